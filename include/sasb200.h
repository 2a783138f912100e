/*
 * sasb200.h -- C-ABI of the B200 sasmodels engine.
 *
 * One shared library per model, libsasb200_<model>.so, exports the symbols
 * below with <model> spliced into each name (SASB200_DECLARE_MODEL).  The
 * libraries for sphere, cylinder, core_shell_sphere, ellipsoid and
 * core_shell_cylinder are declared explicitly at the end of this file.
 *
 * Kernel entry points (one per kernel_iq.c instantiation)
 * --------------------------------------------------------
 *   sasb200_<model>_Iq         replaces <model>_Iq         (1D, CALL_FQ/CALL_IQ)
 *   sasb200_<model>_Iqxy       replaces <model>_Iqxy       (2D, oriented or |q|)
 *   sasb200_<model>_Imagnetic  replaces <model>_Imagnetic  (2D polarised)
 *
 * Reference interface replaced: the generated DLL kernel
 *     void <model>_<variant>(int32_t nq, int32_t pd_start, int32_t pd_stop,
 *         const ProblemDetails *details, const double *values,
 *         const double *q, double *result, double cutoff,
 *         int32_t radius_effective_mode)
 * declared at sasmodels/kernel_iq.c:317-328, named by
 * sasmodels/generate.py:635-642 and bound with ctypes at
 * sasmodels/kerneldll.py:368-375 (called from DllKernel._call_kernel,
 * sasmodels/kerneldll.py:449-475).
 *
 * The first nine arguments keep their meaning:
 *   nq            number of q points (1D) or (qx, qy) pairs (2D)
 *   pd_start/stop half-open range of the dispersity mesh to accumulate;
 *                 pd_start == 0 starts a new sum, pd_start > 0 adds to the
 *                 sums already in result (restartable mesh)
 *   details       int32[4*max_pd + 4]  CallDetails buffer (details.py:43-180)
 *   values        float64 packed parameter / dispersity vector
 *                 (details.py:225-254)
 *   q             float64[nq] (1D) or interleaved float64[2*nq] (2D)
 *   result        float64[nout*nq + 4], nout = 2 for 1D models with Fq
 *                 (F^2 at even, F at odd slots), else 1; the last four
 *                 slots receive sum(w), sum(w V_form), sum(w V_shell),
 *                 sum(w R_eff)
 *   cutoff        mesh points with weight <= cutoff are skipped
 *   radius_effective_mode   0 = skip R_eff, else the model's mode number
 * All arrays are DEVICE pointers (any allocator).  Added arguments:
 *   workspace, workspace_bytes  device scratch; sasb200_<model>_workspace_bytes
 *                 gives the size for a whole mesh in one pass; a smaller
 *                 workspace is used by processing the mesh in chunks.  A
 *                 mesh range small enough for the single-launch path (its
 *                 table fits 32 KB of one block's shared memory: 1024 points
 *                 for sphere, 512 for cylinder 1D) uses no workspace, and
 *                 workspace may then be NULL
 *   tile          iq_main tile code (splits<<16 | warps<<8 | lanes_per_q),
 *                 0 = built-in choice; see sasb200_<model>_tile_code
 *   stream        cudaStream_t (NULL = legacy default stream)
 * Return: 0 on success; -1 bad argument, -2 workspace too small for one
 * 128-point mesh segment, -3 CUDA launch error, -4 variant not available
 * (e.g. Imagnetic for a model without sld parameters).  The calls are
 * asynchronous on *stream*; sasb200_<model>_last_error() describes the last
 * failure on the calling host thread.
 */
#ifndef SASB200_H
#define SASB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SASB200_KERNEL_ARGS \
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details, \
    const double *values, const double *q, double *result, double cutoff, \
    int32_t radius_effective_mode, void *workspace, uint64_t workspace_bytes, \
    int32_t tile, void *stream

#define SASB200_DECLARE_MODEL(M) \
    int32_t sasb200_##M##_Iq(SASB200_KERNEL_ARGS); \
    int32_t sasb200_##M##_Iqxy(SASB200_KERNEL_ARGS); \
    int32_t sasb200_##M##_Imagnetic(SASB200_KERNEL_ARGS); \
    /* bytes of workspace for variant 0=Iq 1=Iqxy 2=Imagnetic; no reference counterpart */ \
    uint64_t sasb200_##M##_workspace_bytes(int32_t variant, int32_t nq, \
                                           int32_t n_mesh, int32_t tile); \
    /* number of instantiated tile shapes and the code of shape i (autotuner) */ \
    int32_t sasb200_##M##_tile_count(void); \
    int32_t sasb200_##M##_tile_code(int32_t i); \
    /* largest mesh range (pd_stop - pd_start) evaluated by the single-launch \
     * path (one kernel, no workspace) for variant 0=Iq 1=Iqxy 2=Imagnetic; \
     * larger ranges take three launches per workspace chunk; no reference \
     * counterpart */ \
    int32_t sasb200_##M##_single_launch_max(int32_t variant); \
    /* tile code the library picks for (variant, nq, n_mesh) when tile == 0 */ \
    int32_t sasb200_##M##_default_tile(int32_t variant, int32_t nq, int32_t n_mesh); \
    /* message of the last failed call on this host thread ("" if none) */ \
    const char *sasb200_##M##_last_error(void);

SASB200_DECLARE_MODEL(sphere)
SASB200_DECLARE_MODEL(cylinder)

/*
 * The cylinder library's sasb200_cylinder_Iqxy runs a hand-rearranged FP64
 * form of the plugin's Iqac (cylinder.c:92-102, lib/sas_J1.c:107-153) with
 * the per-mesh-point work (contrast x volume, scale factor, weight, R, L/2,
 * rotation row) hoisted out of the q loop, fewer divisions in J1 and those
 * left taken as Newton reciprocals; within 1e-12 of the reference DLL like
 * every FP64 entry point.  The plugin's C as
 * translated, without that rearrangement, stays exported under the prefix
 * cylinder_plugin (same arguments) for comparison.
 */
SASB200_DECLARE_MODEL(cylinder_plugin)

/*
 * Allocation-free variant of sasb200_cylinder_Iqxy.  No counterpart in the
 * reference: it is for callers that may not allocate GPU memory (plugins
 * running inside another program's CUDA context or allocator lock, real-time
 * loops).  Same arguments as sasb200_cylinder_Iqxy without workspace and
 * workspace_bytes; the scratch comes from a static 8 MiB device array in the
 * library (SASB200_NOALLOC_SCRATCH_BYTES), held on every GPU that loads the
 * library until the process exits.  Every call looks up the array's device
 * address in the current context (cudaGetSymbolAddress; nothing is cached,
 * so a device reset between calls is harmless).  The first lookup on a
 * device may load the module: make the first call on each device before any
 * stream capture.  Problems whose scratch for one
 * 128-point mesh segment exceeds the array (very large nq) return -2 with a
 * message; larger meshes are processed in chunks.  All calls share the
 * array: calls that overlap on the GPU race, so keep them on one stream.
 */
#define SASB200_NOALLOC_SCRATCH_BYTES (8ull << 20)
int32_t sasb200_cylinder_Iqxy_noalloc(
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details,
    const double *values, const double *q, double *result, double cutoff,
    int32_t radius_effective_mode, int32_t tile, void *stream);

SASB200_DECLARE_MODEL(core_shell_sphere)

/*
 * The core_shell_sphere library's sasb200_core_shell_sphere_Imagnetic
 * evaluates the spin channels of a (q, mesh point) together: the two
 * 3j1(x)/x terms and volumes of core_shell.c:8-30 once, then each channel's
 * contrasts (kernel_iq.c:750-779 calls the model once per channel); within
 * 1e-12 of the reference DLL.  The plugin's C as translated stays exported
 * under the prefix core_shell_sphere_plugin (same arguments).
 */
SASB200_DECLARE_MODEL(core_shell_sphere_plugin)

SASB200_DECLARE_MODEL(ellipsoid)
SASB200_DECLARE_MODEL(core_shell_cylinder)

/*
 * FP32-compensated form of the same five models, exported from the same
 * libraries under the prefix <model>_f32c: identical arguments and result
 * layout; the amplitude arithmetic runs in FP32 (and the MUFU unit) with
 * FP64 phases, FP64 quadrature and dispersity sums and FP64 volumes.
 * Counterpart of the reference's single-precision build of the same kernels
 * (generate.py:449-488 convert_type, FP32 branches of sas_J1.c:155-231 and
 * sas_3j1x_x.c:40-44); max relative error vs the FP64 DLL <= 1e-5.
 */
SASB200_DECLARE_MODEL(sphere_f32c)
SASB200_DECLARE_MODEL(cylinder_f32c)
SASB200_DECLARE_MODEL(core_shell_sphere_f32c)
SASB200_DECLARE_MODEL(ellipsoid_f32c)
SASB200_DECLARE_MODEL(core_shell_cylinder_f32c)

/*
 * Batched evaluation of a whole fit population of one model in one
 * persistent launch (five models: sphere, cylinder, core_shell_sphere,
 * ellipsoid, core_shell_cylinder).
 *
 * Reference interface replaced: a population is evaluated by the reference
 * one parameter set at a time -- bumps Experiment.theory
 * (sasmodels/bumps_model.py:250-261) -> DataMixin._calc_theory
 * (sasmodels/direct_model.py:319-351) -> Kernel.Fq (sasmodels/kernel.py:
 * 101-188) -> one DLL call per set (sasmodels/kerneldll.py:449-475); this
 * one call replaces that loop, with the per-set arrays of each of those
 * calls concatenated.
 *
 *   form          0 FP64 (the plugin's own Fq per q), 1 FP32-compensated,
 *                 2 / 3 the line form (2D kernel along qx at each set's view
 *                 angles, no orientation dispersion) in FP64 / FP32c
 *   warps, blocks persistent grid shape (blocks 0 = occupancy-derived)
 *   sets          int32[8*n_sets]: nq, q_off, det_off, val_off, num_eval,
 *                 raw_off, iq_off, tile_off of each set
 *   q_all, det_all, val_all   concatenated q vectors, CallDetails buffers and
 *                 values vectors of the sets (each as for a single call)
 *   items         int32[4*n_items]: set, first q, mesh start, mesh stop
 *   tile_items_off, tile_items   CSR list of the items of every 32-q tile
 *                 of every set, in mesh order
 *   partials      float64[64*n_items] scratch; norms float64[4*n_sets]
 *   raw_all       float64[sum(2 nq + 4)]: per set the raw result layout
 *   iq_all        float64[sum nq]: per set I(q), normalised as Kernel.Iq
 *   counter       int32 work counter (reset by the call)
 * Same return codes as the kernel entry points.
 */
#define SASB200_DECLARE_BATCH(M) \
    int32_t sasb200_##M##_batch(int32_t form, int32_t warps, int32_t blocks, \
        int32_t n_sets, const int32_t *sets, const double *q_all, const int32_t *det_all, \
        const double *val_all, int32_t n_items, const int32_t *items, \
        const int32_t *tile_items_off, const int32_t *tile_items, double cutoff, \
        int32_t radius_effective_mode, double *partials, double *norms, double *raw_all, \
        double *iq_all, int32_t *counter, void *stream);

SASB200_DECLARE_BATCH(sphere)
SASB200_DECLARE_BATCH(cylinder)
SASB200_DECLARE_BATCH(core_shell_sphere)
SASB200_DECLARE_BATCH(ellipsoid)
SASB200_DECLARE_BATCH(core_shell_cylinder)

#ifdef __cplusplus
}
#endif

#endif /* SASB200_H */
