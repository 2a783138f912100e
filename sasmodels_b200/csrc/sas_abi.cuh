// C-ABI entry points around the driver templates of sas_driver.cuh.
//
// SASB200_EXPORT_MODEL(name, Model) defines, for one generated model binding,
//
//   int32_t  sasb200_<name>_Iq(...), _Iqxy(...), _Imagnetic(...)
//   uint64_t sasb200_<name>_workspace_bytes(variant, nq, n_mesh, tile)
//   int32_t  sasb200_<name>_tile_count(void), sasb200_<name>_tile_code(i)
//   int32_t  sasb200_<name>_single_launch_max(variant)
//   const char *sasb200_<name>_last_error(void)
//
// The three kernels take the arguments of the reference DLL symbols
// <name>_Iq/_Iqxy/_Imagnetic (sasmodels/kernel_iq.c:317-328; ctypes argtypes
// in sasmodels/kerneldll.py:368-375), with every array in device memory,
// followed by a caller-owned device workspace, a tile code and a CUDA stream.
// They return 0 on success and a negative code otherwise; no C++ exception
// crosses the boundary.  See include/sasb200.h.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

namespace sasb200 {

enum Status {
    OK = 0,
    ERR_ARGUMENT = -1,
    ERR_WORKSPACE = -2,
    ERR_CUDA = -3,
    ERR_UNSUPPORTED = -4,
};

struct Tile { int lq, warps, splits; };

// (lq, warps) shapes instantiated for iq_main.
constexpr int N_SHAPES = 6;
__host__ inline Tile shape_at(int i)
{
    static const Tile shapes[N_SHAPES] = {
        {32, 4, 1}, {32, 8, 1}, {8, 4, 1}, {8, 8, 1}, {1, 4, 1}, {1, 8, 1}};
    return shapes[i];
}

// tile code = (splits << 16) | (warps << 8) | lq, or 0 for the built-in choice
__host__ inline int32_t tile_encode(Tile t) { return (t.splits << 16) | (t.warps << 8) | t.lq; }
__host__ inline Tile tile_decode(int32_t code)
{
    return Tile{code & 0xff, (code >> 8) & 0xff, (code >> 16) & 0xffff};
}
__host__ inline bool shape_ok(Tile t)
{
    for (int i = 0; i < N_SHAPES; ++i) {
        const Tile s = shape_at(i);
        if (s.lq == t.lq && s.warps == t.warps) return true;
    }
    return false;
}

__host__ inline int device_sms()
{
    static thread_local int cached_dev = -1, cached_sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cached_sms;
    if (dev != cached_dev) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess
            && sms > 0) cached_sms = sms;
        cached_dev = dev;
    }
    return cached_sms;
}

// Built-in tile choice, fitted to timings of the current kernels on B200
// (cylinder 2D at 4,096 and 65,536 q x 490,000 points, the magnetic
// core_shell_sphere, a 1D ellipsoid with adaptive quadrature):
//   * 1D calls: one q per warp (the 32 lanes take mesh points), 4 warps --
//     every lane of a warp then runs the same quadrature rule (2.3x the
//     8-q tile for the ellipsoid);
//   * 2D calls: 32 neighbouring q per warp from 16,384 q up, 8 below, mesh
//     lanes under 256 q, 4 warps;
//   * then mesh splits for ~512 blocks per SM (at most 128 splits, at most
//     one per 128-point segment): cylinder 2D runs 5 % faster at 32-64
//     splits than at 5.
__host__ inline Tile choose_tile(int nq, int n_mesh, bool one_d)
{
    Tile t;
    if (one_d) t = Tile{1, 4, 1};
    else if (nq >= 16384) t = Tile{32, 4, 1};
    else if (nq >= 256) t = Tile{8, 4, 1};
    else t = Tile{1, 8, 1};
    const long long qtiles = (nq + t.lq - 1)/t.lq;
    const long long nseg = (n_mesh + SEG - 1)/SEG;
    const long long want = (long long)device_sms()*512;
    long long splits = qtiles > 0 ? (want + qtiles - 1)/qtiles : 1;
    if (splits > nseg) splits = nseg;
    if (splits > 128) splits = 128;
    if (splits < 1) splits = 1;
    t.splits = (int)splits;
    return t;
}

// Built-in shape of the single-launch path (no mesh splits): 8 q per warp
// and 4 warps, so a mesh of a few dozen points still spreads over the lanes
// (sphere 1D: 2.85 us per call against 4.1 with one q per warp); one q per
// warp for 1D meshes of 128 points and more, where every lane of a warp
// then runs the same quadrature rule.
__host__ inline Tile choose_small_tile(int n_mesh, bool one_d)
{
    return (one_d && n_mesh >= 128) ? Tile{1, 4, 1} : Tile{8, 4, 1};
}

__host__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class M, int VAR>
struct Workspace {
    using L = Layout<M, VAR>;
    size_t table, counts, norms, points, partial, total;
    Workspace(int nq, long long chunk, int splits)
    {
        const long long nseg = (chunk + SEG - 1)/SEG;
        table = align256((size_t)nseg*SEG*L::NF*sizeof(double));
        counts = align256((size_t)nseg*sizeof(int));
        norms = align256((size_t)nseg*4*sizeof(double));
        points = align256((size_t)nseg*SEG*4*sizeof(double));   // per-point norm terms
        partial = align256((size_t)(splits > 0 ? splits : 1)*L::NOUT*(size_t)nq*sizeof(double));
        total = table + counts + norms + points + partial;
    }
};

template <class M, int VAR, int LQ, int WARPS>
__host__ void launch_main(dim3 grid, cudaStream_t st, int nq, const double *q,
                          const double *values, const double *table,
                          const int *counts, int nseg, double *partial)
{
    // the staged segment is dynamic shared memory: SEG rows of the table
    constexpr size_t stage = (size_t)SEG*Layout<M, VAR>::NF*sizeof(double);
    if (stage > 48*1024) {
        // the opt-in limit is per device; setting it again is harmless
        static int raised[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !raised[dev]) {
            cudaFuncSetAttribute(iq_main<M, VAR, LQ, WARPS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage);
            if (dev >= 0 && dev < 64) raised[dev] = 1;
        }
    }
    iq_main<M, VAR, LQ, WARPS><<<grid, 32*WARPS, stage, st>>>(
        nq, q, values, table, counts, nseg, partial);
}

template <class M, int VAR>
__host__ bool dispatch_main(Tile t, dim3 grid, cudaStream_t st, int nq, const double *q,
                            const double *values, const double *table,
                            const int *counts, int nseg, double *partial)
{
    switch (t.lq*100 + t.warps) {
    case 3204: launch_main<M, VAR, 32, 4>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    case 3208: launch_main<M, VAR, 32, 8>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    case 804:  launch_main<M, VAR, 8, 4>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    case 808:  launch_main<M, VAR, 8, 8>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    case 104:  launch_main<M, VAR, 1, 4>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    case 108:  launch_main<M, VAR, 1, 8>(grid, st, nq, q, values, table, counts, nseg, partial); return true;
    default: return false;
    }
}

template <class M, int VAR>
__host__ bool dispatch_small(Tile t, int nq, cudaStream_t st, int pd_start, int n_mesh,
                             const int32_t *details, const double *values, const double *q,
                             double cutoff, int reff_mode, double *result, int accumulate)
{
    const dim3 grid(nq > 0 ? (nq + t.lq - 1)/t.lq : 1);
#define SASB200_SMALL(LQ_, W_) \
    iq_small<M, VAR, LQ_, W_><<<grid, 32*(W_), 0, st>>>(nq, pd_start, n_mesh, details, \
        values, q, cutoff, reff_mode, result, accumulate); return true;
    switch (t.lq*100 + t.warps) {
    case 3204: SASB200_SMALL(32, 4)
    case 3208: SASB200_SMALL(32, 8)
    case 804:  SASB200_SMALL(8, 4)
    case 808:  SASB200_SMALL(8, 8)
    case 104:  SASB200_SMALL(1, 4)
    case 108:  SASB200_SMALL(1, 8)
    default: return false;
    }
#undef SASB200_SMALL
}

// Error text of the last failing call on this host thread.
inline char *error_buffer()
{
    static thread_local char buf[256] = "";
    return buf;
}

__host__ inline int32_t fail(int32_t code, const char *msg)
{
    std::snprintf(error_buffer(), 256, "%s", msg);
    return code;
}

template <class M, int VAR>
__host__ uint64_t workspace_bytes(int32_t nq, int32_t n_mesh, int32_t tile_code)
{
    if (nq < 0 || n_mesh < 0) return 0;
    Tile t = tile_code ? tile_decode(tile_code)
                       : choose_tile(nq, n_mesh, Layout<M, VAR>::XY == XY_1D);
    // at least one segment, at most 2^20 mesh points per pass
    const long long chunk = n_mesh < 1 ? 1 : (n_mesh < (1 << 20) ? n_mesh : (1 << 20));
    return Workspace<M, VAR>(nq, chunk, t.splits).total;
}

// One kernel call: mesh [pd_start, pd_stop) is processed in chunks that fit
// the workspace; the first chunk overwrites result unless pd_start > 0
// (restartable mesh, kernel_iq.c:381-423), later chunks add to it.
template <class M, int VAR>
__host__ int32_t run(int32_t nq, int32_t pd_start, int32_t pd_stop,
                     const int32_t *details, const double *values, const double *q,
                     double *result, double cutoff, int32_t reff_mode,
                     void *workspace, uint64_t workspace_bytes, int32_t tile_code,
                     void *stream)
{
    using L = Layout<M, VAR>;
    error_buffer()[0] = 0;
    if constexpr (VAR == VAR_IMAGNETIC && M::NMAG == 0) {
        return fail(ERR_UNSUPPORTED, "model has no magnetic parameters");
    } else {
    if (nq < 0 || pd_start < 0 || pd_stop < pd_start)
        return fail(ERR_ARGUMENT, "need nq >= 0 and 0 <= pd_start <= pd_stop");
    if (!details || !values || !result || (nq > 0 && !q))
        return fail(ERR_ARGUMENT, "null array pointer");
    const int n_mesh = pd_stop - pd_start;
    Tile t = tile_code ? tile_decode(tile_code)
                       : choose_tile(nq, n_mesh, Layout<M, VAR>::XY == XY_1D);
    if (!shape_ok(t) || t.splits < 1)
        return fail(ERR_ARGUMENT, "unknown tile code");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_mesh <= small_mesh_max<M, VAR>()) {
        // the whole mesh range fits one block's shared memory: one launch,
        // no workspace (mesh splits of the tile code do not apply)
        if (!tile_code) t = choose_small_tile(n_mesh, Layout<M, VAR>::XY == XY_1D);
        if (!dispatch_small<M, VAR>(t, nq, st, pd_start, n_mesh, details, values, q,
                                    cutoff, reff_mode, result, pd_start > 0 ? 1 : 0))
            return fail(ERR_ARGUMENT, "unknown tile shape");
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) {
            std::snprintf(error_buffer(), 256, "kernel launch: %s", cudaGetErrorString(err));
            return ERR_CUDA;
        }
        return OK;
    }
    // largest chunk of whole segments whose workspace fits
    const long long nseg_all = n_mesh > 0 ? (n_mesh + SEG - 1)/SEG : 1;
    long long lo = 0, hi = nseg_all;
    while (lo < hi) {
        const long long mid = (lo + hi + 1)/2;
        if (Workspace<M, VAR>(nq, mid*SEG, t.splits).total <= workspace_bytes) lo = mid;
        else hi = mid - 1;
    }
    if (lo == 0 || !workspace)
        return fail(ERR_WORKSPACE, "workspace too small for one mesh segment");
    const long long chunk = lo == nseg_all ? (n_mesh > 0 ? n_mesh : 1) : lo*SEG;
    const Workspace<M, VAR> ws(nq, chunk, t.splits);
    char *base = static_cast<char *>(workspace);
    double *table = reinterpret_cast<double *>(base);
    int *counts = reinterpret_cast<int *>(base + ws.table);
    double *norms = reinterpret_cast<double *>(base + ws.table + ws.counts);
    double *points = reinterpret_cast<double *>(base + ws.table + ws.counts + ws.norms);
    double *partial = reinterpret_cast<double *>(base + ws.table + ws.counts + ws.norms
                                                 + ws.points);
    // the norms in the DLL's own order when an effective radius is asked for
    double *seq = reff_mode != 0 ? points : nullptr;
    const int points_stride = (int)(((chunk + SEG - 1)/SEG)*SEG);
    const int nout_nq = L::NOUT*nq;

    long long start = pd_start;
    do {
        const int n = (int)((pd_stop - start) < chunk ? (pd_stop - start) : chunk);
        const int nseg = (n + SEG - 1)/SEG;
        int splits = t.splits < nseg ? t.splits : nseg;
        if (nseg > 0) {
            mesh_prepare<M, VAR><<<nseg, SEG, 0, st>>>(
                (int)start, n, details, values, cutoff, reff_mode, table, counts, norms,
                seq, points_stride);
        }
        if (nq > 0 && nseg > 0) {
            dim3 grid((nq + t.lq - 1)/t.lq, splits);
            if (!dispatch_main<M, VAR>(t, grid, st, nq, q, values, table, counts, nseg, partial))
                return fail(ERR_ARGUMENT, "unknown tile shape");
        }
        if (nseg == 0) splits = 0;
        const int fblocks = (nout_nq + 255)/256 + 1;
        finalize<0><<<fblocks, 256, 0, st>>>(nout_nq, splits, partial, nseg, norms, result,
                                          start > 0 ? 1 : 0, nseg > 0 ? seq : nullptr, n,
                                          points_stride);
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) {
            std::snprintf(error_buffer(), 256, "kernel launch: %s", cudaGetErrorString(err));
            return ERR_CUDA;
        }
        start += n;
    } while (start < pd_stop);
    return OK;
    }
}

}  // namespace sasb200

#define SASB200_STR2(x) #x
#define SASB200_STR(x) SASB200_STR2(x)

#define SASB200_EXPORT_MODEL(NAME, MODEL)                                               \
extern "C" int32_t sasb200_##NAME##_Iq(                                                 \
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details,              \
    const double *values, const double *q, double *result, double cutoff,               \
    int32_t radius_effective_mode, void *workspace, uint64_t workspace_bytes,           \
    int32_t tile, void *stream)                                                         \
{                                                                                       \
    return sasb200::run<MODEL, sasb200::VAR_IQ>(nq, pd_start, pd_stop, details, values, \
        q, result, cutoff, radius_effective_mode, workspace, workspace_bytes, tile,     \
        stream);                                                                        \
}                                                                                       \
extern "C" int32_t sasb200_##NAME##_Iqxy(                                               \
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details,              \
    const double *values, const double *q, double *result, double cutoff,               \
    int32_t radius_effective_mode, void *workspace, uint64_t workspace_bytes,           \
    int32_t tile, void *stream)                                                         \
{                                                                                       \
    return sasb200::run<MODEL, sasb200::VAR_IQXY>(nq, pd_start, pd_stop, details,       \
        values, q, result, cutoff, radius_effective_mode, workspace, workspace_bytes,   \
        tile, stream);                                                                  \
}                                                                                       \
extern "C" int32_t sasb200_##NAME##_Imagnetic(                                          \
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details,              \
    const double *values, const double *q, double *result, double cutoff,               \
    int32_t radius_effective_mode, void *workspace, uint64_t workspace_bytes,           \
    int32_t tile, void *stream)                                                         \
{                                                                                       \
    return sasb200::run<MODEL, sasb200::VAR_IMAGNETIC>(nq, pd_start, pd_stop, details,  \
        values, q, result, cutoff, radius_effective_mode, workspace, workspace_bytes,   \
        tile, stream);                                                                  \
}                                                                                       \
extern "C" uint64_t sasb200_##NAME##_workspace_bytes(                                   \
    int32_t variant, int32_t nq, int32_t n_mesh, int32_t tile)                          \
{                                                                                       \
    switch (variant) {                                                                  \
    case 0: return sasb200::workspace_bytes<MODEL, sasb200::VAR_IQ>(nq, n_mesh, tile);  \
    case 1: return sasb200::workspace_bytes<MODEL, sasb200::VAR_IQXY>(nq, n_mesh, tile);\
    case 2: return sasb200::workspace_bytes<MODEL, sasb200::VAR_IMAGNETIC>(nq, n_mesh,  \
                                                                           tile);       \
    default: return 0;                                                                  \
    }                                                                                   \
}                                                                                       \
extern "C" int32_t sasb200_##NAME##_single_launch_max(int32_t variant)                  \
{                                                                                       \
    switch (variant) {                                                                  \
    case 0: return sasb200::small_mesh_max<MODEL, sasb200::VAR_IQ>();                   \
    case 1: return sasb200::small_mesh_max<MODEL, sasb200::VAR_IQXY>();                 \
    case 2: return sasb200::small_mesh_max<MODEL, sasb200::VAR_IMAGNETIC>();            \
    default: return 0;                                                                  \
    }                                                                                   \
}                                                                                       \
extern "C" int32_t sasb200_##NAME##_tile_count(void) { return sasb200::N_SHAPES; }      \
extern "C" int32_t sasb200_##NAME##_tile_code(int32_t i)                                \
{                                                                                       \
    if (i < 0 || i >= sasb200::N_SHAPES) return 0;                                      \
    return sasb200::tile_encode(sasb200::shape_at(i));                                  \
}                                                                                       \
extern "C" int32_t sasb200_##NAME##_default_tile(int32_t variant, int32_t nq,          \
                                                  int32_t n_mesh)                       \
{                                                                                       \
    return sasb200::tile_encode(sasb200::choose_tile(nq, n_mesh, variant == 0));         \
}                                                                                       \
extern "C" const char *sasb200_##NAME##_last_error(void)                                \
{                                                                                       \
    return sasb200::error_buffer();                                                     \
}
