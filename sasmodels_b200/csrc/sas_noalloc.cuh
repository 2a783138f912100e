// Entry point for callers that cannot allocate GPU memory.
//
// Some hosts of this engine are not allowed to call cudaMalloc or any other
// allocator: plugins that run inside another program's CUDA context with a
// fixed memory budget, code that runs while that program holds its allocator
// lock, and real-time loops where an allocation could block or fail at an
// unpredictable moment.  They still own the inputs and the result vector, but
// they cannot provide the scratch space the regular entry points ask for
// (mesh table, segment norms, per-split partial sums).
//
// SASB200_EXPORT_NOALLOC adds one entry point that takes its scratch from a
// fixed array in device memory instead:
//
//   * the array is a file-scope `static __device__` array of
//     SASB200_NOALLOC_SCRATCH_BYTES (8 MiB).  Every GPU that loads this
//     library holds those 8 MiB from when the module is loaded until the
//     process exits;
//   * the host cannot pass the array's name to a kernel (in host code it is
//     only a stand-in, not a device address).  Every call looks up the
//     device address with cudaGetSymbolAddress, with the caller's device
//     current, and passes it to the kernels.  Nothing is cached, so a device
//     reset or a recreated primary context between calls is harmless: the
//     next call finds the array where the new context put it.  The first
//     lookup on a device can load the module, so make the first call on each
//     device before any stream capture;
//   * no cudaMalloc, cudaFree or allocating library routine is called;
//   * a problem whose scratch for one 128-point mesh segment exceeds the
//     array (mainly a very large nq) is rejected with ERR_WORKSPACE and a
//     message; larger meshes are fine, they are processed in chunks;
//   * nothing in the scratch has to start at zero: each pass writes every
//     slot it later reads.  All calls share the one array and it keeps the
//     last call's contents, so calls that overlap on the GPU (two streams, or
//     two host threads with different streams) race and corrupt each other's
//     results.  Issue them on one stream, or serialise them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define SASB200_NOALLOC_SCRATCH_BYTES (8ull << 20)

namespace sasb200 {
namespace noalloc {

static __device__ __align__(256) unsigned char scratch[SASB200_NOALLOC_SCRATCH_BYTES];

// Device address of `scratch` in the current device's context.  Looked up on
// every call (cheap once the module is loaded), never cached: a cached
// address would go stale if the caller reset the device or recreated its
// primary context between calls.
inline int32_t scratch_address(void **out)
{
    void *p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, scratch);
    if (err != cudaSuccess || p == nullptr) {
        std::snprintf(error_buffer(), 256, "cudaGetSymbolAddress(scratch): %s",
                      cudaGetErrorString(err));
        return ERR_CUDA;
    }
    *out = p;
    return OK;
}

template <class M, int VAR>
__host__ int32_t run_static(int32_t nq, int32_t pd_start, int32_t pd_stop,
                            const int32_t *details, const double *values,
                            const double *q, double *result, double cutoff,
                            int32_t reff_mode, int32_t tile_code, void *stream)
{
    if (nq < 0 || pd_start < 0 || pd_stop < pd_start)
        return fail(ERR_ARGUMENT, "need nq >= 0 and 0 <= pd_start <= pd_stop");
    const Tile t = tile_code ? tile_decode(tile_code)
                             : choose_tile(nq, pd_stop - pd_start,
                                           Layout<M, VAR>::XY == XY_1D);
    if (!shape_ok(t) || t.splits < 1)
        return fail(ERR_ARGUMENT, "unknown tile code");
    const size_t need = Workspace<M, VAR>(nq, SEG, t.splits).total;
    if (need > SASB200_NOALLOC_SCRATCH_BYTES) {
        std::snprintf(error_buffer(), 256,
                      "nq=%d with %d mesh splits needs %zu bytes of scratch per mesh "
                      "segment; the static scratch holds %llu bytes",
                      nq, t.splits, need, (unsigned long long)SASB200_NOALLOC_SCRATCH_BYTES);
        return ERR_WORKSPACE;
    }
    void *ws = nullptr;
    const int32_t rc = scratch_address(&ws);
    if (rc != OK) return rc;
    return run<M, VAR>(nq, pd_start, pd_stop, details, values, q, result, cutoff,
                       reff_mode, ws, SASB200_NOALLOC_SCRATCH_BYTES,
                       tile_encode(t), stream);
}

}  // namespace noalloc
}  // namespace sasb200

#define SASB200_EXPORT_NOALLOC(NAME, MODEL, VARIANT_NAME, VAR)                         \
extern "C" int32_t sasb200_##NAME##_##VARIANT_NAME##_noalloc(                          \
    int32_t nq, int32_t pd_start, int32_t pd_stop, const int32_t *details,             \
    const double *values, const double *q, double *result, double cutoff,              \
    int32_t radius_effective_mode, int32_t tile, void *stream)                         \
{                                                                                      \
    return sasb200::noalloc::run_static<MODEL, VAR>(nq, pd_start, pd_stop, details,    \
        values, q, result, cutoff, radius_effective_mode, tile, stream);               \
}
