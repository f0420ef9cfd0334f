// Shared helpers of the mrcuda library: status/error plumbing, launch checks,
// 16-bit projection storage. Host and device.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "mrcuda.h"

#include <nvtx3/nvToolsExt.h>

namespace mr {

// Per-thread last error message (mr_last_error).
void set_error(const char *fmt, ...);

inline mr_status fail(mr_status s, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return s;
}

inline mr_status check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return MR_OK;
}

#define MR_CUDA_TRY(call)                                                                                   \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return ::mr::fail(MR_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

#define MR_TRY(expr)                                                                                       \
    do {                                                                                                   \
        const mr_status st_ = (expr);                                                                      \
        if (st_ != MR_OK) return st_;                                                                      \
    } while (0)

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

// Bounds-checked build (-DMR_BOUNDS_CHECK, libmrcuda_checked.so): the index checks at the gather
// and scatter sites record the first failing site and index in their translation unit's word
// and skip the access, instead of reading or writing out of bounds (no trap); the product build
// compiles them to `true`. mr_bounds_status reads and clears every unit's word.
#ifdef MR_BOUNDS_CHECK
static __device__ unsigned long long g_bounds_word = 0; // site << 40 | index, first failure
__device__ __forceinline__ bool bounds_ok(long long idx, long long size, int site)
{
    if (idx >= 0 && idx < size) return true;
    atomicCAS(&g_bounds_word, 0ull,
              (static_cast<unsigned long long>(site) << 40) | (static_cast<unsigned long long>(idx) & ((1ull << 40) - 1)));
    return false;
}
#define MR_IN_BOUNDS(idx, size, site) ::mr::bounds_ok((idx), (size), (site))
#define MR_BOUNDS_TAKE(fn)                                                                                  \
    int fn(unsigned long long *w)                                                                          \
    {                                                                                                      \
        const unsigned long long zero = 0;                                                                 \
        if (cudaMemcpyFromSymbol(w, g_bounds_word, sizeof(*w)) != cudaSuccess) return -1;                   \
        return cudaMemcpyToSymbol(g_bounds_word, &zero, sizeof(zero)) == cudaSuccess ? 0 : -1;              \
    }
#else
#define MR_IN_BOUNDS(idx, size, site) true
#define MR_BOUNDS_TAKE(fn)                                                                                  \
    int fn(unsigned long long *w)                                                                          \
    {                                                                                                      \
        *w = 0;                                                                                            \
        return 0;                                                                                          \
    }
#endif
// site codes of the checks
enum BoundsSite {
    kSiteBpDirect = 1,   // k_bp_parallel: detector column and slice of a sample
    kSiteFdkDirect = 2,  // k_fdk: detector row and column of a sample
    kSiteBpStaged = 3,   // k_bp_par_staged: staged box sample
    kSiteFdkStaged = 4,  // k_fdk_staged: staged box sample (byte offset in the stage buffers)
    kSiteMbpBins = 5,    // k_mbp_forward_smem: bin in shared memory
    kSiteMbpAdjoint = 6, // k_mbp_adjoint: projection sample
    kSiteRingRows = 7,   // k_dwt_rows_t / k_up_rows_t: staged row input
    kSiteSpotNbr = 8     // k_complete: neighbour pixel
};

// NVTX range over an entry point (a no-op unless a profiler is attached): every C-ABI call
// shows up by name on the host timeline around the kernels it launches.
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};
#define MR_TRACE() ::mr::TraceRange mr_trace_range_(__func__)

// Keep memory freed by cudaFreeAsync cached in the current device's default pool (release
// threshold = unlimited) instead of returning it to the driver at every synchronisation, so
// that per-call scratch (up to tens of GB for a block of projections) is mapped once.
// Applied once per device by the entry points that allocate scratch.
void keep_pool_memory();

// Scratch allocation of the entry points: stream-ordered from the device's default pool (kept
// as above), or synchronous. MR_ERR_ALLOCATION when the device has no room, or when the
// allocation-failure hook (mr_debug_fail_allocation) takes this allocation.
mr_status device_alloc(void **p, size_t bytes, cudaStream_t s, const char *what);
mr_status device_alloc_sync(void **p, size_t bytes, const char *what);
template <class T>
inline mr_status device_alloc(T **p, size_t bytes, cudaStream_t s, const char *what)
{
    return device_alloc(reinterpret_cast<void **>(p), bytes, s, what);
}
template <class T>
inline mr_status device_alloc_sync(T **p, size_t bytes, const char *what)
{
    return device_alloc_sync(reinterpret_cast<void **>(p), bytes, what);
}

inline unsigned div_up(size_t a, size_t b) { return static_cast<unsigned>((a + b - 1) / b); }

// ---- 16-bit projection storage: value = stored * scale (scale per projection, a power of two)
template <int DT>
struct Sample;
template <>
struct Sample<MR_F32> {
    using T = float;
    static __device__ __forceinline__ float load(const float *p, size_t i) { return __ldg(p + i); }
};
template <>
struct Sample<MR_BF16> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ float load(const __nv_bfloat16 *p, size_t i)
    {
        return __bfloat162float(__ldg(p + i));
    }
};
template <>
struct Sample<MR_F16> {
    using T = __half;
    static __device__ __forceinline__ float load(const __half *p, size_t i) { return __half2float(__ldg(p + i)); }
};

} // namespace mr
