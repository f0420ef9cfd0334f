// Library plumbing (version, status text, per-thread error message), reference-frame
// averaging, projection dose and the FullLogNorm kernels.
//
// Reference: frameworks/tomography/Preprocessing/StdPreprocModules/src/NormPlugins.cpp
// (FullLogNorm), core/algorithms/ImagingAlgorithms/src/averageimage.cpp (AverageImage),
// frameworks/tomography/Framework/ReconFramework/src/ProjectionReader.cpp:752-783 (dose).
#include "mr_common.cuh"
#include "mr_kipl_filters.cuh"

#include <algorithm>
#include <mutex>
#include <vector>

#include <cmath>
#include <atomic>
#include <cstring>

namespace mr {

void keep_pool_memory()
{
    static std::mutex mu;
    static bool done[256] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    done[dev] = true;
}

// Allocation-failure hook: the allocation that finds the countdown at 0 fails (the countdown
// then stays disarmed at -1); each allocation that finds it above 0 counts it down.
static std::atomic<long long> g_alloc_countdown{-1};

static bool alloc_hook_takes()
{
    long long v = g_alloc_countdown.load();
    while (v >= 0)
        if (g_alloc_countdown.compare_exchange_weak(v, v - 1)) return v == 0;
    return false;
}

mr_status device_alloc(void **p, size_t bytes, cudaStream_t s, const char *what)
{
    *p = nullptr;
    if (alloc_hook_takes()) return fail(MR_ERR_ALLOCATION, "%s: %zu bytes (allocation-failure hook)", what, bytes);
    keep_pool_memory();
    const cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? MR_ERR_ALLOCATION : MR_ERR_CUDA, "%s: %zu bytes: %s", what, bytes,
                    cudaGetErrorString(e));
    }
    return MR_OK;
}

mr_status device_alloc_sync(void **p, size_t bytes, const char *what)
{
    *p = nullptr;
    if (alloc_hook_takes()) return fail(MR_ERR_ALLOCATION, "%s: %zu bytes (allocation-failure hook)", what, bytes);
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? MR_ERR_ALLOCATION : MR_ERR_CUDA, "%s: %zu bytes: %s", what, bytes,
                    cudaGetErrorString(e));
    }
    return MR_OK;
}


static thread_local std::string g_last_error;

void set_error(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

// ------------------------------------------------------------------ reference averaging

// One thread per pixel; frames summed in frame order so the float rounding sequence is the
// reference's (ComputeSum :63-77, ComputeAverage :79-89, ComputeMin/Max :174-219).
__global__ void k_average(const float *__restrict__ frames, size_t npix, int n, int method, float *__restrict__ out)
{
    size_t j = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (j >= npix) return;
    if (method == 0 || method == 1) {
        float s = 0.0f;
        for (int i = 0; i < n; ++i) s = __fadd_rn(s, frames[i * npix + j]);
        if (method == 1) s = __fmul_rn(s, __fdiv_rn(1.0f, static_cast<float>(n)));
        out[j] = s;
    } else if (method == 4 || method == 5) {
        float v = frames[j];
        for (int i = 1; i < n; ++i) {
            float s = frames[i * npix + j];
            v = method == 4 ? (s < v ? s : v) : (s > v ? s : v);
        }
        out[j] = v;
    } else {
        // ImageMedian (:91-106, median_STL): middle of the sorted column; even counts
        // average the two middle values in float.
        float col[64];
        for (int i = 0; i < n; ++i) col[i] = frames[i * npix + j];
        for (int i = 1; i < n; ++i) {
            float key = col[i];
            int q = i - 1;
            while (q >= 0 && col[q] > key) {
                col[q + 1] = col[q];
                --q;
            }
            col[q + 1] = key;
        }
        out[j] = (n & 1) ? col[n / 2] : __fdiv_rn(__fadd_rn(col[n / 2 - 1], col[n / 2]), 2.0f);
    }
}

// ComputeWeightedAverage (averageimage.cpp:123-172) after the per-frame 5x5 StdDevFilter:
// weight 1/sigma, or 1/(number of pixels) where sigma is 0; weight sum and weighted sum in
// frame order, then their quotient.
__global__ void k_weighted_average(const float *__restrict__ frames, const float *__restrict__ sigma, size_t npix,
                                   int n, float *__restrict__ out)
{
    const size_t j = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (j >= npix) return;
    const float zw = __fdiv_rn(1.0f, static_cast<float>(npix));
    float ws = 0.0f, acc = 0.0f;
    for (int i = 0; i < n; ++i) {
        const float sg = sigma[i * npix + j];
        const float wt = sg != 0.0f ? __fdiv_rn(1.0f, sg) : zw;
        ws = __fadd_rn(ws, wt);
        acc = __fadd_rn(acc, __fmul_rn(wt, frames[i * npix + j]));
    }
    out[j] = __fdiv_rn(acc, ws);
}

// ------------------------------------------------------------------ projection dose

// Row means of the dose ROI: one thread per (frame, row), columns summed in order
// (ProjectionReader.cpp:768-774).
template <typename T>
__global__ void k_row_means(const T *__restrict__ in, size_t nu, size_t nv, size_t nframes, size_t x0, size_t y0,
                            size_t w, size_t h, float *__restrict__ means)
{
    size_t y = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    size_t f = blockIdx.y;
    if (y >= h || f >= nframes) return;
    const T *p = in + f * nu * nv + (y0 + y) * nu + x0;
    float s = 0.0f;
    for (size_t x = 0; x < w; ++x) s = __fadd_rn(s, static_cast<float>(p[x]));
    means[f * h + y] = __fdiv_rn(s, static_cast<float>(w));
}

// Median of h row means per frame: bitonic sort in shared memory, then the middle
// element, or 0.5*(a+b) in double for even h (kipl median.hpp:10-22).
__global__ void k_median(const float *__restrict__ means, size_t h, unsigned npow2, float *__restrict__ dose)
{
    extern __shared__ float s[];
    const float *m = means + blockIdx.x * h;
    for (unsigned i = threadIdx.x; i < npow2; i += blockDim.x) s[i] = i < h ? m[i] : INFINITY;
    __syncthreads();
    for (unsigned k = 2; k <= npow2; k <<= 1) {
        for (unsigned j = k >> 1; j > 0; j >>= 1) {
            for (unsigned i = threadIdx.x; i < npow2; i += blockDim.x) {
                unsigned l = i ^ j;
                if (l > i) {
                    bool up = (i & k) == 0;
                    float a = s[i], b = s[l];
                    if ((a > b) == up) {
                        s[i] = b;
                        s[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        float d = (h & 1) ? s[h / 2] : static_cast<float>(0.5 * (static_cast<double>(s[h / 2 - 1]) + s[h / 2]));
        dose[blockIdx.x] = d;
    }
}

__global__ void k_fill(float *p, size_t n, float v)
{
    size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) p[i] = v;
}

// ------------------------------------------------------------------ FullLogNorm

__global__ void k_logflat(const float *__restrict__ dark, const float *__restrict__ flat, size_t npix, int ndc,
                          float dose, float *__restrict__ logflat)
{
    size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= npix) return;
    float p = ndc ? __fsub_rn(flat[i], dark[i]) : flat[i];
    logflat[i] = p <= 0.0f ? 0.0f : logf(__fmul_rn(p, dose));
}

template <typename T>
__device__ __forceinline__ float lognorm_px(T raw, float dark, float logflat, float dose, int ndc, int nob)
{
    float v = ndc ? __fsub_rn(static_cast<float>(raw), dark) : static_cast<float>(raw);
    if (v <= 0.0f) return 0.0f;
    float lg = logf(v);
    return nob ? __fadd_rn(__fsub_rn(logflat, lg), dose) : __fadd_rn(-lg, dose);
}

// Grid-stride over groups of 4 pixels of one projection row block; blockIdx.y = projection.
// Vector loads when npix % 4 == 0 (the common case), scalar tail otherwise.
template <typename T>
__global__ void k_lognorm(const T *__restrict__ in, size_t npix, const float *__restrict__ dark,
                          const float *__restrict__ logflat, const float *__restrict__ doselog, size_t ndose, int ndc,
                          int nob, int vec, float *__restrict__ out)
{
    const size_t j = blockIdx.y;
    const float dose = ndose != 1 ? doselog[j] : doselog[0];
    const T *src = in + j * npix;
    float *dst = out + j * npix;
    const size_t n4 = vec ? npix / 4 : 0;
    for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n4;
         q += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 d = ndc ? reinterpret_cast<const float4 *>(dark)[q] : make_float4(0, 0, 0, 0);
        const float4 f = nob ? reinterpret_cast<const float4 *>(logflat)[q] : make_float4(0, 0, 0, 0);
        float4 r;
        if constexpr (sizeof(T) == 2) {
            const ushort4 v = reinterpret_cast<const ushort4 *>(src)[q];
            r.x = lognorm_px(v.x, d.x, f.x, dose, ndc, nob);
            r.y = lognorm_px(v.y, d.y, f.y, dose, ndc, nob);
            r.z = lognorm_px(v.z, d.z, f.z, dose, ndc, nob);
            r.w = lognorm_px(v.w, d.w, f.w, dose, ndc, nob);
        } else {
            const float4 v = reinterpret_cast<const float4 *>(src)[q];
            r.x = lognorm_px(v.x, d.x, f.x, dose, ndc, nob);
            r.y = lognorm_px(v.y, d.y, f.y, dose, ndc, nob);
            r.z = lognorm_px(v.z, d.z, f.z, dose, ndc, nob);
            r.w = lognorm_px(v.w, d.w, f.w, dose, ndc, nob);
        }
        reinterpret_cast<float4 *>(dst)[q] = r;
    }
    for (size_t i = n4 * 4 + blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        dst[i] = lognorm_px(src[i], ndc ? dark[i] : 0.0f, nob ? logflat[i] : 0.0f, dose, ndc, nob);
    }
}

// FullLogNorm with uselut (NormPlugins.cpp:455-480): LogLUT of I - D, then logflat - l + dose,
// or -l + (dose - doselog[0]) without flats. table: len entries, then lo, hi, slope, intercept;
// an index outside the table (NaN, or a value the float arithmetic maps past it) is clamped.
template <typename T>
__global__ void k_lognorm_lut(const T *__restrict__ in, size_t npix, const float *__restrict__ dark,
                              const float *__restrict__ logflat, const float *__restrict__ doselog, size_t ndose,
                              int ndc, int nob, const float *__restrict__ table, int len, float *__restrict__ out)
{
    const size_t j = blockIdx.y;
    float dose = ndose != 1 ? doselog[j] : doselog[0];
    if (!nob) dose = __fsub_rn(dose, doselog[0]);
    const float lo = table[len], hi = table[len + 1], slope = table[len + 2], icpt = table[len + 3];
    const T *src = in + j * npix;
    float *dst = out + j * npix;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float v = ndc ? __fsub_rn(static_cast<float>(src[i]), dark[i]) : static_cast<float>(src[i]);
        int idx;
        if (v < lo) {
            idx = 0;
        } else if (hi < v) {
            idx = len - 1;
        } else {
            const float f = __fadd_rn(__fmul_rn(v, slope), icpt);
            idx = f >= static_cast<float>(len) ? len - 1 : (f >= 0.0f ? min(static_cast<int>(f), len - 1) : 0);
        }
        const float l = __ldg(table + idx);
        dst[i] = nob ? __fadd_rn(__fsub_rn(logflat[i], l), dose) : __fadd_rn(-l, dose);
    }
}

// LogLUT(1 << 16, 0, 65535) as FullLogNorm constructs it (NormPlugins.cpp:245;
// core/kipl/kipl/src/math/LUTCollection.cpp:11-36): with lo = 0 the first entry is log(1/slope),
// entry i >= 1 is log(x) with x stepping by 1/slope in float from 1/slope, in the double log
// the reference calls (host code, glibc, no contraction). Built once per process.
static const std::vector<float> &log_lut_table()
{
    static std::vector<float> table;
    static std::once_flag once;
    std::call_once(once, [] {
        const size_t len = size_t(1) << 16;
        const float lo = 0.0f, hi = static_cast<float>((1 << 16) - 1);
        const float slope = static_cast<float>(len - 1) / (hi - lo), icpt = -slope * lo + 0.5f;
        const float delta = 1.0f / slope;
        table.resize(len + 4);
        table[0] = static_cast<float>(std::log(static_cast<double>(delta)));
        float x = delta;
        for (size_t i = 1; i < len; ++i, x += delta) table[i] = static_cast<float>(std::log(static_cast<double>(x)));
        table[len] = lo;
        table[len + 1] = hi;
        table[len + 2] = slope;
        table[len + 3] = icpt;
    });
    return table;
}

// ComputeWeights (frameworks/tomography/Framework/ReconFramework/src/ReconHelpers.cpp:365-488)
// on the projection list BuildFileList makes (:100-110, :150-160): each projection keyed by its
// angle modulo 180 in a multimap (equal keys in acquisition order), weight 1 to start.
// Interior weights (next key - previous key) / 360, 0 for a repeated key; over a full arc
// (arc > 175 degrees) the last weight wraps through the first key + 180 (0 when it repeats the
// one before), the first weight wraps through the last key - 180 and is divided by 180 (by 360
// after a repeated last key or for a golden-section scan); over a short arc both ends copy
// the second weight. Runs of repeated keys share the weight of the entry before them. The
// result is a map keyed by the projection angle (a repeated angle keeps the last entry); when
// the weights of all entries sum to 0.5 within 0.001, every weight is doubled. Fewer than 3
// projections: weight 1/n each, keyed by the reduced angle (the first entry of a repeated key
// kept). Outputs in map order; returns the number of entries.
static size_t compute_weights(const float *angles, size_t n, float arc0, float arc1, bool golden, float *out_angles,
                              float *out_weights)
{
    struct Entry {
        float key, angle, weight;
    };
    std::vector<Entry> e(n);
    for (size_t i = 0; i < n; ++i) e[i] = {std::fmod(angles[i], 180.0f), angles[i], 1.0f};
    std::stable_sort(e.begin(), e.end(), [](const Entry &a, const Entry &b) { return a.key < b.key; });
    if (n < 3) {
        // std::map keyed by the reduced angle: a repeated key keeps its first entry
        size_t m = 0;
        for (size_t i = 0; i < n; ++i) {
            if (i > 0 && e[i].key == e[i - 1].key) continue;
            out_angles[m] = e[i].angle;
            out_weights[m] = static_cast<float>(1.0 / static_cast<double>(n));
            ++m;
        }
        return m;
    }
    for (size_t i = 1; i + 1 < n; ++i)
        e[i].weight = e[i].key != e[i - 1].key ? (e[i + 1].key - e[i - 1].key) / 360.0f : 0.0f;
    if (175.0f < arc1 - arc0) {
        bool repeated_last = false;
        if (e[n - 1].key != e[n - 2].key) {
            e[n - 1].weight = ((e[0].key + 180) - e[n - 2].key) / 360.0f;
        } else {
            e[n - 1].weight = 0.0f;
            repeated_last = true;
        }
        const float span = e[1].key - (e[n - 1].key - 180);
        e[0].weight = (repeated_last || golden) ? span / 360.0f : span / 180.0f;
    } else {
        e[0].weight = e[1].weight;
        e[n - 1].weight = e[1].weight;
    }
    for (size_t q = 1; q < n;) {
        if (e[q].weight == 0.0f) {
            const size_t before = q - 1;
            size_t run = 0;
            do {
                ++run;
                ++q;
            } while (q < n && e[q].weight == 0.0f);
            const float w = e[before].weight / static_cast<float>(run + 1);
            for (size_t k = before; k < before + run + 1; ++k) e[k].weight = w;
        } else {
            ++q;
        }
    }
    float sum = 0.0f;
    std::vector<Entry> byangle;
    byangle.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        sum += e[i].weight;
        byangle.push_back(e[i]);
    }
    // std::map<float, .>: sorted by angle, a repeated angle keeps the last entry in list order
    std::stable_sort(byangle.begin(), byangle.end(), [](const Entry &a, const Entry &b) { return a.angle < b.angle; });
    const bool twice = std::fabs(sum - 0.5f) < 0.001f;
    size_t m = 0;
    for (size_t i = 0; i < n; ++i) {
        if (i + 1 < n && byangle[i + 1].angle == byangle[i].angle) continue;
        out_angles[m] = byangle[i].angle;
        out_weights[m] = twice ? byangle[i].weight * 2 : byangle[i].weight;
        ++m;
    }
    return m;
}

// kipl::algorithms::dataValidator (core/kipl/kipl/include/algorithms/datavalidator.h:8-19) as
// ReconEngine::validateImage uses it: NaNs (exponent all ones, mantissa not zero) and infinities
// of either sign, counted by their bits. Grid-stride over float4 runs when the data are 16-byte
// aligned; per-warp sums, one atomic per warp.
__global__ void __launch_bounds__(256) k_nonfinite(const float *__restrict__ d, size_t n,
                                                   unsigned long long *__restrict__ counts)
{
    unsigned cnan = 0, cinf = 0;
    auto count = [&](float v) {
        const uint32_t b = __float_as_uint(v) & 0x7fffffffu;
        cnan += b > 0x7f800000u;
        cinf += b == 0x7f800000u;
    };
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    size_t head = 0;
    if ((reinterpret_cast<uintptr_t>(d) & 15) == 0) {
        const size_t n4 = n / 4;
        const float4 *d4 = reinterpret_cast<const float4 *>(d);
        for (size_t i = tid; i < n4; i += stride) {
            const float4 v = __ldg(d4 + i);
            count(v.x);
            count(v.y);
            count(v.z);
            count(v.w);
        }
        head = n4 * 4;
    }
    for (size_t i = head + tid; i < n; i += stride) count(__ldg(d + i));
    for (int o = 16; o > 0; o >>= 1) {
        cnan += __shfl_down_sync(0xffffffffu, cnan, o);
        cinf += __shfl_down_sync(0xffffffffu, cinf, o);
    }
    if ((threadIdx.x & 31) == 0 && (cnan | cinf)) {
        atomicAdd(counts, static_cast<unsigned long long>(cnan));
        atomicAdd(counts + 1, static_cast<unsigned long long>(cinf));
    }
}

} // namespace mr

using namespace mr;

extern "C" {

int mr_version(void) { return 100; }

const char *mr_status_string(mr_status s)
{
    switch (s) {
    case MR_OK: return "ok";
    case MR_ERR_ARGUMENT: return "invalid argument";
    case MR_ERR_CUDA: return "CUDA error";
    case MR_ERR_ALLOCATION: return "allocation failed";
    case MR_ERR_UNSUPPORTED: return "unsupported";
    case MR_ERR_DEVICE: return "device-side error status";
    default: return "unknown status";
    }
}

const char *mr_last_error(void) { return g_last_error.c_str(); }

mr_status mr_data_validator(const float *data_d, size_t n, unsigned long long *counts_d, void *stream)
{
    MR_TRACE();
    if (!counts_d || (n && !data_d)) return fail(MR_ERR_ARGUMENT, "mr_data_validator: null pointer");
    cudaStream_t s = as_stream(stream);
    MR_CUDA_TRY(cudaMemsetAsync(counts_d, 0, 2 * sizeof(unsigned long long), s));
    if (n == 0) return MR_OK;
    int dev = 0, sms = 148;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>(static_cast<size_t>(sms) * 8, div_up(n, 1024)));
    k_nonfinite<<<blocks, 256, 0, s>>>(data_d, n, counts_d);
    return check_launch("k_nonfinite");
}

mr_status mr_debug_fail_allocation(long long after)
{
    g_alloc_countdown.store(after < 0 ? -1 : after);
    return MR_OK;
}

mr_status mr_trace_push(const char *name)
{
    if (!name) return fail(MR_ERR_ARGUMENT, "mr_trace_push: null name");
    nvtxRangePushA(name);
    return MR_OK;
}

mr_status mr_trace_pop(void)
{
    nvtxRangePop();
    return MR_OK;
}

mr_status mr_reference_average(const float *frames_d, size_t nu, size_t nv, size_t n, int method, float *out_d,
                               void *stream)
{
    MR_TRACE();
    if (!frames_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_reference_average: null pointer");
    if (n == 0) return fail(MR_ERR_ARGUMENT, "mr_reference_average: no frames");
    if (method < 0 || method > 5)
        return fail(MR_ERR_UNSUPPORTED, "mr_reference_average: method %d not supported", method);
    if (method == 2 && n > 64) return fail(MR_ERR_ARGUMENT, "mr_reference_average: median of more than 64 frames");
    const size_t npix = nu * nv;
    if (method == 3) {
        // ImageWeightedAverage: 5x5 StdDevFilter of every frame, then the weighted average
        if (nu < 5 || nv < 5 || npix > (size_t(1) << 31) - 1 || n > 65535)
            return fail(MR_ERR_ARGUMENT, "mr_reference_average: weighted average of %zu frames of %zux%zu "
                                         "(at least 5x5, at most 65535 frames)", n, nu, nv);
        cudaStream_t s = as_stream(stream);
        float *work = nullptr;
        MR_TRY(device_alloc(&work, 4 * n * npix * sizeof(float), s, "mr_reference_average: scratch"));
        float *sigma = work, *sq = work + n * npix, *tmp = sq + n * npix, *s2 = tmp + n * npix;
        kf::stddev_filter<5>(frames_d, static_cast<int>(nu), static_cast<int>(nv), static_cast<unsigned>(n), sq, tmp,
                             s2, sigma, s);
        k_weighted_average<<<div_up(npix, 256), 256, 0, s>>>(frames_d, sigma, npix, static_cast<int>(n), out_d);
        mr_status st = check_launch("k_weighted_average");
        cudaFreeAsync(work, s);
        return st;
    }
    if (npix == 0) return MR_OK;
    k_average<<<div_up(npix, 256), 256, 0, as_stream(stream)>>>(frames_d, npix, static_cast<int>(n), method, out_d);
    return check_launch("k_average");
}

mr_status mr_projection_dose(const void *in_d, int dtype, size_t nu, size_t nv, size_t nframes, const size_t *roi_h,
                             float *dose_d, void *stream)
{
    MR_TRACE();
    if (!in_d || !dose_d || !roi_h) return fail(MR_ERR_ARGUMENT, "mr_projection_dose: null pointer");
    if (dtype != MR_F32 && dtype != MR_U16) return fail(MR_ERR_ARGUMENT, "mr_projection_dose: dtype must be f32 or u16");
    if (nframes == 0) return MR_OK;
    cudaStream_t s = as_stream(stream);
    if ((roi_h[0] * roi_h[1] * roi_h[2] * roi_h[3]) == 0) {
        k_fill<<<div_up(nframes, 256), 256, 0, s>>>(dose_d, nframes, 1.0f);
        return check_launch("k_fill");
    }
    if (roi_h[2] <= roi_h[0] || roi_h[3] <= roi_h[1] || roi_h[2] > nu || roi_h[3] > nv)
        return fail(MR_ERR_ARGUMENT, "mr_projection_dose: ROI outside the projection");
    const size_t w = roi_h[2] - roi_h[0], h = roi_h[3] - roi_h[1];
    if (h > 8192) return fail(MR_ERR_ARGUMENT, "mr_projection_dose: ROI taller than 8192 rows");
    float *means = nullptr;
    MR_TRY(device_alloc(&means, nframes * h * sizeof(float), s, "mr_projection_dose: scratch"));
    dim3 g(div_up(h, 128), static_cast<unsigned>(nframes));
    if (dtype == MR_F32)
        k_row_means<float><<<g, 128, 0, s>>>(static_cast<const float *>(in_d), nu, nv, nframes, roi_h[0], roi_h[1], w, h,
                                             means);
    else
        k_row_means<uint16_t><<<g, 128, 0, s>>>(static_cast<const uint16_t *>(in_d), nu, nv, nframes, roi_h[0],
                                                roi_h[1], w, h, means);
    mr_status st = check_launch("k_row_means");
    if (st == MR_OK) {
        unsigned p2 = 1;
        while (p2 < h) p2 <<= 1;
        k_median<<<static_cast<unsigned>(nframes), 256, p2 * sizeof(float), s>>>(means, h, p2, dose_d);
        st = check_launch("k_median");
    }
    cudaFreeAsync(means, s);
    return st;
}

mr_status mr_lognorm_logflat(const float *dark_d, const float *flat_d, size_t npix, int ndc, float flatdose,
                             float *logflat_d, void *stream)
{
    MR_TRACE();
    if (!flat_d || !logflat_d || (ndc && !dark_d)) return fail(MR_ERR_ARGUMENT, "mr_lognorm_logflat: null pointer");
    const float dose = 1.0f / flatdose; // host division, as the reference (NormPlugins.cpp:306)
    if (dose != dose) return fail(MR_ERR_ARGUMENT, "The reference dose is a NaN");
    if (std::isinf(dose)) return fail(MR_ERR_ARGUMENT, "The reference dose is Inf");
    if (npix == 0) return MR_OK;
    k_logflat<<<div_up(npix, 256), 256, 0, as_stream(stream)>>>(dark_d, flat_d, npix, ndc, dose, logflat_d);
    return check_launch("k_logflat");
}

mr_status mr_lognorm_doselog(const float *dose_h, size_t n, float darkdose, float *doselog_h)
{
    MR_TRACE();
    if ((!dose_h || !doselog_h) && n) return fail(MR_ERR_ARGUMENT, "mr_lognorm_doselog: null pointer");
    for (size_t i = 0; i < n; ++i) {
        float d = dose_h[i] - darkdose;
        doselog_h[i] = std::log(d < 1 ? 1.0f : d); // float overload, as the reference
    }
    return MR_OK;
}

mr_status mr_lognorm_apply(const void *in_d, int in_dtype, size_t npix, size_t nproj, const float *dark_d,
                           const float *logflat_d, const float *doselog_d, size_t ndose, int ndc, int nob,
                           float *out_d, void *stream)
{
    MR_TRACE();
    if (!in_d || !out_d || !doselog_d || (ndc && !dark_d) || (nob && !logflat_d))
        return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply: null pointer");
    if (in_dtype != MR_U16 && in_dtype != MR_F32) return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply: input must be u16 or f32");
    if (ndose != 1 && ndose != nproj) return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply: ndose must be 1 or nproj");
    if (nproj > 65535) return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply: more than 65535 projections per call");
    if (npix == 0 || nproj == 0) return MR_OK;
    const unsigned gx = std::min<unsigned>(div_up(npix / 4 + 1, 256), 64u);
    // 16-byte vector path when every row start is 16-byte aligned
    const uintptr_t align = reinterpret_cast<uintptr_t>(in_d) | reinterpret_cast<uintptr_t>(out_d) |
                            reinterpret_cast<uintptr_t>(dark_d) | reinterpret_cast<uintptr_t>(logflat_d);
    const int vec = (npix % 4 == 0) && (align % 16 == 0);
    dim3 g(gx, static_cast<unsigned>(nproj));
    if (in_dtype == MR_U16)
        k_lognorm<uint16_t><<<g, 256, 0, as_stream(stream)>>>(static_cast<const uint16_t *>(in_d), npix, dark_d,
                                                              logflat_d, doselog_d, ndose, ndc, nob, vec, out_d);
    else
        k_lognorm<float><<<g, 256, 0, as_stream(stream)>>>(static_cast<const float *>(in_d), npix, dark_d, logflat_d,
                                                           doselog_d, ndose, ndc, nob, vec, out_d);
    return check_launch("k_lognorm");
}

mr_status mr_compute_weights(const float *angles_h, size_t n, const float *scanarc_h, int golden_section,
                             float *angles_out_h, float *weights_out_h, size_t *nout_h)
{
    MR_TRACE();
    if ((n && (!angles_h || !angles_out_h || !weights_out_h)) || !scanarc_h || !nout_h)
        return fail(MR_ERR_ARGUMENT, "mr_compute_weights: null pointer");
    *nout_h = compute_weights(angles_h, n, scanarc_h[0], scanarc_h[1], golden_section != 0, angles_out_h,
                              weights_out_h);
    return MR_OK;
}

mr_status mr_lognorm_apply_lut(const void *in_d, int in_dtype, size_t npix, size_t nproj, const float *dark_d,
                               const float *logflat_d, const float *doselog_d, size_t ndose, int ndc, int nob,
                               float *out_d, void *stream)
{
    MR_TRACE();
    if (!in_d || !out_d || !doselog_d || (ndc && !dark_d) || (nob && !logflat_d))
        return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply_lut: null pointer");
    if (in_dtype != MR_U16 && in_dtype != MR_F32)
        return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply_lut: input must be u16 or f32");
    if (ndose != 1 && ndose != nproj) return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply_lut: ndose must be 1 or nproj");
    if (nproj > 65535) return fail(MR_ERR_ARGUMENT, "mr_lognorm_apply_lut: more than 65535 projections per call");
    if (npix == 0 || nproj == 0) return MR_OK;
    const std::vector<float> &table = log_lut_table();
    cudaStream_t s = as_stream(stream);
    float *lut = nullptr;
    MR_TRY(device_alloc(&lut, table.size() * sizeof(float), s, "mr_lognorm_apply_lut: scratch"));
    mr_status st = MR_OK;
    cudaError_t e = cudaMemcpyAsync(lut, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "mr_lognorm_apply_lut: table upload: %s", cudaGetErrorString(e));
    if (st == MR_OK) {
        const int len = static_cast<int>(table.size() - 4);
        dim3 g(std::min<unsigned>(div_up(npix, 256), 256u), static_cast<unsigned>(nproj));
        if (in_dtype == MR_U16)
            k_lognorm_lut<uint16_t><<<g, 256, 0, s>>>(static_cast<const uint16_t *>(in_d), npix, dark_d, logflat_d,
                                                      doselog_d, ndose, ndc, nob, lut, len, out_d);
        else
            k_lognorm_lut<float><<<g, 256, 0, s>>>(static_cast<const float *>(in_d), npix, dark_d, logflat_d, doselog_d,
                                                   ndose, ndc, nob, lut, len, out_d);
        st = check_launch("k_lognorm_lut");
    }
    cudaFreeAsync(lut, s);
    return st;
}

} // extern "C"
