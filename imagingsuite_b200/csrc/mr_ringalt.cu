// Alternative ring cleaners: BasicRingClean and MedianMixRingClean, and the kipl median filter
// both are built on.
//
// References (relative to the reference project root):
//   BasicRingClean::ProcessCore     frameworks/tomography/Preprocessing/StdPreprocModules/src/
//                                   BasicRingClean.cpp:50-95
//   MedianMixRingClean::ProcessCore, ComputeProfile
//                                   frameworks/tomography/Preprocessing/StdPreprocModules/src/
//                                   MedianMixRingClean.cpp:57-138
//   TMedianFilter<float,2>          core/kipl/kipl/include/filters/core/medianfilter.hpp:28-199
//   kipl::heapsort, math::median    core/kipl/kipl/include/algorithms/sortalg.h:10-45,
//                                   core/kipl/kipl/include/math/core/median.hpp:10-22
//   SigmoidLUT, LUTbase::BasicLUT   core/kipl/kipl/src/math/LUTCollection.cpp:38-82,
//                                   core/kipl/kipl/src/math/LUTbase.cpp:12-75
//
// The reference's median of a window copies the window (row-major, with its edge rules),
// heap-sorts it and takes the middle element. Without NaN the middle order statistic is
// unique up to the sign of a zero, so a min/max selection network (mr_median_net.cuh) gives
// the same bits. Windows holding a NaN (caught by a NaN sum), and windows whose middle value
// is a zero while zeros of both signs are present, go through the reference's own heap sort
// on the window instead. The reference reads a few values past the end of an image near its
// bottom-right corner (its edge formulas reach past the row); those read 0 here, the value the
// oracle uses too.
#include "mr_common.cuh"
#include "mr_median_net.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace mr {
namespace ringalt {

template <int N>
struct Net;
template <>
struct Net<1> {
    static __device__ __forceinline__ float run(float (&v)[1]) { return v[0]; }
};
template <>
struct Net<3> {
    static __device__ __forceinline__ float run(float (&v)[3]) { return median_net3(v); }
};
template <>
struct Net<5> {
    static __device__ __forceinline__ float run(float (&v)[5]) { return median_net5(v); }
};
template <>
struct Net<9> {
    static __device__ __forceinline__ float run(float (&v)[9]) { return median_net9(v); }
};
template <>
struct Net<15> {
    static __device__ __forceinline__ float run(float (&v)[15]) { return median_net15(v); }
};
template <>
struct Net<25> {
    static __device__ __forceinline__ float run(float (&v)[25]) { return median_net25(v); }
};

// Value idx of an image of n values; at or past the end (the reference's reads near the
// bottom-right corner) it is 0.
__device__ __forceinline__ float value_at(const float *img, long long n, long long idx)
{
    return idx >= 0 && idx < n ? __ldg(img + idx) : 0.0f;
}

// The window TMedianFilter::ExtractNeighborhood builds at (x, y) (medianfilter.hpp:52-159):
// edge code from the unsigned comparisons, the per-code ranges (the bottom-right one reaching
// one column further), a zero start, then the left, right, top and bottom replications.
// The host admits only sizes at which codes 3, 7 and 11-15 cannot occur.
template <int KX, int KY>
__device__ void kipl_window(const float *img, int w, int h, int x, int y, float *win)
{
    constexpr int hx = KX / 2, hy = KY / 2;
    const int code = (x < hx) + 2 * (w - hx - 1 < x) + 4 * (y < hy) + 8 * (h - hy - 1 < y);
    int sx = -hx, ex = KX - hx, sy = -hy, ey = KY - hy;
    const int rx = KX - hx - (w - x), ry = KY - hy - (h - y);
    switch (code) {
    case 1: sx = -x; break;
    case 2: ex = rx; break;
    case 4: sy = -y; break;
    case 5: sx = -x; sy = -y; break;
    case 6: ex = rx; sy = -y; break;
    case 8: ey = ry; break;
    case 9: sx = -x; ey = ry; break;
    case 10: ey = ry; ex = rx + 1; break;
    default: break;
    }
    for (int i = 0; i < KX * KY; ++i) win[i] = 0.0f;
    const long long n = static_cast<long long>(w) * h, base = static_cast<long long>(y) * w + x;
    for (int dy = sy; dy < ey; ++dy)
        for (int dx = sx; dx < ex; ++dx) win[(dy + hy) * KX + dx + hx] = value_at(img, n, base + static_cast<long long>(dy) * w + dx);
    if (code & 1)
        for (int r = 0; r < KY; ++r)
            for (int d = sx - 1, s = sx; d >= -hx; --d, ++s) win[r * KX + d + hx] = win[r * KX + s + hx];
    if (code & 2)
        for (int r = 0; r < KY; ++r)
            for (int s = ex - 1, d = ex; d < KX - hx; --s, ++d) win[r * KX + d + hx] = win[r * KX + s + hx];
    if (code & 4)
        for (int d = sy - 1, s = sy; d >= -hy; --d, ++s)
            for (int c = 0; c < KX; ++c) win[(d + hy) * KX + c] = win[(s + hy) * KX + c];
    if (code & 8)
        for (int s = ey - 1, d = ey; d < KY - hy; --s, ++d)
            for (int c = 0; c < KX; ++c) win[(d + hy) * KX + c] = win[(s + hy) * KX + c];
}

// Heap sort in the Numerical Recipes sift-down form kipl::heapsort uses (1-based positions,
// strict '<'), so equal keys of different bits and NaN land where the reference puts them.
__device__ void nr_heapsort(float *a, int n)
{
    if (n < 2) return;
    int l = (n >> 1) + 1, ir = n;
    for (;;) {
        float v;
        if (l > 1) {
            --l;
            v = a[l - 1];
        } else {
            v = a[ir - 1];
            a[ir - 1] = a[0];
            if (--ir == 1) {
                a[0] = v;
                break;
            }
        }
        int i = l, j = l + l;
        while (j <= ir) {
            if (j < ir && a[j - 1] < a[j]) j++;
            if (v < a[j - 1]) {
                a[i - 1] = a[j - 1];
                i = j;
                j <<= 1;
            } else {
                j = ir + 1;
            }
        }
        a[i - 1] = v;
    }
}

// The rare cases: a NaN in the window, or a zero middle value. The window is rebuilt in the
// reference's order; a zero middle value with zeros of one sign only is that zero, anything
// else is the heap sort's middle element.
template <int KX, int KY>
__device__ __noinline__ float careful_median(const float *img, int w, int h, int x, int y, bool has_nan)
{
    constexpr int N = KX * KY;
    float win[N];
    kipl_window<KX, KY>(img, w, h, x, y, win);
    if (!has_nan) {
        bool pos = false, neg = false;
        for (int i = 0; i < N; ++i) {
            const unsigned b = __float_as_uint(win[i]);
            pos |= b == 0u;
            neg |= b == 0x80000000u;
        }
        if (!(pos && neg)) return neg ? -0.0f : 0.0f;
    }
    nr_heapsort(win, N);
    return win[N / 2];
}

template <int KX, int KY>
__device__ __forceinline__ float window_median(const float *img, int w, int h, int x, int y)
{
    constexpr int N = KX * KY, hx = KX / 2, hy = KY / 2;
    float v[N];
    if (x >= hx && x < w - hx && y >= hy && y < h - hy) {
        const float *p = img + static_cast<size_t>(y - hy) * w + (x - hx);
#pragma unroll
        for (int r = 0; r < KY; ++r)
#pragma unroll
            for (int c = 0; c < KX; ++c) v[r * KX + c] = __ldg(p + static_cast<size_t>(r) * w + c);
    } else {
        float e[N];
        kipl_window<KX, KY>(img, w, h, x, y, e);
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = e[i];
    }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) s += v[i]; // NaN iff a NaN (or +inf and -inf) is in the window
    const float m = Net<N>::run(v);
    if (isnan(s) || m == 0.0f) return careful_median<KX, KY>(img, w, h, x, y, isnan(s));
    return m;
}

enum { MODE_MEDIAN = 0, MODE_DIFF = 1, MODE_ABSDIFF = 2, MODE_MIX = 3 };

template <int MODE>
__device__ __forceinline__ float median_epilogue(const float *img, const float *wt, size_t i, float m)
{
    if (MODE == MODE_DIFF) return __fsub_rn(__ldg(img + i), m);
    if (MODE == MODE_ABSDIFF) return fabsf(__fsub_rn(__ldg(img + i), m));
    if (MODE == MODE_MIX) {
        const float a = __ldg(wt + i);
        return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, a), __ldg(img + i)), __fmul_rn(a, m));
    }
    return m;
}

// One pixel per thread, images along z. MODE_MEDIAN writes the median, MODE_DIFF the image
// minus it (BasicRingClean.cpp:84-86), MODE_ABSDIFF its absolute difference
// (MedianMixRingClean.cpp:133-135), MODE_MIX (1 - wt) * p + wt * median
// (MedianMixRingClean.cpp:91-93) with the weight image wt shared by all images.
template <int KX, int KY, int MODE>
__global__ void __launch_bounds__(256) k_median(const float *__restrict__ src, int w, int h,
                                                const float *__restrict__ wt, float *__restrict__ dst)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t npix = static_cast<size_t>(w) * h, i = static_cast<size_t>(y) * w + x;
    const float *img = src + blockIdx.z * npix;
    dst[blockIdx.z * npix + i] = median_epilogue<MODE>(img, wt, i, window_median<KX, KY>(img, w, h, x, y));
}

// 5x5 median of two horizontally adjacent pixels per thread. Their windows share the 20 values
// of columns x-1 .. x+2. A value of rank r among those 20 has rank r .. r+5 in either window,
// so only ranks 7..12 (0-based) can be a window's middle (rank 12 of 25), and that middle is
// the middle of the 6 candidates and the window's own 5 values: 168 min/max for the shared
// ranks plus 54 per window, instead of 202 per window. Pixels whose windows leave the image go
// through window_median one by one.
template <int MODE>
__global__ void __launch_bounds__(256) k_median55_pair(const float *__restrict__ src, int w, int h,
                                                       const float *__restrict__ wt, float *__restrict__ dst)
{
    const int x = 2 * (blockIdx.x * 32 + threadIdx.x), y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t npix = static_cast<size_t>(w) * h, i = static_cast<size_t>(y) * w + x;
    const float *img = src + blockIdx.z * npix;
    float *out = dst + blockIdx.z * npix;
    if (x >= 2 && x + 3 < w && y >= 2 && y + 2 < h) {
        float c[20], a[5], b[5];
        const float *p = img + static_cast<size_t>(y - 2) * w + (x - 2);
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            const float *q = p + static_cast<size_t>(r) * w;
            a[r] = __ldg(q);
#pragma unroll
            for (int k = 0; k < 4; ++k) c[r * 4 + k] = __ldg(q + 1 + k);
            b[r] = __ldg(q + 5);
        }
        float sc = 0.0f, sa = 0.0f, sb = 0.0f;
#pragma unroll
        for (int k = 0; k < 20; ++k) sc += c[k];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            sa += a[r];
            sb += b[r];
        }
        sa += sc; // NaN iff a NaN (or +inf and -inf) is in the window
        sb += sc;
        rank_net20_7_12(c);
        float va[11], vb[11];
#pragma unroll
        for (int k = 0; k < 6; ++k) va[k] = vb[k] = c[7 + k];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            va[6 + r] = a[r];
            vb[6 + r] = b[r];
        }
        float m0 = median_net11(va), m1 = median_net11(vb);
        if (isnan(sa) || m0 == 0.0f) m0 = careful_median<5, 5>(img, w, h, x, y, isnan(sa));
        if (isnan(sb) || m1 == 0.0f) m1 = careful_median<5, 5>(img, w, h, x + 1, y, isnan(sb));
        out[i] = median_epilogue<MODE>(img, wt, i, m0);
        out[i + 1] = median_epilogue<MODE>(img, wt, i + 1, m1);
    } else {
        out[i] = median_epilogue<MODE>(img, wt, i, window_median<5, 5>(img, w, h, x, y));
        if (x + 1 < w) out[i + 1] = median_epilogue<MODE>(img, wt, i + 1, window_median<5, 5>(img, w, h, x + 1, y));
    }
}

// Mean projection accumulated in projection order (BasicRingClean.cpp:56-69 starts from a copy
// of the first projection, MedianMixRingClean.cpp:113-125 from zero), times 1 / nproj.
// VEC: four pixels per thread.
template <bool VEC>
__global__ void __launch_bounds__(256) k_mean_projection(const float *__restrict__ proj, size_t npix, size_t nproj,
                                                         int from_zero, float scale, float *__restrict__ mean)
{
    if constexpr (VEC) {
        const size_t j = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
        if (j >= npix) return;
        float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        size_t i = 0;
        if (!from_zero) {
            acc = __ldg(reinterpret_cast<const float4 *>(proj + j));
            i = 1;
        }
#pragma unroll 8
        for (; i < nproj; ++i) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(proj + i * npix + j));
            acc.x = __fadd_rn(acc.x, v.x);
            acc.y = __fadd_rn(acc.y, v.y);
            acc.z = __fadd_rn(acc.z, v.z);
            acc.w = __fadd_rn(acc.w, v.w);
        }
        acc.x = __fmul_rn(acc.x, scale);
        acc.y = __fmul_rn(acc.y, scale);
        acc.z = __fmul_rn(acc.z, scale);
        acc.w = __fmul_rn(acc.w, scale);
        *reinterpret_cast<float4 *>(mean + j) = acc;
    } else {
        const size_t j = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
        if (j >= npix) return;
        float acc = 0.0f;
        size_t i = 0;
        if (!from_zero) {
            acc = __ldg(proj + j);
            i = 1;
        }
#pragma unroll 8
        for (; i < nproj; ++i) acc = __fadd_rn(acc, __ldg(proj + i * npix + j));
        mean[j] = __fmul_rn(acc, scale);
    }
}

// proj[i][j] -= diff[j] for every projection (BasicRingClean.cpp:88-93); grid-stride.
template <bool VEC>
__global__ void __launch_bounds__(256) k_subtract(float *__restrict__ proj, size_t npix, size_t nproj,
                                                  const float *__restrict__ diff)
{
    const size_t total = npix * nproj, stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    if constexpr (VEC) {
        for (size_t q = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < total / 4; q += stride) {
            const size_t e = q * 4, j = e % npix;
            float4 p = *reinterpret_cast<const float4 *>(proj + e);
            const float4 d = __ldg(reinterpret_cast<const float4 *>(diff + j));
            p.x = __fsub_rn(p.x, d.x);
            p.y = __fsub_rn(p.y, d.y);
            p.z = __fsub_rn(p.z, d.z);
            p.w = __fsub_rn(p.w, d.w);
            *reinterpret_cast<float4 *>(proj + e) = p;
        }
    } else {
        for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += stride)
            proj[e] = __fsub_rn(proj[e], __ldg(diff + e % npix));
    }
}

// LUTbase::BasicLUT (LUTbase.cpp:57-75) in place on the weight image. table: len entries, then
// lo, hi, slope, intercept. An index outside the table (a NaN weight, or cancellation in
// slope * v + intercept when lambda is far larger than the width, where the reference reads
// past its table) is clamped to it.
__global__ void __launch_bounds__(256) k_lut(float *__restrict__ v, size_t n, const float *__restrict__ table, int len)
{
    const size_t j = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const float lo = table[len], hi = table[len + 1], slope = table[len + 2], icpt = table[len + 3];
    const float x = v[j];
    float r;
    if (x < lo) {
        r = table[0];
    } else if (hi < x) {
        r = table[len - 1];
    } else {
        const float f = __fadd_rn(__fmul_rn(x, slope), icpt);
        int idx = 0;
        if (f >= static_cast<float>(len)) idx = len - 1;
        else if (f >= 0.0f) idx = min(static_cast<int>(f), len - 1);
        r = table[idx];
    }
    v[j] = r;
}

} // namespace ringalt

// SigmoidLUT(len, lambda, sigma) (LUTCollection.cpp:38-82 over LUTbase.cpp:12-20): the limits
// with the double log the reference calls, slope and intercept in float, entries
// 1 / (1 + exp((lambda - x) / sigma)) in double stored as float, x stepping by 1 / slope in float,
// first entry 0 and last 1. Host code, compiled without contraction.
static void sigmoid_lut(size_t len, float lambda, float sigma, float *lut, float *param)
{
    const float eps = sigma * 1e-3f;
    const float lo = static_cast<float>(static_cast<double>(lambda) -
                                        static_cast<double>(sigma) * std::log(static_cast<double>(1.0f / eps)));
    const float hi = static_cast<float>(static_cast<double>(lambda) -
                                        static_cast<double>(sigma) *
                                            std::log(static_cast<double>(1.0f / (1.0f - eps) - 1.0f)));
    const float slope = static_cast<float>(len - 1) / (hi - lo);
    const float intercept = -slope * lo + 0.5f;
    const float invwidth = 1.0f / sigma, delta = 1.0f / slope;
    float x = lo;
    for (size_t i = 0; i < len; ++i, x += delta)
        lut[i] = static_cast<float>(1.0f / (1.0f + std::exp(static_cast<double>((lambda - x) * invwidth))));
    lut[0] = 0.0f;
    lut[len - 1] = 1.0f;
    param[0] = lo;
    param[1] = hi;
    param[2] = slope;
    param[3] = intercept;
}

// Launch the median kernel for kernel size (kx, ky) and mode over nimg images of w x h.
template <int MODE>
static mr_status launch_median(const float *src, int w, int h, size_t nimg, int kx, int ky, const float *wt,
                               float *dst, cudaStream_t s)
{
    using namespace ringalt;
    const size_t npix = static_cast<size_t>(w) * h;
    for (size_t i0 = 0; i0 < nimg; i0 += 65535) {
        const unsigned nz = static_cast<unsigned>(std::min<size_t>(65535, nimg - i0));
        const dim3 grid(div_up(w, 32), div_up(h, 8), nz), block(32, 8);
        const float *a = src + i0 * npix;
        float *b = dst + i0 * npix;
        if (kx == 5 && ky == 5) {
            k_median55_pair<MODE><<<dim3(div_up(w, 64), div_up(h, 8), nz), block, 0, s>>>(a, w, h, wt, b);
            continue;
        }
#define MR_MEDIAN_CASE(KX, KY)                                                                                         \
    if (kx == KX && ky == KY) {                                                                                        \
        k_median<KX, KY, MODE><<<grid, block, 0, s>>>(a, w, h, wt, b);                                                \
        continue;                                                                                                      \
    }
        MR_MEDIAN_CASE(1, 1)
        MR_MEDIAN_CASE(3, 1)
        MR_MEDIAN_CASE(1, 3)
        MR_MEDIAN_CASE(3, 3)
        MR_MEDIAN_CASE(5, 1)
        MR_MEDIAN_CASE(1, 5)
        MR_MEDIAN_CASE(5, 3)
        MR_MEDIAN_CASE(3, 5)
#undef MR_MEDIAN_CASE
        return fail(MR_ERR_UNSUPPORTED, "median filter: kernel %dx%d", kx, ky);
    }
    return check_launch("k_median");
}

static bool median_size_ok(size_t w, size_t h, int kx, int ky)
{
    return w >= 1 && h >= 1 && w <= (1u << 30) && h <= 524280 && w * h <= (size_t(1) << 31) &&
           w >= static_cast<size_t>(2 * (kx / 2)) && h >= static_cast<size_t>(2 * (ky / 2));
}

static mr_status mean_projection(const float *proj, size_t npix, size_t nproj, int from_zero, float *mean,
                                 cudaStream_t s)
{
    const float scale = 1.0f / static_cast<float>(nproj);
    const bool vec = npix % 4 == 0 && reinterpret_cast<uintptr_t>(proj) % 16 == 0;
    if (vec)
        ringalt::k_mean_projection<true><<<div_up(npix / 4, 256), 256, 0, s>>>(proj, npix, nproj, from_zero, scale, mean);
    else
        ringalt::k_mean_projection<false><<<div_up(npix, 256), 256, 0, s>>>(proj, npix, nproj, from_zero, scale, mean);
    return check_launch("k_mean_projection");
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_median_filter(const float *img_d, size_t nu, size_t nv, size_t nimg, int kx, int ky, float *out_d,
                           void *stream)
{
    MR_TRACE();
    if (!img_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_median_filter: null pointer");
    if (kx < 1 || ky < 1 || kx > 5 || ky > 5 || !(kx & 1) || !(ky & 1))
        return fail(MR_ERR_UNSUPPORTED, "mr_median_filter: kernel %dx%d (odd sizes up to 5)", kx, ky);
    if (!median_size_ok(nu, nv, kx, ky))
        return fail(MR_ERR_ARGUMENT, "mr_median_filter: image %zux%zu for a %dx%d kernel", nu, nv, kx, ky);
    if (img_d == out_d) return fail(MR_ERR_ARGUMENT, "mr_median_filter: the output must not alias the input");
    if (nimg == 0) return MR_OK;
    return launch_median<ringalt::MODE_MEDIAN>(img_d, static_cast<int>(nu), static_cast<int>(nv), nimg, kx, ky,
                                               nullptr, out_d, as_stream(stream));
}

mr_status mr_sigmoid_lut(size_t len, float lambda, float sigma, float *lut_h, float *param_h)
{
    MR_TRACE();
    if (!lut_h || !param_h) return fail(MR_ERR_ARGUMENT, "mr_sigmoid_lut: null pointer");
    if (len < 2) return fail(MR_ERR_ARGUMENT, "mr_sigmoid_lut: at least two entries");
    if (!(sigma > 0.0f) || !std::isfinite(sigma) || !std::isfinite(lambda))
        return fail(MR_ERR_ARGUMENT, "mr_sigmoid_lut: width must be positive and finite");
    sigmoid_lut(len, lambda, sigma, lut_h, param_h);
    return MR_OK;
}

mr_status mr_basicringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, void *stream)
{
    MR_TRACE();
    if (!proj_d) return fail(MR_ERR_ARGUMENT, "mr_basicringclean: null pointer");
    if (!median_size_ok(nu, nv, 3, 3))
        return fail(MR_ERR_ARGUMENT, "mr_basicringclean: projections of %zux%zu (at least 2x2)", nu, nv);
    if (nproj == 0) return MR_OK;
    cudaStream_t s = as_stream(stream);
    const size_t npix = nu * nv;
    float *work = nullptr;
    MR_TRY(device_alloc(&work, 2 * npix * sizeof(float), s, "mr_basicringclean: scratch"));
    float *mean = work, *diff = work + npix;
    mr_status st = mean_projection(proj_d, npix, nproj, 0, mean, s);
    if (st == MR_OK)
        st = launch_median<ringalt::MODE_DIFF>(mean, static_cast<int>(nu), static_cast<int>(nv), 1, 3, 3, nullptr,
                                               diff, s);
    if (st == MR_OK) {
        const bool vec = npix % 4 == 0 && reinterpret_cast<uintptr_t>(proj_d) % 16 == 0;
        const size_t items = vec ? npix * nproj / 4 : npix * nproj;
        const unsigned blocks = static_cast<unsigned>(std::min<size_t>(div_up(items, 256), 148 * 16));
        if (vec)
            ringalt::k_subtract<true><<<blocks, 256, 0, s>>>(proj_d, npix, nproj, diff);
        else
            ringalt::k_subtract<false><<<blocks, 256, 0, s>>>(proj_d, npix, nproj, diff);
        st = check_launch("k_subtract");
    }
    cudaFreeAsync(work, s);
    return st;
}

mr_status mr_medianmixringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, float threshold, float width,
                                void *stream)
{
    MR_TRACE();
    if (!proj_d) return fail(MR_ERR_ARGUMENT, "mr_medianmixringclean: null pointer");
    const int pky = nv < 3 ? 1 : 3, pkx = nv < 3 ? 5 : 3, mky = nv < 5 ? 1 : 5;
    if (!median_size_ok(nu, nv, pkx, pky) || !median_size_ok(nu, nv, 5, mky))
        return fail(MR_ERR_ARGUMENT, "mr_medianmixringclean: projections of %zux%zu (at least 4 wide)", nu, nv);
    if (!(width > 0.0f) || !std::isfinite(width) || !std::isfinite(threshold))
        return fail(MR_ERR_ARGUMENT, "mr_medianmixringclean: width must be positive and finite");
    if (nproj == 0) return MR_OK;
    cudaStream_t s = as_stream(stream);
    const size_t npix = nu * nv, len = 1024;
    std::vector<float> table(len + 4);
    sigmoid_lut(len, threshold, width, table.data(), table.data() + len);
    // batch of projections filtered out of place: about 512 MiB
    const size_t batch = std::max<size_t>(1, std::min<size_t>(nproj, (size_t(1) << 27) / npix));
    float *work = nullptr;
    MR_TRY(device_alloc(&work, (2 * npix + len + 4 + batch * npix) * sizeof(float), s, "mr_medianmixringclean: scratch"));
    float *mean = work, *wt = work + npix, *lut = work + 2 * npix, *out = lut + len + 4;
    mr_status st = MR_OK;
    cudaError_t e = cudaMemcpyAsync(lut, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "mr_medianmixringclean: table upload: %s", cudaGetErrorString(e));
    if (st == MR_OK) st = mean_projection(proj_d, npix, nproj, 1, mean, s);
    if (st == MR_OK)
        st = launch_median<ringalt::MODE_ABSDIFF>(mean, static_cast<int>(nu), static_cast<int>(nv), 1, pkx, pky,
                                                  nullptr, wt, s);
    if (st == MR_OK) {
        ringalt::k_lut<<<div_up(npix, 256), 256, 0, s>>>(wt, npix, lut, static_cast<int>(len));
        st = check_launch("k_lut");
    }
    for (size_t i0 = 0; i0 < nproj && st == MR_OK; i0 += batch) {
        const size_t b = std::min(batch, nproj - i0);
        float *p = proj_d + i0 * npix;
        st = launch_median<ringalt::MODE_MIX>(p, static_cast<int>(nu), static_cast<int>(nv), b, 5, mky, wt, out, s);
        if (st == MR_OK) {
            e = cudaMemcpyAsync(p, out, b * npix * sizeof(float), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "mr_medianmixringclean: copy back: %s", cudaGetErrorString(e));
        }
    }
    cudaFreeAsync(work, s);
    return st;
}

} // extern "C"
