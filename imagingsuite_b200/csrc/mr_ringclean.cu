// Wavelet-FFT ring cleaning: StripeFilter and WaveletRingClean on the GPU.
//
// Reference: core/algorithms/ImagingAlgorithms/src/StripeFilter.cpp:68-250 (Münch-style
// vertical-stripe suppression), the separable DWT/IDWT of core/kipl/kipl/include/wavelets/
// core/wavelets.hpp:452-862 and WaveletRingClean::ProcessSingle (frameworks/tomography/
// Preprocessing/StdPreprocModules/src/WaveletRingClean.cpp:74-103).
//
// A batch of sinograms goes through the steps below. WaveletRingClean's sinograms are the
// detector rows of the projection stack: the first analysis pass reads them and the last
// synthesis pass writes them where they are (a row map, no gathered copy).
//   analysis levels  rows (k_dwt_rows_t: both filters per output) then columns (k_dwt_cols_t:
//                    the four sub-bands), mirror padding as pad_mirror, every output the sum
//                    over the taps in the reference's order;
//   stripe damping   every column of every level's vertical band: zero-padded to 2L, FFT,
//                    times the even response built from CreateFilterWindow, inverse FFT
//                    (k_stripe_fft, shared-memory FFT of mr_fft.cuh, two columns per CTA);
//   synthesis        upsampled convolution of the four bands, rows then columns, summed as
//                    ((a + h) + v) + d, cropped to the sinogram on the last level.
// The DWT/IDWT arithmetic is the reference's operation for operation; only the FFT differs
// from the reference's FFTW in float rounding.
#include "mr_common.cuh"
#include "mr_fft.cuh"
#include "mr_daubechies.h"

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace mr {

MR_BOUNDS_TAKE(bounds_take_ring)

namespace rc {

constexpr int kMaxLevels = 16;

// value at position p of pad_mirror(src, n, fw) (wavelets.hpp:648-667)
__device__ __forceinline__ int mirror_index(int n, int fw, int p)
{
    if (p < fw) return fw - 1 - p;
    if (p < fw + n) return p - fw;
    return n - 1 - (p - fw - n);
}

// index t in dyadup(src, n) padded by pad_mirror(., 2n, fw); odd t are the inserted zeros
__device__ __forceinline__ int up_index(int n, int fw, int q)
{
    if (q < fw) return fw - 1 - q;
    if (q < fw + 2 * n) return q - fw;
    return 2 * n - 1 - (q - fw - 2 * n);
}

// Rows of a stack of sinograms: row r (sinogram b = r / rows, position p = r % rows) starts at
// base + b * bstride + p * rstride. Contiguous sinograms [B][rows][len] have bstride =
// rows * len and rstride = len; the sinograms of a projection stack [ntheta][nv][nu] (detector
// row j0 + b, angle p) have bstride = nu and rstride = nv * nu, so the first analysis and the
// last synthesis pass read and write the projections where they are.
struct RowMap {
    size_t bstride, rstride;
    int rows;
    __host__ __device__ size_t at(int r) const { return (r / rows) * bstride + (r % rows) * rstride; }
};

__host__ __device__ inline RowMap contiguous_rows(int rows, int len)
{
    return RowMap{static_cast<size_t>(rows) * len, static_cast<size_t>(len), rows};
}

// FilterVerticalStripes (StripeFilter.cpp:114-135): every column of the vertical band
// [B][bh][bw] zero-padded, filtered with the even real response, first bh samples kept. Two
// columns of one sinogram (2j, 2j + 1) share a complex transform as its real and imaginary
// parts, so a column's rounding does not depend on how sinograms are batched.
__global__ void k_stripe_fft(float *__restrict__ band, int bw, int bh, int n, int logn,
                             const float2 *__restrict__ twiddle, const float *__restrict__ response)
{
    extern __shared__ float2 buf[];
    const int pairs = (bw + 1) / 2;
    const int sino = blockIdx.x / pairs, c0 = 2 * (blockIdx.x % pairs);
    const bool has1 = c0 + 1 < bw;
    const size_t base0 = static_cast<size_t>(sino) * bw * bh + c0;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        float x0 = 0.0f, x1 = 0.0f;
        if (p < bh) {
            x0 = band[base0 + static_cast<size_t>(p) * bw];
            if (has1) x1 = band[base0 + 1 + static_cast<size_t>(p) * bw];
        }
        buf[fft_slot(p)] = make_float2(x0, x1);
    }
    __syncthreads();
    fft_forward(buf, logn, twiddle);
    fft_apply_response(buf, n, response);
    fft_inverse(buf, logn, twiddle);
    for (int p = threadIdx.x; p < bh; p += blockDim.x) {
        const float2 v = buf[fft_slot(p)];
        band[base0 + static_cast<size_t>(p) * bw] = v.x;
        if (has1) band[base0 + 1 + static_cast<size_t>(p) * bw] = v.y;
    }
}

// ---- the four convolution passes: analysis rows (both filters per output) and columns (the
// four sub-bands, wavelets.hpp:474-487); synthesis rows and columns of upsconvRC (:750-858)
// summed as ((a + h) + v) + d (WaveletTransform::synthesize :626-645). Every output is the sum
// over the taps in the reference's order, with the reference's float operations. The tap count
// K is a template parameter (every daubN the library defines), so the tap loops unroll
// completely and the taps sit in registers (in shared memory when K > 32). Away from the
// borders (where the mirrored index is the identity) the window is read directly; in the
// synthesis passes the interior skips the taps that meet the zeros inserted by the dyadic
// upsampling (adding a product with 0 leaves a nonzero sum unchanged, so only the sign of an
// exactly zero result can differ). Blocks that touch a border take a per-output form with the
// mirrored indices.
constexpr int kConvThreads = 128;
constexpr int kBlk = 8;    // column passes: consecutive outputs per thread
constexpr int kRowBlk = 6; // synthesis rows: consecutive outputs per thread (lanes' inputs 3 words apart)

__device__ __forceinline__ void load_taps(const float *__restrict__ taps, int n, float *sm)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) sm[i] = taps[i];
    __syncthreads();
}

template <int K>
struct Taps {
    static constexpr bool kRegs = K <= 32;
    float r[kRegs ? 2 * K : 1];
    const float *sm;
    __device__ __forceinline__ explicit Taps(const float *shared) : sm(shared)
    {
        if constexpr (kRegs) {
#pragma unroll
            for (int i = 0; i < 2 * K; ++i) r[i] = shared[i];
        }
    }
    // tap i of the pair [first K | second K]
    __device__ __forceinline__ float operator[](int i) const
    {
        if constexpr (kRegs) return r[i];
        else return sm[i];
    }
};

// Analysis rows: aH[k] = sum_j tH[j] x[2k + 1 - j], aG the same with tG (j ascending), x the
// row mirror-padded as pad_mirror. A CTA covers kConvThreads * kRowOut outputs of a row; it
// stages the inputs they read, mirrored indices resolved, split by parity (E[e] = x[2e],
// O[e] = x[2e + 1]), so that consecutive outputs read consecutive words (no bank conflicts) and
// the border outputs need no separate path. A thread computes outputs kConvThreads apart; the
// two products of a tap are one paired multiply (each element rounded as the scalar one; a
// paired multiply feeding scalar adds is not contracted).
constexpr int kRowOut = 4;

template <int K>
__global__ void __launch_bounds__(kConvThreads) k_dwt_rows_t(const float *__restrict__ src, RowMap in, int sx,
                                                             int nrows, const float *__restrict__ taps, int dx,
                                                             float *__restrict__ tmpH, float *__restrict__ tmpG)
{
    constexpr int SEG = kConvThreads * kRowOut, KH = K / 2, NE = SEG + KH - 1;
    __shared__ float2 tp2[K];
    __shared__ float ev[NE], od[NE];
    for (int i = threadIdx.x; i < K; i += kConvThreads) tp2[i] = make_float2(taps[i], taps[K + i]);
    const int kc = blockIdx.x * SEG;
    const int e0 = kc - KH + 1; // E[i] = x[2 (e0 + i)], O[i] = x[2 (e0 + i) + 1]
    for (int row = blockIdx.y; row < nrows; row += gridDim.y) {
        const float *r = src + in.at(row);
        __syncthreads(); // the previous row's inputs are consumed
        for (int i = threadIdx.x; i < NE; i += kConvThreads) {
            const int p = K + 2 * (e0 + i); // position in the padded row
            // positions no output of this row reads (past the last output) are not staged
            const bool used = e0 + i <= dx - 1;
            ev[i] = used ? r[mirror_index(sx, K, p)] : 0.0f;
            od[i] = used ? r[mirror_index(sx, K, p + 1)] : 0.0f;
        }
        __syncthreads();
        float aH[kRowOut], aG[kRowOut];
#pragma unroll
        for (int o = 0; o < kRowOut; ++o) aH[o] = aG[o] = 0.0f;
        const int t0 = threadIdx.x + KH - 1; // (k - kc) + KH - 1 for o = 0
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const float2 tt = tp2[j];
#pragma unroll
            for (int o = 0; o < kRowOut; ++o) {
                const int i = t0 + o * kConvThreads;
                const int ix = (j & 1) ? i - (j - 1) / 2 : i - j / 2;
                if (!MR_IN_BOUNDS(ix, NE, kSiteRingRows)) continue;
                const float x = (j & 1) ? ev[ix] : od[ix];
                const float2 pr = __fmul2_rn(tt, make_float2(x, x));
                aH[o] = __fadd_rn(aH[o], pr.x);
                aG[o] = __fadd_rn(aG[o], pr.y);
            }
        }
#pragma unroll
        for (int o = 0; o < kRowOut; ++o) {
            const int k = kc + threadIdx.x + o * kConvThreads;
            if (k < dx) {
                tmpH[static_cast<size_t>(row) * dx + k] = aH[o];
                tmpG[static_cast<size_t>(row) * dx + k] = aG[o];
            }
        }
    }
}

// Analysis columns: the four sub-bands a = tH.H, h = tG.H, v = tH.G, d = tG.G of output row k
// (rows 2k + 1 - m, m ascending). A thread computes kBlk consecutive outputs of a column and
// walks their shared input rows once, from the last to the first, adding each row into every
// output whose tap index m is in range: per output the rows arrive with m ascending.
template <int K>
__global__ void __launch_bounds__(kConvThreads) k_dwt_cols_t(const float *__restrict__ tmpH,
                                                             const float *__restrict__ tmpG, int dx, int sy,
                                                             const float *__restrict__ taps, int dy,
                                                             float *__restrict__ a, float *__restrict__ h,
                                                             float *__restrict__ v, float *__restrict__ d)
{
    __shared__ float tp[2 * K];
    load_taps(taps, 2 * K, tp);
    const int x = blockIdx.x * kConvThreads + threadIdx.x, k0 = blockIdx.y * kBlk, b = blockIdx.z;
    if (x >= dx) return;
    const Taps<K> t(tp);
    const size_t base = static_cast<size_t>(b) * sy * dx + x;
    const int k1 = min(k0 + kBlk, dy);
    const bool inner = 2 * k0 - K + 2 >= 0 && 2 * (k1 - 1) + 1 < sy && k1 - k0 == kBlk;
    if (inner) {
        float sa[kBlk], sh[kBlk], sv[kBlk], sd[kBlk];
#pragma unroll
        for (int o = 0; o < kBlk; ++o) sa[o] = sh[o] = sv[o] = sd[o] = 0.0f;
        const float *cH = tmpH + base + static_cast<size_t>(2 * k0) * dx;
        const float *cG = tmpG + base + static_cast<size_t>(2 * k0) * dx;
#pragma unroll
        for (int e = 2 * kBlk - 1; e >= 2 - K; --e) { // row 2 k0 + e
            const float ph = __ldg(cH + static_cast<ptrdiff_t>(e) * dx), pg = __ldg(cG + static_cast<ptrdiff_t>(e) * dx);
#pragma unroll
            for (int o = 0; o < kBlk; ++o) {
                const int m = 2 * o + 1 - e;
                if (m >= 0 && m < K) {
                    const float th = t[m], tg = t[K + m];
                    sa[o] = __fadd_rn(sa[o], __fmul_rn(th, ph));
                    sh[o] = __fadd_rn(sh[o], __fmul_rn(tg, ph));
                    sv[o] = __fadd_rn(sv[o], __fmul_rn(th, pg));
                    sd[o] = __fadd_rn(sd[o], __fmul_rn(tg, pg));
                }
            }
        }
#pragma unroll
        for (int o = 0; o < kBlk; ++o) {
            const size_t q = (static_cast<size_t>(b) * dy + k0 + o) * dx + x;
            a[q] = sa[o];
            h[q] = sh[o];
            v[q] = sv[o];
            d[q] = sd[o];
        }
        return;
    }
    for (int k = k0; k < k1; ++k) {
        const bool in = 2 * k - K + 2 >= 0 && 2 * k + 1 < sy;
        float sa = 0.0f, sh = 0.0f, sv = 0.0f, sd = 0.0f;
        for (int m = 0; m < K; ++m) {
            const int row = in ? 2 * k - m + 1 : mirror_index(sy, K, K + 2 * k - m + 1);
            const size_t idx = base + static_cast<size_t>(row) * dx;
            const float ph = tmpH[idx], pg = tmpG[idx];
            sa = __fadd_rn(sa, __fmul_rn(tp[m], ph));
            sh = __fadd_rn(sh, __fmul_rn(tp[K + m], ph));
            sv = __fadd_rn(sv, __fmul_rn(tp[m], pg));
            sd = __fadd_rn(sd, __fmul_rn(tp[K + m], pg));
        }
        const size_t q = (static_cast<size_t>(b) * dy + k) * dx + x;
        a[q] = sa;
        h[q] = sh;
        v[q] = sv;
        d[q] = sd;
    }
}

// Synthesis rows of band q = blockIdx.z (a, h with the first synthesis filter, v, d with the
// second): out[k] = sum over m of the parity of k + c, ascending, of src[(k + c - m) / 2] f[m].
// A CTA covers kConvThreads * kRowBlk outputs of a row; their inputs are staged in shared
// memory and the outputs leave through shared memory (coalesced rows both ways). With k0 even
// and c = K - 2 even, output o of a thread's block uses m = o - 2 g for the input
// src[(k0 + c) / 2 + g]. F is the band's filter offset in the tap pair.
template <int K, int F>
__device__ __forceinline__ void up_rows_block(const float *tp, const float *xin, int in0, int xoff, int k0, int kc,
                                              int w, int dx, float *yout)
{
    constexpr int c = K - 2, KH = K / 2;
    if (k0 >= 1 && k0 + kRowBlk - 1 < 2 * w - K + 2 && k0 + kRowBlk <= dx) {
        float f[K];
#pragma unroll
        for (int m = 0; m < K; ++m) f[m] = tp[F + m];
        float acc[kRowBlk];
#pragma unroll
        for (int o = 0; o < kRowBlk; ++o) acc[o] = 0.0f;
        const float *s0 = xin + xoff; // src[(k0 + c) / 2]
#pragma unroll
        for (int g = kRowBlk / 2 - 1; g >= 1 - KH; --g) {
            if (!MR_IN_BOUNDS(xoff + g, kConvThreads * kRowBlk / 2 + KH + 2, kSiteRingRows)) continue;
            const float xv = s0[g];
#pragma unroll
            for (int o = 0; o < kRowBlk; ++o) {
                const int m = o - 2 * g;
                if (m >= 0 && m < K) acc[o] = __fadd_rn(acc[o], __fmul_rn(xv, f[m]));
            }
        }
#pragma unroll
        for (int o = 0; o < kRowBlk; ++o) yout[k0 - kc + o] = acc[o];
        return;
    }
    // a block that reaches a border: its interior outputs here, its border outputs in the CTA's
    // border phase (k_up_rows_t), one per thread
    for (int k = k0; k < min(k0 + kRowBlk, dx); ++k) {
        if (k < 1 || k >= 2 * w - K + 2) continue;
        float acc = 0.0f;
        for (int m = (k + c) & 1; m < K; m += 2) acc = __fadd_rn(acc, __fmul_rn(xin[((k + c - m) >> 1) - in0], tp[F + m]));
        yout[k - kc] = acc;
    }
}

// A border output of the synthesis rows: every tap of the mirror-padded upsampled row (the
// inserted zeros included, as the reference adds them). The staged inputs hold the indices it
// reads except, in a CTA that starts within the right border band, some mirrored ones (read from
// the row itself).
template <int K>
__device__ __forceinline__ float up_rows_border(const float *__restrict__ src, const float *f, const float *xin,
                                                int in0, int nin, int k, int w)
{
    constexpr int c = K - 2;
    float acc = 0.0f;
    for (int m = 0; m < K; ++m) {
        const int ti = up_index(w, K, K + k + c - m);
        float xv = 0.0f;
        if (!(ti & 1)) {
            const int i = (ti >> 1) - in0;
            xv = (i >= 0 && i < nin) ? xin[i] : __ldg(src + (ti >> 1));
        }
        acc = __fadd_rn(acc, __fmul_rn(xv, f[m]));
    }
    return acc;
}

template <int K>
__global__ void __launch_bounds__(kConvThreads) k_up_rows_t(const float *__restrict__ a, const float *__restrict__ hb,
                                                            const float *__restrict__ vb, const float *__restrict__ db,
                                                            int w, int nrows, const float *__restrict__ taps, int dx,
                                                            float *__restrict__ out)
{
    constexpr int c = K - 2, KH = K / 2, SEG = kConvThreads * kRowBlk, NIN = SEG / 2 + KH + 2;
    __shared__ float tp[2 * K];
    __shared__ float xin[NIN];
    __shared__ float yout[SEG];
    load_taps(taps + 2 * K, 2 * K, tp);
    const int q = blockIdx.z;
    const int kc = blockIdx.x * SEG;                  // first output of the CTA (even)
    const int k0 = kc + threadIdx.x * kRowBlk;         // first output of the thread (even)
    const int in0 = (kc + c) / 2 - KH + 1;             // input index held in xin[0]
    const int xoff = (k0 + c) / 2 - in0;               // = 3 * threadIdx.x + KH - 1
    const float *band = q == 0 ? a : q == 1 ? hb : q == 2 ? vb : db;
    const size_t plane = static_cast<size_t>(nrows) * dx;
    for (int row = blockIdx.y; row < nrows; row += gridDim.y) {
        const float *src = band + static_cast<size_t>(row) * w;
        __syncthreads(); // the previous row's xin and yout are consumed
        for (int i = threadIdx.x; i < NIN; i += kConvThreads) {
            const int e = in0 + i;
            xin[i] = (e >= 0 && e < w) ? __ldg(src + e) : 0.0f;
        }
        __syncthreads();
        if (k0 < dx) {
            if (q < 2) up_rows_block<K, 0>(tp, xin, in0, xoff, k0, kc, w, dx, yout);
            else up_rows_block<K, K>(tp, xin, in0, xoff, k0, kc, w, dx, yout);
        }
        // border outputs of the CTA (output 0, and 2w - K + 2 .. dx - 1), one per thread
        {
            const int r0 = max(kc, 2 * w - K + 2), r1 = min(kc + SEG, dx);
            const int nleft = kc == 0 ? 1 : 0, nright = max(0, r1 - r0);
            for (int i = threadIdx.x; i < nleft + nright; i += kConvThreads) {
                const int k = i < nleft ? 0 : r0 + (i - nleft);
                yout[k - kc] = up_rows_border<K>(src, tp + (q < 2 ? 0 : K), xin, in0, NIN, k, w);
            }
        }
        __syncthreads();
        float *o_ = out + q * plane + static_cast<size_t>(row) * dx + kc;
        for (int i = threadIdx.x; i < SEG && kc + i < dx; i += kConvThreads) o_[i] = yout[i];
    }
}

// Synthesis columns: the four row-synthesised planes through their column filters, summed as
// ((a + h) + v) + d per output; output row k of sinogram b starts at out + om.at(b * oy + k).
template <int K>
__global__ void __launch_bounds__(kConvThreads) k_up_cols_t(const float *__restrict__ rows, int dx, int h, int nb,
                                                            const float *__restrict__ taps, int ox, int oy,
                                                            float *__restrict__ out, RowMap om)
{
    __shared__ float tp[2 * K];
    load_taps(taps + 2 * K, 2 * K, tp);
    const int x = blockIdx.x * kConvThreads + threadIdx.x, k0 = blockIdx.y * kBlk, b = blockIdx.z;
    if (x >= ox) return;
    const Taps<K> t(tp);
    constexpr int c = K - 2, KH = K / 2;
    const size_t plane = static_cast<size_t>(nb) * h * dx;
    const size_t base = static_cast<size_t>(b) * h * dx + x;
    const int k1 = min(k0 + kBlk, oy);
    const bool inner = k0 >= 1 && k1 - 1 < 2 * h - K + 2 && k1 - k0 == kBlk;
    if (inner) {
        float sum[kBlk];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int f = (q == 0 || q == 2) ? 0 : K;
            const float *col = rows + q * plane + base + static_cast<size_t>((k0 + c) / 2) * dx;
            float acc[kBlk];
#pragma unroll
            for (int o = 0; o < kBlk; ++o) acc[o] = 0.0f;
#pragma unroll
            for (int g = kBlk / 2 - 1; g >= 1 - KH; --g) {
                const float xv = __ldg(col + static_cast<ptrdiff_t>(g) * dx);
#pragma unroll
                for (int o = 0; o < kBlk; ++o) {
                    const int m = o - 2 * g;
                    if (m >= 0 && m < K) acc[o] = __fadd_rn(acc[o], __fmul_rn(xv, t[f + m]));
                }
            }
#pragma unroll
            for (int o = 0; o < kBlk; ++o) sum[o] = q == 0 ? acc[o] : __fadd_rn(sum[o], acc[o]);
        }
#pragma unroll
        for (int o = 0; o < kBlk; ++o) out[b * om.bstride + (k0 + o) * om.rstride + x] = sum[o];
        return;
    }
    for (int k = k0; k < k1; ++k) {
        const bool in = k >= 1 && k < 2 * h - K + 2;
        float s4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int f = (q == 0 || q == 2) ? 0 : K;
            const float *col = rows + q * plane + base;
            float acc = 0.0f;
            if (in) {
                for (int m = (k + c) & 1; m < K; m += 2)
                    acc = __fadd_rn(acc, __fmul_rn(col[static_cast<size_t>((k + c - m) >> 1) * dx], tp[f + m]));
            } else {
                for (int m = 0; m < K; ++m) {
                    const int ti = up_index(h, K, K + k + c - m);
                    const float xv = (ti & 1) ? 0.0f : col[static_cast<size_t>(ti >> 1) * dx];
                    acc = __fadd_rn(acc, __fmul_rn(xv, tp[f + m]));
                }
            }
            s4[q] = acc;
        }
        out[b * om.bstride + k * om.rstride + x] = __fadd_rn(__fadd_rn(__fadd_rn(s4[0], s4[1]), s4[2]), s4[3]);
    }
}

struct Plan {
    int K = 0, begin = 0, end = 0, levels = 0;
    int sx[kMaxLevels + 1], sy[kMaxLevels + 1];
    int nfft[kMaxLevels];
    std::vector<float> taps;                 // tH | tG | sH | sG
    std::vector<std::vector<float>> resp;    // responses per level (length nfft), digit-reversed order
};

} // namespace rc

// WaveletKernel<float> for 'daubN' (wavelets.hpp:100-405: CopyKernel(k, 0, 2N-1)); the
// reference's daub3 table has the sign of its fifth coefficient flipped, kept here for parity.
static mr_status wavelet_taps(const char *wname, int *begin, int *end, std::vector<float> &taps)
{
    std::string name(wname ? wname : "");
    if (name.compare(0, 4, "daub") != 0) return fail(MR_ERR_UNSUPPORTED, "unsupported wavelet '%s' (daub1..daub30)", name.c_str());
    const int n = std::atoi(name.c_str() + 4);
    if (n < 1 || n > kDaubMax) return fail(MR_ERR_UNSUPPORTED, "Daubechies are only supported for N<=30");
    // kipl's daub28 table has 48 entries for its 56 taps (wavelets.hpp, WaveletKernel case 28):
    // the reference kernel copies 8 values from past the array, so its result is undefined
    if (n == 28)
        return fail(MR_ERR_UNSUPPORTED, "daub28 is not supported: the reference's table is shorter than the filter");
    const int K = 2 * n, e = K - 1;
    std::vector<double> k(kDaub[n - 1], kDaub[n - 1] + K);
    if (n == 3) k[4] = -k[4];
    taps.assign(4 * K, 0.0f);
    double sgn = -1.0; // start = 0 is even
    std::vector<float> tG(K);
    for (int i = 0; i < K; ++i) {
        taps[i] = static_cast<float>(k[e - i]);          // analysis H
        tG[i] = static_cast<float>(sgn * k[i]);          // analysis G
        taps[2 * K + i] = static_cast<float>(k[i]);      // synthesis H
        sgn *= -1.0;
    }
    for (int i = 0; i < K; ++i) {
        taps[K + i] = tG[i];
        taps[3 * K + i] = tG[e - i];                     // synthesis G
    }
    *begin = 0;
    *end = e;
    return MR_OK;
}

static size_t next_power2(size_t n)
{
    const double logtwo = std::log(2.0);
    return static_cast<size_t>(std::floor(std::exp(logtwo * std::ceil(std::log(static_cast<double>(n)) / logtwo)) + 0.5));
}

static int ilog2i(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

static mr_status make_plan(size_t nu, size_t ntheta, const char *wname, int decnum, float sigma, rc::Plan &P)
{
    mr_status st = wavelet_taps(wname, &P.begin, &P.end, P.taps);
    if (st != MR_OK) return st;
    P.K = P.end - P.begin + 1;
    if (decnum < 1 || decnum > rc::kMaxLevels) return fail(MR_ERR_ARGUMENT, "decomposition levels must be 1..%d", rc::kMaxLevels);
    P.levels = decnum;
    P.sx[0] = static_cast<int>(nu);
    P.sy[0] = static_cast<int>(ntheta);
    for (int l = 0; l < decnum; ++l) {
        if (P.sx[l] < P.K || P.sy[l] < P.K) return fail(MR_ERR_ARGUMENT, "Image smaller than wavelet kernel size");
        P.sx[l + 1] = (P.sx[l] + P.K - 1 + (P.sx[l] & 1)) / 2;
        P.sy[l + 1] = (P.sy[l] + P.K - 1 + (P.sy[l] & 1)) / 2;
    }
    // CreateFilterWindow (StripeFilter.cpp:68-81) and configure's FFT lengths (:222-235): the
    // reference filters each column of a level's vertical band (bh samples) zero-padded to
    // N = 2L with the even response R[k] = damp(min(k, N - k)) (1/N included), keeping the first
    // bh samples: y[p] = sum_q x[q] h[p - q] with h[l] = sum_k R[k] cos(2 pi k l / N). Only the
    // lags |l| < bh enter, so a circular convolution of length M >= 2 bh - 1 with h cut to those
    // lags is the same operator; it runs at the shortest power of two M (response
    // G = DFT_M(h cut) / M, unnormalised inverse), which is N / 2 for the usual sizes. h and G
    // are computed in double.
    const float s = -1.0f / (2.0f * sigma * sigma);
    P.resp.resize(decnum);
    for (int l = 0; l < decnum; ++l) {
        const size_t L = next_power2(static_cast<size_t>(1.25 * static_cast<int>(ntheta)) >> l);
        const size_t N = 2 * L;
        if (N > 16384) return fail(MR_ERR_UNSUPPORTED, "stripe filter FFT length %zu above 16384", N);
        const size_t bh = static_cast<size_t>(P.sy[l + 1]);
        if (bh > N) return fail(MR_ERR_ARGUMENT, "band taller than its FFT length");
        const float scale = 1.0f / (2.0f * L);
        std::vector<float> damp(N);
        for (size_t i = 0; i < N; ++i) {
            float w = static_cast<float>(i) * scale;
            damp[i] = (1.0f - std::exp(w * w * s)) * scale;
        }
        // full-length response (the c2r reads bins 0..N/2: damp on 0..N/2, mirrored above)
        std::vector<double> h(N), zero(N, 0.0);
        for (size_t k = 0; k < N; ++k) h[k] = damp[k <= N / 2 ? k : N - k];
        const size_t M = std::min(N, next_power2(2 * bh - 1));
        std::vector<float> resp(M);
        if (M == N) {
            for (size_t k = 0; k < N; ++k) resp[k] = static_cast<float>(h[k]);
        } else {
            host_dft(h, zero, +1); // h[l] = sum_k R[k] exp(+2 pi i k l / N), real
            std::vector<double> g(M, 0.0), gi(M, 0.0);
            g[0] = h[0];
            for (size_t j = 1; j < bh; ++j) g[j] = g[M - j] = h[j];
            host_dft(g, gi, -1);
            for (size_t k = 0; k < M; ++k) resp[k] = static_cast<float>(g[k] / static_cast<double>(M));
        }
        P.nfft[l] = static_cast<int>(M);
        // in the order of the forward transform's output
        P.resp[l] = fft_permute_response(resp, ilog2i(static_cast<int>(M)));
    }
    return MR_OK;
}


// The convolution passes with the tap count as a template parameter.
template <int K>
static void conv_analysis_t(const float *src, rc::RowMap in, int sx, int sy, int dx, int dy, int nb,
                            const float *taps_d, float *tH, float *tG, float *a, float *h, float *v, float *d,
                            cudaStream_t st)
{
    using namespace rc;
    const int rows = nb * sy;
    k_dwt_rows_t<K><<<dim3(div_up(dx, kConvThreads * kRowOut), std::min(rows, 65535)), kConvThreads, 0, st>>>(
        src, in, sx, rows, taps_d, dx, tH, tG);
    k_dwt_cols_t<K><<<dim3(div_up(dx, kConvThreads), div_up(dy, kBlk), nb), kConvThreads, 0, st>>>(
        tH, tG, dx, sy, taps_d, dy, a, h, v, d);
}

template <int K>
static void conv_synthesis_t(const float *a, const float *h, const float *v, const float *d, int w, int hgt, int dx,
                             int ox, int oy, int nb, const float *taps_d, float *tmp, float *out, rc::RowMap om,
                             cudaStream_t st)
{
    using namespace rc;
    const int rows = nb * hgt;
    k_up_rows_t<K><<<dim3(div_up(dx, kConvThreads * kRowBlk), std::min(rows, 65535), 4), kConvThreads, 0, st>>>(
        a, h, v, d, w, rows, taps_d, dx, tmp);
    k_up_cols_t<K><<<dim3(div_up(ox, kConvThreads), div_up(oy, kBlk), nb), kConvThreads, 0, st>>>(
        tmp, dx, hgt, nb, taps_d, ox, oy, out, om);
}

// every daubN filter length (2N) except daub28's, which the library refuses
#define MR_RC_TAPS(X)                                                                                         \
    X(2) X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(18) X(20) X(22) X(24) X(26) X(28) X(30) X(32) X(34) X(36) \
        X(38) X(40) X(42) X(44) X(46) X(48) X(50) X(52) X(54) X(58) X(60)

static bool conv_analysis(int K, const float *src, rc::RowMap in, int sx, int sy, int dx, int dy, int nb,
                          const float *taps_d, float *tH, float *tG, float *a, float *h, float *v, float *d,
                          cudaStream_t st)
{
    switch (K) {
#define MR_RC_CASE(k)                                                                                          \
    case k: conv_analysis_t<k>(src, in, sx, sy, dx, dy, nb, taps_d, tH, tG, a, h, v, d, st); return true;
        MR_RC_TAPS(MR_RC_CASE)
#undef MR_RC_CASE
    default: return false;
    }
}

static bool conv_synthesis(int K, const float *a, const float *h, const float *v, const float *d, int w, int hgt,
                           int dx, int ox, int oy, int nb, const float *taps_d, float *tmp, float *out, rc::RowMap om,
                           cudaStream_t st)
{
    switch (K) {
#define MR_RC_CASE(k)                                                                                          \
    case k: conv_synthesis_t<k>(a, h, v, d, w, hgt, dx, ox, oy, nb, taps_d, tmp, out, om, st); return true;
        MR_RC_TAPS(MR_RC_CASE)
#undef MR_RC_CASE
    default: return false;
    }
}

// Stripe filter of nb sinograms in place: row r of the batch's level-0 image is data + io.at(r)
// (io.rows = ntheta rows of nu samples).
static mr_status stripe_batch(float *data, rc::RowMap io, int nb, const rc::Plan &P, const float *taps_d,
                              const std::vector<float2 *> &tw_d, const std::vector<float *> &resp_d, float *scratch,
                              cudaStream_t st)
{
    using namespace rc;
    const int K = P.K, L = P.levels;
    // scratch layout: per level l=1..L: a, h, v, d [nb][sy][sx]; tmp: H/G rows or up rows [4][nb][h][dx]
    size_t off = 0;
    float *A[kMaxLevels + 1], *Hb[kMaxLevels + 1], *Vb[kMaxLevels + 1], *Db[kMaxLevels + 1];
    A[0] = data;
    for (int l = 1; l <= L; ++l) {
        const size_t n = static_cast<size_t>(nb) * P.sx[l] * P.sy[l];
        A[l] = scratch + off; off += n;
        Hb[l] = scratch + off; off += n;
        Vb[l] = scratch + off; off += n;
        Db[l] = scratch + off; off += n;
    }
    float *tmp = scratch + off;
    for (int l = 0; l < L; ++l) {
        const int sx = P.sx[l], sy = P.sy[l], dx = P.sx[l + 1], dy = P.sy[l + 1];
        float *tH = tmp, *tG = tmp + static_cast<size_t>(nb) * sy * dx;
        const RowMap in = l == 0 ? io : contiguous_rows(sy, sx);
        if (!conv_analysis(K, A[l], in, sx, sy, dx, dy, nb, taps_d, tH, tG, A[l + 1], Hb[l + 1], Vb[l + 1], Db[l + 1],
                           st))
            return fail(MR_ERR_UNSUPPORTED, "stripe filter: no kernel for %d taps", K);
    }
    for (int l = 0; l < L; ++l) {
        const int bw = P.sx[l + 1], bh = P.sy[l + 1], n = P.nfft[l];
        k_stripe_fft<<<nb * ((bw + 1) / 2), std::min(512, std::max(64, n / 8)), fft_buffer_slots(n) * sizeof(float2),
                       st>>>(Vb[l + 1], bw, bh, n, ilog2i(n), tw_d[l], resp_d[l]);
    }
    for (int l = L - 1; l >= 0; --l) {
        const int w = P.sx[l + 1], h = P.sy[l + 1];
        const int dx = l == 0 ? 2 * P.sx[1] : P.sx[l], dy = l == 0 ? 2 * P.sy[1] : P.sy[l];
        const int ox = l == 0 ? P.sx[0] : dx, oy = l == 0 ? P.sy[0] : dy;
        const RowMap om = l == 0 ? io : contiguous_rows(oy, ox);
        if (!conv_synthesis(K, A[l + 1], Hb[l + 1], Vb[l + 1], Db[l + 1], w, h, dx, ox, oy, nb, taps_d, tmp, A[l], om,
                            st))
            return fail(MR_ERR_UNSUPPORTED, "stripe filter: no kernel for %d taps", K);
    }
    return check_launch("stripe filter");
}

// Scratch floats for a batch of nb sinograms.
static size_t stripe_scratch(const rc::Plan &P, int nb)
{
    size_t bands = 0;
    for (int l = 1; l <= P.levels; ++l) bands += 4 * static_cast<size_t>(P.sx[l]) * P.sy[l];
    size_t tmp = 0;
    for (int l = 0; l < P.levels; ++l) {
        tmp = std::max(tmp, 2 * static_cast<size_t>(P.sy[l]) * P.sx[l + 1]);
        const int dx = l == 0 ? 2 * P.sx[1] : P.sx[l];
        tmp = std::max(tmp, 4 * static_cast<size_t>(P.sy[l + 1]) * dx);
    }
    return static_cast<size_t>(nb) * (bands + tmp);
}

// interleaved: data is a projection stack [ntheta][nsino][nu] (the sinograms are its detector
// rows); else nsino contiguous sinograms [nsino][ntheta][nu].
static mr_status run_stripes(float *data_d, bool interleaved, size_t nu, size_t nv_or_nsino, size_t ntheta,
                             const char *wname, int decnum, float sigma, void *stream)
{
    rc::Plan P;
    mr_status st = make_plan(nu, ntheta, wname, decnum, sigma, P);
    if (st != MR_OK) return st;
    cudaStream_t s = as_stream(stream);
    // batch size: about 1 GiB of scratch, at most 65535 sinograms (grid z)
    const size_t per = stripe_scratch(P, 1);
    const size_t nsino = nv_or_nsino;
    const int nb = static_cast<int>(std::max<size_t>(1, std::min<size_t>({nsino, (size_t(1) << 28) / per, size_t(65535)})));
    float *taps_d = nullptr, *work = nullptr;
    std::vector<float2 *> tw_d(P.levels, nullptr);
    std::vector<float *> resp_d(P.levels, nullptr);
    size_t total = 4 * P.K;
    for (int l = 0; l < P.levels; ++l) total += P.nfft[l] * 2 + P.nfft[l];
    total += stripe_scratch(P, nb);
    MR_TRY(device_alloc(&work, total * sizeof(float), s, "stripe filter: scratch"));
    size_t off = 0;
    taps_d = work;
    off += 4 * P.K;
    std::vector<std::vector<float2>> tws(P.levels);
    for (int l = 0; l < P.levels; ++l) {
        tw_d[l] = reinterpret_cast<float2 *>(work + off); // n float2 (offsets stay even: 8-byte aligned)
        off += 2 * static_cast<size_t>(P.nfft[l]);
        resp_d[l] = work + off;
        off += P.nfft[l];
        tws[l] = fft_twiddles(P.nfft[l]);
    }
    float *scratch = work + off;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(rc::k_stripe_fft, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             fft_buffer_slots(16384) * sizeof(float2));
        attr = true;
    }
    cudaError_t e = cudaMemcpyAsync(taps_d, P.taps.data(), P.taps.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    for (int l = 0; l < P.levels && e == cudaSuccess; ++l) {
        e = cudaMemcpyAsync(tw_d[l], tws[l].data(), tws[l].size() * sizeof(float2), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(resp_d[l], P.resp[l].data(), P.resp[l].size() * sizeof(float), cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "stripe filter tables: %s", cudaGetErrorString(e));
    const int rows = static_cast<int>(ntheta);
    for (size_t j0 = 0; j0 < nsino && st == MR_OK; j0 += nb) {
        const int b = static_cast<int>(std::min<size_t>(nb, nsino - j0));
        if (interleaved)
            st = stripe_batch(data_d + j0 * nu, rc::RowMap{nu, nsino * nu, rows}, b, P, taps_d, tw_d, resp_d, scratch, s);
        else
            st = stripe_batch(data_d + j0 * nu * ntheta, rc::contiguous_rows(rows, static_cast<int>(nu)), b, P, taps_d,
                              tw_d, resp_d, scratch, s);
    }
    cudaFreeAsync(work, s);
    return st;
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_wavelet_kernel(const char *wname, int *begin, int *end, float *taps_h)
{
    MR_TRACE();
    if (!begin || !end) return fail(MR_ERR_ARGUMENT, "mr_wavelet_kernel: null pointer");
    std::vector<float> t;
    mr_status st = wavelet_taps(wname, begin, end, t);
    if (st == MR_OK && taps_h) std::copy(t.begin(), t.end(), taps_h);
    return st;
}

mr_status mr_stripefilter(float *sino_d, size_t nu, size_t ntheta, size_t nsino, const char *wname, int decnum,
                          float sigma, void *stream)
{
    MR_TRACE();
    if (!sino_d) return fail(MR_ERR_ARGUMENT, "mr_stripefilter: null pointer");
    if (nsino == 0) return MR_OK;
    return run_stripes(sino_d, false, nu, nsino, ntheta, wname, decnum, sigma, stream);
}

mr_status mr_waveletringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, const char *wname, int decnum,
                              float sigma, void *stream)
{
    MR_TRACE();
    if (!proj_d) return fail(MR_ERR_ARGUMENT, "mr_waveletringclean: null pointer");
    if (nv == 0) return MR_OK;
    return run_stripes(proj_d, true, nu, nv, nproj, wname, decnum, sigma, stream);
}

} // extern "C"
