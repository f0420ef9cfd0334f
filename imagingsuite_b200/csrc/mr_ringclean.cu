// Wavelet-FFT ring cleaning: StripeFilter and WaveletRingClean on the GPU.
//
// Reference: core/algorithms/ImagingAlgorithms/src/StripeFilter.cpp:68-250 (Münch-style
// vertical-stripe suppression), the separable DWT/IDWT of core/kipl/kipl/include/wavelets/
// core/wavelets.hpp:452-862 and WaveletRingClean::ProcessSingle (frameworks/tomography/
// Preprocessing/StdPreprocModules/src/WaveletRingClean.cpp:74-103).
//
// A batch of sinograms [B][ntheta][nu] goes through:
//   analysis levels  rows (k_dwt_rows: both filters per output) then columns (k_dwt_cols:
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

#include <cmath>
#include <string>
#include <vector>

namespace mr {
namespace rc {

constexpr int kMaxTaps = 60;
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

__global__ void k_gather(const float *__restrict__ proj, int nu, int nv, int nproj, int j0, int nb,
                         float *__restrict__ s)
{
    const size_t total = static_cast<size_t>(nb) * nproj * nu;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int u = static_cast<int>(i % nu);
        const size_t r = i / nu;
        const int th = static_cast<int>(r % nproj), b = static_cast<int>(r / nproj);
        s[i] = proj[(static_cast<size_t>(th) * nv + j0 + b) * nu + u];
    }
}

__global__ void k_scatter(const float *__restrict__ s, int nu, int nv, int nproj, int j0, int nb,
                          float *__restrict__ proj)
{
    const size_t total = static_cast<size_t>(nb) * nproj * nu;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int u = static_cast<int>(i % nu);
        const size_t r = i / nu;
        const int th = static_cast<int>(r % nproj), b = static_cast<int>(r / nproj);
        proj[(static_cast<size_t>(th) * nv + j0 + b) * nu + u] = s[i];
    }
}

// FilterVerticalStripes (StripeFilter.cpp:114-135): every column of the vertical band
// [B][bh][bw] zero-padded to n, filtered with the even real response, first bh samples kept.
__global__ void k_stripe_fft(float *__restrict__ band, int bw, int bh, int ncols, int n, int logn,
                             const float2 *__restrict__ twiddle, const float *__restrict__ response)
{
    extern __shared__ float2 buf[];
    const int c0 = 2 * blockIdx.x, c1 = c0 + 1;
    const bool has1 = c1 < ncols;
    const size_t base0 = static_cast<size_t>(c0 / bw) * bw * bh + c0 % bw;
    const size_t base1 = has1 ? static_cast<size_t>(c1 / bw) * bw * bh + c1 % bw : 0;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        float x0 = 0.0f, x1 = 0.0f;
        if (p < bh) {
            x0 = band[base0 + static_cast<size_t>(p) * bw];
            if (has1) x1 = band[base1 + static_cast<size_t>(p) * bw];
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
        if (has1) band[base1 + static_cast<size_t>(p) * bw] = v.y;
    }
}

// ---- the four convolution passes: analysis rows (both filters per output) and columns (the
// four sub-bands, wavelets.hpp:474-487); synthesis rows and columns of upsconvRC
// (:750-858) summed as ((a + h) + v) + d (WaveletTransform::synthesize :626-645). Every output
// is the sum over the taps in the reference's order; indices are 32-bit from the grid, the
// taps sit in shared memory, and away from the borders (where the mirrored index is the
// identity) the window is read directly. In the synthesis passes the interior skips the taps that meet
// the zeros inserted by the dyadic upsampling (adding a product with 0 leaves a nonzero sum
// unchanged, so only the sign of an exactly zero result can differ).
constexpr int kConvThreads = 128;

__device__ __forceinline__ void load_taps(const float *__restrict__ taps, int n, float *sm)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) sm[i] = taps[i];
    __syncthreads();
}

__global__ void __launch_bounds__(kConvThreads) k_dwt_rows2(const float *__restrict__ src, int sx, int nrows,
                                                            const float *__restrict__ taps, int K, int dx,
                                                            float *__restrict__ tmpH, float *__restrict__ tmpG)
{
    __shared__ float tp[2 * kMaxTaps];
    load_taps(taps, 2 * K, tp);
    const float *tH = tp, *tG = tp + K;
    const int k = blockIdx.x * kConvThreads + threadIdx.x;
    if (k >= dx) return;
    const bool inner = 2 * k - K + 2 >= 0 && 2 * k + 1 < sx;
    for (int row = blockIdx.y; row < nrows; row += gridDim.y) {
        const float *r = src + static_cast<size_t>(row) * sx;
        float aH = 0.0f, aG = 0.0f;
        if (inner) {
            const float *w = r + 2 * k + 1; // x_j = w[-j]
            for (int j = 0; j < K; ++j) {
                const float x = w[-j];
                aH = __fadd_rn(aH, __fmul_rn(tH[j], x));
                aG = __fadd_rn(aG, __fmul_rn(tG[j], x));
            }
        } else {
            for (int j = 0; j < K; ++j) {
                const float x = r[mirror_index(sx, K, K + 2 * k - j + 1)];
                aH = __fadd_rn(aH, __fmul_rn(tH[j], x));
                aG = __fadd_rn(aG, __fmul_rn(tG[j], x));
            }
        }
        tmpH[static_cast<size_t>(row) * dx + k] = aH;
        tmpG[static_cast<size_t>(row) * dx + k] = aG;
    }
}

// out[q][row][k], q = blockIdx.z (a, h, v, d), rows over all batch images.
__global__ void __launch_bounds__(kConvThreads) k_up_rows2(const float *__restrict__ a, const float *__restrict__ hb,
                                                           const float *__restrict__ vb, const float *__restrict__ db,
                                                           int w, int nrows, const float *__restrict__ taps, int K,
                                                           int dx, float *__restrict__ out)
{
    __shared__ float tp[2 * kMaxTaps];
    load_taps(taps + 2 * K, 2 * K, tp);
    const int q = blockIdx.z;
    const float *kh = q < 2 ? tp : tp + K;
    const float *band = q == 0 ? a : q == 1 ? hb : q == 2 ? vb : db;
    const int k = blockIdx.x * kConvThreads + threadIdx.x;
    if (k >= dx) return;
    const int c = K - 2;
    const bool inner = k >= 1 && k < 2 * w - K + 2;
    const size_t plane = static_cast<size_t>(nrows) * dx;
    for (int row = blockIdx.y; row < nrows; row += gridDim.y) {
        const float *src = band + static_cast<size_t>(row) * w;
        float acc = 0.0f;
        if (inner) {
            // t = k + c - m; even t only: m of the parity of k + c
            for (int m = (k + c) & 1; m < K; m += 2) acc = __fadd_rn(acc, __fmul_rn(src[(k + c - m) >> 1], kh[m]));
        } else {
            for (int m = 0; m < K; ++m) {
                const int t = up_index(w, K, K + k + c - m);
                const float xv = (t & 1) ? 0.0f : src[t >> 1];
                acc = __fadd_rn(acc, __fmul_rn(xv, kh[m]));
            }
        }
        out[q * plane + static_cast<size_t>(row) * dx + k] = acc;
    }
}

// Column passes with kColBlock consecutive outputs per thread. The outputs of a block share
// most of their input rows, so the thread walks the rows it needs once, from the last to
// the first, and adds each row into every output whose tap m = (output position) - (row
// position) falls in [0, K): per output the rows arrive in descending order, i.e. the taps
// in the reference's ascending order, so every sum equals the one-output-per-thread form
// bit for bit. Blocks that reach a border (mirrored or upsampled-zero indices) use the
// per-output form.
constexpr int kColBlock = 8;

__global__ void __launch_bounds__(kConvThreads) k_dwt_cols3(const float *__restrict__ tmpH,
                                                            const float *__restrict__ tmpG, int dx, int sy,
                                                            const float *__restrict__ taps, int K, int dy,
                                                            float *__restrict__ a, float *__restrict__ h,
                                                            float *__restrict__ v, float *__restrict__ d)
{
    __shared__ float tp[2 * kMaxTaps];
    load_taps(taps, 2 * K, tp);
    const float *tH = tp, *tG = tp + K;
    const int x = blockIdx.x * kConvThreads + threadIdx.x, k0 = blockIdx.y * kColBlock, b = blockIdx.z;
    if (x >= dx) return;
    const size_t base = static_cast<size_t>(b) * sy * dx + x;
    const int k1 = min(k0 + kColBlock, dy); // outputs k0 .. k1-1
    const bool inner = 2 * k0 - K + 2 >= 0 && 2 * (k1 - 1) + 1 < sy;
    if (inner && k1 - k0 == kColBlock) {
        float sa[kColBlock], sh[kColBlock], sv[kColBlock], sd[kColBlock];
#pragma unroll
        for (int r = 0; r < kColBlock; ++r) sa[r] = sh[r] = sv[r] = sd[r] = 0.0f;
        // output k uses rows 2k + 1 - m, m = 0 .. K-1
        for (int i = 2 * (k0 + kColBlock - 1) + 1; i >= 2 * k0 + 2 - K; --i) {
            const size_t idx = base + static_cast<size_t>(i) * dx;
            const float ph = tmpH[idx], pg = tmpG[idx];
#pragma unroll
            for (int r = 0; r < kColBlock; ++r) {
                const int m = 2 * (k0 + r) + 1 - i;
                if (static_cast<unsigned>(m) < static_cast<unsigned>(K)) {
                    const float th = tH[m], tg = tG[m];
                    sa[r] = __fadd_rn(sa[r], __fmul_rn(th, ph));
                    sh[r] = __fadd_rn(sh[r], __fmul_rn(tg, ph));
                    sv[r] = __fadd_rn(sv[r], __fmul_rn(th, pg));
                    sd[r] = __fadd_rn(sd[r], __fmul_rn(tg, pg));
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kColBlock; ++r) {
            const size_t o = (static_cast<size_t>(b) * dy + k0 + r) * dx + x;
            a[o] = sa[r];
            h[o] = sh[r];
            v[o] = sv[r];
            d[o] = sd[r];
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
            sa = __fadd_rn(sa, __fmul_rn(tH[m], ph));
            sh = __fadd_rn(sh, __fmul_rn(tG[m], ph));
            sv = __fadd_rn(sv, __fmul_rn(tH[m], pg));
            sd = __fadd_rn(sd, __fmul_rn(tG[m], pg));
        }
        const size_t o = (static_cast<size_t>(b) * dy + k) * dx + x;
        a[o] = sa;
        h[o] = sh;
        v[o] = sv;
        d[o] = sd;
    }
}

__global__ void __launch_bounds__(kConvThreads) k_up_cols3(const float *__restrict__ rows, int dx, int h, int nb,
                                                           const float *__restrict__ taps, int K, int ox, int oy,
                                                           float *__restrict__ out)
{
    __shared__ float tp[2 * kMaxTaps];
    load_taps(taps + 2 * K, 2 * K, tp);
    const int x = blockIdx.x * kConvThreads + threadIdx.x, k0 = blockIdx.y * kColBlock, b = blockIdx.z;
    if (x >= ox) return;
    const size_t plane = static_cast<size_t>(nb) * h * dx;
    const size_t base = static_cast<size_t>(b) * h * dx + x;
    const int c = K - 2;
    const int k1 = min(k0 + kColBlock, oy);
    const bool inner = k0 >= 1 && k1 - 1 < 2 * h - K + 2;
    if (inner && k1 - k0 == kColBlock) {
        // output k uses rows (k + c - m) / 2 for the m of the parity of k + c
        float s4[4][kColBlock];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float *kv = (q == 0 || q == 2) ? tp : tp + K;
            const float *col = rows + q * plane + base;
#pragma unroll
            for (int r = 0; r < kColBlock; ++r) s4[q][r] = 0.0f;
            for (int i = (k0 + kColBlock - 1 + c) >> 1; 2 * i >= k0 + c - (K - 1); --i) {
                const float xv = col[static_cast<size_t>(i) * dx];
#pragma unroll
                for (int r = 0; r < kColBlock; ++r) {
                    const int m = k0 + r + c - 2 * i;
                    if (static_cast<unsigned>(m) < static_cast<unsigned>(K)) s4[q][r] = __fadd_rn(s4[q][r], __fmul_rn(xv, kv[m]));
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kColBlock; ++r)
            out[(static_cast<size_t>(b) * oy + k0 + r) * ox + x] =
                __fadd_rn(__fadd_rn(__fadd_rn(s4[0][r], s4[1][r]), s4[2][r]), s4[3][r]);
        return;
    }
    for (int k = k0; k < k1; ++k) {
        const bool in = k >= 1 && k < 2 * h - K + 2;
        float s4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float *kv = (q == 0 || q == 2) ? tp : tp + K;
            const float *col = rows + q * plane + base;
            float acc = 0.0f;
            if (in) {
                for (int m = (k + c) & 1; m < K; m += 2)
                    acc = __fadd_rn(acc, __fmul_rn(col[static_cast<size_t>((k + c - m) >> 1) * dx], kv[m]));
            } else {
                for (int m = 0; m < K; ++m) {
                    const int t = up_index(h, K, K + k + c - m);
                    const float xv = (t & 1) ? 0.0f : col[static_cast<size_t>(t >> 1) * dx];
                    acc = __fadd_rn(acc, __fmul_rn(xv, kv[m]));
                }
            }
            s4[q] = acc;
        }
        out[(static_cast<size_t>(b) * oy + k) * ox + x] = __fadd_rn(__fadd_rn(__fadd_rn(s4[0], s4[1]), s4[2]), s4[3]);
    }
}

struct Plan {
    int K = 0, begin = 0, end = 0, levels = 0;
    int sx[kMaxLevels + 1], sy[kMaxLevels + 1];
    int nfft[kMaxLevels];
    std::vector<float> taps;                 // tH | tG | sH | sG
    std::vector<std::vector<float>> resp;    // full-length responses per level
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
    // CreateFilterWindow (StripeFilter.cpp:68-81) and configure's FFT lengths (:222-235)
    const float s = -1.0f / (2.0f * sigma * sigma);
    P.resp.resize(decnum);
    for (int l = 0; l < decnum; ++l) {
        const size_t L = next_power2(static_cast<size_t>(1.25 * static_cast<int>(ntheta)) >> l);
        const size_t N = 2 * L;
        if (N > 16384) return fail(MR_ERR_UNSUPPORTED, "stripe filter FFT length %zu above 16384", N);
        if (static_cast<size_t>(P.sy[l + 1]) > N) return fail(MR_ERR_ARGUMENT, "band taller than its FFT length");
        P.nfft[l] = static_cast<int>(N);
        const float scale = 1.0f / (2.0f * L);
        std::vector<float> damp(N);
        for (size_t i = 0; i < N; ++i) {
            float w = static_cast<float>(i) * scale;
            damp[i] = (1.0f - std::exp(w * w * s)) * scale;
        }
        // the c2r reads bins 0..N/2: response damp[k] on 0..N/2, mirrored above
        P.resp[l].resize(N);
        for (size_t k = 0; k < N; ++k) P.resp[l][k] = damp[k <= N / 2 ? k : N - k];
        // in the order of the forward transform's output
        P.resp[l] = fft_permute_response(P.resp[l], ilog2i(static_cast<int>(N)));
    }
    return MR_OK;
}


// Stripe filter of nb contiguous sinograms s [nb][ntheta][nu], in place.
static mr_status stripe_batch(float *s_d, int nb, const rc::Plan &P, const float *taps_d,
                              const std::vector<float2 *> &tw_d, const std::vector<float *> &resp_d, float *scratch,
                              cudaStream_t st)
{
    using namespace rc;
    const int K = P.K, L = P.levels;
    // scratch layout: per level l=1..L: a, h, v, d [nb][sx][sy]; tmp H/G; up rows [4][nb][h][dx]
    size_t off = 0;
    float *A[kMaxLevels + 1], *Hb[kMaxLevels + 1], *Vb[kMaxLevels + 1], *Db[kMaxLevels + 1];
    A[0] = s_d;
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
        const int rows = nb * sy;
        k_dwt_rows2<<<dim3(div_up(dx, kConvThreads), std::min(rows, 65535)), kConvThreads, 0, st>>>(A[l], sx, rows,
                                                                                                  taps_d, K, dx, tH, tG);
        k_dwt_cols3<<<dim3(div_up(dx, kConvThreads), div_up(dy, kColBlock), nb), kConvThreads, 0, st>>>(
            tH, tG, dx, sy, taps_d, K, dy, A[l + 1], Hb[l + 1], Vb[l + 1], Db[l + 1]);
    }
    for (int l = 0; l < L; ++l) {
        const int bw = P.sx[l + 1], bh = P.sy[l + 1], n = P.nfft[l];
        const int ncols = nb * bw;
        k_stripe_fft<<<(ncols + 1) / 2, std::min(512, std::max(64, n / 8)), fft_buffer_slots(n) * sizeof(float2), st>>>(
            Vb[l + 1], bw, bh, ncols, n, ilog2i(n), tw_d[l], resp_d[l]);
    }
    for (int l = L - 1; l >= 0; --l) {
        const int w = P.sx[l + 1], h = P.sy[l + 1];
        const int dx = l == 0 ? 2 * P.sx[1] : P.sx[l], dy = l == 0 ? 2 * P.sy[1] : P.sy[l];
        const int rows = nb * h;
        k_up_rows2<<<dim3(div_up(dx, kConvThreads), std::min(rows, 65535), 4), kConvThreads, 0, st>>>(
            A[l + 1], Hb[l + 1], Vb[l + 1], Db[l + 1], w, rows, taps_d, K, dx, tmp);
        const int ox = l == 0 ? P.sx[0] : dx, oy = l == 0 ? P.sy[0] : dy;
        k_up_cols3<<<dim3(div_up(ox, kConvThreads), div_up(oy, kColBlock), nb), kConvThreads, 0, st>>>(
            tmp, dx, h, nb, taps_d, K, ox, oy, A[l]);
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

static mr_status run_stripes(float *data_d, bool interleaved, size_t nu, size_t nv_or_nsino, size_t ntheta,
                             const char *wname, int decnum, float sigma, void *stream)
{
    rc::Plan P;
    mr_status st = make_plan(nu, ntheta, wname, decnum, sigma, P);
    if (st != MR_OK) return st;
    cudaStream_t s = as_stream(stream);
    // batch size: about 1 GiB of scratch plus the gathered sinograms
    const size_t per = stripe_scratch(P, 1) + nu * ntheta;
    const size_t nsino = nv_or_nsino;
    const int nb = static_cast<int>(std::max<size_t>(1, std::min<size_t>(nsino, (size_t(1) << 28) / per)));
    float *taps_d = nullptr, *work = nullptr;
    std::vector<float2 *> tw_d(P.levels, nullptr);
    std::vector<float *> resp_d(P.levels, nullptr);
    size_t total = 4 * P.K;
    for (int l = 0; l < P.levels; ++l) total += P.nfft[l] * 2 + P.nfft[l];
    total += stripe_scratch(P, nb) + (interleaved ? static_cast<size_t>(nb) * nu * ntheta : 0);
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
    off += stripe_scratch(P, nb);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(rc::k_stripe_fft, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             fft_buffer_slots(16384) * sizeof(float2));
        attr = true;
    }
    float *gathered = interleaved ? work + off : nullptr;
    cudaError_t e = cudaMemcpyAsync(taps_d, P.taps.data(), P.taps.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    for (int l = 0; l < P.levels && e == cudaSuccess; ++l) {
        e = cudaMemcpyAsync(tw_d[l], tws[l].data(), tws[l].size() * sizeof(float2), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(resp_d[l], P.resp[l].data(), P.resp[l].size() * sizeof(float), cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "stripe filter tables: %s", cudaGetErrorString(e));
    for (size_t j0 = 0; j0 < nsino && st == MR_OK; j0 += nb) {
        const int b = static_cast<int>(std::min<size_t>(nb, nsino - j0));
        float *S;
        if (interleaved) {
            rc::k_gather<<<148 * 8, 256, 0, s>>>(data_d, static_cast<int>(nu), static_cast<int>(nsino),
                                                 static_cast<int>(ntheta), static_cast<int>(j0), b, gathered);
            S = gathered;
        } else {
            S = data_d + j0 * nu * ntheta;
        }
        st = stripe_batch(S, b, P, taps_d, tw_d, resp_d, scratch, s);
        if (st == MR_OK && interleaved)
            rc::k_scatter<<<148 * 8, 256, 0, s>>>(gathered, static_cast<int>(nu), static_cast<int>(nsino),
                                                  static_cast<int>(ntheta), static_cast<int>(j0), b, data_d);
        if (st == MR_OK) st = check_launch("ring clean scatter");
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
