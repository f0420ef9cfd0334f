// In-place mixed-radix complex FFT in shared memory, shared by the row filters
// (mr_rowfilter.cu) and the stripe filter (mr_ringclean.cu). One CTA transforms one complex
// sequence of length n = 2^logn (two real rows packed as re/im).
//
// Forward: decimation in frequency, radix-8 stages from the full length down, the last stage
// radix 4 or 2 when logn is not a multiple of 3. Each stage reads the R inputs of a
// butterfly from shared memory into registers, takes their R-point DFT, multiplies output m
// by W_N^(j m) (N the stage's sub-length) and writes the outputs back to the input
// positions: natural order in, digit-reversed spectrum out. The inverse undoes the stages in
// reverse order (conjugate twiddle, inverse R-point DFT), so it takes the digit-reversed
// spectrum and returns the natural-order, unnormalised inverse transform. A real frequency
// response is applied at the digit-reversed positions (fft_permute_response on the host).
// Twiddles: exp(-2 pi i k / n), k < n (fft_twiddles on the host).
//
// Element e of a sequence sits at fft_slot(e) = e + e/16 of the shared buffer (one float2 of
// padding after every 16): the strided stages would otherwise put up to 16 lanes of a warp on
// one bank (8x the minimum wavefronts in the last radix-8 stage of n = 4096); with the padding
// every stage of n = 2^9 .. 2^13 runs at the minimum of two wavefronts per warp access.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

namespace mr {

constexpr int kFftMaxStages = 16;

__host__ __device__ __forceinline__ int fft_slot(int e) { return e + (e >> 4); }

// float2 slots of the shared buffer of an n-point transform
__host__ __device__ __forceinline__ int fft_buffer_slots(int n) { return n + n / 16; }

// radix (as log2) of each stage, from the full length down
__host__ __device__ __forceinline__ int fft_stages(int logn, int *rl)
{
    int ns = 0;
    for (int rem = logn; rem > 0; rem -= rl[ns - 1]) rl[ns++] = rem >= 3 ? 3 : rem;
    return ns;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); } // a * conj(b)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); } // a * (-i)
__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }

// Forward R-point DFT in registers (x -> X, X[m] = sum_q x[q] W_R^(q m)).
template <int R>
__device__ __forceinline__ void dft_small(float2 (&x)[R])
{
    if constexpr (R == 2) {
        const float2 a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const float2 e0 = cadd(x[0], x[2]), e1 = csub(x[0], x[2]);
        const float2 f0 = cadd(x[1], x[3]), f1 = mul_mi(csub(x[1], x[3]));
        x[0] = cadd(e0, f0);
        x[2] = csub(e0, f0);
        x[1] = cadd(e1, f1);
        x[3] = csub(e1, f1);
    } else {
        constexpr float r = 0.70710678118654752440f;
        float2 a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[k] = cadd(x[k], x[k + 4]);
            b[k] = csub(x[k], x[k + 4]);
        }
        // b[k] *= W8^k
        b[1] = make_float2(r * (b[1].x + b[1].y), r * (b[1].y - b[1].x));
        b[2] = mul_mi(b[2]);
        b[3] = make_float2(r * (b[3].y - b[3].x), -r * (b[3].x + b[3].y));
        dft_small<4>(a);
        dft_small<4>(b);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x[2 * k] = a[k];
            x[2 * k + 1] = b[k];
        }
    }
}

// One forward (DIF) stage of radix 2^RL on sub-transforms of length 2^nsl.
template <int RL>
__device__ __forceinline__ void fft_dif_stage(float2 *buf, int logn, int nsl, const float2 *__restrict__ tw)
{
    constexpr int R = 1 << RL;
    const int qsl = nsl - RL;               // log2 of the input stride N/R
    const int nb = 1 << (logn - RL);        // butterflies
    const int tws = logn - nsl;             // W_N^e = tw[e << tws]
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int j = b & ((1 << qsl) - 1);
        const int base = ((b >> qsl) << nsl) + j;
        float2 x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = buf[fft_slot(base + (q << qsl))];
        dft_small<R>(x);
        buf[fft_slot(base)] = x[0];
#pragma unroll
        for (int m = 1; m < R; ++m) buf[fft_slot(base + (m << qsl))] = cmul(x[m], __ldg(tw + ((j * m) << tws)));
    }
}

// The inverse of fft_dif_stage (times R): conjugate twiddle, inverse R-point DFT.
template <int RL>
__device__ __forceinline__ void fft_inv_stage(float2 *buf, int logn, int nsl, const float2 *__restrict__ tw)
{
    constexpr int R = 1 << RL;
    const int qsl = nsl - RL;
    const int nb = 1 << (logn - RL);
    const int tws = logn - nsl;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int j = b & ((1 << qsl) - 1);
        const int base = ((b >> qsl) << nsl) + j;
        float2 x[R];
        x[0] = conj2(buf[fft_slot(base)]);
#pragma unroll
        for (int m = 1; m < R; ++m) x[m] = conj2(cmulc(buf[fft_slot(base + (m << qsl))], __ldg(tw + ((j * m) << tws))));
        dft_small<R>(x); // inverse DFT = conj(DFT(conj(.)))
#pragma unroll
        for (int q = 0; q < R; ++q) buf[fft_slot(base + (q << qsl))] = conj2(x[q]);
    }
}

// Forward transform: natural order -> digit-reversed spectrum (buffer slots fft_slot(e)).
__device__ __forceinline__ void fft_forward(float2 *buf, int logn, const float2 *__restrict__ tw)
{
    int rl[kFftMaxStages];
    const int ns = fft_stages(logn, rl);
    int nsl = logn;
    for (int s = 0; s < ns; ++s) {
        if (rl[s] == 3) fft_dif_stage<3>(buf, logn, nsl, tw);
        else if (rl[s] == 2) fft_dif_stage<2>(buf, logn, nsl, tw);
        else fft_dif_stage<1>(buf, logn, nsl, tw);
        nsl -= rl[s];
        __syncthreads();
    }
}

// Unnormalised inverse transform: digit-reversed spectrum -> natural order.
__device__ __forceinline__ void fft_inverse(float2 *buf, int logn, const float2 *__restrict__ tw)
{
    int rl[kFftMaxStages];
    const int ns = fft_stages(logn, rl);
    int nsl = 0;
    for (int s = ns - 1; s >= 0; --s) {
        nsl += rl[s];
        if (rl[s] == 3) fft_inv_stage<3>(buf, logn, nsl, tw);
        else if (rl[s] == 2) fft_inv_stage<2>(buf, logn, nsl, tw);
        else fft_inv_stage<1>(buf, logn, nsl, tw);
        __syncthreads();
    }
}

// Multiply by a real frequency response given at the digit-reversed positions, p < n.
__device__ __forceinline__ void fft_apply_response(float2 *buf, int n, const float *__restrict__ h)
{
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float r = __ldg(h + k);
        const float2 v = buf[fft_slot(k)];
        buf[fft_slot(k)] = make_float2(v.x * r, v.y * r);
    }
    __syncthreads();
}

// ---- host side

// exp(-2 pi i k / n), k < n, in double then rounded
inline std::vector<float2> fft_twiddles(int n)
{
    std::vector<float2> t(n);
    for (int k = 0; k < n; ++k) {
        const double ang = -2.0 * 3.14159265358979323846264338327950288 * static_cast<double>(k) / n;
        t[k] = make_float2(static_cast<float>(std::cos(ang)), static_cast<float>(std::sin(ang)));
    }
    return t;
}

// Frequency held at position p of the forward transform's output.
inline int fft_frequency_at(int p, int logn)
{
    int rl[kFftMaxStages];
    const int ns = fft_stages(logn, rl);
    int k = 0, mult = 1, nsl = logn;
    for (int s = 0; s < ns; ++s) {
        const int qsl = nsl - rl[s];
        const int m = (p >> qsl) & ((1 << rl[s]) - 1); // output m of this stage
        k += m * mult;
        mult <<= rl[s];
        p &= (1 << qsl) - 1;
        nsl = qsl;
    }
    return k;
}

// resp (natural frequency order, n values) -> the order of the forward transform's output
inline std::vector<float> fft_permute_response(const std::vector<float> &resp, int logn)
{
    const int n = 1 << logn;
    std::vector<float> out(n);
    for (int p = 0; p < n; ++p) out[p] = resp[fft_frequency_at(p, logn)];
    return out;
}

} // namespace mr

// In-place radix-2 DFT in double of a power-of-two length (re, im), sign -1 forward, +1
// inverse (unnormalised); for the filter responses on the host.
inline void host_dft(std::vector<double> &re, std::vector<double> &im, int sign)
{
    const size_t n = re.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2;
        for (size_t k = 0; k < half; ++k) {
            const double a = sign * 2.0 * M_PI * static_cast<double>(k) / static_cast<double>(len);
            const double wr = std::cos(a), wi = std::sin(a);
            for (size_t i = k; i < n; i += len) {
                const double xr = re[i + half] * wr - im[i + half] * wi, xi = re[i + half] * wi + im[i + half] * wr;
                re[i + half] = re[i] - xr;
                im[i + half] = im[i] - xi;
                re[i] += xr;
                im[i] += xi;
            }
        }
    }
}
