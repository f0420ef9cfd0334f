// In-place radix-2 complex FFT stages in shared memory, shared by the row filters
// (mr_rowfilter.cu) and the stripe filter (mr_ringclean.cu). One CTA transforms one
// complex sequence of length n = 2^logn; twiddles are exp(-2 pi i k / n), k < n/2.
#pragma once

#include <cuda_runtime.h>

namespace mr {

__device__ __forceinline__ unsigned fft_bitrev(unsigned x, int logn) { return __brev(x) >> (32 - logn); }

// Decimation in time: bit-reversed input -> natural-order spectrum (forward transform).
__device__ __forceinline__ void fft_forward_dit(float2 *buf, int n, int logn, const float2 *__restrict__ twiddle)
{
    const int nh = n >> 1;
    for (int s = 1; s <= logn; ++s) {
        const int half = 1 << (s - 1);
        const int tstride = n >> s;
        for (int b = threadIdx.x; b < nh; b += blockDim.x) {
            const int j = b & (half - 1);
            const int i0 = ((b >> (s - 1)) << s) + j;
            const int i1 = i0 + half;
            const float2 w = __ldg(twiddle + j * tstride);
            const float2 x = buf[i0];
            const float2 y = buf[i1];
            const float2 t = make_float2(y.x * w.x - y.y * w.y, y.x * w.y + y.y * w.x);
            buf[i0] = make_float2(x.x + t.x, x.y + t.y);
            buf[i1] = make_float2(x.x - t.x, x.y - t.y);
        }
        __syncthreads();
    }
}

// Decimation in frequency with conjugate twiddles: natural-order spectrum -> bit-reversed,
// unnormalised inverse transform.
__device__ __forceinline__ void fft_inverse_dif(float2 *buf, int n, int logn, const float2 *__restrict__ twiddle)
{
    const int nh = n >> 1;
    for (int s = logn; s >= 1; --s) {
        const int half = 1 << (s - 1);
        const int tstride = n >> s;
        for (int b = threadIdx.x; b < nh; b += blockDim.x) {
            const int j = b & (half - 1);
            const int i0 = ((b >> (s - 1)) << s) + j;
            const int i1 = i0 + half;
            const float2 w = __ldg(twiddle + j * tstride);
            const float2 x = buf[i0];
            const float2 y = buf[i1];
            buf[i0] = make_float2(x.x + y.x, x.y + y.y);
            const float2 d = make_float2(x.x - y.x, x.y - y.y);
            buf[i1] = make_float2(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);
        }
        __syncthreads();
    }
}

// Multiply by a real frequency response h[k], k < n.
__device__ __forceinline__ void fft_apply_response(float2 *buf, int n, const float *__restrict__ h)
{
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float r = __ldg(h + k);
        const float2 v = buf[k];
        buf[k] = make_float2(v.x * r, v.y * r);
    }
    __syncthreads();
}

} // namespace mr
