// kipl filters with EdgeMirror edges, shared by SpotClean2 and the weighted reference average.
//
// kipl::filters::TFilterBase<float,2> (core/kipl/kipl/include/filters/core/filterbase.hpp:
// 83-408) computes the interior directly and each edge band from a padded buffer: outputs in
// the top and bottom ky/2 rows read a buffer mirrored vertically about the edge row (no
// repeat) and padded horizontally with the edge value; outputs in the left and right kx/2
// columns of the other rows read a buffer mirrored horizontally. Every output sums (TFilter,
// from 0), or takes min / max of (TErode from FLT_MAX, TDilate from -FLT_MAX), its nonzero taps
// in row-major order.
#pragma once

#include "mr_common.cuh"

namespace mr {
namespace kf {

constexpr float kFloatMax = 3.402823466e+38f; // std::numeric_limits<float>::max()

// Source value for output (x, y) at (xx, yy) for a kx x ky kernel.
template <int KX, int KY>
__device__ __forceinline__ float mirror_at(const float *img, int w, int h, int x, int y, int xx, int yy)
{
    constexpr int cx = KX / 2, cy = KY / 2;
    if (y < cy || y >= h - cy) {
        yy = yy < 0 ? -yy : (yy >= h ? 2 * (h - 1) - yy : yy);
        xx = min(max(xx, 0), w - 1);
    } else if (x < cx || x >= w - cx) {
        xx = xx < 0 ? -xx : (xx >= w ? 2 * (w - 1) - xx : xx);
    }
    return __ldg(img + static_cast<size_t>(yy) * w + xx);
}

enum { OP_SUM = 0, OP_MIN = 1, OP_MAX = 2 };

// A line of L ones along x or y, one image per grid z: the sum of the box filters
// (StdDevFilter::BoxFilter, SpotClean::BoxFilter), std::min(dest, src) from FLT_MAX (TErode),
// std::max(dest, src) from -FLT_MAX (TDilate).
template <int L, bool ALONG_Y, int OP>
__global__ void __launch_bounds__(256) k_line(const float *__restrict__ src, int w, int h, float *__restrict__ dst)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t npix = static_cast<size_t>(w) * h;
    const float *img = src + blockIdx.z * npix;
    float acc = OP == OP_SUM ? 0.0f : (OP == OP_MIN ? kFloatMax : -kFloatMax);
#pragma unroll
    for (int t = 0; t < L; ++t) {
        const int d = t - L / 2;
        const float v = ALONG_Y ? mirror_at<1, L>(img, w, h, x, y, x, y + d) : mirror_at<L, 1>(img, w, h, x, y, x + d, y);
        if (OP == OP_SUM) acc = __fadd_rn(acc, v);
        else if (OP == OP_MIN) acc = v < acc ? v : acc;
        else acc = acc < v ? v : acc;
    }
    dst[blockIdx.z * npix + static_cast<size_t>(y) * w + x] = acc;
}

template <int L, bool ALONG_Y, int OP>
inline void line(const float *src, int w, int h, unsigned nimg, float *dst, cudaStream_t s)
{
    k_line<L, ALONG_Y, OP><<<dim3(div_up(w, 32), div_up(h, 8), nimg), dim3(32, 8), 0, s>>>(src, w, h, dst);
}

// Box sum over dim (3, 5 or 7) along x, then along y.
inline void box(const float *src, int w, int h, unsigned nimg, int dim, float *tmp, float *dst, cudaStream_t s)
{
    if (dim == 3) {
        line<3, false, OP_SUM>(src, w, h, nimg, tmp, s);
        line<3, true, OP_SUM>(tmp, w, h, nimg, dst, s);
    } else if (dim == 5) {
        line<5, false, OP_SUM>(src, w, h, nimg, tmp, s);
        line<5, true, OP_SUM>(tmp, w, h, nimg, dst, s);
    } else {
        line<7, false, OP_SUM>(src, w, h, nimg, tmp, s);
        line<7, true, OP_SUM>(tmp, w, h, nimg, dst, s);
    }
}

// x * x (kipl::math::sqr). Internal linkage: every translation unit that includes this
// header gets its own copy.
static __global__ void __launch_bounds__(256) k_square(const float *__restrict__ a, size_t n, float *__restrict__ out)
{
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = __fmul_rn(a[i], a[i]);
}

// sqrt(M1 * (s2 - M * m * m)) with M = 1/(dim*dim), M1 = 1/(dim*dim - 1) in float
// (kipl::filters::StdDevFilter::operator(), core/kipl/kipl/src/filters/stddevfilter.cpp:25-44;
// SpotClean::StdDevDetection, SpotClean.cpp:521-545).
template <int DIM>
__global__ void __launch_bounds__(256) k_stddev(const float *__restrict__ s2, const float *__restrict__ m, size_t n,
                                                float *__restrict__ out)
{
    constexpr float M = 1.0f / static_cast<float>(DIM * DIM), M1 = 1.0f / static_cast<float>(DIM * DIM - 1);
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float v = m[i];
        out[i] = __fsqrt_rn(__fmul_rn(M1, __fsub_rn(s2[i], __fmul_rn(__fmul_rn(M, v), v))));
    }
}

inline unsigned flat_blocks(size_t n) { return static_cast<unsigned>(std::min<size_t>(div_up(n, 256), 148 * 16)); }

// Standard deviation filter of dim x dim with EdgeMirror edges on nimg images: sq, tmp scratch
// images of the batch; out receives the result (may not alias img).
template <int DIM>
inline void stddev_filter(const float *img, int w, int h, unsigned nimg, float *sq, float *tmp, float *s2,
                          float *out, cudaStream_t s)
{
    const size_t n = static_cast<size_t>(w) * h * nimg;
    k_square<<<flat_blocks(n), 256, 0, s>>>(img, n, sq);
    box(sq, w, h, nimg, DIM, tmp, s2, s);
    box(img, w, h, nimg, DIM, tmp, sq, s);
    k_stddev<DIM><<<flat_blocks(n), 256, 0, s>>>(s2, sq, n, out);
}

} // namespace kf
} // namespace mr
