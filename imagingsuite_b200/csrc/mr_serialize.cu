// Slice serialisation to 16 bits on the GPU.
//
// Reference: ReconEngine::Serialize (frameworks/tomography/Framework/ReconFramework/src/
// ReconEngine.cpp:576-700) writes the reconstructed block with kipl::io::WriteImageStack
// (core/kipl/kipl/include/io/io_stack.h:114-230): each slice is cut out with ExtractSlice
// (core/kipl/kipl/include/base/core/textractor.hpp:17-125; plane XY for MatrixXYZ volumes,
// plane YZ for the z-fastest MatrixZXY volumes of the parallel-beam backprojectors, with an
// optional inclusive ROI) and stored as TIFF16 by WriteTIFF(src, fname, lo, hi)
// (io/io_tiff.h:181-200), which casts with ImageCaster<unsigned short, float>::cast
// (base/core/imagecast.hpp:33-52):
//   scale = float(65535) / (hi - lo)      (float)
//   out   = unsigned short((min(max(v, lo), hi) - lo) * scale)   (truncation)
// with std::max / std::min semantics (a NaN passes both and becomes 0). Here the cast runs on
// the device and only the uint16 slices leave it (half the bytes of the float volume); the
// file writing stays with the caller.
#include "mr_common.cuh"

#include <algorithm>

namespace mr {
namespace ser {

__device__ __forceinline__ uint16_t to_u16(float v, float lo, float hi, float scale)
{
    const float m = v < lo ? lo : v;  // std::max(v, lo)
    const float c = hi < m ? hi : m;  // std::min(m, hi)
    const float val = __fmul_rn(__fsub_rn(c, lo), scale);
    return static_cast<uint16_t>(min(__float2uint_rz(val), 65535u)); // NaN -> 0
}

// Plane XY of a volume with dims (d0, d1, d2), d0 fastest: slice s = vol[first + s], rows
// b0 .. b0 + h - 1, columns a0 .. a0 + w - 1. Blocks loop over the count * h output rows; a
// row is converted four values per thread (16-byte loads, 8-byte stores) when its source and
// destination starts are 4-aligned (VEC), else one value per thread.
template <bool VEC>
__global__ void __launch_bounds__(256) k_slices_xy(const float *__restrict__ vol, int d0, int d1, int first, int count,
                                                   int a0, int b0, int w, int h, float lo, float hi, float scale,
                                                   uint16_t *__restrict__ out)
{
    const size_t rows = static_cast<size_t>(count) * h;
    for (size_t r = blockIdx.x; r < rows; r += gridDim.x) {
        const int s = static_cast<int>(r / h), b = static_cast<int>(r % h);
        const float *src = vol + (static_cast<size_t>(first + s) * d1 + (b0 + b)) * d0 + a0;
        uint16_t *dst = out + r * w;
        if constexpr (VEC) {
            for (int a = 4 * threadIdx.x; a < w; a += 4 * blockDim.x) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(src + a));
                ushort4 o;
                o.x = to_u16(v.x, lo, hi, scale);
                o.y = to_u16(v.y, lo, hi, scale);
                o.z = to_u16(v.z, lo, hi, scale);
                o.w = to_u16(v.w, lo, hi, scale);
                *reinterpret_cast<ushort4 *>(dst + a) = o;
            }
        } else {
            for (int a = threadIdx.x; a < w; a += blockDim.x) dst[a] = to_u16(__ldg(src + a), lo, hi, scale);
        }
    }
}

// Plane YZ of a volume with dims (d0, d1, d2) = (z, x, y), z fastest: out[s][b][a] =
// vol[b0 + b][a0 + a][first + s]. A block transposes a 32 (a) x 32 (s) tile of one row b
// through shared memory so that both the z-fastest reads and the a-fastest writes coalesce.
__global__ void __launch_bounds__(256) k_slices_yz(const float *__restrict__ vol, int d0, int d1, int first,
                                                   int count, int a0, int b0, int w, int h, float lo, float hi,
                                                   float scale, uint16_t *__restrict__ out)
{
    __shared__ uint16_t tile[32][33];
    const int ta = blockIdx.x * 32, ts = blockIdx.y * 32, b = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y; // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int a = ta + r, s = ts + tx;
        if (a < w && s < count) {
            const size_t src = (static_cast<size_t>(b0 + b) * d1 + (a0 + a)) * d0 + (first + s);
            tile[tx][r] = to_u16(vol[src], lo, hi, scale);
        }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int s = ts + r, a = ta + tx;
        if (a < w && s < count) out[(static_cast<size_t>(s) * h + b) * w + a] = tile[r][tx];
    }
}

} // namespace ser
} // namespace mr

using namespace mr;

extern "C" mr_status mr_slices_u16(const float *vol_d, int plane, size_t d0, size_t d1, size_t d2, size_t first,
                                   size_t count, const size_t *roi_h, float lo, float hi, uint16_t *out_d,
                                   void *stream)
{
    MR_TRACE();
    if (!vol_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_slices_u16: null pointer");
    if (plane != MR_PLANE_XY && plane != MR_PLANE_YZ) return fail(MR_ERR_ARGUMENT, "mr_slices_u16: plane");
    if (d0 == 0 || d1 == 0 || d2 == 0 || d0 > 65535 || d1 > 65535 || d2 > 65535)
        return fail(MR_ERR_ARGUMENT, "mr_slices_u16: unsupported size");
    if (!(lo < hi)) return fail(MR_ERR_ARGUMENT, "mr_slices_u16: the gray interval needs lo < hi");
    // slice axis and the two in-slice axes (fast a, slow b)
    const size_t nslices = plane == MR_PLANE_XY ? d2 : d0;
    const size_t na = plane == MR_PLANE_XY ? d0 : d1, nb = plane == MR_PLANE_XY ? d1 : d2;
    if (first > nslices || count > nslices - first)
        return fail(MR_ERR_ARGUMENT, "mr_slices_u16: slice range outside the volume");
    size_t a0 = 0, b0 = 0, w = na, h = nb;
    if (roi_h) {
        // ExtractSlice: inclusive bounds, swapped when given in reverse order
        const size_t x0 = std::min(roi_h[0], roi_h[2]), x1 = std::max(roi_h[0], roi_h[2]);
        const size_t y0 = std::min(roi_h[1], roi_h[3]), y1 = std::max(roi_h[1], roi_h[3]);
        if (x1 >= na || y1 >= nb) return fail(MR_ERR_ARGUMENT, "mr_slices_u16: roi outside the slice");
        a0 = x0;
        b0 = y0;
        w = x1 - x0 + 1;
        h = y1 - y0 + 1;
    }
    if (count == 0) return MR_OK;
    const float scale = 65535.0f / (hi - lo); // float, as the reference's ImageCaster
    cudaStream_t s = as_stream(stream);
    const int ia0 = static_cast<int>(a0), ib0 = static_cast<int>(b0), iw = static_cast<int>(w), ih = static_cast<int>(h);
    if (plane == MR_PLANE_XY) {
        const unsigned blocks = static_cast<unsigned>(std::min<size_t>(count * h, 148 * 8));
        const bool vec = d0 % 4 == 0 && a0 % 4 == 0 && w % 4 == 0 &&
                         reinterpret_cast<uintptr_t>(vol_d) % 16 == 0 && reinterpret_cast<uintptr_t>(out_d) % 8 == 0;
        if (vec)
            ser::k_slices_xy<true><<<blocks, 256, 0, s>>>(vol_d, static_cast<int>(d0), static_cast<int>(d1),
                                                          static_cast<int>(first), static_cast<int>(count), ia0, ib0,
                                                          iw, ih, lo, hi, scale, out_d);
        else
            ser::k_slices_xy<false><<<blocks, 256, 0, s>>>(vol_d, static_cast<int>(d0), static_cast<int>(d1),
                                                           static_cast<int>(first), static_cast<int>(count), ia0, ib0,
                                                           iw, ih, lo, hi, scale, out_d);
        return check_launch("k_slices_xy");
    }
    dim3 grid(div_up(w, 32), div_up(count, 32), static_cast<unsigned>(h));
    ser::k_slices_yz<<<grid, dim3(32, 8), 0, s>>>(vol_d, static_cast<int>(d0), static_cast<int>(d1),
                                                  static_cast<int>(first), static_cast<int>(count), ia0, ib0, iw, ih,
                                                  lo, hi, scale, out_d);
    return check_launch("k_slices_yz");
}
