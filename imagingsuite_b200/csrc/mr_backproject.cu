// Backprojectors: MultiProjectionBPparallel (parallel beam, linear interpolation) and
// FDKbp_single (cone beam, nearest neighbour), with the host-side geometry that the
// reference computes per projection.
//
// Exactness. The host geometry uses the same float expressions as the reference (compiled
// without contraction), and the kernels evaluate every per-voxel float operation of the
// reference in its order with explicitly rounded intrinsics, accumulating projections in
// the reference's order. With identical filtered projections the FP32 volumes are
// bit-identical to the reference modules'.
//
// Kernel layout. Lanes run along x (consecutive detector columns -> coalesced gathers);
// each thread keeps CZ slices of one (x, y) voxel column in registers across all
// projections and writes them once.
#include "mr_common.cuh"

#include <cmath>
#include <vector>

namespace mr {

MR_BOUNDS_TAKE(bounds_take_direct)

mr_status fdk_tma_launch(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv, size_t nproj,
                         const float *xip_d, const float *yip_d, const float *zip_d, const uint32_t *mask_d,
                         int accumulate, int kbegin, int kend, float *vol_d, int bw, int bh, cudaStream_t s);

static const float kFPi = 3.1415926535897932384626f;
static const double kDPi = 3.1415926535897932384626433832795028841971693993751;

template <int DT>
__device__ __forceinline__ float sample(const void *base, size_t idx)
{
    return Sample<DT>::load(static_cast<const typename Sample<DT>::T *>(base), idx);
}

// ------------------------------------------------------------------ parallel beam

// MultiProjectionBPparallel::BackProject (MultiProjBPparallel.cpp:39-170). x1, y1 are the
// reference's 1-based loop indices; the voxel is vol[y1-1][x1-1][z]; rows y1-1 in
// [ybegin, yend) are processed. `variant` selects the factory's other two parallel-beam
// backprojectors on the same loop structure:
//   1 MultiProjectionBP (MultiProjBP.cpp:36-146): identical without tilt; with tilt the centre
//     offset is subtracted after the x term and each 4-slice group g takes the weight
//     |(u - n) - g * tinc| (one shift per group, :81-84);
//   2 NearestNeighborBP (NNMultiProjBP.cpp:36-121): the sample at the truncated position only,
//     no weights, the centre offset (tilt) subtracted after the x term, no per-slice shift.
template <int DT, int CZ>
__global__ void __launch_bounds__(128) k_bp_parallel(const void *__restrict__ proj, const float *__restrict__ scale,
                                                     const float *__restrict__ weight, const int32_t *__restrict__ index,
                                                     const float *__restrict__ sinv,
                                                     const float *__restrict__ cosv, const float *__restrict__ startu,
                                                     int nproj, int nu, int nv, const uint32_t *__restrict__ mask,
                                                     int tilt, float toff, float tinc, int ybegin, int yend,
                                                     int variant, float *__restrict__ vol)
{
    const int x1 = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y1 = ybegin + blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int z0 = blockIdx.z * CZ;
    if (x1 > nu || y1 > yend) return;
    const uint32_t first = mask[2 * (y1 - 1)], second = mask[2 * (y1 - 1) + 1];
    if (static_cast<uint32_t>(x1) <= first || static_cast<uint32_t>(x1) > second) return;
    const int nz4 = (nv / 4) * 4;
    float *col = vol + (static_cast<size_t>(y1 - 1) * nu + (x1 - 1)) * nv;
    float acc[CZ];
#pragma unroll
    for (int c = 0; c < CZ; ++c) acc[c] = (z0 + c < nz4) ? col[z0 + c] : 0.0f;
    const float fx = static_cast<float>(x1), fy = static_cast<float>(y1);
    const int um2 = nu - 2;
    const size_t pstride = static_cast<size_t>(nu) * nv;

    for (int i = 0; i < nproj; ++i) {
        float local = __fadd_rn(startu[i], __fmul_rn(cosv[i], fy));
        if (tilt && variant == 0) local = __fsub_rn(local, toff);
        float posu = __fsub_rn(local, __fmul_rn(sinv[i], fx));
        if (tilt && variant != 0) posu = __fsub_rn(posu, toff);
        const int n = __float2int_rz(posu);
        if (n < 0 || um2 < n) continue;
        if (!MR_IN_BOUNDS(n + 1, nu, kSiteBpDirect)) continue;
        const int slab = index ? index[i] : i;
        float w = weight ? weight[i] : 1.0f;
        if (DT != MR_F32) w = scale[slab] * w;
        const size_t base = static_cast<size_t>(slab) * pstride + n;
        if (variant == 2) {
#pragma unroll
            for (int c = 0; c < CZ; ++c) {
                const int z = z0 + c;
                if (z < nz4) {
                    float pa = sample<DT>(proj, base + static_cast<size_t>(z) * nu);
                    if (weight || DT != MR_F32) pa = __fmul_rn(pa, w);
                    acc[c] = __fadd_rn(acc[c], pa);
                }
            }
        } else if (variant == 1) {
            // MultiProjBP.cpp:87-98 (tilt) and :128-143: column B is column A plus SizeV/4
            // vectors, i.e. 4*(nv/4) slices further in the transposed, 4-padded projection
            // buffer. With nv a multiple of 4 that is the next detector column; otherwise the
            // sample of slice z is slice 4*(nv/4)+z of column n, the zero padding, or slice
            // 4*(nv/4)+z-nvpad of column n+1.
            const float d = __fsub_rn(posu, static_cast<float>(n));
            const int nvpad = (nv & 3) ? nz4 + 4 : nv;
#pragma unroll
            for (int c = 0; c < CZ; c += 4) {
                const int g = (z0 + c) / 4;
                const float wb = tilt ? fabsf(__fsub_rn(d, __fmul_rn(static_cast<float>(g), tinc))) : fabsf(d);
                const float wa = __fsub_rn(1.0f, wb);
#pragma unroll
                for (int q = 0; q < 4 && c + q < CZ; ++q) {
                    const int z = z0 + c + q;
                    if (z < nz4) {
                        float pa = sample<DT>(proj, base + static_cast<size_t>(z) * nu);
                        float pb;
                        if (nvpad == nv) {
                            pb = sample<DT>(proj, base + static_cast<size_t>(z) * nu + 1);
                        } else {
                            const int k = nz4 + z;
                            pb = k < nv ? sample<DT>(proj, base + static_cast<size_t>(k) * nu)
                                 : k < nvpad ? 0.0f
                                             : sample<DT>(proj, base + static_cast<size_t>(k - nvpad) * nu + 1);
                        }
                        if (weight || DT != MR_F32) {
                            pa = __fmul_rn(pa, w);
                            pb = __fmul_rn(pb, w);
                        }
                        acc[c + q] = __fadd_rn(acc[c + q], __fadd_rn(__fmul_rn(pa, wa), __fmul_rn(pb, wb)));
                    }
                }
            }
        } else if (!tilt) {
            const float wb = fabsf(__fsub_rn(posu, static_cast<float>(n)));
            const float wa = __fsub_rn(1.0f, wb);
#pragma unroll
            for (int c = 0; c < CZ; ++c) {
                const int z = z0 + c;
                if (z < nz4) {
                    float pa = sample<DT>(proj, base + static_cast<size_t>(z) * nu);
                    float pb = sample<DT>(proj, base + static_cast<size_t>(z) * nu + 1);
                    if (weight || DT != MR_F32) {
                        pa = __fmul_rn(pa, w);
                        pb = __fmul_rn(pb, w);
                    }
                    acc[c] = __fadd_rn(acc[c], __fadd_rn(__fmul_rn(pa, wa), __fmul_rn(pb, wb)));
                }
            }
        } else {
            // tilt branch: one weight per group of 4 slices, the position drifting by tinc per
            // group, evaluated as the reference's sequence (:86-105)
            posu = __fsub_rn(posu, static_cast<float>(n));
            const int g0 = z0 / 4;
            for (int g = 0; g < g0; ++g) posu = __fsub_rn(posu, tinc);
#pragma unroll
            for (int c = 0; c < CZ; c += 4) {
                const int g = g0 + c / 4;
                const float wb = fabsf(__fsub_rn(posu, __fmul_rn(static_cast<float>(g), tinc)));
                const float wa = __fsub_rn(1.0f, wb);
#pragma unroll
                for (int q = 0; q < 4 && c + q < CZ; ++q) {
                    const int z = z0 + c + q;
                    if (z < nz4) {
                        float pa = sample<DT>(proj, base + static_cast<size_t>(z) * nu);
                        float pb = sample<DT>(proj, base + static_cast<size_t>(z) * nu + 1);
                        if (weight || DT != MR_F32) {
                            pa = __fmul_rn(pa, w);
                            pb = __fmul_rn(pb, w);
                        }
                        acc[c + q] = __fadd_rn(acc[c + q], __fadd_rn(__fmul_rn(pa, wa), __fmul_rn(pb, wb)));
                    }
                }
                posu = __fsub_rn(posu, tinc);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < CZ; ++c)
        if (z0 + c < nz4) col[z0 + c] = acc[c];
}

// ------------------------------------------------------------------ FDK

// FDKbp_single::project_volume_onto_image_c main loop (fdkbp_single.cpp:488-525) with
// get_pixel_value_c (:641-683); i, j, k index cbct_volume (x fastest), k in [kbegin, kend).
// The result is stored at the final position of FdkReconBase::Process
// (fdkreconbase.cpp:259-270): volume[nv-1-k][j][nu-1-i].
template <int DT, int CZ>
__global__ void __launch_bounds__(128) k_fdk(const void *__restrict__ proj, const float *__restrict__ scale, int nu,
                                             int nv, int nproj, const float *__restrict__ xip,
                                             const float *__restrict__ yip, const float *__restrict__ zip,
                                             int uniform_z, const uint32_t *__restrict__ mask, int accumulate,
                                             int kend, int kbegin, float *__restrict__ vol)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = kbegin + blockIdx.z * CZ;
    if (i >= nu || j >= nu) return;
    const size_t plane = static_cast<size_t>(nu) * nu;
    const size_t out_xy = static_cast<size_t>(j) * nu + (nu - 1 - i);
    float acc[CZ];
#pragma unroll
    for (int c = 0; c < CZ; ++c) {
        const int k = k0 + c;
        acc[c] = (accumulate && k < kend) ? vol[static_cast<size_t>(nv - 1 - k) * plane + out_xy] : 0.0f;
    }
    const bool inside = static_cast<uint32_t>(i) > mask[2 * j] && static_cast<uint32_t>(i) <= mask[2 * j + 1];
    if (inside) {
        const float fh = static_cast<float>(nv), fw = static_cast<float>(nu);
        const size_t pstride = static_cast<size_t>(nu) * nv;
        for (int p = 0; p < nproj; ++p) {
            const float *X = xip + (static_cast<size_t>(p) * nu + i) * 3;
            const float *Y = yip + (static_cast<size_t>(p) * nu + j) * 3;
            const float *Z = zip + static_cast<size_t>(p) * nv * 3;
            const float s = DT == MR_F32 ? 1.0f : scale[p];
            const float x0 = X[0], x1 = X[1], x2 = X[2];
            const float y0 = Y[0], y1 = Y[1], y2 = Y[2];
            if (uniform_z) {
                const float a2 = __fadd_rn(Z[3 * k0 + 2], y2);
                const float dw = __fdiv_rn(1.0f, __fadd_rn(a2, x2));
                const float a0 = __fadd_rn(Z[3 * k0], y0);
                const float c = __fadd_rn(__fmul_rn(dw, __fadd_rn(a0, x0)), 0.5f);
                if (c < 0.0f || c >= fw) continue;
                const int cc = __float2int_rz(c);
                const float dw2 = __fmul_rn(dw, dw);
                const size_t base = static_cast<size_t>(p) * pstride + cc;
#pragma unroll
                for (int q = 0; q < CZ; ++q) {
                    const int k = k0 + q;
                    if (k >= kend) break;
                    const float a1 = __fadd_rn(Z[3 * k + 1], y1);
                    const float r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, x1)), 0.5f);
                    if (r < 0.0f || r >= fh) continue; // value 0: acc + dw2*0 == acc
                    if (!MR_IN_BOUNDS(__float2int_rz(r), nv, kSiteFdkDirect) || !MR_IN_BOUNDS(cc, nu, kSiteFdkDirect)) continue;
                    float v = sample<DT>(proj, base + static_cast<size_t>(__float2int_rz(r)) * nu);
                    if (DT != MR_F32) v = v * s;
                    acc[q] = __fadd_rn(acc[q], __fmul_rn(dw2, v));
                }
            } else {
#pragma unroll
                for (int q = 0; q < CZ; ++q) {
                    const int k = k0 + q;
                    if (k >= kend) break;
                    const float a0 = __fadd_rn(Z[3 * k], y0);
                    const float a1 = __fadd_rn(Z[3 * k + 1], y1);
                    const float a2 = __fadd_rn(Z[3 * k + 2], y2);
                    const float dw = __fdiv_rn(1.0f, __fadd_rn(a2, x2));
                    const float r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, x1)), 0.5f);
                    const float c = __fadd_rn(__fmul_rn(dw, __fadd_rn(a0, x0)), 0.5f);
                    if (r < 0.0f || r >= fh || c < 0.0f || c >= fw) continue;
                    if (!MR_IN_BOUNDS(__float2int_rz(r), nv, kSiteFdkDirect) ||
                        !MR_IN_BOUNDS(__float2int_rz(c), nu, kSiteFdkDirect))
                        continue;
                    float v = sample<DT>(proj, static_cast<size_t>(p) * pstride +
                                                   static_cast<size_t>(__float2int_rz(r)) * nu + __float2int_rz(c));
                    if (DT != MR_F32) v = v * s;
                    acc[q] = __fadd_rn(acc[q], __fmul_rn(__fmul_rn(dw, dw), v));
                }
            }
        }
    }
#pragma unroll
    for (int c = 0; c < CZ; ++c) {
        const int k = k0 + c;
        if (k < kend) vol[static_cast<size_t>(nv - 1 - k) * plane + out_xy] = acc[c];
    }
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_bp_parallel_geometry(const float *angles_h, size_t nproj, size_t nu, float center, int direction,
                                  float *sin_h, float *cos_h, float *startu_h)
{
    MR_TRACE();
    if (nproj && (!angles_h || !sin_h || !cos_h || !startu_h))
        return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_geometry: null pointer");
    // StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:72-79); eDirection 0 = CW
    const float dirweight = 2.0f * (static_cast<float>(direction) - 0.5f);
    const size_t mcx = nu / 2; // MatrixCenterX = volume.Size(1)/2 (:195)
    for (size_t k = 0; k < nproj; ++k) {
        sin_h[k] = std::sin(dirweight * angles_h[k] * kFPi / 180.0f);
        cos_h[k] = std::cos(dirweight * angles_h[k] * kFPi / 180.0f);
        startu_h[k] = mcx * (sin_h[k] - cos_h[k]) + center;
    }
    return MR_OK;
}

mr_status mr_bp_circle_mask(size_t nx, size_t ny, int correcttilt, float tiltangle, size_t nslices, uint32_t *mask_h)
{
    MR_TRACE();
    if (!mask_h) return fail(MR_ERR_ARGUMENT, "mr_bp_circle_mask: null pointer");
    // BackProjectorModuleBase::BuildCircleMask (BackProjectorModuleBase.cpp:153-218), no matrix ROI
    const float cx = static_cast<float>(nx >> 1);
    const float cy = static_cast<float>(ny >> 1);
    float R = cx - 1;
    if (correcttilt) {
        const float slices = static_cast<float>(nslices);
        R -= std::floor(std::tan(std::fabs(tiltangle) * kFPi / 180.0f) * slices);
    }
    const float R2 = R * R;
    for (size_t i = 0; i < ny; ++i) {
        const float y = static_cast<float>(i) - cy;
        const float y2 = y * y;
        if (y2 <= R2) {
            const float x = std::sqrt(R2 - y2);
            mask_h[2 * i] = static_cast<uint32_t>(static_cast<size_t>(std::ceil(cx - x)));
            const size_t s = static_cast<size_t>(std::floor(cx + x));
            mask_h[2 * i + 1] = static_cast<uint32_t>(std::min(nx - 1u, s));
        } else {
            mask_h[2 * i] = 0;
            mask_h[2 * i + 1] = 0;
        }
    }
    return MR_OK;
}

mr_status mr_bp_parallel_tilt(float tiltangle, float tiltpivot, size_t roi_y0, float *tiltoffset, float *tiltinc)
{
    MR_TRACE();
    if (!tiltoffset || !tiltinc) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_tilt: null pointer");
    // MultiProjBPparallel.cpp:64-65,73
    *tiltoffset = (roi_y0 - tiltpivot) * std::tan(tiltangle * kFPi / 180);
    *tiltinc = 4 * std::tan(tiltangle * kFPi / 180);
    return MR_OK;
}

} // extern "C"

namespace mr {
// mr_bp_parallel for the volume rows [y_begin, y_end) (y_end <= nu, checked by the callers)
mr_status bp_parallel_rows(const void *proj_d, int dtype, const float *scale_d, const float *weight_d,
                           const int32_t *index_d, const float *sin_d, const float *cos_d, const float *startu_d,
                           size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d, int correcttilt,
                           float tiltoffset, float tiltinc, size_t y_begin, size_t y_end, int variant, float *vol_d,
                           void *stream)
{
    if (!proj_d || !sin_d || !cos_d || !startu_d || !mask_d || !vol_d)
        return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: null pointer");
    if (variant < 0 || variant > 2) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: unknown backprojector variant %d", variant);
    if (dtype != MR_F32 && dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: dtype");
    if (dtype != MR_F32 && !scale_d) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: 16-bit projections need scale_d");
    if (nu < 2 || nu > 65536 || nv > 65536) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: unsupported size");
    if (nproj > 0x7fffffff) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: too many projections");
    if (y_begin > y_end || y_end > nu) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel: row range outside [0, nu]");
    if (nproj == 0 || nv < 4 || y_begin == y_end) return MR_OK;
    constexpr int CZ = 8;
    dim3 block(32, 4);
    dim3 grid(div_up(nu, 32), div_up(y_end - y_begin, 4), div_up(nv, CZ));
    cudaStream_t s = as_stream(stream);
    const int np = static_cast<int>(nproj), iu = static_cast<int>(nu), iv = static_cast<int>(nv);
    const int yb = static_cast<int>(y_begin), ye = static_cast<int>(y_end);
    switch (dtype) {
    case MR_F32:
        k_bp_parallel<MR_F32, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, np, iu, iv,
                                                         mask_d, correcttilt, tiltoffset, tiltinc, yb, ye, variant, vol_d);
        break;
    case MR_BF16:
        k_bp_parallel<MR_BF16, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, np, iu, iv,
                                                          mask_d, correcttilt, tiltoffset, tiltinc, yb, ye, variant, vol_d);
        break;
    default:
        k_bp_parallel<MR_F16, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, np, iu, iv,
                                                         mask_d, correcttilt, tiltoffset, tiltinc, yb, ye, variant, vol_d);
    }
    return check_launch("k_bp_parallel");
}
} // namespace mr

extern "C" {

mr_status mr_bp_parallel(const void *proj_d, int dtype, const float *scale_d, const float *weight_d,
                         const int32_t *index_d, const float *sin_d, const float *cos_d, const float *startu_d,
                         size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d, int correcttilt, float tiltoffset,
                         float tiltinc, float *vol_d, void *stream)
{
    MR_TRACE();
    return bp_parallel_rows(proj_d, dtype, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, nproj, nu, nv, mask_d,
                            correcttilt, tiltoffset, tiltinc, 0, nu, 0, vol_d, stream);
}

// FDKbp_single::getProjMatrix (fdkbp_single.cpp:83-255), float arithmetic as written there.
static void fdk_projmatrix(const mr_fdk_geom *g, float roi0, float angles, float *pm)
{
    float extrinsic[16] = {0};
    float intrinsic[12] = {0};
    const float sad = g->sod, sid = g->sdd;
    const float offcenter = (g->ppoint[0] - roi0 - g->center) * g->voxelsize[0];
    float cam[3] = {0.0f, 0.0f, 0.0f};
    if (g->direction == 0) {
        cam[0] = sad * std::cos(-angles * kFPi / 180.0f);
        cam[1] = sad * std::sin(-angles * kFPi / 180.0f);
    } else {
        cam[0] = sad * std::cos(angles * kFPi / 180.0f);
        cam[1] = sad * std::sin(angles * kFPi / 180.0f);
    }
    float plt[3], pup[3], nrm[3];
    const float vup[3] = {0.0f, 0.0f, 1.0f};
    const float tgt[3] = {0.0f, 0.0f, 0.0f};
    nrm[0] = cam[0] - tgt[0];
    nrm[1] = cam[1] - tgt[1];
    nrm[2] = cam[2] - tgt[2];
    const float nn = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    nrm[0] /= nn;
    nrm[1] /= nn;
    nrm[2] /= nn;
    plt[0] = nrm[1] * vup[2] - nrm[2] * vup[1];
    plt[1] = nrm[2] * vup[0] - nrm[0] * vup[2];
    plt[2] = nrm[0] * vup[1] - nrm[1] * vup[0];
    const float np = std::sqrt(plt[0] * plt[0] + plt[1] * plt[1] + plt[2] * plt[2]);
    plt[0] /= np;
    plt[1] /= np;
    plt[2] /= np;
    pup[0] = plt[1] * nrm[2] - plt[2] * nrm[1];
    pup[1] = plt[2] * nrm[0] - plt[0] * nrm[2];
    pup[2] = plt[0] * nrm[1] - plt[1] * nrm[0];
    const float nq = std::sqrt(pup[0] * pup[0] + pup[1] * pup[1] + pup[2] * pup[2]);
    pup[0] /= nq;
    pup[1] /= nq;
    pup[2] /= nq;
    extrinsic[0] = -1.0f * plt[0];
    extrinsic[1] = -1.0f * plt[1];
    extrinsic[2] = -1.0f * plt[2];
    extrinsic[4] = -1.0f * pup[0];
    extrinsic[5] = -1.0f * pup[1];
    extrinsic[6] = -1.0f * pup[2];
    extrinsic[8] = -1.0f * nrm[0];
    extrinsic[9] = -1.0f * nrm[1];
    extrinsic[10] = -1.0f * nrm[2];
    extrinsic[15] = 1.0f;
    extrinsic[3] = plt[0] * tgt[0] + plt[1] * tgt[1] + plt[2] * tgt[2] - offcenter;
    extrinsic[7] = pup[0] * tgt[0] + pup[1] * tgt[1] + pup[2] * tgt[2];
    extrinsic[11] = nrm[0] * tgt[0] + nrm[1] * tgt[1] + nrm[2] * tgt[2] + sad;
    intrinsic[0] = 1.0f / g->resolution[0];
    intrinsic[5] = 1.0f / g->resolution[1];
    intrinsic[10] = 1.0f / sid;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) {
            float acc = 0.0f;
            for (int k = 0; k < 4; ++k) acc += intrinsic[i * 4 + k] * extrinsic[k * 4 + j];
            pm[i * 4 + j] = acc;
        }
}

// Volume origin and the CBCT row window of project_volume_onto_image_c (fdkbp_single.cpp:302-372)
// for roi = projection_roi = {0, 0, nu, nv} and a volume of nu x nu x nv, float as written there.
static void fdk_frame(const mr_fdk_geom *g, size_t nu, size_t nv, float origin[3], size_t cb[4])
{
    const size_t roi[4] = {0, 0, nu, nv};
    const size_t proi3 = nv;
    const float *spacing = g->voxelsize;
    const float U = static_cast<float>(roi[2] - roi[0]);
    const float V = static_cast<float>(roi[3] - roi[1]);
    origin[0] = -(U - g->center) * spacing[0] - spacing[0] / 2;
    origin[1] = -(U - g->center) * spacing[1] - spacing[1] / 2;
    origin[2] = -(V - (g->ppoint[1] - roi[1])) * spacing[2] - spacing[2] / 2;
    const float radius = static_cast<float>(nu) * g->voxelsize[0] / 2;
    cb[0] = roi[0];
    cb[1] = 0;
    cb[2] = roi[2];
    cb[3] = 0;
    const float fp1 = g->ppoint[1];
    const float r1 = static_cast<float>(roi[1]), r3 = static_cast<float>(roi[3]);
    const float vx = g->voxelsize[0], sdd = g->sdd, sod = g->sod, res0 = g->resolution[0];
    if (fp1 >= r1 && fp1 >= r3) {
        cb[3] = static_cast<size_t>(fp1 - ((fp1 - r3) * vx * sdd / (sod + radius)) / res0);
        const float value = fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0;
        cb[1] = value <= 0 ? 0 : static_cast<size_t>(fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0);
    }
    if (fp1 < r1 && fp1 < r3) {
        const float value = fp1 + ((r1 - fp1) * vx * sdd / (sod + radius)) / res0;
        cb[1] = static_cast<size_t>(value);
        const float value2 = fp1 + ((r3 - fp1) * vx * sdd / (sod - radius)) / res0;
        cb[3] = value2 >= proi3 ? proi3 : static_cast<size_t>(static_cast<float>(value2));
    }
    if (fp1 >= r1 && fp1 < r3) {
        const float value = fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0;
        cb[1] = value <= 0 ? 0 : static_cast<size_t>(fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0);
        const float value2 = fp1 + ((r3 - fp1) * vx * sdd / (sod - radius)) / res0;
        cb[3] = value2 >= proi3 ? proi3 : static_cast<size_t>(static_cast<float>(value2));
    }
    if (cb[1] != 0) cb[1] -= 8; // the reference's unsigned test cb[1]-8 >= 0 always holds (:369-372)
    if (cb[3] + 8 <= proi3) cb[3] += 8;
}

mr_status mr_fdk_partials(const mr_fdk_geom *g, size_t nu, size_t nv, const float *angles_h, size_t nproj,
                          float *xip_h, float *yip_h, float *zip_h, float *sad_sid_2, float *scale, int *uniform_z)
{
    MR_TRACE();
    if (!g || (nproj && (!angles_h || !xip_h || !yip_h || !zip_h)) || !sad_sid_2 || !scale || !uniform_z)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_partials: null pointer");
    if (nu == 0 || nv == 0) return fail(MR_ERR_ARGUMENT, "mr_fdk_partials: empty detector");
    const size_t roi[4] = {0, 0, nu, nv};
    const float *spacing = g->voxelsize;
    float origin[3];
    size_t cb[4];
    fdk_frame(g, nu, nv, origin, cb);
    const float ic[2] = {g->ppoint[0] - cb[0], g->ppoint[1] - cb[1]};
    *sad_sid_2 = (g->sod * g->sod) / (g->sdd * g->sdd);
    *scale = g->sod / g->sdd;
    int uniform = 1;
    for (size_t p = 0; p < nproj; ++p) {
        float pm[12];
        fdk_projmatrix(g, static_cast<float>(roi[0]), angles_h[p], pm);
        float *X = xip_h + p * nu * 3;
        float *Y = yip_h + p * nu * 3;
        float *Z = zip_h + p * nv * 3;
        for (size_t i = 0; i < nu; ++i) {
            const float x = static_cast<float>(origin[0] + static_cast<long>(i) * spacing[0]);
            X[i * 3 + 0] = x * (pm[0] + ic[0] * pm[8]);
            X[i * 3 + 1] = x * (pm[4] + ic[1] * pm[8]);
            X[i * 3 + 2] = x * pm[8];
        }
        for (size_t j = 0; j < nu; ++j) {
            const float y = static_cast<float>(origin[1] + static_cast<long>(j) * spacing[1]);
            Y[j * 3 + 0] = y * (pm[1] + ic[0] * pm[9]);
            Y[j * 3 + 1] = y * (pm[5] + ic[1] * pm[9]);
            Y[j * 3 + 2] = y * pm[9];
        }
        for (size_t k = 0; k < nv; ++k) {
            const float z = static_cast<float>(origin[2] + static_cast<long>(k) * spacing[2]);
            if (g->correcttilt) {
                // :438-444 (sequential semantics; the reference races on pm[3] under OpenMP)
                const float pos = static_cast<float>(cb[3]) - static_cast<float>(k) - static_cast<float>(g->tiltpivot);
                const float cor = std::tan(-g->tiltangle * kDPi / 180) * pos + g->center;
                pm[3] = ((cor - (g->ppoint[0] - roi[0])) * g->voxelsize[0]) / g->resolution[0];
            }
            Z[k * 3 + 0] = z * (pm[2] + ic[0] * pm[10]) + ic[0] * pm[11] + pm[3];
            Z[k * 3 + 1] = z * (pm[6] + ic[1] * pm[10]) + ic[1] * pm[11] + pm[7];
            Z[k * 3 + 2] = z * pm[10] + pm[11];
            if (k > 0 && (Z[k * 3] != Z[0] || Z[k * 3 + 2] != Z[2])) uniform = 0;
        }
    }
    *uniform_z = uniform;
    return MR_OK;
}

// FDKbp::getProjMatrix (fdkbp.cpp:83-255): the projection matrix in double.
static void fdk_projmatrix64(const mr_fdk_geom *g, double angle, double *pm)
{
    double ext[16] = {0}, intr[12] = {0};
    const double sad = g->sod, sid = g->sdd;
    const double offcenter = (static_cast<double>(g->ppoint[0]) - g->center) * g->voxelsize[0];
    const double a = (g->direction == 0 ? -angle : angle) * kDPi / 180.0;
    const double cam[3] = {sad * std::cos(a), sad * std::sin(a), 0.0};
    const double nn = std::sqrt(cam[0] * cam[0] + cam[1] * cam[1] + cam[2] * cam[2]);
    const double nrm[3] = {cam[0] / nn, cam[1] / nn, cam[2] / nn};
    // plt = nrm x vup, pup = plt x nrm with vup = (0, 0, 1)
    double plt[3] = {nrm[1], -nrm[0], 0.0};
    const double np = std::sqrt(plt[0] * plt[0] + plt[1] * plt[1]);
    plt[0] /= np;
    plt[1] /= np;
    double pup[3] = {plt[1] * nrm[2] - plt[2] * nrm[1], plt[2] * nrm[0] - plt[0] * nrm[2], plt[0] * nrm[1] - plt[1] * nrm[0]};
    const double nq = std::sqrt(pup[0] * pup[0] + pup[1] * pup[1] + pup[2] * pup[2]);
    pup[0] /= nq;
    pup[1] /= nq;
    pup[2] /= nq;
    for (int c = 0; c < 3; ++c) {
        ext[c] = -plt[c];
        ext[4 + c] = -pup[c];
        ext[8 + c] = -nrm[c];
    }
    ext[3] = -offcenter;
    ext[7] = 0.0;
    ext[11] = sad;
    ext[15] = 1.0;
    intr[0] = 1.0 / g->resolution[0];
    intr[5] = 1.0 / g->resolution[1];
    intr[10] = 1.0 / sid;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 4; ++k) acc += intr[i * 4 + k] * ext[k * 4 + j];
            pm[i * 4 + j] = acc;
        }
}

mr_status mr_fdk_maps64(const mr_fdk_geom *g, size_t nu, size_t nv, const float *angles_h, size_t nproj,
                        double *maps_h)
{
    MR_TRACE();
    if (!g || (nproj && (!angles_h || !maps_h))) return fail(MR_ERR_ARGUMENT, "mr_fdk_maps64: null pointer");
    if (nu == 0 || nv == 0) return fail(MR_ERR_ARGUMENT, "mr_fdk_maps64: empty detector");
    float originf[3];
    size_t cb[4];
    fdk_frame(g, nu, nv, originf, cb); // the row window decides the image centre as in the float path
    const double s0 = g->voxelsize[0], s1 = g->voxelsize[1], s2 = g->voxelsize[2];
    const double U = static_cast<double>(nu), V = static_cast<double>(nv);
    const double o0 = -(U - g->center) * s0 - s0 / 2, o1 = -(U - g->center) * s1 - s1 / 2;
    const double o2 = -(V - static_cast<double>(g->ppoint[1])) * s2 - s2 / 2;
    const double ic0 = static_cast<double>(g->ppoint[0]) - static_cast<double>(cb[0]);
    const double ic1 = static_cast<double>(g->ppoint[1]) - static_cast<double>(cb[1]);
    // tilt: pm[3] of slice k = ((cor(k) - ppoint[0]) * vx) / res0, cor(k) = tan(-tilt) (cb3 - k - pivot) + centre
    const double tt = g->correcttilt ? std::tan(-static_cast<double>(g->tiltangle) * kDPi / 180.0) : 0.0;
    for (size_t p = 0; p < nproj; ++p) {
        double pm[12];
        fdk_projmatrix64(g, angles_h[p], pm);
        double pm3 = pm[3], pm3k = 0.0;
        if (g->correcttilt) {
            const double c0 = tt * (static_cast<double>(cb[3]) - g->tiltpivot) + g->center;
            pm3 = ((c0 - g->ppoint[0]) * g->voxelsize[0]) / g->resolution[0];
            pm3k = -tt * g->voxelsize[0] / g->resolution[0];
        }
        const double A[3] = {pm[0] + ic0 * pm[8], pm[4] + ic1 * pm[8], pm[8]};
        const double B[3] = {pm[1] + ic0 * pm[9], pm[5] + ic1 * pm[9], pm[9]};
        const double C[3] = {pm[2] + ic0 * pm[10], pm[6] + ic1 * pm[10], pm[10]};
        const double D[3] = {ic0 * pm[11] + pm3, ic1 * pm[11] + pm[7], pm[11]};
        const double Dk[3] = {pm3k, 0.0, 0.0};
        double *m = maps_h + p * 12;
        for (int r = 0; r < 3; ++r) {
            m[4 * r + 0] = A[r] * s0;
            m[4 * r + 1] = B[r] * s1;
            m[4 * r + 2] = C[r] * s2 + Dk[r];
            m[4 * r + 3] = A[r] * o0 + B[r] * o1 + C[r] * o2 + D[r];
        }
    }
    return MR_OK;
}

mr_status mr_fdk_backproject_slab(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                                  size_t nproj, const float *xip_d, const float *yip_d, const float *zip_d, int uniform_z,
                                  const uint32_t *mask_d, int box_w, int box_h, int accumulate, size_t k_begin,
                                  size_t k_end, float *vol_d, void *stream)
{
    MR_TRACE();
    if (!proj_d || !xip_d || !yip_d || !zip_d || !mask_d || !vol_d)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: null pointer");
    if (dtype != MR_F32 && dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: dtype");
    if (dtype != MR_F32 && !scale_d) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: 16-bit projections need scale_d");
    if (nu == 0 || nv == 0 || nu > 65536 || nv > 65536) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: unsupported size");
    if (nproj > 0x7fffffff) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: too many projections");
    if (k_begin > k_end || k_end > nv) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject: slice range outside [0, nv]");
    if (k_begin == k_end) return MR_OK;
    cudaStream_t s = as_stream(stream);
    if (uniform_z && box_w > 0 && box_h > 0 && nproj > 0) {
        mr_status st = fdk_tma_launch(proj_d, dtype, scale_d, nu, nv, nproj, xip_d, yip_d, zip_d, mask_d, accumulate,
                                      static_cast<int>(k_begin), static_cast<int>(k_end), vol_d, box_w, box_h, s);
        if (st != MR_ERR_UNSUPPORTED) return st;
    }
    constexpr int CZ = 8;
    dim3 block(32, 4);
    dim3 grid(div_up(nu, 32), div_up(nu, 4), div_up(k_end - k_begin, CZ));
    const int np = static_cast<int>(nproj), iu = static_cast<int>(nu), iv = static_cast<int>(nv);
    const int kb = static_cast<int>(k_begin), ke = static_cast<int>(k_end);
    switch (dtype) {
    case MR_F32:
        k_fdk<MR_F32, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, iu, iv, np, xip_d, yip_d, zip_d, uniform_z, mask_d,
                                                 accumulate, ke, kb, vol_d);
        break;
    case MR_BF16:
        k_fdk<MR_BF16, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, iu, iv, np, xip_d, yip_d, zip_d, uniform_z, mask_d,
                                                  accumulate, ke, kb, vol_d);
        break;
    default:
        k_fdk<MR_F16, CZ><<<grid, block, 0, s>>>(proj_d, scale_d, iu, iv, np, xip_d, yip_d, zip_d, uniform_z, mask_d,
                                                 accumulate, ke, kb, vol_d);
    }
    return check_launch("k_fdk");
}

mr_status mr_fdk_backproject(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv, size_t nproj,
                             const float *xip_d, const float *yip_d, const float *zip_d, int uniform_z,
                             const uint32_t *mask_d, int box_w, int box_h, int accumulate, float *vol_d, void *stream)
{
    MR_TRACE();
    return mr_fdk_backproject_slab(proj_d, dtype, scale_d, nu, nv, nproj, xip_d, yip_d, zip_d, uniform_z, mask_d, box_w,
                                   box_h, accumulate, 0, nv, vol_d, stream);
}

} // extern "C"
