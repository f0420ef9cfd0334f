// Parallel-beam backprojection with TMA-staged projection rows (sm_100a).
//
// Arithmetic of MultiProjectionBPparallel::BackProject (MultiProjBPparallel.cpp:39-170),
// every float operation in the reference's order with explicitly rounded intrinsics, so the
// volume is bit-identical to the plain kernel and to the reference (no-tilt branch):
//   u = (startu_i + cos_i y) - sin_i x,  n = (int)u in [0, nu-2],  f = |u - n|,
//   vol[y-1][x-1][z] += (P[z][n] (1 - f) + P[z][n+1] f)          (P pre-multiplied by weight_i)
//
// Tiling: a CTA owns 32 (x) x 8 (y) voxel columns x 32 slices; a thread keeps its 32 slices
// in registers over all projections. In this geometry the detector column of a voxel does
// not depend on its slice, so one projection's footprint on the tile is at most ~34 columns
// by the tile's 32 detector rows: a producer warp projects the 4 tile corners with the voxel
// formula (affine in x and y, so the corners bound every voxel exactly; the per-projection
// sin/cos/startu are copied into shared memory with cp.async three batches ahead and the
// corners use those copies, as the voxels do), and one TMA tile
// load (cp.async.bulk.tensor.3d, no multicast) brings a 48 x 32 box per projection into
// shared memory, batches of 8 projections on two stages with bounded mbarrier waits. The
// box pitch is a compile-time constant, so the slice loop addresses its two samples with
// immediate offsets; the two interpolation products are one f32x2 mul (an f32x2 mul feeding
// scalar adds is not contracted). Rows beyond the detector are zero-filled by the TMA unit
// and never read (only z < 4*(nv/4) is updated). A footprint that does not fit the box falls
// back to guarded global loads for that tile and projection (same arithmetic). The volume
// (z fastest) is read and written as float4 runs.
#include "mr_common.cuh"
#include "mr_tma.cuh"

#include <algorithm>
#include <cmath>

namespace mr {

// Error word of this file's bounded waits (device globals are per translation unit);
// mr_device_status reads and clears it with the FDK kernels' word.
__device__ int g_bp_error = 0;

MR_BOUNDS_TAKE(bounds_take_bp)

int bp_device_status_take()
{
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_bp_error, sizeof(int)) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(g_bp_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

namespace bp2 {

constexpr int TX = 32, TY = 8, TZ = 32, THREADS = TX * TY, NB = 8, G = 4, BW = 48;
constexpr int CTAS_PER_SM = 2;
constexpr int BOXBYTES = BW * TZ * 4;
constexpr int GEO = 8; // sin, cos, startu, weight, slab (as int bits), pad

struct Params {
    const float *proj;
    const float *weight;
    const int32_t *index;
    const float *sinv, *cosv, *startu;
    const uint32_t *mask;
    float *vol;
    int nproj, nu, nv, nz4;
    int wait_limit; // tries of each per-batch wait
    int ybegin, yend; // volume rows y1 - 1 in [ybegin, yend)
};

struct Smem {
    float *box;      // [2][NB][TZ][BW]
    float *geo;      // [3][NB][GEO]
    int4 *meta;      // [2][NB]: x0, mode
    uint64_t *bars;  // [2]
    __device__ explicit Smem(unsigned char *base)
    {
        box = reinterpret_cast<float *>(base);
        geo = reinterpret_cast<float *>(base + 2 * NB * BOXBYTES);
        meta = reinterpret_cast<int4 *>(geo + 3 * NB * GEO);
        bars = reinterpret_cast<uint64_t *>(meta + 2 * NB);
    }
    static constexpr size_t bytes()
    {
        return 2 * NB * static_cast<size_t>(BOXBYTES) + 3 * NB * GEO * sizeof(float) + 2 * NB * sizeof(int4) +
               2 * sizeof(uint64_t);
    }
};

// Detector position of voxel (x1, y1) (1-based) for list entry i, reference order.
__device__ __forceinline__ float posu(float sn, float cs, float su, float fx, float fy)
{
    return __fsub_rn(__fadd_rn(su, __fmul_rn(cs, fy)), __fmul_rn(sn, fx));
}

// Slices of one voxel column for one staged projection: p points at the sample pair of slice 0
// (row pitch BW). FULL: all TZ slices exist.
template <bool HASW, bool FULL>
__device__ __forceinline__ void staged_column(float (&acc)[TZ], const float *p, float wa, float wb, float w, int zmax)
{
    const float2 wab = make_float2(wa, wb);
#pragma unroll
    for (int q = 0; q < TZ; ++q) {
        if (!FULL && q >= zmax) break;
        float pa = p[q * BW], pb = p[q * BW + 1];
        if (HASW) {
            pa = __fmul_rn(pa, w);
            pb = __fmul_rn(pb, w);
        }
        const float2 prod = __fmul2_rn(make_float2(pa, pb), wab);
        acc[q] = __fadd_rn(acc[q], __fadd_rn(prod.x, prod.y));
    }
}

// NearestNeighborBP's column (NNMultiProjBP.cpp:84-90): the sample at the truncated position.
template <bool HASW, bool FULL>
__device__ __forceinline__ void staged_column_nn(float (&acc)[TZ], const float *p, float w, int zmax)
{
#pragma unroll
    for (int q = 0; q < TZ; ++q) {
        if (!FULL && q >= zmax) break;
        float pa = p[q * BW];
        if (HASW) pa = __fmul_rn(pa, w);
        acc[q] = __fadd_rn(acc[q], pa);
    }
}

// NN selects NearestNeighborBP (NNMultiProjBP.cpp:36-121, no tilt): same positions, the one
// sample at n instead of the interpolation.
template <bool HASW, bool NN>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) k_bp_par_staged(const __grid_constant__ CUtensorMap tmap, const Params P)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    Smem S(smem);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = blockIdx.x * TX, j0 = P.ybegin + blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const int x1 = i0 + lane + 1, y1 = j0 + warp + 1;
    const int zmax = min(TZ, P.nz4 - z0);
    const bool valid = x1 <= P.nu && y1 <= P.yend;
    const bool inside = valid && static_cast<uint32_t>(x1) > P.mask[2 * (y1 - 1)] &&
                        static_cast<uint32_t>(x1) <= P.mask[2 * (y1 - 1) + 1];
    float *col = P.vol + (static_cast<size_t>(valid ? y1 - 1 : 0) * P.nu + (valid ? x1 - 1 : 0)) * P.nv + z0;
    const bool vec = (P.nv & 3) == 0 && zmax == TZ;

    float acc[TZ];
#pragma unroll
    for (int q = 0; q < TZ; q += 4) {
        if (inside && vec) {
            const float4 v = *reinterpret_cast<const float4 *>(col + q);
            acc[q] = v.x;
            acc[q + 1] = v.y;
            acc[q + 2] = v.z;
            acc[q + 3] = v.w;
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[q + e] = (inside && q + e < zmax) ? col[q + e] : 0.0f;
        }
    }
    if (!__syncthreads_or(inside)) return;

    if (threadIdx.x == 0) {
        tma::mbar_init(&S.bars[0], 1);
        tma::mbar_init(&S.bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int xa = i0 + 1, xb = min(i0 + TX, P.nu), ya = j0 + 1, yb = min(j0 + TY, P.yend);
    const int nbatch = (P.nproj + NB - 1) / NB;

    // Geometry of batch s into geometry buffer gb (cp.async by all threads, three batches
    // ahead; the weight only with HASW, the slab only with an index list).
    auto stage_geometry = [&](int s, int gb) {
        for (int idx = threadIdx.x; idx < NB * GEO; idx += THREADS) {
            const int b = idx / GEO, e = idx % GEO, i = s * NB + b;
            const float *src = e == 0 ? P.sinv : e == 1 ? P.cosv : e == 2 ? P.startu : e == 3 ? P.weight
                                                                                              : reinterpret_cast<const float *>(P.index);
            const bool ok = i < P.nproj && (e < 3 || (e == 3 && HASW) || (e == 4 && P.index));
            tma::copy4_zfill(S.geo + gb * NB * GEO + idx, ok ? src + i : P.sinv, ok);
        }
    };
    // Batch s (geometry in buffer gb) into stage st: warp 0 forms the footprints from the
    // staged geometry (4 corner lanes per projection) and issues the TMA copies.
    auto issue_batch = [&](int s, int st, int gb) {
        if (warp != 0) return;
        const int b = lane >> 2, corner = lane & 3;
        const int i = s * NB + b;
        const float *g = S.geo + (gb * NB + b) * GEO;
        int nmin = 0, nmax = 0;
        bool ok = i < P.nproj;
        if (ok) {
            const float u = posu(g[0], g[1], g[2], static_cast<float>((corner & 1) ? xb : xa),
                                 static_cast<float>((corner & 2) ? yb : ya));
            ok = fabsf(u) < 1.0e9f;
            nmin = nmax = ok ? __float2int_rz(u) : 0;
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            nmin = min(nmin, __shfl_xor_sync(0xffffffffu, nmin, o));
            nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
            ok = __shfl_xor_sync(0xffffffffu, static_cast<int>(ok), o) && ok;
        }
        // 0: global fallback, 1: staged, 2: no voxel of the tile has n in [0, nu-2]
        int mode = 0, x0 = 0;
        if (i < P.nproj && ok) {
            if (nmax < 0 || nmin > P.nu - 2) {
                mode = 2;
            } else {
                x0 = nmin >= 0 ? (nmin & ~3) : -(((-nmin) + 3) & ~3);
                if (nmax + 1 < x0 + BW) mode = 1;
            }
        }
        const unsigned staged = __ballot_sync(0xffffffffu, corner == 0 && mode == 1);
        if (lane == 0) tma::mbar_expect_tx(&S.bars[st], static_cast<uint32_t>(__popc(staged)) * BOXBYTES);
        __syncwarp();
        if (corner == 0 && i < P.nproj) {
            S.meta[st * NB + b] = make_int4(x0, mode, 0, 0);
            if (mode == 1) {
                const int slab = P.index ? __float_as_int(g[4]) : i;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                tma::load_3d(S.box + (st * NB + b) * (BW * TZ), &tmap, x0, z0, slab, &S.bars[st]);
            }
        }
    };

    for (int s = 0; s < 3 && s < nbatch; ++s) stage_geometry(s, s);
    tma::copy_wait_all();
    __syncthreads();
    for (int s = 0; s < 2 && s < nbatch; ++s) issue_batch(s, s, s);
    __syncthreads();

    uint32_t phase0 = 0, phase1 = 0;
    bool failed = false;
    const float fx = static_cast<float>(x1), fy = static_cast<float>(y1);
    const int um2 = P.nu - 2;
    int s = 0;
    for (int gb = 0; s < nbatch; ++s, gb = gb == 2 ? 0 : gb + 1) {
        const int st = s & 1; // stage buffer; geometry buffer gb = s % 3
        // a wait that timed out skips the batch in its whole warp; the block then leaves the
        // loop together at the barrier below
        const bool got = __all_sync(0xffffffffu, tma::mbar_wait(&S.bars[st], st ? phase1 : phase0, P.wait_limit));
        if (got) {
            if (st) phase1 ^= 1; else phase0 ^= 1;
        } else {
            failed = true;
            if (lane == 0) atomicExch(&g_bp_error, 1);
        }
        if (got && inside) {
            // per-projection set-up of this voxel column: 0 nothing to add, 1 staged, 2 guarded
            // global loads; n the detector column, off the sample offset in the stage
            auto setup = [&](int b, int &n, uint32_t &off, float &wa, float &wb) -> int {
                const int i = s * NB + b;
                n = 0;
                off = 0;
                wa = wb = 0.0f;
                if (i >= P.nproj) return 0;
                const int4 m = S.meta[st * NB + b];
                const float *g = S.geo + (gb * NB + b) * GEO;
                const float u = posu(g[0], g[1], g[2], fx, fy);
                n = __float2int_rz(u);
                if (m.y == 2 || n < 0 || n > um2) return 0;
                off = static_cast<uint32_t>((st * NB + b) * (BW * TZ) + (n - m.x));
                wb = fabsf(__fsub_rn(u, static_cast<float>(n)));
                wa = __fsub_rn(1.0f, wb);
                return m.y == 1 ? 1 : 2;
            };
#pragma unroll 1
            for (int b0 = 0; b0 < NB; b0 += G) {
                // the set-up of a group is formed first so its latency overlaps, then the
                // group's slice loops run in projection order (the reference's summation order)
                int q_mode[G], q_n[G];
                uint32_t q_off[G];
                float q_wa[G], q_wb[G];
#pragma unroll
                for (int e = 0; e < G; ++e) q_mode[e] = setup(b0 + e, q_n[e], q_off[e], q_wa[e], q_wb[e]);
                // a footprint that did not fit its box (rare; uniform over the CTA) sends the
                // whole group through the in-order path with guarded global loads
                bool fallback = false;
#pragma unroll
                for (int e = 0; e < G; ++e)
                    fallback |= s * NB + b0 + e < P.nproj && S.meta[st * NB + b0 + e].y == 0;
                if (!fallback) {
#pragma unroll
                    for (int e = 0; e < G; ++e) {
                        if (q_mode[e] != 1) continue;
                        if (!MR_IN_BOUNDS(q_off[e] + (zmax - 1) * BW + 1, 2 * NB * BW * TZ, kSiteBpStaged)) continue;
                        const float w = HASW ? S.geo[(gb * NB + b0 + e) * GEO + 3] : 1.0f;
                        if (NN) {
                            if (zmax == TZ) staged_column_nn<HASW, true>(acc, S.box + q_off[e], w, zmax);
                            else staged_column_nn<HASW, false>(acc, S.box + q_off[e], w, zmax);
                        } else if (zmax == TZ) {
                            staged_column<HASW, true>(acc, S.box + q_off[e], q_wa[e], q_wb[e], w, zmax);
                        } else {
                            staged_column<HASW, false>(acc, S.box + q_off[e], q_wa[e], q_wb[e], w, zmax);
                        }
                    }
                    continue;
                }
#pragma unroll 1
                for (int e = 0; e < G; ++e) {
                    const int b = b0 + e;
                    int n;
                    uint32_t off;
                    float wa, wb;
                    const int mode = setup(b, n, off, wa, wb); // formed again: no indexed arrays
                    const float w = HASW ? S.geo[(gb * NB + b) * GEO + 3] : 1.0f;
                    if (mode == 1 && !MR_IN_BOUNDS(off + (zmax - 1) * BW + 1, 2 * NB * BW * TZ, kSiteBpStaged)) continue;
                    if (mode == 1) {
                        if (NN) staged_column_nn<HASW, false>(acc, S.box + off, w, zmax);
                        else staged_column<HASW, false>(acc, S.box + off, wa, wb, w, zmax);
                    } else if (mode == 2) {
                        const int i = s * NB + b;
                        const int slab = P.index ? __float_as_int(S.geo[(gb * NB + b) * GEO + 4]) : i;
                        const float *img = P.proj + (static_cast<size_t>(slab) * P.nv + z0) * P.nu + n;
#pragma unroll
                        for (int q = 0; q < TZ; ++q) {
                            if (q >= zmax) break;
                            if (NN) {
                                float pa = __ldg(img + static_cast<size_t>(q) * P.nu);
                                if (HASW) pa = __fmul_rn(pa, w);
                                acc[q] = __fadd_rn(acc[q], pa);
                                continue;
                            }
                            float pa = __ldg(img + static_cast<size_t>(q) * P.nu), pb = __ldg(img + static_cast<size_t>(q) * P.nu + 1);
                            if (HASW) {
                                pa = __fmul_rn(pa, w);
                                pb = __fmul_rn(pb, w);
                            }
                            acc[q] = __fadd_rn(acc[q], __fadd_rn(__fmul_rn(pa, wa), __fmul_rn(pb, wb)));
                        }
                    }
                }
            }
        }
        // batch s+2's geometry complete and published; stage st and geometry buffer gb free
        tma::copy_wait_all();
        if (__syncthreads_or(failed)) break;
        if (s + 2 < nbatch) issue_batch(s + 2, st, gb == 0 ? 2 : gb - 1);
        if (s + 3 < nbatch) stage_geometry(s + 3, gb);
    }
    if (failed) {
        // copies still in flight: batch s (its wait expired) and batch s+1 when it was issued;
        // wait for them (bounded) before the block's shared memory is released
        const int st = s & 1;
        tma::mbar_wait(&S.bars[st], st ? phase1 : phase0);
        if (s + 1 < nbatch) tma::mbar_wait(&S.bars[st ^ 1], st ? phase0 : phase1);
    }
    if (inside) {
#pragma unroll
        for (int q = 0; q < TZ; q += 4) {
            if (vec) {
                *reinterpret_cast<float4 *>(col + q) = make_float4(acc[q], acc[q + 1], acc[q + 2], acc[q + 3]);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (q + e < zmax) col[q + e] = acc[q + e];
            }
        }
    }
}

} // namespace bp2

// Returns MR_ERR_UNSUPPORTED when staging does not apply (the caller uses the plain kernel).
mr_status bp_parallel_staged_launch(const float *proj_d, size_t nslabs, const float *weight_d, const int32_t *index_d,
                                    const float *sin_d, const float *cos_d, const float *startu_d, size_t nproj,
                                    size_t nu, size_t nv, const uint32_t *mask_d, size_t y_begin, size_t y_end,
                                    bool nn, float *vol_d, cudaStream_t s)
{
    using namespace bp2;
    if ((nu * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(proj_d) % 16) != 0 || nv < 4 || nslabs == 0 ||
        nu < static_cast<size_t>(BW))
        return MR_ERR_UNSUPPORTED;
    PFN_cuTensorMapEncodeTiled enc = tma::encode_fn();
    if (!enc) return MR_ERR_UNSUPPORTED;
    CUtensorMap map;
    cuuint64_t dims[3] = {nu, nv, nslabs};
    cuuint64_t strides[2] = {nu * 4, nu * nv * 4};
    cuuint32_t box[3] = {static_cast<cuuint32_t>(BW), static_cast<cuuint32_t>(TZ), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(proj_d), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(MR_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", static_cast<int>(cr));
    Params P;
    P.proj = proj_d;
    P.weight = weight_d;
    P.index = index_d;
    P.sinv = sin_d;
    P.cosv = cos_d;
    P.startu = startu_d;
    P.mask = mask_d;
    P.vol = vol_d;
    P.nproj = static_cast<int>(nproj);
    P.nu = static_cast<int>(nu);
    P.nv = static_cast<int>(nv);
    P.nz4 = static_cast<int>((nv / 4) * 4);
    P.wait_limit = tma::g_batch_wait_limit.load();
    P.ybegin = static_cast<int>(y_begin);
    P.yend = static_cast<int>(y_end);
    const size_t smem = Smem::bytes();
    dim3 grid(div_up(nu, TX), div_up(y_end - y_begin, TY), div_up(static_cast<size_t>(P.nz4), TZ));
    auto launch = [&](auto kernel) -> mr_status {
        MR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        kernel<<<grid, THREADS, smem, s>>>(map, P);
        return check_launch("k_bp_par_staged");
    };
    if (nn) return weight_d ? launch(k_bp_par_staged<true, true>) : launch(k_bp_par_staged<false, true>);
    return weight_d ? launch(k_bp_par_staged<true, false>) : launch(k_bp_par_staged<false, false>);
}

// mr_backproject.cu: the direct-load kernel for a range of volume rows
mr_status bp_parallel_rows(const void *proj_d, int dtype, const float *scale_d, const float *weight_d,
                           const int32_t *index_d, const float *sin_d, const float *cos_d, const float *startu_d,
                           size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d, int correcttilt,
                           float tiltoffset, float tiltinc, size_t y_begin, size_t y_end, int variant, float *vol_d,
                           void *stream);

} // namespace mr

using namespace mr;

extern "C" mr_status mr_bp_parallel_variant(int variant, const void *proj_d, size_t nslabs, int dtype,
                                            const float *scale_d, const float *weight_d, const int32_t *index_d,
                                            const float *sin_d, const float *cos_d, const float *startu_d, size_t nproj,
                                            size_t nu, size_t nv, const uint32_t *mask_d, int correcttilt,
                                            float tiltoffset, float tiltinc, size_t y_begin, size_t y_end, float *vol_d,
                                            void *stream)
{
    MR_TRACE();
    if (!proj_d || !sin_d || !cos_d || !startu_d || !mask_d || !vol_d)
        return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_variant: null pointer");
    if (variant < MR_BP_MULTIPROJ_PARALLEL || variant > MR_BP_NEAREST)
        return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_variant: unknown backprojector variant %d", variant);
    if (y_begin > y_end || y_end > nu) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_variant: row range outside [0, nu]");
    // the serial MultiProjectionBP computes exactly what MultiProjectionBPparallel computes
    // unless the tilt is corrected or the slice count is not a multiple of 4 (its second
    // interpolation sample is then read from another place of its projection buffer)
    if (variant == MR_BP_MULTIPROJ_SERIAL && !correcttilt && (nv & 3) == 0) variant = MR_BP_MULTIPROJ_PARALLEL;
    if (variant != MR_BP_MULTIPROJ_SERIAL && dtype == MR_F32 && !correcttilt && nproj > 0 && nproj <= 0x7fffffff &&
        nu >= 2 && nu <= 65536 && nv <= 65536 && y_begin < y_end) {
        if (!index_d && nslabs < nproj) return fail(MR_ERR_ARGUMENT, "mr_bp_parallel_variant: nslabs below nproj");
        mr_status st = bp_parallel_staged_launch(static_cast<const float *>(proj_d), nslabs, weight_d, index_d, sin_d,
                                                 cos_d, startu_d, nproj, nu, nv, mask_d, y_begin, y_end,
                                                 variant == MR_BP_NEAREST, vol_d, as_stream(stream));
        if (st != MR_ERR_UNSUPPORTED) return st;
    }
    return bp_parallel_rows(proj_d, dtype, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, nproj, nu, nv, mask_d,
                            correcttilt, tiltoffset, tiltinc, y_begin, y_end, variant, vol_d, stream);
}

extern "C" mr_status mr_bp_parallel_rows(const void *proj_d, size_t nslabs, int dtype, const float *scale_d,
                                         const float *weight_d, const int32_t *index_d, const float *sin_d,
                                         const float *cos_d, const float *startu_d, size_t nproj, size_t nu, size_t nv,
                                         const uint32_t *mask_d, int correcttilt, float tiltoffset, float tiltinc,
                                         size_t y_begin, size_t y_end, float *vol_d, void *stream)
{
    MR_TRACE();
    return mr_bp_parallel_variant(MR_BP_MULTIPROJ_PARALLEL, proj_d, nslabs, dtype, scale_d, weight_d, index_d, sin_d,
                                  cos_d, startu_d, nproj, nu, nv, mask_d, correcttilt, tiltoffset, tiltinc, y_begin,
                                  y_end, vol_d, stream);
}

extern "C" mr_status mr_bp_parallel_staged(const void *proj_d, size_t nslabs, int dtype, const float *scale_d,
                                           const float *weight_d, const int32_t *index_d, const float *sin_d,
                                           const float *cos_d, const float *startu_d, size_t nproj, size_t nu, size_t nv,
                                           const uint32_t *mask_d, int correcttilt, float tiltoffset, float tiltinc,
                                           float *vol_d, void *stream)
{
    MR_TRACE();
    return mr_bp_parallel_rows(proj_d, nslabs, dtype, scale_d, weight_d, index_d, sin_d, cos_d, startu_d, nproj, nu, nv,
                               mask_d, correcttilt, tiltoffset, tiltinc, 0, nu, vol_d, stream);
}
