// FDK backprojection with TMA-staged projection footprints (sm_100a).
//
// Same arithmetic as FDKbp_single::project_volume_onto_image_c (fdkbp_single.cpp:488-525)
// and get_pixel_value_c (:641-683), evaluated per voxel in the reference's order with
// explicitly rounded intrinsics, so the FP32 volume is bit-identical to the reference's
// for identical filtered projections. What changes is where the samples come from:
//
//  * CTA tile = 32 (x) x 8 (y) voxel columns x 32 slices; a thread owns one (x, y) column
//    and keeps its 32 slices in registers for all projections.
//  * Projections are consumed in batches of 4. For every projection one warp projects the
//    8 tile corners (the same float formulas as the voxels), takes the footprint's row and
//    column range with a 1-pixel margin and issues one TMA tile load of a fixed box
//    (bw x bh) of the projection into shared memory. Rows/columns outside the detector are
//    zero-filled by the TMA unit, which is exactly the reference's "outside -> 0" rule, so
//    the per-voxel loop needs no bounds test. Two stages are in flight (double buffering
//    on two mbarriers with bounded waits).
//  * The detector row is floor(r) of r = dw*(a1+x1)+0.5 (the reference truncates r >= 0
//    and rejects r < 0; floor sends r < 0 to a zero row), computed as the bit pattern of
//    r + 1.5*2^23 added with round-toward-minus-infinity: one FP32 add, no F2I.
//  * When a footprint does not fit the box, that projection falls back to guarded global
//    loads for this tile (same arithmetic, same result).
#include "mr_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace mr {

__device__ int g_device_error = 0;

namespace fdk2 {

constexpr int TI = 32, TJ = 8, TK = 32, NB = 4, THREADS = TI * TJ;
constexpr float kMagic = 12582912.0f; // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr int kWaitLimit = 1 << 22;

struct Params {
    const void *proj;
    const float *scale;
    const float *xip, *yip, *zip;
    const uint32_t *mask;
    float *vol;
    int nu, nv, nproj;
    int bw, bh;        // TMA box (elements)
    int boxbytes;      // per-projection shared buffer, 128-byte multiple
    int accumulate;
    int xalign;        // x coordinate alignment of a TMA load (elements)
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; false when the limit expired.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < kWaitLimit; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
                 "r"(smem_addr(bar))
                 : "memory");
}

template <int DT>
__device__ __forceinline__ float to_f32(typename Sample<DT>::T v)
{
    if constexpr (DT == MR_F32) return v;
    else if constexpr (DT == MR_BF16) return __bfloat162float(v);
    else return __half2float(v);
}

// Exact per-voxel detector coordinates (float, reference order), for the corner footprints.
__device__ __forceinline__ void project(const Params &P, int p, int i, int j, int k, float &r, float &c)
{
    const float *X = P.xip + (static_cast<size_t>(p) * P.nu + i) * 3;
    const float *Y = P.yip + (static_cast<size_t>(p) * P.nu + j) * 3;
    const float *Z = P.zip + (static_cast<size_t>(p) * P.nv + k) * 3;
    const float a0 = __fadd_rn(Z[0], Y[0]), a1 = __fadd_rn(Z[1], Y[1]), a2 = __fadd_rn(Z[2], Y[2]);
    const float dw = __fdiv_rn(1.0f, __fadd_rn(a2, X[2]));
    r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, X[1])), 0.5f);
    c = __fadd_rn(__fmul_rn(dw, __fadd_rn(a0, X[0])), 0.5f);
}

// Slices of one voxel column for one staged projection. FULL: all TK slices exist.
template <int DT, bool FULL>
__device__ __forceinline__ void staged_column(float (&acc)[TK], const typename Sample<DT>::T *col, const float4 *z4,
                                              float dw, float dw2, float x1f, float y1f, int off, int bw, float sc,
                                              int kmax)
{
#pragma unroll
    for (int q4 = 0; q4 < TK / 4; ++q4) {
        const float4 zz = z4[q4];
        const float zv[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (!FULL && q4 * 4 + e >= kmax) continue;
            const float a1 = __fadd_rn(zv[e], y1f);
            const float r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, x1f)), 0.5f);
            const int row = __float_as_int(__fadd_rd(r, kMagic)) - off;
            float v = to_f32<DT>(col[row * bw]);
            if constexpr (DT != MR_F32) v = v * sc;
            acc[q4 * 4 + e] = __fadd_rn(acc[q4 * 4 + e], __fmul_rn(dw2, v));
        }
    }
}

template <int DT>
__global__ void __launch_bounds__(THREADS, 2) k_fdk_tma(const __grid_constant__ CUtensorMap tmap, const Params P)
{
    using T = typename Sample<DT>::T;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *stage = smem;                                                      // [2][NB] boxes
    float *zipbuf = reinterpret_cast<float *>(smem + 2 * NB * P.boxbytes);            // [2][NB][TK]
    int4 *meta = reinterpret_cast<int4 *>(zipbuf + 2 * NB * TK);                     // [2][NB]
    uint64_t *bars = reinterpret_cast<uint64_t *>(meta + 2 * NB);                     // [2]

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ, k0 = blockIdx.z * TK;
    const int i = i0 + lane, j = j0 + warp;
    const int kmax = min(TK, P.nv - k0);
    const bool valid = i < P.nu && j < P.nu;
    const bool inside = valid && static_cast<uint32_t>(i) > P.mask[2 * j] && static_cast<uint32_t>(i) <= P.mask[2 * j + 1];
    const size_t plane = static_cast<size_t>(P.nu) * P.nu;
    const size_t out_xy = valid ? static_cast<size_t>(j) * P.nu + (P.nu - 1 - i) : 0;

    float acc[TK];
#pragma unroll
    for (int q = 0; q < TK; ++q)
        acc[q] = (valid && P.accumulate && q < kmax) ? P.vol[static_cast<size_t>(P.nv - 1 - (k0 + q)) * plane + out_xy]
                                                     : 0.0f;

    if (!__syncthreads_or(inside)) {
        if (valid) {
#pragma unroll
            for (int q = 0; q < TK; ++q)
                if (q < kmax) P.vol[static_cast<size_t>(P.nv - 1 - (k0 + q)) * plane + out_xy] = acc[q];
        }
        return;
    }

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int i_hi = min(i0 + TI - 1, P.nu - 1), j_hi = min(j0 + TJ - 1, P.nu - 1), k_hi = k0 + kmax - 1;
    const int nbatch = (P.nproj + NB - 1) / NB;

    // Footprints + TMA issue for batch s into stage st (warp 0); zip rows for all threads.
    auto produce = [&](int s, int st) {
        if (warp == 0) {
            const int b = lane >> 3, corner = lane & 7;
            const int p = s * NB + b;
            int rmin = 0, rmax = 0, cmin = 0, cmax = 0;
            bool ok = p < P.nproj;
            if (ok) {
                float r, c;
                project(P, p, (corner & 1) ? i_hi : i0, (corner & 2) ? j_hi : j0, (corner & 4) ? k_hi : k0, r, c);
                ok = fabsf(r) < 4.0e6f && fabsf(c) < 4.0e6f;
                rmin = rmax = ok ? __float2int_rd(r) : 0;
                cmin = cmax = ok ? __float2int_rd(c) : 0;
            }
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
                rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
                cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
                cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
                ok = __shfl_xor_sync(0xffffffffu, static_cast<int>(ok), o) && ok;
            }
            // 0: footprint does not fit (global fallback), 1: staged, 2: nothing to read
            int mode = 0, x0 = 0, y0 = 0;
            if (p < P.nproj && ok) {
                if (cmax < -1 || cmin > P.nu || rmax < -1 || rmin > P.nv) {
                    mode = 2;
                } else {
                    x0 = cmin - 1;
                    x0 = x0 >= 0 ? (x0 / P.xalign) * P.xalign : -(((-x0) + P.xalign - 1) / P.xalign) * P.xalign;
                    y0 = rmin - 1;
                    if (cmax + 1 < x0 + P.bw && rmax + 1 < y0 + P.bh) mode = 1;
                }
            }
            const unsigned staged = __ballot_sync(0xffffffffu, corner == 0 && mode == 1);
            if (lane == 0) mbar_expect_tx(&bars[st], static_cast<uint32_t>(__popc(staged)) * P.bw * P.bh * sizeof(T));
            __syncwarp();
            if (corner == 0 && p < P.nproj) {
                meta[st * NB + b] = make_int4(x0, y0, mode, 0);
                if (mode == 1) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    tma_load_3d(stage + (st * NB + b) * P.boxbytes, &tmap, x0, y0, p, &bars[st]);
                }
            }
        }
        for (int idx = threadIdx.x; idx < NB * TK; idx += THREADS) {
            const int b = idx / TK, q = idx % TK, p = s * NB + b;
            zipbuf[st * NB * TK + idx] = (p < P.nproj && q < kmax) ? P.zip[(static_cast<size_t>(p) * P.nv + k0 + q) * 3 + 1] : 0.0f;
        }
    };

    produce(0, 0);
    if (nbatch > 1) produce(1, 1);
    __syncthreads();

    uint32_t phase0 = 0, phase1 = 0;
    bool failed = false;
    const float fw = static_cast<float>(P.nu), fh = static_cast<float>(P.nv);
    for (int s = 0; s < nbatch; ++s) {
        const int st = s & 1;
        const uint32_t par = st ? phase1 : phase0;
        if (!mbar_wait(&bars[st], par)) {
            failed = true;
            atomicExch(&g_device_error, 1);
            break;
        }
        if (st) phase1 ^= 1; else phase0 ^= 1;

        if (inside) {
#pragma unroll 1
            for (int b = 0; b < NB; ++b) {
                const int p = s * NB + b;
                if (p >= P.nproj) break;
                const int4 m = meta[st * NB + b];
                if (m.z == 2) continue;
                const float *X = P.xip + (static_cast<size_t>(p) * P.nu + i) * 3;
                const float *Y = P.yip + (static_cast<size_t>(p) * P.nu + j) * 3;
                const float *Z = P.zip + static_cast<size_t>(p) * P.nv * 3;
                const float x0f = __ldg(X), x1f = __ldg(X + 1), x2f = __ldg(X + 2);
                const float y0f = __ldg(Y), y1f = __ldg(Y + 1), y2f = __ldg(Y + 2);
                const float dw = __fdiv_rn(1.0f, __fadd_rn(__fadd_rn(__ldg(Z + 2), y2f), x2f));
                const float c = __fadd_rn(__fmul_rn(dw, __fadd_rn(__fadd_rn(__ldg(Z), y0f), x0f)), 0.5f);
                if (c < 0.0f || c >= fw) continue;
                const int cc = static_cast<int>(c);
                float dw2 = __fmul_rn(dw, dw);
                const float sc = DT == MR_F32 ? 1.0f : __ldg(P.scale + p);
                const float4 *z4 = reinterpret_cast<const float4 *>(zipbuf + (st * NB + b) * TK);
                if (m.z == 1) {
                    const T *col = reinterpret_cast<const T *>(stage + (st * NB + b) * P.boxbytes) + (cc - m.x);
                    const int off = kMagicBits + m.y; // bits(r + magic) - off = floor(r) - y0
                    if (kmax == TK)
                        staged_column<DT, true>(acc, col, z4, dw, dw2, x1f, y1f, off, P.bw, sc, kmax);
                    else
                        staged_column<DT, false>(acc, col, z4, dw, dw2, x1f, y1f, off, P.bw, sc, kmax);
                } else {
                    const T *img = static_cast<const T *>(P.proj) + static_cast<size_t>(p) * P.nu * P.nv + cc;
#pragma unroll
                    for (int q4 = 0; q4 < TK / 4; ++q4) {
                        const float4 zz = z4[q4];
                        const float zv[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            if (q4 * 4 + e >= kmax) continue;
                            const float a1 = __fadd_rn(zv[e], y1f);
                            const float r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, x1f)), 0.5f);
                            if (r < 0.0f || r >= fh) continue;
                            float v = to_f32<DT>(img[static_cast<size_t>(static_cast<int>(r)) * P.nu]);
                            if constexpr (DT != MR_F32) v = v * sc;
                            acc[q4 * 4 + e] = __fadd_rn(acc[q4 * 4 + e], __fmul_rn(dw2, v));
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (s + 2 < nbatch) {
            produce(s + 2, st);
        }
    }
    if (failed) {
        // the other stage may still have a copy in flight: wait for it (bounded) before exit
        mbar_wait(&bars[0], phase0);
        mbar_wait(&bars[1], phase1);
    }
    if (valid) {
#pragma unroll
        for (int q = 0; q < TK; ++q)
            if (q < kmax) P.vol[static_cast<size_t>(P.nv - 1 - (k0 + q)) * plane + out_xy] = acc[q];
    }
}

// ---------------------------------------------------------------- host side

static PFN_cuTensorMapEncodeTiled encode_fn()
{
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    });
    return fn;
}

// Footprint of a tile for one projection, in double from the float partials (host guess of
// the box size; the kernel re-checks every footprint and falls back when one does not fit).
static void tile_footprint(const float *X, const float *Y, const float *Z, int i0, int i1, int j0, int j1, int k0,
                           int k1, double &rspan, double &cspan)
{
    double rmin = 1e30, rmax = -1e30, cmin = 1e30, cmax = -1e30;
    for (int corner = 0; corner < 8; ++corner) {
        const int i = corner & 1 ? i1 : i0, j = corner & 2 ? j1 : j0, k = corner & 4 ? k1 : k0;
        const double a0 = static_cast<double>(Z[3 * k]) + Y[3 * j];
        const double a1 = static_cast<double>(Z[3 * k + 1]) + Y[3 * j + 1];
        const double a2 = static_cast<double>(Z[3 * k + 2]) + Y[3 * j + 2];
        const double dw = 1.0 / (a2 + X[3 * i + 2]);
        const double r = dw * (a1 + X[3 * i + 1]) + 0.5, c = dw * (a0 + X[3 * i]) + 0.5;
        rmin = std::min(rmin, r);
        rmax = std::max(rmax, r);
        cmin = std::min(cmin, c);
        cmax = std::max(cmax, c);
    }
    rspan = std::floor(rmax) - std::floor(rmin);
    cspan = std::floor(cmax) - std::floor(cmin);
}

} // namespace fdk2

// Box size (bw, bh) that holds the tile footprints of (a sample of) the geometry.
static void fdk_box_guess(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                          int xalign, int &bw, int &bh)
{
    using namespace fdk2;
    double rs = 0, cs = 0;
    const int ti = static_cast<int>((nu + TI - 1) / TI), tj = static_cast<int>((nu + TJ - 1) / TJ);
    const int tk = static_cast<int>((nv + TK - 1) / TK);
    const size_t pstep = std::max<size_t>(1, nproj / 64);
    const int istep = std::max(1, ti / 8), jstep = std::max(1, tj / 16);
    for (size_t p = 0; p < nproj; p += pstep) {
        const float *X = xip_h + p * nu * 3, *Y = yip_h + p * nu * 3, *Z = zip_h + p * nv * 3;
        for (int a = 0; a < ti; a += (a + istep < ti ? istep : std::max(1, ti - 1 - a)))
            for (int b = 0; b < tj; b += (b + jstep < tj ? jstep : std::max(1, tj - 1 - b)))
                for (int kk : {0, tk - 1}) {
                    const int i0 = a * TI, j0 = b * TJ, k0 = kk * TK;
                    double r, c;
                    tile_footprint(X, Y, Z, i0, std::min<int>(i0 + TI - 1, static_cast<int>(nu) - 1), j0,
                                   std::min<int>(j0 + TJ - 1, static_cast<int>(nu) - 1), k0,
                                   std::min<int>(k0 + TK - 1, static_cast<int>(nv) - 1), r, c);
                    rs = std::max(rs, r);
                    cs = std::max(cs, c);
                }
    }
    // +1 margin each side, +1 for the inclusive range, + alignment slack on x
    bw = static_cast<int>(cs) + 3 + (xalign - 1);
    bh = static_cast<int>(rs) + 3;
    bw = (bw + xalign - 1) / xalign * xalign;
    bw = std::min(bw, 256);
    bh = std::min(bh, 256);
}

// Launches the TMA-staged FDK kernel; returns MR_ERR_UNSUPPORTED when the layout does not
// allow TMA (the caller then uses the plain kernel).
mr_status fdk_tma_launch(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv, size_t nproj,
                         const float *xip_d, const float *yip_d, const float *zip_d, const uint32_t *mask_d,
                         int accumulate, float *vol_d, int bw, int bh, cudaStream_t s)
{
    using namespace fdk2;
    const size_t es = dtype == MR_F32 ? 4 : 2;
    const int xalign = static_cast<int>(16 / es);
    if ((nu * es) % 16 != 0 || (reinterpret_cast<uintptr_t>(proj_d) % 16) != 0) return MR_ERR_UNSUPPORTED;
    if (bw <= 0 || bh <= 0 || bw > 256 || bh > 256 || bw % xalign) return MR_ERR_UNSUPPORTED;
    PFN_cuTensorMapEncodeTiled enc = encode_fn();
    if (!enc) return fail(MR_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    CUtensorMap map;
    cuuint64_t dims[3] = {nu, nv, nproj};
    cuuint64_t strides[2] = {nu * es, nu * nv * es};
    cuuint32_t box[3] = {static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMapDataType t = dtype == MR_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                            : dtype == MR_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                               : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    CUresult cr = enc(&map, t, 3, const_cast<void *>(proj_d), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(MR_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", static_cast<int>(cr));
    Params P;
    P.proj = proj_d;
    P.scale = scale_d;
    P.xip = xip_d;
    P.yip = yip_d;
    P.zip = zip_d;
    P.mask = mask_d;
    P.vol = vol_d;
    P.nu = static_cast<int>(nu);
    P.nv = static_cast<int>(nv);
    P.nproj = static_cast<int>(nproj);
    P.bw = bw;
    P.bh = bh;
    P.boxbytes = static_cast<int>((bw * bh * es + 127) / 128 * 128);
    P.accumulate = accumulate;
    P.xalign = xalign;
    const size_t smem = 2 * NB * static_cast<size_t>(P.boxbytes) + 2 * NB * TK * sizeof(float) + 2 * NB * sizeof(int4) +
                        2 * sizeof(uint64_t);
    if (smem > 110 * 1024) return MR_ERR_UNSUPPORTED;
    dim3 grid(div_up(nu, TI), div_up(nu, TJ), div_up(nv, TK));
    switch (dtype) {
    case MR_F32:
        MR_CUDA_TRY(cudaFuncSetAttribute(k_fdk_tma<MR_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024));
        k_fdk_tma<MR_F32><<<grid, THREADS, smem, s>>>(map, P);
        break;
    case MR_BF16:
        MR_CUDA_TRY(cudaFuncSetAttribute(k_fdk_tma<MR_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024));
        k_fdk_tma<MR_BF16><<<grid, THREADS, smem, s>>>(map, P);
        break;
    default:
        MR_CUDA_TRY(cudaFuncSetAttribute(k_fdk_tma<MR_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024));
        k_fdk_tma<MR_F16><<<grid, THREADS, smem, s>>>(map, P);
    }
    return check_launch("k_fdk_tma");
}

mr_status fdk_box_for(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                      int dtype, int *bw, int *bh)
{
    const int xalign = dtype == MR_F32 ? 4 : 8;
    fdk_box_guess(xip_h, yip_h, zip_h, nu, nv, nproj, xalign, *bw, *bh);
    return MR_OK;
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_fdk_box(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                     int dtype, int *box_w, int *box_h)
{
    if (!xip_h || !yip_h || !zip_h || !box_w || !box_h) return fail(MR_ERR_ARGUMENT, "mr_fdk_box: null pointer");
    if (dtype != MR_F32 && dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_fdk_box: dtype");
    if (nu == 0 || nv == 0 || nproj == 0) {
        *box_w = *box_h = 0;
        return MR_OK;
    }
    return fdk_box_for(xip_h, yip_h, zip_h, nu, nv, nproj, dtype, box_w, box_h);
}

mr_status mr_device_status(int *status)
{
    if (!status) return fail(MR_ERR_ARGUMENT, "mr_device_status: null pointer");
    int v = 0, zero = 0;
    MR_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)));
    MR_CUDA_TRY(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)));
    *status = v;
    return MR_OK;
}

} // extern "C"
