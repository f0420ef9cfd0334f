// FDK backprojection with TMA-staged projection footprints (sm_100a).
//
// Two kernels share one tiling and pipeline:
//
//  * k_fdk_exact (FP32, the reference path): the arithmetic of
//    FDKbp_single::project_volume_onto_image_c (fdkbp_single.cpp:488-525) and
//    get_pixel_value_c (:641-683), every per-voxel float operation in the reference's order
//    with explicitly rounded intrinsics, so the FP32 volume is bit-identical to the
//    reference's for identical filtered projections. The warp-uniform sums zip+yip of every slice are formed once per warp
//    and projection in shared memory.
//  * k_fdk_fast (16-bit projections, the precision form): per-projection affine detector
//    maps computed in FP64 on the host (FDKbp, fdkbp.cpp:83-640, is the double-geometry
//    variant of the same backprojector) and rounded once to float; per voxel column and
//    projection the distance weight and the detector column are formed once, the detector
//    row advances by a constant step per slice, and the weighted sample is accumulated in
//    FP32 by one mixed-precision fma (f32 += bf16 x bf16, or f16 x f16) with the weight
//    rounded to the storage type.
//
// Tiling and staging (both kernels):
//  * CTA tile = 32 (x) x 8 (y) voxel columns x 32 slices; a thread owns one (x, y) column
//    and keeps its 32 slices in registers for all projections.
//  * Projections are consumed in batches of NB (4 or 8). For every projection a producer
//    warp projects the 8 tile corners with the same formulas as the voxels, takes the
//    footprint's row and column range with a 1-pixel margin and issues one TMA tile load of
//    a fixed box (bw x bh) of the projection into shared memory. Rows/columns outside the
//    detector are zero-filled by the TMA unit, which is exactly the reference's
//    "outside -> 0" rule, so the per-voxel loop needs no bounds test. Two stages are in
//    flight (double buffering on two mbarriers with bounded waits).
//  * The per-projection geometry (detector maps, or the exact kernel's xip/yip/zip entries
//    of the tile) is copied with cp.async three batches ahead, and the footprints are formed
//    from those shared-memory copies, so no global load sits between two block barriers.
//  * The detector row is floor(r), taken from the bit pattern of r + 1.5*2^23 added with
//    round-toward-minus-infinity; the shared-memory address of the sample is one integer
//    multiply-add of those bits.
//  * When a footprint does not fit the box, that projection falls back to guarded global
//    loads for this tile (same arithmetic, same result).
#include "mr_common.cuh"
#include "mr_tma.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace mr {

__device__ int g_device_error = 0;
int bp_device_status_take();  // mr_bp_tma.cu
// bounds words of the bounds-checked build, one per translation unit with checks
int bounds_take_bp(unsigned long long *w);      // mr_bp_tma.cu
int bounds_take_direct(unsigned long long *w);  // mr_backproject.cu
int bounds_take_matched(unsigned long long *w); // mr_matched.cu
int bounds_take_ring(unsigned long long *w);    // mr_ringclean.cu
int bounds_take_spot(unsigned long long *w);    // mr_spotclean.cu
MR_BOUNDS_TAKE(bounds_take_fdk)
int msc_device_status_take(); // mr_spotclean.cu

namespace fdk2 {

constexpr int TI = 32, TJ = 8, TK = 32, THREADS = TI * TJ, NWARPS = THREADS / 32;
constexpr int CTAS_PER_SM = 2;
constexpr float kMagic = 12582912.0f; // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
// per-projection geometry staged in shared memory (floats)
constexpr int GEO_EXACT = TK + 3 * TI + 3 * TJ + 4; // zip1[TK], xip[TI][3], yip[TJ][3], Z0, Z2
constexpr int GEO_FAST = 32;                        // FP64 map[12] (24 words), scale, pad
// per-projection tile geometry of the fast kernel (floats, formed from the FP64 map)
constexpr int TGEO = 16;
enum { TG_W0, TG_M8, TG_M9, TG_AU, TG_BU, TG_AV, TG_BV, TG_M6, TG_FC, TG_FR, TG_C0, TG_R0, TG_SCALE };

struct Params {
    const void *proj;
    const float *scale;
    const float *xip, *yip, *zip; // exact kernel
    const double *maps;           // fast kernel: [nproj][12] (FP64)
    const uint32_t *mask;
    float *vol;
    int nu, nv, nproj;
    int bw, bh;       // TMA box (elements)
    int boxbytes;     // per-projection shared buffer, 128-byte multiple
    int rowbytes;     // bw * element size
    int accumulate;
    int kbegin, kend; // cbct slices backprojected: [kbegin, kend)
    int xalign;       // x coordinate alignment of a TMA load (elements)
    int wait_limit;   // tries of each per-batch wait
};

using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::copy4_zfill;
using tma::copy_wait_all;
using tma::smem_addr;

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    tma::load_3d(dst, map, x, y, z, bar);
}

// f32 accumulator += a * b with a, b in 16-bit storage (one instruction on sm_100).
template <int DT>
__device__ __forceinline__ float mixed_fma(unsigned short a, unsigned short b, float c)
{
    float d;
    if constexpr (DT == MR_BF16)
        asm("fma.rn.f32.bf16 %0, %1, %2, %3;" : "=f"(d) : "h"(a), "h"(b), "f"(c));
    else
        asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(a), "h"(b), "f"(c));
    return d;
}

template <int DT>
__device__ __forceinline__ unsigned short to_storage(float w)
{
    if constexpr (DT == MR_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(w));
    else return __half_as_ushort(__float2half_rn(w));
}

template <int DT>
__device__ __forceinline__ float from_storage(unsigned short v)
{
    if constexpr (DT == MR_BF16) return __bfloat162float(__ushort_as_bfloat16(v));
    else return __half2float(__ushort_as_half(v));
}

// Fast-kernel coordinates. The detector column and row of the tile's origin voxel
// (i0, j0, k0) are formed in FP64 from the FP64 map and split into an integer part and an FP32
// fraction; the other voxels add FP32 offsets from the origin, which stay within the tile's
// footprint (tens of pixels), so a coordinate carries an error of a few 1e-6 pixel instead of
// the ~1e-4 of an FP32 evaluation at detector magnitudes. With the map
// u = m0 i + m1 j + m3, v = m4 i + m5 j + m6 k + m7, w = m8 i + m9 j + m11 and
// c = u/w + 1/2, r = v/w + 1/2 (the FP64 oracle's formulas), the offsets from the origin are
// exactly  c - c0 = (au di + bu dj) / w,  r - r0 = (av di + bv dj + m6 dk) / w  with
// au = m0 - (c0 - 1/2) m8, bu = m1 - (c0 - 1/2) m9, av = m4 - (r0 - 1/2) m8,
// bv = m5 - (r0 - 1/2) m9. False when the origin is behind the source or out of range.
__device__ __forceinline__ bool tile_geometry(const double *m, int i0, int j0, int k0, float scale, float (&t)[TGEO])
{
    const double fi = i0, fj = j0, fk = k0;
    const double w0 = m[8] * fi + m[9] * fj + m[11];
    const double u0 = m[0] * fi + m[1] * fj + m[3];
    const double v0 = m[4] * fi + m[5] * fj + m[6] * fk + m[7];
    const bool ok = w0 > 0.0;
    const double cu = ok ? u0 / w0 : 0.0, rv = ok ? v0 / w0 : 0.0;
    const bool inrange = fabs(cu) < 1.0e9 && fabs(rv) < 1.0e9;
    const double c = inrange ? cu + 0.5 : 0.0, r = inrange ? rv + 0.5 : 0.0;
    const double cf = floor(c), rf = floor(r);
    t[TG_W0] = static_cast<float>(w0);
    t[TG_M8] = static_cast<float>(m[8]);
    t[TG_M9] = static_cast<float>(m[9]);
    t[TG_AU] = static_cast<float>(m[0] - cu * m[8]);
    t[TG_BU] = static_cast<float>(m[1] - cu * m[9]);
    t[TG_AV] = static_cast<float>(m[4] - rv * m[8]);
    t[TG_BV] = static_cast<float>(m[5] - rv * m[9]);
    t[TG_M6] = static_cast<float>(m[6]);
    t[TG_FC] = static_cast<float>(c - cf);
    t[TG_FR] = static_cast<float>(r - rf);
    t[TG_C0] = __int_as_float(static_cast<int>(cf));
    t[TG_R0] = __int_as_float(static_cast<int>(rf));
    t[TG_SCALE] = scale;
    return ok && inrange;
}

// Voxel (i0 + di, j0 + dj) relative to the tile origin: inverse depth dw, column
// c0 + tc, row of slice k0 + q: r0 + tr0 + q dr (tc, tr0 fractions relative to the integer
// parts TG_C0, TG_R0). The footprints and the voxels use this same function. The inverse
// depth is the hardware's approximate reciprocal (relative error ~1e-7, far below the 16-bit
// samples' 4e-3 and 5e-4 steps).
template <typename TG>
__device__ __forceinline__ void fast_coord(const TG &t, float di, float dj, float &dw, float &tc, float &tr0, float &dr)
{
    const float w = fmaf(t[TG_M8], di, fmaf(t[TG_M9], dj, t[TG_W0]));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(dw) : "f"(w));
    tc = fmaf(fmaf(t[TG_AU], di, t[TG_BU] * dj), dw, t[TG_FC]);
    tr0 = fmaf(fmaf(t[TG_AV], di, t[TG_BV] * dj), dw, t[TG_FR]);
    dr = t[TG_M6] * dw;
}

// Slices of one voxel column for one staged projection (exact arithmetic). a1: the 32
// per-slice sums zip1 + yip1 of this warp. FULL: all TK slices exist.
//
// Two slices per step on the paired FP32 pipe: (a1 + x1) and dw * (...) as f32x2 add and mul,
// + 0.5 as two scalar adds, the magic-number floor as one f32x2 add rounded down, and
// dw2 * v as one f32x2 mul followed by two scalar adds into the accumulators. Every operation
// is IEEE-rounded on its own, so each slice gets exactly the reference's float sequence; an
// f32x2 mul is never followed directly by an f32x2 add, because ptxas contracts that pair into
// an f32x2 fma even with explicit rounding.
template <bool FULL>
__device__ __forceinline__ void exact_column(float2 (&acc)[TK / 2], const unsigned char *smem, uint32_t base,
                                             uint32_t rowbytes, const float *a1, float x1f, float dw, float dw2,
                                             int kmax, uint32_t stage_bytes)
{
    (void)stage_bytes; // the stage buffers' size, for the bounds-checked build
    const float2 x1 = make_float2(x1f, x1f), dwp = make_float2(dw, dw), dw2p = make_float2(dw2, dw2);
    const float2 mg = make_float2(kMagic, kMagic);
#pragma unroll
    for (int q4 = 0; q4 < TK / 4; ++q4) {
        const float4 a4 = reinterpret_cast<const float4 *>(a1)[q4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = 4 * q4 + 2 * h; // slices q and q + 1 -> acc[q / 2]
            if (!FULL && q >= kmax) break;
            const bool two = FULL || q + 1 < kmax;
            const float2 m = __fmul2_rn(dwp, __fadd2_rn(h ? make_float2(a4.z, a4.w) : make_float2(a4.x, a4.y), x1));
            const float2 b = __fadd2_rd(make_float2(__fadd_rn(m.x, 0.5f), __fadd_rn(m.y, 0.5f)), mg);
            const uint32_t o0 = __float_as_uint(b.x) * rowbytes + base, o1 = __float_as_uint(b.y) * rowbytes + base;
            const float v0 = MR_IN_BOUNDS(o0, stage_bytes, kSiteFdkStaged) ? *reinterpret_cast<const float *>(smem + o0) : 0.0f;
            const float v1 = two && MR_IN_BOUNDS(o1, stage_bytes, kSiteFdkStaged)
                                 ? *reinterpret_cast<const float *>(smem + o1)
                                 : 0.0f;
            const float2 p = __fmul2_rn(dw2p, make_float2(v0, v1));
            acc[q >> 1].x = __fadd_rn(acc[q >> 1].x, p.x);
            if (two) acc[q >> 1].y = __fadd_rn(acc[q >> 1].y, p.y);
        }
    }
}

// Slices of one voxel column for one staged projection (fast arithmetic, 16-bit samples).
template <int DT, bool FULL>
__device__ __forceinline__ void fast_column_staged(float2 (&acc)[TK / 2], const unsigned char *smem, uint32_t base,
                                                   uint32_t rowbytes, float r0, float dr, unsigned short wt, int kmax)
{
    float2 rr = make_float2(r0, __fadd_rn(r0, dr));
    const float2 step = make_float2(2.0f * dr, 2.0f * dr), mg = make_float2(kMagic, kMagic);
#pragma unroll
    for (int q = 0; q < TK / 2; ++q) {
        if (!FULL && 2 * q >= kmax) break;
        const float2 b = __fadd2_rd(rr, mg);
        const unsigned short v0 = *reinterpret_cast<const unsigned short *>(smem + (__float_as_uint(b.x) * rowbytes + base));
        acc[q].x = mixed_fma<DT>(v0, wt, acc[q].x);
        if (FULL || 2 * q + 1 < kmax) {
            const unsigned short v1 =
                *reinterpret_cast<const unsigned short *>(smem + (__float_as_uint(b.y) * rowbytes + base));
            acc[q].y = mixed_fma<DT>(v1, wt, acc[q].y);
        }
        rr = __fadd2_rn(rr, step);
    }
}

// Shared-memory layout of both kernels. Geometry is triple-buffered: batch s+3's copies
// are in flight while batch s is consumed, and batch s+2's is complete for its footprints.
template <int NB, int GEO, bool A1>
struct Smem {
    unsigned char *stage; // [2][NB] boxes
    float *geo;           // [3][NB][GEO]
    float *a1;            // [NWARPS][NB][TK] (exact kernel)
    float2 *zy;           // [NWARPS][NB]: Z0 + y0, Z2 + y2 of the warp's voxel row (exact kernel)
    float *tg;            // [2][NB][TGEO] (fast kernel)
    int4 *meta;           // [2][NB]: x0, y0, mode; .w of a group's first entry: a footprint of the group
                          // did not fit its box
    uint64_t *bars;       // [2]
    uint32_t *gdesc;      // [NB][GEO]: source of each geometry element (exact kernel)
    __device__ Smem(unsigned char *base, int boxbytes)
    {
        stage = base;
        geo = reinterpret_cast<float *>(base + 2 * NB * boxbytes);
        a1 = geo + 3 * NB * GEO;
        zy = reinterpret_cast<float2 *>(a1 + (A1 ? NWARPS * NB * TK : 0));
        tg = reinterpret_cast<float *>(zy + (A1 ? NWARPS * NB : 0));
        meta = reinterpret_cast<int4 *>(tg + (A1 ? 0 : 2 * NB * TGEO));
        bars = reinterpret_cast<uint64_t *>(meta + 2 * NB);
        gdesc = reinterpret_cast<uint32_t *>(bars + 2);
    }
    static size_t bytes(int boxbytes)
    {
        return 2 * NB * static_cast<size_t>(boxbytes) +
               (3 * NB * GEO + (A1 ? NWARPS * NB * (TK + 2) : 2 * NB * TGEO)) * sizeof(float) +
               2 * NB * sizeof(int4) + 2 * sizeof(uint64_t) + (A1 ? NB * GEO * sizeof(uint32_t) : 0);
    }
};

// Sources of the exact kernel's geometry elements of a batch, fixed for the tile: element idx
// (projection b = idx / GEO_EXACT of the batch) is array[offset + p * stride], p the projection;
// bits 0-25 the offset, 26-27 the array (0 zip, 1 xip, 2 yip, 3 none: zero), 28-31 b.
template <int NB>
__device__ __forceinline__ void geometry_sources(const Params &P, uint32_t *gdesc, int i0, int j0, int k0, int kmax)
{
    for (int idx = threadIdx.x; idx < NB * GEO_EXACT; idx += THREADS) {
        const int b = idx / GEO_EXACT, e = idx % GEO_EXACT;
        uint32_t arr = 3, off = 0;
        if (e < TK) {
            if (e < kmax) arr = 0, off = static_cast<uint32_t>((k0 + e) * 3 + 1);
        } else if (e < TK + 3 * TI) {
            const int ii = i0 + (e - TK) / 3;
            if (ii < P.nu) arr = 1, off = static_cast<uint32_t>(ii * 3 + (e - TK) % 3);
        } else if (e < TK + 3 * TI + 3 * TJ) {
            const int jj = j0 + (e - TK - 3 * TI) / 3;
            if (jj < P.nu) arr = 2, off = static_cast<uint32_t>(jj * 3 + (e - TK - 3 * TI) % 3);
        } else if (e == TK + 3 * TI + 3 * TJ) {
            arr = 0, off = 0;
        } else if (e == TK + 3 * TI + 3 * TJ + 1) {
            arr = 0, off = 2;
        }
        gdesc[idx] = off | arr << 26 | static_cast<uint32_t>(b) << 28;
    }
}

// Starts the asynchronous copy of batch s's per-projection geometry into geometry buffer gb
// (all threads; zero where a projection, column, row or slice does not exist).
template <bool EXACT, int NB>
__device__ __forceinline__ void stage_geometry(const Params &P, float *geo, int s, int i0, int j0, int k0, int kmax,
                                               const uint32_t *gdesc)
{
    if constexpr (EXACT) {
        const size_t zstride = static_cast<size_t>(P.nv) * 3, xstride = static_cast<size_t>(P.nu) * 3;
        for (int idx = threadIdx.x; idx < NB * GEO_EXACT; idx += THREADS) {
            const uint32_t d = gdesc[idx];
            const uint32_t arr = (d >> 26) & 3;
            const int p = s * NB + static_cast<int>(d >> 28);
            const bool ok = arr != 3 && p < P.nproj;
            const float *base = arr == 0 ? P.zip : arr == 1 ? P.xip : P.yip;
            const float *src = base + (d & 0x3FFFFFFu) + static_cast<size_t>(p) * (arr == 0 ? zstride : xstride);
            copy4_zfill(geo + idx, ok ? src : P.zip, ok);
        }
    } else {
        const float *maps = reinterpret_cast<const float *>(P.maps); // 24 words per projection
        for (int idx = threadIdx.x; idx < NB * GEO_FAST; idx += THREADS) {
            const int b = idx / GEO_FAST, e = idx % GEO_FAST, p = s * NB + b;
            const bool ok = p < P.nproj && e <= 24;
            const float *src = !ok ? P.scale : e < 24 ? maps + static_cast<size_t>(p) * 24 + e : P.scale + p;
            copy4_zfill(geo + idx, src, ok);
        }
    }
}

// Footprints of batch s's NB projections from its staged geometry (4 projections per producer
// warp, 8 corner lanes each, the same arithmetic as the voxels), then the TMA copies into
// stage st.
template <int DT, bool EXACT, int NB>
__device__ __forceinline__ void issue_batch(const Params &P, const CUtensorMap *tmap, Smem<NB, EXACT ? GEO_EXACT : GEO_FAST, EXACT> &S,
                                            const float *geo, int s, int st, int i0, int j0, int k0, int i_hi, int j_hi,
                                            int kmax)
{
    using T = typename Sample<DT>::T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= NB / 4) return;
    const int b = warp * 4 + (lane >> 3), corner = lane & 7;
    const int p = s * NB + b;
    int rmin = 0, rmax = 0, cmin = 0, cmax = 0;
    bool ok = p < P.nproj;
    if (ok) {
        const int ci = (corner & 1) ? i_hi : i0, cj = (corner & 2) ? j_hi : j0;
        float r, c;
        if constexpr (EXACT) {
            const float *g = geo + b * GEO_EXACT;
            const float *X = g + TK + 3 * (ci - i0), *Y = g + TK + 3 * TI + 3 * (cj - j0);
            const float Z0 = g[TK + 3 * TI + 3 * TJ], Z2 = g[TK + 3 * TI + 3 * TJ + 1];
            const float a1 = __fadd_rn(g[(corner & 4) ? kmax - 1 : 0], Y[1]);
            const float dw = __frcp_rn(__fadd_rn(__fadd_rn(Z2, Y[2]), X[2]));
            r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1, X[1])), 0.5f);
            c = __fadd_rn(__fmul_rn(dw, __fadd_rn(__fadd_rn(Z0, Y[0]), X[0])), 0.5f);
        } else {
            // every lane of the projection forms the tile geometry (same inputs, same values);
            // the first stores it for the voxels
            const float *g = geo + b * GEO_FAST;
            float t[TGEO];
            ok = tile_geometry(reinterpret_cast<const double *>(g), i0, j0, k0, g[24], t);
            if (corner == 0) {
#pragma unroll
                for (int e = 0; e < TGEO; ++e) S.tg[(st * NB + b) * TGEO + e] = t[e];
            }
            float dw, tc, tr0, dr;
            fast_coord(t, static_cast<float>(ci - i0), static_cast<float>(cj - j0), dw, tc, tr0, dr);
            c = tc;
            r = (corner & 4) ? fmaf(static_cast<float>(kmax - 1), dr, tr0) : tr0;
            ok = ok && dw > 0.0f && fabsf(r) < 4.0e6f && fabsf(c) < 4.0e6f;
            if (ok) {
                // footprint in detector pixels: integer part + floor of the fraction
                rmin = rmax = __float_as_int(t[TG_R0]) + __float2int_rd(r);
                cmin = cmax = __float_as_int(t[TG_C0]) + __float2int_rd(c);
            }
        }
        if constexpr (EXACT) {
            ok = ok && fabsf(r) < 4.0e6f && fabsf(c) < 4.0e6f;
            rmin = rmax = ok ? __float2int_rd(r) : 0;
            cmin = cmax = ok ? __float2int_rd(c) : 0;
        }
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
    const bool unfit = __ballot_sync(0xffffffffu, corner == 0 && p < P.nproj && mode == 0) != 0; // this warp's group
    if (lane == 0) mbar_expect_tx(&S.bars[st], static_cast<uint32_t>(__popc(staged)) * P.bw * P.bh * sizeof(T));
    __syncwarp();
    if (corner == 0 && p < P.nproj) {
        S.meta[st * NB + b] = make_int4(x0, y0, mode, (b & 3) == 0 && unfit);
        if (mode == 1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tma_load_3d(S.stage + (st * NB + b) * P.boxbytes, tmap, x0, y0, p, &S.bars[st]);
        }
    }
}

template <int DT, bool EXACT, int NB>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) k_fdk_staged(const __grid_constant__ CUtensorMap tmap, const Params P)
{
    constexpr int GEO = EXACT ? GEO_EXACT : GEO_FAST;
    using T = typename Sample<DT>::T;
    extern __shared__ __align__(1024) unsigned char smem[];
    Smem<NB, GEO, EXACT> S(smem, P.boxbytes);
    const uint32_t stage_bytes = static_cast<uint32_t>(2 * NB * P.boxbytes);
    (void)stage_bytes;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ, k0 = P.kbegin + blockIdx.z * TK;
    const int i = i0 + lane, j = j0 + warp;
    const int kmax = min(TK, P.kend - k0);
    const bool valid = i < P.nu && j < P.nu;
    const bool inside = valid && static_cast<uint32_t>(i) > P.mask[2 * j] && static_cast<uint32_t>(i) <= P.mask[2 * j + 1];
    const size_t plane = static_cast<size_t>(P.nu) * P.nu;
    const size_t out_xy = valid ? static_cast<size_t>(j) * P.nu + (P.nu - 1 - i) : 0;

    // 16-bit storage: weights are scaled by 2^-G (G = largest scale exponent), the sum by 2^G
    float gscale = 1.0f, ginv = 1.0f;
    if constexpr (!EXACT && DT == MR_F16) {
        float mx = 0.0f;
        for (int p = threadIdx.x; p < P.nproj; p += THREADS) mx = fmaxf(mx, P.scale[p]);
        mx = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mx))); // non-negative floats order as integers
        __shared__ float wmax[NWARPS];
        if (lane == 0) wmax[warp] = mx;
        __syncthreads();
        mx = 0.0f;
#pragma unroll
        for (int w = 0; w < NWARPS; ++w) mx = fmaxf(mx, wmax[w]);
        if (mx > 0.0f) {
            gscale = mx;            // a power of two
            ginv = 1.0f / mx;       // exact
        }
    }

    // slices 2q, 2q+1 of the column in acc[q].x, acc[q].y
    float2 acc[TK / 2];
#pragma unroll
    for (int q = 0; q < TK; ++q) {
        const float v = (valid && P.accumulate && q < kmax)
                            ? P.vol[static_cast<size_t>(P.nv - 1 - (k0 + q)) * plane + out_xy] * ginv
                            : 0.0f;
        if (q & 1) acc[q >> 1].y = v; else acc[q >> 1].x = v;
    }

    auto write_out = [&]() {
        if (valid) {
#pragma unroll
            for (int q = 0; q < TK; ++q)
                if (q < kmax)
                    P.vol[static_cast<size_t>(P.nv - 1 - (k0 + q)) * plane + out_xy] =
                        ((q & 1) ? acc[q >> 1].y : acc[q >> 1].x) * gscale;
        }
    };

    if (!__syncthreads_or(inside)) {
        write_out();
        return;
    }

    if (threadIdx.x == 0) {
        mbar_init(&S.bars[0], NB / 4);
        mbar_init(&S.bars[1], NB / 4);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int i_hi = min(i0 + TI - 1, P.nu - 1), j_hi = min(j0 + TJ - 1, P.nu - 1);
    const int nbatch = (P.nproj + NB - 1) / NB;

    // geometry of batches 0-2, footprints and copies of batches 0-1
    if constexpr (EXACT) {
        geometry_sources<NB>(P, S.gdesc, i0, j0, k0, kmax);
        __syncthreads();
    }
    for (int s = 0; s < 3 && s < nbatch; ++s)
        stage_geometry<EXACT, NB>(P, S.geo + s * NB * GEO, s, i0, j0, k0, kmax, S.gdesc);
    copy_wait_all();
    __syncthreads();
    for (int s = 0; s < 2 && s < nbatch; ++s)
        issue_batch<DT, EXACT, NB>(P, &tmap, S, S.geo + s * NB * GEO, s, s, i0, j0, k0, i_hi, j_hi, kmax);
    __syncthreads();

    uint32_t phase0 = 0, phase1 = 0;
    bool failed = false;
    const float fw = static_cast<float>(P.nu), fh = static_cast<float>(P.nv);
    const float fdi = static_cast<float>(lane), fdj = static_cast<float>(warp); // voxel offset in the tile
    const uint32_t rowbytes = static_cast<uint32_t>(P.rowbytes);
    const bool warp_inside = __any_sync(0xffffffffu, inside);
    int s = 0;
    for (int gb = 0; s < nbatch; ++s, gb = gb == 2 ? 0 : gb + 1) {
        const int st = s & 1;  // stage buffer
        const float *geo = S.geo + gb * NB * GEO; // geometry buffer s % 3
        const uint32_t par = st ? phase1 : phase0;
        // a wait that timed out skips the batch in its whole warp; the block then leaves the
        // loop together at the barrier below
        const bool got = __all_sync(0xffffffffu, mbar_wait(&S.bars[st], par, P.wait_limit));
        if (got) {
            if (st) phase1 ^= 1; else phase0 ^= 1;
        } else {
            failed = true;
            if (lane == 0) atomicExch(&g_device_error, 1);
        }

        if constexpr (EXACT) {
            // per-warp slice sums a1[k] = zip1[k] + yip1[j] (lane = slice)
            if (got && warp_inside) {
                for (int idx = lane; idx < NB * TK; idx += 32) {
                    const float *g = geo + (idx / TK) * GEO_EXACT;
                    S.a1[warp * NB * TK + idx] = __fadd_rn(g[idx % TK], g[TK + 3 * TI + 3 * warp + 1]);
                }
                if (lane < NB) { // the warp-uniform first sums of the set-up: (Z0 + y0), (Z2 + y2)
                    const float *g = geo + lane * GEO_EXACT;
                    S.zy[warp * NB + lane] = make_float2(__fadd_rn(g[TK + 3 * TI + 3 * TJ], g[TK + 3 * TI + 3 * warp]),
                                                         __fadd_rn(g[TK + 3 * TI + 3 * TJ + 1], g[TK + 3 * TI + 3 * warp + 2]));
                }
                __syncwarp();
            }
        }
        if (got && inside) {
            // projections in groups of G: the per-projection set-up of a group (reciprocal,
            // detector column, shared-memory base) is formed first, so its latency overlaps
            // per-projection set-up of this voxel column: false when the projection adds
            // nothing here or is not staged (exact: dw, dw^2, x1; fast: row fraction, row
            // step, weight bits; base: shared-memory address of row 0 in magic-bit form)
            auto setup = [&](int b, float &qa, float &qb, float &qc, uint32_t &qbase) -> bool {
                const int p = s * NB + b;
                const int4 m = S.meta[st * NB + b];
                const uint32_t boxoff = static_cast<uint32_t>((st * NB + b) * P.boxbytes);
                qa = qb = qc = 0.0f;
                qbase = 0;
                if (p >= P.nproj || m.z != 1) return false;
                if constexpr (EXACT) {
                    const float *g = geo + b * GEO;
                    const float x0f = g[TK + 3 * lane], x1f = g[TK + 3 * lane + 1], x2f = g[TK + 3 * lane + 2];
                    const float2 zy = S.zy[warp * NB + b];
                    const float dw = __frcp_rn(__fadd_rn(zy.y, x2f));
                    const float c = __fadd_rn(__fmul_rn(dw, __fadd_rn(zy.x, x0f)), 0.5f);
                    const int cc = static_cast<int>(c);
                    qa = dw;
                    qb = __fmul_rn(dw, dw);
                    qc = x1f;
                    // bits(r + magic) * rowbytes + base = (floor(r) - y0) * rowbytes + (cc - x0) * 4 + box
                    qbase = boxoff + static_cast<uint32_t>(cc - m.x) * 4u - static_cast<uint32_t>(kMagicBits + m.y) * rowbytes;
                    return c >= 0.0f && c < fw;
                } else {
                    float t[TGEO]; // the tile geometry, four vector loads
#pragma unroll
                    for (int e = 0; e < TGEO / 4; ++e) {
                        const float4 t4 = reinterpret_cast<const float4 *>(S.tg + (st * NB + b) * TGEO)[e];
                        t[4 * e] = t4.x;
                        t[4 * e + 1] = t4.y;
                        t[4 * e + 2] = t4.z;
                        t[4 * e + 3] = t4.w;
                    }
                    float dw, tc, tr0, dr;
                    fast_coord(t, fdi, fdj, dw, tc, tr0, dr);
                    const int cc = __float_as_int(__fadd_rd(tc, kMagic)) - kMagicBits + __float_as_int(t[TG_C0]);
                    qa = tr0;
                    qb = dr;
                    qc = __uint_as_float(to_storage<DT>(dw * dw * (t[TG_SCALE] * ginv)));
                    // bits(t + magic) * rowbytes + base = (r0 + floor(t) - y0) * rowbytes + ...
                    qbase = boxoff + static_cast<uint32_t>(cc - m.x) * 2u -
                            static_cast<uint32_t>(kMagicBits + m.y - __float_as_int(t[TG_R0])) * rowbytes;
                    return true;
                }
            };
            constexpr int G = 4;
#pragma unroll 1
            for (int b0 = 0; b0 < NB; b0 += G) {
                float q_a[G], q_b[G], q_c[G];
                uint32_t q_base[G];
                bool q_on[G];
#pragma unroll
                for (int e = 0; e < G; ++e) q_on[e] = setup(b0 + e, q_a[e], q_b[e], q_c[e], q_base[e]);
                // a footprint that did not fit its box (rare; uniform over the CTA) sends the
                // whole group through the in-order path below, so that every voxel still sums
                // its projections in the reference's order
                static_assert(G == 4, "groups of four projections are the producer warps' groups");
                const bool fallback = S.meta[st * NB + b0].w != 0;
                if (!fallback) {
#pragma unroll
                    for (int e = 0; e < G; ++e) {
                        if (!q_on[e]) continue;
                        if constexpr (EXACT) {
                            const float *a1 = S.a1 + (warp * NB + b0 + e) * TK;
                            if (kmax == TK)
                                exact_column<true>(acc, smem, q_base[e], rowbytes, a1, q_c[e], q_a[e], q_b[e], kmax,
                                                   stage_bytes);
                            else
                                exact_column<false>(acc, smem, q_base[e], rowbytes, a1, q_c[e], q_a[e], q_b[e], kmax,
                                                    stage_bytes);
                        } else {
                            const unsigned short wt = static_cast<unsigned short>(__float_as_uint(q_c[e]));
                            if (kmax == TK)
                                fast_column_staged<DT, true>(acc, smem, q_base[e], rowbytes, q_a[e], q_b[e], wt, kmax);
                            else
                                fast_column_staged<DT, false>(acc, smem, q_base[e], rowbytes, q_a[e], q_b[e], wt, kmax);
                        }
                    }
                    continue;
                }
                // in order: staged footprints from shared memory, the others by guarded global loads
#pragma unroll 1
                for (int e = 0; e < G; ++e) {
                    const int b = b0 + e, p = s * NB + b;
                    float qa, qb, qc;
                    uint32_t qbase;
                    if (setup(b, qa, qb, qc, qbase)) { // set-up formed again: no indexed arrays
                        if constexpr (EXACT)
                            exact_column<false>(acc, smem, qbase, rowbytes, S.a1 + (warp * NB + b) * TK, qc, qa, qb, kmax,
                                                stage_bytes);
                        else
                            fast_column_staged<DT, false>(acc, smem, qbase, rowbytes, qa, qb,
                                                          static_cast<unsigned short>(__float_as_uint(qc)), kmax);
                        continue;
                    }
                    if (p >= P.nproj || S.meta[st * NB + b].z != 0) continue;
                    const float *g = geo + b * GEO;
                    if constexpr (EXACT) {
                        const float x0f = g[TK + 3 * lane], x1f = g[TK + 3 * lane + 1], x2f = g[TK + 3 * lane + 2];
                        const float y0f = g[TK + 3 * TI + 3 * warp], y2f = g[TK + 3 * TI + 3 * warp + 2];
                        const float Z0 = g[TK + 3 * TI + 3 * TJ], Z2 = g[TK + 3 * TI + 3 * TJ + 1];
                        const float dw = __frcp_rn(__fadd_rn(__fadd_rn(Z2, y2f), x2f));
                        const float c = __fadd_rn(__fmul_rn(dw, __fadd_rn(__fadd_rn(Z0, y0f), x0f)), 0.5f);
                        if (c < 0.0f || c >= fw) continue;
                        const float dw2 = __fmul_rn(dw, dw);
                        const float *a1 = S.a1 + (warp * NB + b) * TK;
                        const float *img = static_cast<const float *>(P.proj) + static_cast<size_t>(p) * P.nu * P.nv +
                                           static_cast<int>(c);
#pragma unroll
                        for (int q = 0; q < TK; ++q) {
                            if (q >= kmax) break;
                            const float r = __fadd_rn(__fmul_rn(dw, __fadd_rn(a1[q], x1f)), 0.5f);
                            if (r < 0.0f || r >= fh) continue;
                            const float v = __ldg(img + static_cast<size_t>(static_cast<int>(r)) * P.nu);
                            float &a = (q & 1) ? acc[q >> 1].y : acc[q >> 1].x;
                            a = __fadd_rn(a, __fmul_rn(dw2, v));
                        }
                    } else {
                        const float *t = S.tg + (st * NB + b) * TGEO;
                        float dw, tc, tr0, dr;
                        fast_coord(t, fdi, fdj, dw, tc, tr0, dr);
                        const int col = __float_as_int(t[TG_C0]) + __float2int_rd(tc);
                        if (col < 0 || col >= P.nu) continue;
                        const unsigned short wt = to_storage<DT>(dw * dw * (t[TG_SCALE] * ginv));
                        const T *img = static_cast<const T *>(P.proj) + static_cast<size_t>(p) * P.nu * P.nv + col;
                        const float wf = from_storage<DT>(wt);
                        const int r0 = __float_as_int(t[TG_R0]);
                        float2 rr = make_float2(tr0, __fadd_rn(tr0, dr));
                        const float2 step = make_float2(2.0f * dr, 2.0f * dr);
#pragma unroll
                        for (int q = 0; q < TK; ++q) {
                            if (q >= kmax) break;
                            // the rows of the staged loop: pairs advanced by 2 dr
                            const int row = r0 + __float2int_rd((q & 1) ? rr.y : rr.x);
                            if (q & 1) rr = __fadd2_rn(rr, step);
                            if (row < 0 || row >= P.nv) continue;
                            const unsigned short v = reinterpret_cast<const unsigned short *>(img)[static_cast<size_t>(row) * P.nu];
                            float &a = (q & 1) ? acc[q >> 1].y : acc[q >> 1].x;
                            a = fmaf(from_storage<DT>(v), wf, a);
                        }
                    }
                }
            }
        }
        // batch s+2's geometry (in flight since batch s-1) complete and published; stage st and
        // geometry buffer gb free
        copy_wait_all();
        if (__syncthreads_or(failed)) break;
        if (s + 2 < nbatch) {
            const int g2 = gb == 0 ? 2 : gb - 1;
            issue_batch<DT, EXACT, NB>(P, &tmap, S, S.geo + g2 * NB * GEO, s + 2, st, i0, j0, k0, i_hi, j_hi, kmax);
        }
        if (s + 3 < nbatch) stage_geometry<EXACT, NB>(P, S.geo + gb * NB * GEO, s + 3, i0, j0, k0, kmax, S.gdesc);
    }
    if (failed) {
        // copies still in flight: batch s (its wait expired) and batch s+1 when it was issued;
        // wait for them (bounded) before the block's shared memory is released
        const int st = s & 1;
        mbar_wait(&S.bars[st], st ? phase1 : phase0);
        if (s + 1 < nbatch) mbar_wait(&S.bars[st ^ 1], st ? phase0 : phase1);
    }
    write_out();
}

// ---------------------------------------------------------------- FP64 error oracle

// FP64 backprojection of FP32 filtered projections through the FP64 maps, for the listed
// output slices (out[s][j][i] = final volume slice slices[s]). One thread per voxel column.
__global__ void k_fdk_f64(const float *__restrict__ proj, int nu, int nv, int nproj, const double *__restrict__ maps,
                          const uint32_t *__restrict__ mask, const int *__restrict__ slices, int nslices,
                          double *__restrict__ out)
{
    constexpr int MAXS = 16;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nu || j >= nu) return;
    double acc[MAXS];
    int ks[MAXS];
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
        acc[s] = 0.0;
        ks[s] = s < nslices ? nv - 1 - slices[s] : 0;
    }
    const bool inside = static_cast<uint32_t>(i) > mask[2 * j] && static_cast<uint32_t>(i) <= mask[2 * j + 1];
    if (inside) {
        const double di = i, dj = j;
        for (int p = 0; p < nproj; ++p) {
            const double *m = maps + static_cast<size_t>(p) * 12;
            const float *img = proj + static_cast<size_t>(p) * nu * nv;
#pragma unroll
            for (int s = 0; s < MAXS; ++s) {
                if (s >= nslices) break;
                const double dk = ks[s];
                const double u = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], di), __dmul_rn(m[1], dj)), __dmul_rn(m[2], dk)), m[3]);
                const double v = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[4], di), __dmul_rn(m[5], dj)), __dmul_rn(m[6], dk)), m[7]);
                const double w = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[8], di), __dmul_rn(m[9], dj)), __dmul_rn(m[10], dk)), m[11]);
                const double dw = __ddiv_rn(1.0, w);
                const double r = __dadd_rn(__dmul_rn(dw, v), 0.5), c = __dadd_rn(__dmul_rn(dw, u), 0.5);
                if (r < 0.0 || r >= nv || c < 0.0 || c >= nu) continue;
                const double val = img[static_cast<size_t>(static_cast<int>(r)) * nu + static_cast<int>(c)];
                acc[s] = __dadd_rn(acc[s], __dmul_rn(__dmul_rn(dw, dw), val));
            }
        }
    }
#pragma unroll
    for (int s = 0; s < MAXS; ++s)
        if (s < nslices) out[(static_cast<size_t>(s) * nu + j) * nu + (nu - 1 - i)] = acc[s];
}

// ---------------------------------------------------------------- host side

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

static void tile_footprint_maps(const double *m, int i0, int i1, int j0, int j1, int k0, int k1, double &rspan,
                                double &cspan)
{
    double rmin = 1e30, rmax = -1e30, cmin = 1e30, cmax = -1e30;
    for (int corner = 0; corner < 8; ++corner) {
        const double i = corner & 1 ? i1 : i0, j = corner & 2 ? j1 : j0, k = corner & 4 ? k1 : k0;
        const double dw = 1.0 / (m[8] * i + m[9] * j + m[10] * k + m[11]);
        const double r = dw * (m[4] * i + m[5] * j + m[6] * k + m[7]) + 0.5;
        const double c = dw * (m[0] * i + m[1] * j + m[2] * k + m[3]) + 0.5;
        rmin = std::min(rmin, r);
        rmax = std::max(rmax, r);
        cmin = std::min(cmin, c);
        cmax = std::max(cmax, c);
    }
    rspan = std::floor(rmax) - std::floor(rmin);
    cspan = std::floor(cmax) - std::floor(cmin);
}

// Largest footprint over a sample of tiles and projections -> box (bw, bh).
template <typename F>
static void box_guess(size_t nu, size_t nv, size_t nproj, int xalign, int &bw, int &bh, F footprint)
{
    double rs = 0, cs = 0;
    const int ti = static_cast<int>((nu + TI - 1) / TI), tj = static_cast<int>((nu + TJ - 1) / TJ);
    const int tk = static_cast<int>((nv + TK - 1) / TK);
    const size_t pstep = std::max<size_t>(1, nproj / 64);
    const int istep = std::max(1, ti / 8), jstep = std::max(1, tj / 16);
    for (size_t p = 0; p < nproj; p += pstep)
        for (int a = 0; a < ti; a += (a + istep < ti ? istep : std::max(1, ti - 1 - a)))
            for (int b = 0; b < tj; b += (b + jstep < tj ? jstep : std::max(1, tj - 1 - b)))
                for (int kk : {0, tk - 1}) {
                    const int i0 = a * TI, j0 = b * TJ, k0 = kk * TK;
                    double r, c;
                    footprint(p, i0, std::min<int>(i0 + TI - 1, static_cast<int>(nu) - 1), j0,
                              std::min<int>(j0 + TJ - 1, static_cast<int>(nu) - 1), k0,
                              std::min<int>(k0 + TK - 1, static_cast<int>(nv) - 1), r, c);
                    rs = std::max(rs, r);
                    cs = std::max(cs, c);
                }
    // +1 margin each side, +1 for the inclusive range, + alignment slack on x
    bw = static_cast<int>(cs) + 3 + (xalign - 1);
    bh = static_cast<int>(rs) + 3;
    bw = (bw + xalign - 1) / xalign * xalign;
    bw = std::min(bw, 256);
    bh = std::min(bh, 256);
}

} // namespace fdk2

// Launches a staged FDK kernel; returns MR_ERR_UNSUPPORTED when the layout does not allow
// TMA or the box does not fit shared memory (the caller then uses the plain kernel).
static mr_status staged_launch(bool exact, const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                               size_t nproj, const float *xip_d, const float *yip_d, const float *zip_d,
                               const double *maps_d, const uint32_t *mask_d, int accumulate, int kbegin, int kend,
                               float *vol_d, int bw,
                               int bh, cudaStream_t s)
{
    using namespace fdk2;
    const size_t es = dtype == MR_F32 ? 4 : 2;
    const int xalign = static_cast<int>(16 / es);
    if ((nu * es) % 16 != 0 || (reinterpret_cast<uintptr_t>(proj_d) % 16) != 0) return MR_ERR_UNSUPPORTED;
    if (bw <= 0 || bh <= 0 || bw > 256 || bh > 256 || bw % xalign) return MR_ERR_UNSUPPORTED;
    PFN_cuTensorMapEncodeTiled enc = tma::encode_fn();
    if (!enc) return fail(MR_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    constexpr size_t kMaxSmem = (227 * 1024) / CTAS_PER_SM - 1024; // CTAS_PER_SM CTAs per SM
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
    P.maps = maps_d;
    P.mask = mask_d;
    P.vol = vol_d;
    P.nu = static_cast<int>(nu);
    P.nv = static_cast<int>(nv);
    P.nproj = static_cast<int>(nproj);
    P.bw = bw;
    P.bh = bh;
    P.boxbytes = static_cast<int>((bw * bh * es + 127) / 128 * 128);
    P.rowbytes = static_cast<int>(bw * es);
    P.accumulate = accumulate;
    P.kbegin = kbegin;
    P.kend = kend;
    P.xalign = xalign;
    P.wait_limit = tma::g_batch_wait_limit.load();
    dim3 grid(div_up(nu, TI), div_up(nu, TJ), div_up(static_cast<size_t>(kend - kbegin), TK));
    auto go = [&](auto kernel, size_t smem) -> mr_status {
        MR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kMaxSmem)));
        kernel<<<grid, THREADS, smem, s>>>(map, P);
        return check_launch(exact ? "k_fdk_exact" : "k_fdk_fast");
    };
    if (exact) {
        if (dtype != MR_F32) return MR_ERR_UNSUPPORTED;
        const size_t s8 = Smem<8, GEO_EXACT, true>::bytes(P.boxbytes), s4 = Smem<4, GEO_EXACT, true>::bytes(P.boxbytes);
        if (s8 <= kMaxSmem) return go(k_fdk_staged<MR_F32, true, 8>, s8);
        if (s4 <= kMaxSmem) return go(k_fdk_staged<MR_F32, true, 4>, s4);
        return MR_ERR_UNSUPPORTED;
    }
    const size_t s8 = Smem<8, GEO_FAST, false>::bytes(P.boxbytes), s4 = Smem<4, GEO_FAST, false>::bytes(P.boxbytes);
    if (dtype == MR_BF16) {
        if (s8 <= kMaxSmem) return go(k_fdk_staged<MR_BF16, false, 8>, s8);
        if (s4 <= kMaxSmem) return go(k_fdk_staged<MR_BF16, false, 4>, s4);
    } else if (dtype == MR_F16) {
        if (s8 <= kMaxSmem) return go(k_fdk_staged<MR_F16, false, 8>, s8);
        if (s4 <= kMaxSmem) return go(k_fdk_staged<MR_F16, false, 4>, s4);
    }
    return MR_ERR_UNSUPPORTED;
}

mr_status fdk_tma_launch(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv, size_t nproj,
                         const float *xip_d, const float *yip_d, const float *zip_d, const uint32_t *mask_d,
                         int accumulate, int kbegin, int kend, float *vol_d, int bw, int bh, cudaStream_t s)
{
    return staged_launch(true, proj_d, dtype, scale_d, nu, nv, nproj, xip_d, yip_d, zip_d, nullptr, mask_d, accumulate,
                         kbegin, kend, vol_d, bw, bh, s);
}

mr_status fdk_box_for(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                      int dtype, int *bw, int *bh)
{
    const int xalign = dtype == MR_F32 ? 4 : 8;
    fdk2::box_guess(nu, nv, nproj, xalign, *bw, *bh,
                    [&](size_t p, int i0, int i1, int j0, int j1, int k0, int k1, double &r, double &c) {
                        fdk2::tile_footprint(xip_h + p * nu * 3, yip_h + p * nu * 3, zip_h + p * nv * 3, i0, i1, j0, j1,
                                             k0, k1, r, c);
                    });
    return MR_OK;
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_fdk_box(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                     int dtype, int *box_w, int *box_h)
{
    MR_TRACE();
    if (!xip_h || !yip_h || !zip_h || !box_w || !box_h) return fail(MR_ERR_ARGUMENT, "mr_fdk_box: null pointer");
    if (dtype != MR_F32 && dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_fdk_box: dtype");
    if (nu == 0 || nv == 0 || nproj == 0) {
        *box_w = *box_h = 0;
        return MR_OK;
    }
    return fdk_box_for(xip_h, yip_h, zip_h, nu, nv, nproj, dtype, box_w, box_h);
}

mr_status mr_fdk_box_maps(const double *maps_h, size_t nu, size_t nv, size_t nproj, int dtype, int *box_w, int *box_h)
{
    MR_TRACE();
    if (!maps_h || !box_w || !box_h) return fail(MR_ERR_ARGUMENT, "mr_fdk_box_maps: null pointer");
    if (dtype != MR_F32 && dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_fdk_box_maps: dtype");
    if (nu == 0 || nv == 0 || nproj == 0) {
        *box_w = *box_h = 0;
        return MR_OK;
    }
    const int xalign = dtype == MR_F32 ? 4 : 8;
    fdk2::box_guess(nu, nv, nproj, xalign, *box_w, *box_h,
                    [&](size_t p, int i0, int i1, int j0, int j1, int k0, int k1, double &r, double &c) {
                        fdk2::tile_footprint_maps(maps_h + p * 12, i0, i1, j0, j1, k0, k1, r, c);
                    });
    return MR_OK;
}

mr_status mr_fdk_backproject_fast(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                                  size_t nproj, const double *maps_d, const uint32_t *mask_d, int box_w, int box_h,
                                  int accumulate, float *vol_d, void *stream)
{
    MR_TRACE();
    if (!proj_d || !scale_d || !maps_d || !mask_d || !vol_d)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_fast: null pointer");
    if (dtype != MR_BF16 && dtype != MR_F16)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_fast: dtype must be MR_BF16 or MR_F16");
    if (nu == 0 || nv == 0 || nu > 65536 || nv > 65536)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_fast: unsupported size");
    if (nproj == 0 || nproj > 0x7fffffff) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_fast: projection count");
    mr_status st = staged_launch(false, proj_d, dtype, scale_d, nu, nv, nproj, nullptr, nullptr, nullptr, maps_d,
                                 mask_d, accumulate, 0, static_cast<int>(nv), vol_d, box_w, box_h, as_stream(stream));
    if (st == MR_ERR_UNSUPPORTED)
        return fail(MR_ERR_UNSUPPORTED,
                    "mr_fdk_backproject_fast: layout or box not supported (row pitch must be a multiple of 16 bytes, "
                    "box from mr_fdk_box_maps)");
    return st;
}

mr_status mr_fdk_backproject_f64(const float *proj_d, size_t nu, size_t nv, size_t nproj, const double *maps_d,
                                 const uint32_t *mask_d, const int *slices_d, size_t nslices, double *out_d,
                                 void *stream)
{
    MR_TRACE();
    if (!proj_d || !maps_d || !mask_d || !slices_d || !out_d)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_f64: null pointer");
    if (nslices == 0 || nslices > 16) return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_f64: 1 to 16 slices");
    if (nu == 0 || nv == 0 || nu > 65536 || nv > 65536 || nproj > 0x7fffffff)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_backproject_f64: unsupported size");
    dim3 grid(div_up(nu, 128), static_cast<unsigned>(nu));
    fdk2::k_fdk_f64<<<grid, 128, 0, as_stream(stream)>>>(proj_d, static_cast<int>(nu), static_cast<int>(nv),
                                                         static_cast<int>(nproj), maps_d, mask_d, slices_d,
                                                         static_cast<int>(nslices), out_d);
    return check_launch("k_fdk_f64");
}

mr_status mr_bounds_status(unsigned long long *first)
{
    MR_TRACE();
    if (!first) return fail(MR_ERR_ARGUMENT, "mr_bounds_status: null pointer");
    unsigned long long w[6] = {};
    int bad = 0;
    bad |= bounds_take_fdk(&w[0]);
    bad |= bounds_take_bp(&w[1]);
    bad |= bounds_take_direct(&w[2]);
    bad |= bounds_take_matched(&w[3]);
    bad |= bounds_take_ring(&w[4]);
    bad |= bounds_take_spot(&w[5]);
    if (bad) return fail(MR_ERR_CUDA, "mr_bounds_status: reading a bounds word failed");
    *first = 0;
    for (unsigned long long v : w)
        if (v) {
            *first = v;
            break;
        }
    return MR_OK;
}

mr_status mr_set_wait_limit(int tries)
{
    tma::g_batch_wait_limit.store(tries < 0 ? tma::kWaitLimit : tries);
    return MR_OK;
}

mr_status mr_device_status(int *status)
{
    MR_TRACE();
    if (!status) return fail(MR_ERR_ARGUMENT, "mr_device_status: null pointer");
    int v = 0, zero = 0;
    MR_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)));
    MR_CUDA_TRY(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)));
    const int b = bp_device_status_take(), m = msc_device_status_take();
    if (b < 0 || m < 0) return fail(MR_ERR_CUDA, "mr_device_status: reading an error word failed");
    *status = v | b | m;
    return MR_OK;
}

} // extern "C"
