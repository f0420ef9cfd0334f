// Differentiation form matched to the parallel-beam backprojector: a forward projector that is
// the exact transpose of MultiProjectionBPparallel's linear-interpolation backprojection
// (MultiProjBPparallel.cpp:39-170), and that backprojection with a per-slice detector centre.
//
// Backprojection (the adjoint), voxel (x, y, z) with 1-based x, y inside the circle mask, every
// projection i (no buffer-drop rule, weight 1):
//     u = (startu[i][z] + cos_i * y) - sin_i * x,   n = (int)u in [0, nu - 2],
//     wb = |u - n|, wa = 1 - wb,   vol[y-1][x-1][z] += P_i[z][n] * wa + P_i[z][n+1] * wb
// with the reference's float operations in its order; startu[i][z] = (nu/2)(sin_i - cos_i) + c_z
// and c_z = centre + tan(tilt) (z - pivot) (the detector centre of slice z). With tilt 0 this is
// the production backprojector bit for bit (mr_bp_parallel with no weights).
//
// Forward projection (the exact transpose): detector bin m of slice z and projection i collects
// wa * vol from every voxel whose n is m and wb * vol from every voxel whose n is m - 1, with the
// same u, n, wa and wb evaluated by the same expressions, so <A x, p> = <x, A^T p> holds to float
// summation. Two kernels: a voxel-driven one (k_mbp_forward_smem, below) while a projection's
// bins for 32 slices fit in shared memory, else a ray-driven one: a warp owns one (i, m) and 32 consecutive slices (lanes), walks the
// volume rows when |sin_i| >= |cos_i| (else the columns) and, in each, only the candidate
// voxels whose u can fall in [m - 1, m + 1): the interval of the affine u, widened by one voxel
// on each side for the float evaluation (u is exact to ~1e-4 pixel, the walk's step is at least
// 1/sqrt(2) pixel). Each candidate's contribution is decided by its own n, as in the adjoint.
// The derivative d proj / d c_z (-vol for the wa term, +vol for the wb term: d wa / du = -1,
// d wb / du = +1, du / dc_z = 1) comes out of the same walk.
#include "mr_common.cuh"
#include "mr_tma.cuh"

#include <cmath>
#include <vector>

namespace mr {

static const float kFPi = 3.1415926535897932384626f;

MR_BOUNDS_TAKE(bounds_take_matched)

// The adjoint with its projection rows staged in shared memory: a CTA owns 32 (x) x 8 (y) voxel
// columns x 32 slices, a thread one column's 32 slices in registers over all projections. For a
// batch of kAdjNB projections the CTA stages, per projection, the detector columns its tile can
// reach in each of its slices: u is affine in x, y and (through the slice centre) z, so its
// truncation is extreme at the tile's corners; the window starts one column before the smallest
// and ends two after the largest (the sample pair n, n + 1 and a column of margin for the
// float rounding), kAdjBW columns at most, else that projection is read from global memory for
// this tile. Rows are copied with cp.async (zero outside the detector), the next batch while
// the current one is summed. Every voxel adds its projections in order with the same float
// operations as the plain kernel: the result is the same bit for bit.
constexpr int kAdjTX = 32, kAdjTY = 8, kAdjTZ = 32, kAdjNB = 8, kAdjBW = 48;
constexpr int kAdjThreads = kAdjTX * kAdjTY;
constexpr int kAdjNoWindow = -0x40000000;

__host__ __device__ constexpr size_t adj_smem_bytes()
{
    return sizeof(float) * (2ull * kAdjNB * kAdjTZ * kAdjBW + 2ull * kAdjNB * kAdjTZ) + sizeof(float2) * 2 * kAdjNB +
           sizeof(int) * 2 * kAdjNB;
}

__global__ void __launch_bounds__(kAdjThreads) k_mbp_adjoint_staged(const float *__restrict__ proj,
                                                                    const float2 *__restrict__ sc,
                                                                    const float *__restrict__ startu, int nproj,
                                                                    int n, int nz, const uint32_t *__restrict__ mask,
                                                                    int accumulate, float *__restrict__ vol)
{
    extern __shared__ __align__(16) float adj_smem[];
    float *box = adj_smem;                                   // [2][NB][TZ][BW]
    float *sus = box + 2 * kAdjNB * kAdjTZ * kAdjBW;         // [2][NB][TZ] slice start positions
    float2 *scs = reinterpret_cast<float2 *>(sus + 2 * kAdjNB * kAdjTZ); // [2][NB]
    int *win = reinterpret_cast<int *>(scs + 2 * kAdjNB);    // [2][NB] first staged column
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x0 = blockIdx.x * kAdjTX, y0 = blockIdx.y * kAdjTY, z0 = blockIdx.z * kAdjTZ;
    const int x1 = x0 + lane + 1, y1 = y0 + warp + 1; // 1-based voxel
    const bool valid = x1 <= n && y1 <= n;
    const bool inside = valid && static_cast<uint32_t>(x1) > mask[2 * (y1 - 1)] &&
                        static_cast<uint32_t>(x1) <= mask[2 * (y1 - 1) + 1];
    const int zmax = min(kAdjTZ, nz - z0);
    float *col = vol + (static_cast<size_t>(valid ? y1 - 1 : 0) * n + (valid ? x1 - 1 : 0)) * nz + z0;
    float acc[kAdjTZ];
#pragma unroll
    for (int c = 0; c < kAdjTZ; ++c) acc[c] = (accumulate && inside && c < zmax) ? col[c] : 0.0f;
    const int nbatch = (nproj + kAdjNB - 1) / kAdjNB;
    const size_t pstride = static_cast<size_t>(n) * nz;
    const int xa = x0 + 1, xb = min(x0 + kAdjTX, n), ya = y0 + 1, yb = min(y0 + kAdjTY, n);
    // geometry and window of batch b into stage st, then its rows by cp.async
    auto stage = [&](int b, int st) {
        for (int e = threadIdx.x; e < kAdjNB * kAdjTZ; e += kAdjThreads) {
            const int i = b * kAdjNB + e / kAdjTZ, z = z0 + e % kAdjTZ;
            sus[st * kAdjNB * kAdjTZ + e] = (i < nproj && z < nz) ? startu[static_cast<size_t>(i) * nz + z] : 0.0f;
        }
        if (threadIdx.x < kAdjNB) {
            const int i = b * kAdjNB + threadIdx.x;
            scs[st * kAdjNB + threadIdx.x] = i < nproj ? sc[i] : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
        if (warp < kAdjNB) { // warp w: the window of projection w of the batch, lanes 0-7 the corners
            const int i = b * kAdjNB + warp;
            int lo = INT_MAX, hi = INT_MIN;
            if (lane < 8 && i < nproj) {
                const float2 s = scs[st * kAdjNB + warp];
                const float fx = static_cast<float>((lane & 1) ? xb : xa), fy = static_cast<float>((lane & 2) ? yb : ya);
                const float su = sus[st * kAdjNB * kAdjTZ + warp * kAdjTZ + ((lane & 4) ? zmax - 1 : 0)];
                const float u = __fsub_rn(__fadd_rn(su, __fmul_rn(s.y, fy)), __fmul_rn(s.x, fx));
                lo = hi = __float2int_rz(u);
            }
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (lane == 0) win[st * kAdjNB + warp] = (i < nproj && hi + 2 - (lo - 1) < kAdjBW) ? lo - 1 : kAdjNoWindow;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kAdjNB * kAdjTZ * kAdjBW; e += kAdjThreads) {
            const int bb = e / (kAdjTZ * kAdjBW), r = e - bb * kAdjTZ * kAdjBW;
            const int z = r / kAdjBW, c = r - z * kAdjBW;
            const int i = b * kAdjNB + bb, w0 = win[st * kAdjNB + bb];
            const int m = w0 + c;
            const bool ok = w0 != kAdjNoWindow && i < nproj && z < zmax && m >= 0 && m < n;
            const float *src = ok ? proj + static_cast<size_t>(i) * pstride + static_cast<size_t>(z0 + z) * n + m : proj;
            tma::copy4_zfill(box + st * kAdjNB * kAdjTZ * kAdjBW + e, src, ok);
        }
    };
    if (nbatch > 0) stage(0, 0);
    tma::copy_wait_all();
    __syncthreads();
    const float fx = static_cast<float>(x1), fy = static_cast<float>(y1);
    for (int b = 0; b < nbatch; ++b) {
        const int st = b & 1;
        if (b + 1 < nbatch) stage(b + 1, st ^ 1); // its barriers only order the staging
        if (inside) {
            for (int e = 0; e < kAdjNB; ++e) {
                const int i = b * kAdjNB + e;
                if (i >= nproj) break;
                const float2 s = scs[st * kAdjNB + e];
                const float cy = __fmul_rn(s.y, fy), sx = __fmul_rn(s.x, fx);
                const float *su = sus + (st * kAdjNB + e) * kAdjTZ;
                const int w0 = win[st * kAdjNB + e];
                if (w0 != kAdjNoWindow) {
                    const float *bx = box + (st * kAdjNB + e) * kAdjTZ * kAdjBW - w0;
                    // branch-free over the slices: a voxel whose column is off the detector reads
                    // a staged column and keeps its sum (a select, not an added zero)
#pragma unroll
                    for (int c = 0; c < kAdjTZ; ++c) {
                        if (c >= zmax) break;
                        const float u = __fsub_rn(__fadd_rn(su[c], cy), sx);
                        const int m = __float2int_rz(u);
                        const bool ok = m >= 0 && m <= n - 2 && MR_IN_BOUNDS(m - w0 + 1, kAdjBW, kSiteMbpAdjoint);
                        const float wb = fabsf(__fsub_rn(u, static_cast<float>(m)));
                        const float wa = __fsub_rn(1.0f, wb);
                        const float *row = bx + c * kAdjBW + (ok ? m : w0);
                        const float t = __fadd_rn(__fmul_rn(row[0], wa), __fmul_rn(row[1], wb));
                        acc[c] = ok ? __fadd_rn(acc[c], t) : acc[c];
                    }
                } else {
                    const float *img = proj + static_cast<size_t>(i) * pstride + static_cast<size_t>(z0) * n;
#pragma unroll
                    for (int c = 0; c < kAdjTZ; ++c) {
                        if (c >= zmax) break;
                        const float u = __fsub_rn(__fadd_rn(su[c], cy), sx);
                        const int m = __float2int_rz(u);
                        if (m < 0 || m > n - 2) continue;
                        const float wb = fabsf(__fsub_rn(u, static_cast<float>(m)));
                        const float wa = __fsub_rn(1.0f, wb);
                        const float *row = img + static_cast<size_t>(c) * n + m;
                        acc[c] = __fadd_rn(acc[c], __fadd_rn(__fmul_rn(__ldg(row), wa), __fmul_rn(__ldg(row + 1), wb)));
                    }
                }
            }
        }
        // batch b+1's rows have landed; stage st is free for batch b+2
        tma::copy_wait_all();
        __syncthreads();
    }
    if (valid && (inside || !accumulate)) {
#pragma unroll
        for (int c = 0; c < kAdjTZ; ++c)
            if (c < zmax) col[c] = acc[c];
    }
}

// One warp per (projection i, bin m), lanes = 32 consecutive slices from z0.
template <bool DERIV>
__global__ void __launch_bounds__(128) k_mbp_forward(const float *__restrict__ vol, const float2 *__restrict__ sc,
                                                     const float *__restrict__ startu, int nproj, int n, int nz,
                                                     const uint32_t *__restrict__ mask, float *__restrict__ proj,
                                                     float *__restrict__ dproj)
{
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int i = blockIdx.y;
    const int z0 = blockIdx.z * 32, z = z0 + lane;
    if (m >= n) return;
    const bool zok = z < nz;
    const float2 s = sc[i];
    const float *su = startu + static_cast<size_t>(i) * nz;
    const float suz = zok ? su[z] : 0.0f;
    // the warp's extreme start positions (startu is affine in z), for the candidate interval
    const int zl = min(z0 + 31, nz - 1);
    const float sua = fminf(su[z0], su[zl]), sub = fmaxf(su[z0], su[zl]);
    const float fm = static_cast<float>(m);
    float acc = 0.0f, dacc = 0.0f;
    auto visit = [&](int x1, int y1) {
        const float u = __fsub_rn(__fadd_rn(suz, __fmul_rn(s.y, static_cast<float>(y1))), __fmul_rn(s.x, static_cast<float>(x1)));
        const int k = __float2int_rz(u);
        if (k < 0 || k > n - 2 || (k != m && k != m - 1)) return;
        const float wb = fabsf(__fsub_rn(u, static_cast<float>(k)));
        const float v = __ldg(vol + (static_cast<size_t>(y1 - 1) * n + (x1 - 1)) * nz + z);
        if (k == m) {
            acc = __fadd_rn(acc, __fmul_rn(v, __fsub_rn(1.0f, wb)));
            if (DERIV) dacc = __fsub_rn(dacc, v);
        } else {
            acc = __fadd_rn(acc, __fmul_rn(v, wb));
            if (DERIV) dacc = __fadd_rn(dacc, v);
        }
    };
    if (fabsf(s.x) >= fabsf(s.y)) {
        // walk the rows y; in row y, u = (su + cos y) - sin x lies in [m - 1, m + 1) for x in
        // ((su + cos y - m - 1) / sin, (su + cos y - m + 1) / sin] (sin > 0; reversed for sin < 0)
        const float inv = 1.0f / s.x;
        for (int y1 = 1; y1 <= n; ++y1) {
            const uint32_t first = mask[2 * (y1 - 1)], second = mask[2 * (y1 - 1) + 1];
            if (second <= first) continue;
            const float cy = s.y * static_cast<float>(y1);
            const float e0 = (sua + cy - fm - 1.0f) * inv, e1 = (sub + cy - fm + 1.0f) * inv;
            int xa = static_cast<int>(floorf(fminf(e0, e1))) - 1, xb = static_cast<int>(ceilf(fmaxf(e0, e1))) + 1;
            xa = max(xa, static_cast<int>(first) + 1);
            xb = min(xb, static_cast<int>(second));
            if (zok)
                for (int x1 = xa; x1 <= xb; ++x1) visit(x1, y1);
        }
    } else {
        // walk the columns x; u lies in [m - 1, m + 1) for y in
        // ((m - 1 - su + sin x) / cos, (m + 1 - su + sin x) / cos] (cos > 0; reversed otherwise)
        const float inv = 1.0f / s.y;
        for (int x1 = 1; x1 <= n; ++x1) {
            const float sx = s.x * static_cast<float>(x1);
            const float e0 = (fm - 1.0f - sub + sx) * inv, e1 = (fm + 1.0f - sua + sx) * inv;
            int ya = max(static_cast<int>(floorf(fminf(e0, e1))) - 1, 1);
            int yb = min(static_cast<int>(ceilf(fmaxf(e0, e1))) + 1, n);
            if (zok)
                for (int y1 = ya; y1 <= yb; ++y1) {
                    const uint32_t first = mask[2 * (y1 - 1)], second = mask[2 * (y1 - 1) + 1];
                    if (static_cast<uint32_t>(x1) > first && static_cast<uint32_t>(x1) <= second) visit(x1, y1);
                }
        }
    }
    if (zok) {
        const size_t o = (static_cast<size_t>(i) * nz + z) * n + m;
        proj[o] = acc;
        if (DERIV) dproj[o] = dacc;
    }
}

// The same forward projection, voxel-driven (used while the bins fit in shared memory): one CTA
// per (projection i, 32 slices) holds that projection's bins of its slices in shared memory
// (bin-major rows padded to 33 words, so the 32 lanes - one slice each - of a warp hit 32 banks
// and the write-out reads 32 consecutive bins without conflicts). Its warps walk the masked
// voxels line by line, along the axis on which u changes least (x when |sin| <= |cos|, else y;
// |du| <= 1/sqrt(2) per step, so a lane's bin moves by at most one between steps), each voxel
// once, with the adjoint's u, n, wa and wb. A lane keeps the running sums of its current pair of
// bins (n, n + 1) in registers and adds a bin to shared memory (atomically) when its walk leaves
// it, so most voxels cost no shared-memory access. The order of the additions into a bin depends
// on the warps' timing: results agree with the ray-driven kernel to float summation, not bit for
// bit.
constexpr int kFwdPad = 33;
constexpr int kFwdThreads = 1024;

__host__ __device__ inline size_t fwd_smem_bytes(int n, bool deriv)
{
    return static_cast<size_t>(n) * kFwdPad * sizeof(float) * (deriv ? 2 : 1) + static_cast<size_t>(n) * sizeof(uint2) * 2;
}

template <bool DERIV>
struct BinRun {
    int mc = -2; // current bin (-2: none yet)
    float a0 = 0.0f, a1 = 0.0f, d0 = 0.0f, d1 = 0.0f;
    // one voxel: bin m (0 <= m <= n - 2), weights wa, wb, value v
    __device__ __forceinline__ void add(float *bins, float *dbins, int lane, int m, float wa, float wb, float v)
    {
        (void)dbins; // (the derivative bins follow the value bins)
        const float pa = __fmul_rn(v, wa), pb = __fmul_rn(v, wb);
        const int diff = m - mc;
        if (diff == 0) {
            a0 = __fadd_rn(a0, pa);
            a1 = __fadd_rn(a1, pb);
            if (DERIV) {
                d0 = __fsub_rn(d0, v);
                d1 = __fadd_rn(d1, v);
            }
        } else if (diff == -1) { // bin mc + 1 is left behind
            atomicAdd(bins + (mc + 1) * kFwdPad + lane, a1);
            a1 = __fadd_rn(a0, pb);
            a0 = pa;
            if (DERIV) {
                atomicAdd(dbins + (mc + 1) * kFwdPad + lane, d1);
                d1 = __fadd_rn(d0, v);
                d0 = -v;
            }
            mc = m;
        } else if (diff == 1) { // bin mc is left behind
            atomicAdd(bins + mc * kFwdPad + lane, a0);
            a0 = __fadd_rn(a1, pa);
            a1 = pb;
            if (DERIV) {
                atomicAdd(dbins + mc * kFwdPad + lane, d0);
                d0 = __fsub_rn(d1, v);
                d1 = v;
            }
            mc = m;
        } else {
            done(bins, dbins, lane);
            a0 = pa;
            a1 = pb;
            if (DERIV) {
                d0 = -v;
                d1 = v;
            }
            mc = m;
        }
    }
    __device__ __forceinline__ void done(float *bins, float *dbins, int lane) const
    {
        if (mc < 0) return;
        atomicAdd(bins + mc * kFwdPad + lane, a0);
        atomicAdd(bins + (mc + 1) * kFwdPad + lane, a1);
        if (DERIV) {
            atomicAdd(dbins + mc * kFwdPad + lane, d0);
            atomicAdd(dbins + (mc + 1) * kFwdPad + lane, d1);
        }
    }
};

template <bool DERIV>
__global__ void __launch_bounds__(kFwdThreads, 1) k_mbp_forward_smem(const float *__restrict__ vol, const float2 *__restrict__ sc,
                                                                  const float *__restrict__ startu, int nproj, int n,
                                                                  int nz, const uint32_t *__restrict__ mask,
                                                                  float *__restrict__ proj, float *__restrict__ dproj)
{
    extern __shared__ float bins[]; // [n][kFwdPad] (+ [n][kFwdPad] for the derivative), then the masks
    float *dbins = bins + static_cast<size_t>(n) * kFwdPad;
    uint2 *rowmask = reinterpret_cast<uint2 *>(bins + static_cast<size_t>(n) * kFwdPad * (DERIV ? 2 : 1));
    uint2 *colspan = rowmask + n; // per column x: the rows [lo, hi] that hold voxels of it
    const int i = blockIdx.x, z0 = blockIdx.y * 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int z = z0 + lane;
    const bool zok = z < nz;
    for (int e = threadIdx.x; e < n * kFwdPad * (DERIV ? 2 : 1); e += blockDim.x) bins[e] = 0.0f;
    for (int y = threadIdx.x; y < n; y += blockDim.x) rowmask[y] = make_uint2(mask[2 * y], mask[2 * y + 1]);
    const float2 s = sc[i];
    const bool by_rows = fabsf(s.x) <= fabsf(s.y);
    __syncthreads();
    if (!by_rows)
        for (int x = threadIdx.x; x < n; x += blockDim.x) {
            const uint32_t x1 = static_cast<uint32_t>(x) + 1;
            int lo = 0, hi = -1;
            for (int y = 0; y < n; ++y)
                if (x1 > rowmask[y].x && x1 <= rowmask[y].y) {
                    lo = y;
                    break;
                }
            for (int y = n - 1; y >= lo; --y)
                if (x1 > rowmask[y].x && x1 <= rowmask[y].y) {
                    hi = y;
                    break;
                }
            colspan[x] = make_uint2(static_cast<uint32_t>(lo), static_cast<uint32_t>(hi + 1));
        }
    __syncthreads();
    BinRun<DERIV> run;
    const float suz = zok ? startu[static_cast<size_t>(i) * nz + z] : 0.0f;
    if (zok) {
        if (by_rows) {
            // line y: voxels x in (first, second], u = (su + cos y) - sin x
            for (int y = warp; y < n; y += nwarps) {
                const uint2 r = rowmask[y];
                const float a = __fadd_rn(suz, __fmul_rn(s.y, static_cast<float>(y + 1)));
                const float *p = vol + (static_cast<size_t>(y) * n + r.x) * nz + z;
                constexpr int U = 4;
                int x = static_cast<int>(r.x);
                const int xe = min(static_cast<int>(r.y), n);
                for (; x < xe; x += U) {
                    float v[U];
#pragma unroll
                    for (int j = 0; j < U; ++j) v[j] = (x + j < xe) ? __ldg(p + static_cast<size_t>(j) * nz) : 0.0f;
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        if (x + j >= xe) continue;
                        const float u = __fsub_rn(a, __fmul_rn(s.x, static_cast<float>(x + j + 1)));
                        const int m = __float2int_rz(u);
                        if (m < 0 || m > n - 2) continue;
                        const float wb = fabsf(__fsub_rn(u, static_cast<float>(m)));
                        if (!MR_IN_BOUNDS(m + 1, n, kSiteMbpBins)) continue;
                        run.add(bins, dbins, lane, m, __fsub_rn(1.0f, wb), wb, v[j]);
                    }
                    p += static_cast<size_t>(U) * nz;
                }
            }
        } else {
            // line x: voxels y in the column's span that the row masks hold
            for (int x = warp; x < n; x += nwarps) {
                const uint2 span = colspan[x];
                const uint32_t x1 = static_cast<uint32_t>(x) + 1;
                const float sx = __fmul_rn(s.x, static_cast<float>(x1));
                const size_t ystride = static_cast<size_t>(n) * nz;
                const float *p = vol + (static_cast<size_t>(span.x) * n + x) * nz + z;
                constexpr int U = 4;
                int y = static_cast<int>(span.x);
                const int ye = static_cast<int>(span.y);
                for (; y < ye; y += U) {
                    float v[U];
                    bool in[U];
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        in[j] = y + j < ye && x1 > rowmask[y + j].x && x1 <= rowmask[y + j].y;
                        v[j] = in[j] ? __ldg(p + static_cast<size_t>(j) * ystride) : 0.0f;
                    }
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        if (!in[j]) continue;
                        const float u = __fsub_rn(__fadd_rn(suz, __fmul_rn(s.y, static_cast<float>(y + j + 1))), sx);
                        const int m = __float2int_rz(u);
                        if (m < 0 || m > n - 2) continue;
                        const float wb = fabsf(__fsub_rn(u, static_cast<float>(m)));
                        if (!MR_IN_BOUNDS(m + 1, n, kSiteMbpBins)) continue;
                        run.add(bins, dbins, lane, m, __fsub_rn(1.0f, wb), wb, v[j]);
                    }
                    p += static_cast<size_t>(U) * ystride;
                }
            }
        }
        run.done(bins, dbins, lane);
    }
    __syncthreads();
    // write-out: consecutive threads take consecutive bins of one slice (coalesced stores)
    const int zs = min(32, nz - z0);
    for (int e = threadIdx.x; e < zs * n; e += blockDim.x) {
        const int zz = e / n, m = e - zz * n;
        const size_t o = (static_cast<size_t>(i) * nz + z0 + zz) * n + m;
        proj[o] = bins[m * kFwdPad + zz];
        if (DERIV) dproj[o] = dbins[m * kFwdPad + zz];
    }
}

} // namespace mr

using namespace mr;

extern "C" {

mr_status mr_mbp_geometry(const float *angles_h, size_t nproj, size_t n, size_t nz, float centre, float tan_tilt,
                          float pivot, int direction, float *sincos_h, float *startu_h)
{
    MR_TRACE();
    if (nproj && (!angles_h || !sincos_h || !startu_h)) return fail(MR_ERR_ARGUMENT, "mr_mbp_geometry: null pointer");
    if (n < 2) return fail(MR_ERR_ARGUMENT, "mr_mbp_geometry: n must be at least 2");
    // StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:72-79) with the centre of slice z
    const float dirweight = 2.0f * (static_cast<float>(direction) - 0.5f);
    const size_t mcx = n / 2;
    for (size_t k = 0; k < nproj; ++k) {
        const float s = std::sin(dirweight * angles_h[k] * kFPi / 180.0f);
        const float c = std::cos(dirweight * angles_h[k] * kFPi / 180.0f);
        sincos_h[2 * k] = s;
        sincos_h[2 * k + 1] = c;
        for (size_t z = 0; z < nz; ++z) {
            const float cz = centre + tan_tilt * (static_cast<float>(z) - pivot);
            startu_h[k * nz + z] = mcx * (s - c) + cz;
        }
    }
    return MR_OK;
}

mr_status mr_mbp_adjoint(const float *proj_d, size_t n, size_t nz, const float *sincos_d, const float *startu_d,
                         size_t nproj, const uint32_t *mask_d, int accumulate, float *vol_d, void *stream)
{
    MR_TRACE();
    if (!proj_d || !sincos_d || !startu_d || !mask_d || !vol_d) return fail(MR_ERR_ARGUMENT, "mr_mbp_adjoint: null pointer");
    if (n < 2 || n > 65536 || nz == 0 || nz > 65536 || nproj > 0x7fffffff)
        return fail(MR_ERR_ARGUMENT, "mr_mbp_adjoint: unsupported size");
    static bool attr = false;
    if (!attr) {
        MR_CUDA_TRY(cudaFuncSetAttribute(k_mbp_adjoint_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(adj_smem_bytes())));
        attr = true;
    }
    dim3 grid(div_up(n, kAdjTX), div_up(n, kAdjTY), div_up(nz, kAdjTZ));
    k_mbp_adjoint_staged<<<grid, kAdjThreads, adj_smem_bytes(), as_stream(stream)>>>(
        proj_d, reinterpret_cast<const float2 *>(sincos_d), startu_d, static_cast<int>(nproj), static_cast<int>(n),
        static_cast<int>(nz), mask_d, accumulate, vol_d);
    return check_launch("k_mbp_adjoint_staged");
}

mr_status mr_mbp_forward(const float *vol_d, size_t n, size_t nz, const float *sincos_d, const float *startu_d,
                         size_t nproj, const uint32_t *mask_d, float *proj_d, float *dproj_d, void *stream)
{
    MR_TRACE();
    if (!vol_d || !sincos_d || !startu_d || !mask_d || !proj_d) return fail(MR_ERR_ARGUMENT, "mr_mbp_forward: null pointer");
    if (n < 2 || n > 65536 || nz == 0 || nz > 65536 || nproj == 0 || nproj > 65535)
        return fail(MR_ERR_ARGUMENT, "mr_mbp_forward: unsupported size");
    const float2 *sc = reinterpret_cast<const float2 *>(sincos_d);
    int dev = 0, optin = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem = fwd_smem_bytes(static_cast<int>(n), dproj_d != nullptr);
    if (smem <= static_cast<size_t>(optin)) {
        dim3 sgrid(static_cast<unsigned>(nproj), div_up(nz, 32));
        auto launch = [&](auto kernel, float *d) -> mr_status {
            MR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
            kernel<<<sgrid, kFwdThreads, smem, as_stream(stream)>>>(vol_d, sc, startu_d, static_cast<int>(nproj),
                                                                   static_cast<int>(n), static_cast<int>(nz), mask_d,
                                                                   proj_d, d);
            return check_launch("k_mbp_forward_smem");
        };
        return dproj_d ? launch(k_mbp_forward_smem<true>, dproj_d) : launch(k_mbp_forward_smem<false>, nullptr);
    }
    // bins beyond shared memory: the ray-driven kernel
    dim3 grid(div_up(n, 4), static_cast<unsigned>(nproj), div_up(nz, 32));
    if (dproj_d)
        k_mbp_forward<true><<<grid, 128, 0, as_stream(stream)>>>(vol_d, reinterpret_cast<const float2 *>(sincos_d),
                                                               startu_d, static_cast<int>(nproj), static_cast<int>(n),
                                                               static_cast<int>(nz), mask_d, proj_d, dproj_d);
    else
        k_mbp_forward<false><<<grid, 128, 0, as_stream(stream)>>>(vol_d, reinterpret_cast<const float2 *>(sincos_d),
                                                                startu_d, static_cast<int>(nproj), static_cast<int>(n),
                                                                static_cast<int>(nz), mask_d, proj_d, nullptr);
    return check_launch("k_mbp_forward");
}

} // extern "C"
