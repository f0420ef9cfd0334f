// MorphSpotClean (replace mode) on the GPU.
//
// Reference: core/algorithms/ImagingAlgorithms/src/MorphSpotClean.cpp:41-175,264-351 with the
// grey-scale reconstructions of core/kipl/kipl/include/morphology/morphgeo.h:151-371 and the
// markers of morphextrema.h:265-328.
//
// Per image: optional inf/NaN replacement and clamping; padding by 5 (zero columns, the
// first/last 5 rows mirrored) and an in-place sliding median along the first and last
// padded rows (sequential, one thread per edge row, as the reference's loop); the
// reconstructions; threshold replacement or sigmoid blend; unpadding.
//
// Reconstructions. FillHole (erosion) and the dual FillPeaks of the 'both' mode are
// textbook reconstructions, unique fixpoints of min/max operations, so any order of
// monotone updates reaches exactly the reference's result. FillPeaks (peaks mode) runs
// RecByDilation, whose forward raster scan compares the running image but assigns the
// marker value (morphgeo.h:213-214); after that scan the reference computes the exact
// reconstruction of the scanned marker. The scanned marker differs from the initial one
// only on the border and on pixels with a border pixel among their backward neighbours
// (every other value stays the marker's interior minimum), so one thread per image replays
// the scan over that band in raster order, and the exact reconstruction follows.
//
// Each reconstruction runs in two kernels, one CTA per image in both. The sweep kernel
// alternates downward and upward row sweeps for a few rounds (it stops early when a round
// changes nothing). A sweep combines each row with the neighbouring row just finished
// (vertical and, for 8-connectivity, diagonal neighbours), then propagates along the row in
// both directions with a CTA-wide scan: the row update v[c] = min(g[c], max(v[c], v[c-1]))
// (dilation) or max(g[c], min(v[c], v[c-1])) (erosion) is a clamp x -> min(hi, max(lo, x)),
// and clamps compose into clamps, so the sequential recurrence is a parallel prefix. On noisy
// projections the sweeps alone need 20-30 rounds (every change of vertical direction along a
// propagation path costs a round), while after a few rounds only a thin set of pixels still
// changes; the completion kernel finishes from there with a worklist (k_complete).
#include "mr_common.cuh"

#include <cfloat>
#include <climits>
#include <cmath>
#include <type_traits>

namespace mr {

// Error word of this file's bounded loops (device globals are per translation unit without
// relocatable device code); mr_device_status reads and clears it with the other kernels' words.
__device__ int g_msc_error = 0;

MR_BOUNDS_TAKE(bounds_take_spot)

int msc_device_status_take()
{
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_msc_error, sizeof(int)) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(g_msc_error, &zero, sizeof(int)) != cudaSuccess) return -1;
    return v;
}

namespace msc {

constexpr int kMargin = 5;
constexpr int kSweepRounds = 3; // dense sweep rounds before the worklist completion (2-6 measured: 3 is fastest)
constexpr int kMaxEdge = 63;

struct Clamp {
    float lo, hi;
};

// g2 after g1 (apply g1 first).
__device__ __forceinline__ Clamp compose(const Clamp g1, const Clamp g2)
{
    return Clamp{fminf(fmaxf(g1.lo, g2.lo), g2.hi), fminf(fmaxf(g1.hi, g2.lo), g2.hi)};
}

// ---- preparation

__global__ void k_finite_max(const float *__restrict__ img, size_t per, float *__restrict__ out)
{
    const float *p = img + blockIdx.x * per;
    float m = -FLT_MAX;
    for (size_t i = threadIdx.x; i < per; i += blockDim.x)
        if (isfinite(p[i]) && m < p[i]) m = p[i];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x + 31) / 32 ? s[threadIdx.x] : -FLT_MAX;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) out[blockIdx.x] = m;
    }
}

// Padded image (MorphSpotClean::PadEdges :264-281) after replaceInfNaN (:514-536) and
// LimitDynamics (core/kipl/kipl/include/segmentation/thresholds.h:60-85).
__global__ void k_pad(const float *__restrict__ img, int w, int h, const float *__restrict__ finite_max, int clamp,
                      float lo, float hi, float *__restrict__ pad)
{
    const int pw = w + 2 * kMargin, ph = h + 2 * kMargin;
    const size_t n = static_cast<size_t>(pw) * ph;
    const int b = blockIdx.y;
    const float *src = img + static_cast<size_t>(b) * w * h;
    float *dst = pad + b * n;
    (void)n;
    for (int y = blockIdx.x; y < ph; y += gridDim.x) {
        int sy = y - kMargin;
        if (sy < 0) sy = -1 - sy;              // padded row m-1-i <- image row i
        else if (sy >= h) sy = 2 * h - 1 - sy; // padded row ph-m+i <- image row h-1-i
        const float *srow = src + static_cast<size_t>(sy) * w;
        float *drow = dst + static_cast<size_t>(y) * pw;
        for (int xp = threadIdx.x; xp < pw; xp += blockDim.x) {
            const int x = xp - kMargin;
            float v = 0.0f;
            if (x >= 0 && x < w) {
                v = srow[x];
                if (finite_max && !isfinite(v)) v = finite_max[b];
                if (clamp) v = v < lo ? lo : (v > hi ? hi : v);
            }
            drow[xp] = v;
        }
    }
}

// Sliding in-place median of E samples in registers: the window holds the E samples of the
// current position, the median just written enters it at its place, the next sample at its
// end. The samples are ordered by an odd-even transposition sort, which swaps only adjacent
// samples in strictly decreasing order and so ends in the same (stable) order as the
// reference's insertion sort for any input without NaN.
template <int E>
__device__ void edge_median_reg(float *srow, int pw)
{
    constexpr int l2 = E / 2;
    float win[E];
#pragma unroll
    for (int q = 0; q < E; ++q) win[q] = q < pw ? srow[q] : 0.0f;
    for (int i = l2; i < pw - l2; ++i) {
        float b[E];
#pragma unroll
        for (int q = 0; q < E; ++q) b[q] = win[q];
#pragma unroll
        for (int pass = 0; pass < E; ++pass) {
#pragma unroll
            for (int k = pass & 1; k + 1 < E; k += 2) {
                const float a = b[k], c = b[k + 1];
                const bool sw = a > c;
                b[k] = sw ? c : a;
                b[k + 1] = sw ? a : c;
            }
        }
        const float m = (E & 1) ? b[E / 2] : static_cast<float>(0.5 * (static_cast<double>(b[E / 2 - 1]) + b[E / 2]));
        srow[i] = m;
#pragma unroll
        for (int q = 0; q + 1 < E; ++q) win[q] = win[q + 1];
        win[l2 - 1 >= 0 ? l2 - 1 : 0] = l2 >= 1 ? m : win[0];
        win[E - 1] = i + 1 + l2 < pw ? srow[i + 1 + l2] : 0.0f;
    }
}

// In-place sliding median of `edge` samples along padded rows 0 and ph-1 (:283-299). One warp
// per edge row: the row is staged in shared memory, lane 0 runs the sequential in-place loop
// there (each median sees the medians already written to its left, as in the reference), and
// the warp writes the row back. Edges 3, 5, 7 and 9 of a row without NaN run in registers.
__global__ void k_edge_median(float *__restrict__ pad, int pw, int ph, int edge)
{
    extern __shared__ float srow[];
    const int lane = threadIdx.x;
    float *row = pad + static_cast<size_t>(blockIdx.x >> 1) * pw * ph + ((blockIdx.x & 1) ? static_cast<size_t>(ph - 1) * pw : 0);
    bool nan = false;
    for (int i = lane; i < pw; i += 32) {
        srow[i] = row[i];
        nan |= isnan(srow[i]);
    }
    nan = __any_sync(0xffffffffu, nan);
    __syncwarp();
    if (lane == 0 && !nan && (edge == 3 || edge == 5 || edge == 7 || edge == 9)) {
        if (edge == 3) edge_median_reg<3>(srow, pw);
        else if (edge == 5) edge_median_reg<5>(srow, pw);
        else if (edge == 7) edge_median_reg<7>(srow, pw);
        else edge_median_reg<9>(srow, pw);
    } else if (lane == 0) {
        const int l2 = edge / 2;
        float buf[kMaxEdge];
        for (int i = l2; i < pw - l2; ++i) {
            for (int q = 0; q < edge; ++q) buf[q] = srow[i - l2 + q];
            for (int a = 1; a < edge; ++a) { // insertion sort
                float key = buf[a];
                int c = a - 1;
                while (c >= 0 && buf[c] > key) {
                    buf[c + 1] = buf[c];
                    --c;
                }
                buf[c + 1] = key;
            }
            srow[i] = (edge & 1) ? buf[edge / 2]
                                 : static_cast<float>(0.5 * (static_cast<double>(buf[edge / 2 - 1]) + buf[edge / 2]));
        }
    }
    __syncwarp();
    for (int i = lane; i < pw; i += 32) row[i] = srow[i];
}

__global__ void k_minmax(const float *__restrict__ pad, size_t n, float *__restrict__ mn, float *__restrict__ mx)
{
    const float *p = pad + blockIdx.x * n;
    float a = FLT_MAX, b = -FLT_MAX;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        a = fminf(a, p[i]);
        b = fmaxf(b, p[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    __shared__ float sa[32], sb[32];
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = (blockDim.x + 31) / 32;
        a = threadIdx.x < nw ? sa[threadIdx.x] : FLT_MAX;
        b = threadIdx.x < nw ? sb[threadIdx.x] : -FLT_MAX;
        for (int o = 16; o > 0; o >>= 1) {
            a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if (threadIdx.x == 0) {
            mn[blockIdx.x] = a;
            mx[blockIdx.x] = b;
        }
    }
}

// Marker of FillHole (interior = image maximum) or FillPeaks (interior = minimum), the image
// on its border (morphextrema.h:268-283, 299-314). sign -1 builds the marker of the negated
// image (FillHole of -padded in the 'both' mode).
__global__ void k_marker(const float *__restrict__ pad, int pw, int ph, const float *__restrict__ interior,
                         float sign, float *__restrict__ v)
{
    const size_t n = static_cast<size_t>(pw) * ph;
    const int b = blockIdx.y;
    const float in = sign * interior[b]; // max(-P) = -min(P) for the negated image
    for (int y = blockIdx.x; y < ph; y += gridDim.x) {
        const size_t ro = b * n + static_cast<size_t>(y) * pw;
        for (int x = threadIdx.x; x < pw; x += blockDim.x) {
            const bool border = y == 0 || y == ph - 1 || x == 0 || x == pw - 1;
            v[ro + x] = border ? sign * pad[ro + x] : in;
        }
    }
}

__device__ __forceinline__ bool is_border(int x, int y, int pw, int ph)
{
    return y == 0 || y == ph - 1 || x == 0 || x == pw - 1;
}

// Replay of RecByDilation's forward scan (morphgeo.h:207-215) over the pixels that can
// change: the border and every pixel with a border pixel among its backward neighbours.
// One thread per image, raster order. v holds the marker on entry.
__global__ void k_peaks_forward_band(const float *__restrict__ pad, int pw, int ph, int nimg, int conn8,
                                     const float *__restrict__ minval, float *__restrict__ v)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nimg) return;
    const size_t n = static_cast<size_t>(pw) * ph;
    const float *g = pad + b * n;
    float *t = v + b * n;
    const float mnv = minval[b];
    const int bx[4] = {-1, 0, -1, 1}, by[4] = {0, -1, -1, -1};
    const int nb = conn8 ? 4 : 2;
    auto visit = [&](int x, int y) {
        const size_t pos = static_cast<size_t>(y) * pw + x;
        float mx = t[pos];
        for (int i = 0; i < nb; ++i) {
            const int qx = x + bx[i], qy = y + by[i];
            if (qx < 0 || qx >= pw || qy < 0) continue;
            const size_t q = static_cast<size_t>(qy) * pw + qx;
            if (t[q] > mx) mx = is_border(qx, qy, pw, ph) ? g[q] : mnv; // assigns the marker value
        }
        t[pos] = mx < g[pos] ? mx : g[pos];
    };
    for (int y = 0; y < ph; ++y) {
        if (y <= 1 || y == ph - 1) {
            for (int x = 0; x < pw; ++x) visit(x, y);
        } else {
            visit(0, y);
            visit(1, y);
            if (conn8 && pw - 2 > 1) visit(pw - 2, y);
            if (pw - 1 > 1) visit(pw - 1, y);
        }
    }
}

// One or two reconstructions of the same images in one launch (FillHole of the image and of its
// negation in the 'both' mode): CTA b < nimg works on image b with sign[0] into vol[0], CTA
// nimg + b on image b with sign[1] into vol[1]. Independent images share the SMs, so the long
// completions of either set overlap.
struct RecJobs {
    float sign[2];
    float *vol[2];
    int nimg;
    const float *interior[2]; // per-image interior value of the marker, formed by the sweeps; null:
                              // the marker is in vol already
};

// Exact reconstruction by alternating row sweeps (see the file comment), one warp per image.
// DILATE: v = min(g, max over neighbourhood); else v = max(g, min over neighbourhood); g is
// `sign * pad`. Rows are staged in shared memory (coalesced global traffic); lane l owns the
// contiguous chunk [l*C, l*C + C) of a row, C odd so that the 32 lanes' chunk positions fall
// in 32 different banks. Positions beyond the row hold the neutral value (-inf for
// dilation, +inf for erosion), which neither propagates into the row nor changes.

template <bool DILATE>
__device__ __forceinline__ float rec_op(float g, float v, float x)
{
    return DILATE ? fminf(g, fmaxf(v, x)) : fmaxf(g, fminf(v, x));
}

__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Barrier of the RW warps of one image (named barrier 1 + image slot; the block holds one image).
template <int RW>
__device__ __forceinline__ void image_sync()
{
    if constexpr (RW == 1) __syncwarp();
    else asm volatile("bar.sync 1, %0;" ::"n"(RW * 32) : "memory");
}

// Clamp pair of a run of elements: for dilation F(x) = min(hi, max(lo, x)) with lo = F(-inf),
// hi = F(+inf); for erosion the same with min/max exchanged (lo = F(+inf), hi = F(-inf)).
// (a then b): apply a first.
template <bool DILATE>
__device__ __forceinline__ void clamp_then(float al, float ah, float &bl, float &bh)
{
    const float nl = rec_op<DILATE>(bh, bl, al), nh = rec_op<DILATE>(bh, bl, ah);
    bl = nl;
    bh = nh;
}

// Order-preserving integer keys of floats (the completion's atomics compare them as ints).
__device__ __forceinline__ int fkey(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}

__device__ __forceinline__ float funkey(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

// One image per block of RW warps; lane t of the image owns the row chunk [t*C, t*C + C), held
// in registers across the vertical step and both scans. C odd: the lanes' chunk positions in
// the shared row buffers fall in distinct banks.
//
// The marker leaves this kernel as keys (fkey): the upward sweep of the last round stores them,
// and an image that converged earlier is converted by one more pass. That sweep also lists the
// pixels it changed (at most cap, then only counted) as the completion's first worklist: after
// it every pixel has been relaxed from its neighbours' current values except from those in the
// row above it that changed later in the sweep, and exactly those are listed. An image whose
// round changed nothing is finished and lists nothing.
template <bool DILATE, int RW, int C>
__global__ void __launch_bounds__(32 * RW) k_reconstruct(const float *__restrict__ pad, RecJobs jobs, int pw, int ph,
                                                         int conn8, int rounds, int *__restrict__ lists, int cap,
                                                         int *__restrict__ counts)
{
    static_assert(C <= 64, "per-pixel change mask");
    const int job = blockIdx.x >= jobs.nimg, img = blockIdx.x - job * jobs.nimg;
    const float sign = jobs.sign[job];
    constexpr int T = 32 * RW, L = T * C + 2 + 1; // row buffer: a neutral element before and after
    extern __shared__ float rows_sm[];
    float(*Gb)[L] = reinterpret_cast<float(*)[L]>(rows_sm);         // [2][L] mask rows
    float(*Rb)[L] = reinterpret_cast<float(*)[L]>(rows_sm + 2 * L); // [3][L] marker rows
    __shared__ float wagg[2][RW][2];
    __shared__ int any_changed[2];
    __shared__ int listed;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const size_t n = static_cast<size_t>(pw) * ph;
    const float *g = pad + img * n;
    float *v = jobs.vol[job] + img * n;
    int *list = lists + blockIdx.x * 2 * static_cast<size_t>(cap);
    const float neutral = DILATE ? -FLT_MAX : FLT_MAX;
    for (int c = t; c < L; c += T) {
        Gb[0][c] = Gb[1][c] = neutral * sign; // sign * stored = neutral
        Rb[0][c] = Rb[1][c] = Rb[2][c] = neutral;
    }
    if (t < 2) any_changed[t] = 0;
    if (t == 0) listed = 0;
    __syncthreads();
    const int c0 = 1 + t * C; // buffer index of the chunk's first element (index 0 is the lead)
    // row y of the mask into G and of the marker into V; from_marker: the initial marker row,
    // formed here (the image on the border, the interior value inside; morphextrema.h:268-283)
    const float *inter = jobs.interior[job];
    const float in_val = inter ? sign * inter[img] : 0.0f;
    auto fetch = [&](int y, float *G, float *V, bool from_marker) {
        const size_t ro = static_cast<size_t>(y) * pw;
        const bool brow = y == 0 || y == ph - 1;
        for (int c = t; c < pw; c += T) {
            cp_async4(G + 1 + c, g + ro + c);
            if (!from_marker) cp_async4(V + 1 + c, v + ro + c);
            else V[1 + c] = brow || c == 0 || c == pw - 1 ? sign * g[ro + c] : in_val;
        }
    };
    // exclusive scan over the image's lanes of clamp pairs; returns the carry into this lane
    auto carry_in = [&](float xl, float xh, bool fwd, int slot) -> float {
        for (int o = 1; o < 32; o <<= 1) {
            const float pl = fwd ? __shfl_up_sync(0xffffffffu, xl, o) : __shfl_down_sync(0xffffffffu, xl, o);
            const float pu = fwd ? __shfl_up_sync(0xffffffffu, xh, o) : __shfl_down_sync(0xffffffffu, xh, o);
            if (fwd ? lane >= o : lane + o < 32) clamp_then<DILATE>(pl, pu, xl, xh);
        }
        // (xl, xh): inclusive prefix within the warp
        float before_l = neutral, before_h = -neutral; // identity
        if constexpr (RW > 1) {
            if (fwd ? lane == 31 : lane == 0) {
                wagg[slot][warp][0] = xl;
                wagg[slot][warp][1] = xh;
            }
            image_sync<RW>();
            // warps earlier in the scan direction, in order (copies: wagg is shared)
            for (int k = 0; k < RW; ++k) {
                const int w = fwd ? k : RW - 1 - k;
                if (fwd ? w >= warp : w <= warp) break;
                float bl = wagg[slot][w][0], bh = wagg[slot][w][1];
                clamp_then<DILATE>(before_l, before_h, bl, bh);
                before_l = bl;
                before_h = bh;
            }
        }
        // lanes before this one within the warp
        float il = fwd ? __shfl_up_sync(0xffffffffu, xl, 1) : __shfl_down_sync(0xffffffffu, xl, 1);
        float ih = fwd ? __shfl_up_sync(0xffffffffu, xh, 1) : __shfl_down_sync(0xffffffffu, xh, 1);
        if (fwd ? lane > 0 : lane < 31) {
            clamp_then<DILATE>(before_l, before_h, il, ih);
            before_l = il;
        }
        return before_l; // the prefix applied to the neutral input
    };

    // one sweep (pass 0 downward, 1 upward); LAST: the upward sweep of the last round, which lists
    // the pixels it changes and stores keys. Returns whether this thread's chunks changed.
    auto sweep = [&](int pass, bool from_marker, auto last_tag) -> bool {
        constexpr bool LAST = decltype(last_tag)::value;
        bool changed = false;
        int gi = 0, vi = 0;
        fetch(pass == 0 ? 0 : ph - 1, Gb[0], Rb[0], from_marker);
        cp_async_wait_all();
        image_sync<RW>();
        for (int step = 0; step < ph; ++step) {
            const int y = pass == 0 ? step : ph - 1 - step;
            const float *G = Gb[gi];
            float *V = Rb[vi];
            const float *Pv = Rb[(vi + 2) % 3];
            if (step + 1 < ph) fetch(pass == 0 ? y + 1 : y - 1, Gb[gi ^ 1], Rb[(vi + 1) % 3], from_marker);
            float gv[C], cv[C];
            unsigned long long chg = 0; // LAST: bit j = element j of the chunk changed in this step
            auto note = [&](int j, bool moved) {
                if constexpr (LAST) chg |= static_cast<unsigned long long>(moved) << j;
                else changed |= moved;
            };
#pragma unroll
            for (int j = 0; j < C; ++j) {
                gv[j] = sign * G[c0 + j];
                cv[j] = V[c0 + j];
            }
            if (step > 0) {
#pragma unroll
                for (int j = 0; j < C; ++j) {
                    float nb = Pv[c0 + j];
                    if (conn8)
                        nb = DILATE ? fmaxf(nb, fmaxf(Pv[c0 + j - 1], Pv[c0 + j + 1]))
                                    : fminf(nb, fminf(Pv[c0 + j - 1], Pv[c0 + j + 1]));
                    const float nvl = rec_op<DILATE>(gv[j], cv[j], nb);
                    note(j, nvl != cv[j]);
                    cv[j] = nvl;
                }
            }
            // forward along the row
            {
                float lo = neutral, hi = -neutral;
#pragma unroll
                for (int j = 0; j < C; ++j) {
                    lo = rec_op<DILATE>(gv[j], cv[j], lo);
                    hi = rec_op<DILATE>(gv[j], cv[j], hi);
                }
                float run = carry_in(lo, hi, true, 0);
#pragma unroll
                for (int j = 0; j < C; ++j) {
                    run = rec_op<DILATE>(gv[j], cv[j], run);
                    note(j, run != cv[j]);
                    cv[j] = run;
                }
            }
            // backward
            {
                float lo = neutral, hi = -neutral;
#pragma unroll
                for (int j = C - 1; j >= 0; --j) {
                    lo = rec_op<DILATE>(gv[j], cv[j], lo);
                    hi = rec_op<DILATE>(gv[j], cv[j], hi);
                }
                float run = carry_in(lo, hi, false, 1);
#pragma unroll
                for (int j = C - 1; j >= 0; --j) {
                    run = rec_op<DILATE>(gv[j], cv[j], run);
                    note(j, run != cv[j]);
                    cv[j] = run;
                }
            }
            if constexpr (LAST) {
                changed |= chg != 0;
                // positions past the row never change (neutral), so every bit is a pixel
                if (chg) {
#pragma unroll
                    for (int j = 0; j < C; ++j) {
                        if (!((chg >> j) & 1)) continue;
                        const int pos = atomicAdd(&listed, 1);
                        if (pos < cap) list[pos] = y * pw + c0 + j - 1;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < C; ++j) V[c0 + j] = cv[j];
            image_sync<RW>();
            const size_t ro = static_cast<size_t>(y) * pw;
            if constexpr (LAST) {
                int *vk = reinterpret_cast<int *>(v);
                for (int c = t; c < pw; c += T) vk[ro + c] = fkey(V[1 + c]);
            } else {
                for (int c = t; c < pw; c += T) v[ro + c] = V[1 + c];
            }
            cp_async_wait_all(); // the next row has landed
            image_sync<RW>();
            gi ^= 1;
            vi = (vi + 1) % 3;
        }
        return changed;
    };

    bool keys = false; // the marker in global memory is stored as keys
    for (int round = 0; round < rounds; ++round) {
        bool changed = sweep(0, round == 0 && inter, std::false_type{});
        if (round == rounds - 1) {
            changed |= sweep(1, false, std::true_type{});
            keys = true;
        } else {
            changed |= sweep(1, false, std::false_type{});
        }
        // image-wide vote (alternating flags: the one read now is cleared for the round after)
        if (changed) any_changed[round & 1] = 1;
        image_sync<RW>();
        const int any = any_changed[round & 1];
        if (t == 0) any_changed[(round + 1) & 1] = 0;
        image_sync<RW>();
        if (!any) break;
    }
    if (!keys) {
        // converged before the last round: nothing to list; store the marker as keys
        int *vk = reinterpret_cast<int *>(v);
        for (size_t i = t; i < n; i += T) vk[i] = fkey(__int_as_float(vk[i]));
    }
    if (t == 0) counts[blockIdx.x] = listed; // the pushes precede the barriers of the last vote
}

template <bool DILATE, int RW, int C>
static mr_status launch_rec(const RecJobs &jobs, int njobs, const float *pad, int pw, int ph, int conn8, int *lists,
                            int cap, int *counts, cudaStream_t s)
{
    const size_t smem = 5 * static_cast<size_t>(32 * RW * C + 3) * sizeof(float);
    MR_CUDA_TRY(cudaFuncSetAttribute(k_reconstruct<DILATE, RW, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    k_reconstruct<DILATE, RW, C><<<jobs.nimg * njobs, 32 * RW, smem, s>>>(pad, jobs, pw, ph, conn8, kSweepRounds,
                                                                          lists, cap, counts);
    return check_launch("k_reconstruct");
}

// ---- completion: worklist relaxation
//
// After the sweeps the remaining changes are sparse (thin, winding paths through the noise),
// so each image's CTA finishes the reconstruction with a worklist. Values are order-preserving
// integer keys (the sweeps leave them so) so that the relaxation is one atomicMin (erosion:
// v[q] = min(v[q], max(g[q], v[p]))) or atomicMax (dilation: v[q] = max(v[q], min(g[q], v[p])))
// per neighbour. The first list is the sweeps' (the pixels their last sweep changed); an image
// whose sweeps converged lists nothing and is done. A relaxation is issued, without waiting for
// its result, when its candidate improves the neighbour's value as loaded, and the neighbour is
// then listed for the next iteration (or followed, below): every change of a value is made by
// such an update, whose pixel is listed with the value written, so the last value of every
// pixel is propagated; a listing whose update lost to a better concurrent one only repeats
// work. It then relaxes its neighbours with its current value. When a list overflows, the next
// iteration relaxes every pixel from its neighbours instead. The reconstruction ends when an
// iteration lists nothing: every pixel then satisfies the fixpoint equations with all its
// neighbours, and the fixpoint is unique, so the result equals the reference's whatever the
// order of the updates. Values are read through L2 (ld.cg), where the atomics resolve. Latency
// shapes the code: an entry issues all its neighbour loads, then all its updates, and the dense
// passes handle kUnroll pixels per thread at a time.

constexpr int kFrontThreads = 512;
constexpr int kMaxIterations = 1 << 22;
constexpr int kUnroll = 4;
constexpr int kChase = 32; // pixels one thread follows within an iteration

template <bool DILATE>
__device__ __forceinline__ void relax(int *addr, int c)
{
    if (DILATE) atomicMax(addr, c);
    else atomicMin(addr, c);
}

template <bool DILATE, bool CONN8>
__global__ void __launch_bounds__(kFrontThreads) k_complete(const float *__restrict__ pad, RecJobs jobs, int pw,
                                                            int ph, int *__restrict__ lists, int cap,
                                                            const int *__restrict__ counts)
{
    const int first = counts[blockIdx.x]; // the sweeps' list (uniform over the CTA)
    if (first == 0) return;
    const int t = threadIdx.x;
    const int n = pw * ph;
    const int job = blockIdx.x >= jobs.nimg, img = blockIdx.x - job * jobs.nimg;
    const float sign = jobs.sign[job];
    const float *g = pad + img * static_cast<size_t>(n);
    int *v = reinterpret_cast<int *>(jobs.vol[job] + img * static_cast<size_t>(n));
    int *cur = lists + blockIdx.x * 2 * static_cast<size_t>(cap), *next = cur + cap;
    __shared__ int count[3];
    if (t < 3) count[t] = 0;
    __syncthreads();

    const int nx[8] = {-1, 1, 0, 0, -1, 1, -1, 1}, ny[8] = {0, 0, -1, 1, -1, -1, 1, 1};
    constexpr int NN = CONN8 ? 8 : 4;
    auto improves = [](int c, int old) { return DILATE ? c > old : c < old; };
    auto push = [&](int q, int it) {
        const int pos = atomicAdd(&count[it % 3], 1);
        if (pos < cap) next[pos] = q;
    };

    bool dense = first > cap;
    int nf = min(first, cap), it = 0;
    for (; it < kMaxIterations; ++it) {
        if (dense) {
            // every pixel from the extreme of its neighbours, kUnroll pixels at a time
            for (int i0 = t; i0 < n; i0 += kUnroll * kFrontThreads) {
                int c[kUnroll], kv[kUnroll];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    const int i = i0 + u * kFrontThreads;
                    const int y = i / pw, x = i % pw;
                    int kn = DILATE ? INT_MIN : INT_MAX;
#pragma unroll
                    for (int k = 0; k < NN; ++k) {
                        const int qx = x + nx[k], qy = y + ny[k];
                        if (i >= n || qx < 0 || qx >= pw || qy < 0 || qy >= ph) continue;
                        const int kq = __ldcg(v + qy * pw + qx);
                        kn = DILATE ? max(kn, kq) : min(kn, kq);
                    }
                    const int kg = i < n ? fkey(sign * __ldg(g + i)) : 0;
                    c[u] = DILATE ? min(kg, kn) : max(kg, kn);
                    kv[u] = i < n ? __ldcg(v + i) : c[u];
                }
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    if (!improves(c[u], kv[u])) continue;
                    relax<DILATE>(v + i0 + u * kFrontThreads, c[u]);
                    push(i0 + u * kFrontThreads, it);
                }
            }
        } else {
            for (int e = t; e < nf; e += kFrontThreads) {
                // relax the neighbours of p; the thread then follows the first neighbour it moved
                // (chasing) for up to kChase steps and lists the others it moved, so a change
                // travels along a path without waiting for a barrier per pixel. Every moved
                // pixel is relaxed afterwards, by this thread's chase or from the next list.
                int p = cur[e];
                // value of p: read for a listed pixel; for a chased one, the value this thread
                // just gave it (a lower value someone else gave it meanwhile is propagated by that
                // thread, and a candidate from a higher one is still an upper bound of the
                // result), which saves a round trip to L2 per step
                int kp = __ldcg(v + p);
                for (int step = 0; p >= 0; ++step) {
                    const int y = p / pw, x = p % pw;
                    int c[NN], kv[NN];
                    unsigned ok = 0;
#pragma unroll
                    for (int k = 0; k < NN; ++k) {
                        const int qx = x + nx[k], qy = y + ny[k];
                        const bool in = qx >= 0 && qx < pw && qy >= 0 && qy < ph;
                        const int q = qy * pw + qx;
                        const int kg = in ? fkey(sign * __ldg(g + q)) : 0;
                        kv[k] = in ? __ldcg(v + q) : 0;
                        c[k] = DILATE ? min(kg, kp) : max(kg, kp);
                        if (in && improves(c[k], kv[k])) ok |= 1u << k;
                    }
                    int follow = -1, kf = 0;
#pragma unroll
                    for (int k = 0; k < NN; ++k) {
                        if (!((ok >> k) & 1)) continue;
                        const int q = p + ny[k] * pw + nx[k];
                        if (!MR_IN_BOUNDS(q, n, kSiteSpotNbr)) continue;
                        relax<DILATE>(v + q, c[k]);
                        if (follow < 0 && step + 1 < kChase) {
                            follow = q;
                            kf = c[k];
                        } else {
                            push(q, it);
                        }
                    }
                    p = follow;
                    kp = kf;
                }
            }
        }
        __syncthreads();
        // count[it % 3] is final; count[(it + 2) % 3] was read by everyone before this barrier
        // and is next written in iteration it + 2
        const int pushed = count[it % 3];
        if (t == 0) count[(it + 2) % 3] = 0;
        int *tmp = cur;
        cur = next;
        next = tmp;
        if (pushed == 0) break;
        dense = pushed > cap;
        nf = min(pushed, cap);
    }
    if (it == kMaxIterations && t == 0) atomicExch(&g_msc_error, 2);
}

// Worklist capacity per image (entries); a larger frontier falls back to a dense iteration.
inline int complete_cap(size_t n) { return static_cast<int>(std::min<size_t>(n, std::max<size_t>(256, n / 16))); }

// Sweeps, then the completion, of jobs.nimg x njobs reconstructions (one CTA each). lists: two
// worklists of complete_cap entries per CTA; counts: one word per CTA (the sweeps' list length).
template <bool DILATE>
static mr_status launch_reconstruct(const RecJobs &jobs, int njobs, const float *pad, int pw, int ph, int conn8,
                                    int *lists, int *counts, cudaStream_t s)
{
    constexpr int RW = 4;
    const int per = (pw + 32 * RW - 1) / (32 * RW);
    const int cap = complete_cap(static_cast<size_t>(pw) * ph);
    mr_status st;
    if (per <= 3) st = launch_rec<DILATE, RW, 3>(jobs, njobs, pad, pw, ph, conn8, lists, cap, counts, s);
    else if (per <= 5) st = launch_rec<DILATE, RW, 5>(jobs, njobs, pad, pw, ph, conn8, lists, cap, counts, s);
    else if (per <= 9) st = launch_rec<DILATE, RW, 9>(jobs, njobs, pad, pw, ph, conn8, lists, cap, counts, s);
    else if (per <= 17) st = launch_rec<DILATE, RW, 17>(jobs, njobs, pad, pw, ph, conn8, lists, cap, counts, s);
    else if (per <= 33) st = launch_rec<DILATE, RW, 33>(jobs, njobs, pad, pw, ph, conn8, lists, cap, counts, s);
    else return fail(MR_ERR_UNSUPPORTED, "mr_morphspotclean: rows longer than %d pixels", 32 * RW * 33 - 2 * kMargin);
    if (st != MR_OK) return st;
    const int nb = jobs.nimg * njobs;
    if (conn8) k_complete<DILATE, true><<<nb, kFrontThreads, 0, s>>>(pad, jobs, pw, ph, lists, cap, counts);
    else k_complete<DILATE, false><<<nb, kFrontThreads, 0, s>>>(pad, jobs, pw, ph, lists, cap, counts);
    return check_launch("k_complete");
}

// Replacement / blend and unpadding (MorphSpotClean::ProcessReplace :108-175,
// kipl::math::SigmoidWeights mathfunctions.hpp:92-99).
__global__ void k_replace(const float *__restrict__ pad, const float *__restrict__ holes, const float *__restrict__ peaks,
                          int w, int h, int detect, float th0, float th1, float s0, float s1, float *__restrict__ img)
{
    const int pw = w + 2 * kMargin, ph = h + 2 * kMargin;
    const size_t n = static_cast<size_t>(pw) * ph;
    const int b = blockIdx.y;
    const size_t per = static_cast<size_t>(w) * h;
    for (int y = blockIdx.x; y < h; y += gridDim.x)
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
        const size_t idx = static_cast<size_t>(y) * w + x;
        const size_t pi = b * n + static_cast<size_t>(y + kMargin) * pw + x + kMargin;
        const float val = pad[pi];
        float out = val;
        // the reconstructions are stored as keys
        const float hv = holes ? funkey(__float_as_int(holes[pi])) : 0.0f;
        const float pk = peaks ? funkey(__float_as_int(peaks[pi])) : 0.0f;
        const float pv = detect == 2 ? -pk : pk;
        if (s0 == 0.0f && s1 == 0.0f) {
            if (detect != 1 && th0 < fabsf(__fsub_rn(val, hv))) out = hv;
            if (detect != 0 && th1 < fabsf(__fsub_rn(pv, val))) out = pv;
        } else {
            auto sw = [](float x, float a, float bb, float level, float width) {
                const float wgt = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(__fdiv_rn(__fsub_rn(level, x), width))));
                return __fadd_rn(a, __fmul_rn(__fsub_rn(bb, a), wgt));
            };
            if (detect == 0) out = sw(__fsub_rn(hv, val), val, hv, th0, s0);
            else if (detect == 1) out = sw(__fsub_rn(val, pv), val, pv, th1, s1);
            else {
                const float dp = __fsub_rn(val, pv), dh = __fsub_rn(hv, val);
                out = fabsf(dh) < fabsf(dp) ? sw(dp, val, pv, th0, s0) : sw(dh, val, hv, th1, s1);
            }
        }
        img[static_cast<size_t>(b) * per + idx] = out;
    }
}

} // namespace msc
} // namespace mr

using namespace mr;
using namespace mr::msc;

extern "C" {

mr_status mr_morphspotclean(float *proj_d, size_t nu, size_t nv, size_t nproj, int detect, int conn8,
                            const float *th_h, const float *sigma_h, int edge, int clamp, float minlevel,
                            float maxlevel, int removeinfnan, void *stream)
{
    MR_TRACE();
    if (!proj_d || !th_h || !sigma_h) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: null pointer");
    if (detect < 0 || detect > 2) return fail(MR_ERR_ARGUMENT, "Unkown detection method selected");
    if (nv < 5) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: images need at least 5 rows (the edge padding mirrors 5 rows)");
    if (edge < 1 || edge > kMaxEdge) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: edge smoothing length must be 1..%d", kMaxEdge);
    if (nu == 0 || nproj == 0) return MR_OK;
    const int w = static_cast<int>(nu), h = static_cast<int>(nv);
    const int pw = w + 2 * kMargin, ph = h + 2 * kMargin;
    if (pw > 128 * 33) return fail(MR_ERR_UNSUPPORTED, "mr_morphspotclean: rows longer than %d pixels", 128 * 33 - 2 * kMargin);
    const size_t n = static_cast<size_t>(pw) * ph;
    cudaStream_t s = as_stream(stream);
    // images per batch: three padded buffers and two worklists each; up to a quarter of the
    // free device memory, so that a block of projections is cleaned concurrently (one CTA per
    // image)
    const size_t cap = static_cast<size_t>(complete_cap(n));
    const size_t per_img = 3 * n * sizeof(float) + 4 * cap * sizeof(int); // two worklists per reconstruction
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = size_t(1) << 30;
    const size_t budget = std::max<size_t>(size_t(1) << 30, free_b / 4);
    const size_t batch = std::max<size_t>(1, std::min<size_t>(nproj, budget / per_img));
    float *scratch = nullptr;
    MR_TRY(device_alloc(&scratch, batch * per_img + 5 * batch * sizeof(float), s, "mr_morphspotclean: scratch"));
    float *P = scratch, *H = P + batch * n, *K = H + batch * n, *stats = K + batch * n;
    float *fmax = stats, *mn = stats + batch, *mx = stats + 2 * batch;
    int *counts = reinterpret_cast<int *>(stats + 3 * batch); // two words per image (the sweeps' list lengths)
    int *lists = reinterpret_cast<int *>(stats + 5 * batch);
    mr_status st = MR_OK;
    for (size_t b0 = 0; b0 < nproj && st == MR_OK; b0 += batch) {
        const int nb = static_cast<int>(std::min(batch, nproj - b0));
        float *img = proj_d + b0 * nu * nv;
        const unsigned gx = std::min<unsigned>(div_up(n, 256), 128u);
        if (removeinfnan) k_finite_max<<<nb, 256, 0, s>>>(img, nu * nv, fmax);
        k_pad<<<dim3(gx, nb), 256, 0, s>>>(img, w, h, removeinfnan ? fmax : nullptr, clamp, minlevel, maxlevel, P);
        k_edge_median<<<2 * nb, 32, pw * sizeof(float), s>>>(P, pw, ph, edge);
        k_minmax<<<nb, 1024, 0, s>>>(P, n, mn, mx);
        if (detect == 0) { // FillHole: erosion from a max marker (formed by the first sweep)
            const RecJobs jobs{{1.0f, 1.0f}, {H, H}, nb, {mx, mx}};
            if ((st = launch_reconstruct<false>(jobs, 1, P, pw, ph, conn8, lists, counts, s)) != MR_OK) break;
        }
        if (detect == 1) { // FillPeaks: forward-scan band replay, then the exact dilation
            k_marker<<<dim3(gx, nb), 256, 0, s>>>(P, pw, ph, mn, 1.0f, K);
            k_peaks_forward_band<<<div_up(nb, 32), 32, 0, s>>>(P, pw, ph, nb, conn8, mn, K);
            const RecJobs jobs{{1.0f, 1.0f}, {K, K}, nb, {nullptr, nullptr}};
            if ((st = launch_reconstruct<true>(jobs, 1, P, pw, ph, conn8, lists, counts, s)) != MR_OK) break;
        }
        if (detect == 2) {
            // FillHole of the image, and -FillHole(-padded): erosion of the negated image from
            // marker max(-P) = -min(P); both erosions in the same launches
            const RecJobs jobs{{1.0f, -1.0f}, {H, K}, nb, {mx, mn}};
            if ((st = launch_reconstruct<false>(jobs, 2, P, pw, ph, conn8, lists, counts, s)) != MR_OK) break;
        }
        if ((st = check_launch("morphspotclean reconstruction")) != MR_OK) break;
        k_replace<<<dim3(gx, nb), 256, 0, s>>>(P, detect != 1 ? H : nullptr, detect != 0 ? K : nullptr, w, h, detect,
                                               th_h[0], th_h[1], sigma_h[0], sigma_h[1], img);
        st = check_launch("k_replace");
    }
    cudaFreeAsync(scratch, s);
    return st;
}

} // extern "C"
