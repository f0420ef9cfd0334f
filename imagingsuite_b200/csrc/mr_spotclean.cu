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
// The reconstruction kernel runs one CTA per image and alternates downward and upward row
// sweeps until a full round changes nothing (bounded; the bound sets the device error
// word). A sweep combines each row with the neighbouring row just finished (vertical and,
// for 8-connectivity, diagonal neighbours), then propagates along the row in both
// directions with a CTA-wide scan: the row update v[c] = min(g[c], max(v[c], v[c-1]))
// (dilation) or max(g[c], min(v[c], v[c-1])) (erosion) is a clamp x -> min(hi, max(lo, x)),
// and clamps compose into clamps, so the sequential recurrence is a parallel prefix.
#include "mr_common.cuh"

#include <cfloat>
#include <cmath>

namespace mr {

extern __device__ int g_device_error;

namespace msc {

constexpr int kMargin = 5;
constexpr int kThreads = 1024;
constexpr int kMaxRounds = 4096;
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
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < n;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(idx / pw), x = static_cast<int>(idx % pw) - kMargin;
        float v = 0.0f;
        if (x >= 0 && x < w) {
            int sy = y - kMargin;
            if (sy < 0) sy = -1 - sy;                 // padded row m-1-i <- image row i
            else if (sy >= h) sy = 2 * h - 1 - sy;    // padded row ph-m+i <- image row h-1-i
            v = src[static_cast<size_t>(sy) * w + x];
            if (finite_max && !isfinite(v)) v = finite_max[b];
            if (clamp) v = v < lo ? lo : (v > hi ? hi : v);
        }
        dst[idx] = v;
    }
}

// In-place sliding median of `edge` samples along padded rows 0 and ph-1 (:283-299).
__global__ void k_edge_median(float *__restrict__ pad, int pw, int ph, int nimg, int edge)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * nimg) return;
    float *row = pad + static_cast<size_t>(t >> 1) * pw * ph + ((t & 1) ? static_cast<size_t>(ph - 1) * pw : 0);
    const int l2 = edge / 2;
    float buf[kMaxEdge];
    for (int i = l2; i < pw - l2; ++i) {
        for (int q = 0; q < edge; ++q) buf[q] = row[i - l2 + q];
        for (int a = 1; a < edge; ++a) { // insertion sort
            float key = buf[a];
            int c = a - 1;
            while (c >= 0 && buf[c] > key) {
                buf[c + 1] = buf[c];
                --c;
            }
            buf[c + 1] = key;
        }
        row[i] = (edge & 1) ? buf[edge / 2]
                            : static_cast<float>(0.5 * (static_cast<double>(buf[edge / 2 - 1]) + buf[edge / 2]));
    }
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
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < n;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(idx / pw), x = static_cast<int>(idx % pw);
        const bool border = y == 0 || y == ph - 1 || x == 0 || x == pw - 1;
        v[b * n + idx] = border ? sign * pad[b * n + idx] : in;
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

// Exact reconstruction by alternating row sweeps (see the file comment). DILATE: v = min(g,
// max over neighbourhood); else v = max(g, min over neighbourhood). g is `sign * pad`.
template <bool DILATE>
__global__ void __launch_bounds__(kThreads) k_reconstruct(const float *__restrict__ pad, float sign, int pw, int ph,
                                                          int conn8, float *__restrict__ vol)
{
    extern __shared__ float sm[];
    float *prev = sm;                       // finished neighbouring row [pw]
    Clamp *wagg = reinterpret_cast<Clamp *>(sm + pw); // per-warp aggregates [32]
    __shared__ int changed_s;
    const size_t n = static_cast<size_t>(pw) * ph;
    const float *g = pad + blockIdx.x * n;
    float *v = vol + blockIdx.x * n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // consecutive chunk of the row per thread
    const int per = (pw + kThreads - 1) / kThreads;
    const int c0 = min(tid * per, pw), c1 = min(c0 + per, pw);
    constexpr int kMaxPer = 8;

    int round = 0;
    for (; round < kMaxRounds; ++round) {
        if (tid == 0) changed_s = 0;
        __syncthreads();
        int changed = 0;
        for (int pass = 0; pass < 2; ++pass) {
            const int dir = pass == 0 ? 1 : -1;
            for (int step = 0; step < ph; ++step) {
                const int y = dir > 0 ? step : ph - 1 - step;
                float val[kMaxPer], gg[kMaxPer];
                // vertical / diagonal neighbours from the row finished just before
                for (int e = 0; e < c1 - c0; ++e) {
                    const int c = c0 + e;
                    const size_t idx = static_cast<size_t>(y) * pw + c;
                    float cand = v[idx];
                    const float gv = sign * g[idx];
                    if (step > 0) {
                        float nbv = prev[c];
                        if (conn8) {
                            if (c > 0) nbv = DILATE ? fmaxf(nbv, prev[c - 1]) : fminf(nbv, prev[c - 1]);
                            if (c + 1 < pw) nbv = DILATE ? fmaxf(nbv, prev[c + 1]) : fminf(nbv, prev[c + 1]);
                        }
                        cand = DILATE ? fminf(gv, fmaxf(cand, nbv)) : fmaxf(gv, fminf(cand, nbv));
                    }
                    val[e] = cand;
                    gg[e] = gv;
                }
                // along the row, both directions: clamp prefix scans
                for (int sweep = 0; sweep < 2; ++sweep) {
                    const bool fwd = sweep == 0;
                    Clamp acc{-FLT_MAX, FLT_MAX}; // identity
                    const int cnt = c1 - c0;
                    for (int k = 0; k < cnt; ++k) {
                        const int e = fwd ? k : cnt - 1 - k;
                        const Clamp f = DILATE ? Clamp{val[e], gg[e]} : Clamp{gg[e], val[e]};
                        acc = compose(acc, f);
                    }
                    // exclusive scan of thread aggregates in the sweep direction
                    Clamp x = acc;
                    for (int o = 1; o < 32; o <<= 1) {
                        Clamp y2;
                        y2.lo = fwd ? __shfl_up_sync(0xffffffffu, x.lo, o) : __shfl_down_sync(0xffffffffu, x.lo, o);
                        y2.hi = fwd ? __shfl_up_sync(0xffffffffu, x.hi, o) : __shfl_down_sync(0xffffffffu, x.hi, o);
                        const bool ok = fwd ? lane >= o : lane + o < 32;
                        if (ok) x = compose(y2, x);
                    }
                    if ((fwd && lane == 31) || (!fwd && lane == 0)) wagg[warp] = x;
                    __syncthreads();
                    Clamp before{-FLT_MAX, FLT_MAX};
                    const int nwarps = kThreads / 32;
                    if (fwd) {
                        for (int q = 0; q < warp; ++q) before = compose(before, wagg[q]);
                    } else {
                        for (int q = nwarps - 1; q > warp; --q) before = compose(before, wagg[q]);
                    }
                    // within the warp: everything before this lane
                    Clamp inwarp;
                    inwarp.lo = fwd ? __shfl_up_sync(0xffffffffu, x.lo, 1) : __shfl_down_sync(0xffffffffu, x.lo, 1);
                    inwarp.hi = fwd ? __shfl_up_sync(0xffffffffu, x.hi, 1) : __shfl_down_sync(0xffffffffu, x.hi, 1);
                    if ((fwd && lane > 0) || (!fwd && lane < 31)) before = compose(before, inwarp);
                    // apply along this thread's chunk
                    Clamp run = before;
                    for (int k = 0; k < cnt; ++k) {
                        const int e = fwd ? k : cnt - 1 - k;
                        const Clamp f = DILATE ? Clamp{val[e], gg[e]} : Clamp{gg[e], val[e]};
                        run = compose(run, f);
                        val[e] = DILATE ? run.lo : run.hi; // F(-inf) for dilation, F(+inf) for erosion
                    }
                    __syncthreads(); // wagg reused
                }
                for (int e = 0; e < c1 - c0; ++e) {
                    const int c = c0 + e;
                    const size_t idx = static_cast<size_t>(y) * pw + c;
                    if (v[idx] != val[e]) {
                        changed = 1;
                        v[idx] = val[e];
                    }
                    prev[c] = val[e];
                }
                __syncthreads();
            }
        }
        if (changed) atomicOr(&changed_s, 1);
        __syncthreads();
        const int any = changed_s;
        __syncthreads();
        if (!any) break;
    }
    if (round == kMaxRounds && tid == 0) atomicExch(&g_device_error, 2);
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
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < per;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(idx / w), x = static_cast<int>(idx % w);
        const size_t pi = b * n + static_cast<size_t>(y + kMargin) * pw + x + kMargin;
        const float val = pad[pi];
        float out = val;
        const float hv = holes ? holes[pi] : 0.0f;
        const float pv = peaks ? (detect == 2 ? -peaks[pi] : peaks[pi]) : 0.0f;
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
    if (!proj_d || !th_h || !sigma_h) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: null pointer");
    if (detect < 0 || detect > 2) return fail(MR_ERR_ARGUMENT, "Unkown detection method selected");
    if (nv < 5) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: images need at least 5 rows (the edge padding mirrors 5 rows)");
    if (edge < 1 || edge > kMaxEdge) return fail(MR_ERR_ARGUMENT, "mr_morphspotclean: edge smoothing length must be 1..%d", kMaxEdge);
    if (nu == 0 || nproj == 0) return MR_OK;
    const int w = static_cast<int>(nu), h = static_cast<int>(nv);
    const int pw = w + 2 * kMargin, ph = h + 2 * kMargin;
    if (pw > kThreads * 8) return fail(MR_ERR_UNSUPPORTED, "mr_morphspotclean: rows longer than %d pixels", kThreads * 8 - 10);
    const size_t n = static_cast<size_t>(pw) * ph;
    cudaStream_t s = as_stream(stream);
    // images per batch: three padded buffers each, about 1 GiB of scratch at most
    const size_t per_img = 3 * n * sizeof(float);
    const size_t batch = std::max<size_t>(1, std::min<size_t>(nproj, (size_t(1) << 30) / per_img));
    float *scratch = nullptr;
    MR_CUDA_TRY(cudaMallocAsync(&scratch, batch * per_img + 4 * batch * sizeof(float), s));
    float *P = scratch, *H = P + batch * n, *K = H + batch * n, *stats = K + batch * n;
    float *fmax = stats, *mn = stats + batch, *mx = stats + 2 * batch;
    mr_status st = MR_OK;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_reconstruct<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
        cudaFuncSetAttribute(k_reconstruct<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
        attr = true;
    }
    const size_t rsmem = (pw + 64) * sizeof(float);
    for (size_t b0 = 0; b0 < nproj && st == MR_OK; b0 += batch) {
        const int nb = static_cast<int>(std::min(batch, nproj - b0));
        float *img = proj_d + b0 * nu * nv;
        const unsigned gx = std::min<unsigned>(div_up(n, 256), 128u);
        if (removeinfnan) k_finite_max<<<nb, 256, 0, s>>>(img, nu * nv, fmax);
        k_pad<<<dim3(gx, nb), 256, 0, s>>>(img, w, h, removeinfnan ? fmax : nullptr, clamp, minlevel, maxlevel, P);
        k_edge_median<<<div_up(2 * nb, 64), 64, 0, s>>>(P, pw, ph, nb, edge);
        k_minmax<<<nb, 1024, 0, s>>>(P, n, mn, mx);
        if (detect == 0 || detect == 2) { // FillHole: erosion from a max marker
            k_marker<<<dim3(gx, nb), 256, 0, s>>>(P, pw, ph, mx, 1.0f, H);
            k_reconstruct<false><<<nb, kThreads, rsmem, s>>>(P, 1.0f, pw, ph, conn8, H);
        }
        if (detect == 1) { // FillPeaks: forward-scan band replay, then the exact dilation
            k_marker<<<dim3(gx, nb), 256, 0, s>>>(P, pw, ph, mn, 1.0f, K);
            k_peaks_forward_band<<<div_up(nb, 32), 32, 0, s>>>(P, pw, ph, nb, conn8, mn, K);
            k_reconstruct<true><<<nb, kThreads, rsmem, s>>>(P, 1.0f, pw, ph, conn8, K);
        }
        if (detect == 2) { // -FillHole(-padded): erosion of the negated image from marker max(-P) = -min(P)
            k_marker<<<dim3(gx, nb), 256, 0, s>>>(P, pw, ph, mn, -1.0f, K);
            k_reconstruct<false><<<nb, kThreads, rsmem, s>>>(P, -1.0f, pw, ph, conn8, K);
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
