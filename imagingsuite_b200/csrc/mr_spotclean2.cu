// SpotClean2: ImagingAlgorithms::SpotClean on the GPU.
//
// References (relative to the reference project root):
//   SpotClean2::ProcessCore        frameworks/tomography/Preprocessing/StdPreprocModules/src/
//                                  SpotClean2.cpp:117-130
//   SpotClean::Process, DetectSpots, ExcludeLargeRegions, CleanByArray, PrepareNeighborhood,
//   Neighborhood, DetectionImage and the five detectors
//                                  core/algorithms/ImagingAlgorithms/src/SpotClean.cpp:78-545
//   TFilterBase / TFilter / TErode / TDilate with EdgeMirror
//                                  core/kipl/kipl/include/filters/core/filterbase.hpp:83-408,
//                                  filters/core/filter.hpp, morphology/core/morphfilters.hpp
//   LabelImage, LabelArea, RemoveConnectedRegion
//                                  core/kipl/kipl/include/morphology/label.h
//   kipl::math::statistics         core/kipl/kipl/include/math/core/image_statistics.hpp:197-219
//
// Per batch of projections (one image per grid z):
//   1. detection image (ring 5x5 filter, 3x3 standard deviation from box sums, 1x5 + 5x1
//      medians, 1x5 + 5x1 erosion/dilation, or the three-box TriKernel), each filter summing
//      or taking min/max over its taps in the reference's order with its EdgeMirror regions;
//   2. SigmoidLUT(1 << 15, gamma, sigma) on it;
//   3. large regions excluded: 8-connected components of the nonzero weights by union-find,
//      component areas, and the reference's rule (a component with area > maxarea goes, and so
//      do the components next to the last background pixel when the background is larger
//      than maxarea: RemoveConnectedRegion floods from every label's last pixel, the
//      background label's included);
//   4. spots marked (outside [minlevel, maxlevel]: weight 1; else a nonzero weight) and listed;
//   5. one CTA per image runs CleanByArray's rounds: every listed spot with unmarked
//      neighbours moves by weight * (mean - value), the new values written after the round.
// The TriKernel statistics are a two-pass double reduction in a fixed order instead of the
// reference's running (Welford) update; both are exact to about 1e-15, far below the float
// rounding of the level they produce.
#include "mr_common.cuh"
#include "mr_kipl_filters.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace mr {
namespace spot2 {

constexpr float kMark = kf::kFloatMax;
using kf::mirror_at;

// RingDetection (SpotClean.cpp:402-427): 5x5 kernel with 1/12 on the ring and -1 in the
// centre, its 13 nonzero taps summed in row-major order from 0, then |.|.
__global__ void __launch_bounds__(256) k_ring(const float *__restrict__ src, int w, int h, float *__restrict__ det)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t npix = static_cast<size_t>(w) * h;
    const float *img = src + blockIdx.z * npix;
    constexpr float wv = 1.0f / 12.0f;
    constexpr int dx[13] = {-1, 0, 1, -2, 2, -2, 0, 2, -2, 2, -1, 0, 1};
    constexpr int dy[13] = {-2, -2, -2, -1, -1, 0, 0, 0, 1, 1, 2, 2, 2};
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < 13; ++t) {
        const float k = t == 6 ? -1.0f : wv;
        acc = __fadd_rn(acc, __fmul_rn(mirror_at<5, 5>(img, w, h, x, y, x + dx[t], y + dy[t]), k));
    }
    det[blockIdx.z * npix + static_cast<size_t>(y) * w + x] = fabsf(acc);
}

// |a - b| (kipl::math::abs of an image difference).
__global__ void __launch_bounds__(256) k_absdiff(const float *__restrict__ a, const float *__restrict__ b, size_t n,
                                                 float *__restrict__ out)
{
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = fabsf(__fsub_rn(a[i], b[i]));
}

// TriKernel statistics (kipl::math::statistics: mean and sqrt(sum (x - mean)^2 / N)) per image
// in two passes of fixed-order double sums: block partials, then one block per image.
constexpr int kStatBlocks = 64;

template <bool SECOND>
__global__ void __launch_bounds__(256) k_stat_partial(const float *__restrict__ f, size_t npix,
                                                      const double *__restrict__ mean, double *__restrict__ partial)
{
    __shared__ double red[256];
    const float *img = f + blockIdx.y * npix;
    const double m = SECOND ? mean[blockIdx.y] : 0.0;
    double acc = 0.0;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const double v = img[i];
        acc += SECOND ? (v - m) * (v - m) : v;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * kStatBlocks + blockIdx.x] = red[0];
}

// SECOND = false: mean = sum / N; SECOND = true: level = (float)(mean + gamma * sqrt(var)).
template <bool SECOND>
__global__ void k_stat_final(const double *__restrict__ partial, size_t npix, float gamma, double *__restrict__ mean,
                             float *__restrict__ level)
{
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int b = 0; b < kStatBlocks; ++b) s += partial[blockIdx.x * kStatBlocks + b];
    if (!SECOND) {
        mean[blockIdx.x] = s / static_cast<double>(npix);
    } else {
        const double sd = sqrt(s / static_cast<double>(npix));
        level[blockIdx.x] = static_cast<float>(mean[blockIdx.x] + static_cast<double>(gamma) * sd);
    }
}

// OneKernel's accumulation (SpotClean.cpp:478-500): det = det || (level < f).
__global__ void __launch_bounds__(256) k_tri_threshold(float *__restrict__ det, const float *__restrict__ f,
                                                       size_t npix, const float *__restrict__ level)
{
    const float lv = level[blockIdx.y];
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = blockIdx.y * npix + i;
        det[j] = (det[j] != 0.0f || lv < f[j]) ? 1.0f : 0.0f;
    }
}

// LUTbase::BasicLUT (LUTbase.cpp:57-75) of SigmoidLUT(1 << 15, gamma, sigma), index clamped to
// the table (the reference reads past it on a NaN or through cancellation).
__global__ void __launch_bounds__(256) k_lut(float *__restrict__ v, size_t n, const float *__restrict__ table, int len)
{
    const float lo = table[len], hi = table[len + 1], slope = table[len + 2], icpt = table[len + 3];
    for (size_t j = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
         j += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float x = v[j];
        float r;
        if (x < lo) {
            r = table[0];
        } else if (hi < x) {
            r = table[len - 1];
        } else {
            const float f = __fadd_rn(__fmul_rn(x, slope), icpt);
            int idx = 0;
            if (f >= static_cast<float>(len)) idx = len - 1;
            else if (f >= 0.0f) idx = min(static_cast<int>(f), len - 1);
            r = table[idx];
        }
        v[j] = r;
    }
}

// ------------------------------------------------------------ connected components

// Union-find over pixel indices of one image: parents only decrease (a root is linked under
// the smaller root by atomicMin), so every find ends; a union retries only when another thread
// changed the root it tried to link, which lowers that root, so retries are finite as well.
__device__ __forceinline__ int uf_find(const volatile int *L, int x)
{
    int p = L[x];
    while (p != x) {
        x = p;
        p = L[x];
    }
    return x;
}

__device__ void uf_union(int *L, int a, int b)
{
    for (;;) {
        a = uf_find(L, a);
        b = uf_find(L, b);
        if (a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(L + b, a);
        if (old == b) return;
        b = old;
    }
}

// label = own index on the nonzero weights (kipl thresholds them with != 0, NaN included), -1
// elsewhere; per-image counters zeroed.
__global__ void __launch_bounds__(256) k_cc_init(const float *__restrict__ det, int w, int h, int *__restrict__ lab,
                                                 int *__restrict__ area)
{
    const size_t npix = static_cast<size_t>(w) * h;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = blockIdx.y * npix + i;
        lab[j] = det[j] != 0.0f ? static_cast<int>(i) : -1;
        area[j] = 0;
    }
}

// 8-connectivity: each pixel unites with its left, upper-left, upper and upper-right
// neighbours inside the image (kipl's CNeighborhood rejects positions outside it).
__global__ void __launch_bounds__(256) k_cc_union(int *__restrict__ lab, int w, int h)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    if (x >= w || y >= h) return;
    int *L = lab + blockIdx.z * static_cast<size_t>(w) * h;
    const int i = y * w + x;
    if (L[i] < 0) return;
    if (x > 0 && L[i - 1] >= 0) uf_union(L, i, i - 1);
    if (y > 0) {
        if (x > 0 && L[i - w - 1] >= 0) uf_union(L, i, i - w - 1);
        if (L[i - w] >= 0) uf_union(L, i, i - w);
        if (x + 1 < w && L[i - w + 1] >= 0) uf_union(L, i, i - w + 1);
    }
}

// Roots, component areas, the background count and the last background index (LabelArea).
// stat per image: [0] background count, [1] last background index (-1 if none),
// [2] status, [3] spot count.
__global__ void __launch_bounds__(256) k_cc_area(int *__restrict__ lab, int w, int h, int *__restrict__ area,
                                                 int *__restrict__ stat)
{
    const size_t npix = static_cast<size_t>(w) * h;
    int *L = lab + blockIdx.y * npix;
    int *A = area + blockIdx.y * npix;
    int *S = stat + blockIdx.y * 4;
    int bg = 0, last = -1;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        if (L[i] < 0) {
            ++bg;
            last = static_cast<int>(i);
        } else {
            atomicAdd(A + uf_find(L, static_cast<int>(i)), 1);
        }
    }
    if (bg) atomicAdd(S, bg);
    if (last >= 0) atomicMax(S + 1, last);
}

// RemoveConnectedRegion's flood from the background's last pixel: the components next to it
// are removed (flagged by a negative area) when the background is larger than maxarea.
__global__ void k_cc_background(const int *__restrict__ lab, int w, int h, int *__restrict__ area,
                                const int *__restrict__ stat, int maxarea)
{
    if (threadIdx.x != 0) return;
    const size_t npix = static_cast<size_t>(w) * h;
    const int *L = lab + blockIdx.x * npix;
    int *A = area + blockIdx.x * npix;
    const int *S = stat + blockIdx.x * 4;
    const int last = S[1];
    if (last < 0 || !(static_cast<size_t>(maxarea) < static_cast<size_t>(S[0]))) return;
    const int x = last % w, y = last / w;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx, yy = y + dy;
            if ((dx || dy) && xx >= 0 && xx < w && yy >= 0 && yy < h && L[yy * w + xx] >= 0)
                A[uf_find(L, yy * w + xx)] = -1;
        }
}

// Weights of removed components (area > maxarea, or flagged) become 0.
__global__ void __launch_bounds__(256) k_cc_apply(float *__restrict__ det, const int *__restrict__ lab, int w, int h,
                                                  const int *__restrict__ area, int maxarea)
{
    const size_t npix = static_cast<size_t>(w) * h;
    const int *L = lab + blockIdx.y * npix;
    const int *A = area + blockIdx.y * npix;
    float *D = det + blockIdx.y * npix;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        if (L[i] < 0) continue;
        const int a = A[uf_find(L, static_cast<int>(i))];
        if (a < 0 || static_cast<size_t>(maxarea) < static_cast<size_t>(a)) D[i] = 0.0f;
    }
}

// --------------------------------------------------------------------- spots

// DetectSpots' marking (SpotClean.cpp:219-232): outside [minlevel, maxlevel] weight 1, else a
// nonzero weight; the original value kept, the pixel marked with FLT_MAX, its index listed.
__global__ void __launch_bounds__(256) k_mark(float *__restrict__ proj, float *__restrict__ det, size_t npix,
                                              float minlevel, float maxlevel, float *__restrict__ orig,
                                              int *__restrict__ list, int *__restrict__ stat)
{
    float *P = proj + blockIdx.y * npix;
    float *D = det + blockIdx.y * npix;
    float *O = orig + blockIdx.y * npix;
    int *Lst = list + blockIdx.y * npix;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < npix;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float v = P[i];
        float wt;
        if (v < minlevel || maxlevel < v) wt = 1.0f;
        else if (D[i] != 0.0f) wt = D[i];
        else continue;
        D[i] = wt;
        O[i] = v;
        P[i] = kMark;
        Lst[atomicAdd(stat + blockIdx.y * 4 + 3, 1)] = static_cast<int>(i);
    }
}

// CleanByArray (SpotClean.cpp:287-336) for one image per CTA. Neighbours are the linear offsets
// {-w-1, -w, -w+1, -1, 1, w-1, w, w+1} from PrepareNeighborhood; Neighborhood (:350-365) starts
// at the 4th for indices up to w (the 5th at index 0) and stops after the 5th in the last row;
// an index past the image end reads 0. Every round reads the image as it was when the round
// began (corrected values are written after it), so the list order does not matter. A round
// that corrects nothing while spots remain sets status 1 (the reference loops forever); spots
// only leave the list, so there are at most as many rounds as spots.
__global__ void __launch_bounds__(512) k_clean(float *__restrict__ proj, int w, int h, const float *__restrict__ det,
                                               const float *__restrict__ orig, float *__restrict__ newv,
                                               int *__restrict__ list0, int *__restrict__ list1,
                                               int *__restrict__ stat)
{
    __shared__ int s_next, s_corr;
    const size_t npix = static_cast<size_t>(w) * h;
    float *P = proj + blockIdx.x * npix;
    const float *D = det + blockIdx.x * npix, *O = orig + blockIdx.x * npix;
    float *NV = newv + blockIdx.x * npix;
    int *cur = list0 + blockIdx.x * npix, *nxt = list1 + blockIdx.x * npix;
    int *S = stat + blockIdx.x * 4;
    int count = S[3];
    const long long n = static_cast<long long>(npix), first_line = w, last_line = n - w;
    const long long off[8] = {-w - 1, -w, -w + 1, -1, 1, w - 1, w, w + 1};
    while (count > 0) {
        if (threadIdx.x == 0) {
            s_next = 0;
            s_corr = 0;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < count; k += blockDim.x) {
            const int pos = cur[k];
            const long long idx = pos;
            const int start = first_line < idx ? 0 : (idx != 0 ? 3 : 4);
            const int stop = idx < last_line ? 8 : 5;
            float sum = 0.0f;
            int cnt = 0;
            for (int t = start; t < stop; ++t) {
                const long long q = idx + off[t];
                const float v = q < n ? P[q] : 0.0f;
                if (v != kMark) {
                    sum = __fadd_rn(sum, v);
                    ++cnt;
                }
            }
            if (cnt) {
                const float mean = __fdiv_rn(sum, static_cast<float>(cnt));
                const float val = O[pos];
                NV[pos] = __fadd_rn(val, __fmul_rn(D[pos], __fsub_rn(mean, val)));
                cur[k] = -pos - 1;
                atomicAdd(&s_corr, 1);
            } else {
                nxt[atomicAdd(&s_next, 1)] = pos;
            }
        }
        __syncthreads();
        const int corrected = s_corr, remaining = s_next;
        if (corrected == 0) {
            if (threadIdx.x == 0) S[2] = 1;
            return;
        }
        for (int k = threadIdx.x; k < count; k += blockDim.x) {
            const int c = cur[k];
            if (c < 0) P[-c - 1] = NV[-c - 1];
        }
        __syncthreads();
        int *t = cur;
        cur = nxt;
        nxt = t;
        count = remaining;
    }
}

} // namespace spot2

extern "C" mr_status mr_median_filter(const float *img_d, size_t nu, size_t nv, size_t nimg, int kx, int ky,
                                      float *out_d, void *stream);
extern "C" mr_status mr_sigmoid_lut(size_t len, float lambda, float sigma, float *lut_h, float *param_h);

namespace {

using kf::box;
using kf::line;
unsigned ew_blocks(size_t n) { return kf::flat_blocks(n); }

// Detection image of nimg projections into det; X1..X3 are scratch images of the batch.
mr_status detection(const float *img, int w, int h, unsigned nimg, int method, float gamma, float *det, float *X1,
                    float *X2, float *X3, double *stats, float *level, cudaStream_t s)
{
    using namespace spot2;
    const size_t npix = static_cast<size_t>(w) * h, n = npix * nimg;
    const dim3 grid(div_up(w, 32), div_up(h, 8), nimg), block(32, 8);
    switch (method) {
    case MR_SPOT_RING:
        k_ring<<<grid, block, 0, s>>>(img, w, h, det);
        break;
    case MR_SPOT_STDDEV:
        kf::stddev_filter<3>(img, w, h, nimg, X1, X3, X2, det, s);
        break;
    case MR_SPOT_MEDIAN: {
        mr_status st = mr_median_filter(img, w, h, nimg, 1, 5, X1, s);
        if (st == MR_OK) st = mr_median_filter(X1, w, h, nimg, 5, 1, X2, s);
        if (st != MR_OK) return st;
        k_absdiff<<<ew_blocks(n), 256, 0, s>>>(img, X2, n, det);
        break;
    }
    case MR_SPOT_MINMAX:
        line<5, true, kf::OP_MIN>(img, w, h, nimg, X1, s);
        line<5, false, kf::OP_MIN>(X1, w, h, nimg, X2, s);
        line<5, true, kf::OP_MAX>(img, w, h, nimg, X1, s);
        line<5, false, kf::OP_MAX>(X1, w, h, nimg, X3, s);
        k_absdiff<<<ew_blocks(n), 256, 0, s>>>(X3, X2, n, det);
        break;
    case MR_SPOT_TRIKERNEL: {
        MR_CUDA_TRY(cudaMemsetAsync(det, 0, n * sizeof(float), s));
        double *partial = stats, *mean = stats + static_cast<size_t>(nimg) * kStatBlocks;
        for (int size = 3; size <= 7; size += 2) {
            box(img, w, h, nimg, size, X3, X1, s);
            k_absdiff<<<ew_blocks(n), 256, 0, s>>>(img, X1, n, X2);
            k_stat_partial<false><<<dim3(kStatBlocks, nimg), 256, 0, s>>>(X2, npix, mean, partial);
            k_stat_final<false><<<nimg, 32, 0, s>>>(partial, npix, gamma, mean, level);
            k_stat_partial<true><<<dim3(kStatBlocks, nimg), 256, 0, s>>>(X2, npix, mean, partial);
            k_stat_final<true><<<nimg, 32, 0, s>>>(partial, npix, gamma, mean, level);
            k_tri_threshold<<<dim3(std::min<unsigned>(div_up(npix, 256), 1024), nimg), 256, 0, s>>>(det, X2, npix,
                                                                                                     level);
        }
        break;
    }
    default:
        return fail(MR_ERR_ARGUMENT, "mr_spotclean2: unknown detection method %d", method);
    }
    return check_launch("spot detection");
}

} // namespace

} // namespace mr

using namespace mr;

extern "C" mr_status mr_spotclean2(float *proj_d, size_t nu, size_t nv, size_t nproj, int method, float gamma,
                                   float sigma, int iterations, float minlevel, float maxlevel, int maxarea,
                                   void *stream)
{
    MR_TRACE();
    using namespace spot2;
    if (!proj_d) return fail(MR_ERR_ARGUMENT, "mr_spotclean2: null pointer");
    if (nu < 16 || nv < 16 || nu * nv > (size_t(1) << 31) - 1)
        return fail(MR_ERR_ARGUMENT, "mr_spotclean2: projections of %zux%zu (16 to 2^31 pixels, 16 wide and high)",
                    nu, nv);
    if (method < MR_SPOT_STDDEV || method > MR_SPOT_TRIKERNEL)
        return fail(MR_ERR_ARGUMENT, "mr_spotclean2: unknown detection method %d", method);
    if (!(sigma > 0.0f) || !std::isfinite(sigma) || !std::isfinite(gamma))
        return fail(MR_ERR_ARGUMENT, "mr_spotclean2: sigma must be positive and finite");
    if (nproj == 0 || iterations <= 0) return MR_OK;
    cudaStream_t s = as_stream(stream);
    const int w = static_cast<int>(nu), h = static_cast<int>(nv);
    const size_t npix = nu * nv, len = size_t(1) << 15;
    std::vector<float> table(len + 4);
    mr_sigmoid_lut(len, gamma, sigma, table.data(), table.data() + len);
    // batch: five float/int images per projection, about 1 GiB in all
    const size_t per = 5 * npix * sizeof(float);
    const unsigned batch = static_cast<unsigned>(
        std::max<size_t>(1, std::min<size_t>({nproj, (size_t(1) << 30) / per, 65535})));
    const size_t bytes = (len + 4) * sizeof(float) + static_cast<size_t>(batch) * per +
                         static_cast<size_t>(batch) * (4 * sizeof(int) + sizeof(float)) +
                         static_cast<size_t>(batch) * (kStatBlocks + 1) * sizeof(double);
    char *work = nullptr;
    MR_TRY(device_alloc(&work, bytes, s, "mr_spotclean2: scratch"));
    double *stats = reinterpret_cast<double *>(work);
    float *lut = reinterpret_cast<float *>(stats + static_cast<size_t>(batch) * (kStatBlocks + 1));
    float *X0 = lut + len + 4;
    float *X1 = X0 + batch * npix, *X2 = X1 + batch * npix, *X3 = X2 + batch * npix, *X4 = X3 + batch * npix;
    int *stat = reinterpret_cast<int *>(X4 + batch * npix);
    float *level = reinterpret_cast<float *>(stat + 4 * static_cast<size_t>(batch));
    mr_status st = MR_OK;
    cudaError_t e = cudaMemcpyAsync(lut, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = fail(MR_ERR_CUDA, "mr_spotclean2: table upload: %s", cudaGetErrorString(e));
    std::vector<int> stat_h(4 * static_cast<size_t>(batch));
    for (int it = 0; it < iterations && st == MR_OK; ++it) {
        for (size_t i0 = 0; i0 < nproj && st == MR_OK; i0 += batch) {
            const unsigned b = static_cast<unsigned>(std::min<size_t>(batch, nproj - i0));
            float *P = proj_d + i0 * npix;
            const size_t n = npix * b;
            const dim3 grid(div_up(w, 32), div_up(h, 8), b), block(32, 8), flat(std::min<unsigned>(div_up(npix, 256), 1024), b);
            st = detection(P, w, h, b, method, gamma, X0, X1, X2, X3, stats, level, s);
            if (st != MR_OK) break;
            k_lut<<<ew_blocks(n), 256, 0, s>>>(X0, n, lut, static_cast<int>(len));
            e = cudaMemsetAsync(stat, 0, 4 * sizeof(int) * b, s);
            if (e == cudaSuccess) {
                // last background index starts at -1 (no background)
                std::vector<int> init(4 * static_cast<size_t>(b), 0);
                for (unsigned k = 0; k < b; ++k) init[4 * k + 1] = -1;
                e = cudaMemcpyAsync(stat, init.data(), init.size() * sizeof(int), cudaMemcpyHostToDevice, s);
            }
            if (e != cudaSuccess) {
                st = fail(MR_ERR_CUDA, "mr_spotclean2: %s", cudaGetErrorString(e));
                break;
            }
            int *lab = reinterpret_cast<int *>(X1), *area = reinterpret_cast<int *>(X2);
            if (maxarea != 0) {
                k_cc_init<<<flat, 256, 0, s>>>(X0, w, h, lab, area);
                k_cc_union<<<grid, block, 0, s>>>(lab, w, h);
                k_cc_area<<<flat, 256, 0, s>>>(lab, w, h, area, stat);
                k_cc_background<<<b, 32, 0, s>>>(lab, w, h, area, stat, maxarea);
                k_cc_apply<<<flat, 256, 0, s>>>(X0, lab, w, h, area, maxarea);
            }
            // lists reuse the label and area images; original values in X3, new values in X4
            k_mark<<<flat, 256, 0, s>>>(P, X0, npix, minlevel, maxlevel, X3, lab, stat);
            k_clean<<<b, 512, 0, s>>>(P, w, h, X0, X3, X4, lab, area, stat);
            st = check_launch("mr_spotclean2");
            if (st != MR_OK) break;
            e = cudaMemcpyAsync(stat_h.data(), stat, 4 * sizeof(int) * b, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                st = fail(MR_ERR_CUDA, "mr_spotclean2: %s", cudaGetErrorString(e));
                break;
            }
            for (unsigned k = 0; k < b; ++k)
                if (stat_h[4 * k + 2]) {
                    st = fail(MR_ERR_DEVICE,
                              "mr_spotclean2: projection %zu: spots with no unmarked neighbour remain (the reference "
                              "loops forever here)",
                              i0 + k);
                    break;
                }
        }
    }
    cudaFreeAsync(work, s);
    return st;
}
