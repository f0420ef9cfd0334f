// Row filters: ProjectionFilterSingle and the FDK ramp filter, as one batched FFT kernel.
//
// Both reference filters are linear, shift-invariant filters of zero/taper-padded detector
// rows with a real, even frequency response:
//   ProjectionFilterSingle (frameworks/tomography/Preprocessing/StdPreprocModules/src/
//     ProjectionFilter.cpp:301-362): r2c of the padded row, bins 0..N/2-1 times the filter,
//     bin N/2 untouched, c2r. As a full-length response: H[k] = filter[min(k, N-k)],
//     H[N/2] = 1.
//   FDKbp_single::ramp_filter_tuned (frameworks/tomography/Backprojectors/
//     FDKBackProjectors/src/fdkbp_single.cpp:832-958): c2c of the padded row times the
//     ramp on all bins, inverse, real part; ramp[k] = ramp[N-k].
// A real even response maps the spectrum of a real row to a Hermitian spectrum, so two
// rows are filtered together as the real and imaginary parts of one complex row (one
// forward and one inverse complex FFT per two rows, no real-FFT pre/post twiddles).
//
// Kernel: one CTA per pair of rows. The padded complex row is built in shared memory in
// bit-reversed order, transformed with in-place radix-2 decimation-in-time stages,
// multiplied by H, transformed back with decimation-in-frequency stages (natural in,
// bit-reversed out) and the crop window is gathered out. Twiddles are a float2 table
// exp(-2 pi i k / N), k < N/2, built in double on the host.
#include "mr_common.cuh"
#include "mr_fft.cuh"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace mr {

// kipl math constants (core/kipl/kipl/include/math/mathconstants.h:7-8)
static const double kDPi = 3.1415926535897932384626433832795028841971693993751;
static const float kFPi = 3.1415926535897932384626f;

enum PadMode { kPadProjFilter = 0, kPadFdk = 1, kPadProjCore = 2 };

struct RowFilterArgs {
    const float *in;
    float *out;           // f32 output (or NULL when out16 is used)
    uint16_t *out16;      // 16-bit output (bf16/f16 bits), NULL for f32
    const float *out_scale_inv; // per-projection 1/scale for 16-bit output
    const float2 *twiddle;
    const float *response; // full-length real response H[k], k < n
    const float *pad;      // projection filter taper (ninsert values)
    const float *tl, *tr;  // projection filter, short form: the tapers' responses per output column
    const float *row_weight;
    size_t rows_per_weight;
    size_t nrows;
    int nu;          // row length (detector columns)
    int nv;          // rows per projection held (FDK edge-row replication)
    int row0;        // FDK: absolute detector row of the first row held
    int nvfull;      // FDK: detector rows of the whole projection
    int n;           // FFT length
    int logn;
    int ninsert;     // projection filter: data offset; FDK: pad_factor/2
    int mode;
    int out16_kind;  // MR_BF16 / MR_F16
    float scale;     // projection filter: pi/(4*N/2); FDK: 1/padwidth
    float post1, post2; // FDK: sad_sid_2, scale (two sequential products); 1 for the projection filter
};

// Value of padded position p (0 <= p < n) of one row, reference padding rules.
__device__ __forceinline__ float padded_value(const RowFilterArgs &a, const float *row, size_t rowidx, int p)
{
    if (a.mode == kPadProjCore) return p < a.nu ? row[p] : 0.0f; // the row alone, zero-padded
    if (a.mode == kPadProjFilter) {
        // ProjectionFilterSingle::Pad (:346-362): dest length n+16; data at ninsert;
        // left taper dest[i] = src[0]*pad[i]; right taper dest[n+15-i] = src[nu-1]*pad[i]
        // (written last), only the first n entries reach the FFT.
        const int ins = a.ninsert;
        const int ri = a.n + 15 - p; // right-taper index if in range
        if (ri >= 0 && ri < ins) return __fmul_rn(row[a.nu - 1], a.pad[ri]);
        if (p < ins) return __fmul_rn(row[0], a.pad[p]);
        const int q = p - ins;
        return q < a.nu ? row[q] : 0.0f;
    } else {
        // ramp_filter_tuned (:850-888): zero pad with the row at pad_factor/2, first and
        // last 5 columns replicated from columns 5 and n-6 (replication of rows is done by
        // the caller choosing the source row).
        int c = p;
        if (c < 5) c = 5;
        if (c >= a.n - 5) c = a.n - 6;
        const int q = c - a.ninsert;
        if (q < 0 || q >= a.nu) return 0.0f;
        float v = row[q];
        if (a.row_weight) v = __fmul_rn(v, a.row_weight[rowidx / a.rows_per_weight]); // img *= weight
        return v;
    }
}

// FDK edge-row replication (ramp_filter_tuned :874-880): detector rows 0..4 take row 5, rows
// nvfull-5..nvfull-1 take row nvfull-6 (after the first copy). The rows held are the window
// [row0, row0 + nv) of each projection (the whole detector: row0 = 0, nvfull = nv); the rule
// applies to the absolute rows and the callers check that every source row is in the window.
__device__ __forceinline__ size_t fdk_source_row(size_t r, int nv, int row0, int nvfull)
{
    const size_t proj = r / nv;
    int v = static_cast<int>(r - proj * nv) + row0;
    if (v >= nvfull - 5) {
        int q = nvfull - 6;
        v = q < 5 ? 5 : q;
    } else if (v < 5) {
        v = 5;
    }
    return proj * nv + (v - row0);
}

__global__ void __launch_bounds__(512) k_rowfilter(RowFilterArgs a)
{
    extern __shared__ float2 buf[];
    const size_t r0 = 2 * static_cast<size_t>(blockIdx.x);
    const size_t r1 = r0 + 1;
    const bool has1 = r1 < a.nrows;
    const int n = a.n;
    const size_t src0 = a.mode == kPadFdk ? fdk_source_row(r0, a.nv, a.row0, a.nvfull) : r0;
    const size_t src1 = a.mode == kPadFdk ? fdk_source_row(r1, a.nv, a.row0, a.nvfull) : r1;
    const float *row0 = a.in + src0 * a.nu;
    const float *row1 = a.in + src1 * a.nu;

    // padded complex row (two real rows as re/im), natural order
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        float x0 = padded_value(a, row0, r0, p);
        float x1 = has1 ? padded_value(a, row1, r1, p) : 0.0f;
        buf[fft_slot(p)] = make_float2(x0, x1);
    }
    __syncthreads();

    fft_forward(buf, a.logn, a.twiddle);
    fft_apply_response(buf, n, a.response);
    fft_inverse(buf, a.logn, a.twiddle);

    // crop and write
    const float l0 = a.mode == kPadProjCore ? row0[0] : 0.0f, r0v = a.mode == kPadProjCore ? row0[a.nu - 1] : 0.0f;
    const float l1 = a.mode == kPadProjCore && has1 ? row1[0] : 0.0f;
    const float r1v = a.mode == kPadProjCore && has1 ? row1[a.nu - 1] : 0.0f;
    for (int i = threadIdx.x; i < a.nu; i += blockDim.x) {
        float2 v = buf[fft_slot(i + (a.mode == kPadProjCore ? 0 : a.ninsert))];
        if (a.mode == kPadProjCore) {
            // the row's part plus the tapers' (scaled by the edge samples they repeat)
            const float tl = a.tl[i], tr = a.tr[i];
            v.x = __fadd_rn(__fadd_rn(v.x, __fmul_rn(l0, tl)), __fmul_rn(r0v, tr));
            v.y = __fadd_rn(__fadd_rn(v.y, __fmul_rn(l1, tl)), __fmul_rn(r1v, tr));
        }
        float y0 = __fmul_rn(v.x, a.scale);
        float y1 = __fmul_rn(v.y, a.scale);
        if (a.mode != kPadFdk) {
            if (a.row_weight) {
                y0 = __fmul_rn(y0, a.row_weight[r0 / a.rows_per_weight]);
                if (has1) y1 = __fmul_rn(y1, a.row_weight[r1 / a.rows_per_weight]);
            }
        } else {
            y0 = __fmul_rn(__fmul_rn(y0, a.post1), a.post2);
            y1 = __fmul_rn(__fmul_rn(y1, a.post1), a.post2);
        }
        if (a.out16) {
            const float s0 = a.out_scale_inv[r0 / a.nv];
            const float s1 = has1 ? a.out_scale_inv[r1 / a.nv] : 0.0f;
            if (a.out16_kind == MR_BF16) {
                a.out16[r0 * a.nu + i] = __bfloat16_as_ushort(__float2bfloat16_rn(y0 * s0));
                if (has1) a.out16[r1 * a.nu + i] = __bfloat16_as_ushort(__float2bfloat16_rn(y1 * s1));
            } else {
                a.out16[r0 * a.nu + i] = __half_as_ushort(__float2half_rn(y0 * s0));
                if (has1) a.out16[r1 * a.nu + i] = __half_as_ushort(__float2half_rn(y1 * s1));
            }
        } else {
            a.out[r0 * a.nu + i] = y0;
            if (has1) a.out[r1 * a.nu + i] = y1;
        }
    }
}

static size_t next_pow2_size(size_t n)
{
    size_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

static int ilog2(size_t n)
{
    int l = 0;
    while ((static_cast<size_t>(1) << l) < n) ++l;
    return l;
}

mr_status launch_rowfilter(RowFilterArgs a, cudaStream_t s)
{
    if (a.nrows == 0) return MR_OK;
    const size_t smem = static_cast<size_t>(fft_buffer_slots(a.n)) * sizeof(float2);
    static bool attr_set = false;
    if (!attr_set) {
        MR_CUDA_TRY(cudaFuncSetAttribute(k_rowfilter, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set = true;
    }
    const unsigned threads = static_cast<unsigned>(std::min(512, std::max(64, a.n / 8))); // one radix-8 butterfly each
    const size_t blocks = (a.nrows + 1) / 2;
    if (blocks > 0x7fffffffu) return fail(MR_ERR_ARGUMENT, "row filter: too many rows in one call");
    k_rowfilter<<<static_cast<unsigned>(blocks), threads, smem, s>>>(a);
    return check_launch("k_rowfilter");
}

// Per-projection power-of-two scale for 16-bit storage: the largest |value| maps below
// 2^14 (f16) or 2^100 (bf16, range is never the issue; the scale keeps one code path).
__global__ void k_absmax(const float *__restrict__ x, size_t per, float *__restrict__ amax)
{
    const float *p = x + blockIdx.y * per;
    float m = 0.0f;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < per;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        m = fmaxf(m, fabsf(p[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(amax + blockIdx.y), __float_as_int(m));
}

__global__ void k_pow2_scales(const float *__restrict__ amax, size_t nproj, int kind, float *__restrict__ scale,
                              float *__restrict__ scale_inv)
{
    size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= nproj) return;
    const float m = amax[i];
    int e = 0;
    if (m > 0.0f && isfinite(m)) {
        frexpf(m, &e); // m = f * 2^e, f in [0.5, 1)
        e -= kind == MR_F16 ? 14 : 0;
    }
    scale[i] = ldexpf(1.0f, e);
    scale_inv[i] = ldexpf(1.0f, -e);
}

template <int KIND>
__global__ void k_quantize(const float *__restrict__ x, size_t per, size_t total, const float *__restrict__ scale_inv,
                           uint16_t *__restrict__ out)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float v = x[i] * scale_inv[i / per];
        out[i] = KIND == MR_BF16 ? __bfloat16_as_ushort(__float2bfloat16_rn(v)) : __half_as_ushort(__float2half_rn(v));
    }
}

// Quantize nproj projections of `per` floats to 16 bits with per-projection scales.
mr_status quantize_projections(const float *x_d, size_t per, size_t nproj, int kind, uint16_t *out_d, float *scale_d,
                               cudaStream_t s)
{
    float *amax = nullptr, *inv = nullptr;
    MR_TRY(device_alloc(&amax, 2 * nproj * sizeof(float), s, "16-bit quantisation: scratch"));
    inv = amax + nproj;
    mr_status st = MR_OK;
    if (cudaMemsetAsync(amax, 0, nproj * sizeof(float), s) != cudaSuccess) st = fail(MR_ERR_CUDA, "memset");
    if (st == MR_OK) {
        dim3 g(std::min<unsigned>(div_up(per, 256), 64u), static_cast<unsigned>(nproj));
        k_absmax<<<g, 256, 0, s>>>(x_d, per, amax);
        st = check_launch("k_absmax");
    }
    if (st == MR_OK) {
        k_pow2_scales<<<div_up(nproj, 128), 128, 0, s>>>(amax, nproj, kind, scale_d, inv);
        st = check_launch("k_pow2_scales");
    }
    if (st == MR_OK) {
        const size_t total = per * nproj;
        const unsigned blocks = std::min<unsigned>(div_up(total, 256), 148u * 16u);
        if (kind == MR_BF16)
            k_quantize<MR_BF16><<<blocks, 256, 0, s>>>(x_d, per, total, inv, out_d);
        else
            k_quantize<MR_F16><<<blocks, 256, 0, s>>>(x_d, per, total, inv, out_d);
        st = check_launch("k_quantize");
    }
    cudaFreeAsync(amax, s);
    return st;
}

// ---- allocation-free quantization (mr_quantize_noalloc)
//
// Scratch of the no-allocation entry point: the per-projection |max| (kQuantScratchMax
// floats) followed by the reciprocal scales (kQuantScratchMax floats), 512 KiB in all.
// Every device that loads this library holds the array until the process exits.
constexpr size_t kQuantScratchMax = 65536;
static __device__ __align__(256) float g_quant_scratch[2 * kQuantScratchMax];

// Device address of g_quant_scratch per device ordinal, looked up on the first call made
// with that device current. In host code the symbol itself is only a host-side stand-in,
// never a device address, so kernels always receive the looked-up pointer. The cache lives
// as long as the process; a cudaDeviceReset makes the cached address stale (documented in
// the header).
static float *quant_scratch_ptr(int device, mr_status *st)
{
    constexpr int kMaxDevices = 64;
    static float *ptrs[kMaxDevices] = {};
    static std::mutex mu;
    if (device < 0 || device >= kMaxDevices) {
        *st = fail(MR_ERR_UNSUPPORTED, "mr_quantize_noalloc: device ordinal %d above %d", device, kMaxDevices - 1);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_quant_scratch);
        if (e != cudaSuccess || !p) {
            *st = fail(MR_ERR_CUDA, "mr_quantize_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
        ptrs[device] = static_cast<float *>(p);
    }
    *st = MR_OK;
    return ptrs[device];
}

} // namespace mr

using namespace mr;

struct mr_filter_plan {
    size_t nu = 0, nfft = 0, ninsert = 0;
    size_t m = 0; // transform length on the device (m < nfft: the short form)
    std::vector<float> filter, pad;
    float2 *twiddle_d = nullptr;
    float *response_d = nullptr;
    float *pad_d = nullptr;
    float *tl_d = nullptr, *tr_d = nullptr; // short form: taper responses per output column
};

extern "C" {

mr_status mr_projfilter_tables(size_t nu, const char *filtertype, float cutoff, float order, int usebias,
                               float biasweight, int paddingdoubler, size_t *nfft_out, size_t *ninsert_out,
                               float *filter_h, float *pad_h)
{
    MR_TRACE();
    if (!filtertype) return fail(MR_ERR_ARGUMENT, "mr_projfilter_tables: null filter type");
    if (nu < 2) return fail(MR_ERR_ARGUMENT, "mr_projfilter_tables: row length must be at least 2");
    if (paddingdoubler < 0 || paddingdoubler > 4) return fail(MR_ERR_ARGUMENT, "mr_projfilter_tables: paddingdoubler out of range");
    std::string ft(filtertype);
    std::transform(ft.begin(), ft.end(), ft.begin(), [](unsigned char c) { return std::tolower(c); });
    int type;
    // string2enum(ProjectionFilterBase::FilterType) (ProjectionFilter.cpp:33-48)
    if (ft == "ram-lak") type = 0;
    else if (ft == "shepp-logan") type = 1;
    else if (ft == "hanning") type = 2;
    else if (ft == "hamming") type = 3;
    else if (ft == "butterworth") type = 4;
    else return fail(MR_ERR_ARGUMENT, "Could not convert filter string to enum.");
    // ComputeFilterSize (:120-125)
    const double e = std::log(static_cast<double>(nu)) / std::log(2.0);
    const size_t nfft = static_cast<size_t>(1) << (static_cast<size_t>(std::ceil(e)) + static_cast<size_t>(paddingdoubler));
    if (nfft > 16384) return fail(MR_ERR_UNSUPPORTED, "mr_projfilter: FFT length %zu above 16384", nfft);
    const size_t n2 = nfft / 2;
    if (!((0 < cutoff) && (cutoff <= 0.5f))) return fail(MR_ERR_ARGUMENT, "Cut off frequency is not in valid range");
    const size_t ins = n2 - nu / 2;
    if (nfft_out) *nfft_out = nfft;
    if (ninsert_out) *ninsert_out = ins;
    if (!filter_h) return MR_OK;
    // BuildFilter (:254-299), same float expressions
    float *filter = filter_h;
    for (size_t i = 0; i < n2; ++i) filter[i] = 0.0f;
    const float forder = type == 4 ? order : 0.0f;
    const size_t cut = static_cast<size_t>(2 * cutoff * n2);
    const float rampstep = 1.0f / ((n2 - 1.0f));
    for (size_t i = 0; i < n2; ++i) filter[i] = i * rampstep;
    const float fstep = 1.0f / ((cut - 1.0f));
    for (size_t i = 0; i < cut && i < n2; ++i) {
        switch (type) {
        case 0: break;
        case 1: filter[i] = static_cast<float>(std::sin(kDPi * i * fstep * cutoff)) / n2; break;
        case 2: filter[i] *= static_cast<float>(0.5f + 0.5f * std::cos(i * fstep * kFPi * cutoff)); break;
        case 3: filter[i] *= static_cast<float>(0.54 + 0.46 * std::cos(i * fstep * kDPi * cutoff)); break;
        case 4: filter[i] /= static_cast<float>(1 + std::pow(i * fstep * cutoff, forder)); break;
        }
    }
    for (size_t i = cut; i < n2; ++i) filter[i] = 0.0f;
    if (usebias) filter[0] = biasweight * filter[1];
    // PreparePadding (:364-376) with kipl::math::Sigmoid(x, 0, 0.07)
    if (pad_h)
        for (size_t i = 0; i < ins; ++i) {
            float x = static_cast<float>(i) / static_cast<float>(ins) - 0.5f;
            pad_h[i] = static_cast<float>(1.0 / (1.0 + std::exp(-(x - 0.0f) / 0.07f)));
        }
    return MR_OK;
}

mr_status mr_projfilter_create(size_t nu, const char *filtertype, float cutoff, float order, int usebias,
                               float biasweight, int paddingdoubler, mr_filter_plan **plan)
{
    MR_TRACE();
    if (!plan) return fail(MR_ERR_ARGUMENT, "mr_projfilter_create: null pointer");
    *plan = nullptr;
    size_t nfft = 0, ins = 0;
    mr_status st = mr_projfilter_tables(nu, filtertype, cutoff, order, usebias, biasweight, paddingdoubler, &nfft, &ins,
                                        nullptr, nullptr);
    if (st != MR_OK) return st;
    const size_t n2 = nfft / 2;
    std::vector<float> filter(n2), pad(ins);
    st = mr_projfilter_tables(nu, filtertype, cutoff, order, usebias, biasweight, paddingdoubler, &nfft, &ins,
                              filter.data(), pad.data());
    if (st != MR_OK) return st;
    // full-length response: filter on 0..n2-1 and mirrored, Nyquist bin passes
    std::vector<float> full(nfft);
    for (size_t k = 0; k < nfft; ++k) full[k] = k == n2 ? 1.0f : filter[k < n2 ? k : nfft - k];
    // Short form. The reference's output column i is sum_p h[(i + ins - p) mod N] d[p] over the
    // padded row d (the row at ins, the left taper row[0] * pad[p] before it, the right taper
    // row[nu-1] * pad[N + 15 - p] after it), h = IDFT_N(full) (unnormalised). Split by source:
    // the row's part needs h only at lags |l| < nu, i.e. a circular convolution of length
    // M >= 2 nu - 1 with h cut to those lags (response DFT_M(h cut) / M); the tapers' parts are
    // row[0] * TL[i] + row[nu-1] * TR[i] with TL, TR fixed by the configuration. All computed
    // in double. Used when M < N (the padding doubler makes N 2 to 4 times M).
    const size_t m = next_pow2_size(2 * nu - 1);
    std::vector<float> resp, tl, tr;
    size_t tlen = nfft;
    if (m < nfft) {
        tlen = m;
        std::vector<double> H(full.begin(), full.end());
        std::vector<double> h(H), hi(nfft, 0.0);
        host_dft(h, hi, +1); // h[l] = sum_k H[k] exp(+2 pi i k l / N)
        std::vector<double> g(m, 0.0), gi(m, 0.0);
        g[0] = h[0];
        for (size_t j = 1; j < nu; ++j) g[j] = g[m - j] = h[j];
        host_dft(g, gi, -1);
        resp.resize(m);
        for (size_t k = 0; k < m; ++k) resp[k] = static_cast<float>(g[k] / static_cast<double>(m));
        // taper responses: IDFT(H * DFT(taper)) at column i + ins
        auto taper_response = [&](bool left) {
            std::vector<double> t(nfft, 0.0), ti(nfft, 0.0);
            for (size_t i = 0; i < ins; ++i) {
                if (left) t[i] = pad[i];
                else if (nfft + 15 - i < nfft) t[nfft + 15 - i] = pad[i];
            }
            host_dft(t, ti, -1);
            for (size_t k = 0; k < nfft; ++k) {
                t[k] *= H[k];
                ti[k] *= H[k];
            }
            host_dft(t, ti, +1);
            std::vector<float> out(nu);
            for (size_t i = 0; i < nu; ++i) out[i] = static_cast<float>(t[(i + ins) % nfft]);
            return out;
        };
        tl = taper_response(true);
        tr = taper_response(false);
    } else {
        resp = full;
    }
    resp = fft_permute_response(resp, ilog2(tlen)); // in the order of the forward transform's output
    std::vector<float2> tw = fft_twiddles(static_cast<int>(tlen));

    mr_filter_plan *p = new mr_filter_plan;
    p->nu = nu;
    p->nfft = nfft;
    p->m = tlen;
    p->ninsert = ins;
    p->filter = filter;
    p->pad = pad;
    mr_status ast = device_alloc_sync(&p->twiddle_d, tw.size() * sizeof(float2), "mr_projfilter_create: twiddles");
    if (ast == MR_OK) ast = device_alloc_sync(&p->response_d, tlen * sizeof(float), "mr_projfilter_create: response");
    if (ast == MR_OK)
        ast = device_alloc_sync(&p->pad_d, std::max<size_t>(ins, 1) * sizeof(float), "mr_projfilter_create: pad");
    if (ast == MR_OK && !tl.empty()) ast = device_alloc_sync(&p->tl_d, nu * sizeof(float), "mr_projfilter_create: tapers");
    if (ast == MR_OK && !tr.empty()) ast = device_alloc_sync(&p->tr_d, nu * sizeof(float), "mr_projfilter_create: tapers");
    if (ast != MR_OK) {
        mr_projfilter_destroy(p);
        return ast;
    }
    cudaError_t err = cudaMemcpy(p->twiddle_d, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(p->response_d, resp.data(), tlen * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && ins)
        err = cudaMemcpy(p->pad_d, pad.data(), ins * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !tl.empty()) err = cudaMemcpy(p->tl_d, tl.data(), nu * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !tr.empty()) err = cudaMemcpy(p->tr_d, tr.data(), nu * sizeof(float), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        mr_projfilter_destroy(p);
        return fail(MR_ERR_CUDA, "mr_projfilter_create: %s", cudaGetErrorString(err));
    }
    *plan = p;
    return MR_OK;
}

mr_status mr_projfilter_destroy(mr_filter_plan *plan)
{
    MR_TRACE();
    if (!plan) return MR_OK;
    cudaFree(plan->twiddle_d);
    cudaFree(plan->response_d);
    cudaFree(plan->pad_d);
    if (plan->tl_d) cudaFree(plan->tl_d);
    if (plan->tr_d) cudaFree(plan->tr_d);
    delete plan;
    return MR_OK;
}

mr_status mr_projfilter_info(const mr_filter_plan *plan, size_t *nfft, size_t *ninsert, float *filter_h, float *pad_h)
{
    MR_TRACE();
    if (!plan) return fail(MR_ERR_ARGUMENT, "mr_projfilter_info: null plan");
    if (nfft) *nfft = plan->nfft;
    if (ninsert) *ninsert = plan->ninsert;
    if (filter_h) std::copy(plan->filter.begin(), plan->filter.end(), filter_h);
    if (pad_h) std::copy(plan->pad.begin(), plan->pad.end(), pad_h);
    return MR_OK;
}

mr_status mr_projfilter_apply(const mr_filter_plan *plan, const float *in_d, float *out_d, size_t nrows,
                              const float *row_weight_d, size_t rows_per_weight, void *stream)
{
    MR_TRACE();
    if (!plan || !in_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_projfilter_apply: null pointer");
    if (row_weight_d && rows_per_weight == 0) return fail(MR_ERR_ARGUMENT, "mr_projfilter_apply: rows_per_weight is 0");
    RowFilterArgs a{};
    a.in = in_d;
    a.out = out_d;
    a.twiddle = plan->twiddle_d;
    a.response = plan->response_d;
    a.pad = plan->pad_d;
    a.row_weight = row_weight_d;
    a.rows_per_weight = rows_per_weight ? rows_per_weight : 1;
    a.nrows = nrows;
    a.nu = static_cast<int>(plan->nu);
    a.nv = 1;
    a.n = static_cast<int>(plan->m);
    a.logn = ilog2(plan->m);
    a.ninsert = static_cast<int>(plan->ninsert);
    a.mode = plan->m < plan->nfft ? kPadProjCore : kPadProjFilter;
    a.tl = plan->tl_d;
    a.tr = plan->tr_d;
    a.scale = kFPi / (4.0f * static_cast<float>(plan->nfft / 2)); // the reference's N
    a.post1 = a.post2 = 1.0f;
    return launch_rowfilter(a, as_stream(stream));
}

mr_status mr_quantize(const float *in_d, size_t per, size_t nproj, int dtype, uint16_t *out_d, float *scale_d,
                      void *stream)
{
    MR_TRACE();
    if (!in_d || !out_d || !scale_d) return fail(MR_ERR_ARGUMENT, "mr_quantize: null pointer");
    if (dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_quantize: dtype must be bf16 or f16");
    if (nproj > 65535) return fail(MR_ERR_ARGUMENT, "mr_quantize: more than 65535 projections per call");
    if (per == 0 || nproj == 0) return MR_OK;
    return quantize_projections(in_d, per, nproj, dtype, out_d, scale_d, as_stream(stream));
}

mr_status mr_quantize_noalloc(const float *in_d, size_t per, size_t nproj, int dtype, uint16_t *out_d, float *scale_d,
                              void *stream)
{
    MR_TRACE();
    if (!in_d || !out_d || !scale_d) return fail(MR_ERR_ARGUMENT, "mr_quantize_noalloc: null pointer");
    if (dtype != MR_BF16 && dtype != MR_F16) return fail(MR_ERR_ARGUMENT, "mr_quantize_noalloc: dtype must be bf16 or f16");
    if (nproj > kQuantScratchMax)
        return fail(MR_ERR_ARGUMENT, "mr_quantize_noalloc: %zu projections exceed the built-in scratch of %zu projections",
                    nproj, kQuantScratchMax);
    if (per == 0 || nproj == 0) return MR_OK;
    int device = 0;
    MR_CUDA_TRY(cudaGetDevice(&device));
    mr_status st = MR_OK;
    float *amax = quant_scratch_ptr(device, &st);
    if (st != MR_OK) return st;
    float *inv = amax + kQuantScratchMax;
    cudaStream_t s = as_stream(stream);
    // the array keeps the previous call's values: the running maxima must start at zero
    MR_CUDA_TRY(cudaMemsetAsync(amax, 0, nproj * sizeof(float), s));
    // one grid row per projection; gridDim.y stops at 65535, so the array's full 65536
    // projections take two launches
    constexpr size_t kGridYMax = 65535;
    for (size_t p0 = 0; p0 < nproj; p0 += kGridYMax) {
        const size_t np = std::min(kGridYMax, nproj - p0);
        dim3 g(std::min<unsigned>(div_up(per, 256), 64u), static_cast<unsigned>(np));
        k_absmax<<<g, 256, 0, s>>>(in_d + p0 * per, per, amax + p0);
        if ((st = check_launch("k_absmax")) != MR_OK) return st;
    }
    k_pow2_scales<<<div_up(nproj, 128), 128, 0, s>>>(amax, nproj, dtype, scale_d, inv);
    if ((st = check_launch("k_pow2_scales")) != MR_OK) return st;
    const size_t total = per * nproj;
    const unsigned blocks = std::min<unsigned>(div_up(total, 256), 148u * 16u);
    if (dtype == MR_BF16)
        k_quantize<MR_BF16><<<blocks, 256, 0, s>>>(in_d, per, total, inv, out_d);
    else
        k_quantize<MR_F16><<<blocks, 256, 0, s>>>(in_d, per, total, inv, out_d);
    return check_launch("k_quantize");
}

mr_status mr_fdk_filter(const float *in_d, size_t nu, size_t nv, size_t nproj, const float *weight_d, float sad_sid_2,
                        float scale, int out_dtype, void *out_d, float *scale_out_d, void *stream)
{
    MR_TRACE();
    return mr_fdk_filter_rows(in_d, nu, nv, 0, nv, nproj, weight_d, sad_sid_2, scale, out_dtype, out_d, scale_out_d,
                              stream);
}

mr_status mr_fdk_filter_rows(const float *in_d, size_t nu, size_t nrows, size_t row0, size_t nv, size_t nproj,
                             const float *weight_d, float sad_sid_2, float scale, int out_dtype, void *out_d,
                             float *scale_out_d, void *stream)
{
    MR_TRACE();
    if (!in_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: null pointer");
    if (nv < 11) return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: the edge-row replication needs at least 11 rows");
    if (nrows == 0 || row0 + nrows > nv) return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: row window outside the detector");
    // rows 0..4 are copies of row 5 and rows nv-5.. of row nv-6: those rows must be held too
    if ((row0 < 5 && row0 + nrows <= 5) || (row0 + nrows > nv - 5 && row0 > nv - 6))
        return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: the row window [%zu, %zu) misses the edge rows it copies", row0,
                    row0 + nrows);
    const size_t nvfull = nv;
    nv = nrows; // rows held per projection from here on
    if (out_dtype != MR_F32 && out_dtype != MR_BF16 && out_dtype != MR_F16)
        return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: unknown output dtype");
    if (out_dtype != MR_F32 && !scale_out_d) return fail(MR_ERR_ARGUMENT, "mr_fdk_filter: 16-bit output needs scale_out_d");
    // prepareFFT (:960-964): padwidth = 2*2^ceil(log2(width)), double arithmetic
    const unsigned padwidth = static_cast<unsigned>(2 * std::pow(2, std::ceil(std::log(static_cast<double>(static_cast<unsigned>(nu))) / std::log(2))));
    if (padwidth > 16384) return fail(MR_ERR_UNSUPPORTED, "mr_fdk_filter: padded width %u above 16384", padwidth);
    // ramp (:890-910), same float/double expressions as the reference
    std::vector<float> ramp(padwidth);
    for (unsigned i = 0; i < padwidth / 2; ++i) ramp[i] = static_cast<float>(i);
    for (unsigned i = padwidth / 2; i < padwidth; ++i) ramp[i] = static_cast<float>(padwidth - i);
    const float degtorad = kFPi / 180.0f;
    for (unsigned i = 0; i < padwidth; ++i) {
        ramp[i] *= (0.54 + 0.46 * (std::cos(i * degtorad * 360 / padwidth) + 1));
        ramp[i] /= padwidth * 0.5;
    }
    ramp = fft_permute_response(ramp, ilog2(padwidth)); // in the order of the forward transform's output
    std::vector<float2> tw = fft_twiddles(static_cast<int>(padwidth));
    cudaStream_t s = as_stream(stream);
    float2 *tw_d = nullptr;
    float *resp_d = nullptr;
    float *tmp = nullptr;
    mr_status st = MR_OK;
    const size_t total = nu * nv * nproj;
    st = device_alloc(&tw_d, tw.size() * sizeof(float2), s, "mr_fdk_filter: twiddles");
    if (st == MR_OK) st = device_alloc(&resp_d, padwidth * sizeof(float), s, "mr_fdk_filter: response");
    if (st == MR_OK && out_dtype != MR_F32) st = device_alloc(&tmp, total * sizeof(float), s, "mr_fdk_filter: f32 staging buffer");
    if (st == MR_OK) {
        if (cudaMemcpyAsync(tw_d, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(resp_d, ramp.data(), padwidth * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess)
            st = fail(MR_ERR_CUDA, "mr_fdk_filter: table upload");
    }
    if (st == MR_OK) {
        RowFilterArgs a{};
        a.in = in_d;
        a.out = out_dtype == MR_F32 ? static_cast<float *>(out_d) : tmp;
        a.twiddle = tw_d;
        a.response = resp_d;
        a.row_weight = weight_d;
        a.rows_per_weight = nv;
        a.nrows = nv * nproj;
        a.nu = static_cast<int>(nu);
        a.nv = static_cast<int>(nv);
        a.row0 = static_cast<int>(row0);
        a.nvfull = static_cast<int>(nvfull);
        a.n = static_cast<int>(padwidth);
        a.logn = ilog2(padwidth);
        a.ninsert = static_cast<int>((padwidth - nu) / 2);
        a.mode = kPadFdk;
        a.scale = 1.0f / padwidth;
        a.post1 = sad_sid_2;
        a.post2 = scale;
        st = launch_rowfilter(a, s);
    }
    if (st == MR_OK && out_dtype != MR_F32)
        st = quantize_projections(tmp, nu * nv, nproj, out_dtype, static_cast<uint16_t *>(out_d), scale_out_d, s);
    // pageable-host uploads above are synchronous with respect to the host buffers, so the
    // vectors may go out of scope; device tables are released in stream order
    if (tw_d) cudaFreeAsync(tw_d, s);
    if (resp_d) cudaFreeAsync(resp_d, s);
    if (tmp) cudaFreeAsync(tmp, s);
    return st;
}

} // extern "C"
