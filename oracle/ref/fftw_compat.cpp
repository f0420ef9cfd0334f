// FFTW3 API subset for building the reference oracle (test infrastructure only).
//
// FFTW is not installed in this environment and its source is not vendored with the
// reference (only external/include/fftw3.h and Windows DLLs ship). The reference hot
// path calls FFTW through kipl (core/kipl/kipl/src/fft/fftbasef.cpp:86-246,
// fftbase.cpp:80-240) and directly in FDK (frameworks/tomography/Backprojectors/
// FDKBackProjectors/src/fdkbp_single.cpp:960-982). This file implements the FFTW3
// planner/execute calls those sites use, from the DFT definition:
//     X[k] = sum_n x[n] exp(sign * 2 pi i k n / N),  unnormalised (FFTW convention),
// with an iterative radix-2 Cooley-Tukey transform for powers of two and a direct
// O(N^2) sum otherwise. Arithmetic is FP64 for both the float and double APIs, so
// float results differ from FFTW's own float rounding by a few ulp.
// Multi-dimensional plans are row-major (last dimension fastest), computed as
// successive 1-D transforms; r2c/c2r keep n_last/2+1 complex values on the last axis.
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include <fftw3.h>

namespace {

using cd = std::complex<double>;

enum Kind { kC2C, kR2C, kC2R };

struct PlanCommon {
    Kind kind;
    int rank;
    int n[3];
    int sign;
    void *in;
    void *out;
    bool single;
};

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// exp(sign * 2 pi i m / n) for m < n/2, each evaluated directly (no recurrence), cached per
// thread and size: the butterflies read the same values they would compute
const std::vector<cd> &twiddles(int n, int sign)
{
    thread_local std::map<std::pair<int, int>, std::vector<cd>> cache;
    std::vector<cd> &t = cache[{n, sign}];
    if (t.empty()) {
        t.resize(static_cast<size_t>(n / 2));
        for (int m = 0; m < n / 2; ++m) {
            const double ang = sign * 2.0 * M_PI * static_cast<double>(m) / n;
            t[static_cast<size_t>(m)] = cd(std::cos(ang), std::sin(ang));
        }
    }
    return t;
}

void fft1d(cd *a, int n, int sign)
{
    if (n <= 1) return;
    if (!is_pow2(n)) {
        std::vector<cd> r(n);
        for (int k = 0; k < n; ++k) {
            cd s = 0.0;
            for (int j = 0; j < n; ++j) {
                long long kj = (static_cast<long long>(k) * j) % n;
                double ang = sign * 2.0 * M_PI * static_cast<double>(kj) / n;
                s += a[j] * cd(std::cos(ang), std::sin(ang));
            }
            r[k] = s;
        }
        std::copy(r.begin(), r.end(), a);
        return;
    }
    // split real and imaginary parts (plain double loops; the butterflies are the same
    // operations as with std::complex's finite-value product), bit-reversed order
    thread_local std::vector<double> re, im;
    re.resize(static_cast<size_t>(n));
    im.resize(static_cast<size_t>(n));
    for (int i = 0, j = 0; i < n; ++i) {
        re[static_cast<size_t>(j)] = a[i].real();
        im[static_cast<size_t>(j)] = a[i].imag();
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
    }
    const std::vector<cd> &tw = twiddles(n, sign);
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        const int stride = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < half; ++k) {
                const cd w = tw[static_cast<size_t>(k) * stride];
                const size_t p = static_cast<size_t>(i + k), q = p + static_cast<size_t>(half);
                const double vr = re[q] * w.real() - im[q] * w.imag();
                const double vi = re[q] * w.imag() + im[q] * w.real();
                const double ur = re[p], ui = im[p];
                re[p] = ur + vr;
                im[p] = ui + vi;
                re[q] = ur - vr;
                im[q] = ui - vi;
            }
        }
    }
    for (int i = 0; i < n; ++i) a[i] = cd(re[static_cast<size_t>(i)], im[static_cast<size_t>(i)]);
}

// In-place multi-dimensional c2c over a row-major array of dims n[0..rank-1].
void fftnd(cd *a, const int *n, int rank, int sign)
{
    size_t total = 1;
    for (int d = 0; d < rank; ++d) total *= static_cast<size_t>(n[d]);
    for (int d = 0; d < rank; ++d) {
        size_t inner = 1;
        for (int e = d + 1; e < rank; ++e) inner *= static_cast<size_t>(n[e]);
        const size_t len = static_cast<size_t>(n[d]);
        const size_t outer = total / (inner * len);
        std::vector<cd> line(len);
        for (size_t o = 0; o < outer; ++o)
            for (size_t in = 0; in < inner; ++in) {
                cd *base = a + o * len * inner + in;
                for (size_t k = 0; k < len; ++k) line[k] = base[k * inner];
                fft1d(line.data(), static_cast<int>(len), sign);
                for (size_t k = 0; k < len; ++k) base[k * inner] = line[k];
            }
    }
}

template <typename R>
void execute_plan(const PlanCommon *p)
{
    size_t total = 1;
    for (int d = 0; d < p->rank; ++d) total *= static_cast<size_t>(p->n[d]);
    const int nl = p->n[p->rank - 1];
    const size_t nh = static_cast<size_t>(nl / 2 + 1);
    const size_t outer = total / static_cast<size_t>(nl);
    std::vector<cd> buf(total);
    if (p->kind == kC2C) {
        const R *src = static_cast<const R *>(p->in);
        for (size_t i = 0; i < total; ++i) buf[i] = cd(src[2 * i], src[2 * i + 1]);
        fftnd(buf.data(), p->n, p->rank, p->sign);
        R *dst = static_cast<R *>(p->out);
        for (size_t i = 0; i < total; ++i) {
            dst[2 * i] = static_cast<R>(buf[i].real());
            dst[2 * i + 1] = static_cast<R>(buf[i].imag());
        }
    } else if (p->kind == kR2C) {
        const R *src = static_cast<const R *>(p->in);
        for (size_t i = 0; i < total; ++i) buf[i] = cd(src[i], 0.0);
        fftnd(buf.data(), p->n, p->rank, -1);
        R *dst = static_cast<R *>(p->out);
        for (size_t o = 0; o < outer; ++o)
            for (size_t k = 0; k < nh; ++k) {
                const cd v = buf[o * nl + k];
                dst[2 * (o * nh + k)] = static_cast<R>(v.real());
                dst[2 * (o * nh + k) + 1] = static_cast<R>(v.imag());
            }
    } else {
        // c2r: rebuild the Hermitian-symmetric full spectrum, inverse transform, real part.
        // Like FFTW, the imaginary parts of self-conjugate bins are ignored.
        const R *src = static_cast<const R *>(p->in);
        std::vector<cd> half(outer * nh);
        for (size_t i = 0; i < outer * nh; ++i) half[i] = cd(src[2 * i], src[2 * i + 1]);
        // index helpers over the leading dims (row-major)
        std::vector<int> lead(p->n, p->n + p->rank - 1);
        for (size_t o = 0; o < outer; ++o) {
            // conjugate partner of the leading multi-index o
            size_t rem = o, partner = 0, mul = 1;
            std::vector<size_t> idx(lead.size());
            for (int d = static_cast<int>(lead.size()) - 1; d >= 0; --d) {
                idx[d] = rem % lead[d];
                rem /= lead[d];
            }
            for (int d = static_cast<int>(lead.size()) - 1; d >= 0; --d) {
                size_t pd = (lead[d] - idx[d]) % lead[d];
                partner += pd * mul;
                mul *= lead[d];
            }
            for (int k = 0; k < nl; ++k) {
                if (static_cast<size_t>(k) < nh)
                    buf[o * nl + k] = half[o * nh + k];
                else
                    buf[o * nl + k] = std::conj(half[partner * nh + (nl - k)]);
            }
            if (lead.empty()) {
                buf[o * nl + 0] = cd(buf[o * nl + 0].real(), 0.0);
                if ((nl & 1) == 0) buf[o * nl + nl / 2] = cd(buf[o * nl + nl / 2].real(), 0.0);
            }
        }
        fftnd(buf.data(), p->n, p->rank, +1);
        R *dst = static_cast<R *>(p->out);
        for (size_t i = 0; i < total; ++i) dst[i] = static_cast<R>(buf[i].real());
    }
}

PlanCommon *make_plan(Kind kind, int rank, const int *n, int sign, void *in, void *out, bool single)
{
    PlanCommon *p = new PlanCommon;
    p->kind = kind;
    p->rank = rank;
    for (int d = 0; d < 3; ++d) p->n[d] = d < rank ? n[d] : 1;
    p->sign = sign;
    p->in = in;
    p->out = out;
    p->single = single;
    return p;
}

} // namespace

struct fftw_plan_s : PlanCommon {};
struct fftwf_plan_s : PlanCommon {};

extern "C" {

// ---- double API
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned)
{ int d[1] = {n}; return static_cast<fftw_plan>(make_plan(kC2C, 1, d, sign, in, out, false)); }
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftw_plan>(make_plan(kC2C, 2, d, sign, in, out, false)); }
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftw_plan>(make_plan(kC2C, 3, d, sign, in, out, false)); }
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned)
{ int d[1] = {n}; return static_cast<fftw_plan>(make_plan(kR2C, 1, d, -1, in, out, false)); }
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftw_plan>(make_plan(kR2C, 2, d, -1, in, out, false)); }
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftw_plan>(make_plan(kR2C, 3, d, -1, in, out, false)); }
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned)
{ int d[1] = {n}; return static_cast<fftw_plan>(make_plan(kC2R, 1, d, +1, in, out, false)); }
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftw_plan>(make_plan(kC2R, 2, d, +1, in, out, false)); }
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftw_plan>(make_plan(kC2R, 3, d, +1, in, out, false)); }
void fftw_execute(const fftw_plan p) { execute_plan<double>(p); }
void fftw_destroy_plan(fftw_plan p) { delete static_cast<PlanCommon *>(p); }
void *fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void *p) { std::free(p); }

// ---- float API
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned)
{ int d[1] = {n}; return static_cast<fftwf_plan>(make_plan(kC2C, 1, d, sign, in, out, true)); }
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftwf_plan>(make_plan(kC2C, 2, d, sign, in, out, true)); }
fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out, int sign, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftwf_plan>(make_plan(kC2C, 3, d, sign, in, out, true)); }
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned)
{ int d[1] = {n}; return static_cast<fftwf_plan>(make_plan(kR2C, 1, d, -1, in, out, true)); }
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftwf_plan>(make_plan(kR2C, 2, d, -1, in, out, true)); }
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in, fftwf_complex *out, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftwf_plan>(make_plan(kR2C, 3, d, -1, in, out, true)); }
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned)
{ int d[1] = {n}; return static_cast<fftwf_plan>(make_plan(kC2R, 1, d, +1, in, out, true)); }
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned)
{ int d[2] = {n0, n1}; return static_cast<fftwf_plan>(make_plan(kC2R, 2, d, +1, in, out, true)); }
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in, float *out, unsigned)
{ int d[3] = {n0, n1, n2}; return static_cast<fftwf_plan>(make_plan(kC2R, 3, d, +1, in, out, true)); }
void fftwf_execute(const fftwf_plan p) { execute_plan<float>(p); }
void fftwf_destroy_plan(fftwf_plan p) { delete static_cast<PlanCommon *>(p); }
void *fftwf_malloc(size_t n) { return std::malloc(n); }
void fftwf_free(void *p) { std::free(p); }

} // extern "C"
