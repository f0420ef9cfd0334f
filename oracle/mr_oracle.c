/* CPU restatement of the MuhRec reconstruction hot path (test infrastructure only).
 * See mr_oracle.h for the contract. Reference citations are relative to the reference
 * project root. Built with -ffp-contract=off: every float operation rounds separately,
 * in the order the reference writes it.
 */
#include "mr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* kipl math constants (core/kipl/kipl/include/math/mathconstants.h:7-8) */
static const double kDPi = 3.1415926535897932384626433832795028841971693993751;
static const float kFPi = 3.1415926535897932384626f;

/* ------------------------------------------------------------------ helpers */

static int cmp_float(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

/* kipl::math::median (core/kipl/kipl/include/math/core/median.hpp:10-22): sorted copy,
 * middle element, or 0.5*(a+b) in double for even counts. */
static float median_f(const float *v, size_t n)
{
    float *tmp = (float *)malloc(n * sizeof(float));
    memcpy(tmp, v, n * sizeof(float));
    qsort(tmp, n, sizeof(float), cmp_float);
    float med;
    if (n & 1)
        med = tmp[n / 2];
    else
        med = (float)(0.5 * ((double)tmp[n / 2 - 1] + (double)tmp[n / 2]));
    free(tmp);
    return med;
}

/* iterative radix-2 complex FFT in FP64, sign -1 forward, +1 backward, unnormalised */
static void fft_c2c(double *re, double *im, size_t n, int sign)
{
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len >> 1;
        for (size_t k = 0; k < half; ++k) {
            double ang = sign * 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (size_t i = 0; i < n; i += len) {
                double ur = re[i + k], ui = im[i + k];
                double xr = re[i + k + half], xi = im[i + k + half];
                double vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
                re[i + k] = ur + vr; im[i + k] = ui + vi;
                re[i + k + half] = ur - vr; im[i + k + half] = ui - vi;
            }
        }
    }
}

/* ------------------------------------------------------- reference averaging */

static void stddev_filter(const float *img, int w, int h, int dim, float *out);
static float lut_apply(const float *lut, size_t len, const float *param, float v);

/* AverageImage::operator() (core/algorithms/ImagingAlgorithms/src/averageimage.cpp:35-219). */
int orc_average(const float *stack, size_t nu, size_t nv, size_t n, int method, float *out)
{
    const size_t npix = nu * nv;
    if (n == 0) return -1;
    switch (method) {
    case ORC_AVG_WEIGHTED: {
        /* ComputeWeightedAverage (:123-172): per frame a 5x5 StdDevFilter (EdgeMirror); per
         * pixel weight 1/sigma, or 1/(number of pixels) where sigma is 0; the weighted sum and
         * the weight sum in frame order, then their quotient. */
        if (nu < 5 || nv < 5) return -1;
        float *sig = (float *)malloc(n * npix * sizeof(float));
        for (size_t i = 0; i < n; ++i) stddev_filter(stack + i * npix, (int)nu, (int)nv, 5, sig + i * npix);
        const float zw = 1.0f / (float)npix;
        for (size_t j = 0; j < npix; ++j) {
            float ws = 0.0f, acc = 0.0f;
            for (size_t i = 0; i < n; ++i) {
                const float sg = sig[i * npix + j];
                const float wt = sg != 0.0f ? 1.0f / sg : zw;
                ws += wt;
                acc += wt * stack[i * npix + j];
            }
            out[j] = acc / ws;
        }
        free(sig);
        return 0;
    }
    case ORC_AVG_SUM:
    case ORC_AVG_AVERAGE: {
        for (size_t j = 0; j < npix; ++j) out[j] = 0.0f;
        for (size_t i = 0; i < n; ++i)
            for (size_t j = 0; j < npix; ++j) out[j] += stack[i * npix + j];
        if (method == ORC_AVG_AVERAGE) {
            float q = 1.0f / (float)n;
            for (size_t j = 0; j < npix; ++j) out[j] *= q;
        }
        return 0;
    }
    case ORC_AVG_MEDIAN: {
        /* median_STL: partial sort, middle element; even counts average the two middle
         * values in float (median.hpp:24-41) */
        float *col = (float *)malloc(n * sizeof(float));
        for (size_t j = 0; j < npix; ++j) {
            for (size_t i = 0; i < n; ++i) col[i] = stack[i * npix + j];
            qsort(col, n, sizeof(float), cmp_float);
            out[j] = (n & 1) ? col[n / 2] : (col[n / 2 - 1] + col[n / 2]) / 2.0f;
        }
        free(col);
        return 0;
    }
    case ORC_AVG_MIN:
    case ORC_AVG_MAX: {
        for (size_t j = 0; j < npix; ++j) {
            float v = stack[j];
            for (size_t i = 1; i < n; ++i) {
                float s = stack[i * npix + j];
                v = method == ORC_AVG_MIN ? (s < v ? s : v) : (s > v ? s : v);
            }
            out[j] = v;
        }
        return 0;
    }
    default:
        return -1;
    }
}

/* ProjectionReader::GetProjectionDose (ReconFramework/src/ProjectionReader.cpp:752-783) */
float orc_frame_dose(const float *frame, size_t nu, const size_t *roi)
{
    if ((roi[0] * roi[1] * roi[2] * roi[3]) == 0) return 1.0f;
    size_t w = roi[2] - roi[0], h = roi[3] - roi[1];
    float *means = (float *)calloc(h, sizeof(float));
    for (size_t y = 0; y < h; ++y) {
        const float *p = frame + (roi[1] + y) * nu + roi[0];
        for (size_t x = 0; x < w; ++x) means[y] += p[x];
        means[y] = means[y] / (float)w;
    }
    float d = median_f(means, h);
    free(means);
    return d;
}

/* ------------------------------------------------------------ FullLogNorm */

/* FullLogNorm::SetReferenceImages (NormPlugins.cpp:300-341) */
void orc_lognorm_logflat(const float *dark, const float *flat, size_t npix, int ndc, float flatdose, float *logflat)
{
    float dose = 1.0f / flatdose;
    for (size_t i = 0; i < npix; ++i) {
        float p = ndc ? flat[i] - dark[i] : flat[i];
        logflat[i] = p <= 0 ? 0.0f : logf(p * dose);
    }
}

/* FullLogNorm::ProcessCore 3D dose list (NormPlugins.cpp:416-425) */
void orc_lognorm_doselog(const float *doses, size_t nproj, float darkdose, float *doselog)
{
    for (size_t i = 0; i < nproj; ++i) {
        float d = doses[i] - darkdose;
        doselog[i] = logf(d < 1 ? 1.0f : d);
    }
}

/* FullLogNorm::ProcessCore 3D, non-LUT branches (NormPlugins.cpp:481-549) */
void orc_lognorm_apply(float *proj, size_t npix, size_t nproj, const float *dark, const float *logflat,
                       const float *doselog, size_t ndose, int ndc, int nob)
{
    for (size_t j = 0; j < nproj; ++j) {
        float *p = proj + j * npix;
        float dose = ndose != 1 ? doselog[j] : doselog[0];
        for (size_t i = 0; i < npix; ++i) {
            float v = ndc ? p[i] - dark[i] : p[i];
            if (v <= 0.0f)
                p[i] = 0.0f;
            else
                p[i] = nob ? (logflat[i] - logf(v)) + dose : -logf(v) + dose;
        }
    }
}

/* kipl::math::LogLUT(1 << 16, 0, 65535) as FullLogNorm builds it (NormPlugins.cpp:245;
 * core/kipl/kipl/src/math/LUTCollection.cpp:11-36 over LUTbase.cpp:12-20): slope
 * (len - 1) / (hi - lo) and intercept -slope * lo + 0.5 in float; with lo = 0 the first entry
 * is log(1 / slope) and entry i >= 1 log(x), x stepping from 1 / slope by 1 / slope in float;
 * the double log the reference calls, stored as float. param: lo, hi, slope, intercept. */
void orc_log_lut(float *lut, float *param)
{
    const size_t len = (size_t)1 << 16;
    const float lo = 0.0f, hi = (float)((1 << 16) - 1);
    const float slope = (float)(len - 1) / (hi - lo), intercept = -slope * lo + 0.5f;
    const float delta = 1.0f / slope;
    float x = delta;
    lut[0] = (float)log((double)delta);
    for (size_t i = 1; i < len; ++i, x += delta) lut[i] = (float)log((double)x);
    param[0] = lo;
    param[1] = hi;
    param[2] = slope;
    param[3] = intercept;
}

/* FullLogNorm::ProcessCore 3D with uselut (NormPlugins.cpp:455-480): I - D (when there are
 * darks), the LogLUT of that (BasicLUT: below lo the first entry, above hi the last, else entry
 * (size_t)(v * slope + intercept), clamped to the table where the reference reads past it),
 * then logflat - l + dose, or -l + (dose - doselog[0]) without flats. */
void orc_lognorm_apply_lut(float *proj, size_t npix, size_t nproj, const float *dark, const float *logflat,
                           const float *doselog, size_t ndose, int ndc, int nob)
{
    const size_t len = (size_t)1 << 16;
    float *lut = (float *)malloc(len * sizeof(float)), param[4];
    orc_log_lut(lut, param);
    for (size_t j = 0; j < nproj; ++j) {
        float *p = proj + j * npix;
        float dose = ndose != 1 ? doselog[j] : doselog[0];
        if (!nob) dose -= doselog[0];
        for (size_t i = 0; i < npix; ++i) {
            const float v = ndc ? p[i] - dark[i] : p[i];
            const float l = lut_apply(lut, len, param, v);
            p[i] = nob ? (logflat[i] - l) + dose : -l + dose;
        }
    }
    free(lut);
}

/* -------------------------------------------------- ProjectionFilterSingle */

/* ProjectionFilterBase::ComputeFilterSize (ProjectionFilter.cpp:120-125) */
size_t orc_projfilter_size(size_t nu, int paddingdoubler)
{
    double e = log((double)nu) / log(2.0);
    return (size_t)1 << ((size_t)ceil(e) + (size_t)paddingdoubler);
}

/* ProjectionFilterSingle::BuildFilter + PreparePadding (ProjectionFilter.cpp:254-299,364-376),
 * with kipl::math::Sigmoid (core/kipl/kipl/include/math/core/mathfunctions.hpp:60-63). */
int orc_projfilter_build(size_t nu, int filtertype, float cutoff, float order, int usebias, float biasweight,
                         int paddingdoubler, float *filter, float *pad, size_t *ninsert)
{
    size_t nfft = orc_projfilter_size(nu, paddingdoubler);
    size_t n2 = nfft / 2;
    if (!((0 < cutoff) && (cutoff <= 0.5f))) return -1;
    float forder = filtertype == ORC_FILTER_BUTTERWORTH ? order : 0.0f;
    size_t cut = (size_t)(2 * cutoff * n2);
    float rampstep = 1.0f / ((n2 - 1.0f));
    for (size_t i = 0; i < n2; ++i) filter[i] = i * rampstep;
    float fstep = 1.0f / ((cut - 1.0f));
    for (size_t i = 0; i < cut; ++i) {
        switch (filtertype) {
        case ORC_FILTER_RAMLAK: break;
        case ORC_FILTER_SHEPPLOGAN: filter[i] = (float)sin(kDPi * i * fstep * cutoff) / n2; break;
        case ORC_FILTER_HANNING: filter[i] *= (float)(0.5f + 0.5f * cosf(i * fstep * kFPi * cutoff)); break;
        case ORC_FILTER_HAMMING: filter[i] *= (float)(0.54 + 0.46 * cos(i * fstep * kDPi * cutoff)); break;
        case ORC_FILTER_BUTTERWORTH: filter[i] /= (float)(1 + powf(i * fstep * cutoff, forder)); break;
        default: return -1;
        }
    }
    for (size_t i = cut; i < n2; ++i) filter[i] = 0.0f;
    if (usebias) filter[0] = biasweight * filter[1];

    size_t ins = n2 - nu / 2;
    for (size_t i = 0; i < ins; ++i) {
        float x = (float)i / (float)ins - 0.5f;
        pad[i] = (float)(1.0 / (1.0 + expf(-(x - 0.0f) / 0.07f)));
    }
    *ninsert = ins;
    return 0;
}

/* ProjectionFilterSingle::FilterProjection + Pad (ProjectionFilter.cpp:301-362) */
void orc_projfilter_apply(float *proj, size_t nu, size_t nrows, const float *filter, const float *pad,
                          size_t nfft, size_t ninsert)
{
    const size_t n2 = nfft / 2;
    const size_t nlen = nfft + 16;
    const float scale = kFPi / (4.0f * n2);
#pragma omp parallel
    {
        float *line = (float *)malloc(nlen * sizeof(float));
        double *re = (double *)malloc(nfft * sizeof(double));
        double *im = (double *)malloc(nfft * sizeof(double));
#pragma omp for schedule(static)
        for (long r = 0; r < (long)nrows; ++r) {
            float *src = proj + (size_t)r * nu;
            memset(line, 0, nlen * sizeof(float));
            memcpy(line + ninsert, src, nu * sizeof(float));
            for (size_t i = 0; i < ninsert; ++i) {
                line[i] = src[0] * pad[i];
                line[nlen - 1 - i] = src[nu - 1] * pad[i];
            }
            for (size_t i = 0; i < nfft; ++i) { re[i] = line[i]; im[i] = 0.0; }
            fft_c2c(re, im, nfft, -1);
            /* bins 0..n2-1 are filtered; bin n2 (Nyquist) keeps its value */
            for (size_t i = 0; i < n2; ++i) {
                double f = (double)(float)((float)re[i] * filter[i]);
                double g = (double)(float)((float)im[i] * filter[i]);
                re[i] = f; im[i] = g;
            }
            /* c2r: Hermitian extension of bins 0..n2, imaginary parts of 0 and n2 ignored */
            im[0] = 0.0;
            im[n2] = 0.0;
            for (size_t k = 1; k < n2; ++k) { re[nfft - k] = re[k]; im[nfft - k] = -im[k]; }
            fft_c2c(re, im, nfft, +1);
            for (size_t i = 0; i < nu; ++i) src[i] = (float)re[i + ninsert] * scale;
        }
        free(line); free(re); free(im);
    }
}

/* ------------------------------------------------------ parallel-beam BP */

/* BackProjectorModuleBase::BuildCircleMask (ReconFramework/src/BackProjectorModuleBase.cpp:153-218),
 * no matrix ROI. mask[2*i] = first, mask[2*i+1] = second. */
static void circle_mask(size_t nx, size_t ny, int correcttilt, float tiltangle, size_t nslices, size_t *mask)
{
    const float cx = (float)(nx >> 1);
    const float cy = (float)(ny >> 1);
    float R = cx - 1;
    if (correcttilt) {
        float slices = (float)nslices;
        R -= floorf(tanf(fabsf(tiltangle) * kFPi / 180.0f) * slices);
    }
    const float R2 = R * R;
    for (size_t i = 0; i < ny; ++i) {
        float y = (float)i - cy;
        float y2 = y * y;
        if (y2 <= R2) {
            float x = sqrtf(R2 - y2);
            mask[2 * i] = (size_t)ceilf(cx - x);
            size_t s = (size_t)floorf(cx + x);
            mask[2 * i + 1] = (nx - 1u) < s ? (nx - 1u) : s;
        } else {
            mask[2 * i] = 0;
            mask[2 * i + 1] = 0;
        }
    }
}

/* One buffer flush of MultiProjectionBPparallel::BackProject (MultiProjBPparallel.cpp:39-170).
 * buf: [count][nu][nvpad] weighted, transposed projections. */
/* variant 0: MultiProjectionBPparallel::BackProject (MultiProjBPparallel.cpp:39-170);
 * 1: the serial MultiProjectionBP (MultiProjBP.cpp:36-146), which differs only under tilt
 * correction (centre offset subtracted after the x term, one weight shift per 4-slice group);
 * 2: NearestNeighborBP (NNMultiProjBP.cpp:36-121): the sample at the truncated position, no
 * weights, under tilt a constant centre offset only. */
static void bp_flush(const float *buf, size_t count, size_t nu, size_t nv, size_t nvpad, const float *fsin,
                     const float *fcos, const float *fstartu, const size_t *mask, int correcttilt,
                     float tiltangle, float tiltpivot, size_t roi_y0, int variant, float *vol)
{
    const size_t sizez = nv / 4;
    const int sizeum2 = (int)(nu - 2);
    const float centeroffset = ((float)roi_y0 - tiltpivot) * tanf(tiltangle * kFPi / 180);
    const float centerinc = 4 * tanf(tiltangle * kFPi / 180);
#pragma omp parallel for schedule(static)
    for (long y = 1; y <= (long)nu; ++y) {
        float local[1024 * 4];
        for (size_t i = 0; i < count; ++i)
            local[i] = correcttilt && variant == 0 ? (fstartu[i] + fcos[i] * (float)y) - centeroffset
                                                   : fstartu[i] + fcos[i] * (float)y;
        const size_t x0 = mask[2 * (y - 1)], x1 = mask[2 * (y - 1) + 1];
        for (size_t x = x0 + 1; x <= x1; ++x) {
            float *col = vol + ((size_t)(y - 1) * nu + (x - 1)) * nv;
            for (size_t i = 0; i < count; ++i) {
                float posu = local[i] - fsin[i] * (float)x;
                if (correcttilt && variant != 0) posu = posu - centeroffset;
                int n = (int)posu;
                if (n < 0 || sizeum2 < n) continue;
                const float *a = buf + (i * nu + (size_t)n) * nvpad;
                /* MultiProjBP.cpp:92,147 steps to column B by SizeV/4 vectors, not the padded
                 * column length: with nv not a multiple of 4 it reads inside the padded buffer */
                const float *b = a + (variant == 1 ? 4 * (nv / 4) : nvpad);
                if (variant == 2) {
                    for (size_t z = 0; z < 4 * sizez; ++z) col[z] = col[z] + a[z];
                } else if (correcttilt && variant == 1) {
                    for (size_t zg = 0; zg < sizez; ++zg) {
                        const float wb = fabsf((posu - (float)n) - (float)zg * centerinc);
                        const float wa = 1.0f - wb;
                        for (size_t q = 0; q < 4; ++q) {
                            size_t z = 4 * zg + q;
                            col[z] = col[z] + (a[z] * wa + b[z] * wb);
                        }
                    }
                } else if (!correcttilt) {
                    const float wb = fabsf(posu - (float)n);
                    const float wa = 1.0f - wb;
                    for (size_t z = 0; z < 4 * sizez; ++z) col[z] = col[z] + (a[z] * wa + b[z] * wb);
                } else {
                    posu -= (float)n;
                    for (size_t zg = 0; zg < sizez; ++zg) {
                        const float wb = fabsf(posu - (float)zg * centerinc);
                        const float wa = 1.0f - wb;
                        for (size_t q = 0; q < 4; ++q) {
                            size_t z = 4 * zg + q;
                            col[z] = col[z] + (a[z] * wa + b[z] * wb);
                        }
                        posu -= centerinc;
                    }
                }
            }
        }
    }
}

int orc_bp_parallel(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
                    const float *weights, float center, int direction, size_t buffersize, int correcttilt,
                    float tiltangle, float tiltpivot, size_t roi_y0, size_t nslices, float *vol)
{
    return orc_bp_parallel_variant(proj, nu, nv, nproj, angles, weights, center, direction, buffersize, correcttilt,
                                   tiltangle, tiltpivot, roi_y0, nslices, 0, vol);
}

int orc_bp_parallel_variant(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
                            const float *weights, float center, int direction, size_t buffersize, int correcttilt,
                            float tiltangle, float tiltpivot, size_t roi_y0, size_t nslices, int variant, float *vol)
{
    if (variant < 0 || variant > 2) return -1;
    if (buffersize == 0 || buffersize > 1024 || nu < 2) return -1;
    const size_t rest = (nv & 3) ? 4 - (nv & 3) : 0;
    const size_t nvpad = nv + rest;
    size_t *mask = (size_t *)malloc(2 * nu * sizeof(size_t));
    circle_mask(nu, nu, correcttilt, tiltangle, nslices, mask);
    float *buf = (float *)calloc(buffersize * nu * nvpad, sizeof(float));
    float fsin[1024], fcos[1024], fstartu[1024];
    memset(vol, 0, nu * nu * nv * sizeof(float));
    const size_t mcx = nu / 2;
    /* StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:64-118) */
    const float dirweight = 2.0f * ((float)direction - 0.5f);
    size_t counter = 0;
    for (size_t k = 0; k < nproj; ++k) {
        fsin[counter] = sinf(dirweight * angles[k] * kFPi / 180.0f);
        fcos[counter] = cosf(dirweight * angles[k] * kFPi / 180.0f);
        fstartu[counter] = mcx * (fsin[counter] - fcos[counter]) + center;
        const float *p = proj + k * nu * nv;
        float *dst = buf + counter * nu * nvpad;
        for (size_t u = 0; u < nu; ++u)
            for (size_t v = 0; v < nv; ++v) dst[u * nvpad + v] = p[v * nu + u] * weights[k];
        counter++;
        const int last = k == nproj - 1;
        if (last || buffersize <= counter) {
            if (buffersize <= counter) counter--; /* the buffer-full flush drops its last entry */
            bp_flush(buf, counter, nu, nv, nvpad, fsin, fcos, fstartu, mask, correcttilt, tiltangle, tiltpivot,
                     roi_y0, variant, vol);
            counter = 0;
        }
    }
    free(buf);
    free(mask);
    return 0;
}

/* ----------------------------------------------------------------- FDK */

/* FDKbp_single::getProjMatrix (fdkbp_single.cpp:83-255) */
void orc_fdk_projmatrix(const orc_fdk_geom *g, size_t nu, float angle, float *pm)
{
    (void)nu;
    float extrinsic[16] = {0};
    float intrinsic[12] = {0};
    const float sad = g->sod, sid = g->sdd;
    const float offcenter = (g->ppoint[0] - (float)0 - g->center) * g->voxelsize[0];
    float cam[3] = {0.0f, 0.0f, 0.0f};
    if (g->direction == 0) {
        cam[0] = sad * cosf(-angle * kFPi / 180.0f);
        cam[1] = sad * sinf(-angle * kFPi / 180.0f);
    } else {
        cam[0] = sad * cosf(angle * kFPi / 180.0f);
        cam[1] = sad * sinf(angle * kFPi / 180.0f);
    }
    float plt[3], pup[3], nrm[3];
    const float vup[3] = {0.0f, 0.0f, 1.0f};
    const float tgt[3] = {0.0f, 0.0f, 0.0f};
    nrm[0] = cam[0] - tgt[0];
    nrm[1] = cam[1] - tgt[1];
    nrm[2] = cam[2] - tgt[2];
    float nn = sqrtf(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    nrm[0] /= nn; nrm[1] /= nn; nrm[2] /= nn;
    plt[0] = nrm[1] * vup[2] - nrm[2] * vup[1];
    plt[1] = nrm[2] * vup[0] - nrm[0] * vup[2];
    plt[2] = nrm[0] * vup[1] - nrm[1] * vup[0];
    float np = sqrtf(plt[0] * plt[0] + plt[1] * plt[1] + plt[2] * plt[2]);
    plt[0] /= np; plt[1] /= np; plt[2] /= np;
    pup[0] = plt[1] * nrm[2] - plt[2] * nrm[1];
    pup[1] = plt[2] * nrm[0] - plt[0] * nrm[2];
    pup[2] = plt[0] * nrm[1] - plt[1] * nrm[0];
    float nq = sqrtf(pup[0] * pup[0] + pup[1] * pup[1] + pup[2] * pup[2]);
    pup[0] /= nq; pup[1] /= nq; pup[2] /= nq;
    extrinsic[0] = -1.0f * plt[0]; extrinsic[1] = -1.0f * plt[1]; extrinsic[2] = -1.0f * plt[2];
    extrinsic[4] = -1.0f * pup[0]; extrinsic[5] = -1.0f * pup[1]; extrinsic[6] = -1.0f * pup[2];
    extrinsic[8] = -1.0f * nrm[0]; extrinsic[9] = -1.0f * nrm[1]; extrinsic[10] = -1.0f * nrm[2];
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

/* FDKbp_single::ramp_filter_tuned + prepareFFT (fdkbp_single.cpp:832-982) on one
 * projection [height][width]; FFTs in FP64. */
void orc_fdk_ramp(float *img, size_t width, size_t height)
{
    const unsigned margin = 5;
    const unsigned padwidth = (unsigned)(2 * pow(2, ceil(log((double)(unsigned)width) / log(2))));
    const unsigned padfactor = padwidth - (unsigned)width;
    float *pad = (float *)calloc((size_t)padwidth * height, sizeof(float));
    for (size_t r = 0; r < height; ++r) memcpy(pad + r * padwidth + padfactor / 2, img + r * width, width * sizeof(float));
    for (unsigned r = 0; r < margin; ++r) memcpy(pad + r * padwidth, pad + margin * padwidth, padwidth * sizeof(float));
    for (unsigned r = (unsigned)height - margin; r < height; ++r)
        memcpy(pad + (size_t)r * padwidth, pad + (height - margin - 1) * padwidth, padwidth * sizeof(float));
    for (size_t r = 0; r < height; ++r) {
        for (unsigned c = 0; c < margin; ++c) pad[r * padwidth + c] = pad[r * padwidth + margin];
        for (unsigned c = padwidth - margin; c < padwidth; ++c) pad[r * padwidth + c] = pad[r * padwidth + padwidth - margin - 1];
    }
    float *ramp = (float *)malloc(padwidth * sizeof(float));
    for (unsigned i = 0; i < padwidth / 2; ++i) ramp[i] = (float)i;
    for (unsigned i = padwidth / 2; i < padwidth; ++i) ramp[i] = (float)(padwidth - i);
    const float degtorad = kFPi / 180.0f;
    for (unsigned i = 0; i < padwidth; ++i) {
        ramp[i] = (float)(ramp[i] * (0.54 + 0.46 * (cosf(i * degtorad * 360 / padwidth) + 1)));
        ramp[i] = (float)(ramp[i] / (padwidth * 0.5));
    }
    const float rpad = 1.0f / padwidth;
#pragma omp parallel
    {
        double *re = (double *)malloc(padwidth * sizeof(double));
        double *im = (double *)malloc(padwidth * sizeof(double));
#pragma omp for schedule(static)
        for (long r = 0; r < (long)height; ++r) {
            float *row = pad + (size_t)r * padwidth;
            for (unsigned c = 0; c < padwidth; ++c) { re[c] = row[c]; im[c] = 0.0; }
            fft_c2c(re, im, padwidth, -1);
            for (unsigned c = 0; c < padwidth; ++c) {
                re[c] = (double)(float)((float)re[c] * ramp[c]);
                im[c] = (double)(float)((float)im[c] * ramp[c]);
            }
            fft_c2c(re, im, padwidth, +1);
            for (unsigned c = 0; c < padwidth; ++c) row[c] = (float)re[c] * rpad;
        }
        free(re); free(im);
    }
    for (size_t r = 0; r < height; ++r) memcpy(img + r * width, pad + r * padwidth + padfactor / 2, width * sizeof(float));
    free(ramp);
    free(pad);
}

/* Volume origin and CBCT row window of project_volume_onto_image_c (fdkbp_single.cpp:302-372)
 * for roi = projection_roi = {0, 0, nu, nv}, volume nu x nu x nv. */
static void fdk_frame(const orc_fdk_geom *g, size_t nu, size_t nv, float origin[3], size_t cb[4])
{
    const size_t sy = nu;
    const size_t roi[4] = {0, 0, nu, nv}, proi3 = nv;
    const float *spacing = g->voxelsize;
    const float U = (float)(roi[2] - roi[0]);
    const float V = (float)(roi[3] - roi[1]);
    origin[0] = -(U - g->center) * spacing[0] - spacing[0] / 2;
    origin[1] = -(U - g->center) * spacing[1] - spacing[1] / 2;
    origin[2] = -(V - (g->ppoint[1] - (float)roi[1])) * spacing[2] - spacing[2] / 2;
    const float radius = (float)sy * g->voxelsize[0] / 2;
    cb[0] = roi[0]; cb[1] = 0; cb[2] = roi[2]; cb[3] = 0;
    const float fp1 = g->ppoint[1], r1 = (float)roi[1], r3 = (float)roi[3];
    const float vx = g->voxelsize[0], sdd = g->sdd, sod = g->sod, res0 = g->resolution[0];
    if (fp1 >= r1 && fp1 >= r3) {
        cb[3] = (size_t)(fp1 - ((fp1 - r3) * vx * sdd / (sod + radius)) / res0);
        float value = fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0;
        cb[1] = value <= 0 ? 0 : (size_t)(fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0);
    }
    if (fp1 < r1 && fp1 < r3) {
        float value = fp1 + ((r1 - fp1) * vx * sdd / (sod + radius)) / res0;
        cb[1] = (size_t)value;
        float value2 = fp1 + ((r3 - fp1) * vx * sdd / (sod - radius)) / res0;
        cb[3] = value2 >= proi3 ? proi3 : (size_t)(float)value2;
    }
    if (fp1 >= r1 && fp1 < r3) {
        float value = fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0;
        cb[1] = value <= 0 ? 0 : (size_t)(fp1 - ((fp1 - r1) * vx * sdd / (sod - radius)) / res0);
        float value2 = fp1 + ((r3 - fp1) * vx * sdd / (sod - radius)) / res0;
        cb[3] = value2 >= proi3 ? proi3 : (size_t)(float)value2;
    }
    if (cb[1] != 0) cb[1] -= 8;
    if (cb[3] + 8 <= proi3) cb[3] += 8;
}

/* FdkReconBase::Process 3D + FDKbp_single::reconstruct/project_volume_onto_image_c
 * (fdkreconbase.cpp:217-277, fdkbp_single.cpp:259-531,641-683). Full detector ROI
 * (roi = projection_roi = {0,0,nu,nv}), volume nu x nu x nv. */
static int fdk_core(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles, const float *weights,
                    const orc_fdk_geom *g, int prefiltered, float *vol)
{
    const size_t sx = nu, sy = nu, sz = nv;
    const size_t npix = nu * nv;
    size_t *mask = (size_t *)malloc(2 * sy * sizeof(size_t));
    circle_mask(sx, sy, g->correcttilt, g->tiltangle, nv, mask);
    float *cbct = (float *)calloc(sx * sy * sz, sizeof(float));
    float *img = (float *)malloc(npix * sizeof(float));
    float *xip = (float *)malloc(3 * sx * sizeof(float));
    float *yip = (float *)malloc(3 * sy * sizeof(float));
    float *zip = (float *)malloc(3 * sz * sizeof(float));
    const size_t roi[4] = {0, 0, nu, nv};

    const float scale = g->sod / g->sdd;
    const float *spacing = g->voxelsize;
    float origin[3];
    size_t cb[4];
    fdk_frame(g, nu, nv, origin, cb);
    const float ic[2] = {g->ppoint[0] - (float)cb[0], g->ppoint[1] - (float)cb[1]};
    const float sad_sid_2 = (g->sod * g->sod) / (g->sdd * g->sdd);

    for (size_t p = 0; p < nproj; ++p) {
        const float *src = proj + p * npix;
        float pm[12];
        orc_fdk_projmatrix(g, nu, angles[p], pm);
        if (prefiltered) {
            memcpy(img, src, npix * sizeof(float));
        } else {
            for (size_t i = 0; i < npix; ++i) img[i] = src[i] * weights[p];
            orc_fdk_ramp(img, nu, nv);
            for (size_t i = 0; i < npix; ++i) {
                img[i] *= sad_sid_2;
                img[i] *= scale;
            }
        }
        for (size_t i = 0; i < sx; ++i) {
            float x = (float)(origin[0] + (float)i * spacing[0]);
            xip[i * 3 + 0] = x * (pm[0] + ic[0] * pm[8]);
            xip[i * 3 + 1] = x * (pm[4] + ic[1] * pm[8]);
            xip[i * 3 + 2] = x * pm[8];
        }
        for (size_t j = 0; j < sy; ++j) {
            float y = (float)(origin[1] + (float)j * spacing[1]);
            yip[j * 3 + 0] = y * (pm[1] + ic[0] * pm[9]);
            yip[j * 3 + 1] = y * (pm[5] + ic[1] * pm[9]);
            yip[j * 3 + 2] = y * pm[9];
        }
        for (size_t k = 0; k < sz; ++k) {
            float z = (float)(origin[2] + (float)k * spacing[2]);
            if (g->correcttilt) {
                float pos = (float)cb[3] - (float)k - g->tiltpivot;
                float cor = (float)(tan(-g->tiltangle * kDPi / 180) * pos + g->center);
                pm[3] = ((cor - (g->ppoint[0] - (float)roi[0])) * g->voxelsize[0]) / g->resolution[0];
            }
            zip[k * 3 + 0] = z * (pm[2] + ic[0] * pm[10]) + ic[0] * pm[11] + pm[3];
            zip[k * 3 + 1] = z * (pm[6] + ic[1] * pm[10]) + ic[1] * pm[11] + pm[7];
            zip[k * 3 + 2] = z * pm[10] + pm[11];
        }
        const float fh = (float)nv, fw = (float)nu;
#pragma omp parallel for schedule(static)
        for (long k = 0; k < (long)sz; ++k) {
            for (size_t j = 0; j < sy; ++j) {
                const float a0 = zip[3 * k] + yip[3 * j];
                const float a1 = zip[3 * k + 1] + yip[3 * j + 1];
                const float a2 = zip[3 * k + 2] + yip[3 * j + 2];
                float *line = cbct + (size_t)k * sy * sx + j * sx;
                for (size_t i = mask[2 * j] + 1; i <= mask[2 * j + 1]; ++i) {
                    const float dw = 1.0f / (a2 + xip[3 * i + 2]);
                    float r = dw * (a1 + xip[3 * i + 1]);
                    float c = dw * (a0 + xip[3 * i]);
                    float val;
                    r += 0.5f;
                    c += 0.5f;
                    if (r < 0 || r >= fh || c < 0 || c >= fw)
                        val = 0.0f;
                    else
                        val = img[(size_t)(int)r * nu + (size_t)(int)c];
                    line[i] += dw * dw * val;
                }
            }
        }
    }
    /* final per-slice horizontal mirror and z reversal (fdkreconbase.cpp:259-270) */
    for (size_t k = 0; k < sz; ++k)
        for (size_t j = 0; j < sy; ++j)
            for (size_t i = 0; i < sx; ++i)
                vol[(sz - k - 1) * sy * sx + j * sx + i] = cbct[k * sy * sx + j * sx + (sx - 1 - i)];
    free(mask); free(cbct); free(img); free(xip); free(yip); free(zip);
    return 0;
}

int orc_fdk(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles, const float *weights,
            const orc_fdk_geom *g, float *vol)
{
    return fdk_core(proj, nu, nv, nproj, angles, weights, g, 0, vol);
}

/* The per-projection image preparation of FdkReconBase::Process + reconstruct +
 * project_volume_onto_image_c: img *= weight, ramp_filter_tuned, cbi *= sad_sid_2, cbi *= scale. */
void orc_fdk_prepare(float *proj, size_t nu, size_t nv, size_t nproj, const float *weights, const orc_fdk_geom *g)
{
    const float scale = g->sod / g->sdd;
    const float sad_sid_2 = (g->sod * g->sod) / (g->sdd * g->sdd);
    for (size_t p = 0; p < nproj; ++p) {
        float *img = proj + p * nu * nv;
        for (size_t i = 0; i < nu * nv; ++i) img[i] = img[i] * weights[p];
        orc_fdk_ramp(img, nu, nv);
        for (size_t i = 0; i < nu * nv; ++i) {
            img[i] *= sad_sid_2;
            img[i] *= scale;
        }
    }
}

/* ---------------------------------------------------- FDK in FP64 (error oracle)
 *
 * FDKbp (fdkbp.cpp:83-640) is FDKbp_single with double geometry. This is that geometry in
 * double, folded into affine maps of the voxel indices (u, v, w rows; 12 doubles per
 * projection): voxel (i, j, k) samples column floor(u/w + 0.5), row floor(v/w + 0.5) with
 * weight (1/w)^2. The row window and the image centre come from the float frame, as in
 * FDKbp_single. Tilt correction folds its per-slice pm[3] (fdkbp_single.cpp:438-444) into
 * the k coefficient of u. */
static void projmatrix64(const orc_fdk_geom *g, double angle, double *pm)
{
    double ext[16] = {0}, intr[12] = {0};
    const double sad = g->sod, sid = g->sdd;
    const double offcenter = ((double)g->ppoint[0] - g->center) * g->voxelsize[0];
    const double a = (g->direction == 0 ? -angle : angle) * kDPi / 180.0;
    const double cam[3] = {sad * cos(a), sad * sin(a), 0.0};
    const double nn = sqrt(cam[0] * cam[0] + cam[1] * cam[1] + cam[2] * cam[2]);
    const double nrm[3] = {cam[0] / nn, cam[1] / nn, cam[2] / nn};
    double plt[3] = {nrm[1], -nrm[0], 0.0}; /* nrm x (0, 0, 1) */
    const double np = sqrt(plt[0] * plt[0] + plt[1] * plt[1]);
    plt[0] /= np;
    plt[1] /= np;
    double pup[3] = {plt[1] * nrm[2] - plt[2] * nrm[1], plt[2] * nrm[0] - plt[0] * nrm[2], plt[0] * nrm[1] - plt[1] * nrm[0]};
    const double nq = sqrt(pup[0] * pup[0] + pup[1] * pup[1] + pup[2] * pup[2]);
    for (int c = 0; c < 3; ++c) {
        pup[c] /= nq;
        ext[c] = -plt[c];
        ext[4 + c] = -pup[c];
        ext[8 + c] = -nrm[c];
    }
    ext[3] = -offcenter;
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

void orc_fdk_maps64(const orc_fdk_geom *g, size_t nu, size_t nv, const float *angles, size_t nproj, double *maps)
{
    float originf[3];
    size_t cb[4];
    fdk_frame(g, nu, nv, originf, cb);
    const double s0 = g->voxelsize[0], s1 = g->voxelsize[1], s2 = g->voxelsize[2];
    const double o0 = -((double)nu - g->center) * s0 - s0 / 2, o1 = -((double)nu - g->center) * s1 - s1 / 2;
    const double o2 = -((double)nv - (double)g->ppoint[1]) * s2 - s2 / 2;
    const double ic0 = (double)g->ppoint[0] - (double)cb[0], ic1 = (double)g->ppoint[1] - (double)cb[1];
    const double tt = g->correcttilt ? tan(-(double)g->tiltangle * kDPi / 180.0) : 0.0;
    for (size_t p = 0; p < nproj; ++p) {
        double pm[12];
        projmatrix64(g, angles[p], pm);
        double pm3 = pm[3], pm3k = 0.0;
        if (g->correcttilt) {
            const double c0 = tt * ((double)cb[3] - g->tiltpivot) + g->center;
            pm3 = ((c0 - g->ppoint[0]) * g->voxelsize[0]) / g->resolution[0];
            pm3k = -tt * g->voxelsize[0] / g->resolution[0];
        }
        const double A[3] = {pm[0] + ic0 * pm[8], pm[4] + ic1 * pm[8], pm[8]};
        const double B[3] = {pm[1] + ic0 * pm[9], pm[5] + ic1 * pm[9], pm[9]};
        const double C[3] = {pm[2] + ic0 * pm[10], pm[6] + ic1 * pm[10], pm[10]};
        const double D[3] = {ic0 * pm[11] + pm3, ic1 * pm[11] + pm[7], pm[11]};
        const double Dk[3] = {pm3k, 0.0, 0.0};
        double *m = maps + p * 12;
        for (int r = 0; r < 3; ++r) {
            m[4 * r + 0] = A[r] * s0;
            m[4 * r + 1] = B[r] * s1;
            m[4 * r + 2] = C[r] * s2 + Dk[r];
            m[4 * r + 3] = A[r] * o0 + B[r] * o1 + C[r] * o2 + D[r];
        }
    }
}

/* FP64 backprojection of FP32 filtered projections for the listed output slices of the
 * final volume (z reversed, x mirrored as in fdkreconbase.cpp:259-270); projections are
 * accumulated in order, as FdkReconBase::Process does. out [nslices][nu][nu]. */
void orc_fdk_bp64(const float *filtered, size_t nu, size_t nv, size_t nproj, const double *maps, const size_t *mask,
                  const int *slices, size_t nslices, double *out)
{
#pragma omp parallel for schedule(dynamic)
    for (long js = 0; js < (long)(nu * nslices); ++js) {
        const size_t s = (size_t)js / nu, j = (size_t)js % nu;
        const double k = (double)(nv - 1 - (size_t)slices[s]);
        double *line = out + (s * nu + j) * nu;
        for (size_t i = 0; i < nu; ++i) line[nu - 1 - i] = 0.0;
        for (size_t i = mask[2 * j] + 1; i <= mask[2 * j + 1] && i < nu; ++i) {
            double acc = 0.0;
            for (size_t p = 0; p < nproj; ++p) {
                const double *m = maps + p * 12;
                const double u = m[0] * (double)i + m[1] * (double)j + m[2] * k + m[3];
                const double v = m[4] * (double)i + m[5] * (double)j + m[6] * k + m[7];
                const double w = m[8] * (double)i + m[9] * (double)j + m[10] * k + m[11];
                const double dw = 1.0 / w;
                const double r = dw * v + 0.5, c = dw * u + 0.5;
                if (r < 0 || r >= (double)nv || c < 0 || c >= (double)nu) continue;
                const double val = filtered[p * nu * nv + (size_t)(int)r * nu + (size_t)(int)c];
                acc += dw * dw * val;
            }
            line[nu - 1 - i] = acc;
        }
    }
}

/* Backprojection and final mirror only, of projections already prepared by orc_fdk_prepare. */
int orc_fdk_bp(const float *filtered, size_t nu, size_t nv, size_t nproj, const float *angles, const orc_fdk_geom *g,
               float *vol)
{
    return fdk_core(filtered, nu, nv, nproj, angles, NULL, g, 1, vol);
}

/* Host geometry of StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:72-79). */
void orc_bp_geometry(const float *angles, size_t n, size_t nu, float center, int direction, float *fsin, float *fcos,
                     float *fstartu)
{
    const float dirweight = 2.0f * ((float)direction - 0.5f);
    const size_t mcx = nu / 2;
    for (size_t k = 0; k < n; ++k) {
        fsin[k] = sinf(dirweight * angles[k] * kFPi / 180.0f);
        fcos[k] = cosf(dirweight * angles[k] * kFPi / 180.0f);
        fstartu[k] = mcx * (fsin[k] - fcos[k]) + center;
    }
}

void orc_circle_mask(size_t nx, size_t ny, int correcttilt, float tiltangle, size_t nslices, size_t *mask)
{
    circle_mask(nx, ny, correcttilt, tiltangle, nslices, mask);
}

/* ---------------------------------------- pair matched to MultiProjBPparallel */

/* Per-projection sin/cos and per-slice start positions of the matched pair: the geometry of
 * StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:72-79) with the detector centre
 * of slice z, c_z = centre + tan_tilt (z - pivot), in float. */
void orc_mbp_geometry(const float *angles, size_t nproj, size_t n, size_t nz, float centre, float tan_tilt,
                      float pivot, int direction, float *sc, float *su)
{
    const float dirweight = 2.0f * ((float)direction - 0.5f);
    const size_t mcx = n / 2;
    for (size_t k = 0; k < nproj; ++k) {
        const float s = sinf(dirweight * angles[k] * kFPi / 180.0f);
        const float c = cosf(dirweight * angles[k] * kFPi / 180.0f);
        sc[2 * k] = s;
        sc[2 * k + 1] = c;
        for (size_t z = 0; z < nz; ++z) {
            const float cz = centre + tan_tilt * ((float)z - pivot);
            su[k * nz + z] = mcx * (s - c) + cz;
        }
    }
}

/* The backprojection of the pair (MultiProjBPparallel.cpp:39-170 without the buffer-drop rule
 * and weights, start position per slice), float, in the reference's order. vol [n][n][nz]. */
void orc_mbp_adjoint(const float *proj, size_t n, size_t nz, const float *sc, const float *su, size_t nproj,
                     const size_t *mask, float *vol)
{
    memset(vol, 0, n * n * nz * sizeof(float));
#pragma omp parallel for schedule(static)
    for (long y = 1; y <= (long)n; ++y) {
        const size_t x0 = mask[2 * (y - 1)], x1 = mask[2 * (y - 1) + 1];
        for (size_t x = x0 + 1; x <= x1; ++x) {
            float *col = vol + ((size_t)(y - 1) * n + (x - 1)) * nz;
            for (size_t i = 0; i < nproj; ++i) {
                const float s = sc[2 * i], c = sc[2 * i + 1];
                for (size_t z = 0; z < nz; ++z) {
                    const float u = (su[i * nz + z] + c * (float)y) - s * (float)x;
                    const int m = (int)u;
                    if (m < 0 || (int)n - 2 < m) continue;
                    const float wb = fabsf(u - (float)m), wa = 1.0f - wb;
                    const float *row = proj + (i * nz + z) * n + (size_t)m;
                    col[z] = col[z] + (row[0] * wa + row[1] * wb);
                }
            }
        }
    }
}

/* The forward projection of the pair as the explicit transpose (scatter over voxels), FP64
 * accumulation. float_u = 1: positions, bins and weights exactly as the kernels form them
 * (the transpose of orc_mbp_adjoint); float_u = 0: everything in double from the geometry
 * parameters (a smooth model in the centre and the tilt for finite differences). dproj (may be
 * NULL) receives d proj / d c_z. */
void orc_mbp_forward64(const float *vol, size_t n, size_t nz, const float *angles, size_t nproj, double centre,
                       double tan_tilt, double pivot, int direction, const size_t *mask, int float_u, double *proj,
                       double *dproj)
{
    memset(proj, 0, nproj * nz * n * sizeof(double));
    if (dproj) memset(dproj, 0, nproj * nz * n * sizeof(double));
    float *sc = (float *)malloc(2 * nproj * sizeof(float));
    float *su = (float *)malloc(nproj * nz * sizeof(float));
    orc_mbp_geometry(angles, nproj, n, nz, (float)centre, (float)tan_tilt, (float)pivot, direction, sc, su);
    const double dirweight = 2.0 * ((double)direction - 0.5);
    const double mcx = (double)(n / 2);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nproj; ++i) {
        const double ds = sin(dirweight * angles[i] * kDPi / 180.0), dc = cos(dirweight * angles[i] * kDPi / 180.0);
        for (size_t y = 1; y <= n; ++y) {
            const size_t x0 = mask[2 * (y - 1)], x1 = mask[2 * (y - 1) + 1];
            for (size_t x = x0 + 1; x <= x1; ++x) {
                const float *col = vol + ((y - 1) * n + (x - 1)) * nz;
                for (size_t z = 0; z < nz; ++z) {
                    double u, wa, wb;
                    int m;
                    if (float_u) {
                        const float s = sc[2 * i], c = sc[2 * i + 1];
                        const float uf = (su[i * nz + z] + c * (float)y) - s * (float)x;
                        m = (int)uf;
                        if (m < 0 || (int)n - 2 < m) continue;
                        const float wbf = fabsf(uf - (float)m);
                        wb = wbf;
                        wa = 1.0f - wbf;
                    } else {
                        const double cz = centre + tan_tilt * ((double)z - pivot);
                        u = (mcx * (ds - dc) + cz + dc * (double)y) - ds * (double)x;
                        m = (int)u;
                        if (m < 0 || (int)n - 2 < m) continue;
                        wb = fabs(u - (double)m);
                        wa = 1.0 - wb;
                    }
                    double *p = proj + ((size_t)i * nz + z) * n + (size_t)m;
                    p[0] += wa * col[z];
                    p[1] += wb * col[z];
                    if (dproj) {
                        double *d = dproj + ((size_t)i * nz + z) * n + (size_t)m;
                        d[0] -= col[z];
                        d[1] += col[z];
                    }
                }
            }
        }
    }
    free(sc);
    free(su);
}

/* ------------------------------------------------------- morphology (kipl) */

/* 2-D neighbourhoods of kipl::morphology::CNeighborhood (core/kipl/kipl/src/morphology/
 * morphology.cpp:25-40): backward half NGm = {0,-1,-sx,-sx-1,-sx+1}, forward half
 * NGp = {0,1,sx,sx+1,sx-1}, full NG = {1,-1,-sx,sx,-sx-1,-sx+1,sx-1,sx+1}; 4-connectivity
 * uses the first 3 / 4 entries. Positions outside the image are rejected (-1), which is
 * what the edge tables of forward2D/backward2D/neighbor2D (:183-470) amount to. */
static const int kBwd[5][2] = {{0, 0}, {-1, 0}, {0, -1}, {-1, -1}, {1, -1}};
static const int kFwd[5][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}, {-1, 1}};
static const int kNbr[8][2] = {{1, 0}, {-1, 0}, {0, -1}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};

static long nb(size_t pos, size_t w, size_t h, const int *d)
{
    long x = (long)(pos % w) + d[0], y = (long)(pos / w) + d[1];
    if (x < 0 || x >= (long)w || y < 0 || y >= (long)h) return -1;
    return y * (long)w + x;
}

typedef struct {
    size_t *v;
    size_t n, cap;
} stack_t_;

static void st_push(stack_t_ *s, size_t x)
{
    if (s->n == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 1024;
        s->v = (size_t *)realloc(s->v, s->cap * sizeof(size_t));
    }
    s->v[s->n++] = x;
}

/* RecByDilation (core/kipl/kipl/include/morphology/morphgeo.h:151-266), including the
 * forward scan that compares the running image but assigns the marker value (:213-214).
 * g: mask, f: marker (f <= g), out: reconstruction. Returns -1 when f > g somewhere. */
int orc_rec_dilation(const float *g, const float *f, size_t w, size_t h, int conn8, float *t)
{
    const size_t n = w * h;
    for (size_t i = 0; i < n; ++i) {
        if (g[i] < f[i]) return -1;
        t[i] = f[i];
    }
    const int cpm = conn8 ? 5 : 3, cng = conn8 ? 8 : 4;
    for (size_t pos = 0; pos < n; ++pos) {
        float mx = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb(pos, w, h, kBwd[i]);
            if (q != -1 && t[q] > mx) mx = f[q];
        }
        t[pos] = mx < g[pos] ? mx : g[pos];
    }
    stack_t_ st = {0};
    for (long pos = (long)n - 1; pos >= 0; --pos) {
        float mx = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb((size_t)pos, w, h, kFwd[i]);
            if (q != -1 && t[q] > mx) mx = t[q];
        }
        t[pos] = mx < g[pos] ? mx : g[pos];
        const float tp = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb((size_t)pos, w, h, kFwd[i]);
            if (q != -1 && t[q] < tp && t[q] < g[q]) {
                st_push(&st, (size_t)pos);
                break;
            }
        }
    }
    while (st.n) {
        size_t pos = st.v[--st.n];
        const float tp = t[pos];
        for (int i = 0; i < cng; ++i) {
            long q = nb(pos, w, h, kNbr[i]);
            if (q != -1 && t[q] < tp && g[q] != t[q]) {
                t[q] = tp < g[q] ? tp : g[q];
                st_push(&st, (size_t)q);
            }
        }
    }
    free(st.v);
    return 0;
}

/* RecByErosion (morphgeo.h:278-371). g: mask, f: marker (f >= g), out: reconstruction. */
void orc_rec_erosion(const float *g, const float *f, size_t w, size_t h, int conn8, float *t)
{
    const size_t n = w * h;
    memcpy(t, f, n * sizeof(float));
    const int cpm = conn8 ? 5 : 3, cng = conn8 ? 8 : 4;
    for (size_t pos = 0; pos < n; ++pos) {
        float mn = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb(pos, w, h, kBwd[i]);
            if (q != -1 && t[q] < mn) mn = t[q];
        }
        t[pos] = mn > g[pos] ? mn : g[pos];
    }
    stack_t_ st = {0};
    for (long pos = (long)n - 1; pos >= 0; --pos) {
        float mn = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb((size_t)pos, w, h, kFwd[i]);
            if (q != -1 && t[q] < mn) mn = t[q];
        }
        t[pos] = mn > g[pos] ? mn : g[pos];
        const float tp = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb((size_t)pos, w, h, kFwd[i]);
            if (q != -1 && t[q] > tp && t[q] > g[q]) {
                st_push(&st, (size_t)pos);
                break;
            }
        }
    }
    while (st.n) {
        size_t pos = st.v[--st.n];
        const float tp = t[pos];
        for (int i = 0; i < cng; ++i) {
            long q = nb(pos, w, h, kNbr[i]);
            if (q != -1 && t[q] > tp && g[q] != t[q]) {
                t[q] = tp > g[q] ? tp : g[q];
                st_push(&st, (size_t)q);
            }
        }
    }
    free(st.v);
}

/* FillHole / FillPeaks (core/kipl/kipl/include/morphology/morphextrema.h:265-328): marker
 * = the image on its border, the image maximum (holes) or minimum (peaks) inside. */
static void extrema_marker(const float *img, size_t w, size_t h, int peaks, float *fm)
{
    float mn = img[0], mx = img[0];
    for (size_t i = 1; i < w * h; ++i) {
        if (img[i] < mn) mn = img[i];
        if (img[i] > mx) mx = img[i];
    }
    for (size_t i = 0; i < w * h; ++i) fm[i] = peaks ? mn : mx;
    memcpy(fm, img, w * sizeof(float));
    memcpy(fm + (h - 1) * w, img + (h - 1) * w, w * sizeof(float));
    for (size_t r = 1; r + 1 < h; ++r) {
        fm[r * w] = img[r * w];
        fm[r * w + w - 1] = img[r * w + w - 1];
    }
}

void orc_fill_hole(const float *img, size_t w, size_t h, int conn8, float *out)
{
    float *fm = (float *)malloc(w * h * sizeof(float));
    extrema_marker(img, w, h, 0, fm);
    orc_rec_erosion(img, fm, w, h, conn8, out);
    free(fm);
}

int orc_fill_peaks(const float *img, size_t w, size_t h, int conn8, float *out)
{
    float *fm = (float *)malloc(w * h * sizeof(float));
    extrema_marker(img, w, h, 1, fm);
    int rc = orc_rec_dilation(img, fm, w, h, conn8, out);
    free(fm);
    return rc;
}

/* The forward raster scan of RecByDilation alone (the marker after :207-215): exposed so
 * the GPU's border-band replay can be checked directly. */
void orc_fill_peaks_forward(const float *img, size_t w, size_t h, int conn8, float *t)
{
    float *fm = (float *)malloc(w * h * sizeof(float));
    extrema_marker(img, w, h, 1, fm);
    memcpy(t, fm, w * h * sizeof(float));
    const int cpm = conn8 ? 5 : 3;
    for (size_t pos = 0; pos < w * h; ++pos) {
        float mx = t[pos];
        for (int i = 1; i < cpm; ++i) {
            long q = nb(pos, w, h, kBwd[i]);
            if (q != -1 && t[q] > mx) mx = fm[q];
        }
        t[pos] = mx < img[pos] ? mx : img[pos];
    }
    free(fm);
}

/* ------------------------------------------------------------- MorphSpotClean */

/* MorphSpotClean::PadEdges (core/algorithms/ImagingAlgorithms/src/MorphSpotClean.cpp:264-300):
 * margin 5, zero columns, the first/last 5 rows mirrored, then an in-place sliding median of
 * `edge` samples along the first and the last padded row. */
static void pad_edges(const float *img, size_t w, size_t h, size_t edge, float *p)
{
    const size_t m = 5, pw = w + 2 * m, ph = h + 2 * m;
    memset(p, 0, pw * ph * sizeof(float));
    for (size_t i = 0; i < h; ++i) memcpy(p + (i + m) * pw + m, img + i * w, w * sizeof(float));
    for (size_t i = 0; i < m; ++i) {
        memcpy(p + (m - 1 - i) * pw + m, img + i * w, w * sizeof(float));
        memcpy(p + (ph - m + i) * pw + m, img + (h - 1 - i) * w, w * sizeof(float));
    }
    const size_t l2 = edge / 2, n = pw - l2;
    float *buf = (float *)malloc(edge * sizeof(float));
    for (int e = 0; e < 2; ++e) {
        float *row = p + (e ? (ph - 1) * pw : 0);
        for (size_t i = l2; i < n; ++i) {
            memcpy(buf, row + i - l2, edge * sizeof(float));
            row[i] = median_f(buf, edge);
        }
    }
    free(buf);
}

/* kipl::math::SigmoidWeights (core/kipl/kipl/include/math/core/mathfunctions.hpp:92-99) */
static float sigmoid_weights(float val, float a, float b, float level, float width)
{
    float w = 1.0f / (1.0f + expf((level - val) / width));
    return a + (b - a) * w;
}

enum { ORC_DETECT_HOLES = 0, ORC_DETECT_PEAKS = 1, ORC_DETECT_BOTH = 2 };

/* MorphSpotClean::process with MorphCleanReplace (MorphSpotClean.cpp:41-175) on one image
 * [h][w]: optional inf/NaN replacement and clamping, padding, FillHole / FillPeaks /
 * both (FillHole of the negated image for peaks), threshold replacement (sigma == 0) or
 * sigmoid blend, unpadding. Returns -1 on a reconstruction error. */
int orc_morphspotclean(float *img, size_t w, size_t h, int detect, int conn8, const float *th, const float *sigma,
                       size_t edge, int clamp, float minlevel, float maxlevel, int removeinfnan)
{
    const size_t n0 = w * h;
    if (removeinfnan) {
        float mx = -3.402823466e38f;
        for (size_t i = 0; i < n0; ++i)
            if (isfinite(img[i]) && mx < img[i]) mx = img[i];
        for (size_t i = 0; i < n0; ++i)
            if (!isfinite(img[i])) img[i] = mx;
    }
    if (clamp)
        for (size_t i = 0; i < n0; ++i) {
            if (img[i] < minlevel) img[i] = minlevel;
            else if (img[i] > maxlevel) img[i] = maxlevel;
        }
    const size_t pw = w + 10, ph = h + 10, n = pw * ph;
    float *p = (float *)malloc(n * sizeof(float));
    float *holes = (float *)malloc(n * sizeof(float));
    float *peaks = (float *)malloc(n * sizeof(float));
    pad_edges(img, w, h, edge, p);
    int rc = 0;
    if (detect == ORC_DETECT_HOLES || detect == ORC_DETECT_BOTH) orc_fill_hole(p, pw, ph, conn8, holes);
    if (detect == ORC_DETECT_PEAKS) rc = orc_fill_peaks(p, pw, ph, conn8, peaks);
    if (detect == ORC_DETECT_BOTH) {
        for (size_t i = 0; i < n; ++i) p[i] = -p[i];
        orc_fill_hole(p, pw, ph, conn8, peaks);
        for (size_t i = 0; i < n; ++i) {
            p[i] = -p[i];
            peaks[i] = -peaks[i];
        }
    }
    if (rc == 0) {
        if (sigma[0] == 0.0f && sigma[1] == 0.0f) {
            for (size_t i = 0; i < n; ++i) {
                const float val = p[i];
                if ((detect == ORC_DETECT_HOLES || detect == ORC_DETECT_BOTH) && th[0] < fabsf(val - holes[i]))
                    p[i] = holes[i];
                if ((detect == ORC_DETECT_PEAKS || detect == ORC_DETECT_BOTH) && th[1] < fabsf(peaks[i] - val))
                    p[i] = peaks[i];
            }
        } else {
            for (size_t i = 0; i < n; ++i) {
                const float val = p[i];
                if (detect == ORC_DETECT_HOLES)
                    p[i] = sigmoid_weights(holes[i] - val, val, holes[i], th[0], sigma[0]);
                else if (detect == ORC_DETECT_PEAKS)
                    p[i] = sigmoid_weights(val - peaks[i], val, peaks[i], th[1], sigma[1]);
                else {
                    const float dp = val - peaks[i], dh = holes[i] - val;
                    if (fabsf(dh) < fabsf(dp))
                        p[i] = sigmoid_weights(dp, val, peaks[i], th[0], sigma[0]);
                    else
                        p[i] = sigmoid_weights(dh, val, holes[i], th[1], sigma[1]);
                }
            }
        }
        for (size_t i = 0; i < h; ++i) memcpy(img + i * w, p + (i + 5) * pw + 5, w * sizeof(float));
    }
    free(p);
    free(holes);
    free(peaks);
    return rc;
}

/* ------------------------------------------------------------ StripeFilter */

/* WaveletTransform::pad_mirror (core/kipl/kipl/include/wavelets/core/wavelets.hpp:648-667):
 * value at position p of the mirrored buffer (the odd-length extra sample is never read). */
static float mirror_at(const float *src, int n, int fw, int p)
{
    if (p < fw) return src[fw - 1 - p];
    if (p < fw + n) return src[p - fw];
    return src[n - 1 - (p - fw - n)];
}

/* One analysis level (wavelets.hpp:474-600): rows with `hr`, columns with `vc`, output
 * (dx, dy) = ((sx + K - 1 + (sx & 1))/2, (sy + K - 1 + (sy & 1))/2); each output is the sum
 * over the taps in order from 0. */
static void dwt_pass(const float *src, int sx, int sy, const float *hr, const float *vc, int begin, int end, float *dst,
                     int dx, int dy)
{
    const int fw = end - begin + 1;
    float *tmp = (float *)calloc((size_t)dx * sy, sizeof(float));
    for (int y = 0; y < sy; ++y)
        for (int k = 0; k < dx; ++k) {
            float acc = 0.0f;
            for (int j = begin; j <= end; ++j) acc = acc + hr[j] * mirror_at(src + (size_t)y * sx, sx, fw, fw + 2 * k - j + 1);
            tmp[(size_t)y * dx + k] = acc;
        }
    float *col = (float *)malloc(sy * sizeof(float));
    for (int x = 0; x < dx; ++x) {
        for (int y = 0; y < sy; ++y) col[y] = tmp[(size_t)y * dx + x];
        for (int k = 0; k < dy; ++k) {
            float acc = 0.0f;
            for (int m = begin; m <= end; ++m) acc = acc + vc[m] * mirror_at(col, sy, fw, fw + 2 * k - m + 1);
            dst[(size_t)k * dx + x] = acc;
        }
    }
    free(col);
    free(tmp);
}

/* value at position q of pad_mirror(dyadup(src, n), 2n, fw) (wavelets.hpp:741-748, 771-780) */
static float up_at(const float *src, int n, int fw, int q, int stride)
{
    int t;
    if (q < fw) t = fw - 1 - q;
    else if (q < fw + 2 * n) t = q - fw;
    else t = 2 * n - 1 - (q - fw - 2 * n);
    return (t & 1) ? 0.0f : src[(size_t)(t / 2) * stride];
}

/* WaveletTransform::upsconvRC (wavelets.hpp:750-862): src (w, h) -> dst (dx, dy). */
static void upsconv(const float *src, int w, int h, float *dst, int dx, int dy, const float *kh, const float *kv,
                    int begin, int end)
{
    const int fw = end - begin + 1, c = fw - 2;
    float *rows = (float *)calloc((size_t)dx * h, sizeof(float));
    for (int y = 0; y < h; ++y)
        for (int k = 0; k < dx; ++k) {
            float acc = 0.0f;
            for (int m = begin; m <= end; ++m) acc = acc + up_at(src + (size_t)y * w, w, fw, fw + k + c - m, 1) * kh[m];
            rows[(size_t)y * dx + k] = acc;
        }
    for (int x = 0; x < dx; ++x)
        for (int k = 0; k < dy; ++k) {
            float acc = 0.0f;
            for (int m = begin; m <= end; ++m) acc = acc + up_at(rows + x, h, fw, fw + k + c - m, dx) * kv[m];
            dst[(size_t)k * dx + x] = acc;
        }
    free(rows);
}

/* kipl::math::fft::NextPower2 (core/kipl/kipl/src/fft/zeropadding.cpp:10-15) */
static size_t next_power2(size_t n)
{
    const double logtwo = log(2.0);
    return (size_t)floor(exp(logtwo * ceil(log((double)n) / logtwo)) + 0.5);
}

/* StripeFilter::process with VerticalComponentFFT (core/algorithms/ImagingAlgorithms/src/
 * StripeFilter.cpp:68-135,214-250) on one sinogram [ntheta][nu]. kern: the four float
 * filters of WaveletKernel (analysis H, analysis G, synthesis H, synthesis G), each
 * end-begin+1 long. Returns -1 when the image is smaller than the kernel. */
int orc_stripefilter(float *img, size_t nu, size_t ntheta, const float *kern, int begin, int end, int nlevels,
                     float sigma)
{
    const int K = end - begin + 1;
    const float *tH = kern, *tG = kern + K, *sH = kern + 2 * K, *sG = kern + 3 * K;
    int sx[17], sy[17];
    float *a[17], *h[17], *v[17], *d[17];
    sx[0] = (int)nu;
    sy[0] = (int)ntheta;
    a[0] = img;
    for (int l = 0; l < nlevels; ++l) {
        if (sx[l] < K || sy[l] < K) {
            for (int q = 1; q <= l; ++q) { free(a[q]); free(h[q]); free(v[q]); free(d[q]); }
            return -1;
        }
        sx[l + 1] = (sx[l] + K - 1 + (sx[l] & 1)) / 2;
        sy[l + 1] = (sy[l] + K - 1 + (sy[l] & 1)) / 2;
        size_t n = (size_t)sx[l + 1] * sy[l + 1];
        a[l + 1] = (float *)malloc(n * sizeof(float));
        h[l + 1] = (float *)malloc(n * sizeof(float));
        v[l + 1] = (float *)malloc(n * sizeof(float));
        d[l + 1] = (float *)malloc(n * sizeof(float));
        dwt_pass(a[l], sx[l], sy[l], tH, tH, begin, end, a[l + 1], sx[l + 1], sy[l + 1]);
        dwt_pass(a[l], sx[l], sy[l], tH, tG, begin, end, h[l + 1], sx[l + 1], sy[l + 1]);
        dwt_pass(a[l], sx[l], sy[l], tG, tH, begin, end, v[l + 1], sx[l + 1], sy[l + 1]);
        dwt_pass(a[l], sx[l], sy[l], tG, tG, begin, end, d[l + 1], sx[l + 1], sy[l + 1]);
    }
    /* FilterVerticalStripes on every level's v band (:114-135) with CreateFilterWindow (:68-81) */
    const float s = -1.0f / (2.0f * sigma * sigma);
    for (int l = 0; l < nlevels; ++l) {
        const size_t L = next_power2((size_t)(1.25 * (double)(int)ntheta) >> l);
        const size_t N = 2 * L;
        const float scale = 1.0f / (2.0f * L);
        float *damp = (float *)malloc(N * sizeof(float));
        for (size_t i = 0; i < N; ++i) {
            float w = (float)i * scale;
            damp[i] = (1.0f - expf(w * w * s)) * scale;
        }
        double *re = (double *)malloc(N * sizeof(double)), *im = (double *)malloc(N * sizeof(double));
        float *band = v[l + 1];
        const int bw = sx[l + 1], bh = sy[l + 1];
        for (int x = 0; x < bw; ++x) {
            for (size_t i = 0; i < N; ++i) { re[i] = (int)i < bh ? band[(size_t)i * bw + x] : 0.0; im[i] = 0.0; }
            fft_c2c(re, im, N, -1);
            for (size_t i = 0; i <= N / 2; ++i) {
                re[i] = (double)(float)((float)re[i] * damp[i]);
                im[i] = (double)(float)((float)im[i] * damp[i]);
            }
            im[0] = 0.0;
            im[N / 2] = 0.0;
            for (size_t k = 1; k < N / 2; ++k) { re[N - k] = re[k]; im[N - k] = -im[k]; }
            fft_c2c(re, im, N, +1);
            for (int i = 0; i < bh; ++i) band[(size_t)i * bw + x] = (float)re[i];
        }
        free(re);
        free(im);
        free(damp);
    }
    /* synthesize (wavelets.hpp:603-645): approximation of level l from level l+1 */
    for (int l = nlevels - 1; l >= 0; --l) {
        const int dx = l == 0 ? 2 * sx[1] : sx[l], dy = l == 0 ? 2 * sy[1] : sy[l];
        const size_t n = (size_t)dx * dy;
        float *acc = (float *)malloc(n * sizeof(float)), *tmp = (float *)malloc(n * sizeof(float));
        const int w = sx[l + 1], hh = sy[l + 1];
        upsconv(a[l + 1], w, hh, acc, dx, dy, sH, sH, begin, end);
        upsconv(h[l + 1], w, hh, tmp, dx, dy, sH, sG, begin, end);
        for (size_t i = 0; i < n; ++i) acc[i] += tmp[i];
        upsconv(v[l + 1], w, hh, tmp, dx, dy, sG, sH, begin, end);
        for (size_t i = 0; i < n; ++i) acc[i] += tmp[i];
        upsconv(d[l + 1], w, hh, tmp, dx, dy, sG, sG, begin, end);
        for (size_t i = 0; i < n; ++i) acc[i] += tmp[i];
        if (l == 0) {
            for (size_t y = 0; y < ntheta; ++y) memcpy(img + y * nu, acc + y * (size_t)dx, nu * sizeof(float));
        } else {
            memcpy(a[l], acc, n * sizeof(float));
        }
        free(acc);
        free(tmp);
    }
    for (int q = 1; q <= nlevels; ++q) { free(a[q]); free(h[q]); free(v[q]); free(d[q]); }
    return 0;
}

/* ------------------------------------------------ Joseph projector pair (FP64)
 *
 * LinearForwardProjector::project 2-D (linearforwardprojector.cpp:15-144) applied to every
 * slice z of a volume [nz][n][n] (x fastest), with the detector centre of slice z at
 * centre + tan_tilt * (z - pivot) instead of the reference's fixed R/2 (rho = r - centre;
 * centre = nu/2, tan_tilt = 0 is the reference's geometry). Angles in degrees. For
 * |sin| > sqrt(1/2) the ray steps along x (m) and interpolates along y at
 * nf = beta + m alpha, alpha = -cos/sin, beta = (rho - x_min (cos + sin)) / sin, weight
 * 1/|sin|; otherwise it steps along y and interpolates along x with sin/cos swapped. A
 * sample counts when 0 <= nf < n - 1 (the effective range of the reference's mmin/mmax
 * window and in-loop test). Positions are formed as beta + m alpha, not accumulated.
 * proj [nproj][nz][nu]. */
typedef struct {
    int major_y;
    double alpha, inv, d, rho_off;
} joseph_angle;

static joseph_angle joseph_geometry(float angle_deg, size_t n)
{
    joseph_angle g;
    const double x_min = -(double)(long)(n / 2);
    const double th = (double)angle_deg * kDPi / 180.0;
    const double sn = sin(th), cs = cos(th);
    g.rho_off = x_min * (cs + sn);
    if (fabs(sn) > sqrt(0.5)) {
        g.major_y = 0;
        g.alpha = -cs / sn;
        g.inv = 1.0 / sn;
        g.d = 1.0 / fabs(sn);
    } else {
        g.major_y = 1;
        g.alpha = -sn / cs;
        g.inv = 1.0 / cs;
        g.d = 1.0 / fabs(cs);
    }
    return g;
}

void orc_joseph_forward64(const float *vol, size_t n, size_t nz, const float *angles, size_t nproj, size_t nu,
                          double centre, double tan_tilt, double pivot, double *proj, double *dproj_dc)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (long t = 0; t < (long)nproj; ++t)
        for (long z = 0; z < (long)nz; ++z) {
            const joseph_angle g = joseph_geometry(angles[t], n);
            const double cz = centre + tan_tilt * ((double)z - pivot);
            const float *sl = vol + (size_t)z * n * n;
            for (size_t r = 0; r < nu; ++r) {
                const double beta = ((double)r - cz - g.rho_off) * g.inv;
                double sum = 0.0, dsum = 0.0;
                for (size_t k = 0; k < n; ++k) {
                    const double f = beta + (double)k * g.alpha;
                    if (!(f >= 0.0 && f < (double)(n - 1))) continue;
                    const size_t i0 = (size_t)f;
                    const double w = f - (double)i0;
                    double s0, s1;
                    if (g.major_y) {
                        s0 = sl[k * n + i0];
                        s1 = sl[k * n + i0 + 1];
                    } else {
                        s0 = sl[i0 * n + k];
                        s1 = sl[(i0 + 1) * n + k];
                    }
                    sum += s0 + w * (s1 - s0);
                    dsum += s1 - s0;
                }
                proj[((size_t)t * nz + z) * nu + r] = sum * g.d;
                if (dproj_dc) dproj_dc[((size_t)t * nz + z) * nu + r] = -dsum * g.inv * g.d;
            }
        }
}

/* The exact transpose of orc_joseph_forward64 (scatter form). vol [nz][n][n] overwritten. */
void orc_joseph_adjoint64(const double *proj, size_t n, size_t nz, const float *angles, size_t nproj, size_t nu,
                          double centre, double tan_tilt, double pivot, double *vol)
{
#pragma omp parallel for schedule(static)
    for (long z = 0; z < (long)nz; ++z) {
        double *sl = vol + (size_t)z * n * n;
        for (size_t i = 0; i < n * n; ++i) sl[i] = 0.0;
        const double cz = centre + tan_tilt * ((double)z - pivot);
        for (size_t t = 0; t < nproj; ++t) {
            const joseph_angle g = joseph_geometry(angles[t], n);
            for (size_t r = 0; r < nu; ++r) {
                const double v = proj[(t * nz + (size_t)z) * nu + r] * g.d;
                const double beta = ((double)r - cz - g.rho_off) * g.inv;
                for (size_t k = 0; k < n; ++k) {
                    const double f = beta + (double)k * g.alpha;
                    if (!(f >= 0.0 && f < (double)(n - 1))) continue;
                    const size_t i0 = (size_t)f;
                    const double w = f - (double)i0;
                    if (g.major_y) {
                        sl[k * n + i0] += (1.0 - w) * v;
                        sl[k * n + i0 + 1] += w * v;
                    } else {
                        sl[i0 * n + k] += (1.0 - w) * v;
                        sl[(i0 + 1) * n + k] += w * v;
                    }
                }
            }
        }
    }
}

/* Slice serialisation: ReconEngine::Serialize (frameworks/tomography/Framework/ReconFramework/
 * src/ReconEngine.cpp:576-700) -> kipl::io::WriteImageStack (core/kipl/kipl/include/io/
 * io_stack.h:114-230): each slice cut out by ExtractSlice (base/core/textractor.hpp:17-125,
 * plane XY = 1 or YZ = 4, optional inclusive ROI, swapped when reversed) and cast by
 * ImageCaster<unsigned short, float>::cast (base/core/imagecast.hpp:33-52):
 * scale = float(65535) / (hi - lo); out = (unsigned short)((min(max(v, lo), hi) - lo) * scale)
 * with std::max / std::min (a NaN passes both; its cast is undefined in C and gives 0 on x86,
 * which is what is written here). vol: dims (d0, d1, d2), d0 fastest. */
int orc_slices_u16(const float *vol, size_t d0, size_t d1, size_t d2, int plane, size_t first, size_t count,
                   const size_t *roi, float lo, float hi, unsigned short *out)
{
    const size_t nslices = plane == 1 ? d2 : d0;
    const size_t na = plane == 1 ? d0 : d1, nb = plane == 1 ? d1 : d2;
    size_t a0 = 0, b0 = 0, w = na, h = nb;
    if ((plane != 1 && plane != 4) || first + count > nslices) return -1;
    if (roi) {
        const size_t x0 = roi[0] < roi[2] ? roi[0] : roi[2], x1 = roi[0] < roi[2] ? roi[2] : roi[0];
        const size_t y0 = roi[1] < roi[3] ? roi[1] : roi[3], y1 = roi[1] < roi[3] ? roi[3] : roi[1];
        if (x1 >= na || y1 >= nb) return -1;
        a0 = x0;
        b0 = y0;
        w = x1 - x0 + 1;
        h = y1 - y0 + 1;
    }
    const float scale = 65535.0f / (hi - lo);
    for (size_t s = 0; s < count; ++s)
        for (size_t b = 0; b < h; ++b)
            for (size_t a = 0; a < w; ++a) {
                const size_t src = plane == 1 ? ((first + s) * d1 + (b0 + b)) * d0 + (a0 + a)
                                              : ((b0 + b) * d1 + (a0 + a)) * d0 + (first + s);
                const float v = vol[src];
                const float m = v < lo ? lo : v;
                const float c = hi < m ? hi : m;
                const float val = (c - lo) * scale;
                out[(s * h + b) * w + a] = val != val ? 0 : (unsigned short)val;
            }
    return 0;
}

/* ------------------------------------------------------- alternative ring cleaners */

/* Heap sort as kipl::heapsort does it (core/kipl/kipl/include/algorithms/sortalg.h:10-45):
 * the Numerical Recipes sift-down form with 1-based positions and strict '<' comparisons, so
 * that equal keys of different bits (+0 / -0) and NaN (false in both directions) end where
 * the reference puts them. */
static void nr_heapsort(float *a, int n)
{
    if (n < 2) return;
    int l = (n >> 1) + 1, ir = n;
    for (;;) {
        float v;
        if (l > 1) {
            --l;
            v = a[l - 1];
        } else {
            v = a[ir - 1];
            a[ir - 1] = a[0];
            if (--ir == 1) {
                a[0] = v;
                break;
            }
        }
        int i = l, j = l + l;
        while (j <= ir) {
            if (j < ir && a[j - 1] < a[j]) j++;
            if (v < a[j - 1]) {
                a[i - 1] = a[j - 1];
                i = j;
                j <<= 1;
            } else {
                j = ir + 1;
            }
        }
        a[i - 1] = v;
    }
}

/* Element idx of an image of n values; positions at or past its end read 0 (the reference's
 * edge handling reads a few values past the last row; the zero there is the convention this
 * restatement and the CUDA path share, and the reference oracle gives its buffers a zeroed
 * tail so that it reads the same). */
static float img_at(const float *img, size_t n, long long idx)
{
    return idx >= 0 && (size_t)idx < n ? img[idx] : 0.0f;
}

/* The kx*ky window (row-major) that TMedianFilter::ExtractNeighborhood builds at (x, y)
 * (core/kipl/kipl/include/filters/core/medianfilter.hpp:52-159): the edge code from the
 * unsigned comparisons, the per-code ranges (including the bottom-right range that reaches past
 * the row), the zero start, then the left, right, top and bottom replications in that order.
 * Returns -1 for the codes the reference rejects. */
static int kipl_window(const float *img, size_t w, size_t h, int kx, int ky, size_t x, size_t y, float *win)
{
    const int hx = kx >> 1, hy = ky >> 1;
    const int code = (x < (size_t)hx) + 2 * ((w - (size_t)hx - 1) < x) + 4 * (y < (size_t)hy) +
                     8 * ((h - (size_t)hy - 1) < y);
    long long sx = -hx, ex = kx - hx, sy = -hy, ey = ky - hy;
    const long long rx = (long long)kx - hx - (long long)(w - x), ry = (long long)ky - hy - (long long)(h - y);
    switch (code) {
    case 1: sx = -(long long)x; break;
    case 2: ex = rx; break;
    case 3: case 7: return -1;
    case 4: sy = -(long long)y; break;
    case 5: sx = -(long long)x; sy = -(long long)y; break;
    case 6: ex = rx; sy = -(long long)y; break;
    case 8: ey = ry; break;
    case 9: sx = -(long long)x; ey = ry; break;
    case 10: ey = ry; ex = rx + 1; break;
    default: break;
    }
    const size_t n = w * h;
    for (int i = 0; i < kx * ky; ++i) win[i] = 0.0f;
    const long long base = (long long)(y * w + x);
    for (long long dy = sy; dy < ey; ++dy)
        for (long long dx = sx; dx < ex; ++dx)
            win[(dy + hy) * kx + (dx + hx)] = img_at(img, n, base + dy * (long long)w + dx);
    if (code & 1)
        for (int r = 0; r < ky; ++r)
            for (long long d = sx - 1, s = sx; d >= -hx; --d, ++s) win[r * kx + d + hx] = win[r * kx + s + hx];
    if (code & 2)
        for (int r = 0; r < ky; ++r)
            for (long long s = ex - 1, d = ex; d < kx - hx; --s, ++d) win[r * kx + d + hx] = win[r * kx + s + hx];
    if (code & 4)
        for (long long d = sy - 1, s = sy; d >= -hy; --d, ++s)
            for (int c = 0; c < kx; ++c) win[(d + hy) * kx + c] = win[(s + hy) * kx + c];
    if (code & 8)
        for (long long s = ey - 1, d = ey; d < ky - hy; --s, ++d)
            for (int c = 0; c < kx; ++c) win[(d + hy) * kx + c] = win[(s + hy) * kx + c];
    return code;
}

/* kipl::filters::TMedianFilter<float,2>::operator() with odd kx, ky (HeapSortMedianFilter,
 * medianfilter.hpp:173-199, and kipl::math::median, math/core/median.hpp:10-22): per pixel the
 * window above, heap-sorted, middle element. Needs w >= 2*(kx/2) and h >= 2*(ky/2), the sizes
 * at which the reference reads only inside the image and the value-past-the-end above. */
int orc_median_filter(const float *img, size_t w, size_t h, int kx, int ky, float *out)
{
    if (kx < 1 || ky < 1 || !(kx & 1) || !(ky & 1) || kx * ky > 49 || w < 1 || h < 1 ||
        w < (size_t)(2 * (kx >> 1)) || h < (size_t)(2 * (ky >> 1)))
        return -1;
    float win[49];
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            if (kipl_window(img, w, h, kx, ky, x, y, win) < 0) return -1;
            nr_heapsort(win, kx * ky);
            out[y * w + x] = win[(kx * ky) / 2];
        }
    return 0;
}

/* Mean projection of n projections of npix values, accumulated in projection order:
 * from_zero = 0 starts from a copy of the first (BasicRingClean.cpp:56-63), 1 from zero
 * (MedianMixRingClean.cpp:113-121); then times 1.0f / n. */
static void mean_projection(const float *proj, size_t npix, size_t n, int from_zero, float *mean)
{
    size_t i0 = 0;
    if (from_zero) {
        for (size_t j = 0; j < npix; ++j) mean[j] = 0.0f;
    } else {
        memcpy(mean, proj, npix * sizeof(float));
        i0 = 1;
    }
    for (size_t i = i0; i < n; ++i)
        for (size_t j = 0; j < npix; ++j) mean[j] += proj[i * npix + j];
    const float scale = 1.0f / (float)n;
    for (size_t j = 0; j < npix; ++j) mean[j] *= scale;
}

/* BasicRingClean::ProcessCore (frameworks/tomography/Preprocessing/StdPreprocModules/src/
 * BasicRingClean.cpp:50-95): mean projection, its 3x3 median, and every projection minus
 * (mean - median). The debug images the reference writes (mean.tif, med.tif, diff.tif in the
 * working directory) are not part of the result. Projections [n][h][w], in place. */
int orc_basicringclean(float *proj, size_t w, size_t h, size_t n)
{
    if (w < 2 || h < 2) return -1;
    if (n == 0) return 0;
    const size_t npix = w * h;
    float *mean = (float *)malloc(npix * sizeof(float)), *med = (float *)malloc(npix * sizeof(float));
    mean_projection(proj, npix, n, 0, mean);
    orc_median_filter(mean, w, h, 3, 3, med);
    for (size_t j = 0; j < npix; ++j) med[j] = mean[j] - med[j];
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < npix; ++j) proj[i * npix + j] -= med[j];
    free(mean);
    free(med);
    return 0;
}

/* kipl::math::SigmoidLUT (core/kipl/kipl/src/math/LUTCollection.cpp:38-82) on LUTbase
 * (core/kipl/kipl/src/math/LUTbase.cpp:12-20): limits from epsilon = sigma * 1e-3 with the
 * double log the reference calls, slope (len - 1) / (hi - lo) and intercept -slope * lo + 0.5 in
 * float, entries 1 / (1 + exp((lambda - x) / sigma)) in double stored as float with x stepping
 * by 1 / slope in float, first entry 0 and last 1. param: lo, hi, slope, intercept. */
void orc_sigmoid_lut(size_t len, float lambda, float sigma, float *lut, float *param)
{
    const float eps = sigma * 1e-3f;
    const float lo = (float)((double)lambda - (double)sigma * log((double)(1.0f / eps)));
    const float hi = (float)((double)lambda - (double)sigma * log((double)(1.0f / (1.0f - eps) - 1.0f)));
    const float slope = (float)(len - 1) / (hi - lo);
    const float intercept = -slope * lo + 0.5f;
    const float invwidth = 1.0f / sigma, delta = 1.0f / slope;
    float x = lo;
    for (size_t i = 0; i < len; ++i, x += delta) lut[i] = (float)(1.0f / (1.0f + exp((double)((lambda - x) * invwidth))));
    lut[0] = 0.0f;
    lut[len - 1] = 1.0f;
    param[0] = lo;
    param[1] = hi;
    param[2] = slope;
    param[3] = intercept;
}

/* LUTbase::BasicLUT (LUTbase.cpp:57-75) for one value. Where the reference's index leaves the
 * table (a NaN value, or a cancellation in slope * value + intercept when lambda is far larger
 * than the width; the reference then reads past its table) the index is clamped to it. */
static float lut_apply(const float *lut, size_t len, const float *param, float v)
{
    if (v < param[0]) return lut[0];
    if (param[1] < v) return lut[len - 1];
    const float f = v * param[2] + param[3];
    if (!(f >= 0.0f)) return lut[0];
    if (f >= (float)len) return lut[len - 1];
    size_t idx = (size_t)f;
    return lut[idx > len - 1 ? len - 1 : idx];
}

/* MedianMixRingClean::ProcessCore and ComputeProfile (frameworks/tomography/Preprocessing/
 * StdPreprocModules/src/MedianMixRingClean.cpp:57-138): weights = SigmoidLUT(1024, threshold,
 * width) of |mean projection - its 3x3 median| (5x1 when h < 3); every projection becomes
 * (1 - w) * p + w * (its 5x5 median, 5x1 when h < 5). Projections [n][h][w], in place. */
int orc_medianmixringclean(float *proj, size_t w, size_t h, size_t n, float threshold, float width)
{
    if (w < 4 || h < 1) return -1;
    if (n == 0) return 0;
    const size_t npix = w * h, len = 1024;
    float *mean = (float *)malloc(npix * sizeof(float)), *wt = (float *)malloc(npix * sizeof(float));
    float *med = (float *)malloc(npix * sizeof(float)), lut[1024], param[4];
    mean_projection(proj, npix, n, 1, mean);
    if (h < 3)
        orc_median_filter(mean, w, h, 5, 1, wt);
    else
        orc_median_filter(mean, w, h, 3, 3, wt);
    for (size_t j = 0; j < npix; ++j) wt[j] = fabsf(mean[j] - wt[j]);
    orc_sigmoid_lut(len, threshold, width, lut, param);
    for (size_t j = 0; j < npix; ++j) wt[j] = lut_apply(lut, len, param, wt[j]);
    for (size_t i = 0; i < n; ++i) {
        float *p = proj + i * npix;
        orc_median_filter(p, w, h, 5, h < 5 ? 1 : 5, med);
        for (size_t j = 0; j < npix; ++j) p[j] = (1.0f - wt[j]) * p[j] + wt[j] * med[j];
    }
    free(mean);
    free(wt);
    free(med);
    return 0;
}

/* ----------------------------------------------------------- SpotClean (SpotClean2) */

/* Source value for output (x, y) at (xx, yy) as kipl TFilterBase<float,2> with EdgeMirror
 * reads it (core/kipl/kipl/include/filters/core/filterbase.hpp:83-128,246-408): outputs in the
 * top and bottom ky/2 rows come from buffers mirrored vertically about the edge row (no
 * repeat) and padded horizontally with the edge value; outputs in the left and right kx/2
 * columns of the remaining rows from buffers mirrored horizontally; the rest read the image. */
static float mirror_src(const float *img, int w, int h, int kx, int ky, int x, int y, int xx, int yy)
{
    const int cx = kx / 2, cy = ky / 2;
    if (y < cy || y >= h - cy) {
        if (yy < 0) yy = -yy;
        else if (yy >= h) yy = 2 * (h - 1) - yy;
        if (xx < 0) xx = 0;
        else if (xx >= w) xx = w - 1;
    } else if (x < cx || x >= w - cx) {
        if (xx < 0) xx = -xx;
        else if (xx >= w) xx = 2 * (w - 1) - xx;
    }
    return img[(size_t)yy * w + xx];
}

enum { KF_SUM = 0, KF_MIN = 1, KF_MAX = 2 };

/* TFilter (sum of value * kernel from 0, filter.hpp:10-15), TErode (min from FLT_MAX) and
 * TDilate (max from -FLT_MAX, morphology/core/morphfilters.hpp:10-75): the kernel's nonzero
 * entries in row-major order (ProcessCore, filterbase.hpp:83-128), EdgeMirror edges. */
static void kipl_filter(const float *img, int w, int h, const float *k, int kx, int ky, int op, float *out)
{
    const int cx = kx / 2, cy = ky / 2;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            float acc = op == KF_SUM ? 0.0f : op == KF_MIN ? 3.402823466e+38f : -3.402823466e+38f;
            for (int i = 0; i < kx * ky; ++i) {
                if (k[i] == 0.0f) continue;
                const float v = mirror_src(img, w, h, kx, ky, x, y, x + i % kx - cx, y + i / kx - cy);
                if (op == KF_SUM) acc = acc + v * k[i];
                else if (op == KF_MIN) acc = v < acc ? v : acc; /* std::min(dest, src) */
                else acc = acc < v ? v : acc;                  /* std::max(dest, src) */
            }
            out[(size_t)y * w + x] = acc;
        }
}

/* SpotClean::BoxFilter (core/algorithms/ImagingAlgorithms/src/SpotClean.cpp:447-465): a sum
 * over dim values along x, then along y, each with EdgeMirror edges. */
static void box_filter(const float *img, int w, int h, int dim, float *tmp, float *out)
{
    float ones[7] = {1, 1, 1, 1, 1, 1, 1};
    kipl_filter(img, w, h, ones, dim, 1, KF_SUM, tmp);
    kipl_filter(tmp, w, h, ones, 1, dim, KF_SUM, out);
}

/* kipl::filters::StdDevFilter(dim, EdgeMirror)::operator() (core/kipl/kipl/src/filters/
 * stddevfilter.cpp:25-64): box sums of img^2 and img, sqrt(M1 * (s2 - M * m * m)) with
 * M = 1/(dim*dim), M1 = 1/(dim*dim - 1) in float. */
static void stddev_filter(const float *img, int w, int h, int dim, float *out)
{
    const size_t n = (size_t)w * h;
    float *a = (float *)calloc(n, sizeof(float)), *b = (float *)malloc(n * sizeof(float));
    float *c = (float *)malloc(n * sizeof(float)), *d = (float *)malloc(n * sizeof(float));
    for (size_t i = 0; i < n; ++i) a[i] = img[i] * img[i];
    box_filter(a, w, h, dim, c, b); /* s2 */
    box_filter(img, w, h, dim, c, d); /* m */
    const float M = 1 / (float)(dim * dim), M1 = 1 / (float)(dim * dim - 1);
    for (size_t i = 0; i < n; ++i) out[i] = (float)sqrt((double)(M1 * (b[i] - M * d[i] * d[i])));
    free(a);
    free(b);
    free(c);
    free(d);
}

/* kipl::math::statistics (core/kipl/kipl/include/math/core/image_statistics.hpp:197-219):
 * running mean and variance in double, variance / N, standard deviation. */
static void running_stats(const float *x, size_t n, double *mean, double *sd)
{
    double m = 0.0, var = 0.0;
    for (size_t i = 0; i < n;) {
        const double value = x[i];
        const double delta = value - m;
        i++;
        m += delta / (double)i;
        var += delta * (value - m);
    }
    var = var / (double)n;
    *mean = m;
    *sd = sqrt(var);
}

/* SpotClean::DetectionImage (SpotClean.cpp:388-545) for method 0 stddev, 1 ring, 2 median,
 * 3 minmax, 4 trikernel; gamma is the TriKernel level factor. */
static int spot_detection(const float *img, int w, int h, int method, float gamma, float *det)
{
    const size_t n = (size_t)w * h;
    float *a = (float *)malloc(n * sizeof(float)), *b = (float *)malloc(n * sizeof(float));
    float *c = (float *)malloc(n * sizeof(float)), *d = (float *)malloc(n * sizeof(float));
    int rc = 0;
    if (method == 1) { /* RingDetection: 5x5 ring of 1/12, centre -1, then |.| */
        const float wv = 1.0f / 12.0f, cv = -1.0f, z = 0.0f;
        const float k[25] = {z, wv, wv, wv, z, wv, z, z, z, wv, wv, z, cv, z, wv, wv, z, z, z, wv, z, wv, wv, wv, z};
        kipl_filter(img, w, h, k, 5, 5, KF_SUM, det);
        for (size_t i = 0; i < n; ++i) det[i] = fabsf(det[i]);
    } else if (method == 0) { /* StdDevDetection(img, 3): the same arithmetic as StdDevFilter */
        stddev_filter(img, w, h, 3, det);
    } else if (method == 2) { /* MedianDetection: 1x5 then 5x1 median, |img - median| */
        orc_median_filter(img, (size_t)w, (size_t)h, 1, 5, a);
        orc_median_filter(a, (size_t)w, (size_t)h, 5, 1, b);
        for (size_t i = 0; i < n; ++i) det[i] = fabsf(img[i] - b[i]);
    } else if (method == 3) { /* MinMaxDetection: 1x5 then 5x1 erosion and dilation */
        const float se[5] = {1, 1, 1, 1, 1};
        kipl_filter(img, w, h, se, 1, 5, KF_MIN, a);
        kipl_filter(a, w, h, se, 5, 1, KF_MIN, b);
        kipl_filter(img, w, h, se, 1, 5, KF_MAX, a);
        kipl_filter(a, w, h, se, 5, 1, KF_MAX, c);
        for (size_t i = 0; i < n; ++i) det[i] = fabsf(c[i] - b[i]);
    } else if (method == 4) { /* TriKernel: OneKernel for 3, 5, 7 */
        for (size_t i = 0; i < n; ++i) det[i] = 0.0f;
        for (int size = 3; size <= 7; size += 2) {
            box_filter(img, w, h, size, c, a);
            for (size_t i = 0; i < n; ++i) a[i] = fabsf(img[i] - a[i]);
            double m, sd;
            running_stats(a, n, &m, &sd);
            const float level = (float)(m + (double)gamma * sd);
            for (size_t i = 0; i < n; ++i) det[i] = (det[i] != 0.0f || level < a[i]) ? 1.0f : 0.0f;
        }
    } else {
        rc = -1;
    }
    free(a);
    free(b);
    free(c);
    free(d);
    return rc;
}

/* SpotClean::ExcludeLargeRegions (SpotClean.cpp:248-285) with kipl LabelImage (8-connected
 * components of s != 0), LabelArea (every label's count and LAST index, the background label 0
 * included) and RemoveConnectedRegion (morphology/label.h): each label with area > maxarea
 * is removed by a flood from its last pixel through nonzero labels; the flood from the
 * background's last pixel removes the components next to it. Then s = 0 on label 0. */
static void exclude_large_regions(float *s, int w, int h, int maxarea)
{
    if (maxarea == 0) return;
    const size_t n = (size_t)w * h;
    int *lbl = (int *)calloc(n, sizeof(int));
    size_t *stack = (size_t *)malloc(n * sizeof(size_t));
    size_t cnt = 0;
    for (size_t p = 0; p < n; ++p) {
        if (lbl[p] || s[p] == 0.0f) continue;
        ++cnt;
        size_t top = 0;
        lbl[p] = (int)cnt;
        stack[top++] = p;
        while (top) {
            const size_t q = stack[--top];
            for (int j = 0; j < 8; ++j) {
                const long r = nb(q, (size_t)w, (size_t)h, kNbr[j]);
                if (r >= 0 && s[r] != 0.0f && !lbl[r]) {
                    lbl[r] = (int)cnt;
                    stack[top++] = (size_t)r;
                }
            }
        }
    }
    size_t *area = (size_t *)calloc(cnt + 1, sizeof(size_t)), *last = (size_t *)calloc(cnt + 1, sizeof(size_t));
    for (size_t i = 0; i < n; ++i) {
        area[lbl[i]]++;
        last[lbl[i]] = i;
    }
    size_t nseed = 0;
    size_t *seeds = (size_t *)malloc((cnt + 1) * sizeof(size_t));
    for (size_t l = 0; l <= cnt; ++l)
        if ((size_t)maxarea < area[l]) seeds[nseed++] = last[l];
    for (size_t i = 0; i < nseed; ++i) lbl[seeds[i]] = 0;
    for (size_t i = 0; i < nseed; ++i) {
        size_t top = 0;
        stack[top++] = seeds[i];
        while (top) {
            const size_t q = stack[--top];
            for (int j = 0; j < 8; ++j) {
                const long r = nb(q, (size_t)w, (size_t)h, kNbr[j]);
                if (r >= 0 && lbl[r] != 0) {
                    lbl[r] = 0;
                    stack[top++] = (size_t)r;
                }
            }
        }
    }
    for (size_t i = 0; i < n; ++i)
        if (lbl[i] == 0) s[i] = 0.0f;
    free(lbl);
    free(stack);
    free(area);
    free(last);
    free(seeds);
}

/* One projection of SpotClean::Process (SpotClean.cpp:78-108): DetectSpots (:185-246: the
 * detection image through SigmoidLUT(1 << 15, gamma, sigma), large regions excluded, pixels
 * outside [minlevel, maxlevel] or with a nonzero weight become spots and are marked with
 * FLT_MAX) and CleanByArray (:287-336 with PrepareNeighborhood / Neighborhood :338-365: every
 * round, each remaining spot with unmarked neighbours among the linear offsets
 * {-w-1,-w,-w+1,-1,1,w-1,w,w+1} (the first row, up to index w, skips the row above; index 0
 * also the left one; the last row skips the row below; nothing wraps differently at the side
 * columns) moves by weight * (mean - value); the new values are written after the round).
 * Returns -2 when a round corrects nothing while spots remain (the reference loops forever). */
static int spotclean_one(float *img, int w, int h, int method, float gamma, float sigma, float minlevel,
                         float maxlevel, int maxarea, const float *lut, const float *param, size_t len)
{
    const size_t n = (size_t)w * h;
    const float mark = 3.402823466e+38f;
    float *s = (float *)malloc(n * sizeof(float)), *res = (float *)malloc(n * sizeof(float));
    size_t *pos = (size_t *)malloc(n * sizeof(size_t)), *next = (size_t *)malloc(n * sizeof(size_t));
    float *val = (float *)malloc(n * sizeof(float)), *wt = (float *)malloc(n * sizeof(float));
    float *nval = (float *)malloc(n * sizeof(float)), *nwt = (float *)malloc(n * sizeof(float));
    int rc = spot_detection(img, w, h, method, gamma, s);
    if (rc == 0) {
        for (size_t i = 0; i < n; ++i) s[i] = lut_apply(lut, len, param, s[i]);
        exclude_large_regions(s, w, h, maxarea);
        memcpy(res, img, n * sizeof(float));
        size_t np = 0;
        for (size_t i = 0; i < n; ++i) {
            if (res[i] < minlevel || maxlevel < res[i]) {
                pos[np] = i; val[np] = res[i]; wt[np] = 1.0f; np++;
                res[i] = mark;
            } else if (s[i] != 0.0f) {
                pos[np] = i; val[np] = res[i]; wt[np] = s[i]; np++;
                res[i] = mark;
            }
        }
        static const int off_dx[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, off_dy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
        float *newv = (float *)malloc((np ? np : 1) * sizeof(float));
        unsigned char *done = (unsigned char *)malloc(np ? np : 1);
        while (np) {
            size_t nc = 0;
            for (size_t k = 0; k < np; ++k) {
                const long long idx = (long long)pos[k];
                const int start = (long long)w < idx ? 0 : (idx != 0 ? 3 : 4);
                const int stop = idx < (long long)(n - w) ? 8 : 5;
                float sum = 0.0f;
                int cntn = 0;
                for (int i = start; i < stop; ++i) {
                    const float v = img_at(res, n, idx + off_dy[i] * (long long)w + off_dx[i]);
                    if (v != mark) {
                        sum += v;
                        cntn++;
                    }
                }
                done[k] = cntn != 0;
                if (cntn) {
                    const float mean = sum / (float)cntn;
                    newv[k] = val[k] + wt[k] * (mean - val[k]);
                    nc++;
                }
            }
            if (nc == 0) {
                rc = -2;
                break;
            }
            size_t nr = 0;
            for (size_t k = 0; k < np; ++k) {
                if (done[k]) {
                    res[pos[k]] = newv[k];
                } else {
                    next[nr] = pos[k]; nval[nr] = val[k]; nwt[nr] = wt[k]; nr++;
                }
            }
            memcpy(pos, next, nr * sizeof(size_t));
            memcpy(val, nval, nr * sizeof(float));
            memcpy(wt, nwt, nr * sizeof(float));
            np = nr;
        }
        free(newv);
        free(done);
        if (rc == 0) {
            for (size_t i = 0; i < n; ++i)
                if (res[i] == mark) rc = -3;
            memcpy(img, res, n * sizeof(float));
        }
    }
    free(s); free(res); free(pos); free(next); free(val); free(wt); free(nval); free(nwt);
    return rc;
}

/* SpotClean2::ProcessCore 3D -> ImagingAlgorithms::SpotClean::Process (SpotClean.cpp:78-108):
 * `iterations` passes over every projection [n][h][w], in place. method: 0 stddev, 1 ring,
 * 2 median, 3 minmax, 4 trikernel. */
int orc_spotclean(float *proj, size_t w, size_t h, size_t n, int method, float gamma, float sigma, int iterations,
                  float minlevel, float maxlevel, int maxarea)
{
    if (w < 16 || h < 16 || method < 0 || method > 4) return -1;
    const size_t len = (size_t)1 << 15;
    float *lut = (float *)malloc(len * sizeof(float)), param[4];
    orc_sigmoid_lut(len, gamma, sigma, lut, param);
    int rc = 0;
    for (int it = 0; it < iterations && rc == 0; ++it)
        for (size_t i = 0; i < n && rc == 0; ++i)
            rc = spotclean_one(proj + i * w * h, (int)w, (int)h, method, gamma, sigma, minlevel, maxlevel, maxarea, lut,
                               param, len);
    free(lut);
    return rc;
}

/* ------------------------------------------------------------- projection weights */

/* ComputeWeights (frameworks/tomography/Framework/ReconFramework/src/ReconHelpers.cpp:365-488)
 * on BuildFileList's multimap (:100-110): key = angle modulo 180, equal keys in acquisition
 * order (a stable insertion sort here), weight 1 to start. Outputs the resulting map in its
 * order (angle, weight); returns its size. arc0/arc1: ProjectionInfo.fScanArc. */
size_t orc_compute_weights(const float *angles, size_t n, float arc0, float arc1, int golden, float *out_angles,
                           float *out_weights)
{
    float *k = (float *)malloc((n ? n : 1) * sizeof(float)), *a = (float *)malloc((n ? n : 1) * sizeof(float));
    float *w = (float *)malloc((n ? n : 1) * sizeof(float));
    for (size_t i = 0; i < n; ++i) {
        float key = fmodf(angles[i], 180.0f), ang = angles[i];
        size_t j = i;
        while (j > 0 && key < k[j - 1]) { /* after equal keys: multimap insertion order */
            k[j] = k[j - 1];
            a[j] = a[j - 1];
            j--;
        }
        k[j] = key;
        a[j] = ang;
        w[i] = 1.0f;
    }
    size_t m = 0;
    if (n < 3) {
        for (size_t i = 0; i < n; ++i) {
            if (i > 0 && k[i] == k[i - 1]) continue; /* map::insert keeps the first */
            out_angles[m] = a[i];
            out_weights[m++] = (float)(1.0 / (double)n);
        }
    } else {
        for (size_t i = 1; i + 1 < n; ++i) w[i] = k[i] != k[i - 1] ? (k[i + 1] - k[i - 1]) / 360.0f : 0.0f;
        if (175.0f < arc1 - arc0) {
            int repeated_last = 0;
            if (k[n - 1] != k[n - 2]) {
                w[n - 1] = ((k[0] + 180) - k[n - 2]) / 360.0f;
            } else {
                w[n - 1] = 0.0f;
                repeated_last = 1;
            }
            if (repeated_last || golden)
                w[0] = (k[1] - (k[n - 1] - 180)) / 360.0f;
            else
                w[0] = (k[1] - (k[n - 1] - 180)) / 180.0f;
        } else {
            w[0] = w[1];
            w[n - 1] = w[1];
        }
        /* runs of zero weights share the weight of the entry before them (the reference reads
         * past the end of its list when the run reaches it; the run simply ends there) */
        for (size_t q = 1; q < n;) {
            if (w[q] == 0.0f) {
                size_t before = q - 1, run = 0;
                do {
                    run++;
                    q++;
                } while (q < n && w[q] == 0.0f);
                float v = w[before] / (float)(run + 1);
                for (size_t t = before; t <= before + run; ++t) w[t] = v;
            } else {
                q++;
            }
        }
        float sum = 0.0f;
        for (size_t i = 0; i < n; ++i) sum += w[i];
        int twice = fabsf(sum - 0.5f) < 0.001f;
        /* std::map keyed by the angle: sorted, a repeated angle keeps the last entry */
        for (size_t i = 0; i < n; ++i) {
            size_t pos = 0;
            while (pos < m && out_angles[pos] < a[i]) pos++;
            if (pos < m && out_angles[pos] == a[i]) {
                out_weights[pos] = w[i];
                continue;
            }
            for (size_t t = m; t > pos; --t) {
                out_angles[t] = out_angles[t - 1];
                out_weights[t] = out_weights[t - 1];
            }
            out_angles[pos] = a[i];
            out_weights[pos] = w[i];
            m++;
        }
        if (twice)
            for (size_t i = 0; i < m; ++i) out_weights[i] *= 2;
    }
    free(k);
    free(a);
    free(w);
    return m;
}
