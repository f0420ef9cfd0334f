// C-ABI harness around the reference's own CPU modules (test infrastructure only).
//
// This translation unit is compiled against the reference headers and linked with the
// reference sources (see oracle/ref/Makefile). It exposes each hot-path module through
// plain pointers so the tests can run the UNMODIFIED reference code on the same seeded
// inputs as the CUDA path. Nothing here is on the product path: only tests/ and the
// CPU-baseline leg of bench.py load the resulting oracle/_ref/libmuhrec_ref.so.
//
// The reference modules normally receive their inputs through the engine (file reader,
// XML config). The harness sets the same fields in code instead:
//   * ReconConfig fields are assigned directly (frameworks/tomography/Framework/
//     ReconFramework/include/ReconConfig.h:77-175);
//   * per-projection doses and the reference-frame doses follow ProjectionReader::
//     GetProjectionDose (ProjectionReader.cpp:752-783): median of the row means inside
//     the dose ROI;
//   * reference frames are averaged with ImagingAlgorithms::AverageImage exactly as
//     NormBase::ReferenceLoader does (NormPlugins.cpp:91-230), then handed to
//     FullLogNorm::SetReferenceImages (NormPlugins.cpp:300-341).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <functional>
#include <iostream>
#include <iterator>
#include <list>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

// Module internals (reference images, doses, protected ProcessCore) are set/called
// directly, so member access is opened for the reference headers only.
#define protected public
#define private public
#include <base/timage.h>
#include <base/textractor.h>
#include <base/imagecast.h>
#include <ReconConfig.h>
#include <ParameterHandling.h>
#include <averageimage.h>
#include <MorphSpotClean.h>
#include <StripeFilter.h>
#include <math/median.h>
#include "NormPlugins.h"
#include "ProjectionFilter.h"
#include "MorphSpotCleanModule.h"
#include "BasicRingClean.h"
#include "MedianMixRingClean.h"
#include "GammaSpotCleanModule.h"
#include "SpotClean2.h"
#include <ReconHelpers.h>
#include <filters/medianfilter.h>
#include <math/LUTCollection.h>
#include "WaveletRingClean.h"
#include "MultiProjBPparallel.h"
#include "MultiProjBP.h"
#include "NNMultiProjBP.h"
#include "fdkbp_single.h"
#include "fdkbp.h"
#include "linearforwardprojector.h"
#include <wavelets/wavelets.h>
#include <ModuleItem.h>
#include <io/io_matlab.h>
#undef private
#undef protected
#include <dlfcn.h>
#include <tiffio.h>

namespace {

std::string g_error;

std::string list_text(const float *v, size_t n)
{
    std::ostringstream s;
    char buf[64];
    for (size_t i = 0; i < n; ++i) {
        std::snprintf(buf, sizeof(buf), "%.9g", static_cast<double>(v[i]));
        if (i) s << ' ';
        s << buf;
    }
    return s.str();
}

// ProjectionReader::GetProjectionDose restated on an in-memory frame
// (ProjectionReader.cpp:760-782): median over rows of the row mean inside roi.
float frame_dose(const float *frame, size_t nu, const size_t *roi)
{
    if (!(roi[0] * roi[1] * roi[2] * roi[3])) return 1.0f;
    const size_t w = roi[2] - roi[0], h = roi[3] - roi[1];
    std::vector<float> means(h, 0.0f);
    for (size_t y = 0; y < h; ++y) {
        const float *p = frame + (roi[1] + y) * nu + roi[0];
        for (size_t x = 0; x < w; ++x) means[y] += p[x];
        means[y] = means[y] / static_cast<float>(w);
    }
    float dose = 0.0f;
    kipl::math::median(means.data(), h, &dose);
    return dose;
}

template <typename F>
int guarded(F f)
{
    try {
        f();
        return 0;
    } catch (kipl::base::KiplException &e) {
        g_error = e.what();
    } catch (std::exception &e) {
        g_error = e.what();
    } catch (...) {
        g_error = "unknown exception";
    }
    return -1;
}

} // namespace

extern "C" {

const char *ref_last_error() { return g_error.c_str(); }

// The reference modules log through kipl::logging::Logger to standard output. Callers keep
// only errors (which are also thrown), so that their own standard output stays clean.
void ref_quiet_logging() { kipl::logging::Logger::SetLogLevel(kipl::logging::Logger::LogError); }

float ref_frame_dose(const float *frame, size_t nu, const size_t *roi) { return frame_dose(frame, nu, roi); }

// ImagingAlgorithms::AverageImage::operator() (averageimage.cpp:35-61)
int ref_average(const float *stack, size_t nu, size_t nv, size_t n, int method, float *out)
{
    return guarded([&] {
        size_t dims[3] = {nu, nv, n};
        kipl::base::TImage<float, 3> img(dims);
        std::memcpy(img.GetDataPtr(), stack, sizeof(float) * nu * nv * n);
        ImagingAlgorithms::AverageImage avg;
        kipl::base::TImage<float, 2> r = avg(img, static_cast<ImagingAlgorithms::AverageImage::eAverageMethod>(method));
        std::memcpy(out, r.GetDataPtr(), sizeof(float) * nu * nv);
    });
}

// FullLogNorm: reference preparation (ReferenceLoader + SetReferenceImages) and
// ProcessCore 3D (NormPlugins.cpp:411-552) on projections [nproj][nv][nu].
// dose_roi is in projection coordinates (x0,y0,x1,y1); all-zero disables dose ROI use.
// uselut selects the module's LogLUT path.
int ref_fulllognorm(float *proj, size_t nu, size_t nv, size_t nproj,
                    const float *darks, size_t ndark, const float *flats, size_t nflat,
                    int refavg, int usenormregion, const size_t *dose_roi,
                    float *dark_out, float *flat_out, float *doses_out, float *refdoses_out, int uselut)
{
    return guarded([&] {
        FullLogNorm mod;
        ReconConfig cfg;
        cfg.ProjectionInfo.nDCCount = ndark;
        cfg.ProjectionInfo.nOBCount = nflat;
        std::memcpy(cfg.ProjectionInfo.dose_roi, dose_roi, 4 * sizeof(size_t));
        std::map<std::string, std::string> par;
        par["usenormregion"] = usenormregion ? "true" : "false";
        par["uselut"] = uselut ? "true" : "false";
        ImagingAlgorithms::AverageImage::eAverageMethod m =
            static_cast<ImagingAlgorithms::AverageImage::eAverageMethod>(refavg);
        par["referenceaverage"] = enum2string(m);
        mod.Configure(cfg, par);

        size_t d2[2] = {nu, nv};
        ImagingAlgorithms::AverageImage avg;
        kipl::base::TImage<float, 2> dark(d2), flat(d2);
        float darkdose = 0.0f, flatdose = 1.0f;
        if (ndark) {
            size_t d3[3] = {nu, nv, ndark};
            kipl::base::TImage<float, 3> st(d3);
            std::memcpy(st.GetDataPtr(), darks, sizeof(float) * nu * nv * ndark);
            float dose = 0.0f;
            for (size_t i = 0; i < ndark; ++i) {
                float t = usenormregion ? frame_dose(darks + i * nu * nv, nu, dose_roi) : 0.0f;
                dose = i == 0 ? t : dose + t;
            }
            darkdose = dose / static_cast<float>(ndark);
            dark = avg(st, m);
        }
        if (nflat) {
            size_t d3[3] = {nu, nv, nflat};
            kipl::base::TImage<float, 3> st(d3);
            std::memcpy(st.GetDataPtr(), flats, sizeof(float) * nu * nv * nflat);
            float dose = 0.0f;
            for (size_t i = 0; i < nflat; ++i) {
                float t = (usenormregion ? frame_dose(flats + i * nu * nv, nu, dose_roi) : 1.0f) - darkdose;
                dose = i == 0 ? t : dose + t;
            }
            flatdose = dose / static_cast<float>(nflat);
            flat = avg(st, m);
        }
        mod.fDarkDose = darkdose;
        mod.fFlatDose = flatdose;
        if (dark_out) std::memcpy(dark_out, dark.GetDataPtr(), sizeof(float) * nu * nv);
        mod.SetReferenceImages(dark, flat);
        if (flat_out) std::memcpy(flat_out, mod.mFlatField.GetDataPtr(), sizeof(float) * nu * nv);
        if (refdoses_out) {
            refdoses_out[0] = darkdose;
            refdoses_out[1] = flatdose;
        }

        std::vector<float> doses(nproj, 1.0f);
        if (usenormregion)
            for (size_t i = 0; i < nproj; ++i) doses[i] = frame_dose(proj + i * nu * nv, nu, dose_roi);
        if (doses_out) std::memcpy(doses_out, doses.data(), sizeof(float) * nproj);
        std::map<std::string, std::string> coeff;
        coeff["dose"] = list_text(doses.data(), nproj);

        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * nu * nv * nproj);
    });
}

// ProjectionFilterSingle (ProjectionFilter.cpp:254-376) on projections [nproj][nv][nu].
int ref_projfilter(float *proj, size_t nu, size_t nv, size_t nproj, const char *filtertype,
                   float cutoff, float order, int usebias, float biasweight, int paddingdoubler,
                   float *filter_out, size_t *nfft_out)
{
    return guarded([&] {
        ProjectionFilterSingle mod(nullptr);
        ReconConfig cfg;
        cfg.ProjectionInfo.roi[0] = 0;
        cfg.ProjectionInfo.roi[1] = 0;
        cfg.ProjectionInfo.roi[2] = nu;
        cfg.ProjectionInfo.roi[3] = nv;
        std::map<std::string, std::string> par;
        par["filtertype"] = filtertype;
        char b[64];
        std::snprintf(b, sizeof(b), "%.9g", cutoff);
        par["cutoff"] = b;
        std::snprintf(b, sizeof(b), "%.9g", order);
        par["order"] = b;
        par["usebias"] = usebias ? "true" : "false";
        std::snprintf(b, sizeof(b), "%.9g", biasweight);
        par["biasweight"] = b;
        par["paddingdoubler"] = std::to_string(paddingdoubler);
        mod.Configure(cfg, par);
        if (nfft_out) *nfft_out = mod.nFFTsize;
        if (filter_out) std::memcpy(filter_out, mod.mFilter.GetDataPtr(), sizeof(float) * mod.mFilter.Size());
        if (proj && nproj) {
            size_t d3[3] = {nu, nv, nproj};
            kipl::base::TImage<float, 3> img(d3);
            std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
            std::map<std::string, std::string> coeff;
            mod.Process(img, coeff);
            std::memcpy(proj, img.GetDataPtr(), sizeof(float) * nu * nv * nproj);
        }
    });
}

// MultiProjectionBPparallel (MultiProjBPparallel.cpp:39-170) driven through
// StdBackProjectorBase::Process 3D (StdBackProjectorBase.cpp:120-149).
// proj: [nproj][nv][nu]; vol out: ZXY [nu (y)][nu (x)][nv (z)].
// variant 1 selects the serial MultiProjectionBP (MultiProjBP.cpp:36-146), 2 NearestNeighborBP
// (NNMultiProjBP.cpp:36-121).
int ref_bp_parallel(const float *proj, size_t nu, size_t nv, size_t nproj,
                    const float *angles, const float *weights, float center, int direction,
                    size_t buffersize, int correcttilt, float tiltangle, float tiltpivot,
                    size_t roi_y0, int serial, float *vol)
{
    return guarded([&] {
        ReconConfig cfg;
        cfg.ProjectionInfo.fCenter = center;
        cfg.ProjectionInfo.eDirection = static_cast<kipl::base::eRotationDirection>(direction);
        cfg.ProjectionInfo.bCorrectTilt = correcttilt != 0;
        cfg.ProjectionInfo.fTiltAngle = tiltangle;
        cfg.ProjectionInfo.fTiltPivotPosition = tiltpivot;
        cfg.ProjectionInfo.imagetype = ReconConfig::cProjections::ImageType_Projections;
        cfg.ProjectionInfo.beamgeometry = ReconConfig::cProjections::BeamGeometry_Parallel;
        cfg.ProjectionInfo.nDims[0] = nu;
        cfg.ProjectionInfo.nDims[1] = nv;
        cfg.MatrixInfo.bUseROI = false;
        std::map<std::string, std::string> par;
        par["ProjectionBufferSize"] = std::to_string(buffersize);
        par["SliceBlock"] = "32";
        par["SubVolume"] = "1 1";
        StdBackProjectorBase *bp = nullptr;
        if (serial == 1)
            bp = new MultiProjectionBP(nullptr);
        else if (serial == 2)
            bp = new NearestNeighborBP(nullptr);
        else
            bp = new MultiProjectionBPparallel(nullptr);
        std::unique_ptr<StdBackProjectorBase> hold(bp);
        bp->Configure(cfg, par);
        size_t roi[4] = {0, roi_y0, nu, roi_y0 + nv};
        bp->SetROI(roi);
        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        std::map<std::string, std::string> params;
        params["angles"] = list_text(angles, nproj);
        params["weights"] = list_text(weights, nproj);
        bp->Process(img, params);
        std::memcpy(vol, bp->volume.GetDataPtr(), sizeof(float) * bp->volume.Size());
    });
}

struct ref_fdk_geom {
    float sod, sdd;
    float ppoint[2];
    float center;
    float resolution[2];
    float voxelsize[3];
    int direction;
    int correcttilt;
    float tiltangle;
    float tiltpivot;
};

// FDKbp_single (fdkbp_single.cpp:83-994) through FdkReconBase::Process 3D
// (fdkreconbase.cpp:217-277). proj: [nproj][nv][nu]; vol out: XYZ [nv][nu][nu]
// after the final mirror/z-reversal; cbct_out (optional) before it.
extern "C++" {
template <typename Module>
static void run_fdk(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles, const float *weights,
                    const ref_fdk_geom *g, float *vol, float *cbct_out);
}

int ref_fdk(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
            const float *weights, const ref_fdk_geom *g, float *vol, float *cbct_out)
{
    return guarded([&] { run_fdk<FDKbp_single>(proj, nu, nv, nproj, angles, weights, g, vol, cbct_out); });
}

// The factory's FDKbp (double-precision geometry, fdkbp.cpp) on the same inputs.
int ref_fdk_double(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
                   const float *weights, const ref_fdk_geom *g, float *vol, float *cbct_out)
{
    return guarded([&] { run_fdk<FDKbp>(proj, nu, nv, nproj, angles, weights, g, vol, cbct_out); });
}

extern "C++" {
static ReconConfig fdk_config(size_t nu, size_t nv, size_t nproj, const ref_fdk_geom *g)
{
    ReconConfig cfg;
    cfg.ProjectionInfo.fSOD = g->sod;
    cfg.ProjectionInfo.fSDD = g->sdd;
    cfg.ProjectionInfo.fpPoint[0] = g->ppoint[0];
    cfg.ProjectionInfo.fpPoint[1] = g->ppoint[1];
    cfg.ProjectionInfo.fCenter = g->center;
    cfg.ProjectionInfo.fResolution[0] = g->resolution[0];
    cfg.ProjectionInfo.fResolution[1] = g->resolution[1];
    cfg.MatrixInfo.fVoxelSize[0] = g->voxelsize[0];
    cfg.MatrixInfo.fVoxelSize[1] = g->voxelsize[1];
    cfg.MatrixInfo.fVoxelSize[2] = g->voxelsize[2];
    cfg.ProjectionInfo.eDirection = static_cast<kipl::base::eRotationDirection>(g->direction);
    cfg.ProjectionInfo.bCorrectTilt = g->correcttilt != 0;
    cfg.ProjectionInfo.fTiltAngle = g->tiltangle;
    cfg.ProjectionInfo.fTiltPivotPosition = g->tiltpivot;
    cfg.ProjectionInfo.imagetype = ReconConfig::cProjections::ImageType_Projections;
    cfg.ProjectionInfo.beamgeometry = ReconConfig::cProjections::BeamGeometry_Cone;
    cfg.ProjectionInfo.nDims[0] = nu;
    cfg.ProjectionInfo.nDims[1] = nv;
    cfg.ProjectionInfo.nFirstIndex = 0;
    cfg.ProjectionInfo.nLastIndex = nproj - 1;
    cfg.ProjectionInfo.nProjectionStep = 1;
    size_t roi[4] = {0, 0, nu, nv};
    std::memcpy(cfg.ProjectionInfo.roi, roi, sizeof(roi));
    std::memcpy(cfg.ProjectionInfo.projection_roi, roi, sizeof(roi));
    cfg.MatrixInfo.nDims[0] = nu;
    cfg.MatrixInfo.nDims[1] = nu;
    cfg.MatrixInfo.nDims[2] = nv;
    cfg.MatrixInfo.bUseROI = false;
    return cfg;
}
} // extern "C++"

// BackProjectorModuleBase::GetSlice (BackProjectorModuleBase.cpp:62-128) of a volume given
// with its kipl dims (d0 fastest): zxy = 1 on a MultiProjectionBPparallel (MatrixZXY), 0 on an
// FDKbp_single (MatrixXYZ); use_roi/roi set MatrixInfo.bUseROI and MatrixInfo.roi. out gets the
// slice, out_dims its two sizes.
int ref_getslice(const float *vol, size_t d0, size_t d1, size_t d2, int zxy, int use_roi, const size_t *roi,
                 size_t idx, float *out, size_t *out_dims)
{
    return guarded([&] {
        std::unique_ptr<BackProjectorModuleBase> bp;
        if (zxy)
            bp.reset(new MultiProjectionBPparallel(nullptr));
        else
            bp.reset(new FDKbp_single(nullptr));
        size_t d3[3] = {d0, d1, d2};
        bp->volume.Resize(d3);
        std::memcpy(bp->volume.GetDataPtr(), vol, sizeof(float) * d0 * d1 * d2);
        bp->mConfig.MatrixInfo.bUseROI = use_roi != 0;
        if (use_roi) std::memcpy(bp->mConfig.MatrixInfo.roi, roi, 4 * sizeof(size_t));
        kipl::base::TImage<float, 2> s = bp->GetSlice(idx);
        out_dims[0] = s.Size(0);
        out_dims[1] = s.Size(1);
        std::memcpy(out, s.GetDataPtr(), sizeof(float) * s.Size());
    });
}

// A configured FDKbp_single that keeps its volume between Process calls, as ReconEngine
// keeps one backprojector per slice block and hands it projections (Configure and SetROI
// once, then Process 3D; each Process adds into cbct_volume and redoes the final mirror).
// Used to time the reference per projection without its per-block set-up.
struct ref_fdk_session {
    FDKbp_single *fdk;
    size_t nu, nv;
};

void *ref_fdk_session_create(size_t nu, size_t nv, size_t nproj_total, const ref_fdk_geom *g)
{
    ref_fdk_session *s = nullptr;
    int rc = guarded([&] {
        std::unique_ptr<ref_fdk_session> hold(new ref_fdk_session{new FDKbp_single(nullptr), nu, nv});
        std::map<std::string, std::string> par;
        par["ProjectionBufferSize"] = "16";
        par["SliceBlock"] = "32";
        par["SubVolume"] = "1 1";
        hold->fdk->Configure(fdk_config(nu, nv, nproj_total, g), par);
        size_t roi[4] = {0, 0, nu, nv};
        hold->fdk->SetROI(roi);
        s = hold.release();
    });
    return rc == 0 ? s : nullptr;
}

int ref_fdk_session_process(void *session, const float *proj, size_t nproj, const float *angles,
                            const float *weights)
{
    return guarded([&] {
        ref_fdk_session *s = static_cast<ref_fdk_session *>(session);
        size_t d3[3] = {s->nu, s->nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * s->nu * s->nv * nproj);
        std::map<std::string, std::string> params;
        params["angles"] = list_text(angles, nproj);
        params["weights"] = list_text(weights, nproj);
        s->fdk->Process(img, params);
    });
}

// Copies the final volume (after the last Process call's mirror) to vol [nv][nu][nu].
int ref_fdk_session_volume(void *session, float *vol)
{
    return guarded([&] {
        ref_fdk_session *s = static_cast<ref_fdk_session *>(session);
        std::memcpy(vol, s->fdk->volume.GetDataPtr(), sizeof(float) * s->fdk->volume.Size());
    });
}

void ref_fdk_session_destroy(void *session)
{
    ref_fdk_session *s = static_cast<ref_fdk_session *>(session);
    if (!s) return;
    delete[] s->fdk->proj_matrices;
    delete s->fdk;
    delete s;
}

extern "C++" {
template <typename Module>
static void run_fdk(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles, const float *weights,
                    const ref_fdk_geom *g, float *vol, float *cbct_out)
{
    {
        ReconConfig cfg = fdk_config(nu, nv, nproj, g);
        size_t roi[4] = {0, 0, nu, nv};
        std::map<std::string, std::string> par;
        par["ProjectionBufferSize"] = "16";
        par["SliceBlock"] = "32";
        par["SubVolume"] = "1 1";
        Module fdk(nullptr);
        fdk.Configure(cfg, par);
        fdk.SetROI(roi);
        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        std::map<std::string, std::string> params;
        params["angles"] = list_text(angles, nproj);
        params["weights"] = list_text(weights, nproj);
        fdk.Process(img, params);
        std::memcpy(vol, fdk.volume.GetDataPtr(), sizeof(float) * fdk.volume.Size());
        if (cbct_out) std::memcpy(cbct_out, fdk.cbct_volume.GetDataPtr(), sizeof(float) * fdk.cbct_volume.Size());
        delete[] fdk.proj_matrices;
    }
}
} // extern "C++"

// ImagingAlgorithms::MorphSpotClean::process on one image [nv][nu]
// (MorphSpotClean.cpp:41-83), configured like the python binding tests.
int ref_morphspotclean(float *img, size_t nu, size_t nv, int detect, int clean, int conn,
                       const float *th, const float *sigma, int edgesmooth, int maxarea,
                       int clamp, float minlevel, float maxlevel, int removeinfnan)
{
    return guarded([&] {
        ImagingAlgorithms::MorphSpotClean c;
        c.setCleanMethod(static_cast<ImagingAlgorithms::eMorphDetectionMethod>(detect),
                         static_cast<ImagingAlgorithms::eMorphCleanMethod>(clean));
        c.setConnectivity(static_cast<kipl::morphology::MorphConnect>(conn));
        c.setLimits(clamp != 0, minlevel, maxlevel, maxarea);
        c.cleanInfNan(removeinfnan != 0);
        if (edgesmooth > 0) c.setEdgeConditioning(edgesmooth);
        size_t d2[2] = {nu, nv};
        kipl::base::TImage<float, 2> im(d2);
        std::memcpy(im.GetDataPtr(), img, sizeof(float) * nu * nv);
        std::vector<float> t(th, th + 2), s(sigma, sigma + 2);
        c.process(im, t, s);
        std::memcpy(img, im.GetDataPtr(), sizeof(float) * nu * nv);
    });
}

// MorphSpotCleanModule::Configure + ProcessCore 3D (MorphSpotCleanModule.cpp:37-183)
// on projections [nproj][nv][nu]. Parameters use the module's text names.
int ref_morphspotclean_module(float *proj, size_t nu, size_t nv, size_t nproj, const char *connectivity,
                              const char *cleanmethod, const char *detectionmethod, const char *threshold,
                              const char *sigma, int edgesmooth, int maxarea, int removeinfnan, int clampdata,
                              float minlevel, float maxlevel, int threading)
{
    return guarded([&] {
        MorphSpotCleanModule mod(nullptr);
        ReconConfig cfg;
        std::map<std::string, std::string> par;
        par["connectivity"] = connectivity;
        par["cleanmethod"] = cleanmethod;
        par["detectionmethod"] = detectionmethod;
        par["threshold"] = threshold;
        par["sigma"] = sigma;
        par["edgesmooth"] = std::to_string(edgesmooth);
        par["maxarea"] = std::to_string(maxarea);
        par["removeinfnan"] = removeinfnan ? "true" : "false";
        par["clampdata"] = clampdata ? "true" : "false";
        char b[64];
        std::snprintf(b, sizeof(b), "%.9g", minlevel);
        par["minlevel"] = b;
        std::snprintf(b, sizeof(b), "%.9g", maxlevel);
        par["maxlevel"] = b;
        par["threading"] = threading ? "true" : "false";
        if (mod.Configure(cfg, par) != 0) throw std::runtime_error("MorphSpotCleanModule::Configure failed");
        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        std::map<std::string, std::string> coeff;
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * nu * nv * nproj);
    });
}

// ImagingAlgorithms::StripeFilter::process on one sinogram [ntheta][nu]
// (StripeFilter.cpp:83-135).
int ref_stripefilter(float *sino, size_t nu, size_t ntheta, const char *wname, int scale, float sigma, int op)
{
    return guarded([&] {
        // the size_t* constructor copies into an empty std::vector (StripeFilter.cpp:25) and
        // crashes; the std::vector<int> constructor (the python binding's) is used instead
        size_t d2[2] = {nu, ntheta};
        std::vector<int> vd = {static_cast<int>(nu), static_cast<int>(ntheta)};
        ImagingAlgorithms::StripeFilter f(vd, wname, scale, sigma);
        kipl::base::TImage<float, 2> im(d2);
        std::memcpy(im.GetDataPtr(), sino, sizeof(float) * nu * ntheta);
        f.process(im, static_cast<ImagingAlgorithms::eStripeFilterOperation>(op));
        std::memcpy(sino, im.GetDataPtr(), sizeof(float) * nu * ntheta);
    });
}

// StripeFilter damping window for one level (StripeFilter.cpp:183-213).
int ref_stripefilter_window(size_t nu, size_t ntheta, const char *wname, int scale, float sigma, int level,
                            float *out, size_t *n_out)
{
    return guarded([&] {
        std::vector<int> vd = {static_cast<int>(nu), static_cast<int>(ntheta)};
        ImagingAlgorithms::StripeFilter f(vd, wname, scale, sigma);
        std::vector<float> w = f.filterWindow(level);
        *n_out = w.size();
        if (out) std::copy(w.begin(), w.end(), out);
    });
}

// WaveletRingClean::ProcessSingle (WaveletRingClean.cpp:74-103) on projections [nproj][nv][nu]:
// every detector row's sinogram [nproj][nu] through StripeFilter::process. The module itself
// builds its StripeFilter with the size_t* constructor, which crashes (see above), so the
// loop is driven here with the working constructor.
int ref_waveletringclean(float *proj, size_t nu, size_t nv, size_t nproj, const char *wname, int decnum,
                         float sigma)
{
    return guarded([&] {
        std::vector<int> vd = {static_cast<int>(nu), static_cast<int>(nproj)};
        ImagingAlgorithms::StripeFilter f(vd, wname, decnum, sigma);
        size_t d2[2] = {nu, nproj};
        kipl::base::TImage<float, 2> sino(d2);
        for (size_t j = 0; j < nv; ++j) {
            for (size_t i = 0; i < nproj; ++i) std::memcpy(sino.GetLinePtr(i), proj + (i * nv + j) * nu, nu * sizeof(float));
            f.process(sino, ImagingAlgorithms::VerticalComponentFFT);
            for (size_t i = 0; i < nproj; ++i) std::memcpy(proj + (i * nv + j) * nu, sino.GetLinePtr(i), nu * sizeof(float));
        }
    });
}

// The wavelet kernel of kipl::wavelets::WaveletKernel<float> (wavelets.hpp:52-405): begin,
// end and the four filters (analysis H/G, synthesis H/G), size floats each.
int ref_wavelet_kernel(const char *wname, int *begin, int *end, float *th, float *tg, float *sh, float *sg)
{
    return guarded([&] {
        kipl::wavelets::WaveletKernel<float> k(wname);
        *begin = k.begin();
        *end = k.end();
        for (int i = 0; i < k.size(); ++i) {
            th[i] = k.transH()[i];
            tg[i] = k.transG()[i];
            sh[i] = k.synthH()[i];
            sg[i] = k.synthG()[i];
        }
    });
}

// LinearForwardProjector::project 2-D (linearforwardprojector.cpp:15-144): slice [n][n]
// (x fastest), angles in degrees; proj [nangles][n] (detector bin fastest).
int ref_joseph_project(const float *slice, size_t n, const float *angles, size_t nangles, float *proj)
{
    return guarded([&] {
        size_t d[2] = {n, n};
        kipl::base::TImage<float, 2> img(d);
        std::memcpy(img.GetDataPtr(), slice, n * n * sizeof(float));
        std::list<float> a(angles, angles + nangles);
        kipl::base::TImage<float, 2> out;
        LinearForwardProjector fp;
        fp.project(img, a, out);
        std::memcpy(proj, out.GetDataPtr(), n * nangles * sizeof(float));
    });
}

// The uint16 slices ReconEngine::Serialize writes as TIFF16 (ReconEngine.cpp:576-700 ->
// kipl::io::WriteImageStack, io_stack.h:114-230): kipl's own ExtractSlice and the
// ImageCaster<unsigned short, float> cast that WriteTIFF(src, fname, lo, hi) applies
// (io_tiff.h:181-200), without the file. plane: kipl::base::eImagePlanes value (1 XY, 4 YZ).
int ref_slices_u16(const float *vol, size_t d0, size_t d1, size_t d2, int plane, size_t first, size_t count,
                   const size_t *roi, float lo, float hi, unsigned short *out)
{
    return guarded([&] {
        size_t d[3] = {d0, d1, d2};
        kipl::base::TImage<float, 3> img(d);
        std::memcpy(img.GetDataPtr(), vol, d0 * d1 * d2 * sizeof(float));
        size_t o = 0;
        for (size_t i = first; i < first + count; ++i) {
            size_t r[4];
            if (roi) std::memcpy(r, roi, sizeof(r));
            kipl::base::TImage<float, 2> sl =
                kipl::base::ExtractSlice(img, i, static_cast<kipl::base::eImagePlanes>(plane), roi ? r : nullptr);
            kipl::base::TImage<unsigned short, 2> u = kipl::base::ImageCaster<unsigned short, float, 2>::cast(sl, lo, hi);
            std::memcpy(out + o, u.GetDataPtr(), u.Size() * sizeof(unsigned short));
            o += u.Size();
        }
    });
}

// kipl::filters::TMedianFilter<float,2> (core/kipl/kipl/include/filters/core/medianfilter.hpp)
// on one image [h][w].
int ref_median_filter(const float *img, size_t w, size_t h, int kx, int ky, float *out)
{
    return guarded([&] {
        size_t d[2] = {w, h}, k[2] = {static_cast<size_t>(kx), static_cast<size_t>(ky)};
        kipl::base::TImage<float, 2> src(d);
        std::memcpy(src.GetDataPtr(), img, w * h * sizeof(float));
        kipl::filters::TMedianFilter<float, 2> filt(k);
        kipl::base::TImage<float, 2> r = filt(src);
        std::memcpy(out, r.GetDataPtr(), w * h * sizeof(float));
    });
}

// BasicRingClean::ProcessCore (StdPreprocModules/src/BasicRingClean.cpp:50-95) on
// projections [n][h][w], in place.
int ref_basicringclean(float *proj, size_t w, size_t h, size_t n)
{
    return guarded([&] {
        BasicRingClean mod;
        ReconConfig cfg;
        std::map<std::string, std::string> par;
        mod.Configure(cfg, par);
        size_t d3[3] = {w, h, n};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * w * h * n);
        std::map<std::string, std::string> coeff;
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * w * h * n);
    });
}

// kipl::math::SigmoidLUT (core/kipl/kipl/src/math/LUTCollection.cpp:38-82): the table and
// LUTbase's lo, hi, slope, intercept.
int ref_sigmoid_lut(size_t len, float lambda, float sigma, float *lut, float *param)
{
    return guarded([&] {
        kipl::math::SigmoidLUT t(len, lambda, sigma);
        std::memcpy(lut, t.fLUT, len * sizeof(float));
        param[0] = t.Low();
        param[1] = t.High();
        param[2] = t.Slope();
        param[3] = t.Intercept();
    });
}

// MedianMixRingClean::ProcessCore (StdPreprocModules/src/MedianMixRingClean.cpp:57-138) on
// projections [n][h][w], in place.
int ref_medianmixringclean(float *proj, size_t w, size_t h, size_t n, float threshold, float width)
{
    return guarded([&] {
        MedianMixRingClean mod;
        ReconConfig cfg;
        std::map<std::string, std::string> par;
        char b[64];
        std::snprintf(b, sizeof(b), "%.9g", threshold);
        par["threshold"] = b;
        std::snprintf(b, sizeof(b), "%.9g", width);
        par["width"] = b;
        mod.Configure(cfg, par);
        size_t d3[3] = {w, h, n};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * w * h * n);
        std::map<std::string, std::string> coeff;
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * w * h * n);
    });
}

// GammaSpotCleanModule::ProcessCore (StdPreprocModules/src/GammaSpotCleanModule.cpp:58-68)
// on projections [n][h][w], in place, with its parameters.
int ref_gammaspotclean(float *proj, size_t w, size_t h, size_t n, float threshold3, float threshold5,
                       float threshold7, float sigma, int mediansize)
{
    return guarded([&] {
        GammaSpotCleanModule mod;
        ReconConfig cfg;
        std::map<std::string, std::string> par;
        char b[64];
        std::snprintf(b, sizeof(b), "%.9g", threshold3);
        par["threshold3"] = b;
        std::snprintf(b, sizeof(b), "%.9g", threshold5);
        par["threshold5"] = b;
        std::snprintf(b, sizeof(b), "%.9g", threshold7);
        par["threshold7"] = b;
        std::snprintf(b, sizeof(b), "%.9g", sigma);
        par["sigma"] = b;
        par["mediansize"] = std::to_string(mediansize);
        mod.Configure(cfg, par);
        size_t d3[3] = {w, h, n};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * w * h * n);
        std::map<std::string, std::string> coeff;
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * w * h * n);
    });
}

// SpotClean2::ProcessCore 3D (StdPreprocModules/src/SpotClean2.cpp:117-130 ->
// ImagingAlgorithms::SpotClean::Process, SpotClean.cpp:78-108) on projections [n][h][w], in
// place. method: the reference's detection method names.
int ref_spotclean2(float *proj, size_t w, size_t h, size_t n, const char *method, float gamma, float sigma,
                   int iterations, float minlevel, float maxlevel, int maxarea)
{
    return guarded([&] {
        SpotClean2 mod;
        ReconConfig cfg;
        std::map<std::string, std::string> par;
        char b[64];
        std::snprintf(b, sizeof(b), "%.9g", gamma);
        par["gamma"] = b;
        std::snprintf(b, sizeof(b), "%.9g", sigma);
        par["sigma"] = b;
        par["iterations"] = std::to_string(iterations);
        std::snprintf(b, sizeof(b), "%.9g", maxlevel);
        par["maxlevel"] = b;
        std::snprintf(b, sizeof(b), "%.9g", minlevel);
        par["minlevel"] = b;
        par["maxarea"] = std::to_string(maxarea);
        par["detectionmethod"] = method;
        mod.Configure(cfg, par);
        size_t d3[3] = {w, h, n};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * w * h * n);
        std::map<std::string, std::string> coeff;
        mod.Process(img, coeff);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * w * h * n);
    });
}

// ComputeWeights (ReconFramework/src/ReconHelpers.cpp:365-488) on the multimap BuildFileList
// makes (:100-110: key = fmod(angle, 180), ProjectionInfo(name, angle)); the resulting map is
// copied out in its order as (info.angle, info.weight).
int ref_compute_weights(const float *angles, size_t n, float arc0, float arc1, int golden, float *out_angles,
                        float *out_weights, size_t *nout)
{
    return guarded([&] {
        ReconConfig cfg;
        cfg.ProjectionInfo.fScanArc[0] = arc0;
        cfg.ProjectionInfo.fScanArc[1] = arc1;
        cfg.ProjectionInfo.scantype = golden ? ReconConfig::cProjections::GoldenSectionScan
                                             : ReconConfig::cProjections::SequentialScan;
        std::multimap<float, ProjectionInfo> mm;
        for (size_t i = 0; i < n; ++i)
            mm.insert(std::make_pair(std::fmod(angles[i], 180.0f), ProjectionInfo("p", angles[i])));
        std::map<float, ProjectionInfo> out;
        ComputeWeights(&cfg, mm, &out);
        size_t m = 0;
        for (auto &kv : out) {
            out_angles[m] = kv.second.angle;
            out_weights[m] = kv.second.weight;
            ++m;
        }
        *nout = m;
    });
}

// A float written to a std::ostringstream with its default format (how ProjectionReader::Read
// writes the angle and weight lists, ProjectionReader.cpp:918-919); out receives the text.
void ref_stream_float(float v, char *out, size_t len)
{
    std::ostringstream s;
    s << v;
    std::snprintf(out, len, "%s", s.str().c_str());
}

// ---------------------------------------------------------------------------------------
// Module libraries loaded the way ReconEngine loads them: ModuleItem / BackProjItem
// (frameworks/tomography/Framework/ReconFramework/src/ModuleItem.cpp, ModuleItemBase.cpp:
// 97-131) open the library with dlopen and take GetModule / Destroy with dlsym; the module
// then gets Configure, SetROI and Process from the reference's own framework code. A module
// library resolves the framework's symbols from the process, so this library's symbols are
// made global first (it was opened RTLD_LOCAL by the caller).

static void make_self_global()
{
    static bool done = false;
    if (done) return;
    Dl_info info;
    if (dladdr(reinterpret_cast<void *>(&make_self_global), &info) && info.dli_fname)
        dlopen(info.dli_fname, RTLD_NOW | RTLD_NOLOAD | RTLD_GLOBAL);
    done = true;
}

static std::map<std::string, std::string> parse_params(const char *text)
{
    std::map<std::string, std::string> m;
    std::istringstream s(text ? text : "");
    std::string line;
    while (std::getline(s, line)) {
        const size_t eq = line.find('=');
        if (eq != std::string::npos) m[line.substr(0, eq)] = line.substr(eq + 1);
    }
    return m;
}

static std::string params_text(const std::map<std::string, std::string> &m)
{
    std::string t;
    for (const auto &kv : m) t += kv.first + "=" + kv.second + "\n";
    return t;
}

// The reference's own preprocessing module of that name (the module library's factory is not
// part of this build, so the classes are constructed here).
static PreprocModuleBase *reference_preproc(const std::string &name)
{
    if (name == "FullLogNorm") return new FullLogNorm;
    if (name == "MorphSpotClean") return new MorphSpotCleanModule(nullptr);
    if (name == "WaveletRingClean") return new WaveletRingClean(nullptr);
    if (name == "ProjectionFilterSingle") return new ProjectionFilterSingle(nullptr);
    throw std::runtime_error("no reference module " + name);
}

static BackProjectorModuleBase *reference_bp(const std::string &name)
{
    if (name == "MultiProjBPparallel") return new MultiProjectionBPparallel(nullptr);
    if (name == "MultiProjBP") return new MultiProjectionBP(nullptr);
    if (name == "NearestNeighborBP") return new NearestNeighborBP(nullptr);
    if (name == "FDKbp_single") return new FDKbp_single(nullptr);
    throw std::runtime_error("no reference backprojector " + name);
}

// GetModuleList of a module library (application tag `app`) as "module|key=value" lines.
int ref_plugin_module_list(const char *sofile, const char *app, char *out, size_t len)
{
    return guarded([&] {
        make_self_global();
        void *h = dlopen(sofile, RTLD_NOW);
        if (!h) throw std::runtime_error(std::string("dlopen: ") + dlerror());
        typedef int (*list_fn)(const char *, void *);
        list_fn f = reinterpret_cast<list_fn>(dlsym(h, "GetModuleList"));
        if (!f) throw std::runtime_error("GetModuleList not exported");
        std::map<std::string, std::map<std::string, std::string>> modules;
        const int rc = f(app, &modules);
        std::string t = "rc=" + std::to_string(rc) + "\n";
        for (const auto &m : modules)
            for (const auto &kv : m.second) t += m.first + "|" + kv.first + "=" + kv.second + "\n";
        std::snprintf(out, len, "%s", t.c_str());
    });
}

// GetModule of a module library for (app, name): 1 when it returns a module (destroyed again
// through the library's Destroy), 0 for nullptr.
int ref_plugin_has_module(const char *sofile, const char *app, const char *name, int *found)
{
    return guarded([&] {
        make_self_global();
        void *h = dlopen(sofile, RTLD_NOW);
        if (!h) throw std::runtime_error(std::string("dlopen: ") + dlerror());
        typedef void *(*get_fn)(const char *, const char *, void *);
        typedef int (*destroy_fn)(const char *, void *);
        get_fn g = reinterpret_cast<get_fn>(dlsym(h, "GetModule"));
        destroy_fn d = reinterpret_cast<destroy_fn>(dlsym(h, "Destroy"));
        if (!g || !d) throw std::runtime_error("GetModule / Destroy not exported");
        void *m = g(app, name, nullptr);
        *found = m != nullptr;
        if (m && d(app, m) != 0) throw std::runtime_error("Destroy failed");
    });
}

// GetParameters of the reference's own module of that name ("module|key=value" lines).
int ref_module_parameters(const char *name, int backprojector, char *out, size_t len)
{
    return guarded([&] {
        std::map<std::string, std::string> p;
        if (backprojector) {
            std::unique_ptr<BackProjectorModuleBase> m(reference_bp(name));
            p = m->GetParameters();
        } else {
            std::unique_ptr<PreprocModuleBase> m(reference_preproc(name));
            p = m->GetParameters();
        }
        std::string t;
        for (const auto &kv : p) t += std::string(name) + "|" + kv.first + "=" + kv.second + "\n";
        std::snprintf(out, len, "%s", t.c_str());
    });
}

// Writes an image [nv][nu] as a MATLAB file through kipl (the format ProjectionReader reads
// without the image libraries this build lacks).
int ref_write_mat(const float *img, size_t nu, size_t nv, const char *fname)
{
    return guarded([&] {
        size_t d2[2] = {nu, nv};
        kipl::base::TImage<float, 2> im(d2);
        std::memcpy(im.GetDataPtr(), img, sizeof(float) * nu * nv);
        kipl::io::WriteMAT(im, fname, "img");
    });
}

// Configure (+ SetROI when roi is given) + Process 3D of a preprocessing module on proj [nproj][nv][nu]
// in place: the reference's own module (sofile NULL) or module `name` of library `sofile`
// through ModuleItem. params/coeff: "key=value" lines. The ReconConfig fields FullLogNorm reads
// for its reference images: reference path, open beam / dark masks, counts, first indices,
// dose ROI.
int ref_preproc_module(const char *sofile, const char *name, const char *params, const char *coeff,
                       const char *refpath, const char *obmask, size_t nob, size_t obfirst, const char *dcmask,
                       size_t ndc, size_t dcfirst, const size_t *dose_roi, const size_t *roi, float *proj, size_t nu,
                       size_t nv, size_t nproj)
{
    return guarded([&] {
        make_self_global();
        ReconConfig cfg;
        cfg.ProjectionInfo.sReferencePath = refpath ? refpath : "";
        cfg.ProjectionInfo.sOBFileMask = obmask ? obmask : "";
        cfg.ProjectionInfo.nOBCount = nob;
        cfg.ProjectionInfo.nOBFirstIndex = obfirst;
        cfg.ProjectionInfo.sDCFileMask = dcmask ? dcmask : "";
        cfg.ProjectionInfo.nDCCount = ndc;
        cfg.ProjectionInfo.nDCFirstIndex = dcfirst;
        cfg.ProjectionInfo.imagetype = ReconConfig::cProjections::ImageType_Projections;
        cfg.ProjectionInfo.nDims[0] = nu;
        cfg.ProjectionInfo.nDims[1] = nv;
        size_t full[4] = {0, 0, nu, nv};
        std::memcpy(cfg.ProjectionInfo.dose_roi, dose_roi ? dose_roi : full, 4 * sizeof(size_t));
        std::memcpy(cfg.ProjectionInfo.roi, roi ? roi : full, 4 * sizeof(size_t));
        std::memcpy(cfg.ProjectionInfo.projection_roi, roi ? roi : full, 4 * sizeof(size_t));
        std::unique_ptr<ModuleItem> item;
        std::unique_ptr<PreprocModuleBase> own;
        PreprocModuleBase *m = nullptr;
        if (sofile && *sofile) {
            item.reset(new ModuleItem("muhrec", sofile, name));
            m = item->GetModule();
        } else {
            own.reset(reference_preproc(name));
            m = own.get();
        }
        if (m->Configure(cfg, parse_params(params)) != 0) throw std::runtime_error("Configure failed");
        if (roi) {
            size_t r[4] = {roi[0], roi[1], roi[2], roi[3]};
            m->SetROI(r);
        }
        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        std::map<std::string, std::string> c = parse_params(coeff);
        m->Process(img, c);
        std::memcpy(proj, img.GetDataPtr(), sizeof(float) * nu * nv * nproj);
    });
}

struct ref_bp_cfg {
    float center;
    int direction;
    int correcttilt;
    float tiltangle, tiltpivot;
    int cone;
    float sod, sdd, ppoint[2], resolution[2], voxelsize[3];
    int use_matrix_roi;
    size_t matrix_roi[4];
};

// Configure + SetROI(roi) + Process 3D of a backprojector (the reference's own, sofile NULL, or
// module `name` of library `sofile` through BackProjItem), then the framework's GetVolume
// (vol: the module's volume in kipl order) and GetSlice of every slice (slices: nslices
// slices of w x h, the sizes written to slice_dims). proj [nproj][nv][nu], roi (x0, y0, x1, y1).
int ref_bp_module(const char *sofile, const char *name, const char *params, const ref_bp_cfg *c, const size_t *roi,
                  const float *proj, size_t nproj, const float *angles, const float *weights, float *vol,
                  float *slices, size_t *slice_dims)
{
    return guarded([&] {
        make_self_global();
        const size_t nu = roi[2] - roi[0], nv = roi[3] - roi[1];
        ReconConfig cfg;
        cfg.ProjectionInfo.fCenter = c->center;
        cfg.ProjectionInfo.eDirection = static_cast<kipl::base::eRotationDirection>(c->direction);
        cfg.ProjectionInfo.bCorrectTilt = c->correcttilt != 0;
        cfg.ProjectionInfo.fTiltAngle = c->tiltangle;
        cfg.ProjectionInfo.fTiltPivotPosition = c->tiltpivot;
        cfg.ProjectionInfo.imagetype = ReconConfig::cProjections::ImageType_Projections;
        cfg.ProjectionInfo.beamgeometry = c->cone ? ReconConfig::cProjections::BeamGeometry_Cone
                                                  : ReconConfig::cProjections::BeamGeometry_Parallel;
        cfg.ProjectionInfo.nDims[0] = nu;
        cfg.ProjectionInfo.nDims[1] = nv;
        cfg.ProjectionInfo.fSOD = c->sod;
        cfg.ProjectionInfo.fSDD = c->sdd;
        cfg.ProjectionInfo.fpPoint[0] = c->ppoint[0];
        cfg.ProjectionInfo.fpPoint[1] = c->ppoint[1];
        cfg.ProjectionInfo.fResolution[0] = c->resolution[0];
        cfg.ProjectionInfo.fResolution[1] = c->resolution[1];
        cfg.ProjectionInfo.nFirstIndex = 0;
        cfg.ProjectionInfo.nLastIndex = nproj - 1;
        cfg.ProjectionInfo.nProjectionStep = 1;
        std::memcpy(cfg.ProjectionInfo.roi, roi, 4 * sizeof(size_t));
        std::memcpy(cfg.ProjectionInfo.projection_roi, roi, 4 * sizeof(size_t));
        cfg.MatrixInfo.fVoxelSize[0] = c->voxelsize[0];
        cfg.MatrixInfo.fVoxelSize[1] = c->voxelsize[1];
        cfg.MatrixInfo.fVoxelSize[2] = c->voxelsize[2];
        cfg.MatrixInfo.nDims[0] = nu;
        cfg.MatrixInfo.nDims[1] = nu;
        cfg.MatrixInfo.nDims[2] = nv;
        cfg.MatrixInfo.bUseROI = c->use_matrix_roi != 0;
        std::memcpy(cfg.MatrixInfo.roi, c->matrix_roi, 4 * sizeof(size_t));
        std::unique_ptr<BackProjItem> item;
        std::unique_ptr<BackProjectorModuleBase> own;
        BackProjectorModuleBase *m = nullptr;
        if (sofile && *sofile) {
            item.reset(new BackProjItem("muhrecbp", sofile, name));
            m = item->GetModule();
        } else {
            own.reset(reference_bp(name));
            m = own.get();
        }
        m->Configure(cfg, parse_params(params));
        size_t r[4] = {roi[0], roi[1], roi[2], roi[3]};
        m->SetROI(r);
        size_t d3[3] = {nu, nv, nproj};
        kipl::base::TImage<float, 3> img(d3);
        std::memcpy(img.GetDataPtr(), proj, sizeof(float) * nu * nv * nproj);
        std::map<std::string, std::string> p;
        p["angles"] = list_text(angles, nproj);
        p["weights"] = list_text(weights, nproj);
        m->Process(img, p);
        kipl::base::TImage<float, 3> v = m->GetVolume();
        std::memcpy(vol, v.GetDataPtr(), sizeof(float) * v.Size());
        const size_t ns = m->GetNSlices();
        for (size_t i = 0; i < ns; ++i) {
            kipl::base::TImage<float, 2> s = m->GetSlice(i);
            slice_dims[0] = s.Size(0);
            slice_dims[1] = s.Size(1);
            std::memcpy(slices + i * s.Size(), s.GetDataPtr(), sizeof(float) * s.Size());
        }
        slice_dims[2] = ns;
        if (FDKbp_single *f = dynamic_cast<FDKbp_single *>(m)) delete[] f->proj_matrices;
    });
}

// libtiff writers for the debug images BasicRingClean saves to the working directory
// (mean.tif, med.tif, diff.tif; libtiff is absent here): opening for writing gives a handle
// that discards everything, so the module runs to the end without touching the file system.
// Opening for reading still fails.
static char g_tiff_sink;
TIFF *TIFFOpen(const char *, const char *mode)
{
    return mode && mode[0] == 'w' ? reinterpret_cast<TIFF *>(&g_tiff_sink) : nullptr;
}
int TIFFSetField(TIFF *, ttag_t, ...) { return 1; }
int TIFFWriteDirectory(TIFF *) { return 1; }
tsize_t TIFFWriteEncodedStrip(TIFF *, tstrip_t, tdata_t, tsize_t cc) { return cc; }
void TIFFClose(TIFF *) {}

} // extern "C"
