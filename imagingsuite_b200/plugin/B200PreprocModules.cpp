// MuhRec preprocessing modules on the B200 kernels: the classes of B200PreprocModules.h and
// the module library's factory functions (GetModule, Destroy, LibVersion, GetModuleList,
// resolved by ModuleItem with dlsym, core/modules/ModuleConfig/src/ModuleItemBase.cpp:97-131).
#include "B200PreprocModules.h"

#include <cmath>
#include <cstring>
#include <iostream>
#include <sstream>

#include <ModuleException.h>
#include <ParameterHandling.h>
#include <ProjectionReader.h>
#include <base/KiplException.h>
#include <strings/filenames.h>
#include <strings/miscstring.h>
#include <strings/string2array.h>

using b200::check;

namespace {

const char *kApplication = "muhrec";

} // namespace

// ============================================================== FullLogNormCUDA

FullLogNormCUDA::FullLogNormCUDA(kipl::interactors::InteractionBase *interactor)
    : PreprocModuleBase("FullLogNorm", interactor)
{
}

FullLogNormCUDA::~FullLogNormCUDA() = default;

// NormBase::Configure + FullLogNorm::Configure (NormPlugins.cpp:57-83,254-258)
int FullLogNormCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    m_Config = config;
    path = config.ProjectionInfo.sReferencePath;
    flatname = config.ProjectionInfo.sOBFileMask;
    darkname = config.ProjectionInfo.sDCFileMask;
    nOBCount = static_cast<int>(config.ProjectionInfo.nOBCount);
    nOBFirstIndex = static_cast<int>(config.ProjectionInfo.nOBFirstIndex);
    nDCCount = static_cast<int>(config.ProjectionInfo.nDCCount);
    nDCFirstIndex = static_cast<int>(config.ProjectionInfo.nDCFirstIndex);
    bUseNormROI = kipl::strings::string2bool(GetStringParameter(parameters, "usenormregion"));
    try {
        bUseLUT = kipl::strings::string2bool(GetStringParameter(parameters, "uselut"));
    } catch (...) {
        logger(logger.LogWarning, "Parameter uselut missing, using uselut=false");
        bUseLUT = false;
    }
    string2enum(GetStringParameter(parameters, "referenceaverage"), m_ReferenceAverage);
    std::memcpy(nOriginalNormRegion, config.ProjectionInfo.dose_roi, 4 * sizeof(size_t));
    return 0;
}

std::map<std::string, std::string> FullLogNormCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["usenormregion"] = kipl::strings::bool2string(bUseNormROI);
    parameters["uselut"] = kipl::strings::bool2string(bUseLUT);
    parameters["referenceaverage"] = enum2string(m_ReferenceAverage);
    return parameters;
}

// NormBase::SetROI (NormPlugins.cpp:41-54)
bool FullLogNormCUDA::SetROI(size_t *roi)
{
    std::ostringstream msg;
    msg << "ROI=[" << roi[0] << " " << roi[1] << " " << roi[2] << " " << roi[3] << "]";
    logger(kipl::logging::Logger::LogMessage, msg.str());
    LoadReferenceImages(roi);
    return true;
}

// NormBase::ReferenceLoader (NormPlugins.cpp:85-225): the frames are read by the framework's
// ProjectionReader and averaged on the device (mr_reference_average, the AverageImage
// methods in the enum's order).
kipl::base::TImage<float, 2> FullLogNormCUDA::ReferenceLoader(const std::string &fname, int firstIndex, int N,
                                                              size_t *roi, float initialDose, float doseBias,
                                                              float &dose)
{
    kipl::base::TImage<float, 2> img, refimg;
    if (fname.empty() && N != 0) throw ReconException("The reference image file name mask is empty", __FILE__, __LINE__);
    dose = initialDose;
    if (N == 0) {
        logger(kipl::logging::Logger::LogWarning, "Reference image count is zero");
        return refimg;
    }
    ProjectionReader reader;
    const bool nexus = fname.find("hdf") != std::string::npos;
    auto read = [&](int index, float &frame_dose) {
        std::string filename, ext;
        const ReconConfig::cProjections &pi = m_Config.ProjectionInfo;
        if (!nexus) {
            kipl::strings::filenames::MakeFileName(fname, index, filename, ext, '#', '0');
            img = reader.Read(filename, pi.eFlip, pi.eRotate, pi.fBinning, roi);
            frame_dose = bUseNormROI ? reader.GetProjectionDose(filename, pi.eFlip, pi.eRotate, pi.fBinning,
                                                                nOriginalNormRegion)
                                     : initialDose;
        } else {
            img = reader.ReadNexus(fname, index, pi.eFlip, pi.eRotate, pi.fBinning, roi);
            frame_dose = bUseNormROI ? reader.GetProjectionDoseNexus(fname, index, pi.eFlip, pi.eRotate, pi.fBinning,
                                                                     nOriginalNormRegion)
                                     : initialDose;
        }
    };
    float tmpdose = 0.0f;
    read(firstIndex, tmpdose);
    tmpdose = tmpdose - doseBias;
    dose = tmpdose;
    const size_t nu = img.Size(0), nv = img.Size(1), npix = img.Size();
    std::vector<float> stack(npix * static_cast<size_t>(N));
    std::memcpy(stack.data(), img.GetDataPtr(), npix * sizeof(float));
    for (int i = 1; i < N; ++i) {
        read(i + firstIndex, tmpdose);
        if (img.Size() != npix) throw ReconException("Reference images of different sizes", __FILE__, __LINE__);
        std::memcpy(stack.data() + static_cast<size_t>(i) * npix, img.GetDataPtr(), npix * sizeof(float));
        tmpdose = tmpdose - doseBias;
        dose += tmpdose;
    }
    dose /= static_cast<float>(N);
    cudaStream_t s = stream.get();
    float *frames = d_stack.get(stack.size());
    float *avg = d_img.get(npix);
    b200::upload(frames, stack.data(), stack.size(), s);
    check(mr_reference_average(frames, nu, nv, static_cast<size_t>(N), static_cast<int>(m_ReferenceAverage), avg, s),
          "FullLogNorm reference average");
    size_t dims[2] = {nu, nv};
    refimg.Resize(dims);
    b200::download(refimg.GetDataPtr(), avg, npix, s);
    stream.sync();
    if (m_Config.ProjectionInfo.imagetype == ReconConfig::cProjections::ImageType_Proj_RepeatSinogram)
        for (size_t i = 1; i < refimg.Size(1); ++i)
            std::memcpy(refimg.GetLinePtr(i), refimg.GetLinePtr(0), sizeof(float) * refimg.Size(0));
    std::ostringstream msg;
    msg << "Loaded reference image (dose=" << dose << ")";
    logger(logger.LogMessage, msg.str());
    return refimg;
}

// FullLogNorm::LoadReferenceImages (NormPlugins.cpp:260-298)
void FullLogNormCUDA::LoadReferenceImages(size_t *roi)
{
    if (flatname.empty() && nOBCount != 0) throw ReconException("The flat field image mask is empty", __FILE__, __LINE__);
    if (darkname.empty() && nDCCount != 0) throw ReconException("The dark current image mask is empty", __FILE__, __LINE__);
    const std::string flatmask = path + flatname, darkmask = path + darkname;
    kipl::base::TImage<float, 2> dark, flat;
    fDarkDose = 0.0f;
    fFlatDose = 1.0f;
    if (nDCCount != 0)
        dark = ReferenceLoader(darkmask, static_cast<int>(m_Config.ProjectionInfo.nDCFirstIndex),
                               static_cast<int>(m_Config.ProjectionInfo.nDCCount), roi, 0.0f, 0.0f, fDarkDose);
    if (nOBCount != 0)
        flat = ReferenceLoader(flatmask, static_cast<int>(m_Config.ProjectionInfo.nOBFirstIndex),
                               static_cast<int>(m_Config.ProjectionInfo.nOBCount), roi, 1.0f, fDarkDose, fFlatDose);
    SetReferenceImages(dark, flat);
}

// NormBase::SetReferenceImages + FullLogNorm::SetReferenceImages (NormPlugins.cpp:77-81,
// 300-341): the dark and log(flat * 1/flatdose) on the device.
void FullLogNormCUDA::SetReferenceImages(kipl::base::TImage<float, 2> dark, kipl::base::TImage<float, 2> flat)
{
    const float dose = 1.0f / fFlatDose;
    if (dose != dose) throw ReconException("The reference dose is a NaN", __FILE__, __LINE__);
    if (std::isinf(dose)) throw ReconException("The reference dose is Inf", __FILE__, __LINE__);
    cudaStream_t s = stream.get();
    nDarkPix = dark.Size();
    nFlatPix = flat.Size();
    if (nDarkPix) b200::upload(d_dark.get(nDarkPix), dark.GetDataPtr(), nDarkPix, s);
    if (nFlatPix) {
        float *f = d_img.get(nFlatPix);
        b200::upload(f, flat.GetDataPtr(), nFlatPix, s);
        const bool ndc = nDCCount != 0;
        if (ndc && nDarkPix != nFlatPix)
            throw ReconException("The dark and flat field images differ in size", __FILE__, __LINE__);
        check(mr_lognorm_logflat(ndc ? d_dark.data() : f, f, nFlatPix, ndc, fFlatDose, d_logflat.get(nFlatPix), s),
              "FullLogNorm log flat");
        if (m_Config.ProjectionInfo.imagetype == ReconConfig::cProjections::ImageType_Proj_RepeatSinogram)
            for (size_t i = 1; i < flat.Size(1); ++i)
                b200::cuda_check(cudaMemcpyAsync(d_logflat.data() + i * flat.Size(0), d_logflat.data(),
                                                 sizeof(float) * flat.Size(0), cudaMemcpyDeviceToDevice, s),
                                 "device copy");
    }
    stream.sync();
}

// FullLogNorm::ProcessCore 2D (NormPlugins.cpp:343-409): one projection, dose from coeff.
int FullLogNormCUDA::ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("FullLogNormCUDA::ProcessCore");
    float dose = 1.0f;
    if (bUseNormROI) {
        dose = GetFloatParameter(coeff, "dose") - fDarkDose;
        dose = dose <= 0.0f ? 1.0f : dose;
    }
    if (dose != dose) throw ReconException("The projection dose is a NaN", __FILE__, __LINE__);
    const float logdose = std::log(dose);
    const size_t N = img.Size();
    if (nFlatPix != N) {
        std::ostringstream msg;
        msg << "Flat field does not match projection (" << img.Size(0) << ", " << img.Size(1) << ")(N flat=" << nFlatPix
            << ", N proj=" << N << ")";
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
    cudaStream_t s = stream.get();
    float *d = d_img.get(N);
    float *dl = d_doselog.get(1);
    b200::upload(d, img.GetDataPtr(), N, s);
    b200::upload(dl, &logdose, 1, s);
    const int ndc = nDCCount != 0;
    check((bUseLUT ? mr_lognorm_apply_lut : mr_lognorm_apply)(d, MR_F32, N, 1, ndc ? d_dark.data() : nullptr,
                                                             d_logflat.data(), dl, 1, ndc, 1, d, s),
          "FullLogNorm");
    b200::download(img.GetDataPtr(), d, N, s);
    stream.sync();
    return 0;
}

// FullLogNorm::ProcessCore 3D (NormPlugins.cpp:411-552)
int FullLogNormCUDA::ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("FullLogNormCUDA::ProcessCore");
    int nDose = static_cast<int>(img.Size(2));
    std::vector<float> doselist(std::max(nDose, 1));
    if (bUseNormROI) {
        GetFloatParameterVector(coeff, "dose", doselist.data(), nDose);
        check(mr_lognorm_doselog(doselist.data(), static_cast<size_t>(nDose), fDarkDose, doselist.data()),
              "FullLogNorm doses");
    } else {
        nDose = 1;
        doselist[0] = 0.0f;
    }
    const size_t N = img.Size(0) * img.Size(1), nproj = img.Size(2);
    if (nOBCount != 0 && nFlatPix != N) {
        std::ostringstream msg;
        msg << "Flat field does not match projection (" << img.Size(0) << ", " << img.Size(1) << ")(N flat=" << nFlatPix
            << ", N proj=" << img.Size() << ")";
        logger(logger.LogError, msg.str());
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
    if (nDCCount != 0 && nDarkPix != N) {
        std::ostringstream msg;
        msg << "Dark field does not match projection (" << img.Size(0) << ", " << img.Size(1) << ")(N flat=" << nDarkPix
            << ", N proj=" << img.Size() << ")";
        logger(logger.LogError, msg.str());
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
    cudaStream_t s = stream.get();
    float *d = d_img.get(img.Size());
    float *dl = d_doselog.get(static_cast<size_t>(nDose));
    b200::upload(d, img.GetDataPtr(), img.Size(), s);
    b200::upload(dl, doselist.data(), static_cast<size_t>(nDose), s);
    const int ndc = nDCCount != 0, nob = nOBCount != 0;
    // the kernels take at most 65535 projections per call
    for (size_t p0 = 0; p0 < nproj; p0 += 65535) {
        const size_t np = std::min<size_t>(65535, nproj - p0);
        float *blk = d + p0 * N;
        // a per-projection dose list is sliced with the block; without flats the LUT path
        // subtracts the first projection's dose of the whole list (doselog[0])
        const bool perproj = nDose != 1;
        if (bUseLUT && !nob && perproj && p0 > 0)
            throw ReconException("FullLogNorm: more than 65535 projections in one block", __FILE__, __LINE__);
        check((bUseLUT ? mr_lognorm_apply_lut : mr_lognorm_apply)(blk, MR_F32, N, np, ndc ? d_dark.data() : nullptr,
                                                                 nob ? d_logflat.data() : nullptr,
                                                                 perproj ? dl + p0 : dl, perproj ? np : 1, ndc, nob,
                                                                 blk, s),
              "FullLogNorm");
    }
    b200::download(img.GetDataPtr(), d, img.Size(), s);
    stream.sync();
    return 0;
}

// ============================================================== MorphSpotCleanCUDA

MorphSpotCleanCUDA::MorphSpotCleanCUDA(kipl::interactors::InteractionBase *interactor)
    : PreprocModuleBase("MorphSpotClean", interactor)
{
}

MorphSpotCleanCUDA::~MorphSpotCleanCUDA() = default;

// MorphSpotCleanModule::Configure (MorphSpotCleanModule.cpp:37-71)
int MorphSpotCleanCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    (void)config;
    std::ostringstream msg;
    try {
        string2enum(GetStringParameter(parameters, "connectivity"), m_eConnectivity);
        string2enum(GetStringParameter(parameters, "cleanmethod"), m_eCleanMethod);
        string2enum(GetStringParameter(parameters, "detectionmethod"), m_eDetectionMethod);
        kipl::strings::string2vector(GetStringParameter(parameters, "threshold"), m_fThreshold);
        kipl::strings::string2vector(GetStringParameter(parameters, "sigma"), m_fSigma);
        m_nEdgeSmoothLength = GetIntParameter(parameters, "edgesmooth");
        m_nMaxArea = GetIntParameter(parameters, "maxarea");
        m_bRemoveInfNaN = kipl::strings::string2bool(GetStringParameter(parameters, "removeinfnan"));
        m_bClampData = kipl::strings::string2bool(GetStringParameter(parameters, "clampdata"));
        m_fMinLevel = GetFloatParameter(parameters, "minlevel");
        m_fMaxLevel = GetFloatParameter(parameters, "maxlevel");
        m_bThreading = kipl::strings::string2bool(GetStringParameter(parameters, "threading"));
    } catch (ModuleException &e) {
        msg << "Module exception: Failed to get parameters: " << e.what();
        logger(kipl::logging::Logger::LogError, msg.str());
        return -1;
    } catch (kipl::base::KiplException &e) {
        msg << "Kipl Exception: Failed to get parameters: " << e.what();
        logger(kipl::logging::Logger::LogError, msg.str());
        return -1;
    } catch (std::exception &e) {
        msg << "STL exception: Failed to get parameters: " << e.what();
        logger(kipl::logging::Logger::LogError, msg.str());
        return -1;
    }
    return 0;
}

std::map<std::string, std::string> MorphSpotCleanCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["connectivity"] = enum2string(m_eConnectivity);
    parameters["cleanmethod"] = enum2string(m_eCleanMethod);
    parameters["detectionmethod"] = enum2string(m_eDetectionMethod);
    parameters["threshold"] = kipl::strings::Vector2String(m_fThreshold);
    parameters["sigma"] = kipl::strings::Vector2String(m_fSigma);
    parameters["edgesmooth"] = kipl::strings::value2string(m_nEdgeSmoothLength);
    parameters["maxarea"] = kipl::strings::value2string(m_nMaxArea);
    parameters["removeinfnan"] = kipl::strings::bool2string(m_bRemoveInfNaN);
    parameters["clampdata"] = kipl::strings::bool2string(m_bClampData);
    parameters["minlevel"] = kipl::strings::value2string(m_fMinLevel);
    parameters["maxlevel"] = kipl::strings::value2string(m_fMaxLevel);
    parameters["threading"] = kipl::strings::bool2string(m_bThreading);
    return parameters;
}

bool MorphSpotCleanCUDA::SetROI(size_t *roi)
{
    (void)roi;
    return false;
}

void MorphSpotCleanCUDA::clean(float *img_h, size_t nu, size_t nv, size_t n, bool clamp, bool removeinfnan)
{
    if (m_eCleanMethod != ImagingAlgorithms::MorphCleanReplace)
        // MorphSpotClean::ProcessFill assigns the padded, CleanByArray-filled image to its output
        // and the module copies that padded-size image into the projection stack
        // (MorphSpotClean.cpp:177-236, MorphSpotCleanModule.cpp:161-163): not reproduced
        throw ReconException("MorphSpotClean: only morphcleanreplace is supported by this module", __FILE__, __LINE__);
    if (m_fThreshold.size() < 2 || m_fSigma.size() < 2)
        throw ReconException("MorphSpotClean: threshold and sigma need two values", __FILE__, __LINE__);
    const size_t total = nu * nv * n;
    cudaStream_t s = stream.get();
    float *d = d_img.get(total);
    b200::upload(d, img_h, total, s);
    // the module's cleaners keep MorphSpotClean's own edge smoothing length (9)
    check(mr_morphspotclean(d, nu, nv, n, static_cast<int>(m_eDetectionMethod),
                            m_eConnectivity == kipl::morphology::conn8, m_fThreshold.data(), m_fSigma.data(), 9,
                            clamp, m_fMinLevel, m_fMaxLevel, removeinfnan, s),
          "MorphSpotClean");
    b200::download(img_h, d, total, s);
    stream.sync();
    b200::check_device("MorphSpotClean");
}

// MorphSpotCleanModule::ProcessCore 3D (MorphSpotCleanModule.cpp:99-109): the single-threaded
// path sets the cleaner's limits (clamping) and no inf/NaN removal; the threaded path
// (ProcessParallelStd, :226-269) sets neither.
int MorphSpotCleanCUDA::ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("MorphSpotCleanCUDA::ProcessCore");
    (void)coeff;
    clean(img.GetDataPtr(), img.Size(0), img.Size(1), img.Size(2), m_bClampData && !m_bThreading, false);
    return 0;
}

// MorphSpotCleanModule::ProcessCore 2D (:112-148): limits and inf/NaN removal as configured
int MorphSpotCleanCUDA::ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("MorphSpotCleanCUDA::ProcessCore");
    (void)coeff;
    clean(img.GetDataPtr(), img.Size(0), img.Size(1), 1, m_bClampData, m_bRemoveInfNaN);
    return 0;
}

// ============================================================== WaveletRingCleanCUDA

WaveletRingCleanCUDA::WaveletRingCleanCUDA(kipl::interactors::InteractionBase *interactor)
    : PreprocModuleBase("WaveletRingClean", interactor)
{
}

WaveletRingCleanCUDA::~WaveletRingCleanCUDA() = default;

// WaveletRingClean::Configure (WaveletRingClean.cpp:34-43)
int WaveletRingCleanCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    (void)config;
    m_sWName = GetStringParameter(parameters, "wname");
    m_fSigma = GetFloatParameter(parameters, "sigma");
    m_nDecNum = GetIntParameter(parameters, "decnum");
    m_bParallelProcessing = kipl::strings::string2bool(GetStringParameter(parameters, "parallel"));
    string2enum(GetStringParameter(parameters, "method"), m_eCleanMethod);
    return 0;
}

std::map<std::string, std::string> WaveletRingCleanCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["wname"] = m_sWName;
    parameters["sigma"] = kipl::strings::value2string(m_fSigma);
    parameters["decnum"] = kipl::strings::value2string(m_nDecNum);
    parameters["parallel"] = m_bParallelProcessing ? "true" : "false";
    parameters["method"] = enum2string(m_eCleanMethod);
    return parameters;
}

bool WaveletRingCleanCUDA::SetROI(size_t *roi)
{
    (void)roi;
    return false;
}

// WaveletRingClean::ProcessSingle / ProcessParallel (:63-146): every detector row's sinogram
// through the stripe filter. `method` is read but, as in the reference, VerticalComponentFFT
// is always applied.
int WaveletRingCleanCUDA::ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("WaveletRingCleanCUDA::ProcessCore");
    (void)coeff;
    const size_t total = img.Size();
    cudaStream_t s = stream.get();
    float *d = d_img.get(total);
    b200::upload(d, img.GetDataPtr(), total, s);
    const mr_status st = mr_waveletringclean(d, img.Size(0), img.Size(1), img.Size(2), m_sWName.c_str(), m_nDecNum,
                                             m_fSigma, s);
    if (st != MR_OK) {
        std::ostringstream msg;
        msg << "Failed to process the projections using stripe filter. (" << mr_last_error() << ")";
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
    b200::download(img.GetDataPtr(), d, total, s);
    stream.sync();
    return 0;
}

// ============================================================== ProjectionFilterCUDA

ProjectionFilterCUDA::ProjectionFilterCUDA(kipl::interactors::InteractionBase *interactor)
    : PreprocModuleBase("ProjectionFilterSingle", interactor)
{
}

ProjectionFilterCUDA::~ProjectionFilterCUDA()
{
    if (plan) mr_projfilter_destroy(plan);
}

// The filter type names of ProjectionFilterBase's enum2string (ProjectionFilter.cpp:51-63)
static std::string canonical_filter_name(const std::string &s)
{
    const std::string l = kipl::strings::toLower(s);
    if (l == "ram-lak") return "Ram-Lak";
    if (l == "shepp-logan") return "Shepp-Logan";
    if (l == "hanning") return "Hanning";
    if (l == "hamming") return "Hamming";
    if (l == "butterworth") return "Butterworth";
    throw ReconException("Could not convert filter string to enum.", __FILE__, __LINE__);
}

// ProjectionFilterBase::Configure (ProjectionFilter.cpp:78-91), BuildFilter and
// PreparePadding through mr_projfilter_create
int ProjectionFilterCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    const size_t N = config.ProjectionInfo.roi[2] - config.ProjectionInfo.roi[0];
    m_FilterType = canonical_filter_name(GetStringParameter(parameters, "filtertype"));
    m_fCutOff = GetFloatParameter(parameters, "cutoff");
    m_fOrder = GetFloatParameter(parameters, "order");
    m_bUseBias = kipl::strings::string2bool(GetStringParameter(parameters, "usebias"));
    m_fBiasWeight = GetFloatParameter(parameters, "biasweight");
    m_nPaddingDoubler = GetIntParameter(parameters, "paddingdoubler");
    nImageSize = N;
    if (plan) mr_projfilter_destroy(plan);
    plan = nullptr;
    const mr_status st = mr_projfilter_create(N, m_FilterType.c_str(), m_fCutOff, m_fOrder, m_bUseBias, m_fBiasWeight,
                                              m_nPaddingDoubler, &plan);
    if (st != MR_OK) throw ReconException(mr_last_error(), __FILE__, __LINE__);
    return 0;
}

std::map<std::string, std::string> ProjectionFilterCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["filtertype"] = m_FilterType;
    parameters["cutoff"] = kipl::strings::value2string(m_fCutOff);
    parameters["order"] = kipl::strings::value2string(m_fOrder);
    parameters["usebias"] = m_bUseBias ? "true" : "false";
    parameters["biasweight"] = kipl::strings::value2string(m_fBiasWeight);
    parameters["paddingdoubler"] = kipl::strings::value2string(m_nPaddingDoubler);
    return parameters;
}

void ProjectionFilterCUDA::filter(float *img_h, size_t nu, size_t rows)
{
    if (!plan) throw ReconException("ProjectionFilter: the filter is not configured", __FILE__, __LINE__);
    if (nu != nImageSize) {
        std::ostringstream msg;
        msg << "ProjectionFilter: projection width " << nu << " differs from the configured ROI width " << nImageSize;
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
    cudaStream_t s = stream.get();
    float *d = d_img.get(nu * rows);
    b200::upload(d, img_h, nu * rows, s);
    check(mr_projfilter_apply(plan, d, d, rows, nullptr, 1, s), "ProjectionFilter");
    b200::download(img_h, d, nu * rows, s);
    stream.sync();
}

// ProjectionFilterBase::ProcessCore 2D/3D (ProjectionFilter.cpp:93-118)
int ProjectionFilterCUDA::ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("ProjectionFilterCUDA::ProcessCore");
    (void)coeff;
    if (img.Size() == 0) throw ReconException("Empty projection image", __FILE__, __LINE__);
    filter(img.GetDataPtr(), img.Size(0), img.Size(1));
    return 0;
}

int ProjectionFilterCUDA::ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff)
{
    b200::Trace trace("ProjectionFilterCUDA::ProcessCore");
    (void)coeff;
    if (img.Size() == 0) throw ReconException("Empty projection image", __FILE__, __LINE__);
    filter(img.GetDataPtr(), img.Size(0), img.Size(1) * img.Size(2));
    return 0;
}

// ============================================================== factory functions

// StdPreprocModules.cpp:40-118: the application tag must be "muhrec"
void *GetModule(const char *application, const char *name, void *vinteractor)
{
    if (!application || std::strcmp(application, kApplication) != 0) return nullptr;
    auto *interactor = reinterpret_cast<kipl::interactors::InteractionBase *>(vinteractor);
    if (!name) return nullptr;
    const std::string n = name;
    if (n == "FullLogNorm" || n == "FullLogNormCUDA") return static_cast<PreprocModuleBase *>(new FullLogNormCUDA(interactor));
    if (n == "MorphSpotClean" || n == "MorphSpotCleanCUDA")
        return static_cast<PreprocModuleBase *>(new MorphSpotCleanCUDA(interactor));
    if (n == "WaveletRingClean" || n == "WaveletRingCleanCUDA")
        return static_cast<PreprocModuleBase *>(new WaveletRingCleanCUDA(interactor));
    if (n == "ProjectionFilterSingle" || n == "ProjectionFilterCUDA")
        return static_cast<PreprocModuleBase *>(new ProjectionFilterCUDA(interactor));
    return nullptr;
}

// StdPreprocModules.cpp:120-163
int Destroy(const char *application, void *obj)
{
    if (!application || std::strcmp(application, kApplication) != 0) return -1;
    kipl::logging::Logger logger("B200PreprocModules::Destroy");
    std::string name = "No name";
    try {
        if (obj) {
            PreprocModuleBase *module = reinterpret_cast<PreprocModuleBase *>(obj);
            name = module->ModuleName();
            logger(kipl::logging::Logger::LogVerbose, "Destroying " + name);
            delete module;
        }
    } catch (std::exception &e) {
        logger(kipl::logging::Logger::LogError, "Failed to destroy " + name + " with STL exception" + e.what());
        return -1;
    } catch (kipl::base::KiplException &e) {
        logger(kipl::logging::Logger::LogError, "Failed to destroy " + name + " with KIPL exception" + e.what());
        return -1;
    }
    return 0;
}

int LibVersion()
{
    return mr_version();
}

// StdPreprocModules.cpp:170-247: the default parameters of every module of the library
int GetModuleList(const char *application, void *listptr)
{
    if (!application || std::strcmp(application, kApplication) != 0) return -1;
    auto *modulelist = reinterpret_cast<std::map<std::string, std::map<std::string, std::string>> *>(listptr);
    FullLogNormCUDA flnorm;
    (*modulelist)["FullLogNorm"] = flnorm.GetParameters();
    MorphSpotCleanCUDA mscm;
    (*modulelist)["MorphSpotClean"] = mscm.GetParameters();
    WaveletRingCleanCUDA wrc;
    (*modulelist)["WaveletRingClean"] = wrc.GetParameters();
    ProjectionFilterCUDA filter;
    (*modulelist)["ProjectionFilterSingle"] = filter.GetParameters();
    return 0;
}
