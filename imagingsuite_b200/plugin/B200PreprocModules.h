// MuhRec preprocessing modules on the B200 kernels (libB200PreprocModules.so, application
// tag "muhrec").
//
// Each class is a PreprocModuleBase with the reference module's parameter names, defaults,
// Configure/GetParameters/SetROI behaviour and ProcessCore on kipl::base::TImage<float,3>
// (frameworks/tomography/Framework/ReconFramework/include/PreprocModuleBase.h), so that a
// ReconEngine configuration selects it by library file and module name in place of the
// module of frameworks/tomography/Preprocessing/StdPreprocModules. ProcessCore copies the
// block to the device, runs libmrcuda.so and copies it back; the engine's buffers stay on
// the host as the engine expects.
//
// Module names (GetModule): the reference's names and the same names with a CUDA suffix:
//   FullLogNorm / FullLogNormCUDA             (NormPlugins.cpp:243-552)
//   MorphSpotClean / MorphSpotCleanCUDA       (MorphSpotCleanModule.cpp:14-269)
//   WaveletRingClean / WaveletRingCleanCUDA   (WaveletRingClean.cpp:17-146)
//   ProjectionFilterSingle / ProjectionFilterCUDA (ProjectionFilter.cpp:67-376)
#ifndef B200_PREPROC_MODULES_H
#define B200_PREPROC_MODULES_H

#include <map>
#include <string>

#include <MorphSpotClean.h>
#include <PreprocModuleBase.h>
#include <ReconConfig.h>
#include <StripeFilter.h>
#include <averageimage.h>
#include <base/timage.h>
#include <morphology/morphology.h>

#include "b200_common.h"

extern "C" {
void *GetModule(const char *application, const char *name, void *vinteractor);
int Destroy(const char *application, void *obj);
int LibVersion();
int GetModuleList(const char *application, void *listptr);
}

// FullLogNorm: dark/flat normalisation and -log (NormBase + FullLogNorm of NormPlugins.cpp).
// SetROI loads the reference images through the framework's ProjectionReader exactly as
// NormBase::ReferenceLoader does (file masks, doses over the dose ROI) and averages them on
// the device; SetReferenceImages takes averaged images directly, as the reference's does.
class FullLogNormCUDA : public PreprocModuleBase {
public:
    explicit FullLogNormCUDA(kipl::interactors::InteractionBase *interactor = nullptr);
    ~FullLogNormCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    std::map<std::string, std::string> GetParameters() override;
    bool SetROI(size_t *roi) override;
    void LoadReferenceImages(size_t *roi);
    void SetReferenceImages(kipl::base::TImage<float, 2> dark, kipl::base::TImage<float, 2> flat);

protected:
    int ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff) override;
    int ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff) override;

private:
    kipl::base::TImage<float, 2> ReferenceLoader(const std::string &fname, int firstIndex, int N, size_t *roi,
                                                  float initialDose, float doseBias, float &dose);
    ReconConfig m_Config;
    std::string path, flatname, darkname;
    int nOBCount = 0, nOBFirstIndex = 1, nDCCount = 0, nDCFirstIndex = 1;
    ImagingAlgorithms::AverageImage::eAverageMethod m_ReferenceAverage =
        ImagingAlgorithms::AverageImage::ImageWeightedAverage;
    float fFlatDose = 1.0f, fDarkDose = 0.0f;
    bool bUseNormROI = true, bUseLUT = false;
    size_t nOriginalNormRegion[4] = {0, 0, 0, 0};
    size_t nDarkPix = 0, nFlatPix = 0;
    b200::Stream stream;
    b200::DeviceArray<float> d_dark, d_logflat, d_img, d_doselog, d_stack;
};

// MorphSpotClean (MorphSpotCleanModule): spot cleaning by grey-scale reconstruction.
class MorphSpotCleanCUDA : public PreprocModuleBase {
public:
    explicit MorphSpotCleanCUDA(kipl::interactors::InteractionBase *interactor = nullptr);
    ~MorphSpotCleanCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    std::map<std::string, std::string> GetParameters() override;
    bool SetROI(size_t *roi) override;

protected:
    int ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff) override;
    int ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff) override;

private:
    void clean(float *img_h, size_t nu, size_t nv, size_t n, bool clamp, bool removeinfnan);
    kipl::morphology::MorphConnect m_eConnectivity = kipl::morphology::conn4;
    ImagingAlgorithms::eMorphDetectionMethod m_eDetectionMethod = ImagingAlgorithms::MorphDetectPeaks;
    ImagingAlgorithms::eMorphCleanMethod m_eCleanMethod = ImagingAlgorithms::MorphCleanReplace;
    std::vector<float> m_fThreshold{0.1f, 0.1f};
    std::vector<float> m_fSigma{0.01f, 0.01f};
    int m_nEdgeSmoothLength = 5;
    int m_nMaxArea = 30;
    bool m_bRemoveInfNaN = false, m_bClampData = false;
    float m_fMinLevel = -0.1f, m_fMaxLevel = 7.0f;
    bool m_bThreading = false;
    b200::Stream stream;
    b200::DeviceArray<float> d_img;
};

// WaveletRingClean: wavelet-Fourier stripe filtering of every detector row's sinogram.
class WaveletRingCleanCUDA : public PreprocModuleBase {
public:
    explicit WaveletRingCleanCUDA(kipl::interactors::InteractionBase *interactor = nullptr);
    ~WaveletRingCleanCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    std::map<std::string, std::string> GetParameters() override;
    bool SetROI(size_t *roi) override;

protected:
    int ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff) override;

private:
    std::string m_sWName = "daub15";
    float m_fSigma = 0.05f;
    int m_nDecNum = 2;
    bool m_bParallelProcessing = false;
    ImagingAlgorithms::eStripeFilterOperation m_eCleanMethod = ImagingAlgorithms::VerticalComponentFFT;
    b200::Stream stream;
    b200::DeviceArray<float> d_img;
};

// ProjectionFilterSingle: ramp-type filtering of every projection row.
class ProjectionFilterCUDA : public PreprocModuleBase {
public:
    explicit ProjectionFilterCUDA(kipl::interactors::InteractionBase *interactor = nullptr);
    ~ProjectionFilterCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    std::map<std::string, std::string> GetParameters() override;

protected:
    int ProcessCore(kipl::base::TImage<float, 2> &img, std::map<std::string, std::string> &coeff) override;
    int ProcessCore(kipl::base::TImage<float, 3> &img, std::map<std::string, std::string> &coeff) override;

private:
    void filter(float *img_h, size_t nu, size_t rows);
    std::string m_FilterType = "Hamming";
    float m_fCutOff = 0.5f, m_fOrder = 1.0f;
    bool m_bUseBias = true;
    float m_fBiasWeight = 0.1f;
    int m_nPaddingDoubler = 2;
    size_t nImageSize = 0;
    mr_filter_plan *plan = nullptr;
    b200::Stream stream;
    b200::DeviceArray<float> d_img;
};

#endif
