// MuhRec backprojectors on the B200 kernels (libB200BackProjectors.so, application tag
// "muhrecbp").
//
// Each class is a BackProjectorModuleBase (frameworks/tomography/Framework/ReconFramework/
// include/BackProjectorModuleBase.h) with the reference module's parameters, SetROI, Process
// and GetHistogram behaviour; the volume is accumulated on the device and copied into the
// module's `volume` after every Process call, so the framework's own GetVolume / GetSlice /
// GetNSlices (and ReconEngine::TransferMatrix) read it as they read the reference modules'.
// The circle mask is the framework's own BuildCircleMask.
//
// Module names (GetModule):
//   MultiProjBPparallel / MultiProjBPCUDA   MultiProjectionBPparallel (MultiProjBPparallel.cpp:39-170)
//   MultiProjBP                              MultiProjectionBP (MultiProjBP.cpp:36-146)
//   NearestNeighborBP                        NearestNeighborBP (NNMultiProjBP.cpp:36-121)
//   FDKbp_single / FDKbpCUDA                 FDKbp_single (fdkbp_single.cpp:83-994) with FdkReconBase
//                                            (fdkreconbase.cpp:91-277)
#ifndef B200_BACKPROJECTORS_H
#define B200_BACKPROJECTORS_H

#include <map>
#include <string>
#include <vector>

#include <BackProjectorModuleBase.h>
#include <ReconConfig.h>
#include <base/timage.h>

#include "b200_common.h"

extern "C" {
void *GetModule(const char *application, const char *name, void *vinteractor);
int Destroy(const char *application, void *obj);
int LibVersion();
int GetModuleList(const char *application, void *listptr);
}

// The parallel-beam backprojectors of StdBackProjectors (StdBackProjectorBase driver,
// StdBackProjectorBase.cpp:64-201), MatrixZXY. variant: MR_BP_MULTIPROJ_PARALLEL,
// MR_BP_MULTIPROJ_SERIAL or MR_BP_NEAREST.
class MultiProjBPCUDA : public BackProjectorModuleBase {
public:
    MultiProjBPCUDA(int variant, const std::string &name, kipl::interactors::InteractionBase *interactor = nullptr);
    ~MultiProjBPCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    int Initialize() override;
    std::map<std::string, std::string> GetParameters() override;
    void SetROI(size_t *roi) override;
    void GetHistogram(float *axis, size_t *hist, size_t nBins) override;
    size_t Process(kipl::base::TImage<float, 2> proj, float angle, float weight, bool bLastProjection) override;
    size_t Process(kipl::base::TImage<float, 3> proj, std::map<std::string, std::string> parameters) override;

private:
    struct Entry {
        const float *data; // nu * nv floats, projection row-major (detector column fastest)
        float angle, weight;
    };
    void backproject(const std::vector<Entry> &entries);
    int variant;
    size_t nProjectionBufferSize = 16, nSliceBlock = 32, nSubVolume[2] = {1, 1};
    size_t SizeU = 0, SizeV = 0;
    size_t nProjCounter = 0;
    std::vector<float> pending;         // projections buffered by the 2D Process
    std::vector<float> pendingAngle, pendingWeight;
    b200::Stream stream;
    b200::DeviceArray<float> d_vol, d_proj, d_geo;
    b200::DeviceArray<uint32_t> d_mask;
};

// FDKbp_single with the FdkReconBase driver, MatrixXYZ: ramp filter and nearest-neighbour
// cone-beam backprojection on the device; the volume is written at the position of the
// reference's final per-slice mirror and z reversal.
class FDKbpCUDA : public BackProjectorModuleBase {
public:
    explicit FDKbpCUDA(kipl::interactors::InteractionBase *interactor = nullptr);
    ~FDKbpCUDA() override;
    int Configure(ReconConfig config, std::map<std::string, std::string> parameters) override;
    int Initialize() override;
    std::map<std::string, std::string> GetParameters() override;
    void SetROI(size_t *roi) override;
    void GetHistogram(float *axis, size_t *hist, size_t nBins) override;
    size_t Process(kipl::base::TImage<float, 3> proj, std::map<std::string, std::string> parameters) override;

private:
    size_t nProjectionBufferSize = 16, nSliceBlock = 32, nSubVolume[2] = {1, 1};
    size_t SizeU = 0, SizeV = 0;
    bool first = true;
    b200::Stream stream;
    b200::DeviceArray<float> d_vol, d_proj, d_filt, d_weight, d_xip, d_yip, d_zip;
    b200::DeviceArray<uint32_t> d_mask;
};

#endif
