// MuhRec backprojectors on the B200 kernels: the classes of B200BackProjectors.h and the
// module library's factory functions (GetModule, Destroy, LibVersion, GetModuleList, resolved
// by BackProjItem with dlsym, frameworks/tomography/Framework/ReconFramework/src/
// ModuleItem.cpp:93-131).
#include "B200BackProjectors.h"

#include <algorithm>
#include <cstring>
#include <limits>
#include <sstream>

#include <ParameterHandling.h>
#include <strings/miscstring.h>

using b200::check;

namespace {

const char *kApplication = "muhrecbp";

// The framework's circle mask (BackProjectorModuleBase::BuildCircleMask) as the kernels'
// (first, second) pairs per volume row.
std::vector<uint32_t> mask_pairs(const std::vector<std::pair<size_t, size_t>> &mask)
{
    std::vector<uint32_t> m(2 * mask.size());
    for (size_t y = 0; y < mask.size(); ++y) {
        m[2 * y] = static_cast<uint32_t>(mask[y].first);
        m[2 * y + 1] = static_cast<uint32_t>(mask[y].second);
    }
    return m;
}

} // namespace

// ============================================================== MultiProjBPCUDA

MultiProjBPCUDA::MultiProjBPCUDA(int variant_, const std::string &name, kipl::interactors::InteractionBase *interactor)
    : BackProjectorModuleBase("muhrec", name, BackProjectorModuleBase::MatrixZXY, interactor), variant(variant_)
{
}

MultiProjBPCUDA::~MultiProjBPCUDA() = default;

// StdBackProjectorBase::Configure (StdBackProjectorBase.cpp:322-331)
int MultiProjBPCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    mConfig = config;
    nProjectionBufferSize = GetIntParameter(parameters, "ProjectionBufferSize");
    nSliceBlock = GetIntParameter(parameters, "SliceBlock");
    GetUIntParameterVector(parameters, "SubVolume", nSubVolume, 2);
    if (nProjectionBufferSize == 0 || nProjectionBufferSize > 1024)
        // the reference's per-buffer arrays hold 1024 entries (StdBackProjectorBase.h:68-72)
        throw ReconException("ProjectionBufferSize must be 1..1024", __FILE__, __LINE__);
    return 0;
}

int MultiProjBPCUDA::Initialize()
{
    return 0;
}

std::map<std::string, std::string> MultiProjBPCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["ProjectionBufferSize"] = kipl::strings::value2string(nProjectionBufferSize);
    parameters["SliceBlock"] = kipl::strings::value2string(nSliceBlock);
    parameters["SubVolume"] =
        kipl::strings::value2string(nSubVolume[0]) + " " + kipl::strings::value2string(nSubVolume[1]);
    return parameters;
}

// StdBackProjectorBase::SetROI (StdBackProjectorBase.cpp:152-201)
void MultiProjBPCUDA::SetROI(size_t *roi)
{
    SizeU = roi[2] - roi[0];
    SizeV = mConfig.ProjectionInfo.imagetype == ReconConfig::cProjections::ImageType_Proj_RepeatSinogram
                ? roi[3]
                : roi[3] - roi[1];
    std::memcpy(mConfig.ProjectionInfo.roi, roi, 4 * sizeof(size_t));
    MatrixDims[0] = SizeV;
    MatrixDims[1] = SizeU;
    MatrixDims[2] = SizeU;
    volume.Resize(MatrixDims);
    volume = 0.0f;
    BuildCircleMask();
    nProjCounter = 0;
    pending.clear();
    pendingAngle.clear();
    pendingWeight.clear();
    cudaStream_t s = stream.get();
    b200::cuda_check(cudaMemsetAsync(d_vol.get(volume.Size()), 0, volume.Size() * sizeof(float), s), "volume clear");
    const std::vector<uint32_t> m = mask_pairs(mask);
    b200::upload(d_mask.get(m.size()), m.data(), m.size(), s);
    stream.sync();
}

// Backprojects the projections of `block` (nslabs slabs of SizeU x SizeV) listed in `kept`
// (slab indices, in backprojection order) with their angles and weights, adding into the
// device volume, and copies the volume into `volume`.
void MultiProjBPCUDA::backproject(const std::vector<Entry> &entries)
{
    if (entries.empty()) return;
    const size_t n = entries.size(), per = SizeU * SizeV;
    cudaStream_t s = stream.get();
    float *proj = d_proj.get(n * per);
    std::vector<float> ang(n), w(n), sn(n), cs(n), su(n);
    for (size_t i = 0; i < n; ++i) {
        b200::upload(proj + i * per, entries[i].data, per, s);
        ang[i] = entries[i].angle;
        w[i] = entries[i].weight;
    }
    // StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:64-82): per-projection
    // sin, cos and start position with the rotation direction's sign
    check(mr_bp_parallel_geometry(ang.data(), n, SizeU, mConfig.ProjectionInfo.fCenter,
                                  static_cast<int>(mConfig.ProjectionInfo.eDirection), sn.data(), cs.data(), su.data()),
          "backprojection geometry");
    float *geo = d_geo.get(4 * n);
    b200::upload(geo, sn.data(), n, s);
    b200::upload(geo + n, cs.data(), n, s);
    b200::upload(geo + 2 * n, su.data(), n, s);
    b200::upload(geo + 3 * n, w.data(), n, s);
    const ReconConfig::cProjections &pi = mConfig.ProjectionInfo;
    float toff = 0.0f, tinc = 0.0f;
    if (pi.bCorrectTilt)
        check(mr_bp_parallel_tilt(pi.fTiltAngle, pi.fTiltPivotPosition, pi.roi[1], &toff, &tinc), "tilt");
    check(mr_bp_parallel_variant(variant, proj, n, MR_F32, nullptr, geo + 3 * n, nullptr, geo, geo + n, geo + 2 * n, n,
                                 SizeU, SizeV, d_mask.data(), pi.bCorrectTilt, toff, tinc, 0, SizeU, d_vol.data(), s),
          "backprojection");
    b200::download(volume.GetDataPtr(), d_vol.data(), volume.Size(), s);
    stream.sync();
    b200::check_device("backprojection");
}

// StdBackProjectorBase::Process 2D (StdBackProjectorBase.cpp:64-118): projections are
// buffered; a full buffer is backprojected without its last entry, the last projection of a
// scan flushes what is buffered.
size_t MultiProjBPCUDA::Process(kipl::base::TImage<float, 2> proj, float angle, float weight, bool bLastProjection)
{
    b200::Trace trace("MultiProjBPCUDA::Process");
    if (volume.Size() == 0) throw ReconException("The target matrix is not allocated.", __FILE__, __LINE__);
    const size_t per = SizeU * SizeV;
    if (proj.Size() != per) throw ReconException("The projection does not match the ROI", __FILE__, __LINE__);
    pending.insert(pending.end(), proj.GetDataPtr(), proj.GetDataPtr() + per);
    pendingAngle.push_back(angle);
    pendingWeight.push_back(weight);
    nProjCounter++;
    if (bLastProjection || nProjectionBufferSize <= nProjCounter) {
        if (nProjectionBufferSize <= nProjCounter) nProjCounter--;
        std::vector<Entry> entries(nProjCounter);
        for (size_t i = 0; i < nProjCounter; ++i) entries[i] = {pending.data() + i * per, pendingAngle[i], pendingWeight[i]};
        backproject(entries);
        nProjCounter = 0;
        pending.clear();
        pendingAngle.clear();
        pendingWeight.clear();
    }
    return nProjCounter;
}

// StdBackProjectorBase::Process 3D (StdBackProjectorBase.cpp:120-149): every projection
// through the 2D rule; the projections that rule backprojects go to the device in one call.
size_t MultiProjBPCUDA::Process(kipl::base::TImage<float, 3> projections, std::map<std::string, std::string> parameters)
{
    b200::Trace trace("MultiProjBPCUDA::Process");
    if (volume.Size() == 0) throw ReconException("The target matrix is not allocated.", __FILE__, __LINE__);
    const size_t nProj = projections.Size(2), per = SizeU * SizeV;
    if (projections.Size(0) * projections.Size(1) != per)
        throw ReconException("The projections do not match the ROI", __FILE__, __LINE__);
    std::vector<float> weights(nProj + 16), angles(nProj + 16);
    GetFloatParameterVector(parameters, "weights", weights.data(), static_cast<int>(nProj));
    GetFloatParameterVector(parameters, "angles", angles.data(), static_cast<int>(nProj));
    std::vector<Entry> entries;
    // projections buffered by earlier 2D calls come first, as in the reference's buffer
    for (size_t i = 0; i < nProjCounter; ++i) entries.push_back({pending.data() + i * per, pendingAngle[i], pendingWeight[i]});
    size_t counter = nProjCounter;
    size_t start = 0; // first entry of the current buffer
    std::vector<Entry> kept;
    for (size_t i = 0; i < nProj; ++i) {
        entries.push_back({projections.GetLinePtr(0, i), angles[i], weights[i]});
        counter++;
        const bool last = i == nProj - 1;
        if (last || nProjectionBufferSize <= counter) {
            if (nProjectionBufferSize <= counter) counter--;
            kept.insert(kept.end(), entries.begin() + start, entries.begin() + start + counter);
            start = entries.size();
            counter = 0;
        }
    }
    backproject(kept);
    nProjCounter = 0;
    pending.clear();
    pendingAngle.clear();
    pendingWeight.clear();
    return 0;
}

// StdBackProjectorBase::GetHistogram with its Min/Max (StdBackProjectorBase.cpp:240-309). As
// written there, Min and Max take std::min of two pointers, i.e. the first slice's value of
// each masked voxel column.
void MultiProjBPCUDA::GetHistogram(float *axis, size_t *hist, size_t nBins)
{
    float matrixMin = std::numeric_limits<float>::max(), matrixMax = -std::numeric_limits<float>::max();
    for (size_t y = 0; y < mask.size(); ++y)
        for (size_t x = mask[y].first; x < mask[y].second; ++x) {
            const float v = *volume.GetLinePtr(x, y);
            matrixMin = std::min(matrixMin, v);
            matrixMax = std::max(matrixMax, v);
        }
    std::memset(axis, 0, sizeof(float) * nBins);
    std::memset(hist, 0, sizeof(size_t) * nBins);
    const float scale = (matrixMax - matrixMin) / (nBins + 1);
    const float invScale = 1.0f / scale;
    for (size_t y = 0; y < mask.size(); ++y)
        for (size_t x = mask[y].first; x < mask[y].second; ++x) {
            const float *pLine = volume.GetLinePtr(x, y);
            for (size_t z = 0; z < volume.Size(0); ++z) {
                size_t index = static_cast<size_t>(invScale * (pLine[z] - matrixMin));
                if (pLine[z] < matrixMin) index = 0;
                else if (nBins <= index) index = nBins - 1;
                hist[index]++;
            }
        }
    axis[0] = matrixMin + scale / 2.0f;
    for (size_t i = 1; i < nBins; ++i) axis[i] = axis[i - 1] + scale;
}

// ============================================================== FDKbpCUDA

FDKbpCUDA::FDKbpCUDA(kipl::interactors::InteractionBase *interactor)
    : BackProjectorModuleBase("muhrecbp", "FDKbp_single", BackProjectorModuleBase::MatrixXYZ, interactor)
{
}

FDKbpCUDA::~FDKbpCUDA() = default;

// FdkReconBase::Configure (fdkreconbase.cpp:45-58)
int FDKbpCUDA::Configure(ReconConfig config, std::map<std::string, std::string> parameters)
{
    mConfig = config;
    nProjectionBufferSize = GetIntParameter(parameters, "ProjectionBufferSize");
    nSliceBlock = GetIntParameter(parameters, "SliceBlock");
    GetUIntParameterVector(parameters, "SubVolume", nSubVolume, 2);
    return 0;
}

int FDKbpCUDA::Initialize()
{
    return 0;
}

std::map<std::string, std::string> FDKbpCUDA::GetParameters()
{
    std::map<std::string, std::string> parameters;
    parameters["ProjectionBufferSize"] = kipl::strings::value2string(nProjectionBufferSize);
    parameters["SliceBlock"] = kipl::strings::value2string(nSliceBlock);
    parameters["SubVolume"] =
        kipl::strings::value2string(nSubVolume[0]) + " " + kipl::strings::value2string(nSubVolume[1]);
    return parameters;
}

// FdkReconBase::SetROI (fdkreconbase.cpp:91-150). The kernels take the full detector as the
// region (roi = projection_roi = (0, 0, nu, nv)).
void FDKbpCUDA::SetROI(size_t *roi)
{
    if (roi[0] != 0 || roi[1] != 0)
        throw ReconException("FDKbp_single: only a full-detector ROI starting at (0, 0) is supported", __FILE__,
                             __LINE__);
    SizeU = roi[2] - roi[0];
    SizeV = mConfig.ProjectionInfo.imagetype == ReconConfig::cProjections::ImageType_Proj_RepeatSinogram
                ? roi[3]
                : roi[3] - roi[1];
    std::memcpy(mConfig.ProjectionInfo.roi, roi, 4 * sizeof(size_t));
    MatrixDims[0] = SizeU;
    MatrixDims[1] = SizeU;
    MatrixDims[2] = SizeV;
    volume.Resize(MatrixDims);
    volume = 0.0f;
    BuildCircleMask();
    first = true;
    cudaStream_t s = stream.get();
    b200::cuda_check(cudaMemsetAsync(d_vol.get(volume.Size()), 0, volume.Size() * sizeof(float), s), "volume clear");
    const std::vector<uint32_t> m = mask_pairs(mask);
    b200::upload(d_mask.get(m.size()), m.data(), m.size(), s);
    stream.sync();
}

// FdkReconBase::Process 3D (fdkreconbase.cpp:217-277) with FDKbp_single::reconstruct: the
// projections weighted, ramp filtered and backprojected; every call adds into the volume.
size_t FDKbpCUDA::Process(kipl::base::TImage<float, 3> projections, std::map<std::string, std::string> parameters)
{
    b200::Trace trace("FDKbpCUDA::Process");
    if (volume.Size() == 0) throw ReconException("The target matrix is not allocated.", __FILE__, __LINE__);
    const size_t nProj = projections.Size(2), nu = SizeU, nv = SizeV;
    if (projections.Size(0) != nu || projections.Size(1) != nv)
        throw ReconException("The projections do not match the ROI", __FILE__, __LINE__);
    if (nProj == 0) return 0;
    std::vector<float> weights(nProj + 16), angles(nProj);
    GetFloatParameterVector(parameters, "weights", weights.data(), static_cast<int>(nProj));
    GetFloatParameterVector(parameters, "angles", angles.data(), static_cast<int>(nProj));
    const ReconConfig::cProjections &pi = mConfig.ProjectionInfo;
    mr_fdk_geom g;
    g.sod = pi.fSOD;
    g.sdd = pi.fSDD;
    g.ppoint[0] = pi.fpPoint[0];
    g.ppoint[1] = pi.fpPoint[1];
    g.center = pi.fCenter;
    g.resolution[0] = pi.fResolution[0];
    g.resolution[1] = pi.fResolution[1];
    g.voxelsize[0] = mConfig.MatrixInfo.fVoxelSize[0];
    g.voxelsize[1] = mConfig.MatrixInfo.fVoxelSize[1];
    g.voxelsize[2] = mConfig.MatrixInfo.fVoxelSize[2];
    g.direction = static_cast<int>(pi.eDirection);
    g.correcttilt = pi.bCorrectTilt;
    g.tiltangle = pi.fTiltAngle;
    g.tiltpivot = pi.fTiltPivotPosition;
    std::vector<float> xip(nProj * nu * 3), yip(nProj * nu * 3), zip(nProj * nv * 3);
    float s2 = 0.0f, scale = 0.0f;
    int uniform = 0, bw = 0, bh = 0;
    check(mr_fdk_partials(&g, nu, nv, angles.data(), nProj, xip.data(), yip.data(), zip.data(), &s2, &scale, &uniform),
          "FDK geometry");
    if (uniform) check(mr_fdk_box(xip.data(), yip.data(), zip.data(), nu, nv, nProj, MR_F32, &bw, &bh), "FDK box");
    cudaStream_t s = stream.get();
    const size_t total = nProj * nu * nv;
    float *proj = d_proj.get(total), *filt = d_filt.get(total), *w = d_weight.get(nProj);
    b200::upload(proj, projections.GetDataPtr(), total, s);
    b200::upload(w, weights.data(), nProj, s);
    float *X = d_xip.get(xip.size()), *Y = d_yip.get(yip.size()), *Z = d_zip.get(zip.size());
    b200::upload(X, xip.data(), xip.size(), s);
    b200::upload(Y, yip.data(), yip.size(), s);
    b200::upload(Z, zip.data(), zip.size(), s);
    check(mr_fdk_filter(proj, nu, nv, nProj, w, s2, scale, MR_F32, filt, nullptr, s), "FDK ramp filter");
    check(mr_fdk_backproject(filt, MR_F32, nullptr, nu, nv, nProj, X, Y, Z, uniform, d_mask.data(), bw, bh, !first,
                             d_vol.data(), s),
          "FDK backprojection");
    first = false;
    b200::download(volume.GetDataPtr(), d_vol.data(), volume.Size(), s);
    stream.sync();
    b200::check_device("FDK backprojection");
    return 0;
}

// FdkReconBase::GetHistogram with its Min/Max over the whole volume (fdkreconbase.cpp:293-367)
void FDKbpCUDA::GetHistogram(float *axis, size_t *hist, size_t nBins)
{
    float matrixMin = std::numeric_limits<float>::max(), matrixMax = -std::numeric_limits<float>::max();
    const float *p = volume.GetDataPtr();
    for (size_t i = 0; i < volume.Size(); ++i) {
        matrixMin = std::min(matrixMin, p[i]);
        matrixMax = std::max(matrixMax, p[i]);
    }
    std::memset(axis, 0, sizeof(float) * nBins);
    std::memset(hist, 0, sizeof(size_t) * nBins);
    const float scale = (matrixMax - matrixMin) / (nBins + 1);
    const float invScale = 1.0f / scale;
    for (size_t i = 0; i < volume.Size(); ++i) {
        size_t index = static_cast<size_t>(invScale * (p[i] - matrixMin));
        if (p[i] < matrixMin) index = 0;
        else if (nBins <= index) index = nBins - 1;
        hist[index]++;
    }
    axis[0] = matrixMin + scale / 2.0f;
    for (size_t i = 1; i < nBins; ++i) axis[i] = axis[i - 1] + scale;
}

// ============================================================== factory functions

// StdBackProjectors.cpp:25-47 and fdkbackproj.cpp:17-35: the application tag must be "muhrecbp"
void *GetModule(const char *application, const char *name, void *vinteractor)
{
    if (!application || std::strcmp(application, kApplication) != 0 || !name) return nullptr;
    auto *interactor = reinterpret_cast<kipl::interactors::InteractionBase *>(vinteractor);
    const std::string n = name;
    BackProjectorModuleBase *m = nullptr;
    if (n == "MultiProjBPparallel" || n == "MultiProjBPCUDA")
        m = new MultiProjBPCUDA(MR_BP_MULTIPROJ_PARALLEL, "Multi projection BP parallel", interactor);
    else if (n == "MultiProjBP")
        m = new MultiProjBPCUDA(MR_BP_MULTIPROJ_SERIAL, "Multi projection BP", interactor);
    else if (n == "NearestNeighborBP")
        m = new MultiProjBPCUDA(MR_BP_NEAREST, "NearestNeighborBP", interactor);
    else if (n == "FDKbp_single" || n == "FDKbpCUDA")
        m = new FDKbpCUDA(interactor);
    return m;
}

int Destroy(const char *application, void *obj)
{
    if (!application || std::strcmp(application, kApplication) != 0) return -1;
    if (obj) delete reinterpret_cast<BackProjectorModuleBase *>(obj);
    return 0;
}

int LibVersion()
{
    return mr_version();
}

// StdBackProjectors.cpp:70-87 and fdkbackproj.cpp:57-73
int GetModuleList(const char *application, void *listptr)
{
    if (!application || std::strcmp(application, kApplication) != 0) return -1;
    auto *modulelist = reinterpret_cast<std::map<std::string, std::map<std::string, std::string>> *>(listptr);
    MultiProjBPCUDA mpbp(MR_BP_MULTIPROJ_SERIAL, "Multi projection BP");
    (*modulelist)["MultiProjBP"] = mpbp.GetParameters();
    MultiProjBPCUDA mpbpp(MR_BP_MULTIPROJ_PARALLEL, "Multi projection BP parallel");
    (*modulelist)["MultiProjBPparallel"] = mpbpp.GetParameters();
    MultiProjBPCUDA nnbp(MR_BP_NEAREST, "NearestNeighborBP");
    (*modulelist)["NearestNeighborBP"] = nnbp.GetParameters();
    FDKbpCUDA fdk;
    (*modulelist)["FDKbp_single"] = fdk.GetParameters();
    return 0;
}
