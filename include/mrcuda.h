/* mrcuda: B200 (sm_100a) kernels for the MuhRec reconstruction hot path, behind a C ABI.
 *
 * Every entry point takes plain pointers and sizes. Pointers named *_d are device
 * pointers (cudaMalloc'd or otherwise device-accessible); *_h are host pointers.
 * `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 * Calls are asynchronous on `stream` unless stated otherwise; argument errors are
 * reported before anything is launched. Every call returns an mr_status; MR_OK is 0.
 * On failure, mr_last_error() returns a message for the calling thread.
 *
 * Array layouts follow kipl::base::TImage (first index fastest):
 *   projections  [nproj][nv][nu]   u (detector column) fastest
 *   parallel-beam volume (MatrixZXY) [ny][nx][nz]  z fastest, nx = ny = nu, nz = nv
 *   FDK volume (MatrixXYZ)           [nz][ny][nx]  x fastest, nx = ny = nu, nz = nv
 *
 * Entry points that need scratch take it from the device's default stream-ordered memory
 * pool (cudaMallocAsync), whose release threshold they raise so that freed scratch stays
 * cached for the next call.
 *
 * Reference interfaces each group replaces are cited as file:line, relative to the
 * reference project root (DTasev/imagingsuite).
 */
#ifndef MRCUDA_H
#define MRCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mr_status;
enum {
    MR_OK = 0,
    MR_ERR_ARGUMENT = 1,    /* invalid size, pointer or parameter (nothing launched) */
    MR_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    MR_ERR_ALLOCATION = 3,  /* device or host allocation failed */
    MR_ERR_UNSUPPORTED = 4, /* valid request the library does not implement */
    MR_ERR_DEVICE = 5       /* a kernel reported an error status (bounded wait expired, ...) */
};

/* Library version (major*10000 + minor*100 + patch) and status text. */
int mr_version(void);
const char *mr_status_string(mr_status s);
const char *mr_last_error(void);

/* Precision of stored projections. MR_F32 is the reference arithmetic; MR_BF16 and
 * MR_F16 store filtered projections in 16 bits with a per-projection power-of-two
 * scale and accumulate in FP32. */
enum { MR_F32 = 0, MR_BF16 = 1, MR_F16 = 2 };

/* ---------------------------------------------------------------------------------
 * Reference frames and doses (FullLogNorm preparation)
 * replaces ImagingAlgorithms::AverageImage::operator()
 *   (core/algorithms/ImagingAlgorithms/src/averageimage.cpp:35-61) and
 *   ProjectionReader::GetProjectionDose (frameworks/tomography/Framework/ReconFramework/
 *   src/ProjectionReader.cpp:752-783).
 * method: 0 ImageSum, 1 ImageAverage, 2 ImageMedian (at most 64 frames), 3 ImageWeightedAverage
 * (per-frame 5x5 StdDevFilter with EdgeMirror edges, weights 1/sigma, or 1/(number of pixels)
 * where sigma is 0; frames at least 5x5; scratch: four images per frame), 4 ImageMin, 5 ImageMax
 * (averageimage.h:16-23). frames_d: [n][nv][nu] float. */
mr_status mr_reference_average(const float *frames_d, size_t nu, size_t nv, size_t n, int method, float *out_d,
                               void *stream);
/* Dose of each frame: median over the rows of roi (x0,y0,x1,y1) of the row means.
 * in_d holds nframes frames of nu x nv, as float (dtype MR_F32) or uint16 (dtype 3).
 * A ROI with any zero coordinate gives 1.0 like the reference. */
enum { MR_U16 = 3 };
mr_status mr_projection_dose(const void *in_d, int dtype, size_t nu, size_t nv, size_t nframes, const size_t *roi_h,
                             float *dose_d, void *stream);

/* ---------------------------------------------------------------------------------
 * FullLogNorm (frameworks/tomography/Preprocessing/StdPreprocModules/src/NormPlugins.cpp)
 * mr_lognorm_logflat replaces FullLogNorm::SetReferenceImages (:300-341):
 *     logflat = (F - D <= 0) ? 0 : log((F - D) / flatdose)     (ndc = 0: F alone)
 * mr_lognorm_doselog replaces the dose list of ProcessCore 3D (:416-425), on the host:
 *     doselog[j] = log(max(dose[j] - darkdose, 1))
 * mr_lognorm_apply replaces ProcessCore 3D (:481-549), non-LUT path:
 *     p = (I - D <= 0) ? 0 : logflat - log(I - D) + doselog[j]   (nob = 0: -log(I-D)+doselog)
 * in_d: [nproj][npix] of uint16 (in_dtype MR_U16) or float (MR_F32; may alias out_d).
 * ndose: 1 (one value for all projections) or nproj. */
mr_status mr_lognorm_logflat(const float *dark_d, const float *flat_d, size_t npix, int ndc, float flatdose,
                             float *logflat_d, void *stream);
mr_status mr_lognorm_doselog(const float *dose_h, size_t n, float darkdose, float *doselog_h);
mr_status mr_lognorm_apply(const void *in_d, int in_dtype, size_t npix, size_t nproj, const float *dark_d,
                           const float *logflat_d, const float *doselog_d, size_t ndose, int ndc, int nob,
                           float *out_d, void *stream);
/* mr_lognorm_apply_lut: the module's uselut path (NormPlugins.cpp:455-480): LogLUT(1 << 16, 0,
 * 65535) of I - D (log of the value rounded half up, log(1) = 0 at and below 0, log(65535)
 * above), then logflat - l + dose, or -l + (dose - doselog[0]) without flats. The table is
 * built on the host with the reference's double log, so results equal the reference bit for
 * bit. Same arguments as mr_lognorm_apply; scratch: the 256 KiB table. */
mr_status mr_lognorm_apply_lut(const void *in_d, int in_dtype, size_t npix, size_t nproj, const float *dark_d,
                               const float *logflat_d, const float *doselog_d, size_t ndose, int ndc, int nob,
                               float *out_d, void *stream);

/* ---------------------------------------------------------------------------------
 * MorphSpotClean, replace mode: ImagingAlgorithms::MorphSpotClean::process
 * (core/algorithms/ImagingAlgorithms/src/MorphSpotClean.cpp:41-175,264-351) with
 * kipl::morphology FillHole/FillPeaks (core/kipl/kipl/include/morphology/morphextrema.h:265-328,
 * morphgeo.h:151-371), in place on nproj images [nproj][nv][nu].
 * detect: 0 holes, 1 peaks, 2 both; conn8: 0 = 4-connectivity, 1 = 8-connectivity;
 * th_h/sigma_h: two host floats each (holes, peaks); sigma == 0 for both selects threshold
 * replacement, else the sigmoid blend; edge: length of the sliding median along the first
 * and last padded rows (the reference default is 9); clamp/minlevel/maxlevel: LimitDynamics
 * before cleaning; removeinfnan: replace inf/NaN by the largest finite value first.
 * nv must be at least 5 (the reference mirrors 5 rows into its padding and reads outside
 * smaller images). Scratch from the stream-ordered pool: per image in a batch three padded
 * float images and two worklists of 1/16 of their pixels; a batch is as many images as fit
 * in max(1 GiB, a quarter of the free device memory). */
mr_status mr_morphspotclean(float *proj_d, size_t nu, size_t nv, size_t nproj, int detect, int conn8,
                            const float *th_h, const float *sigma_h, int edge, int clamp, float minlevel,
                            float maxlevel, int removeinfnan, void *stream);

/* ---------------------------------------------------------------------------------
 * Wavelet-FFT ring cleaning
 * mr_stripefilter replaces ImagingAlgorithms::StripeFilter::process with
 * VerticalComponentFFT (core/algorithms/ImagingAlgorithms/src/StripeFilter.cpp:68-250,
 * kipl::wavelets::WaveletTransform core/kipl/kipl/include/wavelets/core/wavelets.hpp:452-862)
 * on nsino contiguous sinograms [nsino][ntheta][nu], in place.
 * mr_waveletringclean replaces WaveletRingClean::ProcessCore (frameworks/tomography/
 * Preprocessing/StdPreprocModules/src/WaveletRingClean.cpp:63-103): every detector row's
 * sinogram of projections [nproj][nv][nu], in place.
 * wname: "daub1".."daub30" except daub28 (daub1..15 computed from their definition, equal to
 * kipl's float kernels, daub3 with the reference's sign of its fifth coefficient; daub16..30
 * kipl's own table values; kipl's daub28 table is shorter than its filter, so the reference's
 * daub28 kernel is undefined and it returns MR_ERR_UNSUPPORTED); decnum: decomposition levels;
 * sigma: damping width. Scratch: up to about 1 GiB per call.
 * mr_wavelet_kernel (host) returns begin/end and the four filters (analysis H, analysis G,
 * synthesis H, synthesis G; 4*(end-begin+1) floats) of WaveletKernel<float>. */
mr_status mr_wavelet_kernel(const char *wname, int *begin, int *end, float *taps_h);
mr_status mr_stripefilter(float *sino_d, size_t nu, size_t ntheta, size_t nsino, const char *wname, int decnum,
                          float sigma, void *stream);
mr_status mr_waveletringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, const char *wname, int decnum,
                              float sigma, void *stream);

/* ---------------------------------------------------------------------------------
 * Projection weights (host)
 * replaces ComputeWeights (frameworks/tomography/Framework/ReconFramework/src/ReconHelpers.cpp:
 *   365-488) on the list BuildFileList makes (:100-110): angles_h in acquisition order;
 *   scanarc_h = ProjectionInfo.fScanArc (first, last); golden_section: GoldenSectionScan.
 *   Writes the weighted projection map in its order (sorted by angle; a repeated angle keeps
 *   its last entry; below 3 projections sorted by angle modulo 180) to angles_out_h /
 *   weights_out_h (room for n each) and its size to *nout_h. Times 1 / (0.1 * pixel size)
 *   (ProjectionReader.cpp:907-919) these are the `weights` list the backprojectors take. */
mr_status mr_compute_weights(const float *angles_h, size_t n, const float *scanarc_h, int golden_section,
                             float *angles_out_h, float *weights_out_h, size_t *nout_h);

/* ---------------------------------------------------------------------------------
 * Alternative ring cleaners and the kipl median filter they use
 * mr_median_filter replaces kipl::filters::TMedianFilter<float,2>::operator()
 *   (core/kipl/kipl/include/filters/core/medianfilter.hpp:28-199, HeapSortMedianFilter with
 *   ExtractNeighborhood) on nimg images [nimg][nv][nu], out of place: odd kx, ky up to 5,
 *   nu >= 2*(kx/2), nv >= 2*(ky/2) (at smaller sizes the reference rejects the edge code or
 *   reads outside the image). The reference's window near the bottom-right corner reaches a few
 *   values past the image end; those values are taken as 0. Results equal the reference's
 *   heap-sort median bit for bit, NaN and signed zeros included.
 * mr_basicringclean replaces BasicRingClean::ProcessCore (frameworks/tomography/Preprocessing/
 *   StdPreprocModules/src/BasicRingClean.cpp:50-95): every projection minus (mean projection -
 *   its 3x3 median); nu, nv >= 2. The debug images the reference writes to its working
 *   directory are not written. Scratch: two images.
 * mr_medianmixringclean replaces MedianMixRingClean::ProcessCore / ComputeProfile
 *   (StdPreprocModules/src/MedianMixRingClean.cpp:57-138): w = SigmoidLUT(1024, threshold,
 *   width)(|mean - 3x3 median of mean|) (5x1 when nv < 3), then every projection becomes
 *   (1 - w) * p + w * (its 5x5 median; 5x1 when nv < 5). nu >= 4, width > 0. Scratch: two
 *   images and about 512 MiB of filtered projections.
 * mr_sigmoid_lut (host) returns kipl::math::SigmoidLUT's table (len floats) and param = lo, hi,
 *   slope, intercept (core/kipl/kipl/src/math/LUTCollection.cpp:38-82, LUTbase.cpp:12-20).
 * GammaSpotClean needs no entry point: GammaSpotCleanModule::ProcessCore returns without
 *   touching the projections (StdPreprocModules/src/GammaSpotCleanModule.cpp:58-68). */
mr_status mr_median_filter(const float *img_d, size_t nu, size_t nv, size_t nimg, int kx, int ky, float *out_d,
                           void *stream);
mr_status mr_basicringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, void *stream);
mr_status mr_medianmixringclean(float *proj_d, size_t nu, size_t nv, size_t nproj, float threshold, float width,
                                void *stream);
mr_status mr_sigmoid_lut(size_t len, float lambda, float sigma, float *lut_h, float *param_h);

/* ---------------------------------------------------------------------------------
 * SpotClean2
 * replaces SpotClean2::ProcessCore 3D (frameworks/tomography/Preprocessing/StdPreprocModules/
 *   src/SpotClean2.cpp:117-130) -> ImagingAlgorithms::SpotClean::Process (core/algorithms/
 *   ImagingAlgorithms/src/SpotClean.cpp:78-545) on projections [nproj][nv][nu], in place:
 *   `iterations` passes of detection (method below, kipl filters with EdgeMirror edges),
 *   SigmoidLUT(1 << 15, gamma, sigma), exclusion of 8-connected regions larger than maxarea
 *   (0: none) by the reference's RemoveConnectedRegion rule, spots outside [minlevel, maxlevel]
 *   or with a nonzero weight, and the neighbour-mean fill rounds of CleanByArray.
 *   nu, nv >= 16; sigma > 0. Synchronises the stream once per batch of projections (a batch
 *   is about 1 GiB of scratch: five images per projection). A round that corrects nothing while
 *   spots remain (the reference would loop forever) returns MR_ERR_DEVICE; with the value past
 *   the image end read as 0 the last pixel always has an unmarked neighbour, so this is a
 *   guard, not an expected outcome. TriKernel's level
 *   statistics are fixed-order double sums (the reference's running update differs below
 *   1e-15 relative). */
enum { MR_SPOT_STDDEV = 0, MR_SPOT_RING = 1, MR_SPOT_MEDIAN = 2, MR_SPOT_MINMAX = 3, MR_SPOT_TRIKERNEL = 4 };
mr_status mr_spotclean2(float *proj_d, size_t nu, size_t nv, size_t nproj, int method, float gamma, float sigma,
                        int iterations, float minlevel, float maxlevel, int maxarea, void *stream);

/* ---------------------------------------------------------------------------------
 * ProjectionFilterSingle (StdPreprocModules/src/ProjectionFilter.cpp:78-376)
 * Plan = ProjectionFilterBase::Configure/BuildFilter/PreparePadding (:78-93,254-299,364-376):
 *   nfft = 2^(ceil(log2 nu) + paddingdoubler); filter over bins 0..nfft/2-1.
 *   filtertype: "ram-lak", "shepp-logan", "hanning", "hamming", "butterworth" (any case).
 * Apply = FilterProjection + Pad (:301-362) on nrows rows of nu floats:
 *   sigmoid-tapered padding, r2c, bins 0..nfft/2-1 times the filter (Nyquist untouched),
 *   c2r, times pi/(2 nfft), cropped. in_d may alias out_d.
 * row_weight_d (optional, may be NULL): one factor per group of rows_per_weight rows,
 *   multiplied into the output after the reference's scale (the backprojector weighting
 *   of StdBackProjectorBase::Process, StdBackProjectorBase.cpp:80, fused). */
typedef struct mr_filter_plan mr_filter_plan;
/* Host-only: the filter table (nfft/2 floats, filter_h may be NULL to query sizes) and the
 * padding taper (ninsert floats) exactly as BuildFilter/PreparePadding compute them. */
mr_status mr_projfilter_tables(size_t nu, const char *filtertype, float cutoff, float order, int usebias,
                               float biasweight, int paddingdoubler, size_t *nfft, size_t *ninsert, float *filter_h,
                               float *pad_h);
mr_status mr_projfilter_create(size_t nu, const char *filtertype, float cutoff, float order, int usebias,
                               float biasweight, int paddingdoubler, mr_filter_plan **plan);
mr_status mr_projfilter_destroy(mr_filter_plan *plan);
/* Copies the filter table (nfft/2 floats) and padding table (ninsert floats) to the host. */
mr_status mr_projfilter_info(const mr_filter_plan *plan, size_t *nfft, size_t *ninsert, float *filter_h,
                             float *pad_h);
mr_status mr_projfilter_apply(const mr_filter_plan *plan, const float *in_d, float *out_d, size_t nrows,
                              const float *row_weight_d, size_t rows_per_weight, void *stream);

/* Precision form: 16-bit copy of nproj float projections of `per` values each, with a
 * power-of-two scale per projection (value = stored * scale_d[i]; the largest magnitude
 * maps into [2^13, 2^14) for MR_F16, into [0.5, 1) for MR_BF16). out_d holds bf16/f16 bits. */
mr_status mr_quantize(const float *in_d, size_t per, size_t nproj, int dtype, uint16_t *out_d, float *scale_d,
                      void *stream);
/* mr_quantize for callers that cannot allocate device memory: code running inside a
 * framework that owns every allocation (a fixed memory pool, a plugin host that forbids
 * cudaMalloc) or code that must not allocate while the stream is being used elsewhere.
 * This entry point has no counterpart in the reference. It computes exactly what
 * mr_quantize computes, but its per-projection scratch (the running |max| and the inverse
 * scales) lives in a static device array built into the library instead of cudaMallocAsync
 * memory: at most 65536 projections per call (512 KiB, held on every device that loads the
 * library until the process exits); larger calls are rejected with MR_ERR_ARGUMENT. It
 * allocates nothing. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture. The address is kept for the life of the process: after cudaDeviceReset on a
 * device, do not call this entry point on that device again. All calls share the one array,
 * and each call clears the part it uses first, so calls that overlap on the GPU (on
 * different streams without ordering) race. */
mr_status mr_quantize_noalloc(const float *in_d, size_t per, size_t nproj, int dtype, uint16_t *out_d, float *scale_d,
                              void *stream);

/* ---------------------------------------------------------------------------------
 * Parallel-beam backprojection: MultiProjectionBPparallel
 * (frameworks/tomography/Backprojectors/StdBackProjectors/src/MultiProjBPparallel.cpp:39-170)
 * with the geometry of StdBackProjectorBase::Process/SetROI
 * (StdBackProjectorBase.cpp:64-201) and BackProjectorModuleBase::BuildCircleMask
 * (frameworks/tomography/Framework/ReconFramework/src/BackProjectorModuleBase.cpp:153-218).
 *
 * mr_bp_parallel_geometry (host) fills, per projection, exactly the reference's floats:
 *   sin_h = sin(d*angle*pi/180), cos_h likewise, startu_h = (nu/2)*(sin - cos) + center,
 *   d = +1 for counter-clockwise (direction 1), -1 for clockwise (direction 0).
 * mr_bp_circle_mask (host) fills mask_h[2*y], mask_h[2*y+1] = first, second of row y.
 *
 * mr_bp_parallel accumulates (+=) into vol_d ([nu][nu][nv], z fastest) the linear
 * interpolation backprojection of nproj projections:
 *   vol[z][x-1][y-1] += P_i[z][n]*(1-f) + P_i[z][n+1]*f,   u = startu_i + cos_i*y - sin_i*x,
 *   n = (int)u in [0, nu-2], f = |u - n|, x in (first, second] of mask row y-1,
 * projections applied in list order i = 0..nproj-1, entry i reading projection slab
 * index_d[i] of proj_d (index_d NULL: slab i) and multiplied by weight_d[i] first
 * (weight_d may be NULL for pre-weighted projections); sin/cos/startu are per list entry. Only z < 4*(nv/4) is updated, as in the
 * reference. proj_d: [slabs][nv][nu] in `dtype`; for MR_BF16/MR_F16, scale_d[slab] is the
 * per-projection scale (value = stored * scale). Tilt (correcttilt != 0) follows the
 * reference tilt branch (:47-110) with tiltoffset = (roi_y0 - pivot)*tan(tilt) and
 * tiltinc = 4*tan(tilt), both computed by the caller (see mr_bp_parallel_tilt).
 * sin/cos/startu/weight/mask are device arrays (copy the host results over). */
mr_status mr_bp_parallel_geometry(const float *angles_h, size_t nproj, size_t nu, float center, int direction,
                                  float *sin_h, float *cos_h, float *startu_h);
mr_status mr_bp_circle_mask(size_t nx, size_t ny, int correcttilt, float tiltangle, size_t nslices,
                            uint32_t *mask_h);
mr_status mr_bp_parallel_tilt(float tiltangle, float tiltpivot, size_t roi_y0, float *tiltoffset,
                              float *tiltinc);
mr_status mr_bp_parallel(const void *proj_d, int dtype, const float *scale_d, const float *weight_d,
                         const int32_t *index_d, const float *sin_d, const float *cos_d, const float *startu_d,
                         size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d, int correcttilt, float tiltoffset,
                         float tiltinc, float *vol_d, void *stream);
/* The same backprojection with the projection rows of each 32 x 8 x 32 voxel tile staged in
 * shared memory by TMA (FP32, no tilt correction, row pitch a multiple of 16 bytes);
 * nslabs = number of projection slabs in proj_d (the bound of every TMA load). Other
 * requests run mr_bp_parallel. Results are bit-identical on both paths. */
mr_status mr_bp_parallel_staged(const void *proj_d, size_t nslabs, int dtype, const float *scale_d,
                                const float *weight_d, const int32_t *index_d, const float *sin_d, const float *cos_d,
                                const float *startu_d, size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d,
                                int correcttilt, float tiltoffset, float tiltinc, float *vol_d, void *stream);
/* mr_bp_parallel_staged for the volume rows y in [y_begin, y_end) only (vol_d is still the
 * whole [nu][nu][nv] volume; a row block is contiguous in it): used to copy finished row
 * blocks to the host while the next block is backprojected. Every voxel gets the value the
 * whole-volume call gives it. */
mr_status mr_bp_parallel_rows(const void *proj_d, size_t nslabs, int dtype, const float *scale_d,
                              const float *weight_d, const int32_t *index_d, const float *sin_d, const float *cos_d,
                              const float *startu_d, size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d,
                              int correcttilt, float tiltoffset, float tiltinc, size_t y_begin, size_t y_end,
                              float *vol_d, void *stream);
/* The factory's three parallel-beam backprojectors on the same kernels
 * (StdBackProjectors/src/StdBackProjectors.cpp:25-60), for the volume rows [y_begin, y_end):
 *   MR_BP_MULTIPROJ_PARALLEL  "MultiProjBPparallel" (MultiProjBPparallel.cpp:39-170): as
 *     mr_bp_parallel_rows;
 *   MR_BP_MULTIPROJ_SERIAL    "MultiProjBP" (MultiProjBP.cpp:36-146): the same without tilt
 *     correction; with it, u = ((startu_i + cos_i y) - sin_i x) - tiltoffset and the 4-slice
 *     group g takes the weight |(u - n) - g*tiltinc|;
 *   MR_BP_NEAREST             "NearestNeighborBP" (NNMultiProjBP.cpp:36-121): the same u (minus
 *     tiltoffset after the x term with tilt correction), vol[z] += P_i[z][n] with n = (int)u in
 *     [0, nu-2], no interpolation and no per-slice shift.
 * Results equal each reference module's bit for bit (FP32). */
enum { MR_BP_MULTIPROJ_PARALLEL = 0, MR_BP_MULTIPROJ_SERIAL = 1, MR_BP_NEAREST = 2 };
mr_status mr_bp_parallel_variant(int variant, const void *proj_d, size_t nslabs, int dtype, const float *scale_d,
                                 const float *weight_d, const int32_t *index_d, const float *sin_d, const float *cos_d,
                                 const float *startu_d, size_t nproj, size_t nu, size_t nv, const uint32_t *mask_d,
                                 int correcttilt, float tiltoffset, float tiltinc, size_t y_begin, size_t y_end,
                                 float *vol_d, void *stream);

/* ---------------------------------------------------------------------------------
 * FDK cone-beam backprojection: FDKbp_single
 * (frameworks/tomography/Backprojectors/FDKBackProjectors/src/fdkbp_single.cpp:83-994)
 * driven as FdkReconBase::Process 3D (fdkreconbase.cpp:217-277).
 *
 * Geometry as ReconConfig fields (ReconConfig.h): source-object / source-detector
 * distances, piercing point (detector pixels), centre of rotation, detector pitch,
 * voxel size; direction 0 = clockwise. The detector ROI is the full projection
 * (roi = projection_roi = {0, 0, nu, nv}) and the volume is nu x nu x nv. */
typedef struct {
    float sod, sdd;
    float ppoint[2];
    float center;
    float resolution[2];
    float voxelsize[3];
    int direction;
    int correcttilt;
    float tiltangle;
    float tiltpivot;
} mr_fdk_geom;

/* Per-projection partial projections (host, exact reference float arithmetic):
 * xip [nproj][nu][3], yip [nproj][nu][3], zip [nproj][nv][3] of
 * project_volume_onto_image_c (:293-445), and the image scale factors. *uniform_z is set
 * to 1 when, for every projection, zip[k][0] and zip[k][2] do not depend on k (always the
 * case without tilt correction), which lets the backprojector hoist the detector column
 * and the distance weight out of the slice loop. */
mr_status mr_fdk_partials(const mr_fdk_geom *g, size_t nu, size_t nv, const float *angles_h, size_t nproj,
                          float *xip_h, float *yip_h, float *zip_h, float *sad_sid_2, float *scale, int *uniform_z);
/* Ramp filter (ramp_filter_tuned, :832-958) of nproj projections [nproj][nv][nu] with
 * the input weighting of FdkReconBase::Process (img *= weight, :243) and the image
 * rescale of project_volume_onto_image_c (cbi *= sad_sid_2; cbi *= scale, :380-384)
 * fused. out_dtype MR_F32, or MR_BF16/MR_F16 with scale_out_d[nproj] written. */
mr_status mr_fdk_filter(const float *in_d, size_t nu, size_t nv, size_t nproj, const float *weight_d,
                        float sad_sid_2, float scale, int out_dtype, void *out_d, float *scale_out_d,
                        void *stream);
/* mr_fdk_filter on the detector rows [row0, row0 + nrows) of each projection only (in_d and
 * out_d hold [nproj][nrows][nu]): the rows a slab of slices projects onto (the CBCT row
 * window of ReconEngine's slice blocks, ReconEngine.cpp:954-1008). Each row equals the same
 * row of the whole-detector call; the edge-row replication of the reference (rows 0..4 copy
 * row 5, the last five copy row nv-6) refers to the absolute rows, so a window that reaches
 * those rows must also hold row 5 (row nv-6), else MR_ERR_ARGUMENT. Rows are transformed two
 * at a time (the real and imaginary parts of one complex FFT): with nv even, a window that
 * starts on an even row and holds an even number of rows keeps the whole detector's pairs and
 * its rows equal that call's bit for bit; other windows agree to FFT rounding. */
mr_status mr_fdk_filter_rows(const float *in_d, size_t nu, size_t nrows, size_t row0, size_t nv, size_t nproj,
                             const float *weight_d, float sad_sid_2, float scale, int out_dtype, void *out_d,
                             float *scale_out_d, void *stream);
/* Voxel-driven nearest-neighbour backprojection (:450-525) of nproj filtered
 * projections into the final volume (after FdkReconBase's per-slice mirror and z
 * reversal, fdkreconbase.cpp:259-270). vol_d [nv][nu][nu] is overwritten when
 * accumulate == 0, else added to (continuing a previous batch of projections).
 * xip/yip/zip: device copies of mr_fdk_partials. mask_d: mr_bp_circle_mask(nu, nu, ...). */
mr_status mr_fdk_backproject(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                             size_t nproj, const float *xip_d, const float *yip_d, const float *zip_d, int uniform_z,
                             const uint32_t *mask_d, int box_w, int box_h, int accumulate, float *vol_d, void *stream);
/* mr_fdk_backproject for the cbct_volume slices k in [k_begin, k_end) only (final volume
 * slices nv-1-k; vol_d is still the whole [nv][nu][nu] volume): the slice blocks
 * ReconEngine reconstructs one at a time (ReconEngine.cpp:954-1008), here used to copy
 * finished slabs to the host while the next slab is backprojected. Every voxel gets the
 * value the whole-volume call gives it. */
mr_status mr_fdk_backproject_slab(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                                  size_t nproj, const float *xip_d, const float *yip_d, const float *zip_d, int uniform_z,
                                  const uint32_t *mask_d, int box_w, int box_h, int accumulate, size_t k_begin,
                                  size_t k_end, float *vol_d, void *stream);
/* Shared-memory staging box for mr_fdk_backproject (host): the largest detector footprint
 * (columns box_w, rows box_h) of a 32 x 8 x 32 voxel tile over a sample of the geometry,
 * from the host copies of the partials. With box_w = box_h = 0, or when the projection
 * layout does not allow TMA (row pitch not a multiple of 16 bytes), or without uniform_z,
 * mr_fdk_backproject uses direct global loads; tiles whose footprint exceeds the box fall
 * back to direct loads for that projection. Results are identical on every path. */
mr_status mr_fdk_box(const float *xip_h, const float *yip_h, const float *zip_h, size_t nu, size_t nv, size_t nproj,
                     int dtype, int *box_w, int *box_h);

/* ---- FDK precision form (no counterpart in the reference's API; the geometry restates
 * FDKbp, the double-geometry variant of the cone-beam backprojector, fdkbp.cpp:83-640).
 *
 * Per-projection detector maps in FP64 (host): for voxel (i, j, k) of the nu x nu x nv grid
 * of project_volume_onto_image_c, with m = maps_h + 12 p,
 *   u = m[0] i + m[1] j + m[2] k + m[3],  v = m[4] i + m[5] j + m[6] k + m[7],
 *   w = m[8] i + m[9] j + m[10] k + m[11];
 * the voxel samples detector column floor(u/w + 0.5), row floor(v/w + 0.5) with weight
 * 1/w^2. The row window that sets the image centre is the float path's. */
mr_status mr_fdk_maps64(const mr_fdk_geom *g, size_t nu, size_t nv, const float *angles_h, size_t nproj,
                        double *maps_h);
/* Staging box of mr_fdk_backproject_fast from the FP64 maps (host). */
mr_status mr_fdk_box_maps(const double *maps_h, size_t nu, size_t nv, size_t nproj, int dtype, int *box_w, int *box_h);
/* Nearest-neighbour FDK backprojection of 16-bit filtered projections (MR_BF16 or MR_F16,
 * value = stored * scale_d[p], from mr_fdk_filter or mr_quantize) through the FP64 maps
 * (maps_d [nproj][12] double from mr_fdk_maps64, m[2] = m[10] = 0: no tilt correction), FP32
 * accumulation, into the final volume layout of mr_fdk_backproject. The detector coordinates
 * of each 32 x 8 x 32 voxel tile's origin are formed in FP64; the other voxels add FP32
 * offsets to them. Each weighted sample is one mixed-precision fma with the weight
 * 1/w^2 * scale rounded to the storage type.
 * Requires a TMA-compatible layout (row pitch a multiple of 16 bytes) and a box from
 * mr_fdk_box_maps; returns MR_ERR_UNSUPPORTED otherwise. Accuracy against the FP64
 * backprojection is reported by the tests and the benchmark, not bit-exact. */
mr_status mr_fdk_backproject_fast(const void *proj_d, int dtype, const float *scale_d, size_t nu, size_t nv,
                                  size_t nproj, const double *maps_d, const uint32_t *mask_d, int box_w, int box_h,
                                  int accumulate, float *vol_d, void *stream);
/* FP64 error oracle on the device: backprojection of FP32 filtered projections through the
 * FP64 maps with FP64 accumulation, for 1..16 output slices (indices into the final volume's
 * z); out_d [nslices][nu][nu] in the final layout. Restated on the CPU by the oracle. */
mr_status mr_fdk_backproject_f64(const float *proj_d, size_t nu, size_t nv, size_t nproj, const double *maps_d,
                                 const uint32_t *mask_d, const int *slices_d, size_t nslices, double *out_d,
                                 void *stream);

/* ---------------------------------------------------------------------------------
 * Slice serialisation to 16 bits: the slices ReconEngine::Serialize (frameworks/tomography/
 * Framework/ReconFramework/src/ReconEngine.cpp:576-700) writes through kipl::io::
 * WriteImageStack (core/kipl/kipl/include/io/io_stack.h:114-230) as TIFF16: ExtractSlice
 * (base/core/textractor.hpp:17-125) of plane XY (MatrixXYZ volumes, FDK) or YZ (MatrixZXY
 * volumes, parallel beam), then ImageCaster<unsigned short, float>::cast (base/core/
 * imagecast.hpp:33-52) with the gray interval [lo, hi]:
 *     out = unsigned short((min(max(v, lo), hi) - lo) * (float(65535) / (hi - lo)))
 * (float arithmetic, truncation; NaN gives 0). vol_d: the volume as a kipl TImage of dims
 * (d0, d1, d2), d0 fastest (MatrixXYZ: (nx, ny, nz); MatrixZXY: (nz, nx, ny)); slices
 * first .. first + count - 1 along the plane's slice axis (d2 for XY, d0 for YZ); roi_h:
 * NULL or (x0, y0, x1, y1), inclusive, over the slice's two axes; out_d [count][h][w]
 * uint16 with w, h the slice (or roi) size. Requires lo < hi and dims up to 65535. */
enum { MR_PLANE_XY = 1, MR_PLANE_YZ = 4 }; /* kipl::base::eImagePlanes values */
mr_status mr_slices_u16(const float *vol_d, int plane, size_t d0, size_t d1, size_t d2, size_t first, size_t count,
                        const size_t *roi_h, float lo, float hi, uint16_t *out_d, void *stream);

/* ---- Differentiable parallel-beam projector pair (the Joseph projector of
 * LinearForwardProjector::project, ReconAlgorithms/linearforwardprojector.cpp:15-144, and its
 * exact transpose; the reference has no adjoint and no multi-slice form).
 *
 * Volume [nz][n][n] (x fastest), projections [nproj][nz][nu] (detector bin fastest), angles
 * in degrees. Slice z uses the detector centre c_z = centre + tan_tilt * (z - pivot), in
 * detector bins; centre = nu/2 (integer division) and tan_tilt = 0 give the reference's
 * geometry. */
/* Per-angle parameters in FP64, rounded once to float: params_h [nproj][8]. */
mr_status mr_joseph_geometry(const float *angles_h, size_t nproj, size_t n, float *params_h);
/* proj_d = A(centre, tilt) vol_d; when dproj_d is not NULL it receives d proj / d centre.
 * volt_d: caller scratch of nz * n * n floats (the transposed slices). */
mr_status mr_joseph_forward(const float *vol_d, float *volt_d, size_t n, size_t nz, const float *params_d,
                            size_t nproj, size_t nu, float centre, float tan_tilt, float pivot, float *proj_d,
                            float *dproj_d, void *stream);
/* vol_d (=|+=) A^T proj_d: the exact transpose of mr_joseph_forward (same weights, same
 * sample set), voxel-driven. */
mr_status mr_joseph_adjoint(const float *proj_d, size_t n, size_t nz, const float *params_d, size_t nproj, size_t nu,
                            float centre, float tan_tilt, float pivot, int accumulate, float *vol_d, void *stream);
/* out_d[z] = sum over projections and bins of a_d * b_d for every slice z (FP64), e.g. the
 * centre derivative against a residual: d/d centre = sum_z out_d[z], d/d tan_tilt =
 * sum_z (z - pivot) out_d[z]. */
mr_status mr_slice_dot(const float *a_d, const float *b_d, size_t nproj, size_t nz, size_t nu, double *out_d,
                       void *stream);

/* ---- Differentiable pair matched to the parallel-beam backprojector (no counterpart in the
 * reference's API): mr_mbp_adjoint is MultiProjectionBPparallel's linear-interpolation
 * backprojection (MultiProjBPparallel.cpp:39-170, every projection, weight 1) with a detector
 * centre per slice, c_z = centre + tan_tilt (z - pivot); with tan_tilt = 0 it equals
 * mr_bp_parallel bit for bit. mr_mbp_forward is its exact transpose: each detector bin collects
 * the same weights of the same voxels, so <A x, p> = <x, A^T p> up to float summation.
 * Volume [n][n][nz] (MatrixZXY, z fastest; x, y in the circle mask of mr_bp_circle_mask(n, n, 0,
 * 0, nz)), projections [nproj][nz][n] (the detector is n bins wide, as the reference's
 * backprojector takes it). mr_mbp_geometry (host): sincos_h [nproj][2] = sin, cos of the
 * direction-signed angle and startu_h [nproj][nz] = (n/2)(sin - cos) + c_z, the reference's float
 * expressions. mr_mbp_forward also returns d proj / d c_z in dproj_d when it is not NULL. */
mr_status mr_mbp_geometry(const float *angles_h, size_t nproj, size_t n, size_t nz, float centre, float tan_tilt,
                          float pivot, int direction, float *sincos_h, float *startu_h);
mr_status mr_mbp_adjoint(const float *proj_d, size_t n, size_t nz, const float *sincos_d, const float *startu_d,
                         size_t nproj, const uint32_t *mask_d, int accumulate, float *vol_d, void *stream);
mr_status mr_mbp_forward(const float *vol_d, size_t n, size_t nz, const float *sincos_d, const float *startu_d,
                         size_t nproj, const uint32_t *mask_d, float *proj_d, float *dproj_d, void *stream);

/* Device-side error word of bounded waits inside kernels (0 = none); reading it
 * synchronizes the device and clears the word. */
mr_status mr_device_status(int *status);

/* Failure detection and tracing (no counterpart in the reference, whose engine wraps module
 * exceptions at each level, ReconEngine.cpp:810-833, and times modules with a CPU timer,
 * ProcessModuleBase.cpp:129-149).
 * mr_set_wait_limit: tries of each per-batch mbarrier wait in the TMA-staged backprojectors
 *   (default 4194304; a negative value restores it), read at each launch. A wait that runs
 *   out sets the device error word (mr_device_status returns 1), skips the rest of the block's
 *   projections, waits for the block's copies still in flight (with the default limit) and
 *   returns; the context stays usable. 0 makes every such wait expire at once.
 * mr_debug_fail_allocation: the scratch allocation made after `after` further successful ones
 *   fails with MR_ERR_ALLOCATION, once (a negative value disarms the hook). Process-wide.
 * mr_trace_push / mr_trace_pop: an NVTX range on the calling thread (the host modules put one
 *   around each Process; every entry point of this library opens one named after itself). */
/* ReconEngine::validateImage (ReconEngine.cpp:1724-1740) over kipl::algorithms::dataValidator
 * (datavalidator.h:8-19): counts_d[0] = NaNs and counts_d[1] = infinities (either sign) among
 * the n floats at data_d. counts_d (device, two values) is zeroed first; asynchronous. */
mr_status mr_data_validator(const float *data_d, size_t n, unsigned long long *counts_d, void *stream);
/* Bounds-checked build (libmrcuda_checked.so, compiled with -DMR_BOUNDS_CHECK; no counterpart in
 * the reference): the index checks at the gather sites of the backprojectors, the matched pair,
 * the ring cleaner and the MorphSpotClean worklist record the first failing site and index and
 * skip the access. *first = site << 40 | index of the first failure in any kernel since the last
 * call (0: none), and the record is cleared; the product build always reports 0. Synchronizes. */
mr_status mr_bounds_status(unsigned long long *first);
mr_status mr_set_wait_limit(int tries);
mr_status mr_debug_fail_allocation(long long after);
mr_status mr_trace_push(const char *name);
mr_status mr_trace_pop(void);

/* Diagnostics (no counterpart in the reference): the measured shared-memory load rate of the
 * current device, the on-chip roofline of the staged backprojectors, which gather one 32-bit
 * sample per lane from shared memory. A conflict-free kernel with many loads in flight,
 * timed with CUDA events on the legacy default stream (synchronous; allocates a few bytes).
 * wavefronts_per_s: shared-memory wavefronts served per second (a warp's conflict-free
 * 32-bit load is one wavefront); bytes_per_s = 128 bytes per wavefront. */
mr_status mr_measure_smem(double *wavefronts_per_s, double *bytes_per_s);

#ifdef __cplusplus
}
#endif
#endif /* MRCUDA_H */
