/* CPU restatement of the MuhRec reconstruction hot path (test infrastructure only).
 *
 * This is the oracle the CUDA path is checked against. It restates, in plain C, the
 * algorithms of the reference modules named beside each function (paths relative to the
 * reference project root). Only tests/, __graft_entry__.smoke() and the CPU-baseline leg
 * of bench.py may load it; the product library never links or calls it.
 *
 * Parity pinning: every function here is checked against the reference's own modules
 * compiled from source (oracle/ref, libmuhrec_ref.so) and against the reference's
 * golden vectors (tests/golden). Float arithmetic follows the reference's operation
 * order with no contraction (built with -ffp-contract=off), so results are bit-identical
 * where the reference is deterministic; FFTs run in FP64 (FFTW is not available).
 *
 * Layouts: projections [nproj][nv][nu] (u fastest), the kipl TImage<float,3> order.
 */
#ifndef MR_ORACLE_H
#define MR_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ImagingAlgorithms::AverageImage methods (averageimage.h:16-23) */
enum { ORC_AVG_SUM = 0, ORC_AVG_AVERAGE, ORC_AVG_MEDIAN, ORC_AVG_WEIGHTED, ORC_AVG_MIN, ORC_AVG_MAX };

int orc_average(const float *stack, size_t nu, size_t nv, size_t n, int method, float *out);
float orc_frame_dose(const float *frame, size_t nu, const size_t *roi);

/* FullLogNorm (StdPreprocModules/src/NormPlugins.cpp:300-552) */
void orc_lognorm_logflat(const float *dark, const float *flat, size_t npix, int ndc, float flatdose, float *logflat);
void orc_lognorm_doselog(const float *doses, size_t nproj, float darkdose, float *doselog);
void orc_lognorm_apply(float *proj, size_t npix, size_t nproj, const float *dark, const float *logflat,
                       const float *doselog, size_t ndose, int ndc, int nob);
void orc_log_lut(float *lut, float *param);
void orc_lognorm_apply_lut(float *proj, size_t npix, size_t nproj, const float *dark, const float *logflat,
                           const float *doselog, size_t ndose, int ndc, int nob);

/* ProjectionFilterSingle (StdPreprocModules/src/ProjectionFilter.cpp:120-376) */
enum { ORC_FILTER_RAMLAK = 0, ORC_FILTER_SHEPPLOGAN, ORC_FILTER_HANNING, ORC_FILTER_HAMMING, ORC_FILTER_BUTTERWORTH };
size_t orc_projfilter_size(size_t nu, int paddingdoubler);
int orc_projfilter_build(size_t nu, int filtertype, float cutoff, float order, int usebias, float biasweight,
                         int paddingdoubler, float *filter, float *pad, size_t *ninsert);
void orc_projfilter_apply(float *proj, size_t nu, size_t nrows, const float *filter, const float *pad,
                          size_t nfft, size_t ninsert);

/* MultiProjectionBPparallel through StdBackProjectorBase (StdBackProjectors/src/
 * StdBackProjectorBase.cpp:64-201, MultiProjBPparallel.cpp:39-170,
 * ReconFramework/src/BackProjectorModuleBase.cpp:153-218). vol: ZXY [nu][nu][nv]. */
int orc_bp_parallel(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
                    const float *weights, float center, int direction, size_t buffersize, int correcttilt,
                    float tiltangle, float tiltpivot, size_t roi_y0, size_t nslices, float *vol);
/* variant 0 MultiProjectionBPparallel, 1 the serial MultiProjectionBP, 2 NearestNeighborBP */
int orc_bp_parallel_variant(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles,
                            const float *weights, float center, int direction, size_t buffersize, int correcttilt,
                            float tiltangle, float tiltpivot, size_t roi_y0, size_t nslices, int variant, float *vol);

void orc_bp_geometry(const float *angles, size_t n, size_t nu, float center, int direction, float *fsin, float *fcos,
                     float *fstartu);
void orc_circle_mask(size_t nx, size_t ny, int correcttilt, float tiltangle, size_t nslices, size_t *mask);

/* The parallel-beam pair matched to MultiProjBPparallel (differentiation form). */
void orc_mbp_geometry(const float *angles, size_t nproj, size_t n, size_t nz, float centre, float tan_tilt,
                      float pivot, int direction, float *sc, float *su);
void orc_mbp_adjoint(const float *proj, size_t n, size_t nz, const float *sc, const float *su, size_t nproj,
                     const size_t *mask, float *vol);
void orc_mbp_forward64(const float *vol, size_t n, size_t nz, const float *angles, size_t nproj, double centre,
                       double tan_tilt, double pivot, int direction, const size_t *mask, int float_u, double *proj,
                       double *dproj);

/* FDKbp_single via FdkReconBase (FDKBackProjectors/src/fdkbp_single.cpp:83-994,
 * fdkreconbase.cpp:91-277). vol: XYZ [nv][nu][nu] after the final mirror. */
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
} orc_fdk_geom;
int orc_fdk(const float *proj, size_t nu, size_t nv, size_t nproj, const float *angles, const float *weights,
            const orc_fdk_geom *g, float *vol);
/* pieces of orc_fdk, exposed for kernel-level checks */
void orc_fdk_prepare(float *proj, size_t nu, size_t nv, size_t nproj, const float *weights, const orc_fdk_geom *g);
int orc_fdk_bp(const float *filtered, size_t nu, size_t nv, size_t nproj, const float *angles, const orc_fdk_geom *g,
               float *vol);
void orc_fdk_ramp(float *img, size_t width, size_t height);
void orc_fdk_projmatrix(const orc_fdk_geom *g, size_t nu, float angle, float *pm /*12*/);
/* FP64 error oracle: detector maps in double and the FP64 backprojection of listed slices */
void orc_fdk_maps64(const orc_fdk_geom *g, size_t nu, size_t nv, const float *angles, size_t nproj, double *maps);
void orc_fdk_bp64(const float *filtered, size_t nu, size_t nv, size_t nproj, const double *maps, const size_t *mask,
                  const int *slices, size_t nslices, double *out);

/* kipl morphology and MorphSpotClean (core/kipl/kipl/include/morphology/morphgeo.h,
 * morphextrema.h; core/algorithms/ImagingAlgorithms/src/MorphSpotClean.cpp). Images [h][w]. */
int orc_rec_dilation(const float *g, const float *f, size_t w, size_t h, int conn8, float *out);
void orc_rec_erosion(const float *g, const float *f, size_t w, size_t h, int conn8, float *out);
void orc_fill_hole(const float *img, size_t w, size_t h, int conn8, float *out);
int orc_fill_peaks(const float *img, size_t w, size_t h, int conn8, float *out);
void orc_fill_peaks_forward(const float *img, size_t w, size_t h, int conn8, float *out);
int orc_morphspotclean(float *img, size_t w, size_t h, int detect, int conn8, const float *th, const float *sigma,
                       size_t edge, int clamp, float minlevel, float maxlevel, int removeinfnan);

/* StripeFilter / WaveletRingClean (core/algorithms/ImagingAlgorithms/src/StripeFilter.cpp,
 * core/kipl/kipl/include/wavelets/core/wavelets.hpp). kern: analysis H, analysis G,
 * synthesis H, synthesis G, each end-begin+1 floats. Sinogram [ntheta][nu], in place. */
int orc_stripefilter(float *img, size_t nu, size_t ntheta, const float *kern, int begin, int end, int nlevels,
                     float sigma);

/* Joseph projector pair in FP64 (forward with its centre derivative, and the transpose) */
void orc_joseph_forward64(const float *vol, size_t n, size_t nz, const float *angles, size_t nproj, size_t nu,
                          double centre, double tan_tilt, double pivot, double *proj, double *dproj_dc);
void orc_joseph_adjoint64(const double *proj, size_t n, size_t nz, const float *angles, size_t nproj, size_t nu,
                          double centre, double tan_tilt, double pivot, double *vol);

/* Slice serialisation to 16 bits (ReconEngine::Serialize -> kipl::io::WriteImageStack). */
int orc_slices_u16(const float *vol, size_t d0, size_t d1, size_t d2, int plane, size_t first, size_t count,
                   const size_t *roi, float lo, float hi, unsigned short *out);

/* Alternative ring cleaners: kipl TMedianFilter<float,2> (odd kx, ky), BasicRingClean,
 * kipl SigmoidLUT (param: lo, hi, slope, intercept) and MedianMixRingClean. Images [h][w],
 * projections [n][h][w] in place. */
int orc_median_filter(const float *img, size_t w, size_t h, int kx, int ky, float *out);
int orc_basicringclean(float *proj, size_t w, size_t h, size_t n);
void orc_sigmoid_lut(size_t len, float lambda, float sigma, float *lut, float *param);
int orc_medianmixringclean(float *proj, size_t w, size_t h, size_t n, float threshold, float width);

/* SpotClean2 (ImagingAlgorithms::SpotClean): method 0 stddev, 1 ring, 2 median, 3 minmax,
 * 4 trikernel. Projections [n][h][w] in place, w, h >= 16. Returns -2 when the reference would
 * loop forever (a round with no spot next to an unmarked pixel). */
int orc_spotclean(float *proj, size_t w, size_t h, size_t n, int method, float gamma, float sigma, int iterations,
                  float minlevel, float maxlevel, int maxarea);

/* ComputeWeights (ReconHelpers.cpp:365-488): projection angles in acquisition order -> the
 * weighted projection map (angle, weight), in map order; returns its size. */
size_t orc_compute_weights(const float *angles, size_t n, float arc0, float arc1, int golden, float *out_angles,
                           float *out_weights);

#ifdef __cplusplus
}
#endif
#endif
