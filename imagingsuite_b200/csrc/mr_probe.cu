// Measured on-chip roofline of the gather kernels: the shared-memory load rate of this GPU.
//
// The staged backprojectors read their samples from shared memory with one 32-bit load per
// lane (ld.shared.b32): a warp's load is served in one shared-memory wavefront when its lanes
// hit distinct banks (or the same word), more when they conflict. Their on-chip roofline is
// therefore the number of such wavefronts the SMs serve per second, measured here with a
// conflict-free pattern: every warp reads 32 consecutive words (one wavefront) with 8
// independent loads in flight per iteration, enough to keep the load pipe busy, so the
// kernel is bound by shared-memory wavefronts and not by issue or latency.
#include "mr_common.cuh"

namespace mr {

constexpr int kProbeWords = 8192; // 32 KiB of shared memory per block
constexpr int kProbeThreads = 1024;
constexpr int kProbeLoads = 8;

__global__ void __launch_bounds__(kProbeThreads) k_smem_probe(float *__restrict__ sink, int iters)
{
    __shared__ float buf[kProbeWords];
    for (int i = threadIdx.x; i < kProbeWords; i += kProbeThreads) buf[i] = static_cast<float>(i & 255);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float acc[kProbeLoads];
#pragma unroll
    for (int k = 0; k < kProbeLoads; ++k) acc[k] = 0.0f;
    // off stays below kProbeWords / kProbeLoads, so the k-th load is off + k * 1024 words: one
    // address update per iteration and immediate offsets for the loads
    constexpr int kSpan = kProbeWords / kProbeLoads;
    int off = (warp * 32 + lane) & (kSpan - 1);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < kProbeLoads; ++k) acc[k] += buf[off + k * kSpan];
        off = (off + 32) & (kSpan - 1);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kProbeLoads; ++k) s += acc[k];
    if (s == -1.0f) sink[blockIdx.x] = s; // never true (all values are >= 0); keeps the loads
}

} // namespace mr

using namespace mr;

extern "C" mr_status mr_measure_smem(double *wavefronts_per_s, double *bytes_per_s)
{
    MR_TRACE();
    if (!wavefronts_per_s || !bytes_per_s) return fail(MR_ERR_ARGUMENT, "mr_measure_smem: null pointer");
    int dev = 0, sms = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = 2 * sms; // two 1024-thread blocks per SM (64 warps)
    const int iters = 4096;
    float *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    mr_status st = MR_OK;
    float ms = 0.0f;
    if (cudaMalloc(&sink, blocks * sizeof(float)) != cudaSuccess) return fail(MR_ERR_ALLOCATION, "mr_measure_smem: sink");
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = fail(MR_ERR_CUDA, "events");
    for (int rep = 0; st == MR_OK && rep < 3; ++rep) { // the last of three launches is timed
        if (rep == 2) cudaEventRecord(e0, 0);
        k_smem_probe<<<blocks, kProbeThreads>>>(sink, iters);
        if (rep == 2) cudaEventRecord(e1, 0);
        st = check_launch("k_smem_probe");
    }
    if (st == MR_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        st = fail(MR_ERR_CUDA, "mr_measure_smem: timing");
    if (st == MR_OK) {
        const double wavefronts = static_cast<double>(blocks) * (kProbeThreads / 32) * iters * kProbeLoads;
        *wavefronts_per_s = wavefronts / (ms * 1e-3);
        *bytes_per_s = *wavefronts_per_s * 128.0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    return st;
}
