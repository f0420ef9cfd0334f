// TMA and mbarrier helpers shared by the staged kernels (sm_100a): shared-memory addresses,
// mbarrier init / expect-tx / bounded wait, tiled 3-D TMA loads (no multicast), and the
// driver's tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>

namespace mr {
namespace tma {

constexpr int kWaitLimit = 1 << 22; // bounded mbarrier waits (iterations)

// Iteration limit of the staged kernels' per-batch waits, read by each launch (mr_set_wait_limit
// changes it; the waits that drain copies in flight after an expiry keep kWaitLimit).
inline std::atomic<int> g_batch_wait_limit{kWaitLimit};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; false when `limit` tries expired.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit = kWaitLimit)
{
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

// Tiled 3-D TMA load into this CTA's shared memory, completing on `bar`. x must be a
// multiple of 16 bytes / element size (the caller aligns it).
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
                 "r"(smem_addr(bar))
                 : "memory");
}

// Asynchronous 4-byte global -> shared copy (cp.async); when !valid nothing is read (src may
// be any mapped address) and dst receives zero.
__device__ __forceinline__ void copy4_zfill(float *dst, const float *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}

// Completes this thread's outstanding cp.async copies (a barrier then publishes them).
__device__ __forceinline__ void copy_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

inline PFN_cuTensorMapEncodeTiled encode_fn()
{
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    });
    return fn;
}

} // namespace tma
} // namespace mr
