// Shared pieces of the MuhRec plugin libraries (libB200PreprocModules.so,
// libB200BackProjectors.so): device buffers, the CUDA stream of a module instance, and the
// translation of mrcuda status codes into the framework's ReconException.
//
// The plugins are compiled against the MuhRec framework headers (ReconFramework,
// ModuleConfig, kipl, ImagingAlgorithms) and resolve those libraries' symbols from the
// process that loads them, as MuhRec's own module libraries do: ReconEngine has them loaded
// before it opens a module library with dlopen. All device work goes through libmrcuda.so's C
// ABI (include/mrcuda.h).
#ifndef B200_PLUGIN_COMMON_H
#define B200_PLUGIN_COMMON_H

#include <cuda_runtime.h>

#include <cstddef>
#include <sstream>
#include <string>
#include <vector>

#include <ReconException.h>
#include <base/timage.h>

#include "mrcuda.h"

namespace b200 {

// mrcuda status -> ReconException with the library's message (the framework's error type,
// which ReconEngine catches and re-raises with its context).
inline void check(mr_status st, const char *what)
{
    if (st != MR_OK) {
        std::ostringstream msg;
        msg << what << ": " << mr_last_error() << " (" << mr_status_string(st) << ")";
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
}

inline void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        std::ostringstream msg;
        msg << what << ": " << cudaGetErrorString(e);
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
}

// A device array that grows on demand and is released with its owner (one per module
// instance: the engine reuses a module for every block, so the memory is allocated once).
template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    ~DeviceArray() { release(); }

    T *get(size_t count)
    {
        if (count > capacity_) {
            release();
            cuda_check(cudaMalloc(reinterpret_cast<void **>(&ptr_), count * sizeof(T) + 16), "device allocation");
            capacity_ = count;
        }
        return ptr_;
    }
    T *data() const { return ptr_; }
    size_t capacity() const { return capacity_; }
    void release()
    {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        capacity_ = 0;
    }

private:
    T *ptr_ = nullptr;
    size_t capacity_ = 0;
};

// The module instance's stream, created on first use (construction of a module, e.g. by
// GetModuleList, touches no device).
class Stream {
public:
    Stream() = default;
    Stream(const Stream &) = delete;
    Stream &operator=(const Stream &) = delete;
    ~Stream()
    {
        if (s_) cudaStreamDestroy(s_);
    }
    cudaStream_t get()
    {
        if (!s_) cuda_check(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "stream creation");
        return s_;
    }
    void sync() { cuda_check(cudaStreamSynchronize(get()), "stream synchronisation"); }

private:
    cudaStream_t s_ = nullptr;
};

template <typename T>
inline void upload(T *dst_d, const T *src_h, size_t count, cudaStream_t s)
{
    cuda_check(cudaMemcpyAsync(dst_d, src_h, count * sizeof(T), cudaMemcpyHostToDevice, s), "host to device copy");
}

template <typename T>
inline void download(T *dst_h, const T *src_d, size_t count, cudaStream_t s)
{
    cuda_check(cudaMemcpyAsync(dst_h, src_d, count * sizeof(T), cudaMemcpyDeviceToHost, s), "device to host copy");
}

// NVTX range over a module call (mr_trace_push / mr_trace_pop of mrcuda): the engine's
// per-module timer (ProcessModuleBase.cpp:129-149) as a range on the profiler's timeline.
class Trace {
public:
    explicit Trace(const char *name) { mr_trace_push(name); }
    ~Trace() { mr_trace_pop(); }
    Trace(const Trace &) = delete;
    Trace &operator=(const Trace &) = delete;
};

// Bounded device waits report through mrcuda's error word; a set word becomes an exception.
inline void check_device(const char *what)
{
    int status = 0;
    check(mr_device_status(&status), what);
    if (status != 0) {
        std::ostringstream msg;
        msg << what << ": a kernel reported error status " << status;
        throw ReconException(msg.str(), __FILE__, __LINE__);
    }
}

} // namespace b200

#endif
