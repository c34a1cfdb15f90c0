// oceanlib-b200: host-side error types and RAII device/pinned buffers.
#pragma once

#include "../../include/ocean_b200.h"

#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <utility>

namespace ocean_b200 {

// A CUDA call failed.
struct DeviceError : std::runtime_error {
    cudaError_t code;
    DeviceError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

// A bounded device wait gave up (a persistent kernel's error word was set).
struct TimeoutError : std::runtime_error {
    TimeoutError() : std::runtime_error("device wait timed out") {}
};

inline void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        // Reset the runtime's last-error slot, so a later launch's
        // cudaGetLastError reports that launch and not this failure (sticky
        // errors that poison the context stay set regardless).
        cudaGetLastError();
        throw DeviceError(e, what);
    }
}

inline ocean_status status_of(const DeviceError& e)
{
    return e.code == cudaErrorMemoryAllocation ? OCEAN_ERROR_OUT_OF_MEMORY : OCEAN_ERROR_DEVICE;
}

// Maps the exceptions of a host call to ocean_status (no exception may cross
// the C boundary).
template <typename Fn>
ocean_status guarded(Fn&& fn)
{
    try {
        fn();
        return OCEAN_OK;
    } catch (const std::invalid_argument&) {
        return OCEAN_ERROR_INVALID_ARG;
    } catch (const TimeoutError&) {
        return OCEAN_ERROR_TIMEOUT;
    } catch (const DeviceError& e) {
        return status_of(e);
    } catch (const std::bad_alloc&) {
        return OCEAN_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return OCEAN_ERROR_UNKNOWN;
    }
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) : n(count)
    {
        if (count) check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
        return *this;
    }
    ~DevBuf() { if (p) cudaFree(p); }
};

template <typename T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    HostBuf() = default;
    explicit HostBuf(size_t count, bool zero = true) : n(count)
    {
        if (count) check(cudaMallocHost(&p, count * sizeof(T)), "cudaMallocHost");
        if (p && zero) std::memset(p, 0, count * sizeof(T));
    }
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    HostBuf(HostBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    HostBuf& operator=(HostBuf&& o) noexcept
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
        return *this;
    }
    ~HostBuf() { if (p) cudaFreeHost(p); }
};

}  // namespace ocean_b200
