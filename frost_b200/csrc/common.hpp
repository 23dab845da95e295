// Shared host-side helpers: status codes as exceptions inside the library,
// CUDA error checks, and the thread-local last-error message the C ABI
// reports. Exceptions never cross the extern "C" boundary (capi.cpp catches
// them), mirroring frost's "errors are exceptions" rule
// (docs/architecture.md:78-80, lib/cuda/gpu_utils.cuh:13-20).
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

#include <cuda_runtime_api.h>

#include "frost_b200.h"

namespace fb {

using SizeType  = std::size_t;
using IndexType = std::ptrdiff_t;

/** An error carrying one of the frost_status codes. */
class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), m_code(code) {}
    int code() const noexcept { return m_code; }

private:
    int m_code;
};

[[noreturn]] inline void invalid(const std::string& msg) {
    throw Error(FROST_ERR_INVALID_ARGUMENT, msg);
}

[[noreturn]] inline void fail_state(const std::string& msg) {
    throw Error(FROST_ERR_STATE, msg);
}

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        const int code = e == cudaErrorMemoryAllocation ? FROST_ERR_OUT_OF_MEMORY : FROST_ERR_DEVICE;
        throw Error(code, std::string(what) + " failed: " + cudaGetErrorString(e) + " (" + file +
                              ":" + std::to_string(line) + ")");
    }
}

#define FB_CUDA(call) ::fb::cuda_check((call), #call, __FILE__, __LINE__)

/** Lets kernel `fn` launch with up to the device's opt-in shared memory per
 * block. The attribute is process-wide state of the function: setting it to
 * each launch's own size would race between host threads launching the
 * same kernel with different sizes (served beams, batched cleaners), so it
 * is set once, to the largest value, per function and device. */
inline void allow_large_smem(const void* fn) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (done.count({fn, dev}) != 0)
        return;
    cudaFuncAttributes a{};
    FB_CUDA(cudaFuncGetAttributes(&a, fn));
    int optin = 0;
    FB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    FB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - static_cast<int>(a.sharedSizeBytes)));
    done.insert({fn, dev});
}
#define FB_LAUNCH_CHECK() ::fb::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

void set_last_error(const std::string& msg);

/** RAII device buffer (cudaMalloc/cudaFree) that grows on demand. */
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : m_ptr(o.m_ptr), m_bytes(o.m_bytes) {
        o.m_ptr   = nullptr;
        o.m_bytes = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            m_ptr     = o.m_ptr;
            m_bytes   = o.m_bytes;
            o.m_ptr   = nullptr;
            o.m_bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }

    /** Ensures at least `bytes` of storage; contents are not preserved. */
    void reserve(SizeType bytes) {
        if (bytes <= m_bytes)
            return;
        release();
        if (bytes == 0)
            return;
        void* p = nullptr;
        FB_CUDA(cudaMalloc(&p, bytes));
        m_ptr   = p;
        m_bytes = bytes;
    }
    void release() noexcept {
        if (m_ptr != nullptr)
            cudaFree(m_ptr);
        m_ptr   = nullptr;
        m_bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(m_ptr); }
    void* get() const { return m_ptr; }
    SizeType bytes() const { return m_bytes; }

private:
    void* m_ptr      = nullptr;
    SizeType m_bytes = 0;
};

/** RAII pinned host buffer. */
class PinnedBuffer {
public:
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { release(); }
    void reserve(SizeType bytes) {
        if (bytes <= m_bytes)
            return;
        release();
        void* p = nullptr;
        FB_CUDA(cudaMallocHost(&p, bytes));
        m_ptr   = p;
        m_bytes = bytes;
    }
    void release() noexcept {
        if (m_ptr != nullptr)
            cudaFreeHost(m_ptr);
        m_ptr   = nullptr;
        m_bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(m_ptr); }
    SizeType bytes() const { return m_bytes; }

private:
    void* m_ptr      = nullptr;
    SizeType m_bytes = 0;
};

/** Sets the calling thread's current device for a scope. */
class DeviceGuard {
public:
    explicit DeviceGuard(int device) {
        FB_CUDA(cudaGetDevice(&m_prev));
        if (m_prev != device)
            FB_CUDA(cudaSetDevice(device));
        m_set = m_prev != device;
    }
    ~DeviceGuard() {
        if (m_set)
            cudaSetDevice(m_prev);
    }

private:
    int m_prev = 0;
    bool m_set = false;
};

constexpr int bits_of(int dtype) {
    switch (dtype) {
    case FROST_UINT1: return 1;
    case FROST_UINT2: return 2;
    case FROST_UINT4: return 4;
    case FROST_UINT8: return 8;
    case FROST_UINT16: return 16;
    case FROST_UINT32: return 32;
    case FROST_FLOAT32: return 32;
    default: return 0;
    }
}

inline bool is_finite_bits32(uint32_t bits) { return (bits & 0x7F800000U) != 0x7F800000U; }
inline bool is_finite_bits64(uint64_t bits) {
    return (bits & 0x7FF0000000000000ULL) != 0x7FF0000000000000ULL;
}
bool is_finite(float x);
bool is_finite(double x);
inline bool is_positive_finite(float x) { return is_finite(x) && x > 0.0F; }
inline bool is_positive_finite(double x) { return is_finite(x) && x > 0.0; }

} // namespace fb
