// Self-written stand-in for the few dmt backend types named by the
// reference's lib/prepare/device_rfi.hpp (dmt v0.8.0 is not vendored).
// No device code is built into the oracle; these only let the header parse.
#pragma once
#include <cstddef>
namespace dmt {
enum class Backend { kCPU, kCUDA, kHIP };
struct Stream { void* handle = nullptr; };
template <class T> struct DeviceSpan { T* ptr = nullptr; std::size_t n = 0; };
} // namespace dmt
