// Self-written stand-in for the psrio sample-type enum (psrio v0.5.0 is not
// vendored with the reference). Only the enumerators the reference's
// frost/common/policies.hpp maps to and from are declared. Test
// infrastructure: used only to compile the reference's CPU RFI sources.
#pragma once
#include <cstdint>
namespace psrio {
enum class SampleType : std::uint8_t {
    kUInt1,
    kUInt2,
    kUInt4,
    kUInt8,
    kUInt16,
    kUInt32,
    kFloat32,
    kInt8,
    kInt16,
};
} // namespace psrio
