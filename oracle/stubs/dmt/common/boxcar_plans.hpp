// Self-written stand-in for the dmt peak-finding enum named by the
// reference's include/frost/config/config.hpp:67-68 (dmt v0.8.0 is not
// vendored).
#pragma once
namespace dmt {
enum class PeakFindingMode { kContiguousPeakPerWidth, kContiguousPeakAcrossWidths, kAllAboveThreshold };
} // namespace dmt
