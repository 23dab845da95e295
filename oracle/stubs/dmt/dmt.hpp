// Self-written stand-in for dmt's umbrella header as the reference's
// lib/search/subband_dedup.cpp:9 uses it: the dispersion constant only.
// Its value in dmt v0.8.0 is not available here (dmt is not vendored); the
// oracle and this build both take 4.148808e3 s MHz^2 cm^3 / pc as a double.
#pragma once
#include <dmt/common/candidate.hpp>
namespace dmt {
inline constexpr double kDispConst = 4.148808e3;
} // namespace dmt
