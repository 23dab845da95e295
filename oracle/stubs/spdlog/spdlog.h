// Self-written stand-in for the spdlog calls in the reference's
// lib/search/postprocess.cpp (warnings only; dropped here).
#pragma once
namespace spdlog {
template <class... A> inline void warn(A&&...) {}
template <class... A> inline void info(A&&...) {}
template <class... A> inline void debug(A&&...) {}
} // namespace spdlog
