// Test infrastructure (oracle build only): a no-op stand-in for the logging
// library the reference's CurveBrute.cpp includes. Logging is not on the
// arithmetic path, so dropping it changes no result.
#pragma once
namespace spdlog {
template <class... A> inline void info(A&&...) {}
template <class... A> inline void warn(A&&...) {}
template <class... A> inline void error(A&&...) {}
template <class... A> inline void debug(A&&...) {}
}  // namespace spdlog
