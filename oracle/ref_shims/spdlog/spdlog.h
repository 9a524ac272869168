// Project-written no-op stand-in for the logging calls made by the reference's
// CPU tree path (spdlog is not installed here).  Logging has no effect on any
// computed value.
#pragma once

#define SPDLOG_TRACE(...) ((void)0)

namespace spdlog {

template <typename... Args>
inline void debug(Args&&...) {}
template <typename... Args>
inline void info(Args&&...) {}
template <typename... Args>
inline void warn(Args&&...) {}
template <typename... Args>
inline void error(Args&&...) {}

}  // namespace spdlog
