// Project-written stand-in for spdlog (oracle build only). The reference logs
// progress through rainbow-core/logs/detail/log.hpp:13-35; logging is off the
// arithmetic path, so every call here is a no-op.
#pragma once

namespace spdlog {
template <typename F, typename... A> inline void debug(const F&, const A&...) {}
template <typename F, typename... A> inline void info(const F&, const A&...) {}
template <typename F, typename... A> inline void warn(const F&, const A&...) {}
template <typename F, typename... A> inline void error(const F&, const A&...) {}
} // namespace spdlog
