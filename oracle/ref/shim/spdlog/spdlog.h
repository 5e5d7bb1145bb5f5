// spdlog-API shim (test infrastructure): the logging calls of the reference's
// src/prism/log.h (set_level, debug/info/warn/error/critical with fmt format
// strings), printed to stderr through fmt. The level starts at "off" unless the
// environment variable PRISM_REF_LOG names a level (debug, info, warn, error).
#pragma once

#include <fmt/format.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>

namespace spdlog {
namespace level {
enum level_enum { trace = 0, debug, info, warn, err, critical, off };
}

template <typename... Args>
using format_string_t = fmt::format_string<Args...>;

inline auto currentLevel() -> level::level_enum& {
    static level::level_enum lvl = [] {
        const char* e = std::getenv("PRISM_REF_LOG");
        if (e == nullptr) return level::off;
        if (std::strcmp(e, "debug") == 0) return level::debug;
        if (std::strcmp(e, "info") == 0) return level::info;
        if (std::strcmp(e, "warn") == 0) return level::warn;
        if (std::strcmp(e, "error") == 0) return level::err;
        return level::off;
    }();
    return lvl;
}

inline void set_level(level::level_enum l) {
    if (std::getenv("PRISM_REF_LOG") != nullptr) currentLevel() = l;
}

template <typename... Args>
void log(level::level_enum l, const char* tag, format_string_t<Args...> f, Args&&... args) {
    if (l < currentLevel()) return;
    std::fprintf(stderr, "[%s] %s\n", tag, fmt::format(f, std::forward<Args>(args)...).c_str());
}

template <typename... Args>
void debug(format_string_t<Args...> f, Args&&... args) {
    log(level::debug, "debug", f, std::forward<Args>(args)...);
}
template <typename... Args>
void info(format_string_t<Args...> f, Args&&... args) {
    log(level::info, "info", f, std::forward<Args>(args)...);
}
template <typename... Args>
void warn(format_string_t<Args...> f, Args&&... args) {
    log(level::warn, "warn", f, std::forward<Args>(args)...);
}
template <typename... Args>
void error(format_string_t<Args...> f, Args&&... args) {
    log(level::err, "error", f, std::forward<Args>(args)...);
}
template <typename... Args>
void critical(format_string_t<Args...> f, Args&&... args) {
    log(level::critical, "critical", f, std::forward<Args>(args)...);
}

} // namespace spdlog
