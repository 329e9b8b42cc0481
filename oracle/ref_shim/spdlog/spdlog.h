/*
 * Minimal stand-in for spdlog's free logging functions used by the reference's file loader
 * (source/graph/FileLoader.cpp) and test main. Messages are formatted with {fmt} and written to stderr.
 * Test infrastructure for the oracle only.
 */
#pragma once

#include <fmt/format.h>

#include <cstdio>
#include <utility>

namespace spdlog {
namespace detail {
template <typename... Args>
void log(const char* level, fmt::format_string<Args...> format, Args&&... args) {
    const auto message = fmt::format(format, std::forward<Args>(args)...);
    std::fprintf(stderr, "[%s] %s\n", level, message.c_str());
}
} // namespace detail

template <typename... Args>
void info(fmt::format_string<Args...> format, Args&&... args) {
    detail::log("info", format, std::forward<Args>(args)...);
}
template <typename... Args>
void warn(fmt::format_string<Args...> format, Args&&... args) {
    detail::log("warning", format, std::forward<Args>(args)...);
}
template <typename... Args>
void error(fmt::format_string<Args...> format, Args&&... args) {
    detail::log("error", format, std::forward<Args>(args)...);
}
} // namespace spdlog
