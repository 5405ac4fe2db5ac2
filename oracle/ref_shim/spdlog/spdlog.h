// Logging stand-in for building the reference's headers in the oracle harness: every call is a
// no-op, so the harness needs no spdlog/fmt installation.
#pragma once
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <numeric>
#include <string>
#include <vector>
namespace spdlog {
template <typename... A> inline void info(A &&...) {}
template <typename... A> inline void warn(A &&...) {}
template <typename... A> inline void error(A &&...) {}
template <typename... A> inline void debug(A &&...) {}
}  // namespace spdlog
