// Single-rank shim: range-v3 range traits mapped onto the C++20 standard ones (oracle build only).
#pragma once

#include <ranges>

namespace ranges {
using std::ranges::iterator_t;
using std::ranges::range_difference_t;
using std::ranges::range_reference_t;
using std::ranges::range_value_t;
using std::ranges::sentinel_t;
}  // namespace ranges
