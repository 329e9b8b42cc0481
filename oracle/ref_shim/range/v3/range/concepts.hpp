// Single-rank shim: range-v3 range concepts mapped onto the C++20 standard ones (oracle build only).
#pragma once

#include <ranges>

namespace ranges {
using std::ranges::bidirectional_range;
using std::ranges::contiguous_range;
using std::ranges::forward_range;
using std::ranges::input_range;
using std::ranges::random_access_range;
using std::ranges::range;
using std::ranges::sized_range;
}  // namespace ranges
