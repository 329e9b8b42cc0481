// Single-rank shim: the range-v3 comparison function objects the reference's utility headers name, mapped onto
// their C++20 standard-library equivalents (test infrastructure for the oracle build only).
#pragma once

#include <functional>

namespace ranges {
using std::ranges::equal_to;
using std::ranges::greater;
using std::ranges::greater_equal;
using std::ranges::less;
using std::ranges::less_equal;
using std::ranges::not_equal_to;
}  // namespace ranges
