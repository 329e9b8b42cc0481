// Single-rank shim: range-v3 views::map mapped onto the C++20 standard view (oracle build only).
#pragma once

#include <ranges>

namespace ranges {
namespace views {
using namespace std::views;
}  // namespace views
using std::ranges::begin;
using std::ranges::end;
using std::ranges::size;
}  // namespace ranges
