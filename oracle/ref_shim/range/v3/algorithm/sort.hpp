/*
 * Minimal stand-in for range-v3's sort over a zipped pair of random-access ranges: sorts both ranges together,
 * lexicographically by (first, second), through an index permutation. Test infrastructure for the oracle only.
 */
#pragma once

#include <range/v3/view/zip.hpp>

#include <algorithm>
#include <cstddef>
#include <numeric>
#include <vector>

namespace ranges {
template <typename A, typename B>
void sort(views::zip_pair<A, B> zipped) {
    const auto n = static_cast<std::size_t>(std::size(zipped.first));
    auto order = std::vector<std::size_t>(n);
    std::iota(order.begin(), order.end(), std::size_t{ 0 });
    std::stable_sort(order.begin(), order.end(), [&](std::size_t l, std::size_t r) {
        if (zipped.first[l] < zipped.first[r]) {
            return true;
        }
        if (zipped.first[r] < zipped.first[l]) {
            return false;
        }
        return zipped.second[l] < zipped.second[r];
    });
    auto first_copy = std::vector<std::decay_t<decltype(zipped.first[0])>>(std::begin(zipped.first), std::end(zipped.first));
    auto second_copy = std::vector<std::decay_t<decltype(zipped.second[0])>>(std::begin(zipped.second), std::end(zipped.second));
    for (std::size_t i = 0; i < n; ++i) {
        zipped.first[i] = first_copy[order[i]];
        zipped.second[i] = second_copy[order[i]];
    }
}
} // namespace ranges
