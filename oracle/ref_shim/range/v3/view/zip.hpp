/*
 * Minimal stand-in for range-v3's views::zip, covering the single use in the reference's MPI wrapper
 * (external/mpi-wrapper/core/MPITypes.h:265: ranges::sort(ranges::views::zip(displacements, types))).
 * Test infrastructure for the oracle only.
 */
#pragma once

namespace ranges::views {
template <typename A, typename B>
struct zip_pair {
    A& first;
    B& second;
};

template <typename A, typename B>
[[nodiscard]] zip_pair<A, B> zip(A& a, B& b) {
    return { a, b };
}
} // namespace ranges::views
