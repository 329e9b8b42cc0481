// A host CSR built by the library (loaded network files, contracted graphs): ngx_network of the C ABI.
#pragma once

#include <cstdint>
#include <vector>

struct ngx_network {
    int64_t n = 0;
    std::vector<int64_t> rank_nodes;  // vertices per rank
    std::vector<int64_t> row_ptr;     // n + 1
    std::vector<int32_t> col;         // global target ids, ascending within a row
    std::vector<double> w;            // weights (integers of the reference's 32-bit weight type), never 0
};
