// Host-side state of a graph handle (private to the library).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "ngx_common.cuh"

struct ngx_graph {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;        // the stream all work of the graph is issued on
    cudaStream_t own_stream = nullptr;    // created with the graph; `stream` points here unless the caller set one

    int64_t n = 0;
    int64_t m_user = 0;    // arcs in the caller's CSR (zero weights included)
    int64_t m_stored = 0;  // arcs on the device (zero weights dropped)

    // Forward CSR over stored arcs; two arc arrays, one per metric (|w| and 1/|w|).
    int64_t* d_row_ptr = nullptr;
    ngx::Arc* d_arcs_regular = nullptr;
    ngx::Arc* d_arcs_inverse = nullptr;
    // Reverse CSR (in-arcs) with regular lengths; Arc::col is the arc's source, Arc::id its index in the stored forward CSR.
    int64_t* d_rrow_ptr = nullptr;
    ngx::Arc* d_rarcs = nullptr;

    double mean_len_regular = 1.0;
    double mean_len_inverse = 1.0;
    double min_len_regular = 1.0;
    double max_len_regular = 1.0;
    int64_t max_out_degree = 0;

    // Abort flag in mapped pinned host memory: the host sets it, kernels poll it between phases.
    int* h_abort = nullptr;
    int* d_abort = nullptr;

    uint64_t memory_budget = 0;

    // Cached device workspace, grown on demand and reused across runs.
    void* d_workspace = nullptr;
    size_t workspace_bytes = 0;

    ngx::DeviceCsr csr(int metric) const {
        return ngx::DeviceCsr{ n, m_stored, d_row_ptr, metric == NGX_METRIC_INVERSE ? d_arcs_inverse : d_arcs_regular };
    }
    ngx::DeviceCsr reverse_csr() const { return ngx::DeviceCsr{ n, m_stored, d_rrow_ptr, d_rarcs }; }
};

namespace ngx {

// Grows the graph's cached workspace to at least `bytes`.
int ensure_workspace(ngx_graph* g, size_t bytes);

// Bytes of device memory a run may use for workspaces (budget, or most of the free memory).
size_t workspace_budget(const ngx_graph* g);

}  // namespace ngx
