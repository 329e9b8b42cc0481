// Host-side helpers shared by the APSP, Brandes and gradient runs (private to the library).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"

namespace ngx {

constexpr int64_t kMaxHistBins = 16384;

// Device buffers of one run's reduced outputs, carved from one allocation.
struct RunOutputs {
    unsigned long long* acc = nullptr;       // 2 * kAccDigits: exact sums of d and of 1/d
    unsigned long long* counters = nullptr;  // kCounterCount
    unsigned long long* hist = nullptr;
    double* src_f64 = nullptr;               // 3 * S: per-source sum, max, inverse sum
    unsigned long long* src_u64 = nullptr;   // 2 * S: per-source unreachable, traversed arcs
    double* rows = nullptr;                  // S * n distance rows, when requested
    int* error = nullptr;
    unsigned long long* tile_counter = nullptr;
    void* block = nullptr;
    size_t bytes = 0;
};

// Device buffers of the DAG passes: per-vertex betweenness and per-arc gradients in 128-bit fixed point.
struct DagOutputs {
    unsigned long long* bc = nullptr;        // 2 * n
    unsigned long long* grad_cpl = nullptr;  // 2 * m_user
    unsigned long long* grad_eff = nullptr;  // 2 * m_user
    unsigned long long* levels = nullptr;    // unused
    int* sigma_inexact = nullptr;            // device flag: a pushed sigma sum reached 2^53
    int sigma_pull = 0;                      // run the sigma pass in pull form
};

int check_opts(const ngx_graph* g, const ngx_apsp_opts* opts);
int run_apsp(ngx_graph* g, const ngx_apsp_opts* opts, ngx_apsp_result* result, double* rows, int tile_mode, DagOutputs* extra);
int prepare_sources(const ngx_graph* g, const ngx_apsp_opts* opts, std::vector<int32_t>& sources);
double pick_delta(const ngx_graph* g, int metric, double requested);
int alloc_outputs(ngx_graph* g, int64_t num_sources, int64_t hist_bins, bool want_rows, RunOutputs& o);
void free_outputs(ngx_graph* g, RunOutputs& o);
int device_error_status(int code);
int auto_hist_max(ngx_graph* g, const ngx_apsp_opts* opts, const std::vector<int32_t>& sources, double* out);
int collect(ngx_graph* g, const RunOutputs& o, int64_t num_sources, int64_t hist_bins, double hist_max, ngx_apsp_result* r);
void clear_result_totals(ngx_apsp_result* r);

}  // namespace ngx
