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
    unsigned long long* acc = nullptr;       // per graph 2 * kAccDigits: exact sums of d and of 1/d
    unsigned long long* counters = nullptr;  // per graph kCounterCount
    unsigned long long* hist = nullptr;      // per graph hist_bins
    GraphDesc* graphs = nullptr;             // the run's graph table
    int32_t* sources = nullptr;              // all graphs' sources, graph after graph
    double* src_f64 = nullptr;               // 3 * S: per-source sum, max, inverse sum
    unsigned long long* src_u64 = nullptr;   // 2 * S: per-source unreachable, traversed arcs
    double* rows = nullptr;                  // S * n distance rows, when requested
    int* error = nullptr;
    unsigned long long* tile_counter = nullptr;
    void* block = nullptr;
    bool owned = true;                       // false: the graph's persistent buffer (CUDA graph replays)
    size_t bytes = 0;
    size_t zeroed_bytes = 0;                 // leading bytes (accumulators, counters, flags) reset before each run
    int64_t num_graphs = 0;
    int64_t num_sources = 0;
};

// What one launch covers: a graph table and sources already in the outputs block, and the work items.
struct TileJob {
    int64_t num_graphs = 1;
    int64_t num_items = 0;             // (graph, tile) work items
    const WorkItem* d_items = nullptr; // nullptr: tile t of graph 0
    int64_t num_sources = 0;
    int64_t n_max = 0;                 // largest graph (workspace slot size)
    double plain_delta = 1.0;          // bucket width of the plain form (single graph)
    bool track_reach = false;          // keep per-tile reach lists (a graph of several strongly connected components)
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
// Bucket width when the caller gives none, as a multiple of the mean arc length: 2 / sqrt(mean out-degree), clamped
// to 0.125-2. Dense graphs want narrow buckets (many arcs relax into each bucket: a wide one re-relaxes more pairs),
// sparse ones wide buckets (few arcs per bucket: a narrow one runs many nearly empty phases). Measured best widths:
// 0.15-0.25 x the mean at out-degree 100, 0.5 on a batch of out-degree 5-60, 1.0 or more at out-degree 6.
double default_delta_scale(int64_t n, int64_t m);
double pick_delta(double mean_len, double requested, double scale);
int alloc_outputs(ngx_graph* g, int64_t num_graphs, int64_t num_sources, int64_t hist_bins, bool want_rows, RunOutputs& o, bool persistent);
void free_outputs(ngx_graph* g, RunOutputs& o);
int device_error_status(int code);
int launch_tiles(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, const TileJob& job, int64_t hist_bins, double hist_max, RunOutputs& o,
                 DagOutputs* extra, float* kernel_ms, bool synchronous);
int launch_apsp_in_workspace(ngx_graph* g, const ngx_apsp_opts* opts, const TileJob& job, int64_t hist_bins, double hist_max, RunOutputs& o, void* ws,
                             size_t ws_bytes);
int read_totals(ngx_graph* g, const RunOutputs& o, std::vector<unsigned long long>& acc, std::vector<unsigned long long>& counters);
int collect_graph(ngx_graph* g, const RunOutputs& o, const unsigned long long* acc_all, const unsigned long long* counters_all, int64_t gi,
                  int64_t src_off, int64_t num_sources, int64_t hist_bins, double hist_max, ngx_apsp_result* r,
                  const int32_t* scatter = nullptr);
void clear_result_totals(ngx_apsp_result* r);

}  // namespace ngx
