// Host-side state of a graph handle (private to the library).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "ngx_common.cuh"

namespace ngx {
// Allocator whose element construction without arguments leaves trivial types uninitialized: large host arrays that a
// parallel pass fills completely are then first touched (and paged in) by the threads that fill them.
template <typename T>
struct DefaultInitAllocator : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = DefaultInitAllocator<U>;
    };
    using std::allocator<T>::allocator;
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible_v<U>) {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using HostVector = std::vector<T, DefaultInitAllocator<T>>;

// Host view of one graph of a handle (a single-graph handle holds one; a batch handle holds many, concatenated).
struct GraphPart {
    int64_t n = 0;
    int64_t m_user = 0;         // the caller's arcs (zero weights included)
    int64_t m_stored = 0;       // device arcs (zero weights dropped)
    int64_t row_off = 0;        // start of its n + 1 row offsets in the concatenated row_ptr arrays
    int64_t user_arc_off = 0;   // start of its caller arcs in the concatenated arc numbering (gradients)
    int64_t vertex_off = 0;     // start of its vertices in concatenated per-vertex outputs (betweenness)
    double mean_len_regular = 1.0;
    double mean_len_inverse = 1.0;
};
}  // namespace ngx

struct ngx_graph {
    int device = 0;
    int sm_count = 0;
    size_t l2_bytes = 0;  // the device's L2 cache
    cudaStream_t stream = nullptr;        // the stream all work of the graph is issued on
    cudaStream_t own_stream = nullptr;    // created with the graph; `stream` points here unless the caller set one

    int64_t n = 0;         // vertices of the largest graph (workspace slots are sized for it)
    int64_t n_total = 0;   // vertices of all graphs
    int64_t m_user = 0;    // arcs in the caller's CSRs (zero weights included)
    int64_t m_stored = 0;  // arcs on the device (zero weights dropped)
    std::vector<ngx::GraphPart> parts;  // one per graph
    // batch work items (graph, tile) in scheduling order, on the device; built by ngx_batch_create
    void* d_items = nullptr;
    int64_t num_items = 0;

    // Forward CSR over stored arcs; two arc arrays, one per metric (|w| and 1/|w|).
    int64_t* d_row_ptr = nullptr;
    ngx::Arc* d_arcs_regular = nullptr;
    ngx::Arc* d_arcs_inverse = nullptr;
    // Reverse CSR (in-arcs) with regular lengths; Arc::col is the arc's source, Arc::id its index in the stored forward CSR.
    int64_t* d_rrow_ptr = nullptr;
    ngx::Arc* d_rarcs = nullptr;
    int32_t* d_arc_src = nullptr;  // source vertex (graph-local) of each stored forward arc
    int32_t* d_stored_of_user = nullptr;  // device build: stored index of each caller arc (-1 for zero weights)

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

    // CUDA graph of the last batch run (kernel + output resets), replayed while the run's configuration is unchanged
    void* graph_exec = nullptr;  // cudaGraphExec_t
    uint64_t graph_key = 0;
    void* d_persistent = nullptr;  // output buffers the captured graph writes
    size_t persistent_bytes = 0;

    // Grow-only output buffers of single-graph runs (summaries, per-source outputs; betweenness / gradient sums), so
    // that a run allocates nothing once they have reached their size: stream-ordered frees were measured to stall a
    // synchronizing call for hundreds of milliseconds while the pool returned memory.
    void* d_call_out = nullptr;
    size_t call_out_bytes = 0;
    void* d_call_dag = nullptr;
    size_t call_dag_bytes = 0;

    // bucket width per size class (floor(log2 n)), as a multiple of each graph's mean arc length (ngx_batch_autotune)
    double class_scale[64] = {};
    // launch shape and bucket width picked by ngx_graph_autotune, per task (APSP, Brandes, gradient); runs use them
    // for the options they leave at 0
    ngx_tuning tuned[3] = {};
    // stored forward index of each caller arc (-1 for zero weights), for ngx_graph_update_weights (a device-built
    // handle copies it from d_stored_of_user on first use)
    ngx::HostVector<int32_t> stored_of_user;
    // all-sources processing order of each graph (graph-local ids, graph after graph): clusters of nearby vertices,
    // so that the 32 sources of a tile reach most vertices in the same phases and share arc passes
    ngx::HostVector<int32_t> source_order;
    // strongly connected components of a single graph (ensure_components; 0 = not computed yet). When there are
    // several, the all-sources order keeps each component's sources together and tiles list the vertices they reach.
    int64_t scc_components = 0;   // -1: not known (the pre-pass gave up)
    bool order_grouped = false;
    int64_t scc_pass_cap = 0;     // SCC passes allowed (0 = no cap; the APSP pre-pass sets one)
    int64_t scc_passes = 0;

    ngx::DeviceCsr csr(int metric) const {
        return ngx::DeviceCsr{ n, m_stored, d_row_ptr, metric == NGX_METRIC_INVERSE ? d_arcs_inverse : d_arcs_regular };
    }
    ngx::DeviceCsr reverse_csr() const { return ngx::DeviceCsr{ n, m_stored, d_rrow_ptr, d_rarcs }; }
};

namespace ngx {

// Host form of a handle's graphs, concatenated graph after graph, before the upload.
struct HostGraphs {
    std::vector<GraphPart> parts;
    HostVector<int64_t> row_ptr;   // n + 1 global arc offsets per graph (graph i's at parts[i].row_off)
    HostVector<int64_t> rrow_ptr;  // the same for the reverse CSR
    HostVector<Arc> regular;       // stored arcs (zero weights dropped) with |w|, in caller order within each row
    HostVector<Arc> inverse;       // the same arcs with 1/|w|
    HostVector<Arc> rarcs;         // in-arcs per target, ascending source; col = source, id = stored forward index
    HostVector<int32_t> arc_src;   // graph-local source of each stored arc
    HostVector<int32_t> stored_of_user;  // stored index of each caller arc, -1 for zero weights
    HostVector<int32_t> source_order;    // locality order of each graph, graph after graph
    int64_t n_max = 0;
    int64_t n_total = 0;
    int64_t m_user = 0;
    int64_t max_out_degree = 0;
    double mean_len_regular = 1.0;
    double mean_len_inverse = 1.0;
    double min_len_regular = 1.0;
    double max_len_regular = 1.0;
};

// Validates `count` CSRs and builds their host form on up to `threads` host threads (0: the machine's cores). No
// CUDA calls. The result does not depend on the number of threads.
int build_host_graphs(const ngx_csr* csrs, int64_t count, int threads, HostGraphs* out);

// Validates and uploads `count` CSRs into one handle (concatenated device CSR + reverse CSR). A single graph is built
// on the device (build_graph_on_device) unless `on_host`; batches are built on host threads.
int create_graphs(const ngx_csr* csrs, int64_t count, int device, ngx_graph** out, bool on_host = false);

// Device build of one graph whose rows passed the host checks, into g (device, stream and sm_count already set).
int build_graph_on_device(const ngx_csr* csr, ngx_graph* g);

// The all-sources order of a single-graph handle, computed from its device arrays when a run first needs it.
int ensure_source_order(ngx_graph* g);

// The strongly connected components of a single-graph handle (ngx_scc on its device), counted once per handle.
int ensure_components(ngx_graph* g);

// Copies a device-built handle's stored index of every caller arc to the host (ngx_graph_update_weights needs it).
int ensure_stored_of_user(ngx_graph* g);

// Grows the graph's cached workspace to at least `bytes`.
int ensure_workspace(ngx_graph* g, size_t bytes);
// Grows *buf (capacity *cap) to at least `bytes`; contents are not kept. Frees the old buffer only after the stream
// is idle.
int grow_buffer(ngx_graph* g, void** buf, size_t* cap, size_t bytes);

// Bytes of device memory a run may use for workspaces (budget, or most of the free memory).
size_t workspace_budget(const ngx_graph* g);

}  // namespace ngx
