// APSP summaries without any device allocation: ngx_apsp_noalloc.
//
// Some callers cannot allocate device memory while they run the metrics: a process whose caching allocator (torch's,
// for one) already holds nearly all of the GPU's memory, where a cudaMalloc fails or forces the cache to be emptied;
// and loops with a latency bound, where cudaFree would synchronize the whole device. For them this entry point runs
// the batched APSP tile kernel (the one ngx_apsp uses) with every device buffer - outputs, sources and the per-slot
// delta-stepping workspace - carved from one fixed array of NGX_NOALLOC_SCRATCH_BYTES defined in this file. The graph
// handle itself was allocated when it was created; this call allocates no device memory, and host memory only to build
// an error message.
//
// Because there is one array per device, calls that overlap on the same device (two host threads, or two handles on
// one device used at once) race on it and corrupt each other's results: serialize them.
//
// The array's device address is looked up on every call, with the graph's device current: the lookup allocates
// nothing, and a cached address would go stale if the caller reset the device (cudaDeviceReset) and the library's
// device code were loaded again at another address.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_run.h"

namespace ngx {
namespace {

constexpr size_t kScratchBytes = NGX_NOALLOC_SCRATCH_BYTES;
constexpr int64_t kChunk = 4096;  // sources staged per host -> device copy

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

size_t align256(size_t bytes) { return (bytes + 255) & ~size_t(255); }

// The device address of the current device's scratch array.
int scratch_address(void** out) {
    void* ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&ptr, g_scratch);
    if (err != cudaSuccess) {
        return cuda_fail(err, "ngx_apsp_noalloc: cudaGetSymbolAddress of the scratch array");
    }
    if ((reinterpret_cast<uintptr_t>(ptr) & 255u) != 0u) {
        return fail(NGX_CUDA_ERROR, "ngx_apsp_noalloc: the scratch array is not 256-byte aligned");
    }
    *out = ptr;
    return NGX_OK;
}

}  // namespace

int run_apsp_noalloc(ngx_graph* g, const ngx_apsp_opts* opts, ngx_apsp_result* result) {
    if (const int rc = check_opts(g, opts); rc != NGX_OK) {
        return rc;
    }
    if (result == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: result is NULL");
    }
    if (g->parts.size() != 1) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: this handle holds a batch of graphs");
    }
    if (opts->mode != NGX_MODE_BATCHED) {
        return fail(NGX_UNSUPPORTED, "ngx_apsp_noalloc: only the batched form runs from the fixed scratch array");
    }
    const int64_t n = g->n;
    const int64_t k = opts->sources != nullptr ? opts->num_sources : n;
    if (n > NGX_NOALLOC_MAX_VERTICES) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: the graph has " + std::to_string(n) + " vertices; at most " +
                                              std::to_string(NGX_NOALLOC_MAX_VERTICES) + " fit the fixed scratch array (use ngx_apsp)");
    }
    if (k < 0 || k > NGX_NOALLOC_MAX_SOURCES) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: num_sources must be in [0, " + std::to_string(NGX_NOALLOC_MAX_SOURCES) + "]");
    }
    const int64_t hist_bins = opts->hist_bins;
    const double hist_max = opts->hist_max;
    if (hist_bins > 0 && !(hist_max > 0.0)) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: hist_max must be > 0 when hist_bins > 0 (no automatic bound)");
    }
    for (int64_t i = 0; opts->sources != nullptr && i < k; ++i) {
        if (opts->sources[i] < 0 || opts->sources[i] >= n) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: source " + std::to_string(opts->sources[i]) + " out of range");
        }
    }
    clear_result_totals(result);
    if (k == 0 || n == 0) {
        result->cpl = result->efficiency = NAN;  // no reached pairs
        return NGX_OK;
    }
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    void* scratch = nullptr;
    if (const int rc = scratch_address(&scratch); rc != NGX_OK) {
        return rc;
    }
    *g->h_abort = 0;

    // Scratch layout: [zeroed: accumulators | counters | error | tile counter | histogram] [graph table] [sources]
    // [per-source outputs, when requested] [workspace slots]. Only the zeroed part must start at zero; the kernel
    // initialises its workspace slots itself.
    const bool per_f64 = result->src_sum != nullptr || result->src_max != nullptr || result->src_sum_inverse != nullptr;
    const bool per_u64 = result->src_unreachable != nullptr || result->src_arcs != nullptr;
    size_t off = 0;
    const auto take = [&](size_t bytes) {
        const size_t at = off;
        off += align256(bytes);
        return at;
    };
    const size_t a_acc = take(2 * kAccDigits * 8);
    const size_t a_cnt = take(kCounterCount * 8);
    const size_t a_err = take(8);
    const size_t a_tile = take(8);
    const size_t a_hist = take(static_cast<size_t>(std::max<int64_t>(hist_bins, 1)) * 8);
    const size_t zeroed = off;
    const size_t a_graph = take(sizeof(GraphDesc));
    const size_t a_src = take(static_cast<size_t>(k) * 4);
    const size_t a_f64 = per_f64 ? take(3 * static_cast<size_t>(k) * 8) : 0;
    const size_t a_u64 = per_u64 ? take(2 * static_cast<size_t>(k) * 8) : 0;
    if (off >= kScratchBytes) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_noalloc: outputs exceed the fixed scratch array");
    }
    char* base = static_cast<char*>(scratch);
    RunOutputs o;
    o.block = scratch;
    o.owned = false;
    o.bytes = off;
    o.zeroed_bytes = zeroed;
    o.acc = reinterpret_cast<unsigned long long*>(base + a_acc);
    o.counters = reinterpret_cast<unsigned long long*>(base + a_cnt);
    o.error = reinterpret_cast<int*>(base + a_err);
    o.tile_counter = reinterpret_cast<unsigned long long*>(base + a_tile);
    o.hist = reinterpret_cast<unsigned long long*>(base + a_hist);
    o.graphs = reinterpret_cast<GraphDesc*>(base + a_graph);
    o.sources = reinterpret_cast<int32_t*>(base + a_src);
    o.src_f64 = per_f64 ? reinterpret_cast<double*>(base + a_f64) : nullptr;
    o.src_u64 = per_u64 ? reinterpret_cast<unsigned long long*>(base + a_u64) : nullptr;
    o.num_graphs = 1;
    o.num_sources = k;

    const GraphPart& part = g->parts[0];
    const double delta = pick_delta(opts->metric == NGX_METRIC_INVERSE ? part.mean_len_inverse : part.mean_len_regular, opts->delta,
                                    default_delta_scale(part.n, part.m_stored));
    const GraphDesc desc{ part.n, part.m_stored, part.row_off, 0, k, part.vertex_off, delta };
    NGX_CUDA_TRY(cudaMemsetAsync(scratch, 0, zeroed, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(o.graphs, &desc, sizeof(desc), cudaMemcpyHostToDevice, g->stream));
    // sources: narrowed to 32 bits through a fixed host buffer, chunk by chunk
    int32_t staged[kChunk];
    for (int64_t first = 0; first < k; first += kChunk) {
        const int64_t count = std::min<int64_t>(kChunk, k - first);
        for (int64_t i = 0; i < count; ++i) {
            staged[i] = static_cast<int32_t>(opts->sources != nullptr ? opts->sources[first + i] : first + i);
        }
        NGX_CUDA_TRY(cudaMemcpyAsync(o.sources + first, staged, static_cast<size_t>(count) * 4, cudaMemcpyHostToDevice, g->stream));
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }

    TileJob job;
    job.num_graphs = 1;
    job.num_items = (k + kTile - 1) / kTile;
    job.d_items = nullptr;
    job.num_sources = k;
    job.n_max = n;
    job.plain_delta = delta;
    int rc = launch_apsp_in_workspace(g, opts, job, hist_bins, hist_max, o, base + off, kScratchBytes - off);
    const cudaError_t err = cudaStreamSynchronize(g->stream);
    if (rc != NGX_OK) {
        return rc;
    }
    if (err != cudaSuccess) {
        return cuda_fail(err, "ngx_apsp_noalloc: tile kernel");
    }
    int code = 0;
    NGX_CUDA_TRY(cudaMemcpyAsync(&code, o.error, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    unsigned long long acc[2 * kAccDigits];
    unsigned long long counters[kCounterCount];
    NGX_CUDA_TRY(cudaMemcpyAsync(acc, o.acc, sizeof(acc), cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(counters, o.counters, sizeof(counters), cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if ((rc = device_error_status(code)) != NGX_OK) {
        return rc;
    }
    if ((rc = collect_graph(g, o, acc, counters, 0, 0, k, hist_bins, hist_max, result)) != NGX_OK) {
        return rc;
    }
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return NGX_OK;
}

}  // namespace ngx

extern "C" {

int ngx_apsp_noalloc(ngx_graph* graph, const ngx_apsp_opts* opts, ngx_apsp_result* result) {
    return ngx::guard_host("ngx_apsp_noalloc", [&]() -> int { return ngx::run_apsp_noalloc(graph, opts, result); });
}

}  // extern "C"
