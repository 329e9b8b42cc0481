// Host side of the all-sources APSP run: source tiling, workspace sizing, launch, result reduction.
//
// Replaces AllPairsShortestPath::compute_apsp_impl's per-source loop (source/metrics/paths/AllPairsShortestPath.h:110-163)
// and compute_apsp_impl_delta_stepping (:197-247) with one persistent launch over all source tiles.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_run.h"
#include "sssp_kernels.cuh"

namespace ngx {

namespace {
constexpr int kBatchedUnroll = 4;
constexpr int kPlainWarpsMax = 16;
constexpr int kBatchedDefaultBlock = 384;
}  // namespace

int prepare_sources(const ngx_graph* g, const ngx_apsp_opts* opts, std::vector<int32_t>& sources) {
    if (opts->sources == nullptr) {
        sources.resize(static_cast<size_t>(g->n));
        for (int64_t i = 0; i < g->n; ++i) {
            sources[static_cast<size_t>(i)] = static_cast<int32_t>(i);
        }
        return NGX_OK;
    }
    if (opts->num_sources < 0) {
        return fail(NGX_INVALID_ARGUMENT, "num_sources is negative");
    }
    sources.resize(static_cast<size_t>(opts->num_sources));
    for (int64_t i = 0; i < opts->num_sources; ++i) {
        const int64_t s = opts->sources[i];
        if (s < 0 || s >= g->n) {
            return fail(NGX_INVALID_ARGUMENT, "source " + std::to_string(s) + " is out of range");
        }
        sources[static_cast<size_t>(i)] = static_cast<int32_t>(s);
    }
    return NGX_OK;
}

double pick_delta(const ngx_graph* g, int metric, double requested) {
    if (requested > 0.0 && std::isfinite(requested)) {
        return requested;
    }
    const double mean = metric == NGX_METRIC_INVERSE ? g->mean_len_inverse : g->mean_len_regular;
    return mean > 0.0 && std::isfinite(mean) ? mean : 1.0;
}

int check_opts(const ngx_graph* g, const ngx_apsp_opts* opts) {
    if (g == nullptr || opts == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "graph or opts is NULL");
    }
    if (opts->metric != NGX_METRIC_REGULAR && opts->metric != NGX_METRIC_INVERSE) {
        return fail(NGX_INVALID_ARGUMENT, "unknown metric");
    }
    if (opts->mode != NGX_MODE_BATCHED && opts->mode != NGX_MODE_PLAIN) {
        return fail(NGX_INVALID_ARGUMENT, "unknown mode");
    }
    if (opts->hist_bins < 0 || opts->hist_bins > kMaxHistBins) {
        return fail(NGX_INVALID_ARGUMENT, "hist_bins must be in [0, " + std::to_string(kMaxHistBins) + "]");
    }
    if (opts->block_threads != 0 && (opts->block_threads < 64 || opts->block_threads > 512 || opts->block_threads % 32 != 0)) {
        return fail(NGX_INVALID_ARGUMENT, "block_threads must be a multiple of 32 in [64, 512]");
    }
    return NGX_OK;
}

int alloc_outputs(ngx_graph* g, int64_t num_sources, int64_t hist_bins, bool want_rows, RunOutputs& o) {
    const size_t s = static_cast<size_t>(num_sources);
    size_t off = 0;
    const auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~size_t(255);
        return at;
    };
    const size_t a_acc = take(2 * kAccDigits * 8);
    const size_t a_cnt = take(kCounterCount * 8);
    const size_t a_err = take(8);
    const size_t a_tile = take(8);
    const size_t a_hist = take(static_cast<size_t>(std::max<int64_t>(hist_bins, 1)) * 8);
    const size_t a_f64 = take(3 * s * 8);
    const size_t a_u64 = take(2 * s * 8);
    const size_t a_rows = want_rows ? take(s * static_cast<size_t>(g->n) * 8) : 0;
    NGX_CUDA_TRY(cudaMallocAsync(&o.block, off, g->stream));
    o.bytes = off;
    char* b = static_cast<char*>(o.block);
    o.acc = reinterpret_cast<unsigned long long*>(b + a_acc);
    o.counters = reinterpret_cast<unsigned long long*>(b + a_cnt);
    o.error = reinterpret_cast<int*>(b + a_err);
    o.tile_counter = reinterpret_cast<unsigned long long*>(b + a_tile);
    o.hist = reinterpret_cast<unsigned long long*>(b + a_hist);
    o.src_f64 = reinterpret_cast<double*>(b + a_f64);
    o.src_u64 = reinterpret_cast<unsigned long long*>(b + a_u64);
    o.rows = want_rows ? reinterpret_cast<double*>(b + a_rows) : nullptr;
    NGX_CUDA_TRY(cudaMemsetAsync(o.block, 0, a_f64, g->stream));
    return NGX_OK;
}

void free_outputs(ngx_graph* g, RunOutputs& o) {
    if (o.block != nullptr) {
        cudaFreeAsync(o.block, g->stream);
        o.block = nullptr;
    }
}

int device_error_status(int code) {
    switch (code) {
    case kDevOk: return NGX_OK;
    case kDevTimeout: return fail(NGX_TIMEOUT, "a source tile exceeded max_iterations delta-stepping phases");
    case kDevAborted: return fail(NGX_ABORTED, "run aborted by ngx_graph_request_abort");
    default: return fail(NGX_CUDA_ERROR, "unknown device error code " + std::to_string(code));
    }
}

template <int kMode>
const void* tile_kernel_for_block(int block) {
    switch (block) {
    case 256: return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 256, 3>);
    case 384: return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 384, 2>);
    case 512: return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 512, 2>);
    default: return nullptr;
    }
}

// One persistent launch over `sources` (tile order): SSSP with the fused APSP epilogue, plus Brandes or the adjoint
// when `tile_mode` asks for them (batched form only). Leaves reduced outputs in `o` and the DAG outputs in `extra`.
int launch_tiles(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, const int32_t* d_sources, int64_t num_sources, int64_t hist_bins,
                 double hist_max, RunOutputs& o, DagOutputs* extra, float* kernel_ms) {
    const bool batched = opts->mode == NGX_MODE_BATCHED || tile_mode != kModeApsp;
    const int width = batched ? kTile : 1;
    const int64_t num_tiles = batched ? (num_sources + kTile - 1) / kTile : num_sources;
    const int block = opts->block_threads > 0 ? opts->block_threads : (batched ? kBatchedDefaultBlock : 512);
    const size_t acc_bytes = static_cast<size_t>(2) * (batched ? kTile : kPlainWarpsMax) * kAccDigits * 8;
    const size_t smem = acc_bytes + static_cast<size_t>(hist_bins) * 4;

    const void* kernel = reinterpret_cast<const void*>(&sssp_plain_kernel);
    if (batched) {
        kernel = tile_mode == kModeBrandes ? tile_kernel_for_block<kModeBrandes>(block)
                 : tile_mode == kModeGrad  ? tile_kernel_for_block<kModeGrad>(block)
                                           : tile_kernel_for_block<kModeApsp>(block);
        if (kernel == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "batched mode supports block_threads 256, 384 or 512");
        }
    }
    NGX_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int per_sm = 0;
    NGX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
    if (per_sm <= 0) {
        return fail(NGX_UNSUPPORTED, "kernel does not fit on an SM with this block size and histogram");
    }
    if (opts->ctas_per_sm > 0) {
        per_sm = std::min(per_sm, opts->ctas_per_sm);
    }
    const size_t slot_bytes = sssp_slot_bytes(g->n, width) + (tile_mode != kModeApsp ? brandes_slot_bytes(g->n, tile_mode == kModeGrad) : 0);
    const size_t budget = workspace_budget(g);
    int64_t slots = std::min<int64_t>(num_tiles, static_cast<int64_t>(g->sm_count) * per_sm);
    slots = std::min<int64_t>(slots, static_cast<int64_t>(budget / slot_bytes));
    if (slots <= 0) {
        return fail(NGX_OUT_OF_MEMORY, "not enough device memory for one workspace slot (" + std::to_string(slot_bytes) + " bytes)");
    }
    if (const int rc = ensure_workspace(g, static_cast<size_t>(slots) * slot_bytes); rc != NGX_OK) {
        return rc;
    }
    const int64_t n = g->n;
    char* ws = static_cast<char*>(g->d_workspace);
    SsspParams p{};
    p.g = g->csr(opts->metric);
    p.sources = d_sources;
    p.num_sources = num_sources;
    p.num_tiles = num_tiles;
    p.delta = pick_delta(g, opts->metric, opts->delta);
    p.max_iterations = opts->max_iterations > 0 ? opts->max_iterations : static_cast<unsigned long long>(4 * n + 64);
    p.tile_counter = o.tile_counter;
    p.error = o.error;
    p.abort_flag = g->d_abort;
    p.ws_dist = reinterpret_cast<unsigned long long*>(ws);
    ws += static_cast<size_t>(slots) * n * width * 8;
    p.ws_pend = reinterpret_cast<uint32_t*>(ws);
    ws += static_cast<size_t>(slots) * 2 * n * 4;
    p.ws_far = reinterpret_cast<uint32_t*>(ws);
    ws += static_cast<size_t>(slots) * n * 4;
    p.ws_queue = reinterpret_cast<int32_t*>(ws);
    ws += static_cast<size_t>(slots) * 2 * n * 4;
    p.ws_stamp = reinterpret_cast<uint32_t*>(ws);
    ws += static_cast<size_t>(slots) * n * 4;
    BrandesParams bp{};
    if (tile_mode != kModeApsp) {
        const size_t nt = static_cast<size_t>(n) * kTile;
        ws = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(ws) + 255) & ~uintptr_t(255));
        bp.rg = g->reverse_csr();
        bp.ws_sigma = reinterpret_cast<double*>(ws);
        ws += static_cast<size_t>(slots) * nt * 8;
        bp.ws_delta = reinterpret_cast<double*>(ws);
        ws += static_cast<size_t>(slots) * nt * 8;
        if (tile_mode == kModeGrad) {
            bp.ws_delta_g = reinterpret_cast<double*>(ws);
            ws += static_cast<size_t>(slots) * nt * 8;
        }
        bp.ws_cnt = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * nt * 4;
        bp.ws_lvl = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * nt * 4;
        bp.ws_list = reinterpret_cast<int32_t*>(ws);
        ws += static_cast<size_t>(slots) * nt * 4;
        bp.ws_loff = reinterpret_cast<int32_t*>(ws);
        ws += static_cast<size_t>(slots) * static_cast<size_t>(n + 2) * 4;
        bp.ws_scnt = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * nt * 4;
        bp.ws_soff = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * (nt + 1) * 4;
        // list entries pack (vertex << 5 | source) into 32 bits; larger graphs use the arc-scanning passes
        bp.succ_capacity = n < (int64_t(1) << 26) ? static_cast<int64_t>(nt) * kSuccPerPair : 0;
        bp.ws_succ = reinterpret_cast<uint32_t*>(ws);
        if (extra != nullptr) {
            bp.bc = extra->bc;
            bp.grad_cpl = extra->grad_cpl;
            bp.grad_eff = extra->grad_eff;
            bp.levels = extra->levels;
            bp.sigma_inexact = extra->sigma_inexact;
            bp.sigma_pull = extra->sigma_pull;
        }
    }
    p.out.acc_sum = o.acc;
    p.out.acc_inv = o.acc + kAccDigits;
    p.out.counters = o.counters;
    p.out.hist = hist_bins > 0 ? o.hist : nullptr;
    p.out.hist_bins = static_cast<int>(hist_bins);
    p.out.hist_max = hist_max;
    p.out.hist_width = hist_bins > 0 ? hist_max / static_cast<double>(hist_bins) : 0.0;
    p.out.src_sum = o.src_f64;
    p.out.src_max = o.src_f64 + num_sources;
    p.out.src_inv = o.src_f64 + 2 * num_sources;
    p.out.src_unreach = o.src_u64;
    p.out.src_arcs = o.src_u64 + num_sources;
    p.out.rows = o.rows;

    cudaEvent_t start, stop;
    NGX_CUDA_TRY(cudaEventCreate(&start));
    NGX_CUDA_TRY(cudaEventCreate(&stop));
    cudaEventRecord(start, g->stream);
    if (batched) {
        void* args[] = { &p, &bp };
        const cudaError_t launch = cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(slots)), dim3(block), args, smem, g->stream);
        if (launch != cudaSuccess) {
            cudaEventDestroy(start);
            cudaEventDestroy(stop);
            return cuda_fail(launch, "sssp kernel launch");
        }
    } else {
        sssp_plain_kernel<<<static_cast<unsigned>(slots), block, smem, g->stream>>>(p);
    }
    cudaError_t err = cudaGetLastError();
    cudaEventRecord(stop, g->stream);
    if (err == cudaSuccess) {
        err = cudaEventSynchronize(stop);
    }
    float ms = 0.0f;
    if (err == cudaSuccess) {
        cudaEventElapsedTime(&ms, start, stop);
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    if (err != cudaSuccess) {
        return cuda_fail(err, "sssp kernel");
    }
    if (kernel_ms != nullptr) {
        *kernel_ms += ms;
    }
    int code = 0;
    NGX_CUDA_TRY(cudaMemcpy(&code, o.error, sizeof(int), cudaMemcpyDeviceToHost));
    return device_error_status(code);
}

// Histogram bound when the caller gives none: 1.5 x the largest eccentricity of up to one tile of sources spread
// over the requested list (plus the overflow count for anything beyond it).
int auto_hist_max(ngx_graph* g, const ngx_apsp_opts* opts, const std::vector<int32_t>& sources, double* out) {
    const int64_t k = std::min<int64_t>(kTile, static_cast<int64_t>(sources.size()));
    std::vector<int32_t> sample(static_cast<size_t>(k));
    for (int64_t i = 0; i < k; ++i) {
        sample[static_cast<size_t>(i)] = sources[static_cast<size_t>(i * static_cast<int64_t>(sources.size()) / k)];
    }
    int32_t* d_sample = nullptr;
    NGX_CUDA_TRY(cudaMallocAsync(&d_sample, sizeof(int32_t) * static_cast<size_t>(k), g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(d_sample, sample.data(), sizeof(int32_t) * static_cast<size_t>(k), cudaMemcpyHostToDevice, g->stream));
    RunOutputs o;
    int rc = alloc_outputs(g, k, 0, false, o);
    ngx_apsp_opts sample_opts = *opts;
    sample_opts.mode = NGX_MODE_BATCHED;
    if (rc == NGX_OK) {
        rc = launch_tiles(g, &sample_opts, kModeApsp, d_sample, k, 0, 0.0, o, nullptr, nullptr);
    }
    unsigned long long bits = 0;
    if (rc == NGX_OK && cudaMemcpy(&bits, o.counters + kDiameterBits, 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = fail(NGX_CUDA_ERROR, "copying the sampled eccentricity");
    }
    free_outputs(g, o);
    cudaFreeAsync(d_sample, g->stream);
    double ecc = 0.0;
    std::memcpy(&ecc, &bits, sizeof(double));
    *out = ecc > 0.0 ? 1.5 * ecc : 1.0;
    return rc;
}

int collect(ngx_graph* g, const RunOutputs& o, int64_t num_sources, int64_t hist_bins, double hist_max, ngx_apsp_result* r) {
    unsigned long long acc[2 * kAccDigits];
    unsigned long long counters[kCounterCount];
    NGX_CUDA_TRY(cudaMemcpyAsync(acc, o.acc, sizeof(acc), cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(counters, o.counters, sizeof(counters), cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    acc_normalize(acc);
    acc_normalize(acc + kAccDigits);
    r->sum_distances = acc_round_normalized(acc);
    r->sum_inverse = acc_round_normalized(acc + kAccDigits);
    std::memcpy(&r->diameter, &counters[kDiameterBits], sizeof(double));
    r->unreachable = counters[kUnreachable];
    r->reached_pairs = counters[kReachedPairs];
    r->traversed_arcs = counters[kTraversedArcs];
    r->hist_overflow = counters[kHistOverflow];
    r->hist_max = hist_max;
    r->phases = counters[kIterations];
    r->expansions = counters[kExpansions];
    r->lane_expansions = counters[kLaneExpansions];
    r->dag_levels = counters[kDagLevels];
    r->dag_entries = counters[kDagEntries];
    r->dag_scan_tiles = counters[kDagScanTiles];
    for (int i = 0; i < 5; ++i) {
        r->phase_cycles[i] = counters[kCyclesSssp + i];
    }
    r->cpl = r->sum_distances / static_cast<double>(r->reached_pairs);
    r->efficiency = r->sum_inverse / static_cast<double>(r->reached_pairs);
    const size_t s = static_cast<size_t>(num_sources);
    if (r->hist != nullptr && hist_bins > 0) {
        NGX_CUDA_TRY(cudaMemcpyAsync(r->hist, o.hist, static_cast<size_t>(hist_bins) * 8, cudaMemcpyDeviceToHost, g->stream));
    }
    if (s > 0) {
        if (r->src_sum != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_sum, o.src_f64, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_max != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_max, o.src_f64 + s, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_sum_inverse != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_sum_inverse, o.src_f64 + 2 * s, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_unreachable != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_unreachable, o.src_u64, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_arcs != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_arcs, o.src_u64 + s, s * 8, cudaMemcpyDeviceToHost, g->stream));
    }
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return NGX_OK;
}

void clear_result_totals(ngx_apsp_result* r) {
    r->sum_distances = r->sum_inverse = r->diameter = 0.0;
    r->unreachable = r->reached_pairs = r->traversed_arcs = r->hist_overflow = 0;
    r->hist_max = 0.0;
    r->cpl = r->efficiency = 0.0;
    r->kernel_ms = 0.0;
    r->phases = r->expansions = r->lane_expansions = r->dag_levels = r->dag_entries = r->dag_scan_tiles = 0;
    for (int i = 0; i < 5; ++i) {
        r->phase_cycles[i] = 0;
    }
}

int run_apsp(ngx_graph* g, const ngx_apsp_opts* opts, ngx_apsp_result* result, double* rows, int tile_mode, DagOutputs* extra) {
    if (const int rc = check_opts(g, opts); rc != NGX_OK) {
        return rc;
    }
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    *g->h_abort = 0;
    std::vector<int32_t> sources;
    if (const int rc = prepare_sources(g, opts, sources); rc != NGX_OK) {
        return rc;
    }
    ngx_apsp_result scratch{};
    ngx_apsp_result* r = result != nullptr ? result : &scratch;
    clear_result_totals(r);
    const int64_t num_sources = static_cast<int64_t>(sources.size());
    if (num_sources == 0 || g->n == 0) {
        r->cpl = r->efficiency = NAN;  // no reached pairs, as 0 / 0 in AllPairsShortestPath.h:157-158
        return NGX_OK;
    }
    const int64_t hist_bins = opts->hist_bins;
    double hist_max = opts->hist_max;
    if (hist_bins > 0 && !(hist_max > 0.0)) {
        if (const int rc = auto_hist_max(g, opts, sources, &hist_max); rc != NGX_OK) {
            return rc;
        }
    }
    int32_t* d_sources = nullptr;
    NGX_CUDA_TRY(cudaMallocAsync(&d_sources, sizeof(int32_t) * sources.size(), g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(d_sources, sources.data(), sizeof(int32_t) * sources.size(), cudaMemcpyHostToDevice, g->stream));
    RunOutputs o;
    int rc = alloc_outputs(g, num_sources, hist_bins, rows != nullptr, o);
    float ms = 0.0f;
    if (rc == NGX_OK) {
        rc = launch_tiles(g, opts, tile_mode, d_sources, num_sources, hist_bins, hist_max, o, extra, &ms);
    }
    if (rc == NGX_OK) {
        rc = collect(g, o, num_sources, hist_bins, hist_max, r);
        r->kernel_ms = ms;
    }
    if (rc == NGX_OK && rows != nullptr) {
        const cudaError_t err = cudaMemcpy(rows, o.rows, static_cast<size_t>(num_sources) * static_cast<size_t>(g->n) * 8, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "copying distance rows");
        }
    }
    free_outputs(g, o);
    cudaFreeAsync(d_sources, g->stream);
    cudaStreamSynchronize(g->stream);
    return rc;
}

}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_apsp(ngx_graph* graph, const ngx_apsp_opts* opts, ngx_apsp_result* result) { return run_apsp(graph, opts, result, nullptr, kModeApsp, nullptr); }

int ngx_sssp_rows(ngx_graph* graph, const ngx_apsp_opts* opts, double* rows) {
    if (rows == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_sssp_rows: rows is NULL");
    }
    ngx_apsp_opts o = *opts;
    o.hist_bins = 0;
    return run_apsp(graph, &o, nullptr, rows, kModeApsp, nullptr);
}

}  // extern "C"
