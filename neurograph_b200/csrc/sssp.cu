// Host side of the tile runs: source tiling, workspace sizing, launch, result reduction.
//
// Replaces AllPairsShortestPath::compute_apsp_impl's per-source loop (source/metrics/paths/AllPairsShortestPath.h:110-163)
// and compute_apsp_impl_delta_stepping (:197-247) with one persistent launch over all source tiles, of one graph or of
// a batch of graphs.

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
#ifndef NGX_BATCHED_UNROLL
#define NGX_BATCHED_UNROLL 4  // (arc, source) pairs in flight per lane in the distance phase
#endif
constexpr int kBatchedUnroll = NGX_BATCHED_UNROLL;
constexpr int kPlainWarpsMax = 16;
constexpr int kBatchedDefaultBlock = 512;
constexpr int kMaxGroupSize = 512;  // CTAs sharing one tile at most (above any SM count x resident CTAs per SM used here)

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
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

double default_delta_scale(int64_t n, int64_t m) {
    const double degree = n > 0 ? static_cast<double>(m) / static_cast<double>(n) : 1.0;
    const double scale = 2.0 / std::sqrt(degree > 1.0 ? degree : 1.0);
    return scale < 0.125 ? 0.125 : (scale > 2.0 ? 2.0 : scale);
}

double pick_delta(double mean_len, double requested, double scale) {
    if (requested > 0.0 && std::isfinite(requested)) {
        return requested;
    }
    const double base = mean_len > 0.0 && std::isfinite(mean_len) ? mean_len : 1.0;
    return base * (scale > 0.0 ? scale : 1.0);
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
    if (opts->tile_ctas < 0 || opts->tile_ctas > kMaxGroupSize) {
        return fail(NGX_INVALID_ARGUMENT, "tile_ctas must be in [0, " + std::to_string(kMaxGroupSize) + "]");
    }
    if (opts->block_threads != 0 && (opts->block_threads < 64 || opts->block_threads > 512 || opts->block_threads % 32 != 0)) {
        return fail(NGX_INVALID_ARGUMENT, "block_threads must be a multiple of 32 in [64, 512]");
    }
    return NGX_OK;
}

int alloc_outputs(ngx_graph* g, int64_t num_graphs, int64_t num_sources, int64_t hist_bins, bool want_rows, RunOutputs& o, bool persistent) {
    const size_t s = static_cast<size_t>(num_sources);
    const size_t gcount = static_cast<size_t>(num_graphs);
    size_t off = 0;
    const auto take = [&](size_t bytes) {
        const size_t at = off;
        off += align256(bytes);
        return at;
    };
    const size_t a_acc = take(gcount * 2 * kAccDigits * 8);
    const size_t a_cnt = take(gcount * kCounterCount * 8);
    const size_t a_err = take(8);
    const size_t a_tile = take(8);
    const size_t a_hist = take(gcount * static_cast<size_t>(std::max<int64_t>(hist_bins, 1)) * 8);
    const size_t zeroed = off;  // everything above starts at zero
    const size_t a_graphs = take(gcount * sizeof(GraphDesc));
    const size_t a_sources = take(std::max<size_t>(s, 1) * 4);
    const size_t a_f64 = take(3 * s * 8);
    const size_t a_u64 = take(2 * s * 8);
    const size_t a_rows = want_rows ? take(s * static_cast<size_t>(g->n) * 8) : 0;
    if (persistent) {
        if (off > g->persistent_bytes) {
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            cudaFree(g->d_persistent);
            g->d_persistent = nullptr;
            g->persistent_bytes = 0;
            NGX_CUDA_TRY(cudaMalloc(&g->d_persistent, off));
            g->persistent_bytes = off;
        }
        o.block = g->d_persistent;
        o.owned = false;
    } else {
        if (const int rc = grow_buffer(g, &g->d_call_out, &g->call_out_bytes, off); rc != NGX_OK) {
            return rc;
        }
        o.block = g->d_call_out;
        o.owned = false;
    }
    o.bytes = off;
    o.zeroed_bytes = zeroed;
    char* b = static_cast<char*>(o.block);
    o.acc = reinterpret_cast<unsigned long long*>(b + a_acc);
    o.counters = reinterpret_cast<unsigned long long*>(b + a_cnt);
    o.error = reinterpret_cast<int*>(b + a_err);
    o.tile_counter = reinterpret_cast<unsigned long long*>(b + a_tile);
    o.hist = reinterpret_cast<unsigned long long*>(b + a_hist);
    o.graphs = reinterpret_cast<GraphDesc*>(b + a_graphs);
    o.sources = reinterpret_cast<int32_t*>(b + a_sources);
    o.src_f64 = reinterpret_cast<double*>(b + a_f64);
    o.src_u64 = reinterpret_cast<unsigned long long*>(b + a_u64);
    o.rows = want_rows ? reinterpret_cast<double*>(b + a_rows) : nullptr;
    o.num_graphs = num_graphs;
    o.num_sources = num_sources;
    return NGX_OK;
}

void free_outputs(ngx_graph* g, RunOutputs& o) {
    if (o.block != nullptr && o.owned) {
        cudaFreeAsync(o.block, g->stream);
    }
    o.block = nullptr;
}

int device_error_status(int code) {
    switch (code) {
    case kDevOk: return NGX_OK;
    case kDevTimeout: return fail(NGX_TIMEOUT, "a source tile exceeded max_iterations delta-stepping phases");
    case kDevAborted: return fail(NGX_ABORTED, "run aborted by ngx_graph_request_abort");
    default: return fail(NGX_CUDA_ERROR, "unknown device error code " + std::to_string(code));
    }
}

// The instantiation for a block size; 256 threads with ctas_per_sm >= 4 selects the 4-CTA (64-register) build. Tile
// groups of several CTAs (multi) and reach lists (reach) are built for the default shape only (512 threads x 2 CTAs per
// SM); nullptr for other combinations.
template <int kMode>
const void* tile_kernel_for_block(int block, int ctas_per_sm, bool reach, bool multi) {
    if (reach || multi) {
        if (block != kBatchedDefaultBlock) {
            return nullptr;
        }
        if (multi && reach) return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 512, 2, true, true>);
        if (multi) return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 512, 2, true, false>);
        return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 512, 2, false, true>);
    }
    switch (block) {
    case 256:
        return ctas_per_sm >= 4 ? reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 256, 4>)
                                : reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 256, 3>);
    case 384: return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 384, 2>);
    case 512: return reinterpret_cast<const void*>(&tile_kernel<kMode, kBatchedUnroll, 512, 2>);
    default: return nullptr;
    }
}

// CTAs per tile group: the caller's choice, else the largest of three needs.
//  * L2 residency: the distance phase of a tile touches about 280 bytes per vertex (its 256-byte distance rows, pending
//    marks, queues); when a tile fits in L2, as many tiles are kept in flight as fit in 90 % of it, each worked by
//    resident / that many CTAs (measured: 4 tiles of 74 CTAs on the 100,000-vertex connectome, +20 % for APSP and
//    +18 % for Brandes over one CTA per tile).
//  * Few tiles: a run with fewer tiles than resident CTAs gives each tile the CTAs the others would leave idle.
//  * Memory: when the device affords fewer workspace slots than that, each slot gets enough CTAs to use every SM.
int choose_group_size(int requested, int64_t resident, int64_t num_tiles, int64_t affordable_slots, int64_t n, size_t l2_bytes) {
    if (requested > 0) {
        return static_cast<int>(std::min<int64_t>({ static_cast<int64_t>(requested), resident, static_cast<int64_t>(kMaxGroupSize) }));
    }
    int64_t group = 1;
    const double tile_bytes = 280.0 * static_cast<double>(std::max<int64_t>(n, 1));
    const double room = 0.9 * static_cast<double>(l2_bytes);
    if (tile_bytes <= 0.5 * room) {
        const int64_t in_flight = std::max<int64_t>(1, static_cast<int64_t>(room / tile_bytes));
        group = std::max<int64_t>(group, resident / in_flight);
    }
    group = std::max<int64_t>(group, resident / std::max<int64_t>(1, num_tiles));
    if (affordable_slots < std::min(resident, num_tiles)) {
        // enough CTAs per slot that the affordable slots hold every resident CTA (rounded up: the slot count then
        // follows from the group size, and no CTA is left without a slot)
        const int64_t slots = std::max<int64_t>(1, affordable_slots);
        group = std::max<int64_t>(group, (resident + slots - 1) / slots);
    }
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({ group, resident, static_cast<int64_t>(kMaxGroupSize) })));
}

// Launches the tile kernel: cooperative when several CTAs share a tile (they wait for one another at group barriers,
// so all of them must be resident at once).
cudaError_t launch_tile_kernel(const void* kernel, int64_t grid, int block, size_t smem, cudaStream_t stream, int group_size, void** args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = group_size > 1 ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, kernel, args);
}

int launch_tiles(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, const TileJob& job, int64_t hist_bins, double hist_max, RunOutputs& o,
                 DagOutputs* extra, float* kernel_ms, bool synchronous) {
    // the plain (one source per CTA) form runs APSP and Brandes; the adjoint is batched only
    const bool batched = opts->mode == NGX_MODE_BATCHED || tile_mode == kModeGrad;
    const int width = batched ? kTile : 1;
    const int64_t num_tiles = batched ? job.num_items : job.num_sources;
    const int block = opts->block_threads > 0 ? opts->block_threads : (batched ? kBatchedDefaultBlock : 512);
    const size_t acc_bytes = static_cast<size_t>(2) * (batched ? kTile : kPlainWarpsMax) * kAccDigits * 8;
    const size_t smem = acc_bytes + static_cast<size_t>(hist_bins) * 4;
    if (!batched && job.num_graphs != 1) {
        return fail(NGX_UNSUPPORTED, "the plain form runs one graph at a time");
    }
    if (num_tiles == 0) {
        return NGX_OK;
    }

    const void* kernel = tile_mode == kModeBrandes ? reinterpret_cast<const void*>(&sssp_plain_kernel<true>)
                                                   : reinterpret_cast<const void*>(&sssp_plain_kernel<false>);
    // reach lists (several strongly connected components) and tile groups run with the default block shape only
    const bool default_shape = block == kBatchedDefaultBlock && (opts->ctas_per_sm == 0 || opts->ctas_per_sm >= 2);
    if (batched && opts->tile_ctas > 1 && !default_shape) {
        return fail(NGX_INVALID_ARGUMENT, "tile groups (tile_ctas > 1) run with the default block shape (512 threads, 2 CTAs per SM)");
    }
    const bool track = batched && job.track_reach && default_shape;
    const auto pick = [&](bool reach, bool multi) -> const void* {
        return tile_mode == kModeBrandes ? tile_kernel_for_block<kModeBrandes>(block, opts->ctas_per_sm, reach, multi)
               : tile_mode == kModeGrad  ? tile_kernel_for_block<kModeGrad>(block, opts->ctas_per_sm, reach, multi)
                                         : tile_kernel_for_block<kModeApsp>(block, opts->ctas_per_sm, reach, multi);
    };
    if (batched) {
        kernel = pick(track, false);
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
    const int64_t n = job.n_max;
    const int64_t resident = static_cast<int64_t>(g->sm_count) * per_sm;
    const size_t reach_bytes = track ? static_cast<size_t>(n) * 8 + 512 : 0;  // reach mask + reached list
    const size_t dag_bytes = tile_mode == kModeApsp ? 0 : batched ? brandes_slot_bytes(n, tile_mode == kModeGrad) : plain_brandes_slot_bytes(n);
    const size_t data_bytes = sssp_slot_bytes(n, width) + dag_bytes + reach_bytes;
    const size_t budget = workspace_budget(g);
    // the group size decides the group storage per slot, which the slot count must leave room for
    const int64_t affordable = static_cast<int64_t>(budget / (data_bytes + static_cast<size_t>(group_stride_words(kMaxGroupSize)) * 8));
    const int group = batched && default_shape ? choose_group_size(opts->tile_ctas, resident, num_tiles, affordable, n, g->l2_bytes) : 1;
    if (group > 1) {
        kernel = pick(track, true);  // the same shape and occupancy, built for groups
        NGX_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    }
    const size_t group_bytes = static_cast<size_t>(group_stride_words(group)) * 8;
    const size_t slot_bytes = data_bytes + group_bytes;
    int64_t slots = std::min<int64_t>(num_tiles, resident / group);
    slots = std::min<int64_t>(slots, static_cast<int64_t>(budget / slot_bytes));
    if (slots <= 0) {
        return fail(NGX_OUT_OF_MEMORY, "not enough device memory for one workspace slot (" + std::to_string(slot_bytes) + " bytes)");
    }
    if (const int rc = ensure_workspace(g, static_cast<size_t>(slots) * slot_bytes); rc != NGX_OK) {
        return rc;
    }
    char* ws = static_cast<char*>(g->d_workspace);
    // group storage first (256-byte aligned slots), then the slot arrays
    unsigned long long* group_ws = reinterpret_cast<unsigned long long*>(ws);
    ws += static_cast<size_t>(slots) * group_bytes;
    SsspParams p{};
    p.g = g->csr(opts->metric);
    p.g.n = n;
    p.sources = o.sources;
    p.num_sources = job.num_sources;
    p.num_tiles = num_tiles;
    p.delta = job.plain_delta;
    p.graphs = o.graphs;
    p.items = job.d_items;
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
    p.group_size = group;
    p.group_stride = group_stride_words(group);
    p.group_ws = group_ws;
    if (track) {
        ws = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(ws) + 255) & ~uintptr_t(255));
        p.ws_reach = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * n * 4;
        p.ws_touched = reinterpret_cast<int32_t*>(ws);
        ws += static_cast<size_t>(slots) * n * 4;
    }
    BrandesParams bp{};
    if (tile_mode == kModeBrandes && !batched) {
        // plain form: sigma, delta, predecessor counts and the level list per vertex, the level offsets
        ws = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(ws) + 255) & ~uintptr_t(255));
        bp.rg = g->reverse_csr();
        bp.ws_sigma = reinterpret_cast<double*>(ws);
        ws += static_cast<size_t>(slots) * n * 8;
        bp.ws_delta = reinterpret_cast<double*>(ws);
        ws += static_cast<size_t>(slots) * n * 8;
        bp.ws_cnt = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * n * 4;
        bp.ws_list = reinterpret_cast<int32_t*>(ws);
        ws += static_cast<size_t>(slots) * n * 4;
        bp.ws_loff = reinterpret_cast<int32_t*>(ws);
        if (extra != nullptr) {
            bp.bc = extra->bc;
        }
    } else if (tile_mode != kModeApsp) {
        const size_t nt = static_cast<size_t>(n) * kTile;
        ws = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(ws) + 255) & ~uintptr_t(255));
        bp.rg = g->reverse_csr();
        bp.arc_src = g->d_arc_src;
        bp.m_total = g->m_stored;
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
        bp.ws_tie = reinterpret_cast<uint32_t*>(ws);
        ws += static_cast<size_t>(slots) * n * 4;
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
    p.out.src_max = o.src_f64 + job.num_sources;
    p.out.src_inv = o.src_f64 + 2 * job.num_sources;
    p.out.src_unreach = o.src_u64;
    p.out.src_arcs = o.src_u64 + job.num_sources;
    p.out.rows = o.rows;

    cudaEvent_t start = nullptr, stop = nullptr;
    if (synchronous) {
        NGX_CUDA_TRY(cudaEventCreate(&start));
        NGX_CUDA_TRY(cudaEventCreate(&stop));
        cudaEventRecord(start, g->stream);
    }
    cudaError_t err = cudaSuccess;
    if (batched) {
        void* args[] = { &p, &bp };
        err = cudaMemsetAsync(group_ws, 0, static_cast<size_t>(slots) * group_bytes, g->stream);
        if (err == cudaSuccess) {
            err = launch_tile_kernel(kernel, slots * group, block, smem, g->stream, group, args);
        }
    } else {
        if (tile_mode == kModeBrandes) {
            sssp_plain_kernel<true><<<static_cast<unsigned>(slots), block, smem, g->stream>>>(p, bp);
        } else {
            sssp_plain_kernel<false><<<static_cast<unsigned>(slots), block, smem, g->stream>>>(p, bp);
        }
        err = cudaGetLastError();
    }
    if (!synchronous) {
        return err == cudaSuccess ? NGX_OK : cuda_fail(err, "tile kernel launch");
    }
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
        return cuda_fail(err, "tile kernel");
    }
    if (kernel_ms != nullptr) {
        *kernel_ms += ms;
    }
    int code = 0;
    NGX_CUDA_TRY(cudaMemcpy(&code, o.error, sizeof(int), cudaMemcpyDeviceToHost));
    return device_error_status(code);
}

// Launches the batched APSP tile kernel on the graph's stream with its workspace carved from `ws` (`ws_bytes` bytes,
// 256-byte aligned) instead of the handle's workspace: nothing is allocated. Per-source outputs are written only where
// `o` has them. Returns after the launch; the caller synchronizes.
int launch_apsp_in_workspace(ngx_graph* g, const ngx_apsp_opts* opts, const TileJob& job, int64_t hist_bins, double hist_max, RunOutputs& o, void* ws,
                             size_t ws_bytes) {
    const int block = opts->block_threads > 0 ? opts->block_threads : kBatchedDefaultBlock;
    const void* kernel = tile_kernel_for_block<kModeApsp>(block, opts->ctas_per_sm, false, false);
    if (kernel == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "batched mode supports block_threads 256, 384 or 512");
    }
    if (job.num_items == 0) {
        return NGX_OK;
    }
    const size_t smem = static_cast<size_t>(2) * kTile * kAccDigits * 8 + static_cast<size_t>(hist_bins) * 4;
    NGX_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int per_sm = 0;
    NGX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
    if (per_sm <= 0) {
        return fail(NGX_UNSUPPORTED, "kernel does not fit on an SM with this block size and histogram");
    }
    if (opts->ctas_per_sm > 0) {
        per_sm = std::min(per_sm, opts->ctas_per_sm);
    }
    const int64_t n = job.n_max;
    const size_t group_bytes = static_cast<size_t>(group_stride_words(1)) * 8;  // one CTA per tile
    const size_t slot_bytes = sssp_slot_bytes(n, kTile) + group_bytes;
    int64_t slots = std::min<int64_t>(job.num_items, static_cast<int64_t>(g->sm_count) * per_sm);
    slots = std::min<int64_t>(slots, static_cast<int64_t>(ws_bytes / slot_bytes));
    if (slots <= 0) {
        return fail(NGX_OUT_OF_MEMORY, "the workspace holds no slot of " + std::to_string(slot_bytes) + " bytes");
    }
    char* w = static_cast<char*>(ws);
    unsigned long long* group_ws = reinterpret_cast<unsigned long long*>(w);
    w += static_cast<size_t>(slots) * group_bytes;
    SsspParams p{};
    p.g = g->csr(opts->metric);
    p.g.n = n;
    p.sources = o.sources;
    p.num_sources = job.num_sources;
    p.num_tiles = job.num_items;
    p.delta = job.plain_delta;
    p.graphs = o.graphs;
    p.items = job.d_items;
    p.max_iterations = opts->max_iterations > 0 ? opts->max_iterations : static_cast<unsigned long long>(4 * n + 64);
    p.tile_counter = o.tile_counter;
    p.error = o.error;
    p.abort_flag = g->d_abort;
    p.ws_dist = reinterpret_cast<unsigned long long*>(w);
    w += static_cast<size_t>(slots) * n * kTile * 8;
    p.ws_pend = reinterpret_cast<uint32_t*>(w);
    w += static_cast<size_t>(slots) * 2 * n * 4;
    p.ws_far = reinterpret_cast<uint32_t*>(w);
    w += static_cast<size_t>(slots) * n * 4;
    p.ws_queue = reinterpret_cast<int32_t*>(w);
    w += static_cast<size_t>(slots) * 2 * n * 4;
    p.ws_stamp = reinterpret_cast<uint32_t*>(w);
    p.group_size = 1;
    p.group_stride = group_stride_words(1);
    p.group_ws = group_ws;
    BrandesParams bp{};
    p.out.acc_sum = o.acc;
    p.out.acc_inv = o.acc + kAccDigits;
    p.out.counters = o.counters;
    p.out.hist = hist_bins > 0 ? o.hist : nullptr;
    p.out.hist_bins = static_cast<int>(hist_bins);
    p.out.hist_max = hist_max;
    p.out.hist_width = hist_bins > 0 ? hist_max / static_cast<double>(hist_bins) : 0.0;
    if (o.src_f64 != nullptr) {
        p.out.src_sum = o.src_f64;
        p.out.src_max = o.src_f64 + job.num_sources;
        p.out.src_inv = o.src_f64 + 2 * job.num_sources;
    }
    if (o.src_u64 != nullptr) {
        p.out.src_unreach = o.src_u64;
        p.out.src_arcs = o.src_u64 + job.num_sources;
    }
    void* args[] = { &p, &bp };
    cudaError_t err = cudaMemsetAsync(group_ws, 0, static_cast<size_t>(slots) * group_bytes, g->stream);
    if (err == cudaSuccess) {
        err = cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(slots)), dim3(block), args, smem, g->stream);
    }
    return err == cudaSuccess ? NGX_OK : cuda_fail(err, "tile kernel launch");
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

// Reduces graph `gi`'s accumulators and counters (host copies) into a result; copies its optional device outputs.
int collect_graph(ngx_graph* g, const RunOutputs& o, const unsigned long long* acc_all, const unsigned long long* counters_all, int64_t gi,
                  int64_t src_off, int64_t num_sources, int64_t hist_bins, double hist_max, ngx_apsp_result* r, const int32_t* scatter) {
    unsigned long long acc[2 * kAccDigits];
    std::memcpy(acc, acc_all + gi * 2 * kAccDigits, sizeof(acc));
    const unsigned long long* counters = counters_all + gi * kCounterCount;
    acc_normalize(acc);
    acc_normalize(acc + kAccDigits);
    r->sum_distances = acc_round_normalized(acc);
    r->sum_inverse = acc_round_normalized(acc + kAccDigits);
    if (r->acc_digits != nullptr) {
        std::memcpy(r->acc_digits, acc, sizeof(acc));
    }
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
    // AllPairsShortestPath.h:154-158: both averages are over the R reached ordered pairs (0 / 0 gives NaN, as there)
    r->cpl = r->sum_distances / static_cast<double>(r->reached_pairs);
    r->efficiency = r->sum_inverse / static_cast<double>(r->reached_pairs);
    const size_t s = static_cast<size_t>(num_sources);
    const size_t total = static_cast<size_t>(o.num_sources);
    const size_t at = static_cast<size_t>(src_off);
    if (r->hist != nullptr && hist_bins > 0) {
        NGX_CUDA_TRY(cudaMemcpyAsync(r->hist, o.hist + gi * hist_bins, static_cast<size_t>(hist_bins) * 8, cudaMemcpyDeviceToHost, g->stream));
    }
    if (s > 0 && scatter != nullptr) {
        // the run took the sources in the graph's locality order: entry i belongs to vertex scatter[i]
        std::vector<unsigned long long> tmp(s);
        const auto put = [&](void* dst, const void* src) -> int {
            if (dst == nullptr) {
                return NGX_OK;
            }
            NGX_CUDA_TRY(cudaMemcpyAsync(tmp.data(), src, s * 8, cudaMemcpyDeviceToHost, g->stream));
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            auto* out = static_cast<unsigned long long*>(dst);
            for (size_t i = 0; i < s; ++i) {
                out[scatter[i]] = tmp[i];
            }
            return NGX_OK;
        };
        int rc = put(r->src_sum, o.src_f64 + at);
        if (rc == NGX_OK) rc = put(r->src_max, o.src_f64 + total + at);
        if (rc == NGX_OK) rc = put(r->src_sum_inverse, o.src_f64 + 2 * total + at);
        if (rc == NGX_OK) rc = put(r->src_unreachable, o.src_u64 + at);
        if (rc == NGX_OK) rc = put(r->src_arcs, o.src_u64 + total + at);
        return rc;
    }
    if (s > 0) {
        if (r->src_sum != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_sum, o.src_f64 + at, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_max != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_max, o.src_f64 + total + at, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_sum_inverse != nullptr) {
            NGX_CUDA_TRY(cudaMemcpyAsync(r->src_sum_inverse, o.src_f64 + 2 * total + at, s * 8, cudaMemcpyDeviceToHost, g->stream));
        }
        if (r->src_unreachable != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_unreachable, o.src_u64 + at, s * 8, cudaMemcpyDeviceToHost, g->stream));
        if (r->src_arcs != nullptr) NGX_CUDA_TRY(cudaMemcpyAsync(r->src_arcs, o.src_u64 + total + at, s * 8, cudaMemcpyDeviceToHost, g->stream));
    }
    return NGX_OK;
}

int read_totals(ngx_graph* g, const RunOutputs& o, std::vector<unsigned long long>& acc, std::vector<unsigned long long>& counters) {
    acc.resize(static_cast<size_t>(o.num_graphs) * 2 * kAccDigits);
    counters.resize(static_cast<size_t>(o.num_graphs) * kCounterCount);
    NGX_CUDA_TRY(cudaMemcpyAsync(acc.data(), o.acc, acc.size() * 8, cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(counters.data(), o.counters, counters.size() * 8, cudaMemcpyDeviceToHost, g->stream));
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return NGX_OK;
}

// One single-graph run of `sources` (graph 0 of the handle).
int run_sources(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, const std::vector<int32_t>& sources, int64_t hist_bins, double hist_max,
                bool want_rows, DagOutputs* extra, RunOutputs& o, float* ms) {
    const int64_t num_sources = static_cast<int64_t>(sources.size());
    if (const int rc = alloc_outputs(g, 1, num_sources, hist_bins, want_rows, o, false); rc != NGX_OK) {
        return rc;
    }
    const GraphPart& part = g->parts[0];
    const double delta = pick_delta(opts->metric == NGX_METRIC_INVERSE ? part.mean_len_inverse : part.mean_len_regular, opts->delta,
                                    default_delta_scale(part.n, part.m_stored));
    const GraphDesc desc{ part.n, part.m_stored, part.row_off, 0, num_sources, part.vertex_off, delta };
    NGX_CUDA_TRY(cudaMemsetAsync(o.block, 0, o.zeroed_bytes, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(o.graphs, &desc, sizeof(desc), cudaMemcpyHostToDevice, g->stream));
    NGX_CUDA_TRY(cudaMemcpyAsync(o.sources, sources.data(), sizeof(int32_t) * sources.size(), cudaMemcpyHostToDevice, g->stream));
    TileJob job;
    job.num_graphs = 1;
    job.num_items = (num_sources + kTile - 1) / kTile;
    job.d_items = nullptr;
    job.num_sources = num_sources;
    job.n_max = part.n;
    job.plain_delta = delta;
    job.track_reach = g->scc_components > 1;
    return launch_tiles(g, opts, tile_mode, job, hist_bins, hist_max, o, extra, ms, true);
}

// Histogram bound when the caller gives none: 1.5 x the largest eccentricity of up to one tile of sources spread
// over the requested list (plus the overflow count for anything beyond it).
int auto_hist_max(ngx_graph* g, const ngx_apsp_opts* opts, const std::vector<int32_t>& sources, double* out) {
    const int64_t k = std::min<int64_t>(kTile, static_cast<int64_t>(sources.size()));
    std::vector<int32_t> sample(static_cast<size_t>(k));
    for (int64_t i = 0; i < k; ++i) {
        sample[static_cast<size_t>(i)] = sources[static_cast<size_t>(i * static_cast<int64_t>(sources.size()) / k)];
    }
    ngx_apsp_opts sample_opts = *opts;
    sample_opts.mode = NGX_MODE_BATCHED;
    RunOutputs o;
    int rc = run_sources(g, &sample_opts, kModeApsp, sample, 0, 0.0, false, nullptr, o, nullptr);
    unsigned long long bits = 0;
    if (rc == NGX_OK) {
        std::vector<unsigned long long> acc, counters;
        rc = read_totals(g, o, acc, counters);
        if (rc == NGX_OK) {
            bits = counters[kDiameterBits];
        }
    }
    free_outputs(g, o);
    double ecc = 0.0;
    std::memcpy(&ecc, &bits, sizeof(double));
    *out = ecc > 0.0 ? 1.5 * ecc : 1.0;
    return rc;
}

int run_apsp(ngx_graph* g, const ngx_apsp_opts* caller_opts, ngx_apsp_result* result, double* rows, int tile_mode, DagOutputs* extra) {
    if (const int rc = check_opts(g, caller_opts); rc != NGX_OK) {
        return rc;
    }
    // options left at 0 take the handle's tuned values for this task (ngx_graph_autotune), if any
    ngx_apsp_opts tuned_opts = *caller_opts;
    const ngx_tuning& t = g->tuned[tile_mode];
    if (t.block_threads > 0 && tuned_opts.mode == NGX_MODE_BATCHED) {
        if (tuned_opts.block_threads == 0 && tuned_opts.ctas_per_sm == 0) {
            tuned_opts.block_threads = t.block_threads;
            tuned_opts.ctas_per_sm = t.ctas_per_sm;
        }
        if (tuned_opts.tile_ctas == 0) {
            tuned_opts.tile_ctas = t.tile_ctas;
        }
        if (!(tuned_opts.delta > 0.0) && g->parts.size() == 1) {
            const GraphPart& part = g->parts[0];
            tuned_opts.delta = pick_delta(tuned_opts.metric == NGX_METRIC_INVERSE ? part.mean_len_inverse : part.mean_len_regular, 0.0, t.delta_scale);
        }
    }
    const ngx_apsp_opts* opts = &tuned_opts;
    if (g->parts.size() != 1) {
        return fail(NGX_INVALID_ARGUMENT, "this handle holds a batch of graphs: use ngx_batch_run");
    }
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    *g->h_abort = 0;
    // the strongly connected components decide whether tiles keep reach lists (several components)
    if (const int rc = ensure_components(g); rc != NGX_OK) {
        return rc;
    }
    std::vector<int32_t> sources;
    if (const int rc = prepare_sources(g, opts, sources); rc != NGX_OK) {
        return rc;
    }
    // all sources: in the graph's locality order (tiles of nearby sources), results scattered back by vertex;
    // distance rows keep vertex order
    const int32_t* scatter = nullptr;
    if (opts->sources == nullptr && rows == nullptr) {
        if (const int rc = ensure_source_order(g); rc != NGX_OK) {
            return rc;
        }
    }
    if (opts->sources == nullptr && rows == nullptr && g->source_order.size() == sources.size()) {
        sources.assign(g->source_order.begin(), g->source_order.end());
        scatter = g->source_order.data();
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
    RunOutputs o;
    float ms = 0.0f;
    int rc = run_sources(g, opts, tile_mode, sources, hist_bins, hist_max, rows != nullptr, extra, o, &ms);
    if (rc == NGX_OK) {
        std::vector<unsigned long long> acc, counters;
        rc = read_totals(g, o, acc, counters);
        if (rc == NGX_OK) {
            rc = collect_graph(g, o, acc.data(), counters.data(), 0, 0, num_sources, hist_bins, hist_max, r, scatter);
        }
        r->kernel_ms = ms;
    }
    if (rc == NGX_OK && rows != nullptr) {
        const cudaError_t err = cudaMemcpyAsync(rows, o.rows, static_cast<size_t>(num_sources) * static_cast<size_t>(g->n) * 8, cudaMemcpyDeviceToHost,
                                                g->stream);
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "copying distance rows");
        }
    }
    cudaStreamSynchronize(g->stream);
    free_outputs(g, o);
    cudaStreamSynchronize(g->stream);
    return rc;
}

}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_apsp(ngx_graph* graph, const ngx_apsp_opts* opts, ngx_apsp_result* result) {
    return guard_host("ngx_apsp", [&]() -> int { return run_apsp(graph, opts, result, nullptr, kModeApsp, nullptr); });
}

int ngx_sssp_rows(ngx_graph* graph, const ngx_apsp_opts* opts, double* rows) {
    return guard_host("ngx_sssp_rows", [&]() -> int {
        if (rows == nullptr || opts == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_sssp_rows: opts or rows is NULL");
        }
        ngx_apsp_opts o = *opts;
        o.hist_bins = 0;
        return run_apsp(graph, &o, nullptr, rows, kModeApsp, nullptr);
    });
}

}  // extern "C"
