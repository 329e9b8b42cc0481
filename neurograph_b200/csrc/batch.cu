// Batches of independent graphs in one persistent launch, CUDA-graph replay, the bucket-width autotuner, and in-place
// weight updates.
//
// No reference counterpart: neurograph computes its metrics for one graph per run (source/neurograph.cpp:139-416).
// A batch handle concatenates many graphs (graph.cu); its work items are (graph, 32-source tile) pairs in
// longest-first order (graphs with more arcs first), consumed by the persistent tile kernel from one device counter,
// so small and large graphs share the GPU without per-graph launches or idle tails.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_run.h"

namespace ngx {
namespace {

int size_class(int64_t n) {
    int c = 0;
    while ((int64_t(2) << c) <= n && c < NGX_SIZE_CLASSES - 1) {
        ++c;
    }
    return c;
}

int task_mode(int task) {
    switch (task) {
    case NGX_TASK_APSP: return kModeApsp;
    case NGX_TASK_BRANDES: return kModeBrandes;
    case NGX_TASK_GRAD: return kModeGrad;
    default: return -1;
    }
}

// Builds and uploads the (graph, tile) work items of all graphs, graphs with more arcs first.
int build_items(ngx_graph* g) {
    std::vector<int32_t> order(g->parts.size());
    for (size_t i = 0; i < order.size(); ++i) {
        order[i] = static_cast<int32_t>(i);
    }
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        const auto& pa = g->parts[static_cast<size_t>(a)];
        const auto& pb = g->parts[static_cast<size_t>(b)];
        return pa.m_stored * 1.0 * pa.n > pb.m_stored * 1.0 * pb.n;
    });
    std::vector<WorkItem> items;
    for (const int32_t gi : order) {
        const int64_t tiles = (g->parts[static_cast<size_t>(gi)].n + kTile - 1) / kTile;
        for (int64_t t = 0; t < tiles; ++t) {
            items.push_back(WorkItem{ gi, static_cast<int32_t>(t) });
        }
    }
    cudaFree(g->d_items);
    g->d_items = nullptr;
    g->num_items = static_cast<int64_t>(items.size());
    NGX_CUDA_TRY(cudaMalloc(&g->d_items, std::max<size_t>(1, items.size()) * sizeof(WorkItem)));
    if (!items.empty()) {
        NGX_CUDA_TRY(cudaMemcpy(g->d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice));
    }
    return NGX_OK;
}

std::vector<GraphDesc> graph_table(const ngx_graph* g, int metric, double delta_scale) {
    std::vector<GraphDesc> descs(g->parts.size());
    for (size_t i = 0; i < g->parts.size(); ++i) {
        const GraphPart& part = g->parts[i];
        const double scale = delta_scale > 0.0 ? delta_scale : (g->class_scale[size_class(part.n)] > 0.0 ? g->class_scale[size_class(part.n)]
                                                                                     : default_delta_scale(part.n, part.m_stored));
        const double mean = metric == NGX_METRIC_INVERSE ? part.mean_len_inverse : part.mean_len_regular;
        descs[i] = GraphDesc{ part.n, part.m_stored, part.row_off, part.vertex_off, part.n, part.vertex_off, pick_delta(mean, 0.0, scale) };
    }
    return descs;
}

uint64_t mix(uint64_t h, uint64_t x) {
    h ^= x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h;
}

uint64_t options_key(const ngx_batch_opts* o, const ngx_graph* g) {
    uint64_t h = 0;
    h = mix(h, static_cast<uint64_t>(o->task));
    h = mix(h, static_cast<uint64_t>(o->metric));
    uint64_t bits = 0;
    std::memcpy(&bits, &o->delta_scale, 8);
    h = mix(h, bits);
    h = mix(h, static_cast<uint64_t>(o->block_threads));
    h = mix(h, static_cast<uint64_t>(o->tile_ctas));
    h = mix(h, static_cast<uint64_t>(o->hist_bins));
    std::memcpy(&bits, &o->hist_max, 8);
    h = mix(h, bits);
    h = mix(h, o->max_iterations);
    for (int c = 0; c < NGX_SIZE_CLASSES; ++c) {
        std::memcpy(&bits, &g->class_scale[c], 8);
        h = mix(h, bits);
    }
    for (const ngx_tuning& t : g->tuned) {
        h = mix(h, static_cast<uint64_t>(t.block_threads) << 32 | static_cast<uint64_t>(t.ctas_per_sm) << 16 | static_cast<uint64_t>(t.tile_ctas));
    }
    return h == 0 ? 1 : h;
}

// Times the first wave of graph gi's source tiles (at most 2 x SMs tiles, in the order a run takes them) with bucket
// width `scale` x its mean arc length and the launch options of `aopts`; *rate = traversed arcs per millisecond.
int time_wave(ngx_graph* g, int mode, int32_t gi, double scale, const ngx_apsp_opts& aopts, double* rate) {
    *rate = 0.0;
    const GraphPart& part = g->parts[static_cast<size_t>(gi)];
    const int64_t tiles = std::min<int64_t>((part.n + kTile - 1) / kTile, 2 * g->sm_count);
    std::vector<WorkItem> items(static_cast<size_t>(tiles));
    for (int64_t t = 0; t < tiles; ++t) {
        items[static_cast<size_t>(t)] = WorkItem{ 0, static_cast<int32_t>(t) };
    }
    const std::vector<int32_t> sources(g->source_order.begin() + part.vertex_off, g->source_order.begin() + part.vertex_off + part.n);
    WorkItem* d_items = nullptr;
    NGX_CUDA_TRY(cudaMalloc(&d_items, std::max<size_t>(1, items.size()) * sizeof(WorkItem)));
    struct Free {
        WorkItem* p;
        ~Free() { cudaFree(p); }
    } free_items{ d_items };
    NGX_CUDA_TRY(cudaMemcpy(d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice));
    RunOutputs o;
    int rc = alloc_outputs(g, 1, part.n, 0, false, o, false);
    DagOutputs extra;
    const size_t dag_words = 1 + (mode == kModeBrandes ? 2 * static_cast<size_t>(g->n_total) : 0) +
                             (mode == kModeGrad ? 4 * static_cast<size_t>(g->m_user) : 0);
    if (rc == NGX_OK && mode != kModeApsp) {
        rc = grow_buffer(g, &g->d_call_dag, &g->call_dag_bytes, dag_words * 8);
        if (rc == NGX_OK) {
            auto* dag = static_cast<unsigned long long*>(g->d_call_dag);
            cudaMemsetAsync(dag, 0, dag_words * 8, g->stream);
            extra.sigma_inexact = reinterpret_cast<int*>(dag);
            if (mode == kModeBrandes) extra.bc = dag + 1;
            if (mode == kModeGrad) {
                extra.grad_cpl = dag + 1;
                extra.grad_eff = dag + 1 + 2 * static_cast<size_t>(g->m_user);
            }
        }
    }
    if (rc == NGX_OK) {
        const GraphDesc desc{ part.n, part.m_stored, part.row_off, 0, part.n, part.vertex_off, pick_delta(part.mean_len_regular, 0.0, scale) };
        cudaMemsetAsync(o.block, 0, o.zeroed_bytes, g->stream);
        cudaMemcpyAsync(o.graphs, &desc, sizeof(desc), cudaMemcpyHostToDevice, g->stream);
        cudaMemcpyAsync(o.sources, sources.data(), sources.size() * 4, cudaMemcpyHostToDevice, g->stream);
        TileJob job;
        job.num_graphs = 1;
        job.num_items = tiles;
        job.d_items = d_items;
        job.num_sources = part.n;
        job.n_max = g->n;
        float ms = 0.0f;
        rc = launch_tiles(g, &aopts, mode, job, 0, 0.0, o, mode != kModeApsp ? &extra : nullptr, &ms, true);
        if (rc == NGX_OK) {
            std::vector<unsigned long long> acc, counters;
            rc = read_totals(g, o, acc, counters);
            if (rc == NGX_OK && ms > 0.0f) {
                *rate = static_cast<double>(counters[kTraversedArcs]) / ms;
            }
        }
    }
    free_outputs(g, o);
    cudaStreamSynchronize(g->stream);
    return rc;
}

// Resets the zero-initialised part of the outputs (and the betweenness / gradient sums), then launches.
int enqueue_run(ngx_graph* g, const ngx_apsp_opts& aopts, int mode, const TileJob& job, int64_t hist_bins, double hist_max, RunOutputs& o,
                DagOutputs* extra, void* dag_block, size_t dag_bytes) {
    NGX_CUDA_TRY(cudaMemsetAsync(o.block, 0, o.zeroed_bytes, g->stream));
    if (dag_block != nullptr) {
        NGX_CUDA_TRY(cudaMemsetAsync(dag_block, 0, dag_bytes, g->stream));
    }
    return launch_tiles(g, &aopts, mode, job, hist_bins, hist_max, o, extra, nullptr, false);
}

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_batch_create(const ngx_csr* graphs, int64_t count, int device, ngx_graph** out) {
    return guard_host("ngx_batch_create", [&]() -> int {
        const int rc = create_graphs(graphs, count, device, out);
        if (rc != NGX_OK) {
            return rc;
        }
        const int rc2 = build_items(*out);
        if (rc2 != NGX_OK) {
            ngx_graph_destroy(*out);
            *out = nullptr;
        }
        return rc2;
    });
}

int ngx_batch_run(ngx_graph* g, const ngx_batch_opts* opts, ngx_apsp_result* results, double* bc, double* dcpl, double* deff) {
    return guard_host("ngx_batch_run", [&]() -> int {
        if (g == nullptr || opts == nullptr || results == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_batch_run: batch, opts or results is NULL");
        }
        const int mode = task_mode(opts->task);
        if (mode < 0) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_batch_run: unknown task");
        }
        if (mode != kModeApsp && opts->metric != NGX_METRIC_REGULAR) {
            return fail(NGX_UNSUPPORTED, "ngx_batch_run: betweenness and the gradient are defined for the regular metric");
        }
        if (opts->hist_bins < 0 || opts->hist_bins > kMaxHistBins || (opts->hist_bins > 0 && !(opts->hist_max > 0.0))) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_batch_run: hist_bins must be in [0, 16384] with hist_max > 0");
        }
        if (g->d_items == nullptr) {
            if (const int rc = build_items(g); rc != NGX_OK) {
                return rc;
            }
        }
        NGX_CUDA_TRY(cudaSetDevice(g->device));
        *g->h_abort = 0;
        ngx_apsp_opts aopts{};
        aopts.metric = opts->metric;
        aopts.mode = NGX_MODE_BATCHED;
        aopts.block_threads = opts->block_threads;
        aopts.tile_ctas = opts->tile_ctas;
        const ngx_tuning& tuned = g->tuned[mode];
        if (tuned.block_threads > 0 && aopts.block_threads == 0) {
            aopts.block_threads = tuned.block_threads;  // the launch shape ngx_batch_autotune picked
            aopts.ctas_per_sm = tuned.ctas_per_sm;
        }
        if (tuned.tile_ctas > 0 && aopts.tile_ctas == 0) {
            aopts.tile_ctas = tuned.tile_ctas;
        }
        aopts.max_iterations = opts->max_iterations;
        if (const int rc = check_opts(g, &aopts); rc != NGX_OK) {
            return rc;
        }
        const int64_t count = static_cast<int64_t>(g->parts.size());
        const int64_t hist_bins = opts->hist_bins;
        const double hist_max = opts->hist_max;

        // persistent outputs: the run's block, then the betweenness / gradient fixed-point sums and the sigma flag
        const size_t n_total = static_cast<size_t>(g->n_total);
        const size_t m_total = static_cast<size_t>(g->m_user);
        const size_t dag_words = 1 + (mode == kModeBrandes ? 2 * n_total : 0) + (mode == kModeGrad ? 4 * m_total : 0);
        RunOutputs o;
        if (const int rc = alloc_outputs(g, count, g->n_total, hist_bins, false, o, true); rc != NGX_OK) {
            return rc;
        }
        const size_t run_bytes = (o.bytes + 255) & ~size_t(255);
        if (run_bytes + dag_words * 8 > g->persistent_bytes) {
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            if (g->graph_exec != nullptr) {
                cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(g->graph_exec));
                g->graph_exec = nullptr;
                g->graph_key = 0;
            }
            cudaFree(g->d_persistent);
            g->d_persistent = nullptr;
            g->persistent_bytes = 0;
            NGX_CUDA_TRY(cudaMalloc(&g->d_persistent, run_bytes + dag_words * 8));
            g->persistent_bytes = run_bytes + dag_words * 8;
            if (const int rc = alloc_outputs(g, count, g->n_total, hist_bins, false, o, true); rc != NGX_OK) {
                return rc;
            }
        }
        auto* dag_block = reinterpret_cast<unsigned long long*>(static_cast<char*>(g->d_persistent) + run_bytes);
        DagOutputs extra;
        extra.sigma_inexact = reinterpret_cast<int*>(dag_block);
        if (mode == kModeBrandes) {
            extra.bc = dag_block + 1;
        }
        if (mode == kModeGrad) {
            extra.grad_cpl = dag_block + 1;
            extra.grad_eff = dag_block + 1 + 2 * m_total;
        }

        // graph table and sources (every vertex of every graph) for these options
        const std::vector<GraphDesc> descs = graph_table(g, opts->metric, opts->delta_scale);
        // every graph's sources in its locality order (per-source results are scattered back by vertex)
        const auto& sources = g->source_order;
        NGX_CUDA_TRY(cudaMemcpyAsync(o.graphs, descs.data(), descs.size() * sizeof(GraphDesc), cudaMemcpyHostToDevice, g->stream));
        if (!sources.empty()) {
            NGX_CUDA_TRY(cudaMemcpyAsync(o.sources, sources.data(), sources.size() * 4, cudaMemcpyHostToDevice, g->stream));
        }
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        TileJob job;
        job.num_graphs = count;
        job.num_items = g->num_items;
        job.d_items = static_cast<const WorkItem*>(g->d_items);
        job.num_sources = g->n_total;
        job.n_max = g->n;
        job.plain_delta = 1.0;

        const uint64_t key = options_key(opts, g);
        cudaEvent_t start, stop;
        NGX_CUDA_TRY(cudaEventCreate(&start));
        NGX_CUDA_TRY(cudaEventCreate(&stop));
        int rc = NGX_OK;
        cudaEventRecord(start, g->stream);
        if (opts->use_cuda_graph && g->graph_exec != nullptr && g->graph_key == key) {
            const cudaError_t err = cudaGraphLaunch(static_cast<cudaGraphExec_t>(g->graph_exec), g->stream);
            rc = err == cudaSuccess ? NGX_OK : cuda_fail(err, "replaying the captured batch run");
        } else {
            rc = enqueue_run(g, aopts, mode, job, hist_bins, hist_max, o, &extra, dag_block, dag_words * 8);
        }
        cudaEventRecord(stop, g->stream);
        cudaError_t err = cudaEventSynchronize(stop);
        float ms = 0.0f;
        if (err == cudaSuccess) {
            cudaEventElapsedTime(&ms, start, stop);
        } else if (rc == NGX_OK) {
            rc = cuda_fail(err, "batch run");
        }
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        if (rc == NGX_OK) {
            int code = 0;
            NGX_CUDA_TRY(cudaMemcpy(&code, o.error, sizeof(int), cudaMemcpyDeviceToHost));
            rc = device_error_status(code);
        }
        int inexact = 0;
        if (rc == NGX_OK && mode != kModeApsp) {
            NGX_CUDA_TRY(cudaMemcpy(&inexact, extra.sigma_inexact, sizeof(int), cudaMemcpyDeviceToHost));
            if (inexact != 0) {
                // some path count reached 2^53: rerun with the order-defined pull form for sigma (not captured)
                extra.sigma_pull = 1;
                rc = enqueue_run(g, aopts, mode, job, hist_bins, hist_max, o, &extra, dag_block, dag_words * 8);
                if (rc == NGX_OK) {
                    err = cudaStreamSynchronize(g->stream);
                    rc = err == cudaSuccess ? NGX_OK : cuda_fail(err, "batch rerun");
                }
                extra.sigma_pull = 0;
            }
        }
        // capture the run for later replays (after a plain run has sized the workspace; nothing executes here)
        if (rc == NGX_OK && opts->use_cuda_graph && inexact == 0 && (g->graph_exec == nullptr || g->graph_key != key)) {
            if (g->graph_exec != nullptr) {
                cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(g->graph_exec));
                g->graph_exec = nullptr;
                g->graph_key = 0;
            }
            // The workspace was sized by the run above, so the capture allocates nothing. A capture that fails anyway
            // leaves the handle without a graph; the results of the run above stand and later calls launch normally.
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const int crc = enqueue_run(g, aopts, mode, job, hist_bins, hist_max, o, &extra, dag_block, dag_words * 8);
                const cudaError_t cerr = cudaStreamEndCapture(g->stream, &graph);
                cudaGraphExec_t exec = nullptr;
                if (crc == NGX_OK && cerr == cudaSuccess && graph != nullptr && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                    g->graph_exec = exec;
                    g->graph_key = key;
                }
                if (graph != nullptr) {
                    cudaGraphDestroy(graph);
                }
            }
            cudaGetLastError();
            set_last_error("");
        }
        if (rc != NGX_OK) {
            return rc;
        }

        // per-graph results
        std::vector<unsigned long long> acc, counters;
        if ((rc = read_totals(g, o, acc, counters)) != NGX_OK) {
            return rc;
        }
        for (int64_t gi = 0; gi < count; ++gi) {
            ngx_apsp_result* r = &results[gi];
            clear_result_totals(r);
            const GraphPart& part = g->parts[static_cast<size_t>(gi)];
            if ((rc = collect_graph(g, o, acc.data(), counters.data(), gi, part.vertex_off, part.n, hist_bins, hist_max, r,
                                    g->source_order.data() + part.vertex_off)) != NGX_OK) {
                return rc;
            }
            r->kernel_ms = ms;
        }
        if (mode == kModeBrandes && bc != nullptr) {
            std::vector<unsigned long long> fixed(2 * n_total);
            NGX_CUDA_TRY(cudaMemcpyAsync(fixed.data(), extra.bc, fixed.size() * 8, cudaMemcpyDeviceToHost, g->stream));
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            for (size_t v = 0; v < n_total; ++v) {
                bc[v] = fixed_value(fixed[2 * v], fixed[2 * v + 1]);
            }
        }
        if (mode == kModeGrad && (dcpl != nullptr || deff != nullptr)) {
            std::vector<unsigned long long> fixed(4 * m_total);
            NGX_CUDA_TRY(cudaMemcpyAsync(fixed.data(), extra.grad_cpl, fixed.size() * 8, cudaMemcpyDeviceToHost, g->stream));
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            for (int64_t gi = 0; gi < count; ++gi) {
                const GraphPart& part = g->parts[static_cast<size_t>(gi)];
                const double r = static_cast<double>(results[gi].reached_pairs);
                for (int64_t e = 0; e < part.m_user; ++e) {
                    const size_t i = static_cast<size_t>(part.user_arc_off + e);
                    if (dcpl != nullptr) dcpl[i] = fixed_value(fixed[2 * i], fixed[2 * i + 1]) / r;
                    if (deff != nullptr) deff[i] = -fixed_value(fixed[2 * m_total + 2 * i], fixed[2 * m_total + 2 * i + 1]) / r;
                }
            }
        }
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        return NGX_OK;
    });
}

int ngx_batch_autotune(ngx_graph* g, int task, double* class_scales) {
    return guard_host("ngx_batch_autotune", [&]() -> int {
        if (g == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_batch_autotune: batch is NULL");
        }
        const int mode = task_mode(task);
        if (mode < 0) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_batch_autotune: unknown task");
        }
        NGX_CUDA_TRY(cudaSetDevice(g->device));
        *g->h_abort = 0;
        static const double kScales[] = { 0.125, 0.25, 0.5, 1.0, 2.0, 4.0 };
        g->tuned[mode] = ngx_tuning{};
        // the graph of each size class whose first wave is timed: its median-size member
        int32_t heaviest = -1;
        double heaviest_work = -1.0;
        std::vector<int32_t> probe(NGX_SIZE_CLASSES, -1);
        for (int c = 0; c < NGX_SIZE_CLASSES; ++c) {
            std::vector<int32_t> members;
            double work = 0.0;
            for (size_t i = 0; i < g->parts.size(); ++i) {
                if (size_class(g->parts[i].n) == c && g->parts[i].n > 0) {
                    members.push_back(static_cast<int32_t>(i));
                    work += static_cast<double>(g->parts[i].n) * static_cast<double>(g->parts[i].m_stored);
                }
            }
            if (class_scales != nullptr) {
                class_scales[c] = 0.0;
            }
            if (members.empty()) {
                continue;
            }
            std::sort(members.begin(), members.end(), [&](int32_t a, int32_t b) { return g->parts[static_cast<size_t>(a)].n < g->parts[static_cast<size_t>(b)].n; });
            probe[static_cast<size_t>(c)] = members[members.size() / 2];
            if (work > heaviest_work) {
                heaviest_work = work;
                heaviest = c;
            }
        }
        // bucket width per size class, with the default launch shape
        ngx_apsp_opts aopts{};
        aopts.metric = NGX_METRIC_REGULAR;
        aopts.mode = NGX_MODE_BATCHED;
        for (int c = 0; c < NGX_SIZE_CLASSES; ++c) {
            if (probe[static_cast<size_t>(c)] < 0) {
                continue;
            }
            double best_rate = -1.0, best_scale = 1.0;
            const GraphPart& probe_part = g->parts[static_cast<size_t>(probe[static_cast<size_t>(c)])];
            const double own = default_delta_scale(probe_part.n, probe_part.m_stored);  // the untuned width, tried too
            for (const double scale : { own, kScales[0], kScales[1], kScales[2], kScales[3], kScales[4], kScales[5] }) {
                double rate = 0.0;
                if (const int rc = time_wave(g, mode, probe[static_cast<size_t>(c)], scale, aopts, &rate); rc != NGX_OK) {
                    return rc;
                }
                if (rate > best_rate) {
                    best_rate = rate;
                    best_scale = scale;
                }
            }
            g->class_scale[c] = best_scale;
            if (class_scales != nullptr) {
                class_scales[c] = best_scale;
            }
        }
        // one launch shape for the whole batch (one launch runs every graph): block shape, then CTAs per tile, timed on
        // the size class that holds most of the batch's work
        if (heaviest >= 0) {
            const int32_t gi = probe[static_cast<size_t>(heaviest)];
            const double scale = g->class_scale[heaviest];
            struct Shape {
                int block, per_sm;
            };
            static const Shape kShapes[] = { { 512, 2 }, { 384, 2 }, { 256, 3 }, { 256, 4 } };
            double best_rate = -1.0;
            Shape best_shape = kShapes[0];
            int trials = 0;
            for (const Shape& sh : kShapes) {
                aopts.block_threads = sh.block;
                aopts.ctas_per_sm = sh.per_sm;
                aopts.tile_ctas = 1;
                double rate = 0.0;
                if (const int rc = time_wave(g, mode, gi, scale, aopts, &rate); rc != NGX_OK) {
                    return rc;
                }
                ++trials;
                if (rate > best_rate) {
                    best_rate = rate;
                    best_shape = sh;
                }
            }
            int best_group = 1;
            for (const int gs : { 0, 2, 4 }) {
                // groups of several CTAs per tile run with the default block shape; 0 = the library's own rule (by L2
                // residency and the slots memory affords), which is what a run with tile_ctas 0 gets
                aopts.block_threads = kShapes[0].block;
                aopts.ctas_per_sm = kShapes[0].per_sm;
                aopts.tile_ctas = gs;
                double rate = 0.0;
                if (const int rc = time_wave(g, mode, gi, scale, aopts, &rate); rc != NGX_OK) {
                    return rc;
                }
                ++trials;
                if (rate > best_rate) {
                    best_rate = rate;
                    best_group = gs;
                    best_shape = kShapes[0];
                }
            }
            ngx_tuning& t = g->tuned[mode];
            t.delta_scale = scale;
            t.block_threads = best_shape.block;
            t.ctas_per_sm = best_shape.per_sm;
            t.tile_ctas = best_group;
            t.trials = trials;
            t.gteps = best_rate / 1e6;
        }
        return NGX_OK;
    });
}

int ngx_graph_tuning(const ngx_graph* g, int task, ngx_tuning* out) {
    if (g == nullptr || out == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_tuning: graph or out is NULL");
    }
    const int mode = task_mode(task);
    if (mode < 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_tuning: unknown task");
    }
    *out = g->tuned[mode];
    return NGX_OK;
}

int ngx_graph_update_weights(ngx_graph* g, const double* w) {
    return guard_host("ngx_graph_update_weights", [&]() -> int {
        if (g == nullptr || (w == nullptr && g->m_user > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_update_weights: graph or w is NULL");
        }
        NGX_CUDA_TRY(cudaSetDevice(g->device));
        if (const int rc = ensure_stored_of_user(g); rc != NGX_OK) {
            return rc;
        }
        const size_t m = static_cast<size_t>(g->m_stored);
        std::vector<Arc> regular(m), inverse(m), rarcs(m);
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        NGX_CUDA_TRY(cudaMemcpy(regular.data(), g->d_arcs_regular, m * sizeof(Arc), cudaMemcpyDeviceToHost));
        NGX_CUDA_TRY(cudaMemcpy(rarcs.data(), g->d_rarcs, m * sizeof(Arc), cudaMemcpyDeviceToHost));
        for (int64_t e = 0; e < g->m_user; ++e) {
            const int32_t stored = g->stored_of_user[static_cast<size_t>(e)];
            const double a = std::fabs(w[e]);
            if (!std::isfinite(w[e]) || (stored < 0) != (a == 0.0)) {
                return fail(NGX_INVALID_ARGUMENT, "ngx_graph_update_weights: arc " + std::to_string(e) + " is non-finite or changes between zero and non-zero");
            }
            if (stored >= 0) {
                regular[static_cast<size_t>(stored)].len = a;
            }
        }
        double sum_regular = 0.0, sum_inverse = 0.0, min_regular = INFINITY, max_regular = 0.0;
        for (size_t e = 0; e < m; ++e) {
            inverse[e] = regular[e];
            inverse[e].len = 1.0 / regular[e].len;
            sum_regular += regular[e].len;
            sum_inverse += inverse[e].len;
            min_regular = std::min(min_regular, regular[e].len);
            max_regular = std::max(max_regular, regular[e].len);
        }
        for (size_t r = 0; r < m; ++r) {
            rarcs[r].len = regular[static_cast<size_t>(rarcs[r].id)].len;
        }
        for (GraphPart& part : g->parts) {
            double sr = 0.0, si = 0.0;
            for (int64_t e = 0; e < part.m_user; ++e) {
                const int32_t stored = g->stored_of_user[static_cast<size_t>(part.user_arc_off + e)];
                if (stored >= 0) {
                    sr += regular[static_cast<size_t>(stored)].len;
                    si += inverse[static_cast<size_t>(stored)].len;
                }
            }
            if (part.m_stored > 0) {
                part.mean_len_regular = sr / static_cast<double>(part.m_stored);
                part.mean_len_inverse = si / static_cast<double>(part.m_stored);
            }
        }
        if (m > 0) {
            g->mean_len_regular = sum_regular / static_cast<double>(m);
            g->mean_len_inverse = sum_inverse / static_cast<double>(m);
            g->min_len_regular = min_regular;
            g->max_len_regular = max_regular;
            NGX_CUDA_TRY(cudaMemcpy(g->d_arcs_regular, regular.data(), m * sizeof(Arc), cudaMemcpyHostToDevice));
            NGX_CUDA_TRY(cudaMemcpy(g->d_arcs_inverse, inverse.data(), m * sizeof(Arc), cudaMemcpyHostToDevice));
            NGX_CUDA_TRY(cudaMemcpy(g->d_rarcs, rarcs.data(), m * sizeof(Arc), cudaMemcpyHostToDevice));
        }
        return NGX_OK;
    });
}

}  // extern "C"
