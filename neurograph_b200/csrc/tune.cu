// Autotuning of a single-graph handle (ngx_graph_autotune): bucket width, block shape and CTAs per source tile.
//
// No reference counterpart: the reference runs one Dijkstra per source and has no launch parameters; its
// delta-stepping takes a fixed delta from the command line (source/neurograph.cpp:507-515). Here the choices only
// change speed (the relaxation fixed point, the exact sums and the fixed-point betweenness do not depend on them), so
// they are timed on a sample of the graph's own all-sources order and the fastest is kept in the handle.

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_run.h"

namespace ngx {
namespace {

struct Shape {
    int block_threads;
    int ctas_per_sm;
};

// One timed run of the task over `sources` with the given options; returns traversed arcs per millisecond.
int trial(ngx_graph* g, int task, const std::vector<int64_t>& sources, double delta, const Shape& shape, int tile_ctas, double* rate) {
    ngx_apsp_opts o{};
    o.metric = NGX_METRIC_REGULAR;
    o.mode = NGX_MODE_BATCHED;
    o.sources = sources.data();
    o.num_sources = static_cast<int64_t>(sources.size());
    o.delta = delta;
    o.block_threads = shape.block_threads;
    o.ctas_per_sm = shape.ctas_per_sm;
    o.tile_ctas = tile_ctas;
    ngx_apsp_result r{};
    int rc = NGX_OK;
    if (task == NGX_TASK_APSP) {
        rc = ngx_apsp(g, &o, &r);
    } else if (task == NGX_TASK_BRANDES) {
        std::vector<double> bc(static_cast<size_t>(std::max<int64_t>(1, g->n)));
        rc = ngx_brandes(g, &o, bc.data(), &r);
    } else {
        std::vector<double> dcpl(static_cast<size_t>(std::max<int64_t>(1, g->m_user))), deff(dcpl.size());
        rc = ngx_apsp_grad(g, &o, dcpl.data(), deff.data(), &r);
    }
    *rate = rc == NGX_OK && r.kernel_ms > 0.0 ? static_cast<double>(r.traversed_arcs) / r.kernel_ms : 0.0;
    return rc;
}

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_graph_autotune(ngx_graph* g, int task, int64_t sample_sources, ngx_tuning* best) {
    return guard_host("ngx_graph_autotune", [&]() -> int {
        if (g == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_autotune: graph is NULL");
        }
        if (task != NGX_TASK_APSP && task != NGX_TASK_BRANDES && task != NGX_TASK_GRAD) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_autotune: unknown task");
        }
        if (g->parts.size() != 1) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_autotune: this handle holds a batch of graphs: use ngx_batch_autotune");
        }
        if (sample_sources < 0) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_autotune: sample_sources is negative");
        }
        NGX_CUDA_TRY(cudaSetDevice(g->device));
        if (const int rc = ensure_source_order(g); rc != NGX_OK) {
            return rc;
        }
        ngx_tuning& t = g->tuned[task];
        t = ngx_tuning{};  // trials run untuned
        const int64_t wave = static_cast<int64_t>(g->sm_count) * 2 * kTile;
        const int64_t k = std::min<int64_t>(g->n, sample_sources > 0 ? sample_sources : wave);
        if (k == 0) {
            t.delta_scale = default_delta_scale(g->parts[0].n, g->parts[0].m_stored);
            t.block_threads = 512;
            t.ctas_per_sm = 2;
            t.tile_ctas = 1;
            if (best != nullptr) {
                *best = t;
            }
            return NGX_OK;
        }
        const std::vector<int64_t> sources(g->source_order.begin(), g->source_order.begin() + k);
        const double mean = g->parts[0].mean_len_regular;
        // bucket widths: the library's default for this graph's degree first, then fixed multiples of the mean length
        const double kScales[] = { default_delta_scale(g->parts[0].n, g->parts[0].m_stored), 0.125, 0.25, 0.5, 1.0, 2.0 };
        static const Shape kShapes[] = { { 512, 2 }, { 384, 2 }, { 256, 3 }, { 256, 4 } };
        const int tiles = static_cast<int>((k + kTile - 1) / kTile);
        // CTAs per tile: the library's own choice (0: the bucket-width trials run with it, as untuned runs do), 1, 2,
        // 4, 8, and the size at which the sample's tiles fill the resident CTAs
        std::vector<int> groups = { 1, 2, 4, 8 };
        const int resident = g->sm_count * 2;
        if (tiles < resident) {
            groups.push_back(std::max(1, resident / tiles));
        }
        std::sort(groups.begin(), groups.end());
        groups.erase(std::unique(groups.begin(), groups.end()), groups.end());

        double best_rate = -1.0;
        double scale = 1.0;
        Shape shape = kShapes[0];
        int tile_ctas = 0;
        int trials = 0;
        // one parameter at a time: bucket width, then block shape, then CTAs per tile
        for (const double sc : kScales) {
            double rate = 0.0;
            if (const int rc = trial(g, task, sources, pick_delta(mean, 0.0, sc), shape, tile_ctas, &rate); rc != NGX_OK) {
                return rc;
            }
            ++trials;
            if (rate > best_rate) {
                best_rate = rate;
                scale = sc;
            }
        }
        for (const Shape& sh : kShapes) {
            if (sh.block_threads == shape.block_threads && sh.ctas_per_sm == shape.ctas_per_sm) {
                continue;
            }
            double rate = 0.0;
            if (const int rc = trial(g, task, sources, pick_delta(mean, 0.0, scale), sh, tile_ctas, &rate); rc != NGX_OK) {
                return rc;
            }
            ++trials;
            if (rate > best_rate) {
                best_rate = rate;
                shape = sh;
            }
        }
        // groups of several CTAs per tile run with the default block shape (512 x 2)
        for (const int gs : groups) {
            double rate = 0.0;
            if (const int rc = trial(g, task, sources, pick_delta(mean, 0.0, scale), kShapes[0], gs, &rate); rc != NGX_OK) {
                return rc;
            }
            ++trials;
            if (rate > best_rate) {
                best_rate = rate;
                tile_ctas = gs;
                shape = kShapes[0];
            }
        }
        t.delta_scale = scale;
        t.block_threads = shape.block_threads;
        t.ctas_per_sm = shape.ctas_per_sm;
        t.tile_ctas = tile_ctas;
        t.trials = trials;
        t.gteps = best_rate / 1e6;  // arcs per ms -> 1e9 arcs per s
        if (best != nullptr) {
            *best = t;
        }
        return NGX_OK;
    });
}

}  // extern "C"
