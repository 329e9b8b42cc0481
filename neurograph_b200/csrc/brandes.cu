// Host side of the Brandes and adjoint runs (ngx_brandes, ngx_apsp_grad).
//
// Replaces BetweennessCentrality::compute_average_betweenness_centrality's per-source loop over
// BrandesVariant::accumulate_from_source (source/metrics/paths/BetweennessCentrality.h:46-80,
// BetweennessCentralityVariants/BrandesVariant.h:50-159): one persistent launch computes, per source tile, the
// distances, the APSP summaries, sigma and the dependencies, and accumulates betweenness (or the per-arc gradient).

#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "brandes_kernels.cuh"
#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_run.h"

namespace ngx {
namespace {

int dag_run(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, ngx_apsp_result* result, std::vector<unsigned long long>& host_bc,
            std::vector<unsigned long long>& host_cpl, std::vector<unsigned long long>& host_eff, uint64_t* reached_pairs) {
    if (const int rc = check_opts(g, opts); rc != NGX_OK) {
        return rc;
    }
    if (opts->metric != NGX_METRIC_REGULAR) {
        return fail(NGX_UNSUPPORTED, "betweenness and the gradient are defined for the regular metric (arc length |w|)");
    }
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    ngx_apsp_opts o = *opts;
    o.mode = NGX_MODE_BATCHED;
    const size_t n = static_cast<size_t>(g->n);
    const size_t m = static_cast<size_t>(g->m_user);
    DagOutputs extra;
    const size_t bc_words = tile_mode == kModeBrandes ? 2 * n : 0;
    const size_t grad_words = tile_mode == kModeGrad ? 2 * m : 0;
    const size_t words = 1 + bc_words + 2 * grad_words;
    if (const int rc = grow_buffer(g, &g->d_call_dag, &g->call_dag_bytes, words * 8); rc != NGX_OK) {
        return rc;
    }
    unsigned long long* block = static_cast<unsigned long long*>(g->d_call_dag);
    NGX_CUDA_TRY(cudaMemsetAsync(block, 0, words * 8, g->stream));
    extra.sigma_inexact = reinterpret_cast<int*>(block);
    if (bc_words != 0) {
        extra.bc = block + 1;
    }
    if (grad_words != 0) {
        extra.grad_cpl = block + 1;
        extra.grad_eff = block + 1 + grad_words;
    }
    ngx_apsp_result scratch{};
    ngx_apsp_result* r = result != nullptr ? result : &scratch;
    int rc = run_apsp(g, &o, r, nullptr, tile_mode, &extra);
    if (rc == NGX_OK) {
        // sigma was pushed with atomics; if any path count reached 2^53 the sums may depend on the order of the
        // atomics, so rerun with the order-defined pull form
        int inexact = 0;
        cudaError_t err = cudaMemcpyAsync(&inexact, extra.sigma_inexact, sizeof(int), cudaMemcpyDeviceToHost, g->stream);
        if (err == cudaSuccess) {
            err = cudaStreamSynchronize(g->stream);
        }
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "reading the sigma exactness flag");
        } else if (inexact != 0) {
            const double first_ms = r->kernel_ms;
            extra.sigma_pull = 1;
            NGX_CUDA_TRY(cudaMemsetAsync(block, 0, words * 8, g->stream));
            rc = run_apsp(g, &o, r, nullptr, tile_mode, &extra);
            r->kernel_ms += first_ms;
        }
    }
    if (rc == NGX_OK) {
        host_bc.resize(bc_words);
        host_cpl.resize(grad_words);
        host_eff.resize(grad_words);
        cudaError_t err = cudaSuccess;
        if (bc_words != 0) {
            err = cudaMemcpyAsync(host_bc.data(), extra.bc, bc_words * 8, cudaMemcpyDeviceToHost, g->stream);
        }
        if (err == cudaSuccess && grad_words != 0) {
            err = cudaMemcpyAsync(host_cpl.data(), extra.grad_cpl, grad_words * 8, cudaMemcpyDeviceToHost, g->stream);
        }
        if (err == cudaSuccess && grad_words != 0) {
            err = cudaMemcpyAsync(host_eff.data(), extra.grad_eff, grad_words * 8, cudaMemcpyDeviceToHost, g->stream);
        }
        if (err == cudaSuccess) {
            err = cudaStreamSynchronize(g->stream);
        }
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "copying betweenness / gradients");
        }
        *reached_pairs = r->reached_pairs;
    }
    cudaStreamSynchronize(g->stream);
    return rc;
}

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_brandes(ngx_graph* graph, const ngx_apsp_opts* opts, double* bc, ngx_apsp_result* result) {
    if (graph == nullptr || opts == nullptr || (bc == nullptr && graph->n > 0)) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_brandes: graph, opts or bc is NULL");
    }
    std::vector<unsigned long long> fixed, unused_a, unused_b;
    uint64_t reached = 0;
    const int rc = dag_run(graph, opts, kModeBrandes, result, fixed, unused_a, unused_b, &reached);
    if (rc != NGX_OK) {
        return rc;
    }
    for (int64_t v = 0; v < graph->n; ++v) {
        bc[v] = fixed.empty() ? 0.0 : fixed_value(fixed[static_cast<size_t>(2 * v)], fixed[static_cast<size_t>(2 * v + 1)]);
    }
    return NGX_OK;
}

int ngx_apsp_grad(ngx_graph* graph, const ngx_apsp_opts* opts, double* dcpl, double* deff, ngx_apsp_result* result) {
    if (graph == nullptr || opts == nullptr || ((dcpl == nullptr || deff == nullptr) && graph->m_user > 0)) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_grad: graph, opts, dcpl or deff is NULL");
    }
    std::vector<unsigned long long> unused, fixed_cpl, fixed_eff;
    uint64_t reached = 0;
    const int rc = dag_run(graph, opts, kModeGrad, result, unused, fixed_cpl, fixed_eff, &reached);
    if (rc != NGX_OK) {
        return rc;
    }
    const double r = static_cast<double>(reached);
    for (int64_t e = 0; e < graph->m_user; ++e) {
        const size_t i = static_cast<size_t>(2 * e);
        const double c = fixed_cpl.empty() ? 0.0 : fixed_value(fixed_cpl[i], fixed_cpl[i + 1]);
        const double f = fixed_eff.empty() ? 0.0 : fixed_value(fixed_eff[i], fixed_eff[i + 1]);
        dcpl[e] = c / r;
        deff[e] = -f / r;
    }
    return NGX_OK;
}

}  // extern "C"
