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

// 128-bit fixed-point sums -> doubles, scaled: out[i] = sign * value(sum[i]) / divisor (IEEE division, as on the host).
__global__ void fixed_to_double_kernel(const unsigned long long* sums, int64_t count, double divisor, double sign, double* out) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = fixed_value(sums[2 * i], sums[2 * i + 1]);
        out[i] = divisor == 1.0 ? sign * v : sign * v / divisor;
    }
}

int convert_fixed(ngx_graph* g, const unsigned long long* sums, int64_t count, double divisor, double sign, double* d_out, double* h_out) {
    if (count == 0) {
        return NGX_OK;
    }
    const int block = 256;
    const int64_t want = (count + block - 1) / block;
    const int grid = static_cast<int>(want < 8 * g->sm_count ? want : 8 * g->sm_count);
    fixed_to_double_kernel<<<grid, block, 0, g->stream>>>(sums, count, divisor, sign, d_out);
    NGX_CUDA_TRY(cudaGetLastError());
    NGX_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, static_cast<size_t>(count) * 8, cudaMemcpyDeviceToHost, g->stream));
    return NGX_OK;
}

// Output arrays of one Brandes / adjoint run: converted doubles, or the unconverted 128-bit fixed-point words.
struct DagHostOut {
    double* bc = nullptr;
    double* dcpl = nullptr;
    double* deff = nullptr;
    uint64_t* bc_fixed = nullptr;    // 2 n words
    uint64_t* dcpl_fixed = nullptr;  // 2 m words
    uint64_t* deff_fixed = nullptr;  // 2 m words
};

// One Brandes or adjoint run of a single-graph handle. The fixed-point sums are either converted on the device and
// copied straight into the caller's double arrays, or copied out as words (for exact merging across ranks).
int dag_run(ngx_graph* g, const ngx_apsp_opts* opts, int tile_mode, ngx_apsp_result* result, const DagHostOut& out) {
    if (const int rc = check_opts(g, opts); rc != NGX_OK) {
        return rc;
    }
    if (opts->metric != NGX_METRIC_REGULAR) {
        return fail(NGX_UNSUPPORTED, "betweenness and the gradient are defined for the regular metric (arc length |w|)");
    }
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    ngx_apsp_opts o = *opts;
    if (tile_mode != kModeBrandes || o.mode != NGX_MODE_PLAIN) {
        o.mode = NGX_MODE_BATCHED;  // the adjoint has the batched form only
    }
    const size_t n = static_cast<size_t>(g->n);
    const size_t m = static_cast<size_t>(g->m_user);
    DagOutputs extra;
    const size_t bc_words = tile_mode == kModeBrandes ? 2 * n : 0;
    const size_t grad_words = tile_mode == kModeGrad ? 2 * m : 0;
    const size_t words = 1 + bc_words + 2 * grad_words;
    const size_t out_doubles = tile_mode == kModeBrandes ? n : 2 * m;  // converted results, after the sums
    if (const int rc = grow_buffer(g, &g->d_call_dag, &g->call_dag_bytes, (words + out_doubles) * 8); rc != NGX_OK) {
        return rc;
    }
    unsigned long long* block = static_cast<unsigned long long*>(g->d_call_dag);
    double* d_out = reinterpret_cast<double*>(block + words);
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
    if (rc == NGX_OK && g->n > 0) {
        const auto copy_words = [&](uint64_t* dst, const unsigned long long* src, size_t count) -> int {
            NGX_CUDA_TRY(cudaMemcpyAsync(dst, src, 2 * count * 8, cudaMemcpyDeviceToHost, g->stream));
            return NGX_OK;
        };
        if (tile_mode == kModeBrandes && out.bc_fixed != nullptr) {
            rc = copy_words(out.bc_fixed, extra.bc, n);
        } else if (tile_mode == kModeBrandes) {
            rc = convert_fixed(g, extra.bc, static_cast<int64_t>(n), 1.0, 1.0, d_out, out.bc);
        } else if (out.dcpl_fixed != nullptr) {
            rc = copy_words(out.dcpl_fixed, extra.grad_cpl, m);
            if (rc == NGX_OK) {
                rc = copy_words(out.deff_fixed, extra.grad_eff, m);
            }
        } else {
            // dCPL/dw = c / R and dE/dw = -f / R over the R reached ordered pairs (0 / 0 = NaN without any)
            const double reached = static_cast<double>(r->reached_pairs);
            rc = convert_fixed(g, extra.grad_cpl, static_cast<int64_t>(m), reached, 1.0, d_out, out.dcpl);
            if (rc == NGX_OK) {
                rc = convert_fixed(g, extra.grad_eff, static_cast<int64_t>(m), reached, -1.0, d_out + m, out.deff);
            }
        }
        const cudaError_t err = cudaStreamSynchronize(g->stream);
        if (rc == NGX_OK && err != cudaSuccess) {
            rc = cuda_fail(err, "converting betweenness / gradients");
        }
    }
    cudaStreamSynchronize(g->stream);
    return rc;
}

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_brandes(ngx_graph* graph, const ngx_apsp_opts* opts, double* bc, ngx_apsp_result* result) {
    return guard_host("ngx_brandes", [&]() -> int {
        if (graph == nullptr || opts == nullptr || (bc == nullptr && graph->n > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_brandes: graph, opts or bc is NULL");
        }
        DagHostOut out;
        out.bc = bc;
        return dag_run(graph, opts, kModeBrandes, result, out);
    });
}

int ngx_brandes_fixed(ngx_graph* graph, const ngx_apsp_opts* opts, uint64_t* bc_fixed, ngx_apsp_result* result) {
    return guard_host("ngx_brandes_fixed", [&]() -> int {
        if (graph == nullptr || opts == nullptr || (bc_fixed == nullptr && graph->n > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_brandes_fixed: graph, opts or bc_fixed is NULL");
        }
        DagHostOut out;
        out.bc_fixed = bc_fixed;
        return dag_run(graph, opts, kModeBrandes, result, out);
    });
}

int ngx_apsp_grad(ngx_graph* graph, const ngx_apsp_opts* opts, double* dcpl, double* deff, ngx_apsp_result* result) {
    return guard_host("ngx_apsp_grad", [&]() -> int {
        if (graph == nullptr || opts == nullptr || ((dcpl == nullptr || deff == nullptr) && graph->m_user > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_grad: graph, opts, dcpl or deff is NULL");
        }
        DagHostOut out;
        out.dcpl = dcpl;
        out.deff = deff;
        return dag_run(graph, opts, kModeGrad, result, out);
    });
}

int ngx_apsp_grad_fixed(ngx_graph* graph, const ngx_apsp_opts* opts, uint64_t* dcpl_fixed, uint64_t* deff_fixed, ngx_apsp_result* result) {
    return guard_host("ngx_apsp_grad_fixed", [&]() -> int {
        if (graph == nullptr || opts == nullptr || ((dcpl_fixed == nullptr || deff_fixed == nullptr) && graph->m_user > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_apsp_grad_fixed: graph, opts, dcpl_fixed or deff_fixed is NULL");
        }
        DagHostOut out;
        out.dcpl_fixed = dcpl_fixed;
        out.deff_fixed = deff_fixed;
        return dag_run(graph, opts, kModeGrad, result, out);
    });
}

int ngx_fixed_to_double(const uint64_t* words, int64_t count, double divisor, double sign, double* out) {
    return guard_host("ngx_fixed_to_double", [&]() -> int {
        if (count < 0 || (count > 0 && (words == nullptr || out == nullptr))) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_fixed_to_double: negative count or NULL array");
        }
        for (int64_t i = 0; i < count; ++i) {
            // the same expression as fixed_to_double_kernel, so a merged sum converts to the bits of a single run
            const double v = fixed_value(words[2 * i], words[2 * i + 1]);
            out[i] = divisor == 1.0 ? sign * v : sign * v / divisor;
        }
        return NGX_OK;
    });
}

}  // extern "C"
