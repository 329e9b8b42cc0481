// Graph handle: validation, CSR + reverse CSR upload, status strings and error reporting.
//
// Replaces the reference's DistributedGraph adjacency (source/graph/DistributedGraph.{h,cpp}): per-rank RMA windows of
// 12-byte {rank, id, weight} arcs read through get_out_arcs (DistributedGraph.h:275-311) become one device-resident
// CSR of 16-byte {target, arc id, FP64 length} records, plus a reverse CSR for the pull passes of Brandes and the
// gradient. Zero-weight arcs are left out, as DistributedGraph::upload_out_arcs skips them (DistributedGraph.cpp:223).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"

namespace ngx {

namespace {
thread_local std::string last_error_message;
}

void set_last_error(const std::string& message) { last_error_message = message; }

int fail(int status, const std::string& message) {
    set_last_error(message);
    return status;
}

int cuda_fail(cudaError_t err, const char* what) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(err));
    return err == cudaErrorMemoryAllocation ? NGX_OUT_OF_MEMORY : NGX_CUDA_ERROR;
}

size_t workspace_budget(const ngx_graph* g) {
    size_t free_bytes = 0, total_bytes = 0;
    if (cudaMemGetInfo(&free_bytes, &total_bytes) != cudaSuccess) {
        return 0;
    }
    size_t usable = free_bytes + g->workspace_bytes;
    usable = usable > (size_t(1) << 30) ? usable - (size_t(1) << 30) : usable / 2;  // keep 1 GiB headroom
    if (g->memory_budget != 0 && g->memory_budget < usable) {
        usable = static_cast<size_t>(g->memory_budget);
    }
    return usable;
}

int ensure_workspace(ngx_graph* g, size_t bytes) {
    if (bytes <= g->workspace_bytes) {
        return NGX_OK;
    }
    if (g->d_workspace != nullptr) {
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (g->graph_exec != nullptr) {
            // a captured batch run refers to the old workspace
            cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(g->graph_exec));
            g->graph_exec = nullptr;
            g->graph_key = 0;
        }
        NGX_CUDA_TRY(cudaFree(g->d_workspace));
        g->d_workspace = nullptr;
        g->workspace_bytes = 0;
    }
    NGX_CUDA_TRY(cudaMalloc(&g->d_workspace, bytes));
    g->workspace_bytes = bytes;
    return NGX_OK;
}

int grow_buffer(ngx_graph* g, void** buf, size_t* cap, size_t bytes) {
    if (bytes <= *cap && *buf != nullptr) {
        return NGX_OK;
    }
    if (*buf != nullptr) {
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        NGX_CUDA_TRY(cudaFree(*buf));
        *buf = nullptr;
        *cap = 0;
    }
    const size_t want = bytes + bytes / 4 + 256;  // headroom for source lists that grow a little between calls
    NGX_CUDA_TRY(cudaMalloc(buf, want));
    *cap = want;
    return NGX_OK;
}

namespace {

// Tiles of nearby sources: from each unassigned seed (in id order), the seed and its lightest unassigned out-neighbours,
// then theirs (one hop at a time, lightest first, continuing from the 64 lightest), until a tile of 32 is full or the
// search has looked at 256 vertices. Close sources reach most vertices at similar distances, so more of them are pending on a vertex when it is
// expanded, and one pass over its arcs serves more of them. O(n * 256 * degree) at worst, on the host.
void append_source_order(int64_t n, const int64_t* row_ptr, const Arc* arcs, std::vector<int32_t>& order) {
    std::vector<uint8_t> assigned(static_cast<size_t>(n), 0);
    std::vector<int32_t> seen_stamp(static_cast<size_t>(n), -1);
    std::vector<int32_t> frontier, next;
    std::vector<std::pair<double, int32_t>> cand;
    int32_t stamp = 0;
    for (int64_t seed = 0; seed < n; ++seed) {
        if (assigned[static_cast<size_t>(seed)]) {
            continue;
        }
        ++stamp;
        int taken = 0;
        int looked = 1;
        frontier.assign(1, static_cast<int32_t>(seed));
        seen_stamp[static_cast<size_t>(seed)] = stamp;
        assigned[static_cast<size_t>(seed)] = 1;
        order.push_back(static_cast<int32_t>(seed));
        ++taken;
        while (taken < kTile && !frontier.empty() && looked < 256) {
            cand.clear();
            for (const int32_t u : frontier) {
                for (int64_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
                    const int32_t v = arcs[e].col;
                    if (seen_stamp[static_cast<size_t>(v)] != stamp) {
                        seen_stamp[static_cast<size_t>(v)] = stamp;
                        cand.emplace_back(arcs[e].len, v);
                    }
                }
            }
            std::sort(cand.begin(), cand.end());
            next.clear();
            for (const auto& c : cand) {
                ++looked;
                if (next.size() < 64) {
                    next.push_back(c.second);  // the next hop continues from the lightest candidates only
                }
                if (!assigned[static_cast<size_t>(c.second)]) {
                    assigned[static_cast<size_t>(c.second)] = 1;
                    order.push_back(c.second);
                    if (++taken == kTile) {
                        break;
                    }
                }
            }
            frontier.swap(next);
        }
    }
}

void release(ngx_graph* g) {
    if (g == nullptr) {
        return;
    }
    cudaSetDevice(g->device);
    if (g->stream != nullptr) {
        cudaStreamSynchronize(g->stream);
    }
    cudaFree(g->d_row_ptr);
    cudaFree(g->d_arcs_regular);
    cudaFree(g->d_arcs_inverse);
    cudaFree(g->d_rrow_ptr);
    cudaFree(g->d_rarcs);
    cudaFree(g->d_arc_src);
    cudaFree(g->d_workspace);
    cudaFree(g->d_items);
    cudaFree(g->d_persistent);
    cudaFree(g->d_call_out);
    cudaFree(g->d_call_dag);
    if (g->graph_exec != nullptr) {
        cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(g->graph_exec));
    }
    if (g->h_abort != nullptr) {
        cudaFreeHost(g->h_abort);
    }
    if (g->own_stream != nullptr) {
        cudaStreamDestroy(g->own_stream);
    }
    delete g;
}

int validate(const ngx_csr* csr) {
    if (csr == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: csr is NULL");
    }
    if (csr->n < 0 || csr->m < 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: negative n or m");
    }
    if (csr->n >= (int64_t(1) << 31) - 1 || csr->m >= (int64_t(1) << 31) - 1) {
        return fail(NGX_UNSUPPORTED, "ngx_graph_create: n and m must be below 2^31 - 1 (int32 vertex and arc ids)");
    }
    if (csr->n > 0 && csr->row_ptr == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: row_ptr is NULL");
    }
    if (csr->m > 0 && (csr->col == nullptr || csr->w == nullptr)) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: col or w is NULL");
    }
    if (csr->n == 0) {
        return csr->m == 0 ? NGX_OK : fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: arcs without vertices");
    }
    if (csr->row_ptr[0] != 0 || csr->row_ptr[csr->n] != csr->m) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: row_ptr must start at 0 and end at m");
    }
    for (int64_t u = 0; u < csr->n; ++u) {
        if (csr->row_ptr[u + 1] < csr->row_ptr[u]) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: row_ptr is not monotone at vertex " + std::to_string(u));
        }
    }
    for (int64_t e = 0; e < csr->m; ++e) {
        if (csr->col[e] < 0 || csr->col[e] >= csr->n) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: arc " + std::to_string(e) + " has an out-of-range target");
        }
        if (!std::isfinite(csr->w[e])) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: arc " + std::to_string(e) + " has a non-finite weight");
        }
    }
    return NGX_OK;
}

}  // namespace

int create_graphs(const ngx_csr* csrs, int64_t count, int device, ngx_graph** out) {
    if (out == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: out is NULL");
    }
    *out = nullptr;
    if (csrs == nullptr || count <= 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: no graphs");
    }
    int64_t n_total = 0, m_total = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (const int rc = validate(&csrs[i]); rc != NGX_OK) {
            return count > 1 ? fail(rc, "graph " + std::to_string(i) + ": " + ngx_last_error()) : rc;
        }
        n_total += csrs[i].n;
        m_total += csrs[i].m;
    }
    if (n_total >= (int64_t(1) << 31) - 1 || m_total >= (int64_t(1) << 31) - 1) {
        return fail(NGX_UNSUPPORTED, "ngx_graph_create: total vertices and arcs must be below 2^31 - 1");
    }
    int device_count = 0;
    NGX_CUDA_TRY(cudaGetDeviceCount(&device_count));
    if (device < 0 || device >= device_count) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: no CUDA device " + std::to_string(device));
    }
    NGX_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop{};
    NGX_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        return fail(NGX_UNSUPPORTED, std::string("ngx_graph_create: the kernels are built for sm_100a (B200); device is ") + prop.name);
    }

    auto* g = new (std::nothrow) ngx_graph{};
    if (g == nullptr) {
        return fail(NGX_OUT_OF_MEMORY, "ngx_graph_create: host allocation failed");
    }
    g->device = device;
    g->sm_count = prop.multiProcessorCount;
    g->n_total = n_total;
    g->m_user = m_total;

    const auto finish = [&](int rc) -> int {
        if (rc != NGX_OK) {
            release(g);
            return rc;
        }
        *out = g;
        return NGX_OK;
    };

    if (cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&g->h_abort), sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&g->d_abort), g->h_abort, 0) != cudaSuccess) {
        return finish(fail(NGX_CUDA_ERROR, "ngx_graph_create: stream or abort flag setup failed"));
    }
    *g->h_abort = 0;
    g->stream = g->own_stream;

    // Host compaction, graph after graph: drop zero-weight arcs, keep each arc's caller index (graphs numbered
    // consecutively), precompute both metrics' lengths. Row offsets are global arc indices; targets stay graph-local.
    std::vector<int64_t> row_ptr;
    std::vector<int64_t> rrow_ptr;
    std::vector<Arc> regular;
    std::vector<Arc> inverse;
    std::vector<int32_t> arc_src;
    row_ptr.reserve(static_cast<size_t>(n_total + count));
    rrow_ptr.reserve(static_cast<size_t>(n_total + count));
    regular.reserve(static_cast<size_t>(m_total));
    inverse.reserve(static_cast<size_t>(m_total));
    std::vector<Arc> rarcs(static_cast<size_t>(m_total));
    g->stored_of_user.assign(static_cast<size_t>(m_total), -1);
    double sum_regular = 0.0, sum_inverse = 0.0;
    double min_regular = INFINITY, max_regular = 0.0;
    int64_t user_arc_off = 0, vertex_off = 0;
    g->parts.resize(static_cast<size_t>(count));
    for (int64_t gi = 0; gi < count; ++gi) {
        const ngx_csr* csr = &csrs[gi];
        const int64_t n = csr->n;
        GraphPart& part = g->parts[static_cast<size_t>(gi)];
        part.n = n;
        part.m_user = csr->m;
        part.row_off = static_cast<int64_t>(row_ptr.size());
        part.user_arc_off = user_arc_off;
        part.vertex_off = vertex_off;
        const int64_t first_arc = static_cast<int64_t>(regular.size());
        std::vector<int64_t> in_degree(static_cast<size_t>(n) + 1, 0);
        double part_regular = 0.0, part_inverse = 0.0;
        row_ptr.push_back(first_arc);
        for (int64_t u = 0; u < n; ++u) {
            for (int64_t e = csr->row_ptr[u]; e < csr->row_ptr[u + 1]; ++e) {
                const double a = std::fabs(csr->w[e]);
                if (a == 0.0) {
                    continue;
                }
                const int32_t v = csr->col[e];
                const int32_t id = static_cast<int32_t>(user_arc_off + e);
                g->stored_of_user[static_cast<size_t>(id)] = static_cast<int32_t>(regular.size());
                regular.push_back(Arc{ v, id, a });
                arc_src.push_back(static_cast<int32_t>(u));
                inverse.push_back(Arc{ v, id, 1.0 / a });
                part_regular += a;
                part_inverse += 1.0 / a;
                min_regular = std::min(min_regular, a);
                max_regular = std::max(max_regular, a);
                in_degree[static_cast<size_t>(v) + 1] += 1;
            }
            row_ptr.push_back(static_cast<int64_t>(regular.size()));
            g->max_out_degree = std::max(g->max_out_degree, row_ptr.back() - row_ptr[row_ptr.size() - 2]);
        }
        part.m_stored = static_cast<int64_t>(regular.size()) - first_arc;
        if (part.m_stored > 0) {
            part.mean_len_regular = part_regular / static_cast<double>(part.m_stored);
            part.mean_len_inverse = part_inverse / static_cast<double>(part.m_stored);
        }
        sum_regular += part_regular;
        sum_inverse += part_inverse;
        // reverse CSR of this graph by counting sort over targets; within a target, ascending source order
        const size_t rbase = rrow_ptr.size();
        rrow_ptr.push_back(first_arc);
        for (int64_t v = 0; v < n; ++v) {
            rrow_ptr.push_back(rrow_ptr.back() + in_degree[static_cast<size_t>(v) + 1]);
        }
        std::vector<int64_t> fill(rrow_ptr.begin() + static_cast<std::ptrdiff_t>(rbase), rrow_ptr.end() - 1);
        for (int64_t u = 0; u < n; ++u) {
            for (int64_t e = row_ptr[static_cast<size_t>(part.row_off + u)]; e < row_ptr[static_cast<size_t>(part.row_off + u + 1)]; ++e) {
                const Arc& a = regular[static_cast<size_t>(e)];
                // the reverse record keeps the arc's index in the stored forward CSR (its caller index is arcs[e].id)
                rarcs[static_cast<size_t>(fill[static_cast<size_t>(a.col)]++)] = Arc{ static_cast<int32_t>(u), static_cast<int32_t>(e), a.len };
            }
        }
        // arcs of this graph's rows, with graph-local row offsets
        {
            std::vector<int64_t> local_rows(static_cast<size_t>(n) + 1);
            for (int64_t v = 0; v <= n; ++v) {
                local_rows[static_cast<size_t>(v)] = row_ptr[static_cast<size_t>(part.row_off + v)] - first_arc;
            }
            append_source_order(n, local_rows.data(), regular.data() + first_arc, g->source_order);
        }
        g->n = std::max(g->n, n);
        user_arc_off += csr->m;
        vertex_off += n;
    }
    const int64_t m = static_cast<int64_t>(regular.size());
    rarcs.resize(static_cast<size_t>(m));
    g->m_stored = m;
    if (m > 0) {
        g->mean_len_regular = sum_regular / static_cast<double>(m);
        g->mean_len_inverse = sum_inverse / static_cast<double>(m);
        g->min_len_regular = min_regular;
        g->max_len_regular = max_regular;
    }

    const auto upload = [&](auto** dst, const auto& src) -> int {
        using T = std::remove_reference_t<decltype(src[0])>;
        const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
        NGX_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), bytes));
        if (!src.empty()) {
            NGX_CUDA_TRY(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, g->stream));
        }
        return NGX_OK;
    };
    int rc = upload(&g->d_row_ptr, row_ptr);
    if (rc == NGX_OK) rc = upload(&g->d_arcs_regular, regular);
    if (rc == NGX_OK) rc = upload(&g->d_arcs_inverse, inverse);
    if (rc == NGX_OK) rc = upload(&g->d_rrow_ptr, rrow_ptr);
    if (rc == NGX_OK) rc = upload(&g->d_rarcs, rarcs);
    if (rc == NGX_OK) rc = upload(&g->d_arc_src, arc_src);
    if (rc == NGX_OK) {
        const cudaError_t err = cudaStreamSynchronize(g->stream);
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "ngx_graph_create: upload");
        }
    }
    return finish(rc);
}

}  // namespace ngx

using namespace ngx;

extern "C" {

const char* ngx_status_string(int status) {
    switch (status) {
    case NGX_OK: return "ok";
    case NGX_INVALID_ARGUMENT: return "invalid argument";
    case NGX_OUT_OF_MEMORY: return "out of memory";
    case NGX_CUDA_ERROR: return "CUDA error";
    case NGX_TIMEOUT: return "iteration cap reached";
    case NGX_ABORTED: return "aborted";
    case NGX_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

int ngx_graph_source_order(const ngx_graph* graph, int64_t* order) {
    if (graph == nullptr || (order == nullptr && graph->n_total > 0)) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_source_order: graph or order is NULL");
    }
    for (size_t i = 0; i < graph->source_order.size(); ++i) {
        order[i] = graph->source_order[i];
    }
    return NGX_OK;
}

const char* ngx_last_error(void) { return last_error_message.c_str(); }

const char* ngx_version(void) {
    static const std::string version = [] {
        int runtime = 0;
        cudaRuntimeGetVersion(&runtime);
        return std::string("neurograph-b200 sm_100a, CUDA runtime ") + std::to_string(runtime / 1000) + "." + std::to_string((runtime % 1000) / 10);
    }();
    return version.c_str();
}

int ngx_graph_create(const ngx_csr* csr, int device, ngx_graph** out) {
    if (csr == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: csr is NULL");
    }
    return create_graphs(csr, 1, device, out);
}

void ngx_graph_destroy(ngx_graph* graph) { release(graph); }

int ngx_graph_size(const ngx_graph* graph, int64_t* n, int64_t* m) {
    if (graph == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_size: graph is NULL");
    }
    if (n != nullptr) *n = graph->n_total;
    if (m != nullptr) *m = graph->m_user;
    return NGX_OK;
}

int ngx_graph_request_abort(ngx_graph* graph) {
    if (graph == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_request_abort: graph is NULL");
    }
    *reinterpret_cast<volatile int*>(graph->h_abort) = 1;
    return NGX_OK;
}

int ngx_graph_set_stream(ngx_graph* graph, void* stream) {
    if (graph == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_set_stream: graph is NULL");
    }
    NGX_CUDA_TRY(cudaSetDevice(graph->device));
    NGX_CUDA_TRY(cudaStreamSynchronize(graph->stream));
    graph->stream = stream != nullptr ? static_cast<cudaStream_t>(stream) : graph->own_stream;
    return NGX_OK;
}

int ngx_graph_set_memory_budget(ngx_graph* graph, uint64_t bytes) {
    if (graph == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_set_memory_budget: graph is NULL");
    }
    graph->memory_budget = bytes;
    return NGX_OK;
}

}  // extern "C"
