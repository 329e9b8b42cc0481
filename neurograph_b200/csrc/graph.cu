// Graph handle: validation, CSR + reverse CSR upload, status strings and error reporting.
//
// Replaces the reference's DistributedGraph adjacency (source/graph/DistributedGraph.{h,cpp}): per-rank RMA windows of
// 12-byte {rank, id, weight} arcs read through get_out_arcs (DistributedGraph.h:275-311) become one device-resident
// CSR of 16-byte {target, arc id, FP64 length} records, plus a reverse CSR for the pull passes of Brandes and the
// gradient. Zero-weight arcs are left out, as DistributedGraph::upload_out_arcs skips them (DistributedGraph.cpp:223).

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"
#include "ngx_threads.h"

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
// search has looked at 256 vertices. Close sources reach most vertices at similar distances, so more of them are
// pending on a vertex when it is expanded, and one pass over its arcs serves more of them. Candidates are ordered by
// (length, vertex), a strict order, and only the lightest ones a hop uses are selected and sorted: the unassigned ones
// that fill the tile and, when the hop does not fill it, the 64 that continue the search. O(n * 256 * degree) at
// worst, on the host.
void append_source_order(int64_t n, const int64_t* row_ptr, const Arc* arcs, HostVector<int32_t>& order) {
    std::vector<uint8_t> assigned(static_cast<size_t>(n), 0);
    std::vector<int32_t> seen_stamp(static_cast<size_t>(n), -1);
    std::vector<int32_t> frontier, next;
    std::vector<std::pair<double, int32_t>> cand, free_cand;
    int32_t stamp = 0;
    for (int64_t seed = 0; seed < n; ++seed) {
        if (assigned[static_cast<size_t>(seed)]) {
            continue;
        }
        ++stamp;
        int taken = 0;
        int64_t looked = 1;
        frontier.assign(1, static_cast<int32_t>(seed));
        seen_stamp[static_cast<size_t>(seed)] = stamp;
        assigned[static_cast<size_t>(seed)] = 1;
        order.push_back(static_cast<int32_t>(seed));
        ++taken;
        while (taken < kTile && !frontier.empty() && looked < 256) {
            cand.clear();
            free_cand.clear();
            for (const int32_t u : frontier) {
                for (int64_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
                    const int32_t v = arcs[e].col;
                    if (seen_stamp[static_cast<size_t>(v)] != stamp) {
                        seen_stamp[static_cast<size_t>(v)] = stamp;
                        cand.emplace_back(arcs[e].len, v);
                        if (!assigned[static_cast<size_t>(v)]) {
                            free_cand.emplace_back(arcs[e].len, v);
                        }
                    }
                }
            }
            // the unassigned candidates, lightest first, fill the tile
            const size_t need = static_cast<size_t>(kTile - taken);
            const size_t take = std::min(need, free_cand.size());
            std::partial_sort(free_cand.begin(), free_cand.begin() + static_cast<std::ptrdiff_t>(take), free_cand.end());
            for (size_t i = 0; i < take; ++i) {
                assigned[static_cast<size_t>(free_cand[i].second)] = 1;
                order.push_back(free_cand[i].second);
            }
            taken += static_cast<int>(take);
            if (taken == kTile) {
                break;
            }
            // the hop looked at every candidate; the next one continues from the 64 lightest of them
            looked += static_cast<int64_t>(cand.size());
            const size_t keep = std::min<size_t>(64, cand.size());
            std::partial_sort(cand.begin(), cand.begin() + static_cast<std::ptrdiff_t>(keep), cand.end());
            next.clear();
            for (size_t i = 0; i < keep; ++i) {
                next.push_back(cand[i].second);
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
    cudaFree(g->d_stored_of_user);
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

// Checks the sizes, pointers and row offsets of one CSR (the arcs are checked during the first pass over them).
int validate_rows(const ngx_csr* csr) {
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
    return NGX_OK;
}

// A vertex range of one graph, sized to about kChunkArcs caller arcs: the unit of the parallel passes over arcs.
constexpr int64_t kChunkArcs = int64_t(1) << 20;
struct Chunk {
    int64_t graph = 0;
    int64_t v0 = 0, v1 = 0;
    int64_t bad_arc = -1;  // first arc with an out-of-range target or a non-finite weight
    bool bad_target = false;
    int64_t max_degree = 0;
    double min_len = INFINITY, max_len = 0.0;
};

}  // namespace

int build_host_graphs(const ngx_csr* csrs, int64_t count, int threads, HostGraphs* out) {
    if (csrs == nullptr || count <= 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: no graphs");
    }
    if (threads <= 0) {
        threads = static_cast<int>(std::min<unsigned>(32u, std::max(1u, std::thread::hardware_concurrency())));
    }
    HostGraphs& h = *out;
    // rows of every graph first; the arcs of the graphs before the first bad one are checked by the first pass, so
    // that the first error in graph order is the one reported
    int64_t rows_ok = count;
    int rows_rc = NGX_OK;
    std::string rows_message;
    int64_t n_total = 0, m_total = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (const int rc = validate_rows(&csrs[i]); rc != NGX_OK) {
            rows_ok = i;
            rows_rc = rc;
            rows_message = ngx_last_error();
            break;
        }
        n_total += csrs[i].n;
        m_total += csrs[i].m;
    }
    const auto graph_error = [&](int64_t i, int rc, const std::string& message) {
        return count > 1 ? fail(rc, "graph " + std::to_string(i) + ": " + message) : fail(rc, message);
    };
    if (rows_ok == count && (n_total >= (int64_t(1) << 31) - 1 || m_total >= (int64_t(1) << 31) - 1)) {
        return fail(NGX_UNSUPPORTED, "ngx_graph_create: total vertices and arcs must be below 2^31 - 1");
    }
    if (m_total < (int64_t(1) << 16)) {
        threads = 1;  // not worth a thread
    }
    try {
        // vertex and row offsets per graph
        std::vector<int64_t> vertex_off(static_cast<size_t>(rows_ok) + 1, 0), row_off(static_cast<size_t>(rows_ok) + 1, 0),
            user_off(static_cast<size_t>(rows_ok) + 1, 0);
        for (int64_t i = 0; i < rows_ok; ++i) {
            vertex_off[static_cast<size_t>(i) + 1] = vertex_off[static_cast<size_t>(i)] + csrs[i].n;
            row_off[static_cast<size_t>(i) + 1] = row_off[static_cast<size_t>(i)] + csrs[i].n + 1;
            user_off[static_cast<size_t>(i) + 1] = user_off[static_cast<size_t>(i)] + csrs[i].m;
        }
        std::vector<Chunk> chunks;
        for (int64_t i = 0; i < rows_ok; ++i) {
            const ngx_csr& c = csrs[i];
            const int64_t pieces = std::max<int64_t>(1, std::min<int64_t>(c.n, (c.m + kChunkArcs - 1) / kChunkArcs));
            int64_t v0 = 0;
            for (int64_t p = 1; p <= pieces && c.n > 0; ++p) {
                int64_t v1 = c.n;
                if (p < pieces) {
                    const int64_t target = p * c.m / pieces;
                    v1 = std::max<int64_t>(v0, std::lower_bound(c.row_ptr, c.row_ptr + c.n, target) - c.row_ptr);
                }
                Chunk k;
                k.graph = i;
                k.v0 = v0;
                k.v1 = v1;
                chunks.push_back(k);
                v0 = v1;
            }
        }
        // pass 1: check the arcs, count the stored ones per vertex
        std::vector<int64_t> kept(static_cast<size_t>(vertex_off.back()), 0);
        parallel_for(static_cast<int64_t>(chunks.size()), threads, [&](int64_t t) {
            Chunk& k = chunks[static_cast<size_t>(t)];
            const ngx_csr& c = csrs[k.graph];
            int64_t* kept_row = kept.data() + vertex_off[static_cast<size_t>(k.graph)];
            for (int64_t u = k.v0; u < k.v1; ++u) {
                int64_t stored = 0;
                for (int64_t e = c.row_ptr[u]; e < c.row_ptr[u + 1]; ++e) {
                    const int32_t v = c.col[e];
                    const double w = c.w[e];
                    if (k.bad_arc < 0 && (v < 0 || v >= c.n || !std::isfinite(w))) {
                        k.bad_arc = e;
                        k.bad_target = v < 0 || v >= c.n;
                    }
                    stored += w != 0.0 ? 1 : 0;
                }
                kept_row[u] = stored;
                k.max_degree = std::max(k.max_degree, stored);
            }
        });
        for (int64_t i = 0; i < rows_ok; ++i) {
            int64_t bad = -1;
            bool bad_target = false;
            for (const Chunk& k : chunks) {
                if (k.graph == i && k.bad_arc >= 0 && (bad < 0 || k.bad_arc < bad)) {
                    bad = k.bad_arc;
                    bad_target = k.bad_target;
                }
            }
            if (bad >= 0) {
                return graph_error(i, NGX_INVALID_ARGUMENT, "ngx_graph_create: arc " + std::to_string(bad) +
                                                                (bad_target ? " has an out-of-range target" : " has a non-finite weight"));
            }
        }
        if (rows_ok < count) {
            return graph_error(rows_ok, rows_rc, rows_message);
        }
        // row offsets (global arc indices) and the parts
        h.parts.assign(static_cast<size_t>(count), GraphPart{});
        h.row_ptr.assign(static_cast<size_t>(row_off.back()), 0);
        int64_t m = 0;
        for (int64_t i = 0; i < count; ++i) {
            GraphPart& part = h.parts[static_cast<size_t>(i)];
            part.n = csrs[i].n;
            part.m_user = csrs[i].m;
            part.row_off = row_off[static_cast<size_t>(i)];
            part.user_arc_off = user_off[static_cast<size_t>(i)];
            part.vertex_off = vertex_off[static_cast<size_t>(i)];
            int64_t* rows = h.row_ptr.data() + part.row_off;
            const int64_t* kept_row = kept.data() + part.vertex_off;
            rows[0] = m;
            for (int64_t u = 0; u < part.n; ++u) {
                m += kept_row[u];
                rows[u + 1] = m;
            }
            part.m_stored = m - rows[0];
            h.n_max = std::max(h.n_max, part.n);
        }
        kept = std::vector<int64_t>();
        h.n_total = n_total;
        h.m_user = m_total;
        // pass 2: the stored arcs
        h.regular.resize(static_cast<size_t>(m));
        h.inverse.resize(static_cast<size_t>(m));
        h.arc_src.resize(static_cast<size_t>(m));
        h.stored_of_user.resize(static_cast<size_t>(m_total));  // every caller arc is written by its chunk
        HostVector<int32_t> target(static_cast<size_t>(m));
        parallel_for(static_cast<int64_t>(chunks.size()), threads, [&](int64_t t) {
            Chunk& k = chunks[static_cast<size_t>(t)];
            const ngx_csr& c = csrs[k.graph];
            const GraphPart& part = h.parts[static_cast<size_t>(k.graph)];
            int64_t pos = h.row_ptr[static_cast<size_t>(part.row_off + k.v0)];
            for (int64_t u = k.v0; u < k.v1; ++u) {
                for (int64_t e = c.row_ptr[u]; e < c.row_ptr[u + 1]; ++e) {
                    const double a = std::fabs(c.w[e]);
                    const int32_t id = static_cast<int32_t>(part.user_arc_off + e);
                    if (a == 0.0) {
                        h.stored_of_user[static_cast<size_t>(id)] = -1;
                        continue;
                    }
                    const int32_t v = c.col[e];
                    h.stored_of_user[static_cast<size_t>(id)] = static_cast<int32_t>(pos);
                    h.regular[static_cast<size_t>(pos)] = Arc{ v, id, a };
                    h.inverse[static_cast<size_t>(pos)] = Arc{ v, id, 1.0 / a };
                    h.arc_src[static_cast<size_t>(pos)] = static_cast<int32_t>(u);
                    target[static_cast<size_t>(pos)] = v;
                    k.min_len = std::min(k.min_len, a);
                    k.max_len = std::max(k.max_len, a);
                    ++pos;
                }
            }
        });
        // The locality order needs only the forward arcs. A single graph's order is sequential (each tile depends on
        // the ones before), so it runs on a thread of its own beside the remaining passes; a batch's graphs are
        // ordered in parallel at the end.
        std::vector<HostVector<int32_t>> orders(static_cast<size_t>(count));
        const auto order_graph = [&](int64_t i) {
            const GraphPart& part = h.parts[static_cast<size_t>(i)];
            const int64_t first = h.row_ptr[static_cast<size_t>(part.row_off)];
            std::vector<int64_t> local_rows(static_cast<size_t>(part.n) + 1);
            for (int64_t v = 0; v <= part.n; ++v) {
                local_rows[static_cast<size_t>(v)] = h.row_ptr[static_cast<size_t>(part.row_off + v)] - first;
            }
            orders[static_cast<size_t>(i)].reserve(static_cast<size_t>(part.n));
            append_source_order(part.n, local_rows.data(), h.regular.data() + first, orders[static_cast<size_t>(i)]);
        };
        std::thread order_thread;
        std::exception_ptr order_failure;
        if (count == 1 && threads > 1) {
            try {
                order_thread = std::thread([&] {
                    try {
                        order_graph(0);
                    } catch (...) {
                        order_failure = std::current_exception();
                    }
                });
                --threads;
            } catch (const std::system_error&) {
                // no thread for it: ordered at the end like a batch's graphs
            }
        }
        // joins the order thread on every exit from here on
        struct Joiner {
            std::thread& t;
            ~Joiner() {
                if (t.joinable()) {
                    t.join();
                }
            }
        } joiner{ order_thread };
        double min_regular = INFINITY, max_regular = 0.0;
        for (const Chunk& k : chunks) {
            h.max_out_degree = std::max(h.max_out_degree, k.max_degree);
            min_regular = std::min(min_regular, k.min_len);
            max_regular = std::max(max_regular, k.max_len);
        }
        // Two kinds of tasks run together: each graph's sums of lengths in arc order (the mean lengths; the graphs
        // are then added in order, so the bits do not depend on the threads), and the in-degree counts of the
        // reverse CSR, which is built by counting sort over targets, within a target in ascending stored order
        // (= ascending source); a large graph's targets are split into ranges, each task scanning all its targets.
        struct Range {
            int64_t graph, t0, t1;
        };
        std::vector<Range> ranges;
        for (int64_t i = 0; i < count; ++i) {
            const GraphPart& part = h.parts[static_cast<size_t>(i)];
            const int64_t pieces = part.m_stored >= (int64_t(1) << 21) ? std::min<int64_t>(threads, part.n) : 1;
            for (int64_t r = 0; r < pieces; ++r) {
                ranges.push_back(Range{ i, r * part.n / pieces, (r + 1) * part.n / pieces });
            }
        }
        std::vector<double> part_regular(static_cast<size_t>(count), 0.0), part_inverse(static_cast<size_t>(count), 0.0);
        std::vector<int64_t> cursor(static_cast<size_t>(n_total) + 1, 0);  // in-degree, then the next free slot
        parallel_for(count + static_cast<int64_t>(ranges.size()), threads, [&](int64_t t) {
            if (t < count) {
                const GraphPart& part = h.parts[static_cast<size_t>(t)];
                const int64_t first = h.row_ptr[static_cast<size_t>(part.row_off)];
                double sr = 0.0, si = 0.0;
                for (int64_t e = first; e < first + part.m_stored; ++e) {
                    sr += h.regular[static_cast<size_t>(e)].len;
                    si += h.inverse[static_cast<size_t>(e)].len;
                }
                part_regular[static_cast<size_t>(t)] = sr;
                part_inverse[static_cast<size_t>(t)] = si;
                return;
            }
            const Range& r = ranges[static_cast<size_t>(t - count)];
            const GraphPart& part = h.parts[static_cast<size_t>(r.graph)];
            const int64_t first = h.row_ptr[static_cast<size_t>(part.row_off)];
            int64_t* degree = cursor.data() + part.vertex_off;
            for (int64_t e = first; e < first + part.m_stored; ++e) {
                const int32_t v = target[static_cast<size_t>(e)];
                if (v >= r.t0 && v < r.t1) {
                    ++degree[v];
                }
            }
        });
        double sum_regular = 0.0, sum_inverse = 0.0;
        for (int64_t i = 0; i < count; ++i) {
            GraphPart& part = h.parts[static_cast<size_t>(i)];
            if (part.m_stored > 0) {
                part.mean_len_regular = part_regular[static_cast<size_t>(i)] / static_cast<double>(part.m_stored);
                part.mean_len_inverse = part_inverse[static_cast<size_t>(i)] / static_cast<double>(part.m_stored);
            }
            sum_regular += part_regular[static_cast<size_t>(i)];
            sum_inverse += part_inverse[static_cast<size_t>(i)];
        }
        if (m > 0) {
            h.mean_len_regular = sum_regular / static_cast<double>(m);
            h.mean_len_inverse = sum_inverse / static_cast<double>(m);
            h.min_len_regular = min_regular;
            h.max_len_regular = max_regular;
        }
        h.rrow_ptr.assign(static_cast<size_t>(row_off.back()), 0);
        for (int64_t i = 0; i < count; ++i) {
            const GraphPart& part = h.parts[static_cast<size_t>(i)];
            int64_t* rows = h.rrow_ptr.data() + part.row_off;
            int64_t* slot = cursor.data() + part.vertex_off;
            rows[0] = h.row_ptr[static_cast<size_t>(part.row_off)];
            for (int64_t v = 0; v < part.n; ++v) {
                rows[v + 1] = rows[v] + slot[v];
                slot[v] = rows[v];
            }
        }
        h.rarcs.resize(static_cast<size_t>(m));
        parallel_for(static_cast<int64_t>(ranges.size()), threads, [&](int64_t t) {
            const Range& r = ranges[static_cast<size_t>(t)];
            const GraphPart& part = h.parts[static_cast<size_t>(r.graph)];
            const int64_t first = h.row_ptr[static_cast<size_t>(part.row_off)];
            int64_t* slot = cursor.data() + part.vertex_off;
            for (int64_t e = first; e < first + part.m_stored; ++e) {
                const int32_t v = target[static_cast<size_t>(e)];
                if (v >= r.t0 && v < r.t1) {
                    // the reverse record keeps the arc's index in the stored forward CSR (its caller index is regular[e].id)
                    h.rarcs[static_cast<size_t>(slot[v]++)] = Arc{ h.arc_src[static_cast<size_t>(e)], static_cast<int32_t>(e), h.regular[static_cast<size_t>(e)].len };
                }
            }
        });
        target = HostVector<int32_t>();
        cursor = std::vector<int64_t>();
        if (order_thread.joinable()) {
            order_thread.join();
            if (order_failure) {
                std::rethrow_exception(order_failure);
            }
        } else {
            parallel_for(count, threads, order_graph);
        }
        if (count == 1) {
            h.source_order = std::move(orders[0]);
        } else {
            h.source_order.clear();
            h.source_order.reserve(static_cast<size_t>(n_total));
            for (const auto& o : orders) {
                h.source_order.insert(h.source_order.end(), o.begin(), o.end());
            }
        }
    } catch (const std::bad_alloc&) {
        return fail(NGX_OUT_OF_MEMORY, "ngx_graph_create: host allocation failed");
    } catch (const std::exception& e) {
        return fail(NGX_OUT_OF_MEMORY, std::string("ngx_graph_create: host build failed: ") + e.what());
    }
    return NGX_OK;
}

int create_graphs(const ngx_csr* csrs, int64_t count, int device, ngx_graph** out, bool on_host) {
    if (out == nullptr) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: out is NULL");
    }
    *out = nullptr;
    if (csrs == nullptr || count <= 0) {
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: no graphs");
    }
    // the input is checked (and, on the host path, laid out) before the device, so that a bad graph is reported as
    // such anywhere
    // the device build needs a usable device; without one the host path checks the graph and reports what is wrong
    int devices = 0;
    const bool have_device = cudaGetDeviceCount(&devices) == cudaSuccess && device >= 0 && device < devices;
    if (!have_device) {
        cudaGetLastError();
    }
    const bool on_device = !on_host && have_device && count == 1 && csrs[0].n > 0;
    HostGraphs h;
    if (on_device) {
        if (const int rc = validate_rows(&csrs[0]); rc != NGX_OK) {
            return rc;
        }
    } else if (const int rc = build_host_graphs(csrs, count, 0, &h); rc != NGX_OK) {
        return rc;
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
    g->l2_bytes = static_cast<size_t>(prop.l2CacheSize);
    if (!on_device) {
        g->n_total = h.n_total;
        g->m_user = h.m_user;
        g->n = h.n_max;
        g->m_stored = static_cast<int64_t>(h.regular.size());
        g->parts = std::move(h.parts);
        g->stored_of_user = std::move(h.stored_of_user);
        g->source_order = std::move(h.source_order);
        g->max_out_degree = h.max_out_degree;
        g->mean_len_regular = h.mean_len_regular;
        g->mean_len_inverse = h.mean_len_inverse;
        g->min_len_regular = h.min_len_regular;
        g->max_len_regular = h.max_len_regular;
    }

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
    if (on_device) {
        return finish(build_graph_on_device(&csrs[0], g));
    }

    const auto upload = [&](auto** dst, const auto& src) -> int {
        using T = std::remove_cv_t<std::remove_reference_t<decltype(src[0])>>;
        const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
        NGX_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), bytes));
        if (!src.empty()) {
            NGX_CUDA_TRY(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, g->stream));
        }
        return NGX_OK;
    };
    int rc = upload(&g->d_row_ptr, h.row_ptr);
    if (rc == NGX_OK) rc = upload(&g->d_arcs_regular, h.regular);
    if (rc == NGX_OK) rc = upload(&g->d_arcs_inverse, h.inverse);
    if (rc == NGX_OK) rc = upload(&g->d_rrow_ptr, h.rrow_ptr);
    if (rc == NGX_OK) rc = upload(&g->d_rarcs, h.rarcs);
    if (rc == NGX_OK) rc = upload(&g->d_arc_src, h.arc_src);
    if (rc == NGX_OK) {
        const cudaError_t err = cudaStreamSynchronize(g->stream);
        if (err != cudaSuccess) {
            rc = cuda_fail(err, "ngx_graph_create: upload");
        }
    }
    return finish(rc);
}

// SCC passes (kernel launches with a host flag read, ~10-20 us each) the APSP pre-pass may spend.
constexpr int64_t kSccPrePassCap = 2048;

int ensure_components(ngx_graph* g) {
    if (g->scc_components != 0 || g->parts.size() != 1 || g->n == 0) {
        return NGX_OK;
    }
    // a pre-pass for the runs, so bounded: graphs whose components need more passes (long chains) run without it
    uint64_t count = 0, largest = 0;
    g->scc_pass_cap = kSccPrePassCap;
    g->scc_passes = 0;
    const int rc = ngx_scc(g, nullptr, &count, &largest, nullptr);
    g->scc_pass_cap = 0;
    if (rc == NGX_TIMEOUT) {
        g->scc_components = -1;
        set_last_error("");
        return NGX_OK;
    }
    if (rc != NGX_OK) {
        return rc;
    }
    g->scc_components = static_cast<int64_t>(count);
    return NGX_OK;
}

int ensure_source_order(ngx_graph* g) {
    if (g->parts.size() == 1 && !g->order_grouped && static_cast<int64_t>(g->source_order.size()) == g->n_total) {
        // a graph of several strongly connected components: the sources of each component together (in their
        // locality order), so that a tile's sources reach the same vertices (StronglyConnectedComponents.h:34-35)
        if (const int rc = ensure_components(g); rc != NGX_OK) {
            return rc;
        }
        if (g->scc_components > 1) {
            std::vector<int32_t> comp(static_cast<size_t>(g->n));
            uint64_t count = 0, largest = 0;
            if (const int rc = ngx_scc(g, comp.data(), &count, &largest, nullptr); rc != NGX_OK) {
                return rc;
            }
            std::stable_sort(g->source_order.begin(), g->source_order.end(),
                             [&](int32_t a, int32_t b) { return comp[static_cast<size_t>(a)] < comp[static_cast<size_t>(b)]; });
        }
        g->order_grouped = true;
        return NGX_OK;
    }
    if (static_cast<int64_t>(g->source_order.size()) == g->n_total) {
        return NGX_OK;
    }
    if (g->parts.size() != 1) {
        return fail(NGX_INVALID_ARGUMENT, "a batch handle without its source order");
    }
    // the forward CSR back from the device, then the same order the host build computes
    const int64_t n = g->n;
    std::vector<int64_t> rows(static_cast<size_t>(n) + 1);
    HostVector<Arc> arcs(static_cast<size_t>(g->m_stored));
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    NGX_CUDA_TRY(cudaMemcpyAsync(rows.data(), g->d_row_ptr, rows.size() * 8, cudaMemcpyDeviceToHost, g->stream));
    if (!arcs.empty()) {
        NGX_CUDA_TRY(cudaMemcpyAsync(arcs.data(), g->d_arcs_regular, arcs.size() * sizeof(Arc), cudaMemcpyDeviceToHost, g->stream));
    }
    NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    HostVector<int32_t> order;
    order.reserve(static_cast<size_t>(n));
    append_source_order(n, rows.data(), arcs.data(), order);
    g->source_order = std::move(order);
    return ensure_source_order(g);  // then grouped by component
}

int ensure_stored_of_user(ngx_graph* g) {
    if (static_cast<int64_t>(g->stored_of_user.size()) == g->m_user || g->d_stored_of_user == nullptr) {
        return NGX_OK;
    }
    HostVector<int32_t> map(static_cast<size_t>(g->m_user));
    NGX_CUDA_TRY(cudaSetDevice(g->device));
    if (!map.empty()) {
        NGX_CUDA_TRY(cudaMemcpyAsync(map.data(), g->d_stored_of_user, map.size() * 4, cudaMemcpyDeviceToHost, g->stream));
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    g->stored_of_user = std::move(map);
    return NGX_OK;
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
    return guard_host("ngx_graph_source_order", [&]() -> int {
        if (graph == nullptr || (order == nullptr && graph->n_total > 0)) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_source_order: graph or order is NULL");
        }
        // computed on first use for a device-built handle (a cache, not a change of the graph)
        if (const int rc = ensure_source_order(const_cast<ngx_graph*>(graph)); rc != NGX_OK) {
            return rc;
        }
        for (size_t i = 0; i < graph->source_order.size(); ++i) {
            order[i] = graph->source_order[i];
        }
        return NGX_OK;
    });
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
    return guard_host("ngx_graph_create", [&]() -> int {
        if (csr == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: csr is NULL");
        }
        return create_graphs(csr, 1, device, out);
    });
}

int ngx_graph_create_ex(const ngx_csr* csr, int device, int flags, ngx_graph** out) {
    return guard_host("ngx_graph_create_ex", [&]() -> int {
        if (csr == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create_ex: csr is NULL");
        }
        if ((flags & ~NGX_BUILD_ON_HOST) != 0) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create_ex: unknown flags");
        }
        return create_graphs(csr, 1, device, out, (flags & NGX_BUILD_ON_HOST) != 0);
    });
}

int ngx_graph_layout(const ngx_graph* graph, int64_t* row_ptr, ngx_arc* arcs, ngx_arc* arcs_inverse, int64_t* rrow_ptr, ngx_arc* rarcs,
                     int32_t* arc_src, double* mean_lengths) {
    return guard_host("ngx_graph_layout", [&]() -> int {
        if (graph == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_graph_layout: graph is NULL");
        }
        static_assert(sizeof(ngx_arc) == sizeof(Arc), "ngx_arc mirrors the device arc record");
        NGX_CUDA_TRY(cudaSetDevice(graph->device));
        const size_t rows = static_cast<size_t>(graph->n_total + static_cast<int64_t>(graph->parts.size()));
        const size_t m = static_cast<size_t>(graph->m_stored);
        const auto get = [&](void* dst, const void* src, size_t bytes) -> int {
            if (dst != nullptr && bytes > 0) {
                NGX_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, graph->stream));
            }
            return NGX_OK;
        };
        int rc = get(row_ptr, graph->d_row_ptr, rows * 8);
        if (rc == NGX_OK) rc = get(arcs, graph->d_arcs_regular, m * sizeof(Arc));
        if (rc == NGX_OK) rc = get(arcs_inverse, graph->d_arcs_inverse, m * sizeof(Arc));
        if (rc == NGX_OK) rc = get(rrow_ptr, graph->d_rrow_ptr, rows * 8);
        if (rc == NGX_OK) rc = get(rarcs, graph->d_rarcs, m * sizeof(Arc));
        if (rc == NGX_OK) rc = get(arc_src, graph->d_arc_src, m * 4);
        if (rc != NGX_OK) {
            return rc;
        }
        NGX_CUDA_TRY(cudaStreamSynchronize(graph->stream));
        if (mean_lengths != nullptr) {
            mean_lengths[0] = graph->mean_len_regular;
            mean_lengths[1] = graph->mean_len_inverse;
        }
        return NGX_OK;
    });
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
