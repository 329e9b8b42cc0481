// Brandes betweenness and the CPL / efficiency adjoint on a source tile whose distances are final (sm_100a).
//
// Pull form over the shortest-path DAG, lane s of a warp owning source s of the tile (BrandesVariant.h:79-159 in the
// reference, restated):
//   count  cnt[v][s] = number of in-arcs (u -> v) with fl(d[u][s] + len) == d[v][s]               (reverse CSR)
//   sigma  level-synchronous Kahn order: the sources form level 0; a vertex joins level L + 1 for source s when its
//          last DAG predecessor (at level <= L) is done. On entering its level it pulls
//          sigma[v][s] = sum over DAG in-arcs of sigma[u][s], in reverse-CSR order, so every sum has a fixed order.
//   delta  levels in decreasing order; each vertex pulls over its DAG out-arcs (forward CSR order):
//          Brandes   delta[v][s] = sum sigma[v][s] * ((1 + delta[x][s]) / sigma[x][s])   (BrandesVariant.h:150-155)
//          adjoint   share = sigma[v][s] / sigma[x][s]; c = share * (1 + delta[x][s]); c_g = share * (g[x][s] + dg[x][s])
//                    with g = (1 / d)^2; delta[v] = sum c, dg[v] = sum c_g; each DAG arc e = (v -> x) receives
//                    sum over the tile's sources of c (d sum_t d(s,t) / d len_e) and of c_g (-d sum_t 1/d(s,t) / d len_e).
// Betweenness per vertex and the gradients per arc are summed in 128-bit fixed point (integer adds: per (arc, source)
// term for the gradients, per tile after an exact integer sum over the tile's lanes for betweenness), so the totals do
// not depend on the order in which CTAs finish nor on how the sources are grouped into tiles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "ngx_common.cuh"

namespace ngx {

constexpr uint32_t kNoLevel = 0xFFFFFFFFu;

struct BrandesParams {
    DeviceCsr rg;                   // reverse CSR (in-arcs), regular lengths; Arc::col = source, Arc::id = forward stored index
    const int32_t* arc_src;         // source vertex of each stored forward arc
    int64_t m_total;                // stored forward arcs of all graphs
    uint32_t* ws_tie;               // slots * n: bit s set when a relaxation of (v, s) tied with its distance
    double* ws_sigma;               // slots * n * kTile
    double* ws_delta;               // slots * n * kTile
    double* ws_delta_g;             // slots * n * kTile (adjoint only)
    uint32_t* ws_cnt;               // slots * n * kTile
    uint32_t* ws_lvl;               // slots * n * kTile
    int32_t* ws_list;               // slots * n * kTile: the vertices of each level, level after level
    int32_t* ws_loff;               // slots * (n + 2): start of each level in ws_list
    uint32_t* ws_scnt;              // slots * n * kTile: DAG successors per (vertex, source), then fill positions
    uint32_t* ws_soff;              // slots * (n * kTile + 1): start of each (vertex, source)'s successor list
    uint32_t* ws_succ;              // slots * succ_capacity: successor lists (indices into the forward CSR)
    int64_t succ_capacity;          // entries per slot; a tile with more DAG arcs uses the arc-scanning passes
    unsigned long long* bc;         // 2 * n fixed point (Brandes), or nullptr
    unsigned long long* grad_cpl;   // 2 * m_user fixed point (adjoint), or nullptr
    unsigned long long* grad_eff;   // 2 * m_user fixed point (adjoint), or nullptr
    unsigned long long* levels;     // unused (levels are counted in the run counters)
    int* sigma_inexact;             // set when a pushed sigma sum reaches 2^53 (the host then reruns in pull form)
    int sigma_pull;                 // 1: pull form for sigma
};

constexpr int kSuccPerPair = 2;  // successor-list capacity, in DAG arcs per (vertex, source)

inline size_t brandes_slot_bytes(int64_t n, bool adjoint) {
    const size_t nt = static_cast<size_t>(n) * kTile;
    return nt * (8 + 8 + (adjoint ? 8 : 0) + 4 + 4 + 4) + static_cast<size_t>(n + 2) * 4 +
           nt * 4 + (nt + 1) * 4 + static_cast<size_t>(n) * 4 + nt * kSuccPerPair * 4 + 1024;
}

// Per-CTA bytes of the plain (one source per CTA) Brandes form: sigma, delta, counts, level list, level offsets.
inline size_t plain_brandes_slot_bytes(int64_t n) {
    return static_cast<size_t>(n) * (8 + 8 + 4 + 4) + static_cast<size_t>(n + 2) * 4 + 256;
}

__device__ __forceinline__ bool on_dag(unsigned long long du_bits, double len, unsigned long long dv_bits) {
    return static_cast<unsigned long long>(__double_as_longlong(__dadd_rn(__longlong_as_double(static_cast<long long>(du_bits)), len))) == dv_bits;
}

// Pair-parallel walk over the deg x k (arc, ready source) pairs of one vertex, as in the SSSP expansion: pair
// p = 32 i + lane takes arc p / k and the (p % k)-th ready source. Sums per source are gathered in arc order: in each
// iteration the lanes holding rank r's pairs are l0, l0 + k, ... (increasing arcs), and lane r adds them in that order,
// so every per-source sum runs over the arcs in CSR order, the same order for every run.
struct PairWalk {
    int k;         // ready sources
    int a;         // this lane's arc (relative to the row)
    int r;         // this lane's rank
    int step_a;
    int step_r;
    __device__ __forceinline__ PairWalk(int k_, int lane) : k(k_) {
        a = lane / k;
        r = lane - a * k;
        step_a = 32 / k;
        step_r = 32 - step_a * k;
    }
    __device__ __forceinline__ void advance() {
        a += step_a;
        r += step_r;
        if (r >= k) {
            r -= k;
            a += 1;
        }
    }
};

// Lane r (< k) receives the sum, in lane order, of `value` over the lanes whose pair has rank r in this iteration;
// `first_rank` is the rank of lane 0's pair.
__device__ __forceinline__ double gather_rank_sum(double value, int k, int first_rank, int lane) {
    const int l0 = (lane - first_rank + 32 * k) % k;  // first lane whose rank equals this lane's index
    const int rounds = (32 + k - 1) / k;
    double sum = 0.0;
    for (int q = 0; q < rounds; ++q) {
        const int from = l0 + q * k;
        const double t = __shfl_sync(0xFFFFFFFFu, value, from < 32 ? from : 0);
        if (from < 32) {
            sum += t;
        }
    }
    return sum;
}

// sigma values are path counts: integers, summed exactly in FP64 (in any order) while below 2^53.
constexpr double kSigmaExact = 9007199254740992.0;

// Processes one level-L entry v of the sigma pass, then releases the DAG successors.
// kPull: sigma[v] = sum over DAG in-arcs of sigma[u], gathered in reverse-CSR order (the order-defined form).
// !kPull: sigma[v] is final on entry (pushed by its predecessors); v adds sigma[v] into each DAG successor with an
//         atomic add. While every sum stays below 2^53 these integer sums are exact, so the result equals the pull
//         form's bit for bit whatever the order; a sum reaching 2^53 raises *inexact and the host reruns in pull form.
template <bool kPull, int kUnroll>
__device__ __forceinline__ void brandes_sigma_vertex(const DeviceCsr& g, const DeviceCsr& rg, int v, uint32_t level, int nsrc, int lane,
                                                     const unsigned long long* dist, double* sigma, uint32_t* cnt, uint32_t* lvl, uint32_t* stamp,
                                                     unsigned level_stamp, int32_t* next_list, int* next_len, int* inexact) {
    const int64_t vbase = static_cast<int64_t>(v) * kTile;
    const bool ready = lane < nsrc && __ldcg(&lvl[vbase + lane]) == level;
    const unsigned rmask = __ballot_sync(0xFFFFFFFFu, ready);
    if (rmask == 0u) {
        return;
    }
    const int k = __popc(rmask);
    const int rank_src = lane < k ? static_cast<int>(__fns(rmask, 0, lane + 1)) : 0;
    const unsigned long long rank_dv = __ldcg(&dist[vbase + rank_src]);
    double rank_sv = 0.0;
    if constexpr (kPull) {
        if (level > 0) {
            const int64_t beg = __ldg(&rg.row_ptr[v]);
            const int deg = static_cast<int>(__ldg(&rg.row_ptr[v + 1]) - beg);
            const Arc* arcs = rg.arcs + beg;
            PairWalk w(k, lane);
            double acc = 0.0;
            const int64_t total = static_cast<int64_t>(deg) * k;
            for (int64_t p0 = 0; p0 < total; p0 += 32) {
                const int s = __shfl_sync(0xFFFFFFFFu, rank_src, w.r);
                const unsigned long long dvs = __shfl_sync(0xFFFFFFFFu, rank_dv, w.r);
                double contrib = 0.0;
                if (w.a < deg) {
                    const Arc arc = ldg_arc(&arcs[w.a]);
                    const int64_t urow = static_cast<int64_t>(arc.col) * kTile + s;
                    const unsigned long long du = __ldcg(&dist[urow]);
                    if (du != kInfBits && on_dag(du, arc.len, dvs)) {
                        contrib = __ldcg(&sigma[urow]);
                    }
                }
                acc += gather_rank_sum(contrib, k, static_cast<int>(p0 % k), lane);
                w.advance();
            }
            if (lane < k) {
                sigma[vbase + rank_src] = acc;
            }
            rank_sv = acc;
        } else {
            rank_sv = __ldcg(&sigma[vbase + rank_src]);
        }
    } else {
        rank_sv = __ldcg(&sigma[vbase + rank_src]);
    }
    const int64_t beg = __ldg(&g.row_ptr[v]);
    const int deg = static_cast<int>(__ldg(&g.row_ptr[v + 1]) - beg);
    const Arc* arcs = g.arcs + beg;
    PairWalk w(k, lane);
    const int64_t total = static_cast<int64_t>(deg) * k;
    for (int64_t p0 = 0; p0 < total; p0 += 32 * kUnroll) {
        int x[kUnroll];
        int s[kUnroll];
        double sv[kUnroll];
        unsigned long long dvs[kUnroll], dx[kUnroll];
        double len[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            s[u] = __shfl_sync(0xFFFFFFFFu, rank_src, w.r);
            dvs[u] = __shfl_sync(0xFFFFFFFFu, rank_dv, w.r);
            sv[u] = __shfl_sync(0xFFFFFFFFu, rank_sv, w.r);
            x[u] = 0;
            len[u] = 0.0;
            dx[u] = kInfBits;
            if (w.a < deg) {
                const Arc arc = ldg_arc(&arcs[w.a]);
                x[u] = arc.col;
                len[u] = arc.len;
                dx[u] = __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + s[u]]);
            }
            w.advance();
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            bool released = false;
            if (dx[u] != kInfBits && on_dag(dvs[u], len[u], dx[u])) {
                const int64_t xrow = static_cast<int64_t>(x[u]) * kTile + s[u];
                if constexpr (!kPull) {
                    const double before = atomicAdd(&sigma[xrow], sv[u]);
                    if (before + sv[u] >= kSigmaExact) {
                        atomicExch(inexact, 1);
                    }
                }
                if (atomicSub(&cnt[xrow], 1u) == 1u) {
                    lvl[xrow] = level + 1u;
                    released = atomicExch(&stamp[x[u]], level_stamp) != level_stamp;
                }
            }
            const unsigned pmask = __ballot_sync(0xFFFFFFFFu, released);
            if (pmask != 0u) {
                const int leader = __ffs(pmask) - 1;
                int base = 0;
                if (lane == leader) {
                    base = atomicAdd(next_len, __popc(pmask));
                }
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (released) {
                    unsigned lt;
                    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
                    next_list[base + __popc(pmask & lt)] = x[u];
                }
            }
        }
    }
}

// Processes one level-L entry v of the delta pass (pull over DAG out-arcs), emitting per-arc adjoint terms.
template <int kMode, int kUnroll>
__device__ __forceinline__ void brandes_delta_vertex(const DeviceCsr& g, int v, uint32_t level, int nsrc, int lane, const unsigned long long* dist,
                                                     const double* sigma, double* delta, double* delta_g, const uint32_t* lvl,
                                                     unsigned long long* grad_cpl, unsigned long long* grad_eff) {
    const int64_t vbase = static_cast<int64_t>(v) * kTile;
    const bool ready = lane < nsrc && __ldcg(&lvl[vbase + lane]) == level;
    const unsigned rmask = __ballot_sync(0xFFFFFFFFu, ready);
    if (rmask == 0u) {
        return;
    }
    const int k = __popc(rmask);
    const int rank_src = lane < k ? static_cast<int>(__fns(rmask, 0, lane + 1)) : 0;
    const unsigned long long rank_dv = __ldcg(&dist[vbase + rank_src]);
    const double rank_sv = __ldcg(&sigma[vbase + rank_src]);
    const int64_t beg = __ldg(&g.row_ptr[v]);
    const int deg = static_cast<int>(__ldg(&g.row_ptr[v + 1]) - beg);
    const Arc* arcs = g.arcs + beg;
    PairWalk w(k, lane);
    double acc = 0.0;
    double acc_g = 0.0;
    const int64_t total = static_cast<int64_t>(deg) * k;
    for (int64_t p0 = 0; p0 < total; p0 += 32 * kUnroll) {
        int s[kUnroll];
        unsigned long long dvs[kUnroll], dx[kUnroll];
        double sv[kUnroll], len[kUnroll];
        int x[kUnroll], id[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            s[u] = __shfl_sync(0xFFFFFFFFu, rank_src, w.r);
            dvs[u] = __shfl_sync(0xFFFFFFFFu, rank_dv, w.r);
            sv[u] = __shfl_sync(0xFFFFFFFFu, rank_sv, w.r);
            x[u] = 0;
            id[u] = 0;
            len[u] = 0.0;
            dx[u] = kInfBits;
            if (w.a < deg) {
                const Arc arc = ldg_arc(&arcs[w.a]);
                x[u] = arc.col;
                id[u] = arc.id;
                len[u] = arc.len;
                dx[u] = __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + s[u]]);
            }
            w.advance();
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            double c = 0.0, cg = 0.0;
            if (dx[u] != kInfBits && on_dag(dvs[u], len[u], dx[u])) {
                const int64_t xrow = static_cast<int64_t>(x[u]) * kTile + s[u];
                if constexpr (kMode == kModeBrandes) {
                    c = sv[u] * ((1.0 + __ldcg(&delta[xrow])) / __ldcg(&sigma[xrow]));
                } else {
                    const double share = sv[u] / __ldcg(&sigma[xrow]);
                    const double inv = 1.0 / __longlong_as_double(static_cast<long long>(dx[u]));
                    c = share * (1.0 + __ldcg(&delta[xrow]));
                    cg = share * (inv * inv + __ldcg(&delta_g[xrow]));
                    // per (arc, source) term into the arc's 128-bit fixed-point sum: order-free, deterministic
                    fixed_add(&grad_cpl[2 * static_cast<int64_t>(id[u])], c);
                    fixed_add(&grad_eff[2 * static_cast<int64_t>(id[u])], cg);
                }
            }
            const int first_rank = static_cast<int>((p0 + 32 * u) % k);
            acc += gather_rank_sum(c, k, first_rank, lane);
            if constexpr (kMode == kModeGrad) {
                acc_g += gather_rank_sum(cg, k, first_rank, lane);
            }
        }
    }
    if (lane < k) {
        delta[vbase + rank_src] = acc;
        if constexpr (kMode == kModeGrad) {
            delta_g[vbase + rank_src] = acc_g;
        }
    }
}

// ------------------------------------------------------------------------------------------ successor lists
// The DAG of a tile is about one arc per (vertex, source) without ties, against deg arcs scanned per (vertex, source)
// by the arc-scanning passes. The dense count pass (lane per source, coalesced distance rows) already visits every DAG
// arc; it also counts successors per (vertex, source). A block-wide prefix sum gives each (vertex, source) its list,
// a second dense pass fills the lists (forward-CSR arc indices), and each list is sorted so that every sum over it has
// a fixed order. sigma and delta then touch only DAG arcs.

// Counts the DAG in-arcs of v for the lanes in `scan` by scanning v's in-arcs (ties, or no usable recorded key).
__device__ __forceinline__ void dag_count_scan(const DeviceCsr& rg, int64_t v, unsigned long long dv, bool scan, const unsigned long long* dist,
                                               uint32_t* scnt, int lane, uint32_t& c, uint32_t& first) {
    const int64_t beg = __ldg(&rg.row_ptr[v]);
    const int64_t end = __ldg(&rg.row_ptr[v + 1]);
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
        const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
        Arc a{ 0, 0, 0.0 };
        if (lane < cntr) {
            a = ldg_arc(&rg.arcs[e0 + lane]);
        }
        for (int j = 0; j < cntr; j += 4) {
            unsigned long long du[4];
            double len[4];
            int src[4], fwd[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j + u < cntr ? j + u : 0;
                src[u] = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                fwd[u] = __shfl_sync(0xFFFFFFFFu, a.id, jj);
                len[u] = __shfl_sync(0xFFFFFFFFu, a.len, jj);
                du[u] = (scan && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(src[u]) * kTile + lane]) : kInfBits;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (du[u] != kInfBits && on_dag(du[u], len[u], dv)) {
                    if (c == 0) {
                        first = static_cast<uint32_t>(fwd[u]);
                    }
                    ++c;
                    atomicAdd(&scnt[static_cast<int64_t>(src[u]) * kTile + lane], 1u);
                }
            }
        }
    }
}

// Vertices handled together by one warp in the count and fill passes (their loads are issued side by side).
constexpr int kDagVertices = 2;

// cnt[v][s] = DAG predecessors; scnt[u][s] += 1 for each DAG arc u -> v (warp per vertex, lane per source);
// pred[v][s] = forward-CSR index of a DAG in-arc (the only one when cnt[v][s] == 1).
// A lane whose tie bit stayed clear in the SSSP phase takes its single DAG arc from the predecessor key recorded
// there (pred_key, which shares storage with sigma and is zeroed here for the sigma pass), after checking it; lanes
// with ties (or a key that does not check out) count by scanning v's in-arcs.
__device__ __forceinline__ void dag_count(const DeviceCsr& g, const DeviceCsr& rg, const int32_t* arc_src, int64_t m_total, int64_t n, int nsrc,
                                          const int* s_src, const unsigned long long* dist, const uint32_t* tie, unsigned long long* pred_key,
                                          uint32_t* cnt, uint32_t* scnt, uint32_t* pred, int lane, int warp, int nwarps,
                                          unsigned long long* active_pairs) {
    unsigned long long active_count = 0;
    const int src_lane = lane < nsrc ? s_src[lane] : -1;
    for (int64_t v0 = warp; v0 < n; v0 += static_cast<int64_t>(kDagVertices) * nwarps) {
        int64_t vv[kDagVertices];
        unsigned long long dv[kDagVertices], key[kDagVertices], du[kDagVertices];
        bool active[kDagVertices], fast[kDagVertices];
        uint32_t e[kDagVertices];
        Arc a[kDagVertices];
        int32_t u[kDagVertices];
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            vv[i] = v0 + static_cast<int64_t>(i) * nwarps;
            dv[i] = kInfBits;
            key[i] = 0ull;
            bool tied = true;
            if (vv[i] < n) {
                dv[i] = __ldcg(&dist[vv[i] * kTile + lane]);
                tied = (__ldcg(&tie[vv[i]]) >> lane) & 1u;
                key[i] = __ldcg(&pred_key[vv[i] * kTile + lane]);
                pred_key[vv[i] * kTile + lane] = 0ull;  // sigma = 0.0
            }
            active[i] = vv[i] < n && lane < nsrc && dv[i] != kInfBits && vv[i] != src_lane;
            active_count += active[i] ? 1ull : 0ull;
            e[i] = static_cast<uint32_t>(key[i]);
            fast[i] = active[i] && !tied && (key[i] >> 32) == (dv[i] >> 32) && static_cast<int64_t>(e[i]) < m_total;
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            a[i] = Arc{ -1, 0, 0.0 };
            u[i] = 0;
            if (fast[i]) {
                a[i] = ldg_arc(&g.arcs[e[i]]);
                u[i] = __ldg(&arc_src[e[i]]);
            }
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            fast[i] = fast[i] && a[i].col == static_cast<int32_t>(vv[i]);
            du[i] = fast[i] ? __ldcg(&dist[static_cast<int64_t>(u[i]) * kTile + lane]) : kInfBits;
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            if (vv[i] >= n) {
                continue;  // warp-uniform
            }
            uint32_t c = 0;
            uint32_t first = 0;
            bool scan = active[i];
            if (du[i] != kInfBits && on_dag(du[i], a[i].len, dv[i])) {
                c = 1;
                first = e[i];
                scan = false;
                atomicAdd(&scnt[static_cast<int64_t>(u[i]) * kTile + lane], 1u);
            }
            if (__ballot_sync(0xFFFFFFFFu, scan) != 0u) {
                dag_count_scan(rg, vv[i], dv[i], scan, dist, scnt, lane, c, first);
            }
            cnt[vv[i] * kTile + lane] = c;
            pred[vv[i] * kTile + lane] = first;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        active_count += __shfl_xor_sync(0xFFFFFFFFu, active_count, off);
    }
    if (lane == 0 && active_count != 0ull) {
        atomicAdd(active_pairs, active_count);
    }
}

template <bool kTarget>
__device__ __forceinline__ void dag_fill_scan(const DeviceCsr& rg, int64_t v, bool active, const unsigned long long* dist, const uint32_t* soff,
                                              uint32_t* sfill, uint32_t* succ, int lane);

// Fills the successor lists: each DAG arc u -> v is appended to (u, s), as its target v (kTarget: betweenness needs
// nothing else) or as its forward-CSR index (the adjoint also needs the arc). A (v, s) with a single DAG predecessor
// takes it from pred[v][s] (a forward index); only lanes with several re-scan v's in-arcs.
template <bool kTarget>
__device__ __forceinline__ void dag_fill(const DeviceCsr& rg, const int32_t* arc_src, int64_t n, const unsigned long long* dist, const uint32_t* cnt,
                                         const uint32_t* pred, const uint32_t* soff, uint32_t* sfill, uint32_t* succ, int lane, int warp, int nwarps) {
    for (int64_t v0 = warp; v0 < n; v0 += static_cast<int64_t>(kDagVertices) * nwarps) {
        // single-predecessor lanes of kDagVertices vertices, their loads side by side
        uint32_t c[kDagVertices], e[kDagVertices], pos[kDagVertices], off[kDagVertices];
        int64_t urow[kDagVertices];
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            const int64_t v = v0 + static_cast<int64_t>(i) * nwarps;
            c[i] = v < n ? __ldcg(&cnt[v * kTile + lane]) : 0u;
            e[i] = c[i] == 1u ? __ldcg(&pred[v * kTile + lane]) : 0u;
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            urow[i] = c[i] == 1u ? static_cast<int64_t>(__ldg(&arc_src[e[i]])) * kTile + lane : 0;
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            pos[i] = c[i] == 1u ? atomicAdd(&sfill[urow[i]], 1u) : 0u;
            off[i] = c[i] == 1u ? __ldcg(&soff[urow[i]]) : 0u;
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            if (c[i] == 1u) {
                const int64_t v = v0 + static_cast<int64_t>(i) * nwarps;
                succ[off[i] + pos[i]] = kTarget ? static_cast<uint32_t>(v) : e[i];
            }
        }
#pragma unroll
        for (int i = 0; i < kDagVertices; ++i) {
            const int64_t v = v0 + static_cast<int64_t>(i) * nwarps;
            const bool active = c[i] >= 2u;
            if (v < n && __ballot_sync(0xFFFFFFFFu, active) != 0u) {
                dag_fill_scan<kTarget>(rg, v, active, dist, soff, sfill, succ, lane);
            }
        }
    }
}

// Appends v's DAG in-arcs for the lanes in `active` (several predecessors) by scanning v's in-arcs.
template <bool kTarget>
__device__ __forceinline__ void dag_fill_scan(const DeviceCsr& rg, int64_t v, bool active, const unsigned long long* dist, const uint32_t* soff,
                                              uint32_t* sfill, uint32_t* succ, int lane) {
    {  // one scope, so the scan below keeps its layout
        const unsigned long long dv = __ldcg(&dist[v * kTile + lane]);
        const int64_t beg = __ldg(&rg.row_ptr[v]);
        const int64_t end = __ldg(&rg.row_ptr[v + 1]);
        for (int64_t e0 = beg; e0 < end; e0 += 32) {
            const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
            Arc a{ 0, 0, 0.0 };
            if (lane < cntr) {
                a = ldg_arc(&rg.arcs[e0 + lane]);
            }
            for (int j = 0; j < cntr; j += 4) {
                unsigned long long du[4];
                double len[4];
                int src[4], fwd[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = j + u < cntr ? j + u : 0;
                    src[u] = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                    fwd[u] = __shfl_sync(0xFFFFFFFFu, a.id, jj);
                    len[u] = __shfl_sync(0xFFFFFFFFu, a.len, jj);
                    du[u] = (active && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(src[u]) * kTile + lane]) : kInfBits;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (du[u] != kInfBits && on_dag(du[u], len[u], dv)) {
                        const int64_t urow = static_cast<int64_t>(src[u]) * kTile + lane;
                        const uint32_t pos = atomicAdd(&sfill[urow], 1u);
                        succ[__ldcg(&soff[urow]) + pos] = kTarget ? static_cast<uint32_t>(v) : static_cast<uint32_t>(fwd[u]);
                    }
                }
            }
        }
    }
}

// Sorts each successor list by its entries (the fill order depends on timing; the sums must not). Lists are spread
// over the threads of the group: thread `first` of `stride` takes lists first, first + stride, ...
__device__ __forceinline__ void dag_sort(const uint32_t* soff, uint32_t* succ, int64_t nt, int64_t first, int64_t stride) {
    for (int64_t i = first; i < nt; i += stride) {
        const uint32_t beg = __ldcg(&soff[i]);
        const uint32_t end = __ldcg(&soff[i + 1]);
        for (uint32_t a = beg + 1; a < end; ++a) {
            const uint32_t key = __ldcg(&succ[a]);
            uint32_t b = a;
            while (b > beg && __ldcg(&succ[b - 1]) > key) {
                succ[b] = __ldcg(&succ[b - 1]);
                --b;
            }
            succ[b] = key;
        }
    }
}

// ------------------------------------------------------------------------------------------ level passes
// One level of (vertex, source) entries (entry = v << 5 | s) is processed a warp at a time: the warp takes 32 entries,
// scans their successor-list lengths, and walks the (entry, successor) pairs 32 at a time, kLevelUnroll pairs per lane
// in flight, so hubs with long lists do not serialise a lane and every lane keeps independent loads outstanding.
constexpr int kLevelUnroll = 4;

// The adjoint's delta pass carries twice the values per pair; it unrolls less to stay within 64 registers.
constexpr int delta_level_unroll(int mode) { return mode == kModeGrad ? 2 : 4; }

// Exclusive prefix of x over the warp's lanes; *total receives the sum.
__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t x, int lane, uint32_t* total) {
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) {
            incl += y;
        }
    }
    *total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    return incl - x;
}

// The lane whose list holds pair p: the largest lane L with off[L] <= p (lanes with empty lists share their
// successor's offset, so L always has a non-empty list when p < total).
__device__ __forceinline__ int pair_owner(uint32_t off, uint32_t p) {
    int l = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t o = __shfl_sync(0xFFFFFFFFu, off, l + step);
        if (o <= p) {
            l += step;
        }
    }
    return l;
}

// sigma over one level: every entry adds sigma[v][s] into its DAG successors and releases those whose last
// predecessor this was. The adds are exact integer sums while below 2^53 (see brandes_sigma_vertex); since every
// addend is positive, a final value below 2^53 proves every partial sum was too, so the check is made on each entry's
// final sigma when its own level runs.
template <bool kTarget>
__device__ __forceinline__ void dag_sigma_level(const DeviceCsr& g, const int32_t* entries, int len, uint32_t level, double* sigma, uint32_t* cnt,
                                                uint32_t* lvl, const uint32_t* soff, const uint32_t* succ, int32_t* next_list, int* next_len,
                                                int* inexact, int lane, int warp, int nwarps) {
    for (int base = warp * 32; base < len; base += nwarps * 32) {
        const int i = base + lane;
        uint32_t entry = 0, beg = 0, count = 0;
        double sv = 0.0;
        if (i < len) {
            entry = static_cast<uint32_t>(__ldcg(&entries[i]));
            const int64_t row = static_cast<int64_t>(entry >> 5) * kTile + (entry & 31u);
            sv = __ldcg(&sigma[row]);
            beg = __ldcg(&soff[row]);
            count = __ldcg(&soff[row + 1]) - beg;
            if (sv >= kSigmaExact) {
                atomicExch(inexact, 1);
            }
        }
        uint32_t total = 0;
        const uint32_t off = warp_exclusive_scan(count, lane, &total);
        for (uint32_t p0 = 0; p0 < total; p0 += 32 * kLevelUnroll) {
            uint32_t xrow_s[kLevelUnroll];
            uint32_t x[kLevelUnroll];
            double add[kLevelUnroll];
            bool ok[kLevelUnroll];
#pragma unroll
            for (int u = 0; u < kLevelUnroll; ++u) {
                const uint32_t q = p0 + static_cast<uint32_t>(u * 32 + lane);
                ok[u] = q < total;
                const int owner = pair_owner(off, ok[u] ? q : 0u);
                const uint32_t j = __shfl_sync(0xFFFFFFFFu, beg, owner) + (q - __shfl_sync(0xFFFFFFFFu, off, owner));
                xrow_s[u] = __shfl_sync(0xFFFFFFFFu, entry, owner) & 31u;
                add[u] = __shfl_sync(0xFFFFFFFFu, sv, owner);
                x[u] = 0;
                if (ok[u]) {
                    const uint32_t e = __ldcg(&succ[j]);
                    x[u] = kTarget ? e : static_cast<uint32_t>(ldg_arc(&g.arcs[e]).col);
                }
            }
#pragma unroll
            for (int u = 0; u < kLevelUnroll; ++u) {
                bool push = false;
                const int64_t xrow = static_cast<int64_t>(x[u]) * kTile + xrow_s[u];
                if (ok[u]) {
                    atomicAdd(&sigma[xrow], add[u]);
                    if (atomicSub(&cnt[xrow], 1u) == 1u) {
                        lvl[xrow] = level + 1u;
                        push = true;
                    }
                }
                const unsigned pmask = __ballot_sync(0xFFFFFFFFu, push);
                if (pmask != 0u) {
                    int at = 0;
                    const int leader = __ffs(pmask) - 1;
                    if (lane == leader) {
                        at = atomicAdd(next_len, __popc(pmask));
                    }
                    at = __shfl_sync(0xFFFFFFFFu, at, leader);
                    if (push) {
                        next_list[at + __popc(pmask & lanemask_lt())] = static_cast<int32_t>((x[u] << 5) | xrow_s[u]);
                    }
                }
            }
        }
    }
}

// One level of the sigma pass when the tile's DAGs are trees: every successor gets sigma 1 and joins the next level.
template <bool kTarget>
__device__ __forceinline__ void dag_tree_level(const DeviceCsr& g, const int32_t* entries, int len, double* sigma, const uint32_t* soff,
                                               const uint32_t* succ, int32_t* next_list, int* next_len, int lane, int warp, int nwarps) {
    for (int base = warp * 32; base < len; base += nwarps * 32) {
        const int i = base + lane;
        uint32_t entry = 0, beg = 0, count = 0;
        if (i < len) {
            entry = static_cast<uint32_t>(__ldcg(&entries[i]));
            const int64_t row = static_cast<int64_t>(entry >> 5) * kTile + (entry & 31u);
            beg = __ldcg(&soff[row]);
            count = __ldcg(&soff[row + 1]) - beg;
        }
        uint32_t total = 0;
        const uint32_t off = warp_exclusive_scan(count, lane, &total);
        // every pair pushes exactly one entry: reserve the warp's slots once
        int at = 0;
        if (lane == 0 && total != 0u) {
            at = atomicAdd(next_len, static_cast<int>(total));
        }
        at = __shfl_sync(0xFFFFFFFFu, at, 0);
        for (uint32_t p0 = 0; p0 < total; p0 += 32 * kLevelUnroll) {
            uint32_t x[kLevelUnroll], sx[kLevelUnroll];
            bool ok[kLevelUnroll];
#pragma unroll
            for (int u = 0; u < kLevelUnroll; ++u) {
                const uint32_t q = p0 + static_cast<uint32_t>(u * 32 + lane);
                ok[u] = q < total;
                const int owner = pair_owner(off, ok[u] ? q : 0u);
                const uint32_t j = __shfl_sync(0xFFFFFFFFu, beg, owner) + (q - __shfl_sync(0xFFFFFFFFu, off, owner));
                sx[u] = __shfl_sync(0xFFFFFFFFu, entry, owner) & 31u;
                x[u] = 0;
                if (ok[u]) {
                    const uint32_t e = __ldcg(&succ[j]);
                    x[u] = kTarget ? e : static_cast<uint32_t>(ldg_arc(&g.arcs[e]).col);
                }
            }
#pragma unroll
            for (int u = 0; u < kLevelUnroll; ++u) {
                const uint32_t q = p0 + static_cast<uint32_t>(u * 32 + lane);
                if (ok[u]) {
                    sigma[static_cast<int64_t>(x[u]) * kTile + sx[u]] = 1.0;
                    next_list[at + static_cast<int>(q)] = static_cast<int32_t>((x[u] << 5) | sx[u]);
                }
            }
        }
    }
}

// delta (and the adjoint terms) over one level: each entry pulls over its sorted successor list. Pair contributions
// go through the warp's slice of `buf` (32 values per unrolled pair, twice for the adjoint) and each entry's lane adds
// its own in list order, so every sum runs in the same order as a sequential loop over the list.
template <int kMode, bool kTree>
__device__ __forceinline__ void dag_delta_level(const DeviceCsr& g, const int32_t* entries, int len, const unsigned long long* dist, const double* sigma,
                                                double* delta, double* delta_g, const uint32_t* soff, const uint32_t* succ, unsigned long long* grad_cpl,
                                                unsigned long long* grad_eff, double* buf, int lane, int buf_warp, int warp, int nwarps) {
    constexpr bool kTarget = kMode == kModeBrandes;
    constexpr int kU = delta_level_unroll(kMode);
    double* const wbuf = buf + static_cast<size_t>(buf_warp) * 32 * kU * (kMode == kModeGrad ? 2 : 1);
    for (int base = warp * 32; base < len; base += nwarps * 32) {
        const int i = base + lane;
        uint32_t entry = 0, beg = 0, count = 0;
        double sv = 0.0;
        int64_t row = 0;
        if (i < len) {
            entry = static_cast<uint32_t>(__ldcg(&entries[i]));
            row = static_cast<int64_t>(entry >> 5) * kTile + (entry & 31u);
            sv = kTree ? 1.0 : __ldcg(&sigma[row]);
            beg = __ldcg(&soff[row]);
            count = __ldcg(&soff[row + 1]) - beg;
        }
        uint32_t total = 0;
        const uint32_t off = warp_exclusive_scan(count, lane, &total);
        double acc = 0.0, acc_g = 0.0;
        for (uint32_t p0 = 0; p0 < total; p0 += 32 * kU) {
            double dx[kU], sx[kU], share_sv[kU], gx[kU], dgx[kU];
            int32_t id[kU];
            bool ok[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const uint32_t q = p0 + static_cast<uint32_t>(u * 32 + lane);
                ok[u] = q < total;
                const int owner = pair_owner(off, ok[u] ? q : 0u);
                const uint32_t j = __shfl_sync(0xFFFFFFFFu, beg, owner) + (q - __shfl_sync(0xFFFFFFFFu, off, owner));
                const uint32_t s = __shfl_sync(0xFFFFFFFFu, entry, owner) & 31u;
                share_sv[u] = __shfl_sync(0xFFFFFFFFu, sv, owner);
                dx[u] = 0.0;
                sx[u] = 1.0;
                gx[u] = 0.0;
                dgx[u] = 0.0;
                id[u] = 0;
                if (ok[u]) {
                    const uint32_t e = __ldcg(&succ[j]);
                    uint32_t x = e;
                    if constexpr (!kTarget) {
                        const Arc arc = ldg_arc(&g.arcs[e]);
                        x = static_cast<uint32_t>(arc.col);
                        id[u] = arc.id;
                    }
                    const int64_t xrow = static_cast<int64_t>(x) * kTile + s;
                    dx[u] = __ldcg(&delta[xrow]);
                    sx[u] = kTree ? 1.0 : __ldcg(&sigma[xrow]);  // every sigma is 1 in a tree
                    if constexpr (kMode == kModeGrad) {
                        gx[u] = __longlong_as_double(static_cast<long long>(__ldcg(&dist[xrow])));
                        dgx[u] = __ldcg(&delta_g[xrow]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                double c = 0.0, cg = 0.0;
                if (ok[u]) {
                    if constexpr (kMode == kModeBrandes) {
                        c = share_sv[u] * ((1.0 + dx[u]) / sx[u]);
                    } else {
                        const double share = share_sv[u] / sx[u];
                        const double inv = 1.0 / gx[u];
                        c = share * (1.0 + dx[u]);
                        cg = share * (inv * inv + dgx[u]);
                        fixed_add(&grad_cpl[2 * static_cast<int64_t>(id[u])], c);
                        fixed_add(&grad_eff[2 * static_cast<int64_t>(id[u])], cg);
                    }
                }
                wbuf[u * 32 + lane] = c;
                if constexpr (kMode == kModeGrad) {
                    wbuf[32 * kU + u * 32 + lane] = cg;
                }
            }
            __syncwarp();
            const uint32_t lo = off > p0 ? off : p0;
            const uint32_t end_own = off + count;
            const uint32_t end_chunk = p0 + 32 * kU;
            const uint32_t hi = end_own < end_chunk ? end_own : end_chunk;
            for (uint32_t q = lo; q < hi; ++q) {
                acc += wbuf[q - p0];
                if constexpr (kMode == kModeGrad) {
                    acc_g += wbuf[32 * kU + (q - p0)];
                }
            }
            __syncwarp();
        }
        if (i < len) {
            delta[row] = acc;
            if constexpr (kMode == kModeGrad) {
                delta_g[row] = acc_g;
            }
        }
    }
}

}  // namespace ngx
