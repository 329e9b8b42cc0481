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
// Betweenness per vertex and the gradients per arc are summed across tiles in 128-bit fixed point (fixed_add), so the
// totals do not depend on the order in which CTAs finish; within a tile the lanes are combined by a fixed butterfly.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "ngx_common.cuh"

namespace ngx {

enum TileMode : int { kModeApsp = 0, kModeBrandes = 1, kModeGrad = 2 };

constexpr uint32_t kNoLevel = 0xFFFFFFFFu;

struct BrandesParams {
    DeviceCsr rg;                   // reverse CSR (in-arcs), regular lengths; Arc::col = source of the arc
    double* ws_sigma;               // slots * n * kTile
    double* ws_delta;               // slots * n * kTile
    double* ws_delta_g;             // slots * n * kTile (adjoint only)
    uint32_t* ws_cnt;               // slots * n * kTile
    uint32_t* ws_lvl;               // slots * n * kTile
    int32_t* ws_list;               // slots * n * kTile: the vertices of each level, level after level
    int32_t* ws_loff;               // slots * (n + 2): start of each level in ws_list
    unsigned long long* bc;         // 2 * n fixed point (Brandes), or nullptr
    unsigned long long* grad_cpl;   // 2 * m_user fixed point (adjoint), or nullptr
    unsigned long long* grad_eff;   // 2 * m_user fixed point (adjoint), or nullptr
    unsigned long long* levels;     // total levels over all tiles (statistics)
};

inline size_t brandes_slot_bytes(int64_t n, bool adjoint) {
    const size_t nt = static_cast<size_t>(n) * kTile;
    return nt * (8 + 8 + (adjoint ? 8 : 0) + 4 + 4 + 4) + static_cast<size_t>(n + 2) * 4 + 256;
}

__device__ __forceinline__ bool on_dag(unsigned long long du_bits, double len, unsigned long long dv_bits) {
    return static_cast<unsigned long long>(__double_as_longlong(__dadd_rn(__longlong_as_double(static_cast<long long>(du_bits)), len))) == dv_bits;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        x += __shfl_xor_sync(0xFFFFFFFFu, x, off);
    }
    return x;
}

// cnt[v][s] for every vertex of the graph (warp per vertex, lane per source).
__device__ __forceinline__ void brandes_count(const DeviceCsr& rg, int64_t n, int nsrc, const int* s_src, const unsigned long long* dist, uint32_t* cnt,
                                              int lane, int warp, int nwarps) {
    for (int64_t v = warp; v < n; v += nwarps) {
        const unsigned long long dv = __ldcg(&dist[v * kTile + lane]);
        const bool active = lane < nsrc && dv != kInfBits && v != s_src[lane];
        uint32_t c = 0;
        if (__ballot_sync(0xFFFFFFFFu, active) != 0u) {
            const int64_t beg = __ldg(&rg.row_ptr[v]);
            const int64_t end = __ldg(&rg.row_ptr[v + 1]);
            for (int64_t e0 = beg; e0 < end; e0 += 32) {
                const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
                Arc a{ 0, 0, 0.0 };
                if (lane < cntr) {
                    a = rg.arcs[e0 + lane];
                }
                for (int j = 0; j < cntr; j += 4) {
                    unsigned long long du[4];
                    double len[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int jj = j + u < cntr ? j + u : 0;
                        const int src = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                        len[u] = __shfl_sync(0xFFFFFFFFu, a.len, jj);
                        du[u] = (active && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(src) * kTile + lane]) : kInfBits;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (du[u] != kInfBits && on_dag(du[u], len[u], dv)) {
                            ++c;
                        }
                    }
                }
            }
        }
        cnt[v * kTile + lane] = c;
    }
}

// Processes one level-L entry v of the sigma pass: pull sigma (L > 0), then release the DAG successors.
__device__ __forceinline__ void brandes_sigma_vertex(const DeviceCsr& g, const DeviceCsr& rg, int v, uint32_t level, int nsrc, int lane,
                                                     const unsigned long long* dist, double* sigma, uint32_t* cnt, uint32_t* lvl, uint32_t* stamp,
                                                     unsigned level_stamp, int32_t* next_list, int* next_len) {
    const int64_t vrow = static_cast<int64_t>(v) * kTile + lane;
    const bool ready = lane < nsrc && __ldcg(&lvl[vrow]) == level;
    if (__ballot_sync(0xFFFFFFFFu, ready) == 0u) {
        return;
    }
    const unsigned long long dv = __ldcg(&dist[vrow]);
    if (level > 0) {
        double sig = 0.0;
        const int64_t beg = __ldg(&rg.row_ptr[v]);
        const int64_t end = __ldg(&rg.row_ptr[v + 1]);
        for (int64_t e0 = beg; e0 < end; e0 += 32) {
            const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
            Arc a{ 0, 0, 0.0 };
            if (lane < cntr) {
                a = rg.arcs[e0 + lane];
            }
            for (int j = 0; j < cntr; j += 4) {
                unsigned long long du[4];
                int src[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = j + u < cntr ? j + u : 0;
                    src[u] = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                    du[u] = (ready && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(src[u]) * kTile + lane]) : kInfBits;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const double len = __shfl_sync(0xFFFFFFFFu, a.len, j + u < cntr ? j + u : 0);
                    if (du[u] != kInfBits && on_dag(du[u], len, dv)) {
                        sig += __ldcg(&sigma[static_cast<int64_t>(src[u]) * kTile + lane]);
                    }
                }
            }
        }
        if (ready) {
            sigma[vrow] = sig;
        }
    }
    const int64_t beg = __ldg(&g.row_ptr[v]);
    const int64_t end = __ldg(&g.row_ptr[v + 1]);
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
        const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
        Arc a{ 0, 0, 0.0 };
        if (lane < cntr) {
            a = g.arcs[e0 + lane];
        }
        for (int j = 0; j < cntr; j += 4) {
            unsigned long long dx[4];
            int x[4];
            double len[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j + u < cntr ? j + u : 0;
                x[u] = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                len[u] = __shfl_sync(0xFFFFFFFFu, a.len, jj);
                dx[u] = (ready && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + lane]) : kInfBits;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                bool released = false;
                if (dx[u] != kInfBits && on_dag(dv, len[u], dx[u])) {
                    const int64_t xrow = static_cast<int64_t>(x[u]) * kTile + lane;
                    if (atomicSub(&cnt[xrow], 1u) == 1u) {
                        lvl[xrow] = level + 1u;
                        released = true;
                    }
                }
                const unsigned rmask = __ballot_sync(0xFFFFFFFFu, released);
                if (rmask != 0u && lane == 0) {
                    if (atomicExch(&stamp[x[u]], level_stamp) != level_stamp) {
                        next_list[atomicAdd(next_len, 1)] = x[u];
                    }
                }
            }
        }
    }
}

// Processes one level-L entry v of the delta pass (pull over DAG out-arcs), emitting per-arc adjoint terms.
template <int kMode>
__device__ __forceinline__ void brandes_delta_vertex(const DeviceCsr& g, int v, uint32_t level, int nsrc, int lane, const unsigned long long* dist,
                                                     const double* sigma, double* delta, double* delta_g, const uint32_t* lvl,
                                                     unsigned long long* grad_cpl, unsigned long long* grad_eff) {
    const int64_t vrow = static_cast<int64_t>(v) * kTile + lane;
    const bool ready = lane < nsrc && __ldcg(&lvl[vrow]) == level;
    if (__ballot_sync(0xFFFFFFFFu, ready) == 0u) {
        return;
    }
    const unsigned long long dv = __ldcg(&dist[vrow]);
    const double sv = ready ? __ldcg(&sigma[vrow]) : 0.0;
    double acc = 0.0;
    double acc_g = 0.0;
    const int64_t beg = __ldg(&g.row_ptr[v]);
    const int64_t end = __ldg(&g.row_ptr[v + 1]);
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
        const int cntr = static_cast<int>(end - e0 < 32 ? end - e0 : 32);
        Arc a{ 0, 0, 0.0 };
        if (lane < cntr) {
            a = g.arcs[e0 + lane];
        }
        for (int j = 0; j < cntr; j += 4) {
            unsigned long long dx[4];
            int x[4];
            double len[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j + u < cntr ? j + u : 0;
                x[u] = __shfl_sync(0xFFFFFFFFu, a.col, jj);
                len[u] = __shfl_sync(0xFFFFFFFFu, a.len, jj);
                dx[u] = (ready && j + u < cntr) ? __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + lane]) : kInfBits;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool dag = dx[u] != kInfBits && on_dag(dv, len[u], dx[u]);
                const int64_t xrow = static_cast<int64_t>(x[u]) * kTile + lane;
                if constexpr (kMode == kModeBrandes) {
                    if (dag) {
                        acc += sv * ((1.0 + __ldcg(&delta[xrow])) / __ldcg(&sigma[xrow]));
                    }
                } else {
                    double c = 0.0, cg = 0.0;
                    if (dag) {
                        const double share = sv / __ldcg(&sigma[xrow]);
                        const double inv = 1.0 / __longlong_as_double(static_cast<long long>(dx[u]));
                        c = share * (1.0 + __ldcg(&delta[xrow]));
                        cg = share * (inv * inv + __ldcg(&delta_g[xrow]));
                        acc += c;
                        acc_g += cg;
                    }
                    if (__ballot_sync(0xFFFFFFFFu, dag) != 0u) {
                        const double sc = warp_sum(c);
                        const double sg = warp_sum(cg);
                        const int id = __shfl_sync(0xFFFFFFFFu, a.id, j + u < cntr ? j + u : 0);
                        if (lane == 0) {
                            fixed_add(&grad_cpl[2 * static_cast<int64_t>(id)], sc);
                            fixed_add(&grad_eff[2 * static_cast<int64_t>(id)], sg);
                        }
                    }
                }
            }
        }
    }
    if (ready) {
        delta[vrow] = acc;
        if constexpr (kMode == kModeGrad) {
            delta_g[vrow] = acc_g;
        }
    }
}

}  // namespace ngx
