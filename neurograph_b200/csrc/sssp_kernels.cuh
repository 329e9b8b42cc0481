// Batched and plain multi-source delta-stepping kernels with the fused APSP epilogue (sm_100a).
//
// Both kernels are persistent: one CTA per workspace slot, each CTA takes source tiles from a device work counter until
// none are left. A tile is either NGX_TILE sources (batched form: lane s of every warp owns source s of the tile) or
// one source (plain form: the lanes of a warp stride over one vertex's arcs).
//
// Per tile the CTA runs delta-stepping with a common bucket bound theta for all its sources:
//   near phase   vertices whose pending (vertex, source) pairs lie below theta are expanded; an improvement below
//                theta marks the pair pending for the next iteration, one at or above theta marks it "far"; after
//                the iteration the next queue is compacted from the pending masks (warp ballot + prefix);
//   bucket step  when no near work is left, one pass over the far marks finds the smallest pending distance d_min,
//                theta becomes (floor(d_min / delta) + 1) * delta, and the pairs below it move to the near queue.
// Relaxation is fl(d[u] + len) compared and stored with a 64-bit atomicMin on the bit pattern, which orders
// non-negative doubles like their values. The label-correcting fixed point is the same as the reference Dijkstra's
// (PriorityQueueVariant.h:47-93: d[v] = min over arcs of fl(d[u] + |w|)), so distances are bit-identical.
//
// Race-freedom of the pending marks: expansions of iteration k read and clear pend[k % 2]; improvements made during
// iteration k set pend[(k + 1) % 2] and the far marks; iterations are separated by (group) barriers. A pair improved
// while its vertex is being expanded is therefore always expanded again in the next iteration, with the new distance.
// All distance reads go through L2 (__ldcg), where the atomics are performed.
//
// Epilogue (after a tile's distances are final), per (vertex, source), replacing summarize_distances
// (types/SsspResult.h:42-64) and the aggregation of AllPairsShortestPath::compute_apsp_impl (:110-163): unreachable
// count, exact sums of d and of 1/d (order-independent integer accumulators, rounded once), maximum finite distance,
// traversed arcs, and the distance histogram (bin floor(d / (hist_max / bins)), clamped to the last bin, as
// FixedSizeHistogram::add_data_point, external/cpp-utility/data-structure/Histogram.hpp:166-180). The distances are
// reset to +inf in the same pass, so the N x N distances never leave the per-CTA workspace.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "brandes_kernels.cuh"
#include "ngx_common.cuh"
#include "ngx_group.cuh"

namespace ngx {

constexpr unsigned kFullMask = 0xFFFFFFFFu;

struct TileOutputs {
    unsigned long long* acc_sum;    // per graph: kAccDigits words of the exact sum of distances, then kAccDigits for 1/d
    unsigned long long* acc_inv;    // unused by the tile kernel (acc_sum + kAccDigits of each graph)
    unsigned long long* counters;   // per graph: kCounterCount words (see Counter)
    unsigned long long* hist;       // per graph: hist_bins words (or nullptr)
    int hist_bins;
    double hist_width;
    double hist_max;
    double* src_sum;                // per tile position (or nullptr)
    double* src_max;
    double* src_inv;
    unsigned long long* src_unreach;
    unsigned long long* src_arcs;
    double* rows;                   // num_sources x n distance rows (or nullptr)
};


struct SsspParams {
    DeviceCsr g;                   // concatenated CSR: row_ptr over all graphs' rows, arcs with graph-local targets; g.n = largest n
    const int32_t* sources;        // tile order (graph-local ids)
    int64_t num_sources;
    int64_t num_tiles;             // work items
    double delta;
    const GraphDesc* graphs;       // batch table (tile kernel)
    const WorkItem* items;         // work items in scheduling order, or nullptr: tile t of graph 0
    unsigned long long max_iterations;  // per tile
    unsigned long long* tile_counter;
    int* error;
    const volatile int* abort_flag;
    // workspace, carved per slot (blockIdx.x)
    unsigned long long* ws_dist;   // slots * n * width (width = kTile batched, 1 plain)
    uint32_t* ws_pend;             // slots * 2n
    uint32_t* ws_far;              // slots * n
    int32_t* ws_queue;             // slots * 2n
    uint32_t* ws_stamp;            // slots * n
    // reach lists (graphs of several strongly connected components; nullptr otherwise): per vertex the tile's
    // sources that reached it, and the list of the vertices reached, so that per-tile passes visit only those
    uint32_t* ws_reach;            // slots * n
    int32_t* ws_touched;           // slots * n
    // groups: the CTAs blockIdx.x / group_size share slot (blockIdx.x / group_size) and its tiles
    int group_size;
    int64_t group_stride;          // words of group storage per slot (group_stride_words)
    unsigned long long* group_ws;  // slots * group_stride words, zero at launch
    TileOutputs out;
};

// Bytes of per-slot workspace for a graph with n vertices.
inline size_t sssp_slot_bytes(int64_t n, int width) {
    return static_cast<size_t>(n) * (static_cast<size_t>(width) * 8 + 4 * 2 + 4 + 4 * 2 + 4) + 256;
}


__device__ __forceinline__ double next_theta(double d_min, double delta) {
    const double theta = (floor(__ddiv_rn(d_min, delta)) + 1.0) * delta;
    return theta > d_min ? theta : INFINITY;
}

// Control block of the CTAs working on one tile: one per workspace slot in global memory, and a copy in each CTA's
// shared memory that every group barrier refreshes (ngx_group.cuh). Only atomics and barrier updates change it.
struct TileShared {
    long long tile;
    int qlen[2];
    int cur;
    int stop;
    unsigned stamp;                 // id of the DAG pass about to run (dedup of its level lists)
    int done;                       // bucket step: no pending far pair is left
    double theta;
    double theta_next;              // bucket step: the bound below which pass 2 moves pairs to the near queue
    unsigned long long min_bits;
    unsigned long long iterations;
    unsigned long long overflow;    // histogram overflow of the tile (plain form)
    // Brandes / adjoint levels
    unsigned level;
    int lvl_start;
    int lvl_len;
    int next_len;
    unsigned long long active_pairs;  // reached (vertex, source) pairs other than the sources, counted by the DAG pass
    int grab;                       // next queue entry handed to a warp in the current near iteration
    int touched_len;                // vertices the tile has reached so far (reach lists; see SsspParams::ws_touched)
    // the state of a CTA that left its group (ngx_group.cuh): no tile, nothing queued, pending or levelled
    __device__ void halt() {
        stop = 1;
        tile = 0x7FFFFFFFFFFFFFFFll;
        qlen[0] = 0;
        qlen[1] = 0;
        done = 1;
        level = 0u;
        lvl_start = 0;
        lvl_len = 0;
    }
};
static_assert(sizeof(TileShared) % 8 == 0, "TileShared is copied in 8-byte words");

// Per-slot group storage, in 8-byte words: the control block, the barrier, one scan partial per CTA, and (groups of
// several CTAs) the per-source epilogue sums: exact accumulators of d and 1/d, unreachable, arcs and maximum per source.
constexpr int kCtlWords = static_cast<int>(sizeof(TileShared) / 8);
constexpr int kGroupAccWords = 2 * kTile * kAccDigits + 3 * kTile;
inline int64_t group_stride_words(int group_size) {
    const int64_t words = kCtlWords + 1 + group_size + (group_size > 1 ? kGroupAccWords : 0);
    return (words + 31) / 32 * 32;  // 256-byte aligned slots
}

// This CTA's view of its tile group (see SsspParams::group_*). A group of one CTA keeps the control block in the CTA's
// shared memory (`local`), where its counters are shared-memory atomics; larger groups keep it in global memory.
template <typename Params>
__device__ __forceinline__ Group<TileShared> tile_group(const Params& p, TileShared* local) {
    unsigned long long* const gws = p.group_ws + (blockIdx.x / p.group_size) * p.group_stride;
    TileShared* const ctl = p.group_size == 1 ? local : reinterpret_cast<TileShared*>(gws);
    return Group<TileShared>{ ctl, reinterpret_cast<GroupBarrier*>(gws + kCtlWords), gws + kCtlWords + 1, p.group_size,
                              static_cast<int>(blockIdx.x % p.group_size), p.error };
}

// Queue entries a warp takes at a time (guided self-scheduling): the entries not yet handed out over twice the group's
// warps, clamped to 1..32, so a near iteration starts with large chunks (one round of loads serves many entries) and
// ends with single entries (a vertex expansion takes tens of microseconds: a coarse last chunk would leave the other
// warps of the group waiting at the barrier that closes the iteration).
__device__ __forceinline__ int expand_chunk(int remaining, int group_warps) {
    const int c = remaining / (2 * group_warps);
    return c < 1 ? 1 : (c > 32 ? 32 : c);
}

// The reach list of a tile: mask[v] has bit s set once source s reached v; a vertex is appended to list[] (length
// *len) by the relaxation that gives it its first finite distance of the tile. Disabled when mask is nullptr.
struct Reach {
    uint32_t* mask;
    int32_t* list;
    int* len;
    __device__ __forceinline__ void add(int v, uint32_t bit) const {
        if (atomicOr(&mask[v], bit) == 0u) {
            list[atomicAdd(len, 1)] = v;
        }
    }
};

// The relaxations of kUnroll (arc, source) pairs per lane, their loads done: pair u relaxes d[x[u]][src[u]] with nd[u]
// (cur[u] = the distance read before). The atomic minima are issued back to back and waited for together (APSP mode:
// not waited for at all), then the marks; see batched_expand for what each mode does with an improvement.
template <int kUnroll, bool kTrack, bool kReach>
__device__ __forceinline__ void relax_pairs(const int (&x)[kUnroll], const int (&src)[kUnroll], const double (&nd)[kUnroll],
                                            unsigned long long (&cur)[kUnroll], const uint32_t (&eidx)[kUnroll], const bool (&valid)[kUnroll],
                                            unsigned long long* __restrict__ dist, uint32_t* pend_nxt, uint32_t* far, double theta,
                                            unsigned long long* pred_key, uint32_t* tie, const Reach& reach) {
    // the atomic minima (cur[u] becomes the old value where it is waited for)
    bool tried[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const unsigned long long nb = static_cast<unsigned long long>(__double_as_longlong(nd[u]));
        tried[u] = valid[u] && nb < cur[u];
        if (tried[u]) {
            if constexpr (kTrack) {
                cur[u] = atomicMin(&dist[static_cast<int64_t>(x[u]) * kTile + src[u]], nb);
            } else {
                atomicMin(&dist[static_cast<int64_t>(x[u]) * kTile + src[u]], nb);
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const unsigned long long nb = static_cast<unsigned long long>(__double_as_longlong(nd[u]));
        if (tried[u]) {
            const unsigned long long old = cur[u];
            if constexpr (kTrack) {
                if (nb < old) {
                    atomicMin(&pred_key[static_cast<int64_t>(x[u]) * kTile + src[u]], ((nb >> 32) << 32) | eidx[u]);
                } else if (nb == old) {
                    atomicOr(&tie[x[u]], 1u << src[u]);
                }
            }
            if (nb < old) {
                const uint32_t bit = 1u << src[u];
                if (kReach && old == kInfBits) {
                    reach.add(x[u], bit);  // the first distance of (x, s): x joins the tile's reached vertices
                }
                if (nd[u] < theta) {
                    atomicOr(&pend_nxt[x[u]], bit);
                } else {
                    atomicOr(&far[x[u]], bit);
                }
            }
        } else if (kTrack && valid[u] && nb == cur[u]) {
            atomicOr(&tie[x[u]], 1u << src[u]);
        }
    }
}

// ------------------------------------------------------------------------------------------ batched form
// Expands vertex v for the k sources pending on it. The deg(v) x k (arc, source) pairs are spread over the 32 lanes:
// pair p = 32 i + lane takes arc p / k and the (p % k)-th pending source, so no lane idles when few sources are
// pending, and when all 32 are, every iteration reads one whole distance row d[x][0..31] (256 contiguous bytes).
// An improvement below theta sets the pair's bit in pend_nxt (the next iteration's queue is compacted from those
// masks after the iteration), one at or above theta its far mark. The kUnroll relaxations of a lane are issued back
// to back and waited for together.
// APSP mode: the atomic minimum is not waited for. An improvement is judged against the distance read before it, so
// a relaxation that lost a race to a smaller value may still set a pending bit or a far mark: the pair is then
// expanded once more with its (smaller) current distance, or its superseded far mark is cleared or moved by the next
// expansion or bucket step, which changes the work and never the fixed point.
// kTrack (betweenness / adjoint): the atomic minimum returns the old value. Each improvement of d[x][s] to nb offers
// the key (top 32 bits of nb, arc index) to pred_key[x][s] with an atomic minimum, so the key of the smallest
// distance wins whatever the order of the stores; a relaxation that ties with d[x][s] sets bit s of tie[x]. Every
// DAG arc is relaxed with final distances, so a (x, s) whose tie bit stayed clear has exactly one DAG predecessor: the
// arc in its key (the DAG count pass checks it). For that, no (v, s) may be expanded twice with one distance (the
// repeat would look like a tie): last[v][s] keeps the distance of the latest expansion, and sources whose distance has
// not changed since are dropped from the next.
// The caller has taken v's pending mask (amask, non-zero), cleared it and v's superseded far marks, and read its row
// offsets (beg, deg): see expand_queue.
template <int kUnroll, bool kTrack, bool kReach>
__device__ __forceinline__ void batched_expand(const DeviceCsr& g, int v, uint32_t amask, int64_t beg, int deg, int lane,
                                               unsigned long long* __restrict__ dist, uint32_t* pend_nxt, uint32_t* far, double theta,
                                               unsigned long long& expansions, unsigned long long& lane_expansions, unsigned long long* pred_key,
                                               uint32_t* tie, unsigned long long* last, const Reach& reach) {
    const uint32_t amask0 = amask;
    int k = __popc(amask);
    // lane r < k holds the r-th pending source and its distance to v
    int rank_src = lane < k ? static_cast<int>(__fns(amask, 0, lane + 1)) : 0;
    unsigned long long rank_bits = __ldcg(&dist[static_cast<int64_t>(v) * kTile + rank_src]);
    if constexpr (kTrack) {
        unsigned long long* const slot = &last[static_cast<int64_t>(v) * kTile + rank_src];
        const bool repeat = lane < k && __ldcg(slot) == rank_bits;
        if (lane < k && !repeat) {
            *slot = rank_bits;
        }
        const uint32_t drop = __reduce_or_sync(kFullMask, repeat ? (1u << rank_src) : 0u);
        if (drop != 0u) {
            amask &= ~drop;
            if (amask == 0u) {
                return;
            }
            // re-rank the remaining sources; their distances come from the lanes that read them
            const int new_k = __popc(amask);
            const int src_new = lane < new_k ? static_cast<int>(__fns(amask, 0, lane + 1)) : 0;
            const int old_rank = __popc(amask0 & ((1u << src_new) - 1u));
            rank_bits = __shfl_sync(kFullMask, rank_bits, old_rank);
            rank_src = src_new;
            k = new_k;
        }
    }
    expansions += 1;
    lane_expansions += static_cast<unsigned long long>(k);
    const double rank_dv = __longlong_as_double(static_cast<long long>(rank_bits));
    const Arc* arcs = g.arcs + beg;
    // v's arc records (16 B each) into L1 ahead of the pair loop, one 128-byte line per lane
    if (lane * 8 < deg) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(arcs + lane * 8));
    }
    // position of this lane's first pair, and the per-iteration advance of 32 pairs
    int a = lane / k;
    int r = lane - a * k;
    const int step_a = 32 / k;
    const int step_r = 32 - step_a * k;
    const int64_t total = static_cast<int64_t>(deg) * k;
    for (int64_t p0 = 0; p0 < total; p0 += 32 * kUnroll) {
        int x[kUnroll];
        int src[kUnroll];
        double nd[kUnroll];
        unsigned long long cur[kUnroll];
        uint32_t eidx[kUnroll];
        bool valid[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            valid[u] = a < deg;
            eidx[u] = static_cast<uint32_t>(beg + a);
            src[u] = __shfl_sync(kFullMask, rank_src, r);
            const double dvs = __shfl_sync(kFullMask, rank_dv, r);
            x[u] = 0;
            nd[u] = 0.0;
            cur[u] = 0ull;
            if (valid[u]) {
                const Arc arc = ldg_arc(&arcs[a]);
                x[u] = arc.col;
                nd[u] = __dadd_rn(dvs, arc.len);
                cur[u] = __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + src[u]]);
            }
            a += step_a;
            r += step_r;
            if (r >= k) {
                r -= k;
                a += 1;
            }
        }
        relax_pairs<kUnroll, kTrack, kReach>(x, src, nd, cur, eidx, valid, dist, pend_nxt, far, theta, pred_key, tie, reach);
    }
}

// Queue entries with fewer (arc, pending source) pairs than this fill less than one iteration of batched_expand's
// pair loop (32 lanes x 4 pairs at the library's unroll); consecutive ones are expanded together by packed_expand,
// whose division of a pair index by the entry's source count is exact only below 2^7 pairs per entry.
constexpr int kPackPairs = 128;
static_assert(kPackPairs <= 128, "packed_expand divides pair indices below 2^7 by a 16-bit reciprocal");

// Expands a group of m small queue entries together, so that one iteration of the pair loop serves several vertices.
// Lane i < m holds entry i: its vertex gv, pending mask gmask (non-zero), first arc gbeg and out-degree gdeg; the
// entries have at most 32 pending sources in all. Lane t then holds the t-th (entry, pending source) of the group and
// that source's distance to the entry's vertex, and the group's pairs are dealt to the lanes entry after entry: pair
// q of entry i (0 <= q < k_i deg_i) is arc q / k_i with the (q % k_i)-th pending source, as in batched_expand. The
// relaxations, the repeat check of the DAG modes (a repeated (vertex, source) only drops its own pairs here) and the
// counters are batched_expand's.
template <int kUnroll, bool kTrack, bool kReach>
__device__ __forceinline__ void packed_expand(const DeviceCsr& g, int m, int gv, uint32_t gmask, int64_t gbeg, int gdeg, int lane,
                                              unsigned long long* __restrict__ dist, uint32_t* pend_nxt, uint32_t* far, double theta,
                                              unsigned long long& expansions, unsigned long long& lane_expansions, unsigned long long* pred_key,
                                              uint32_t* tie, unsigned long long* last, const Reach& reach) {
    // per entry (lane i < m): pending sources k_i, pairs, offsets of its ranks and pairs in the group, 16-bit reciprocal
    const int ki = lane < m ? __popc(gmask) : 0;
    const int pi = lane < m ? ki * gdeg : 0;
    int kinc = ki, pinc = pi;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int ku = __shfl_up_sync(kFullMask, kinc, off);
        const int pu = __shfl_up_sync(kFullMask, pinc, off);
        if (lane >= off) {
            kinc += ku;
            pinc += pu;
        }
    }
    const int ri = kinc - ki;
    const int si = pinc - pi;
    const int ktot = __shfl_sync(kFullMask, kinc, 31);
    const int ptot = __shfl_sync(kFullMask, pinc, 31);
    // floor(q / k) = (q * ceil(2^16 / k)) >> 16 exactly for q < 2^7 and k <= 32
    const int mgi = lane < m ? (65536 + ki - 1) / ki : 0;
    // lane t < ktot: its entry (the number of entries whose ranks start at or below t, minus one) and rank
    const unsigned starts = __reduce_or_sync(kFullMask, lane < m ? (1u << ri) : 0u);
    const int et = lane < ktot ? __popc(starts & ((2u << lane) - 1u)) - 1 : 0;
    const uint32_t emask = __shfl_sync(kFullMask, gmask, et);
    const int ev = __shfl_sync(kFullMask, gv, et);
    const int er = __shfl_sync(kFullMask, ri, et);
    const int rank_src = lane < ktot ? static_cast<int>(__fns(emask, 0, lane - er + 1)) : 0;
    const unsigned long long rank_bits = __ldcg(&dist[static_cast<int64_t>(ev) * kTile + rank_src]);
    bool rank_ok = lane < ktot;
    if constexpr (kTrack) {
        unsigned long long* const slot = &last[static_cast<int64_t>(ev) * kTile + rank_src];
        if (rank_ok && __ldcg(slot) == rank_bits) {
            rank_ok = false;  // expanded with this distance already
        } else if (rank_ok) {
            *slot = rank_bits;
        }
    }
    const unsigned ok_mask = __ballot_sync(kFullMask, rank_ok);
    if (ok_mask == 0u) {
        return;
    }
    expansions += static_cast<unsigned long long>(m);
    lane_expansions += static_cast<unsigned long long>(__popc(ok_mask));
    const double rank_dv = __longlong_as_double(static_cast<long long>(rank_bits));
    if (lane < m) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(g.arcs + gbeg));
    }
    for (int p0 = 0; p0 < ptot; p0 += 32 * kUnroll) {
        int x[kUnroll];
        int src[kUnroll];
        double nd[kUnroll];
        unsigned long long cur[kUnroll];
        uint32_t eidx[kUnroll];
        bool valid[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int q = p0 + u * 32 + lane;
            // the entry of pair q: the last one whose pairs start at or below q
            int e = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int c = e + step;
                const int sc = __shfl_sync(kFullMask, si, c & 31);
                e = (c < m && sc <= q) ? c : e;
            }
            const int local = q - __shfl_sync(kFullMask, si, e);
            const int ke = __shfl_sync(kFullMask, ki, e);
            const int a = (local * __shfl_sync(kFullMask, mgi, e)) >> 16;
            const int t = (__shfl_sync(kFullMask, ri, e) + local - a * ke) & 31;
            const int64_t beg_e = __shfl_sync(kFullMask, gbeg, e);
            src[u] = __shfl_sync(kFullMask, rank_src, t);
            const double dvs = __shfl_sync(kFullMask, rank_dv, t);
            valid[u] = q < ptot && ((ok_mask >> t) & 1u);
            eidx[u] = static_cast<uint32_t>(beg_e + a);
            x[u] = 0;
            nd[u] = 0.0;
            cur[u] = 0ull;
            if (valid[u]) {
                const Arc arc = ldg_arc(&g.arcs[beg_e + a]);
                x[u] = arc.col;
                nd[u] = __dadd_rn(dvs, arc.len);
                cur[u] = __ldcg(&dist[static_cast<int64_t>(x[u]) * kTile + src[u]]);
            }
        }
        relax_pairs<kUnroll, kTrack, kReach>(x, src, nd, cur, eidx, valid, dist, pend_nxt, far, theta, pred_key, tie, reach);
    }
}

// One near iteration of a tile: the warps of the group take the queue in chunks (expand_chunk) from a shared counter;
// lane j fetches entry j's vertex, its pending mask, far marks and row offsets (one round of parallel loads), clears the
// mask and the superseded far marks, and the warp then expands the vertices one after another: one at a time when a
// vertex has a loop iteration's worth of (arc, source) pairs or more, else with its small neighbours in the chunk.
template <int kUnroll, bool kTrack, bool kReach>
__device__ __forceinline__ void expand_queue(const DeviceCsr& g, const int32_t* q_cur, int qlen, int lane, int* grab, int group_warps,
                                             unsigned long long* __restrict__ dist, uint32_t* pend_cur, uint32_t* pend_nxt, uint32_t* far,
                                             double theta, unsigned long long& expansions, unsigned long long& lane_expansions,
                                             unsigned long long* pred_key, uint32_t* tie, unsigned long long* last, const Reach& reach) {
    for (;;) {
        int base = 0;
        int chunk = 0;
        if (lane == 0) {
            // the grab counter is in shared memory for single-CTA tiles and in global memory for groups: a volatile
            // generic load reads either (for global memory, from L2)
            chunk = expand_chunk(qlen - *reinterpret_cast<volatile int*>(grab), group_warps);
            base = atomicAdd(grab, chunk);
        }
        base = __shfl_sync(kFullMask, base, 0);
        chunk = __shfl_sync(kFullMask, chunk, 0);
        if (base >= qlen) {
            break;
        }
        const int i = base + lane;
        const int count = qlen - base < chunk ? qlen - base : chunk;
        int vj = 0;
        uint32_t mj = 0;
        int64_t bj = 0;
        int dj = 0;
        if (lane < count) {
            vj = __ldcg(&q_cur[i]);
            mj = __ldcg(&pend_cur[vj]);
            const uint32_t fm = __ldcg(&far[vj]);
            bj = __ldg(&g.row_ptr[vj]);
            dj = static_cast<int>(__ldg(&g.row_ptr[vj + 1]) - bj);
            if (mj != 0u) {
                pend_cur[vj] = 0u;
                if (fm & mj) {
                    atomicAnd(&far[vj], ~mj);  // those far marks are superseded by the near values expanded now
                }
            }
        }
        // entries with fewer pairs than one loop iteration holds go in groups (packed_expand), the others one by one
        const int kj = __popc(mj);
        const unsigned any_mask = __ballot_sync(kFullMask, lane < count && mj != 0u);
        const unsigned small_mask = __ballot_sync(kFullMask, lane < count && mj != 0u && kj * dj < kPackPairs);
        int j = 0;
        while (j < count) {
            const unsigned rest = any_mask & ~((1u << j) - 1u);
            if (rest == 0u) {
                break;
            }
            j = __ffs(rest) - 1;  // the next entry with pending sources
            unsigned fit = 0u;
            if ((small_mask >> j) & 1u) {
                // the small entries from j up to the next large one, as many as hold 32 pending sources
                const unsigned large_after = any_mask & ~small_mask & ~((1u << j) - 1u);
                const int stop = large_after != 0u ? __ffs(large_after) - 1 : 32;
                const unsigned run = small_mask & ~((1u << j) - 1u) & (stop >= 32 ? kFullMask : ((1u << stop) - 1u));
                const bool in_run = (run >> lane) & 1u;
                int kin = in_run ? kj : 0;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int ku = __shfl_up_sync(kFullMask, kin, off);
                    if (lane >= off) {
                        kin += ku;
                    }
                }
                fit = __ballot_sync(kFullMask, in_run && kin <= 32);
            }
            if (__popc(fit) > 1) {
                const int m = __popc(fit);
                const int sl = lane < m ? static_cast<int>(__fns(fit, 0, lane + 1)) : 0;
                const int gv = __shfl_sync(kFullMask, vj, sl);
                const uint32_t gmask = __shfl_sync(kFullMask, mj, sl);
                const int64_t gbeg = __shfl_sync(kFullMask, bj, sl);
                const int gdeg = __shfl_sync(kFullMask, dj, sl);
                packed_expand<kUnroll, kTrack, kReach>(g, m, gv, gmask, gbeg, gdeg, lane, dist, pend_nxt, far, theta, expansions,
                                                       lane_expansions, pred_key, tie, last, reach);
                j = 32 - __clz(fit);
            } else {
                const uint32_t amask = __shfl_sync(kFullMask, mj, j);
                const int v = __shfl_sync(kFullMask, vj, j);
                const int64_t beg = __shfl_sync(kFullMask, bj, j);
                const int deg = __shfl_sync(kFullMask, dj, j);
                batched_expand<kUnroll, kTrack, kReach>(g, v, amask, beg, deg, lane, dist, pend_nxt, far, theta, expansions, lane_expansions,
                                                        pred_key, tie, last, reach);
                ++j;
            }
        }
    }
}

// The next iteration's queue: the group's warps scan the pending masks `pend` (over the tile's reached vertices when
// it keeps a reach list: no other vertex can be pending) and append every vertex with a pending source to `q`, 32 at
// a time with one ballot and one atomic per warp.
template <bool kReach>
__device__ __forceinline__ void compact_queue(const uint32_t* pend, int32_t* q, int* qlen, int64_t span, const Reach& reach, int lane, int gw,
                                              int gwarps) {
    for (int64_t vb = static_cast<int64_t>(gw) * 32; vb < span; vb += static_cast<int64_t>(gwarps) * 32) {
        const int64_t i = vb + lane;
        const int64_t v = i < span ? (kReach ? static_cast<int64_t>(__ldcg(&reach.list[i])) : i) : 0;
        const uint32_t m = i < span ? __ldcg(&pend[v]) : 0u;
        const unsigned bal = __ballot_sync(kFullMask, m != 0u);
        if (bal != 0u) {
            int qb = 0;
            if (lane == 0) {
                qb = atomicAdd(qlen, __popc(bal));
            }
            qb = __shfl_sync(kFullMask, qb, 0);
            if (m != 0u) {
                q[qb + __popc(bal & lanemask_lt())] = static_cast<int32_t>(v);
            }
        }
    }
}

// kMulti: the launch may put several CTAs on a tile (p.group_size > 1, cooperative launch); without it the group is
// the CTA itself, whose control block lives in shared memory. kReach: the tiles keep reach lists.
template <int kMode, int kUnroll, int kBlock, int kMinBlocks, bool kMulti = false, bool kReach = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) tile_kernel(const SsspParams p, const BrandesParams b) {
    extern __shared__ __align__(16) unsigned long long smem[];
    unsigned long long* s_acc_sum = smem;                                // kTile * kAccDigits
    unsigned long long* s_acc_inv = smem + kTile * kAccDigits;          // kTile * kAccDigits
    unsigned int* s_hist = reinterpret_cast<unsigned int*>(smem + 2 * kTile * kAccDigits);
    __shared__ TileShared s;
    __shared__ unsigned s_bar;
    __shared__ int s_src[kTile];
    __shared__ unsigned long long s_unreach[kTile];
    __shared__ unsigned long long s_arcs[kTile];
    __shared__ unsigned long long s_max[kTile];
    __shared__ unsigned long long s_part[kBlock + 3];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int64_t n_slot = p.g.n;  // every slot holds the largest graph of the batch
    // The CTAs blockIdx.x / group_size share workspace slot `slot` and work on its tiles together. The group's
    // pointers and indices are recomputed from the launch parameters where they are used (fewer live registers).
    const int64_t slot = blockIdx.x / p.group_size;
    const auto grp = [&]() { return tile_group(p, &s); };
    const auto ctl = [&]() {
        return kMulti ? reinterpret_cast<TileShared*>(p.group_ws + (blockIdx.x / p.group_size) * p.group_stride) : &s;
    };
    // a group barrier whose last arrival applies `update` to the control block (a block barrier without kMulti)
    const auto sync = [&](auto&& update) {
        if constexpr (kMulti) {
            grp().sync(s, s_bar, update);
        } else {
            __syncthreads();
            if (threadIdx.x == 0) {
                update(s);
            }
            __syncthreads();
        }
    };
    const auto sync0 = [&]() { sync([](volatile TileShared&) {}); };
    // this thread's (warp's) index among the group's threads (warps), and their counts
#define NGX_GT (kMulti ? static_cast<int64_t>(blockIdx.x % p.group_size) * blockDim.x + threadIdx.x : static_cast<int64_t>(threadIdx.x))
#define NGX_GTHREADS (kMulti ? static_cast<int64_t>(p.group_size) * blockDim.x : static_cast<int64_t>(blockDim.x))
#define NGX_GW (kMulti ? static_cast<int>(blockIdx.x % p.group_size) * static_cast<int>(blockDim.x >> 5) + static_cast<int>(threadIdx.x >> 5) \
                       : static_cast<int>(threadIdx.x >> 5))
#define NGX_GWARPS (kMulti ? p.group_size * static_cast<int>(blockDim.x >> 5) : static_cast<int>(blockDim.x >> 5))
    unsigned long long expansions = 0, lane_expansions = 0;

    unsigned long long* dist = p.ws_dist + slot * n_slot * kTile;
    uint32_t* pend0 = p.ws_pend + slot * 2 * n_slot;
    uint32_t* pend1 = pend0 + n_slot;
    uint32_t* far = p.ws_far + slot * n_slot;
    int32_t* q0 = p.ws_queue + slot * 2 * n_slot;
    int32_t* q1 = q0 + n_slot;
    uint32_t* stamp = p.ws_stamp + slot * n_slot;
    // reach lists: compiled in only for the kernels that keep them (kReach), so the others carry no extra registers
    const Reach reach{ kReach ? p.ws_reach + slot * n_slot : nullptr, kReach ? p.ws_touched + slot * n_slot : nullptr,
                       kReach ? &ctl()->touched_len : nullptr };
    const int64_t nt_slot = n_slot * kTile;
    double* sigma = nullptr;
    double* delta = nullptr;
    double* delta_g = nullptr;
    uint32_t* cnt = nullptr;
    uint32_t* lvl = nullptr;
    int32_t* list = nullptr;
    int32_t* loff = nullptr;
    uint32_t* scnt = nullptr;
    uint32_t* soff = nullptr;
    uint32_t* succ = nullptr;
    uint32_t* tie = nullptr;
    if constexpr (kMode != kModeApsp) {
        scnt = b.ws_scnt + slot * nt_slot;
        soff = b.ws_soff + slot * (nt_slot + 1);
        succ = b.ws_succ + slot * b.succ_capacity;
        sigma = b.ws_sigma + slot * nt_slot;
        delta = b.ws_delta + slot * nt_slot;
        delta_g = kMode == kModeGrad ? b.ws_delta_g + slot * nt_slot : nullptr;
        cnt = b.ws_cnt + slot * nt_slot;
        lvl = b.ws_lvl + slot * nt_slot;
        list = b.ws_list + slot * nt_slot;
        loff = b.ws_loff + slot * (n_slot + 2);
        tie = b.ws_tie + slot * n_slot;
        for (int64_t i = NGX_GT; i < n_slot; i += NGX_GTHREADS) {
            tie[i] = 0u;
        }
        for (int64_t i = NGX_GT; i < nt_slot; i += NGX_GTHREADS) {
            scnt[i] = 0u;
            sigma[i] = __longlong_as_double(-1ll);  // all-ones: the empty predecessor key (sigma is zeroed by the count pass)
            delta[i] = __longlong_as_double(-1ll);  // all-ones: no expansion yet (delta holds last[][] in the SSSP phase)
            if constexpr (kMode == kModeGrad) {
                delta_g[i] = 0.0;
            }
            cnt[i] = 0u;
            lvl[i] = kNoLevel;
        }
    }

    for (int64_t i = NGX_GT; i < nt_slot; i += NGX_GTHREADS) {
        dist[i] = kInfBits;
    }
    for (int64_t i = NGX_GT; i < n_slot; i += NGX_GTHREADS) {
        pend0[i] = 0u;
        pend1[i] = 0u;
        far[i] = 0u;
        stamp[i] = 0u;
        if (kReach) {
            reach.mask[i] = 0u;
        }
    }
    for (int i = tid; i < 2 * kTile * kAccDigits; i += blockDim.x) {
        smem[i] = 0ull;
    }
    for (int i = tid; i < p.out.hist_bins; i += blockDim.x) {
        s_hist[i] = 0u;
    }
    if (tid == 0) {
        s_bar = 0u;
    }
    bool first_tile = true;

    for (;;) {
        // ---- the next work item, taken for the whole group; the slot's stamp counts on across tiles
        sync([&](volatile TileShared& c) {
            if (first_tile) {
                c.stamp = 1u;
            }
            c.tile = static_cast<long long>(atomicAdd(p.tile_counter, 1ull));
            c.stop = *reinterpret_cast<volatile int*>(p.error) != 0 ? 1 : 0;
            c.qlen[0] = 0;
            c.qlen[1] = 0;
            c.cur = 0;
            c.done = 0;
            c.iterations = 0;
            c.min_bits = kInfBits;
            c.active_pairs = 0;
            c.grab = 0;
            c.touched_len = 0;
            if (c.tile < p.num_tiles) {
                const WorkItem it = p.items != nullptr ? p.items[c.tile] : WorkItem{ 0, static_cast<int32_t>(c.tile) };
                c.theta = p.graphs[it.graph].delta;
            }
        });
        first_tile = false;
        if (s.stop != 0 || s.tile >= p.num_tiles) {
            break;
        }
        // ---- the work item: tile `item.tile` of graph `item.graph`
        const WorkItem item = p.items != nullptr ? p.items[s.tile] : WorkItem{ 0, static_cast<int32_t>(s.tile) };
        const GraphDesc gd = p.graphs[item.graph];
        const int64_t n = gd.n;
        const int64_t nt = n * kTile;
        const DeviceCsr g{ gd.n, gd.m, p.g.row_ptr + gd.row_off, p.g.arcs };
        const DeviceCsr rg{ gd.n, gd.m, b.rg.row_ptr + gd.row_off, b.rg.arcs };
        unsigned long long* const cnts = p.out.counters + static_cast<int64_t>(item.graph) * kCounterCount;
        unsigned long long* const acc_sum_g = p.out.acc_sum + static_cast<int64_t>(item.graph) * 2 * kAccDigits;
        unsigned long long* const acc_inv_g = acc_sum_g + kAccDigits;
        unsigned long long* const hist_g = p.out.hist != nullptr ? p.out.hist + static_cast<int64_t>(item.graph) * p.out.hist_bins : nullptr;
        unsigned long long* const bc_g = b.bc != nullptr ? b.bc + 2 * gd.bc_off : nullptr;
        const int64_t tile_first = static_cast<int64_t>(item.tile) * kTile;
        const int64_t base = gd.src_off + tile_first;
        const int nsrc = static_cast<int>(gd.num_sources - tile_first < kTile ? gd.num_sources - tile_first : kTile);
        if (tid < kTile) {
            s_src[tid] = tid < nsrc ? p.sources[base + tid] : -1;
            s_unreach[tid] = 0ull;
            s_arcs[tid] = 0ull;
            s_max[tid] = 0ull;
        }
        __syncthreads();
        if ((!kMulti || grp().rank == 0) && warp == 0) {
            const int v = s_src[lane];
            if (v >= 0) {
                dist[static_cast<int64_t>(v) * kTile + lane] = 0ull;
                // pend0 is all zero between tiles: the first lane of a source repeated in the tile queues it
                if (atomicOr(&pend0[v], 1u << lane) == 0u) {
                    q0[atomicAdd(&ctl()->qlen[0], 1)] = v;
                }
                if (kReach) {
                    reach.add(v, 1u << lane);
                }
            }
        }
        sync0();

        // ------------------------------------------------------------ delta-stepping over the tile
        long long t_phase = clock64();
        for (;;) {
            for (;;) {
                const int cur = s.cur;
                const int qlen = s.qlen[cur];
                if (qlen == 0) {
                    break;
                }
                uint32_t* pend_cur = cur ? pend1 : pend0;
                uint32_t* pend_nxt = cur ? pend0 : pend1;
                const int32_t* q_cur = cur ? q1 : q0;
                int32_t* q_nxt = cur ? q0 : q1;
                const double theta = s.theta;
                expand_queue<kUnroll, kMode != kModeApsp, kReach>(g, q_cur, qlen, lane, &ctl()->grab, NGX_GWARPS, dist, pend_cur, pend_nxt,
                                                          far, theta, expansions, lane_expansions, reinterpret_cast<unsigned long long*>(sigma), tie,
                                                          reinterpret_cast<unsigned long long*>(delta), reach);
                sync([&](volatile TileShared& c) {
                    c.qlen[cur] = 0;
                    c.grab = 0;
                    c.iterations = c.iterations + 1;
                    if (c.iterations > p.max_iterations) {
                        atomicCAS(p.error, kDevOk, kDevTimeout);
                        c.stop = 1;
                    } else if (*p.abort_flag != 0) {
                        atomicCAS(p.error, kDevOk, kDevAborted);
                        c.stop = 1;
                    }
                });
                if (s.stop != 0) {
                    break;
                }
                // the next iteration's queue, from its pending masks (reach list: touched_len is final here)
                compact_queue<kReach>(pend_nxt, q_nxt, &ctl()->qlen[cur ^ 1], kReach ? static_cast<int64_t>(s.touched_len) : n, reach, lane,
                                      NGX_GW, NGX_GWARPS);
                sync([&](volatile TileShared& c) { c.cur = cur ^ 1; });
            }
            if (s.stop != 0) {
                break;
            }
            // bucket step, pass 1: smallest pending far distance (min_bits is +inf here: reset at the tile's start and
            // after every bucket step)
            // (over the tile's reached vertices when it keeps a reach list: no other vertex has far marks)
            const int64_t span = kReach ? static_cast<int64_t>(s.touched_len) : n;
            unsigned long long local_min = kInfBits;
            for (int64_t vb = static_cast<int64_t>(NGX_GW) * 32; vb < span; vb += static_cast<int64_t>(NGX_GWARPS) * 32) {
                const int64_t i = vb + lane;
                const int64_t v = i < span ? (kReach ? static_cast<int64_t>(__ldcg(&reach.list[i])) : i) : 0;
                const uint32_t fm = i < span ? __ldcg(&far[v]) : 0u;
                unsigned any = __ballot_sync(kFullMask, fm != 0u);
                while (any != 0u) {
                    const int l = __ffs(any) - 1;
                    any &= any - 1u;
                    const uint32_t f = __shfl_sync(kFullMask, fm, l);
                    const int64_t vl = __shfl_sync(kFullMask, v, l);
                    if ((f >> lane) & 1u) {
                        const unsigned long long d = __ldcg(&dist[vl * kTile + lane]);
                        local_min = d < local_min ? d : local_min;
                    }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const unsigned long long o = __shfl_xor_sync(kFullMask, local_min, off);
                local_min = o < local_min ? o : local_min;
            }
            if (lane == 0 && local_min != kInfBits) {
                atomicMin(&ctl()->min_bits, local_min);
            }
            sync([&](volatile TileShared& c) {
                if (c.min_bits == kInfBits) {
                    c.done = 1;  // nothing pending: the tile's distances are final
                } else {
                    c.theta_next = next_theta(__longlong_as_double(static_cast<long long>(c.min_bits)), gd.delta);
                }
            });
            if (s.done != 0) {
                break;
            }
            const double theta = s.theta_next;
            // pass 2: move the pairs below the new bound into the near queue of the next iteration
            const int cur = s.cur;
            uint32_t* pend_cur = cur ? pend1 : pend0;
            int32_t* q_cur = cur ? q1 : q0;
            for (int64_t vb = static_cast<int64_t>(NGX_GW) * 32; vb < span; vb += static_cast<int64_t>(NGX_GWARPS) * 32) {
                const int64_t i = vb + lane;
                const int64_t v = i < span ? (kReach ? static_cast<int64_t>(__ldcg(&reach.list[i])) : i) : 0;
                const uint32_t fm = i < span ? __ldcg(&far[v]) : 0u;
                unsigned any = __ballot_sync(kFullMask, fm != 0u);
                while (any != 0u) {
                    const int l = __ffs(any) - 1;
                    any &= any - 1u;
                    const uint32_t f = __shfl_sync(kFullMask, fm, l);
                    const int64_t vv = __shfl_sync(kFullMask, v, l);
                    bool near = false;
                    if ((f >> lane) & 1u) {
                        near = __longlong_as_double(static_cast<long long>(__ldcg(&dist[vv * kTile + lane]))) < theta;
                    }
                    const unsigned nmask = __ballot_sync(kFullMask, near);
                    if (nmask != 0u && lane == 0) {
                        far[vv] = f & ~nmask;
                        pend_cur[vv] = nmask;
                        q_cur[atomicAdd(&ctl()->qlen[cur], 1)] = static_cast<int32_t>(vv);
                    }
                }
            }
            sync([&](volatile TileShared& c) {
                c.theta = c.theta_next;
                c.min_bits = kInfBits;
            });
        }
        if (s.stop != 0) {
            break;
        }

        if (tid == 0) {
            const long long now = clock64();
            atomicAdd(&cnts[kCyclesSssp], static_cast<unsigned long long>(now - t_phase));
            t_phase = now;
        }
        if constexpr (kMode != kModeApsp) {
            // ------------------------------------------------------------ shortest-path DAG: counts, sigma, delta
            // the level lists are built only after the successor lists: their storage holds pred[][] until then
            uint32_t* const pred = reinterpret_cast<uint32_t*>(list);
            dag_count(g, rg, b.arc_src, b.m_total, n, nsrc, s_src, dist, tie, reinterpret_cast<unsigned long long*>(sigma), cnt, scnt, pred, lane,
                      NGX_GW, NGX_GWARPS, &ctl()->active_pairs);
            sync0();
            const unsigned long long dag_arcs = group_exclusive_scan(grp(), s, s_bar, scnt, soff, nt, s_part);
            const bool use_lists = dag_arcs <= static_cast<unsigned long long>(b.succ_capacity);
            for (int64_t i = NGX_GT; i < nt; i += NGX_GTHREADS) {
                scnt[i] = 0u;
            }
            sync0();
            if (use_lists) {
                dag_fill<kMode == kModeBrandes>(rg, b.arc_src, n, dist, cnt, pred, soff, scnt, succ, lane, NGX_GW, NGX_GWARPS);
                sync0();
                dag_sort(soff, succ, nt, NGX_GT, NGX_GTHREADS);
            }
            sync([&](volatile TileShared& c) {
                if (!use_lists) {
                    c.stamp = c.stamp + 1u;
                }
                c.level = 0u;
                c.lvl_start = 0;
                c.lvl_len = 0;
                c.next_len = 0;
                loff[0] = 0;
            });
            if (tid == 0) {
                const long long now = clock64();
                atomicAdd(&cnts[kCyclesCount], static_cast<unsigned long long>(now - t_phase));
                t_phase = now;
                if (!use_lists && (!kMulti || grp().rank == 0)) {
                    atomicAdd(&cnts[kDagScanTiles], 1ull);
                }
            }
            // the sources form level 0
            if ((!kMulti || grp().rank == 0) && warp == 0) {
                const int v = s_src[lane];
                if (v >= 0) {
                    const int64_t row = static_cast<int64_t>(v) * kTile + lane;
                    lvl[row] = 0u;
                    sigma[row] = 1.0;
                    if (use_lists) {
                        list[atomicAdd(&ctl()->lvl_len, 1)] = static_cast<int32_t>((static_cast<uint32_t>(v) << 5) | static_cast<uint32_t>(lane));
                    } else if (atomicExch(&stamp[v], s.stamp) != s.stamp) {
                        list[atomicAdd(&ctl()->lvl_len, 1)] = v;
                    }
                }
            }
            sync0();
          if (use_lists) {
            // --- sigma and delta over the successor lists. When every reached pair has exactly one DAG predecessor
            // (as many DAG arcs as reached non-source pairs) the DAGs are trees: every sigma is 1 and every child is
            // released by its only parent, so the sigma levels need neither sums nor counts.
            const bool tree = dag_arcs == s.active_pairs;
            for (;;) {
                const int start = s.lvl_start;
                const int len = s.lvl_len;
                if (len == 0) {
                    break;
                }
                const unsigned level = s.level;
                if (tree) {
                    dag_tree_level<kMode == kModeBrandes>(g, list + start, len, sigma, soff, succ, list + start + len, &ctl()->next_len, lane, NGX_GW,
                                                          NGX_GWARPS);
                } else {
                    dag_sigma_level<kMode == kModeBrandes>(g, list + start, len, level, sigma, cnt, lvl, soff, succ, list + start + len,
                                                           &ctl()->next_len, b.sigma_inexact, lane, NGX_GW, NGX_GWARPS);
                }
                sync([&](volatile TileShared& c) {
                    c.lvl_start = start + len;
                    c.lvl_len = c.next_len;
                    c.next_len = 0;
                    c.level = level + 1u;
                    loff[level + 1u] = start + len;
                });
            }
            if (tid == 0) {
                const long long now = clock64();
                atomicAdd(&cnts[kCyclesSigma], static_cast<unsigned long long>(now - t_phase));
                t_phase = now;
            }
            const int levels = static_cast<int>(s.level);
            const int lowest = kMode == kModeGrad ? 0 : 1;
            for (int level = levels - 1; level >= lowest; --level) {
                const int start = __ldcg(&loff[level]);
                const int end = __ldcg(&loff[level + 1]);
                if (tree) {
                    dag_delta_level<kMode, true>(g, list + start, end - start, dist, sigma, delta, delta_g, soff, succ, b.grad_cpl, b.grad_eff,
                                                 reinterpret_cast<double*>(s_acc_sum), lane, warp, NGX_GW, NGX_GWARPS);
                } else {
                    dag_delta_level<kMode, false>(g, list + start, end - start, dist, sigma, delta, delta_g, soff, succ, b.grad_cpl, b.grad_eff,
                                                  reinterpret_cast<double*>(s_acc_sum), lane, warp, NGX_GW, NGX_GWARPS);
                }
                sync0();
            }
            // the pair buffers borrowed the epilogue's accumulators, which must start the epilogue at zero
            for (int k = tid; k < (kBlock / 32) * 32 * delta_level_unroll(kMode) * (kMode == kModeGrad ? 2 : 1); k += blockDim.x) {
                s_acc_sum[k] = 0ull;
            }
            __syncthreads();
            if (tid == 0) {
                if ((!kMulti || grp().rank == 0)) {
                    atomicAdd(&cnts[kDagLevels], static_cast<unsigned long long>(levels));
                    atomicAdd(&cnts[kDagEntries], static_cast<unsigned long long>(__ldcg(&loff[levels])));
                }
                const long long now = clock64();
                atomicAdd(&cnts[kCyclesDelta], static_cast<unsigned long long>(now - t_phase));
                t_phase = now;
            }
          } else {
            // --- too many DAG arcs for the lists (many ties): the arc-scanning passes, one vertex per warp
            for (;;) {
                const int start = s.lvl_start;
                const int len = s.lvl_len;
                if (len == 0) {
                    break;
                }
                const unsigned level = s.level;
                const unsigned level_stamp = s.stamp + 1u;
                if (b.sigma_pull != 0) {
                    for (int i = NGX_GW; i < len; i += NGX_GWARPS) {
                        brandes_sigma_vertex<true, 2>(g, rg, __ldcg(&list[start + i]), level, nsrc, lane, dist, sigma, cnt, lvl, stamp, level_stamp,
                                                      list + start + len, &ctl()->next_len, b.sigma_inexact);
                    }
                } else {
                    for (int i = NGX_GW; i < len; i += NGX_GWARPS) {
                        brandes_sigma_vertex<false, 2>(g, rg, __ldcg(&list[start + i]), level, nsrc, lane, dist, sigma, cnt, lvl, stamp, level_stamp,
                                                       list + start + len, &ctl()->next_len, b.sigma_inexact);
                    }
                }
                sync([&](volatile TileShared& c) {
                    c.lvl_start = start + len;
                    c.lvl_len = c.next_len;
                    c.next_len = 0;
                    c.stamp = level_stamp;
                    c.level = level + 1u;
                    loff[level + 1u] = start + len;
                });
            }
            if (tid == 0) {
                const long long now = clock64();
                atomicAdd(&cnts[kCyclesSigma], static_cast<unsigned long long>(now - t_phase));
                t_phase = now;
            }
            // s.level is one past the last non-empty level; loff[s.level] is the end of the lists
            const int levels = static_cast<int>(s.level);
            const int lowest = kMode == kModeGrad ? 0 : 1;
            for (int level = levels - 1; level >= lowest; --level) {
                const int start = __ldcg(&loff[level]);
                const int end = __ldcg(&loff[level + 1]);
                for (int i = start + NGX_GW; i < end; i += NGX_GWARPS) {
                    brandes_delta_vertex<kMode, 2>(g, __ldcg(&list[i]), static_cast<unsigned>(level), nsrc, lane, dist, sigma, delta, delta_g, lvl,
                                                   b.grad_cpl, b.grad_eff);
                }
                sync0();
            }
            if (tid == 0) {
                if ((!kMulti || grp().rank == 0)) {
                    atomicAdd(&cnts[kDagLevels], static_cast<unsigned long long>(levels));
                    atomicAdd(&cnts[kDagEntries], static_cast<unsigned long long>(__ldcg(&loff[levels])));
                }
                const long long now = clock64();
                atomicAdd(&cnts[kCyclesDelta], static_cast<unsigned long long>(now - t_phase));
                t_phase = now;
            }
          }
        }

        // ------------------------------------------------------------ epilogue: fused APSP summaries, reset
        const int my_src = s_src[lane];
        const bool valid = lane < nsrc;
        unsigned long long unreach = 0, arcs = 0, mx = 0, overflow = 0;
        // APSP with a reach list visits the reached vertices only: every other vertex is unreached by every source and
        // its state was never touched; the DAG passes have written every vertex's rows, and distance rows need every
        // vertex, so those visit all of them
        const bool by_list = kReach && kMode == kModeApsp && p.out.rows == nullptr;
        const int64_t span = by_list ? static_cast<int64_t>(s.touched_len) : n;
        if (by_list && valid && (!kMulti || grp().rank == 0) && warp == 0) {
            unreach = static_cast<unsigned long long>(n - span);
        }
        for (int64_t i = NGX_GW; i < span; i += NGX_GWARPS) {
            const int64_t v = by_list ? static_cast<int64_t>(__ldcg(&reach.list[i])) : i;
            if (kReach && lane == 0) {
                reach.mask[v] = 0u;
            }
            unsigned long long* slot_ptr = &dist[v * kTile + lane];
            const unsigned long long bits = __ldcg(slot_ptr);
            *slot_ptr = kInfBits;
            if constexpr (kMode != kModeApsp) {
                const int64_t row = v * kTile + lane;
                if constexpr (kMode == kModeBrandes) {
                    // BrandesVariant.h:156: every settled vertex but the source gains its dependency
                    const double dep = (valid && v != my_src && bits != kInfBits) ? __ldcg(&delta[row]) : 0.0;
                    // summed over the tile's sources in fixed point, exactly: betweenness does not depend on how
                    // the sources are grouped into tiles
                    unsigned long long lo, hi;
                    fixed_parts(dep, lo, hi);
                    fixed_warp_sum(lo, hi);
                    if (lane == 0 && (lo | hi) != 0ull) {
                        fixed_add_parts(&bc_g[2 * v], lo, hi);
                    }
                }
                sigma[row] = __longlong_as_double(-1ll);
                delta[row] = __longlong_as_double(-1ll);
                if constexpr (kMode == kModeGrad) {
                    delta_g[row] = 0.0;
                }
                cnt[row] = 0u;
                lvl[row] = kNoLevel;
                scnt[row] = 0u;
                if (lane == 0) {
                    tie[v] = 0u;
                }
            }
            if (!valid) {
                continue;
            }
            const double d = __longlong_as_double(static_cast<long long>(bits));
            if (p.out.rows != nullptr) {
                p.out.rows[(base + lane) * n + v] = d;
            }
            if (bits == kInfBits) {
                ++unreach;
                continue;
            }
            arcs += static_cast<unsigned long long>(__ldg(&g.row_ptr[v + 1]) - __ldg(&g.row_ptr[v]));
            mx = bits > mx ? bits : mx;
            acc_add_shared(&s_acc_sum[lane * kAccDigits], d);
            if (bits != 0ull) {
                acc_add_shared(&s_acc_inv[lane * kAccDigits], __ddiv_rn(1.0, d));
            }
            if (p.out.hist_bins > 0 && v != my_src) {
                if (d >= p.out.hist_max) {
                    ++overflow;
                } else {
                    unsigned long long bin = static_cast<unsigned long long>(__ddiv_rn(d, p.out.hist_width));
                    if (bin >= static_cast<unsigned long long>(p.out.hist_bins)) {
                        bin = static_cast<unsigned long long>(p.out.hist_bins) - 1ull;
                    }
                    atomicAdd(&s_hist[bin], 1u);
                }
            }
        }
        if (valid) {
            atomicAdd(&s_unreach[lane], unreach);
            atomicAdd(&s_arcs[lane], arcs);
            atomicMax(&s_max[lane], mx);
        }
        if (overflow != 0) {
            atomicAdd(&cnts[kHistOverflow], overflow);
        }
        __syncthreads();
        if (kMulti && p.group_size > 1) {
            // the group's CTAs add their per-source sums into the group's (exact integer adds), and the first CTA
            // finishes the tile's per-source outputs from them
            unsigned long long* const g_acc = p.group_ws + slot * p.group_stride + kCtlWords + 1 + p.group_size;  // kGroupAccWords
            for (int i = tid; i < 2 * kTile * kAccDigits; i += blockDim.x) {
                if (smem[i] != 0ull) {
                    atomicAdd(&g_acc[i], smem[i]);
                }
            }
            if (tid < kTile) {
                atomicAdd(&g_acc[2 * kTile * kAccDigits + tid], s_unreach[tid]);
                atomicAdd(&g_acc[2 * kTile * kAccDigits + kTile + tid], s_arcs[tid]);
                atomicMax(&g_acc[2 * kTile * kAccDigits + 2 * kTile + tid], s_max[tid]);
            }
            sync0();
            if ((!kMulti || grp().rank == 0)) {
                for (int i = tid; i < 2 * kTile * kAccDigits; i += blockDim.x) {
                    smem[i] = __ldcg(&g_acc[i]);
                    g_acc[i] = 0ull;
                }
                if (tid < kTile) {
                    unsigned long long* const per = g_acc + 2 * kTile * kAccDigits;
                    s_unreach[tid] = __ldcg(&per[tid]);
                    s_arcs[tid] = __ldcg(&per[kTile + tid]);
                    s_max[tid] = __ldcg(&per[2 * kTile + tid]);
                    per[tid] = 0ull;
                    per[kTile + tid] = 0ull;
                    per[2 * kTile + tid] = 0ull;
                }
            }
            __syncthreads();
        }
        if ((!kMulti || grp().rank == 0)) {
            if (tid < nsrc) {
                unsigned long long* a_sum = &s_acc_sum[tid * kAccDigits];
                unsigned long long* a_inv = &s_acc_inv[tid * kAccDigits];
                acc_normalize(a_sum);
                acc_normalize(a_inv);
                const int64_t pos = base + tid;
                if (p.out.src_sum != nullptr) p.out.src_sum[pos] = acc_round_normalized(a_sum);
                if (p.out.src_inv != nullptr) p.out.src_inv[pos] = acc_round_normalized(a_inv);
                if (p.out.src_max != nullptr) p.out.src_max[pos] = __longlong_as_double(static_cast<long long>(s_max[tid]));
                if (p.out.src_unreach != nullptr) p.out.src_unreach[pos] = s_unreach[tid];
                if (p.out.src_arcs != nullptr) p.out.src_arcs[pos] = s_arcs[tid];
                const unsigned long long reached = static_cast<unsigned long long>(n) - s_unreach[tid];
                atomicAdd(&cnts[kUnreachable], s_unreach[tid]);
                atomicAdd(&cnts[kReachedPairs], reached - 1ull);
                atomicAdd(&cnts[kTraversedArcs], s_arcs[tid]);
                atomicMax(&cnts[kDiameterBits], s_max[tid]);
            }
            __syncthreads();
            for (int i = tid; i < kAccDigits; i += blockDim.x) {
                unsigned long long t_sum = 0, t_inv = 0;
                for (int k = 0; k < nsrc; ++k) {
                    t_sum += s_acc_sum[k * kAccDigits + i];
                    t_inv += s_acc_inv[k * kAccDigits + i];
                }
                if (t_sum != 0) atomicAdd(&acc_sum_g[i], t_sum);
                if (t_inv != 0) atomicAdd(&acc_inv_g[i], t_inv);
            }
            if (tid == 0) {
                atomicAdd(&cnts[kIterations], s.iterations);
            }
        }
        for (int i = tid; i < p.out.hist_bins; i += blockDim.x) {
            if (s_hist[i] != 0u) {
                atomicAdd(&hist_g[i], static_cast<unsigned long long>(s_hist[i]));
                s_hist[i] = 0u;
            }
        }
        __syncthreads();
        for (int i = tid; i < 2 * kTile * kAccDigits; i += blockDim.x) {
            smem[i] = 0ull;
        }
        __syncthreads();
        if (tid == 0) {
            atomicAdd(&cnts[kCyclesEpilogue], static_cast<unsigned long long>(clock64() - t_phase));
        }
    }
    if (lane == 0 && expansions != 0) {
        // whole-launch totals, kept in the first graph's counters
        atomicAdd(&p.out.counters[kExpansions], expansions);
        atomicAdd(&p.out.counters[kLaneExpansions], lane_expansions);
    }
#undef NGX_GT
#undef NGX_GTHREADS
#undef NGX_GW
#undef NGX_GWARPS
}

// ------------------------------------------------------------------------------------------ plain form
__device__ __forceinline__ void plain_push(bool push, int x, int lane, int32_t* q, int* qlen) {
    const unsigned mask = __ballot_sync(kFullMask, push);
    if (mask == 0u) {
        return;
    }
    int base = 0;
    if (lane == __ffs(mask) - 1) {
        base = atomicAdd(qlen, __popc(mask));
    }
    base = __shfl_sync(kFullMask, base, __ffs(mask) - 1);
    if (push) {
        q[base + __popc(mask & lanemask_lt())] = x;
    }
}

// Brandes for the one source of a plain tile (BrandesVariant.h:79-159), by one CTA with warp-per-vertex passes over
// the final distances: DAG predecessor counts from each vertex's in-arcs; Kahn levels over the out-arcs (the last
// predecessor of x to be done appends x to the next level); sigma of each new level pulled over its in-arcs (integer
// sums, exact in FP64 below 2^53); dependencies pulled over the out-arcs, level by level from the last,
// delta[u] = sum over DAG arcs u -> x of sigma[u] * ((1 + delta[x]) / sigma[x]), each lane's terms in arc order and
// the lanes combined by a fixed shuffle tree; every vertex but the source adds delta[u] to its 128-bit fixed-point
// betweenness. The arrays are per CTA: sigma, delta, cnt, list (n each) and loff (n + 2).
__device__ __forceinline__ double warp_sum_fixed_order(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        x += __shfl_xor_sync(kFullMask, x, off);
    }
    return x;
}

__device__ void plain_brandes(const DeviceCsr& g, const DeviceCsr& rg, int64_t n, int src, const unsigned long long* dist, double* sigma,
                              double* delta, uint32_t* cnt, int32_t* list, int32_t* loff, unsigned long long* bc, TileShared& s, int tid,
                              int lane, int warp, int nwarps) {
    // DAG predecessors of every reached vertex
    for (int64_t v = warp; v < n; v += nwarps) {
        const unsigned long long dv = __ldcg(&dist[v]);
        unsigned c = 0;
        if (dv != kInfBits && v != src) {
            const int64_t beg = __ldg(&rg.row_ptr[v]);
            const int64_t end = __ldg(&rg.row_ptr[v + 1]);
            for (int64_t e = beg + lane; e < end; e += 32) {
                const Arc a = ldg_arc(&rg.arcs[e]);
                c += on_dag(__ldcg(&dist[a.col]), a.len, dv) ? 1u : 0u;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            c += __shfl_xor_sync(kFullMask, c, off);
        }
        if (lane == 0) {
            cnt[v] = c;
            sigma[v] = v == src ? 1.0 : 0.0;
            delta[v] = 0.0;
        }
    }
    if (tid == 0) {
        list[0] = src;
        loff[0] = 0;
        loff[1] = 1;
        s.level = 0u;
        s.next_len = 0;
    }
    __syncthreads();
    // Kahn levels, and sigma of each new level
    for (;;) {
        const unsigned level = s.level;
        const int start = loff[level];
        const int len = loff[level + 1] - start;
        if (len == 0) {
            break;
        }
        for (int i = warp; i < len; i += nwarps) {
            const int u = list[start + i];
            const unsigned long long du = __ldcg(&dist[u]);
            const int64_t beg = __ldg(&g.row_ptr[u]);
            const int64_t end = __ldg(&g.row_ptr[u + 1]);
            for (int64_t e0 = beg; e0 < end; e0 += 32) {
                const int64_t e = e0 + lane;
                bool ready = false;
                int x = 0;
                if (e < end) {
                    const Arc a = ldg_arc(&g.arcs[e]);
                    x = a.col;
                    ready = on_dag(du, a.len, __ldcg(&dist[x])) && atomicSub(&cnt[x], 1u) == 1u;
                }
                plain_push(ready, x, lane, list + start + len, &s.next_len);
            }
        }
        __syncthreads();
        const int next = start + len;
        const int next_len = s.next_len;
        for (int i = warp; i < next_len; i += nwarps) {
            const int x = __ldcg(&list[next + i]);
            const unsigned long long dx = __ldcg(&dist[x]);
            const int64_t beg = __ldg(&rg.row_ptr[x]);
            const int64_t end = __ldg(&rg.row_ptr[x + 1]);
            double acc = 0.0;
            for (int64_t e = beg + lane; e < end; e += 32) {
                const Arc a = ldg_arc(&rg.arcs[e]);
                if (on_dag(__ldcg(&dist[a.col]), a.len, dx)) {
                    acc += __ldcg(&sigma[a.col]);
                }
            }
            acc = warp_sum_fixed_order(acc);
            if (lane == 0) {
                sigma[x] = acc;
            }
        }
        __syncthreads();
        if (tid == 0) {
            loff[level + 2] = next + next_len;
            s.level = level + 1u;
            s.next_len = 0;
        }
        __syncthreads();
    }
    // dependencies, from the last level to the source's
    for (int level = static_cast<int>(s.level) - 1; level >= 0; --level) {
        const int start = loff[level];
        const int len = loff[level + 1] - start;
        for (int i = warp; i < len; i += nwarps) {
            const int u = __ldcg(&list[start + i]);
            const unsigned long long du = __ldcg(&dist[u]);
            const double su = __ldcg(&sigma[u]);
            const int64_t beg = __ldg(&g.row_ptr[u]);
            const int64_t end = __ldg(&g.row_ptr[u + 1]);
            double acc = 0.0;
            for (int64_t e = beg + lane; e < end; e += 32) {
                const Arc a = ldg_arc(&g.arcs[e]);
                if (on_dag(du, a.len, __ldcg(&dist[a.col]))) {
                    acc += su * ((1.0 + __ldcg(&delta[a.col])) / __ldcg(&sigma[a.col]));
                }
            }
            acc = warp_sum_fixed_order(acc);
            if (lane == 0) {
                delta[u] = acc;
                if (u != src && acc != 0.0) {
                    unsigned long long lo, hi;
                    fixed_parts(acc, lo, hi);
                    fixed_add_parts(&bc[2 * static_cast<int64_t>(u)], lo, hi);
                }
            }
        }
        __syncthreads();
    }
}

template <bool kBrandes>
__global__ void __launch_bounds__(512, 2) sssp_plain_kernel(const SsspParams p, const BrandesParams b) {
    extern __shared__ __align__(16) unsigned long long smem[];
    const int nwarps_max = 16;
    unsigned long long* s_acc_sum = smem;                             // nwarps_max * kAccDigits (one per warp)
    unsigned long long* s_acc_inv = smem + nwarps_max * kAccDigits;
    unsigned int* s_hist = reinterpret_cast<unsigned int*>(smem + 2 * nwarps_max * kAccDigits);
    __shared__ TileShared s;
    __shared__ unsigned long long s_unreach, s_arcs, s_max;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    const int64_t n = p.g.n;
    const int64_t slot = blockIdx.x;
    unsigned long long expansions = 0;

    unsigned long long* dist = p.ws_dist + slot * n;
    uint32_t* pend0 = p.ws_pend + slot * 2 * n;
    uint32_t* pend1 = pend0 + n;
    uint32_t* far = p.ws_far + slot * n;
    int32_t* q0 = p.ws_queue + slot * 2 * n;
    int32_t* q1 = q0 + n;
    uint32_t* stamp = p.ws_stamp + slot * n;

    for (int64_t i = tid; i < n; i += blockDim.x) {
        dist[i] = kInfBits;
        pend0[i] = 0u;
        pend1[i] = 0u;
        far[i] = 0u;
        stamp[i] = 0u;
    }
    for (int i = tid; i < 2 * nwarps_max * kAccDigits; i += blockDim.x) {
        smem[i] = 0ull;
    }
    for (int i = tid; i < p.out.hist_bins; i += blockDim.x) {
        s_hist[i] = 0u;
    }
    if (tid == 0) {
        s.stamp = 1u;
    }
    __syncthreads();

    for (;;) {
        if (tid == 0) {
            s.tile = static_cast<long long>(atomicAdd(p.tile_counter, 1ull));
            s.stop = (*reinterpret_cast<volatile int*>(p.error) != 0) ? 1 : 0;
            s.qlen[0] = 0;
            s.qlen[1] = 0;
            s.cur = 0;
            s.theta = p.delta;
            s.iterations = 0;
            s.overflow = 0;
            s_unreach = 0;
            s_arcs = 0;
            s_max = 0;
        }
        __syncthreads();
        if (s.stop != 0 || s.tile >= p.num_tiles) {
            break;
        }
        const int64_t pos = s.tile;
        const int src = p.sources[pos];
        if (tid == 0) {
            dist[src] = 0ull;
            pend0[src] = 1u;
            stamp[src] = s.stamp;
            q0[0] = src;
            s.qlen[0] = 1;
        }
        __syncthreads();

        for (;;) {
            for (;;) {
                const int cur = s.cur;
                const int qlen = s.qlen[cur];
                if (qlen == 0) {
                    break;
                }
                uint32_t* pend_cur = cur ? pend1 : pend0;
                uint32_t* pend_nxt = cur ? pend0 : pend1;
                const int32_t* q_cur = cur ? q1 : q0;
                int32_t* q_nxt = cur ? q0 : q1;
                const unsigned next_stamp = s.stamp + 1u;
                const double theta = s.theta;
                for (int i = warp; i < qlen; i += nwarps) {
                    const int v = __ldcg(&q_cur[i]);
                    if (__ldcg(&pend_cur[v]) == 0u) {
                        continue;
                    }
                    const double dv = __longlong_as_double(static_cast<long long>(__ldcg(&dist[v])));
                    expansions += 1;
                    if (lane == 0) {
                        pend_cur[v] = 0u;
                        far[v] = 0u;  // a near value supersedes any far mark; no far mark can be set while d[v] < theta
                    }
                    const int64_t beg = __ldg(&p.g.row_ptr[v]);
                    const int64_t end = __ldg(&p.g.row_ptr[v + 1]);
                    for (int64_t e0 = beg; e0 < end; e0 += 32) {
                        const int64_t e = e0 + lane;
                        bool push = false;
                        int x = 0;
                        if (e < end) {
                            const Arc a = ldg_arc(&p.g.arcs[e]);
                            x = a.col;
                            const double nd = __dadd_rn(dv, a.len);
                            const unsigned long long nb = static_cast<unsigned long long>(__double_as_longlong(nd));
                            if (nb < __ldcg(&dist[x])) {
                                const unsigned long long old = atomicMin(&dist[x], nb);
                                if (nb < old) {
                                    if (nd < theta) {
                                        pend_nxt[x] = 1u;
                                        push = atomicExch(&stamp[x], next_stamp) != next_stamp;
                                    } else {
                                        far[x] = 1u;
                                    }
                                }
                            }
                        }
                        plain_push(push, x, lane, q_nxt, &s.qlen[cur ^ 1]);
                    }
                }
                __syncthreads();
                if (tid == 0) {
                    s.qlen[cur] = 0;
                    s.cur = cur ^ 1;
                    s.stamp = next_stamp;
                    s.iterations += 1;
                    if (s.iterations > p.max_iterations) {
                        atomicCAS(p.error, kDevOk, kDevTimeout);
                        s.stop = 1;
                    } else if (*p.abort_flag != 0) {
                        atomicCAS(p.error, kDevOk, kDevAborted);
                        s.stop = 1;
                    }
                }
                __syncthreads();
                if (s.stop != 0) {
                    break;
                }
            }
            if (s.stop != 0) {
                break;
            }
            if (tid == 0) {
                s.min_bits = kInfBits;
            }
            __syncthreads();
            unsigned long long local_min = kInfBits;
            for (int64_t v = tid; v < n; v += blockDim.x) {
                if (__ldcg(&far[v]) != 0u) {
                    const unsigned long long d = __ldcg(&dist[v]);
                    local_min = d < local_min ? d : local_min;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const unsigned long long o = __shfl_xor_sync(kFullMask, local_min, off);
                local_min = o < local_min ? o : local_min;
            }
            if (lane == 0 && local_min != kInfBits) {
                atomicMin(&s.min_bits, local_min);
            }
            __syncthreads();
            if (s.min_bits == kInfBits) {
                break;
            }
            const double theta = next_theta(__longlong_as_double(static_cast<long long>(s.min_bits)), p.delta);
            const int cur = s.cur;
            uint32_t* pend_cur = cur ? pend1 : pend0;
            int32_t* q_cur = cur ? q1 : q0;
            for (int64_t vb = 0; vb < n; vb += blockDim.x) {
                const int64_t v = vb + tid;
                bool push = false;
                if (v < n && __ldcg(&far[v]) != 0u) {
                    if (__longlong_as_double(static_cast<long long>(__ldcg(&dist[v]))) < theta) {
                        far[v] = 0u;
                        pend_cur[v] = 1u;
                        push = true;
                    }
                }
                plain_push(push, static_cast<int>(v), lane, q_cur, &s.qlen[cur]);
            }
            __syncthreads();
            if (tid == 0) {
                s.theta = theta;
            }
            __syncthreads();
        }
        if (s.stop != 0) {
            break;
        }
        if constexpr (kBrandes) {
            plain_brandes(p.g, b.rg, n, src, dist, b.ws_sigma + slot * n, b.ws_delta + slot * n, b.ws_cnt + slot * n, b.ws_list + slot * n,
                          b.ws_loff + slot * (n + 2), b.bc, s, tid, lane, warp, nwarps);
        }

        // epilogue: one accumulator pair per warp, combined exactly
        unsigned long long* a_sum = &s_acc_sum[warp * kAccDigits];
        unsigned long long* a_inv = &s_acc_inv[warp * kAccDigits];
        unsigned long long unreach = 0, arcs = 0, mx = 0, overflow = 0;
        for (int64_t v = tid; v < n; v += blockDim.x) {
            const unsigned long long bits = __ldcg(&dist[v]);
            dist[v] = kInfBits;
            const double d = __longlong_as_double(static_cast<long long>(bits));
            if (p.out.rows != nullptr) {
                p.out.rows[pos * n + v] = d;
            }
            if (bits == kInfBits) {
                ++unreach;
                continue;
            }
            arcs += static_cast<unsigned long long>(__ldg(&p.g.row_ptr[v + 1]) - __ldg(&p.g.row_ptr[v]));
            mx = bits > mx ? bits : mx;
            acc_add_shared(a_sum, d);
            if (bits != 0ull) {
                acc_add_shared(a_inv, __ddiv_rn(1.0, d));
            }
            if (p.out.hist_bins > 0 && v != src) {
                if (d >= p.out.hist_max) {
                    ++overflow;
                } else {
                    unsigned long long bin = static_cast<unsigned long long>(__ddiv_rn(d, p.out.hist_width));
                    if (bin >= static_cast<unsigned long long>(p.out.hist_bins)) {
                        bin = static_cast<unsigned long long>(p.out.hist_bins) - 1ull;
                    }
                    atomicAdd(&s_hist[bin], 1u);
                }
            }
        }
        atomicAdd(&s_unreach, unreach);
        atomicAdd(&s_arcs, arcs);
        atomicMax(&s_max, mx);
        if (overflow != 0) {
            atomicAdd(&s.overflow, overflow);
        }
        __syncthreads();
        // fold the per-warp accumulators into warp 0's, digit-wise (each digit < 2^33 * adds, far below 2^64)
        for (int i = tid; i < kAccDigits; i += blockDim.x) {
            for (int w = 1; w < nwarps; ++w) {
                s_acc_sum[i] += s_acc_sum[w * kAccDigits + i];
                s_acc_inv[i] += s_acc_inv[w * kAccDigits + i];
                s_acc_sum[w * kAccDigits + i] = 0ull;
                s_acc_inv[w * kAccDigits + i] = 0ull;
            }
        }
        __syncthreads();
        if (tid == 0) {
            acc_normalize(s_acc_sum);
            acc_normalize(s_acc_inv);
            if (p.out.src_sum != nullptr) p.out.src_sum[pos] = acc_round_normalized(s_acc_sum);
            if (p.out.src_inv != nullptr) p.out.src_inv[pos] = acc_round_normalized(s_acc_inv);
            if (p.out.src_max != nullptr) p.out.src_max[pos] = __longlong_as_double(static_cast<long long>(s_max));
            if (p.out.src_unreach != nullptr) p.out.src_unreach[pos] = s_unreach;
            if (p.out.src_arcs != nullptr) p.out.src_arcs[pos] = s_arcs;
            atomicAdd(&p.out.counters[kUnreachable], s_unreach);
            atomicAdd(&p.out.counters[kReachedPairs], static_cast<unsigned long long>(n) - s_unreach - 1ull);
            atomicAdd(&p.out.counters[kTraversedArcs], s_arcs);
            atomicMax(&p.out.counters[kDiameterBits], s_max);
            if (s.overflow != 0) atomicAdd(&p.out.counters[kHistOverflow], s.overflow);
            atomicAdd(&p.out.counters[kIterations], s.iterations);
        }
        __syncthreads();
        for (int i = tid; i < kAccDigits; i += blockDim.x) {
            if (s_acc_sum[i] != 0) atomicAdd(&p.out.acc_sum[i], s_acc_sum[i]);
            if (s_acc_inv[i] != 0) atomicAdd(&p.out.acc_inv[i], s_acc_inv[i]);
        }
        for (int i = tid; i < p.out.hist_bins; i += blockDim.x) {
            if (s_hist[i] != 0u) {
                atomicAdd(&p.out.hist[i], static_cast<unsigned long long>(s_hist[i]));
                s_hist[i] = 0u;
            }
        }
        __syncthreads();
        for (int i = tid; i < kAccDigits; i += blockDim.x) {
            s_acc_sum[i] = 0ull;
            s_acc_inv[i] = 0ull;
        }
        __syncthreads();
    }
    if (lane == 0 && expansions != 0) {
        atomicAdd(&p.out.counters[kExpansions], expansions);
        atomicAdd(&p.out.counters[kLaneExpansions], expansions);
    }
}

}  // namespace ngx
