/*
 * CPU restatement of the reference implementation's all-sources shortest-path hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: the tests, the smoke check and the CPU-baseline leg of the
 * benchmark call it to verify (and to time beside) the CUDA library. It is never part of the product path, which has
 * no CPU fallback.
 *
 * It restates, with FP64 arc lengths, the algorithms of (paths relative to the reference project):
 *   Dijkstra, binary heap with lazy deletion   source/metrics/paths/DijkstraVariants/PriorityQueueVariant.h:47-93
 *   arc length |w| or 1/|w|                     source/metrics/paths/DijkstraVariants/DijkstraCommon.h:36-54
 *   per-source summary                          source/metrics/paths/types/SsspResult.h:42-64
 *   APSP aggregation (R, CPL, efficiency)       source/metrics/paths/AllPairsShortestPath.h:110-163
 *   Brandes betweenness                         source/metrics/paths/BetweennessCentralityVariants/BrandesVariant.h:79-159
 *   distance histogram bin rule                 external/cpp-utility/data-structure/Histogram.hpp:143-180
 *   strongly connected components (Tarjan)      source/metrics/connectivity/SccVariants/TarjanGatheredVariant.h:17-36
 * and adds the exactly rounded sums and the CPL / efficiency gradient that the reference does not have.
 *
 * Parity pin: on integer-weight graphs its distances, per-source summaries, APSP scalars and Brandes values are
 * compared bit for bit with the reference's own code built from source (oracle/_ref), and with the golden values of
 * the reference's test suite.
 */
#ifndef NGX_ORACLE_H
#define NGX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Out-arc CSR. Arc e = (u -> col[e]) for row_ptr[u] <= e < row_ptr[u+1], weight w[e]. */
typedef struct {
    int64_t n;
    int64_t m;
    const int64_t* row_ptr;
    const int32_t* col;
    const double* w;
} ngxo_graph;

enum { NGXO_METRIC_REGULAR = 0, NGXO_METRIC_INVERSE = 1 };

/* Exact accumulator of non-negative doubles: 32-bit digits in 64-bit words, digit 0 weighs 2^-1088. */
#define NGXO_ACC_DIGITS 72
#define NGXO_ACC_EXP0 (-1088)
typedef struct {
    uint64_t digit[NGXO_ACC_DIGITS];
} ngxo_acc;

void ngxo_acc_clear(ngxo_acc* acc);
void ngxo_acc_add(ngxo_acc* acc, double x);
void ngxo_acc_merge(ngxo_acc* into, const ngxo_acc* from);
void ngxo_acc_normalize(ngxo_acc* acc);
double ngxo_acc_round(const ngxo_acc* acc); /* correctly rounded (to nearest, ties to even) value */
double ngxo_exact_sum(const double* x, int64_t count);

typedef struct {
    double sum_distances;        /* exactly rounded sum of all finite d(s,t), t != s */
    double sum_inverse;          /* exactly rounded sum of 1/d(s,t) over finite d != 0 */
    double sum_distances_sequential; /* sum_distances accumulated in the reference's order (per source in id order, then over sources) */
    double sum_inverse_sequential; /* sum_inverse in the reference's order */
    double diameter;             /* maximum finite distance */
    uint64_t unreachable;        /* number of (s, t) with t unreachable from s */
    uint64_t reached_pairs;      /* R = sum over sources of (reached - 1) */
    uint64_t traversed_arcs;     /* sum over sources of the out-degrees of the reached vertices */
    uint64_t hist_overflow;      /* reached pairs t != s with d >= hist_max */
    double cpl;                  /* sum_distances / R */
    double efficiency;           /* sum_inverse / R */
} ngxo_totals;

/* Single-source distances (+inf where unreachable). Returns 0 or a negative error code. */
int ngxo_sssp(const ngxo_graph* g, int64_t source, int metric, double* dist);

/*
 * APSP summaries over the given sources (sources == NULL: all n, in id order).
 * Optional per-source outputs (k entries each, NULL to skip): exactly rounded sum of distances, maximum finite
 * distance, exactly rounded and reference-order sums of 1/d, unreachable count, traversed arcs.
 * hist (bins entries, or NULL): counts of reached t != s by bin floor(d / (hist_max / bins)), clamped to the last bin;
 * d >= hist_max goes to totals->hist_overflow.
 */
int ngxo_apsp(const ngxo_graph* g, const int64_t* sources, int64_t k, int metric, int64_t bins, double hist_max, uint64_t* hist, double* src_sum,
              double* src_max, double* src_sum_inv, double* src_sum_inv_seq, uint64_t* src_unreachable, uint64_t* src_arcs, ngxo_totals* totals);

/* Brandes betweenness of the given sources (NULL: all), added onto bc (n entries), regular metric. */
int ngxo_brandes(const ngxo_graph* g, const int64_t* sources, int64_t k, double* bc);

/*
 * Gradient of CPL and of global efficiency with respect to every arc length |w_e| (regular metric), over the given
 * sources (NULL: all), normalised by R of those sources. dcpl, deff: m entries each, overwritten.
 */
int ngxo_apsp_grad(const ngxo_graph* g, const int64_t* sources, int64_t k, double* dcpl, double* deff, ngxo_totals* totals);

/*
 * Strongly connected components by Tarjan's algorithm (iterative depth-first search; weights and self arcs ignored,
 * zero-weight arcs absent). comp (n entries) receives each vertex's component, named by its largest vertex. Returns
 * the number of components, or a negative error code.
 */
int64_t ngxo_scc(const ngxo_graph* g, int32_t* comp);

#ifdef __cplusplus
}
#endif

#endif
