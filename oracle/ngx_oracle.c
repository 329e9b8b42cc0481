/*
 * CPU restatement of the reference implementation's all-sources shortest-path hot path (see ngx_oracle.h).
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never the product path.
 *
 * Compiled with -ffp-contract=off so that every relaxation is exactly fl(d[u] + len), as in the reference.
 */
#include "ngx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NGXO_OK 0
#define NGXO_EINVAL (-1)
#define NGXO_ENOMEM (-2)

/* ------------------------------------------------------------------------------------------------ exact sums */

void ngxo_acc_clear(ngxo_acc* acc) { memset(acc, 0, sizeof(*acc)); }

/*
 * Adds a finite x >= 0 exactly. x = mant * 2^e with a 53-bit integer mant; its bit 0 lands at absolute bit
 * p = e - NGXO_ACC_EXP0 >= 14. The shifted mantissa spans at most three 32-bit digits; each digit word grows by less
 * than 2^33 per call, so 2^31 calls fit between normalisations.
 */
void ngxo_acc_add(ngxo_acc* acc, double x) {
    uint64_t bits;
    memcpy(&bits, &x, sizeof(bits));
    const uint64_t biased = (bits >> 52) & 0x7FFu;
    const uint64_t fraction = bits & ((UINT64_C(1) << 52) - 1u);
    if (biased == 0 && fraction == 0) {
        return;
    }
    const uint64_t mant = biased == 0 ? fraction : (fraction | (UINT64_C(1) << 52));
    const int64_t e = biased == 0 ? -1074 : (int64_t)biased - 1075;
    const int64_t p = e - NGXO_ACC_EXP0;
    const int64_t i = p >> 5;
    const int r = (int)(p & 31);
    const uint64_t a = (mant & 0xFFFFFFFFu) << r;
    const uint64_t b = (mant >> 32) << r;
    acc->digit[i] += a & 0xFFFFFFFFu;
    acc->digit[i + 1] += (a >> 32) + (b & 0xFFFFFFFFu);
    acc->digit[i + 2] += b >> 32;
}

void ngxo_acc_merge(ngxo_acc* into, const ngxo_acc* from) {
    for (int i = 0; i < NGXO_ACC_DIGITS; ++i) {
        into->digit[i] += from->digit[i];
    }
}

void ngxo_acc_normalize(ngxo_acc* acc) {
    uint64_t carry = 0;
    for (int i = 0; i < NGXO_ACC_DIGITS; ++i) {
        const uint64_t t = acc->digit[i] + carry;
        acc->digit[i] = t & 0xFFFFFFFFu;
        carry = t >> 32;
    }
}

static int acc_bit(const uint64_t* d, int64_t k) { return (int)((d[k >> 5] >> (k & 31)) & 1u); }

static int acc_any_below(const uint64_t* d, int64_t k) {
    /* any bit with absolute index < k set? */
    const int64_t word = k >> 5;
    for (int64_t i = 0; i < word; ++i) {
        if (d[i] != 0) {
            return 1;
        }
    }
    const int r = (int)(k & 31);
    return r != 0 && (d[word] & ((UINT64_C(1) << r) - 1u)) != 0;
}

/*
 * Round to nearest, ties to even. The lowest kept bit is q = max(msb - 52, 14): bit 14 weighs 2^-1074, the
 * smallest subnormal, so results below the normal range round once, at the right position.
 */
double ngxo_acc_round(const ngxo_acc* in) {
    ngxo_acc a = *in;
    ngxo_acc_normalize(&a);
    int64_t top = -1;
    for (int i = NGXO_ACC_DIGITS - 1; i >= 0; --i) {
        if (a.digit[i] != 0) {
            int b = 31;
            while (((a.digit[i] >> b) & 1u) == 0) {
                --b;
            }
            top = (int64_t)i * 32 + b;
            break;
        }
    }
    if (top < 0) {
        return 0.0;
    }
    int64_t q = top - 52;
    if (q < 14) {
        q = 14;
    }
    uint64_t mant = 0;
    for (int64_t k = top; k >= q; --k) {
        mant = (mant << 1) | (uint64_t)acc_bit(a.digit, k);
    }
    const int half = acc_bit(a.digit, q - 1);
    const int sticky = acc_any_below(a.digit, q - 1);
    if (half && (sticky || (mant & 1u))) {
        mant += 1u;
    }
    return ldexp((double)mant, (int)(q + NGXO_ACC_EXP0));
}

double ngxo_exact_sum(const double* x, int64_t count) {
    ngxo_acc acc;
    ngxo_acc_clear(&acc);
    for (int64_t i = 0; i < count; ++i) {
        ngxo_acc_add(&acc, x[i]);
        if ((i & ((INT64_C(1) << 30) - 1)) == ((INT64_C(1) << 30) - 1)) {
            ngxo_acc_normalize(&acc);
        }
    }
    return ngxo_acc_round(&acc);
}

/* ------------------------------------------------------------------------------------------------ binary heap */

/*
 * The reference keeps its Dijkstra queue in std::priority_queue<VertexDistance, vector, GreaterVertexDistance>
 * (PriorityQueueVariant.h:49-54), ordered by distance only. Ties among equal distances are popped in the order the
 * standard binary-heap algorithm leaves them; this heap uses the same sift-up on push and the same
 * sift-the-hole-to-a-leaf-then-up on pop, so that the settle order, and with it Brandes' summation order,
 * follows the reference's exactly.
 */
typedef struct {
    double dist;
    int64_t vertex;
} heap_item;

typedef struct {
    heap_item* items;
    int64_t size;
    int64_t capacity;
} heap;

/* comp(a, b): a has lower priority than b (a is farther). */
static int heap_comp(const heap_item* a, const heap_item* b) { return a->dist > b->dist; }

static void heap_sift_up(heap_item* first, int64_t hole, int64_t top, heap_item value) {
    int64_t parent = (hole - 1) / 2;
    while (hole > top && heap_comp(&first[parent], &value)) {
        first[hole] = first[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    first[hole] = value;
}

static int heap_push(heap* h, double dist, int64_t vertex) {
    if (h->size == h->capacity) {
        const int64_t capacity = h->capacity == 0 ? 256 : 2 * h->capacity;
        heap_item* items = (heap_item*)realloc(h->items, (size_t)capacity * sizeof(heap_item));
        if (items == NULL) {
            return NGXO_ENOMEM;
        }
        h->items = items;
        h->capacity = capacity;
    }
    const heap_item value = { dist, vertex };
    h->items[h->size] = value;
    h->size += 1;
    heap_sift_up(h->items, h->size - 1, 0, value);
    return NGXO_OK;
}

static heap_item heap_pop(heap* h) {
    heap_item* first = h->items;
    const heap_item result = first[0];
    const int64_t len = h->size - 1; /* length of the heap after the pop */
    const heap_item value = first[len];
    first[len] = first[0];
    int64_t hole = 0;
    int64_t child = 0;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (heap_comp(&first[child], &first[child - 1])) {
            child -= 1;
        }
        first[hole] = first[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2 && len >= 2) {
        child = 2 * (child + 1);
        first[hole] = first[child - 1];
        hole = child - 1;
    }
    if (len > 0) {
        heap_sift_up(first, hole, 0, value);
    }
    h->size = len;
    return result;
}

/* ------------------------------------------------------------------------------------------------ graph helpers */

static int graph_valid(const ngxo_graph* g) {
    if (g == NULL || g->n < 0 || g->m < 0 || (g->n > 0 && g->row_ptr == NULL)) {
        return 0;
    }
    if (g->n > 0 && (g->row_ptr[0] != 0 || g->row_ptr[g->n] != g->m)) {
        return 0;
    }
    return 1;
}

/*
 * Arc length under the metric (DijkstraCommon.h:36-54): |w|, or 1/|w|. A zero weight is an absent arc: the reference
 * drops zero-weight arcs when it uploads the graph (DistributedGraph.cpp:174-176, :223-225), and in the inverse
 * metric a zero weight is infinitely long and never relaxed. Both are returned as +inf and skipped.
 */
static double arc_length(double w, int metric) {
    const double a = fabs(w);
    if (a == 0.0) {
        return INFINITY;
    }
    return metric == NGXO_METRIC_INVERSE ? 1.0 / a : a;
}

/* ------------------------------------------------------------------------------------------------ Dijkstra */

typedef struct {
    double* dist;
    heap queue;
    uint64_t traversed_arcs;
} sssp_work;

/* PriorityQueueVariant::compute_distances (PriorityQueueVariant.h:47-93) over the CSR; dist pre-filled here. */
static int dijkstra(const ngxo_graph* g, int64_t source, int metric, sssp_work* work) {
    double* dist = work->dist;
    for (int64_t v = 0; v < g->n; ++v) {
        dist[v] = INFINITY;
    }
    dist[source] = 0.0;
    work->queue.size = 0;
    work->traversed_arcs = 0;
    if (heap_push(&work->queue, 0.0, source) != NGXO_OK) {
        return NGXO_ENOMEM;
    }
    while (work->queue.size > 0) {
        const heap_item top = heap_pop(&work->queue);
        const int64_t u = top.vertex;
        const double du = top.dist;
        if (dist[u] < du) {
            continue; /* stale entry */
        }
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            const double len = arc_length(g->w[e], metric);
            if (isinf(len)) {
                continue;
            }
            work->traversed_arcs += 1;
            const double nd = du + len;
            const int64_t v = g->col[e];
            if (dist[v] <= nd) {
                continue;
            }
            dist[v] = nd;
            if (heap_push(&work->queue, nd, v) != NGXO_OK) {
                return NGXO_ENOMEM;
            }
        }
    }
    return NGXO_OK;
}

int ngxo_sssp(const ngxo_graph* g, int64_t source, int metric, double* dist) {
    if (!graph_valid(g) || source < 0 || source >= g->n || dist == NULL) {
        return NGXO_EINVAL;
    }
    sssp_work work = { dist, { NULL, 0, 0 }, 0 };
    const int rc = dijkstra(g, source, metric, &work);
    free(work.queue.items);
    return rc;
}

/* ------------------------------------------------------------------------------------------------ APSP */

int ngxo_apsp(const ngxo_graph* g, const int64_t* sources, int64_t k, int metric, int64_t bins, double hist_max, uint64_t* hist, double* src_sum,
              double* src_max, double* src_sum_inv, double* src_sum_inv_seq, uint64_t* src_unreachable, uint64_t* src_arcs, ngxo_totals* totals) {
    if (!graph_valid(g) || totals == NULL || (hist != NULL && (bins <= 0 || !(hist_max > 0.0)))) {
        return NGXO_EINVAL;
    }
    if (sources == NULL) {
        k = g->n;
    }
    double* dist = (double*)malloc((size_t)(g->n > 0 ? g->n : 1) * sizeof(double));
    if (dist == NULL) {
        return NGXO_ENOMEM;
    }
    sssp_work work = { dist, { NULL, 0, 0 }, 0 };
    ngxo_acc total_sum, total_inv, row_sum, row_inv;
    ngxo_acc_clear(&total_sum);
    ngxo_acc_clear(&total_inv);
    memset(totals, 0, sizeof(*totals));
    if (hist != NULL) {
        memset(hist, 0, (size_t)bins * sizeof(uint64_t));
    }
    const double width = hist != NULL ? hist_max / (double)bins : 0.0;
    double sum_inverse_sequential = 0.0;
    double sum_distances_sequential = 0.0;
    int rc = NGXO_OK;

    for (int64_t i = 0; i < k; ++i) {
        const int64_t s = sources == NULL ? i : sources[i];
        if (s < 0 || s >= g->n) {
            rc = NGXO_EINVAL;
            break;
        }
        rc = dijkstra(g, s, metric, &work);
        if (rc != NGXO_OK) {
            break;
        }
        /* summarize_distances (SsspResult.h:42-64), in global-id order */
        ngxo_acc_clear(&row_sum);
        ngxo_acc_clear(&row_inv);
        double row_inv_seq = 0.0;
        double row_sum_seq = 0.0;
        double row_max = 0.0;
        uint64_t row_unreachable = 0;
        for (int64_t t = 0; t < g->n; ++t) {
            const double d = dist[t];
            if (isinf(d)) {
                ++row_unreachable;
                continue;
            }
            ngxo_acc_add(&row_sum, d);
            row_sum_seq += d;
            if (d != 0.0) {
                const double inv = 1.0 / d;
                ngxo_acc_add(&row_inv, inv);
                row_inv_seq += inv;
            }
            if (d > row_max) {
                row_max = d;
            }
            if (hist != NULL && t != s) {
                if (d >= hist_max) {
                    totals->hist_overflow += 1;
                } else {
                    uint64_t bin = (uint64_t)(d / width);
                    if (bin >= (uint64_t)bins) {
                        bin = (uint64_t)bins - 1u;
                    }
                    hist[bin] += 1;
                }
            }
        }
        ngxo_acc_normalize(&row_sum);
        ngxo_acc_normalize(&row_inv);
        ngxo_acc_merge(&total_sum, &row_sum);
        ngxo_acc_merge(&total_inv, &row_inv);
        ngxo_acc_normalize(&total_sum);
        ngxo_acc_normalize(&total_inv);
        sum_inverse_sequential += row_inv_seq;
        sum_distances_sequential += row_sum_seq;
        if (row_max > totals->diameter) {
            totals->diameter = row_max;
        }
        totals->unreachable += row_unreachable;
        totals->reached_pairs += (uint64_t)g->n - row_unreachable - 1u;
        totals->traversed_arcs += work.traversed_arcs;
        if (src_sum != NULL) {
            src_sum[i] = ngxo_acc_round(&row_sum);
        }
        if (src_max != NULL) {
            src_max[i] = row_max;
        }
        if (src_sum_inv != NULL) {
            src_sum_inv[i] = ngxo_acc_round(&row_inv);
        }
        if (src_sum_inv_seq != NULL) {
            src_sum_inv_seq[i] = row_inv_seq;
        }
        if (src_unreachable != NULL) {
            src_unreachable[i] = row_unreachable;
        }
        if (src_arcs != NULL) {
            src_arcs[i] = work.traversed_arcs;
        }
    }
    totals->sum_distances = ngxo_acc_round(&total_sum);
    totals->sum_inverse = ngxo_acc_round(&total_inv);
    totals->sum_inverse_sequential = sum_inverse_sequential;
    totals->sum_distances_sequential = sum_distances_sequential;
    /* AllPairsShortestPath.h:154-158: both averages are over the R reached ordered pairs */
    totals->cpl = totals->sum_distances / (double)totals->reached_pairs;
    totals->efficiency = totals->sum_inverse / (double)totals->reached_pairs;
    free(work.queue.items);
    free(dist);
    return rc;
}

/* ------------------------------------------------------------------------------------------------ Brandes */

typedef struct {
    double* dist;
    double* sigma;
    double* delta;
    int64_t* settled;
    int64_t settled_count;
    int64_t* pred_head; /* per vertex: first entry of its predecessor list, -1 if none */
    int64_t* pred_next; /* arena: next entry */
    int64_t* pred_arc;  /* arena: the arc (u -> v) that made u a predecessor */
    int64_t pred_count;
    int64_t pred_capacity;
    heap queue;
} brandes_work;

static void brandes_free(brandes_work* w) {
    free(w->dist);
    free(w->sigma);
    free(w->delta);
    free(w->settled);
    free(w->pred_head);
    free(w->pred_next);
    free(w->pred_arc);
    free(w->queue.items);
}

static int brandes_alloc(brandes_work* w, const ngxo_graph* g) {
    memset(w, 0, sizeof(*w));
    const size_t n = (size_t)(g->n > 0 ? g->n : 1);
    w->dist = (double*)malloc(n * sizeof(double));
    w->sigma = (double*)malloc(n * sizeof(double));
    w->delta = (double*)malloc(n * sizeof(double));
    w->settled = (int64_t*)malloc(n * sizeof(int64_t));
    w->pred_head = (int64_t*)malloc(n * sizeof(int64_t));
    w->pred_capacity = g->m > 0 ? g->m : 1;
    w->pred_next = (int64_t*)malloc((size_t)w->pred_capacity * sizeof(int64_t));
    w->pred_arc = (int64_t*)malloc((size_t)w->pred_capacity * sizeof(int64_t));
    if (!w->dist || !w->sigma || !w->delta || !w->settled || !w->pred_head || !w->pred_next || !w->pred_arc) {
        brandes_free(w);
        return NGXO_ENOMEM;
    }
    return NGXO_OK;
}

/*
 * The forward phase of BrandesVariant::accumulate_from_source (BrandesVariant.h:98-141): Dijkstra that counts
 * shortest paths on exact distance equality and records one predecessor entry per DAG arc.
 * Each arc can become a predecessor entry at most once per source (u is expanded once), so m arena slots suffice.
 */
static int brandes_forward(const ngxo_graph* g, int64_t root, brandes_work* w) {
    for (int64_t v = 0; v < g->n; ++v) {
        w->dist[v] = INFINITY;
        w->sigma[v] = 0.0;
        w->delta[v] = 0.0;
        w->pred_head[v] = -1;
    }
    w->settled_count = 0;
    w->pred_count = 0;
    w->queue.size = 0;
    w->dist[root] = 0.0;
    w->sigma[root] = 1.0;
    if (heap_push(&w->queue, 0.0, root) != NGXO_OK) {
        return NGXO_ENOMEM;
    }
    while (w->queue.size > 0) {
        const heap_item top = heap_pop(&w->queue);
        const int64_t u = top.vertex;
        const double du = top.dist;
        if (w->dist[u] < du) {
            continue;
        }
        w->settled[w->settled_count++] = u;
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            const double len = arc_length(g->w[e], NGXO_METRIC_REGULAR);
            if (isinf(len)) {
                continue;
            }
            const double nd = du + len;
            const int64_t v = g->col[e];
            if (nd < w->dist[v]) {
                w->dist[v] = nd;
                w->sigma[v] = w->sigma[u];
                w->pred_head[v] = -1;
                if (heap_push(&w->queue, nd, v) != NGXO_OK) {
                    return NGXO_ENOMEM;
                }
            } else if (nd == w->dist[v]) {
                w->sigma[v] += w->sigma[u];
            } else {
                continue;
            }
            const int64_t slot = w->pred_count++;
            w->pred_arc[slot] = e;
            w->pred_next[slot] = w->pred_head[v];
            w->pred_head[v] = slot;
        }
    }
    return NGXO_OK;
}

int ngxo_brandes(const ngxo_graph* g, const int64_t* sources, int64_t k, double* bc) {
    if (!graph_valid(g) || bc == NULL) {
        return NGXO_EINVAL;
    }
    if (sources == NULL) {
        k = g->n;
    }
    /* source vertex of every arc, for predecessor lookups */
    int64_t* arc_source = (int64_t*)malloc((size_t)(g->m > 0 ? g->m : 1) * sizeof(int64_t));
    brandes_work w;
    if (arc_source == NULL || brandes_alloc(&w, g) != NGXO_OK) {
        free(arc_source);
        return NGXO_ENOMEM;
    }
    for (int64_t u = 0; u < g->n; ++u) {
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            arc_source[e] = u;
        }
    }
    int rc = NGXO_OK;
    for (int64_t i = 0; i < k && rc == NGXO_OK; ++i) {
        const int64_t root = sources == NULL ? i : sources[i];
        if (root < 0 || root >= g->n) {
            rc = NGXO_EINVAL;
            break;
        }
        rc = brandes_forward(g, root, &w);
        if (rc != NGXO_OK) {
            break;
        }
        /* Backward sweep (BrandesVariant.h:147-158): decreasing settle order, root (index 0) excluded. */
        for (int64_t index = w.settled_count; index > 1;) {
            --index;
            const int64_t v = w.settled[index];
            const double portion = (1.0 + w.delta[v]) / w.sigma[v];
            for (int64_t slot = w.pred_head[v]; slot >= 0; slot = w.pred_next[slot]) {
                const int64_t p = arc_source[w.pred_arc[slot]];
                w.delta[p] += w.sigma[p] * portion;
            }
            bc[v] += w.delta[v];
        }
    }
    brandes_free(&w);
    free(arc_source);
    return rc;
}

/* ------------------------------------------------------------------------------------------------ gradient */

/*
 * d(sum_t d(s,t)) / d len_e = sigma(s,u)/sigma(s,v) * (1 + delta_s(v)) for a shortest-path DAG arc e = (u -> v),
 * the Brandes edge dependency; for efficiency each target t weighs g(t) = 1/d(s,t)^2 instead of 1 and the sign flips.
 * Arcs off every DAG get zero.
 */
int ngxo_apsp_grad(const ngxo_graph* g, const int64_t* sources, int64_t k, double* dcpl, double* deff, ngxo_totals* totals) {
    if (!graph_valid(g) || dcpl == NULL || deff == NULL) {
        return NGXO_EINVAL;
    }
    if (sources == NULL) {
        k = g->n;
    }
    int64_t* arc_source = (int64_t*)malloc((size_t)(g->m > 0 ? g->m : 1) * sizeof(int64_t));
    double* delta_g = (double*)malloc((size_t)(g->n > 0 ? g->n : 1) * sizeof(double));
    brandes_work w;
    if (arc_source == NULL || delta_g == NULL || brandes_alloc(&w, g) != NGXO_OK) {
        free(arc_source);
        free(delta_g);
        return NGXO_ENOMEM;
    }
    for (int64_t u = 0; u < g->n; ++u) {
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            arc_source[e] = u;
        }
    }
    for (int64_t e = 0; e < g->m; ++e) {
        dcpl[e] = 0.0;
        deff[e] = 0.0;
    }
    ngxo_acc total_sum, total_inv;
    ngxo_acc_clear(&total_sum);
    ngxo_acc_clear(&total_inv);
    uint64_t reached_pairs = 0;
    int rc = NGXO_OK;
    for (int64_t i = 0; i < k && rc == NGXO_OK; ++i) {
        const int64_t root = sources == NULL ? i : sources[i];
        if (root < 0 || root >= g->n) {
            rc = NGXO_EINVAL;
            break;
        }
        rc = brandes_forward(g, root, &w);
        if (rc != NGXO_OK) {
            break;
        }
        for (int64_t v = 0; v < g->n; ++v) {
            delta_g[v] = 0.0;
        }
        for (int64_t index = w.settled_count; index > 1;) {
            --index;
            const int64_t v = w.settled[index];
            const double inv = 1.0 / w.dist[v];
            const double weight_count = 1.0 + w.delta[v];
            const double weight_eff = inv * inv + delta_g[v];
            for (int64_t slot = w.pred_head[v]; slot >= 0; slot = w.pred_next[slot]) {
                const int64_t e = w.pred_arc[slot];
                const int64_t u = arc_source[e];
                const double share = w.sigma[u] / w.sigma[v];
                const double c = share * weight_count;
                const double ce = share * weight_eff;
                dcpl[e] += c;
                deff[e] += ce;
                w.delta[u] += c;
                delta_g[u] += ce;
            }
        }
        for (int64_t index = 1; index < w.settled_count; ++index) {
            const double d = w.dist[w.settled[index]];
            ngxo_acc_add(&total_sum, d);
            ngxo_acc_add(&total_inv, 1.0 / d);
        }
        ngxo_acc_normalize(&total_sum);
        ngxo_acc_normalize(&total_inv);
        reached_pairs += (uint64_t)(w.settled_count - 1);
    }
    const double r = (double)reached_pairs;
    for (int64_t e = 0; e < g->m; ++e) {
        dcpl[e] = dcpl[e] / r;
        deff[e] = -deff[e] / r;
    }
    if (totals != NULL) {
        memset(totals, 0, sizeof(*totals));
        totals->reached_pairs = reached_pairs;
        totals->sum_distances = ngxo_acc_round(&total_sum);
        totals->sum_inverse = ngxo_acc_round(&total_inv);
        totals->cpl = totals->sum_distances / r;
        totals->efficiency = totals->sum_inverse / r;
    }
    brandes_free(&w);
    free(arc_source);
    free(delta_g);
    return rc;
}

/* ------------------------------------------------------------------ strongly connected components (Tarjan 1972) */
int64_t ngxo_scc(const ngxo_graph* g, int32_t* comp) {
    if (!graph_valid(g) || comp == NULL) {
        return -1;
    }
    const int64_t n = g->n;
    int64_t* index = malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* low = malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* next_arc = malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* call = malloc(sizeof(int64_t) * (size_t)(n + 1)); /* depth-first path */
    int64_t* stack = malloc(sizeof(int64_t) * (size_t)(n + 1)); /* Tarjan's vertex stack */
    uint8_t* on_stack = calloc((size_t)(n + 1), 1);
    if (!index || !low || !next_arc || !call || !stack || !on_stack) {
        free(index), free(low), free(next_arc), free(call), free(stack), free(on_stack);
        return -2;
    }
    for (int64_t v = 0; v < n; ++v) {
        index[v] = -1;
    }
    int64_t counter = 0, stack_top = 0, components = 0;
    for (int64_t root = 0; root < n; ++root) {
        if (index[root] >= 0) {
            continue;
        }
        int64_t depth = 0;
        call[depth++] = root;
        index[root] = low[root] = counter++;
        next_arc[root] = g->row_ptr[root];
        stack[stack_top++] = root;
        on_stack[root] = 1;
        while (depth > 0) {
            const int64_t v = call[depth - 1];
            if (next_arc[v] < g->row_ptr[v + 1]) {
                const int64_t e = next_arc[v]++;
                const int64_t x = g->col[e];
                if (g->w[e] == 0.0 || x == v) {
                    continue; /* absent arc; self arcs join nothing */
                }
                if (index[x] < 0) {
                    index[x] = low[x] = counter++;
                    next_arc[x] = g->row_ptr[x];
                    stack[stack_top++] = x;
                    on_stack[x] = 1;
                    call[depth++] = x;
                } else if (on_stack[x] && index[x] < low[v]) {
                    low[v] = index[x];
                }
                continue;
            }
            /* v is finished */
            --depth;
            if (low[v] == index[v]) {
                int64_t top = stack_top, largest = -1;
                do {
                    const int64_t x = stack[--top];
                    largest = x > largest ? x : largest;
                } while (stack[top] != v);
                for (int64_t i = top; i < stack_top; ++i) {
                    comp[stack[i]] = (int32_t)largest;
                    on_stack[stack[i]] = 0;
                }
                stack_top = top;
                ++components;
            }
            if (depth > 0) {
                const int64_t parent = call[depth - 1];
                if (low[v] < low[parent]) {
                    low[parent] = low[v];
                }
            }
        }
    }
    free(index), free(low), free(next_arc), free(call), free(stack), free(on_stack);
    return components;
}
