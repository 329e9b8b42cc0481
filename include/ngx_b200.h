/*
 * neurograph-b200: C ABI of the B200 (sm_100a) library for neurograph's all-sources shortest-path hot path.
 *
 * One call covers what the reference computes with one Dijkstra (or delta-stepping, or Brandes) run per source:
 * all sources run as batched multi-source delta-stepping on the GPU, each distance row is reduced on the fly into
 * the APSP summaries, and the N x N distance matrix never reaches memory.
 *
 * Conventions
 *  - Every entry point returns an ngx_status and never aborts or throws; ngx_last_error() describes the last failure
 *    of the calling thread.
 *  - The library owns all device memory it allocates and never frees caller pointers. Output arrays are
 *    caller-allocated HOST arrays of the documented length.
 *  - Handles are opaque. One graph handle owns one CUDA stream and is not thread-safe; separate handles may be used
 *    from separate threads.
 *  - Vertex ids are 0-based and global (the reference's prefix_distribution[rank] + local id, one rank).
 *  - Arc lengths: |w| (regular metric) or 1/|w| (inverse metric), as DijkstraCommon::transform_weight
 *    (source/metrics/paths/DijkstraVariants/DijkstraCommon.h:36-54). A zero weight is an absent arc, as the
 *    reference drops zero-weight arcs when it builds its graph (source/graph/DistributedGraph.cpp:174-176).
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *  - ngx_graph_create        DistributedGraph::construct_graph + the per-rank RMA arc windows
 *                            (source/graph/DistributedGraph.cpp:46-127, DistributedGraph.h:218-311)
 *  - ngx_apsp                AllPairsShortestPath::compute_apsp / compute_apsp_inverse / compute_apsp_delta_stepping
 *                            (source/metrics/paths/AllPairsShortestPath.h:54-98), with the per-source loop over
 *                            Dijkstra::compute_sssp (Dijkstra.h:55-98) or DeltaStepping::compute_shortest_distances
 *                            (DeltaStepping.h:36-82) and summarize_distances (types/SsspResult.h:42-64) fused in
 *  - ngx_sssp_rows           Dijkstra::compute_sssp's distance buffer (Dijkstra.h:55-98), for chosen sources
 *  - ngx_brandes             BetweennessCentrality::compute_average_betweenness_centrality with BrandesVariant
 *                            (BetweennessCentrality.h:46-80, BetweennessCentralityVariants/BrandesVariant.h:50-159)
 *  - ngx_apsp_grad           no reference counterpart: gradient of CPL and efficiency w.r.t. every arc length
 *  - ngx_*_fixed, ngx_fixed_to_double  the per-rank betweenness vectors and their reduce_componentwise_sum
 *                            (BetweennessCentrality.h:74), made exact across ranks
 *  - ngx_exact_*             the sequential double sums of AllPairsShortestPath.h:146-158, made exact across ranks
 *  - ngx_batch_*             the per-graph loop of source/neurograph.cpp:139-416, for many graphs in one launch
 *  - ngx_network_*           DistributedGraph::construct_graph's loading (DistributedGraph.cpp:68-127,
 *                            FileLoader.cpp:96-327, ArcTransformer.cpp:21-69), one process reading every rank's files
 *  - ngx_diameter_*          DiameterApproximation::compute_approximation (metrics/paths/DiameterApproximation.h:54-126)
 *  - ngx_scc                 StronglyConnectedComponents::compute_strongly_connected_components
 *                            (metrics/connectivity/StronglyConnectedComponents.h:17-36)
 *  - ngx_apsp_noalloc, ngx_graph_source_order, ngx_graph_update_weights: no counterpart (see their comments)
 */
#ifndef NGX_B200_H
#define NGX_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define NGX_API __attribute__((visibility("default")))
#else
#define NGX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NGX_OK = 0,
    NGX_INVALID_ARGUMENT = 1,
    NGX_OUT_OF_MEMORY = 2,
    NGX_CUDA_ERROR = 3,
    NGX_TIMEOUT = 4,  /* a kernel hit its iteration cap (opts.max_iterations) and stopped */
    NGX_ABORTED = 5,  /* ngx_graph_request_abort() was called while a run was in flight */
    NGX_UNSUPPORTED = 6
} ngx_status;

typedef enum { NGX_METRIC_REGULAR = 0, NGX_METRIC_INVERSE = 1 } ngx_metric;

/* How sources are mapped onto the GPU. */
typedef enum {
    NGX_MODE_BATCHED = 0, /* a tile of NGX_TILE sources per CTA; lanes of a warp are sources, arcs are shared */
    NGX_MODE_PLAIN = 1    /* one source per CTA; lanes of a warp stride over one vertex's arcs */
} ngx_mode;

#define NGX_TILE 32

/* Host CSR of out-arcs: arc e = (u -> col[e], w[e]) for row_ptr[u] <= e < row_ptr[u + 1]. */
typedef struct {
    int64_t n;
    int64_t m;
    const int64_t* row_ptr; /* n + 1 entries, row_ptr[0] == 0, non-decreasing, row_ptr[n] == m */
    const int32_t* col;     /* m entries in [0, n) */
    const double* w;        /* m entries, finite */
} ngx_csr;

typedef struct ngx_graph ngx_graph;

typedef struct {
    int metric;              /* ngx_metric */
    int mode;                /* ngx_mode */
    const int64_t* sources;  /* host list of source vertices, or NULL for all n in id order */
    int64_t num_sources;     /* entries in sources (ignored when sources is NULL) */
    double delta;            /* bucket width of the delta-stepping; <= 0: the tuned width, else 2 / sqrt(mean out-degree)
                                x the mean arc length (the factor clamped to 0.125-2) */
    int block_threads;       /* threads per CTA; 0 picks the default */
    int ctas_per_sm;         /* concurrent CTAs per SM; 0 picks the default (bounded by the memory budget) */
    int64_t hist_bins;       /* bins of the shortest-path distance histogram; 0 = no histogram */
    double hist_max;         /* exclusive upper bound of the histogram; <= 0 = sampled eccentricity x 1.5 */
    uint64_t max_iterations; /* cap on delta-stepping phases per source tile; 0 = 4 * n + 64 */
    int tile_ctas;           /* CTAs that work on one source tile together (batched form; 1 to 512); 0 picks 1, or more
                                when the device memory affords fewer workspace slots than there are resident CTAs */
} ngx_apsp_opts;

/* Totals over all requested sources; per-source arrays are optional caller-allocated host arrays (NULL to skip). */
typedef struct {
    double sum_distances;     /* exactly rounded sum of finite d(s,t), t != s */
    double sum_inverse;       /* exactly rounded sum of 1/d(s,t), finite d != 0 */
    double diameter;          /* maximum finite distance */
    uint64_t unreachable;     /* pairs (s,t) with t unreachable from s */
    uint64_t reached_pairs;   /* R = sum over sources of (reached vertices - 1) */
    uint64_t traversed_arcs;  /* sum over sources of the out-degrees of the reached vertices (GTEPS numerator) */
    uint64_t hist_overflow;   /* reached pairs with d >= hist_max */
    double hist_max;          /* the histogram bound actually used */
    double cpl;               /* characteristic path length sum_distances / R (AllPairsShortestPath.h:154-157) */
    double efficiency;        /* global efficiency sum_inverse / R (AllPairsShortestPath.h:158) */
    double kernel_ms;         /* device time of the run's kernels (CUDA events) */
    uint64_t phases;          /* delta-stepping phases (near iterations) summed over source tiles */
    uint64_t expansions;      /* vertex expansions: one pass over a vertex's out-arcs */
    uint64_t lane_expansions; /* (vertex, source) expansions; lane_expansions / expansions = sources per arc pass */
    uint64_t dag_levels;      /* Kahn levels of the shortest-path DAGs summed over source tiles (Brandes / adjoint) */
    uint64_t dag_entries;     /* entries of those levels ((vertex, source) pairs, or vertices on the arc-scanning path) */
    uint64_t dag_scan_tiles;  /* tiles whose DAG did not fit the successor lists and used the arc-scanning passes */
    uint64_t phase_cycles[5]; /* SM cycles summed over CTAs: distances, DAG counts, sigma, delta, summaries */
    /* optional outputs */
    uint64_t* hist;           /* hist_bins entries */
    double* src_sum;          /* per source: exactly rounded sum of distances */
    double* src_max;          /* per source: maximum finite distance (eccentricity) */
    double* src_sum_inverse;  /* per source: exactly rounded sum of 1/d */
    uint64_t* src_unreachable;/* per source: unreachable vertices */
    uint64_t* src_arcs;       /* per source: traversed arcs */
    uint64_t* acc_digits;     /* 2 x NGX_ACC_DIGITS: the exact sums of d and of 1/d before rounding (normalized digits,
                                 for merging the runs of several ranks exactly; see ngx_exact_round) */
} ngx_apsp_result;

/*
 * Exact sums. An accumulator is NGX_ACC_DIGITS unsigned 64-bit words, digit i holding a multiple of
 * 2^(32 i + NGX_ACC_EXP0); any non-negative finite double is a sum of at most three such digits. Digit-wise integer
 * addition is associative, so accumulators of different ranks (or runs) can be summed word by word, in any order
 * (e.g. an all-reduce with SUM), as long as each word stays below 2^64: normalized digits are below 2^32, so up to
 * 2^32 accumulators can be summed before ngx_exact_round. Replaces the sequential double sums of
 * AllPairsShortestPath.h:146-158 when results of several ranks are combined.
 */
#define NGX_ACC_DIGITS 72
#define NGX_ACC_EXP0 (-1088)

/* Adds values[0..count) (non-negative finite doubles, else NGX_INVALID_ARGUMENT) into the accumulator `digits` and
 * normalizes it. Host-only: needs no GPU. */
NGX_API int ngx_exact_accumulate(const double* values, int64_t count, uint64_t* digits);

/* Normalizes the accumulator `digits` in place (carries) and returns its value rounded once to nearest-even. */
NGX_API double ngx_exact_round(uint64_t* digits);

NGX_API const char* ngx_status_string(int status);
NGX_API const char* ngx_last_error(void);
/* Library build identifier (compute capability the kernels were built for, CUDA version). */
NGX_API const char* ngx_version(void);

/* Validates and uploads the graph to `device`, building the device CSR and reverse CSR on the GPU: the caller's arcs
 * are checked, zero weights dropped and both arc lengths written by device kernels, and the reverse CSR comes from a
 * stable device sort of the stored arcs by target (replaces DistributedGraph::construct_graph's window construction,
 * source/graph/DistributedGraph.cpp:154-250). */
NGX_API int ngx_graph_create(const ngx_csr* csr, int device, ngx_graph** out);

#define NGX_BUILD_ON_HOST 1 /* ngx_graph_create_ex: build the arrays on host threads and upload them */
/* ngx_graph_create with flags (0 or NGX_BUILD_ON_HOST); both builds give bit-identical device arrays. */
NGX_API int ngx_graph_create_ex(const ngx_csr* csr, int device, int flags, ngx_graph** out);

/* One stored arc as the device holds it (16 bytes): forward CSR {target, caller arc index, length}; reverse CSR
 * {source, stored forward index, |w|}. */
typedef struct {
    int32_t col;
    int32_t id;
    double len;
} ngx_arc;

/* Copies a handle's device arrays to host arrays (any pointer may be NULL): row_ptr and rrow_ptr n + 1 entries per
 * graph (global stored-arc offsets), arcs (|w| lengths), arcs_inverse (1/|w|), rarcs and arc_src (source vertex of
 * each stored arc) m_stored entries, mean_lengths[2] = the mean |w| and 1/|w| that default bucket widths derive from.
 * m_stored = row_ptr[n] of the last graph. No reference counterpart (inspection of DistributedGraph's windows). */
NGX_API int ngx_graph_layout(const ngx_graph* graph, int64_t* row_ptr, ngx_arc* arcs, ngx_arc* arcs_inverse, int64_t* rrow_ptr,
                             ngx_arc* rarcs, int32_t* arc_src, double* mean_lengths);
NGX_API void ngx_graph_destroy(ngx_graph* graph);
NGX_API int ngx_graph_size(const ngx_graph* graph, int64_t* n, int64_t* m);
/* Asks an in-flight run on this graph to stop at its next phase boundary; the run returns NGX_ABORTED. */
NGX_API int ngx_graph_request_abort(ngx_graph* graph);
/*
 * Runs the graph's work on `stream` (a cudaStream_t of the graph's device, owned by the caller, who keeps it alive
 * while the graph uses it); NULL restores the graph's own stream. Lets a caller time or order the library's kernels
 * with its own events.
 */
NGX_API int ngx_graph_set_stream(ngx_graph* graph, void* stream);
/* Caps the device memory the graph's runs may use for workspaces (bytes; 0 = no cap beyond free memory). */
NGX_API int ngx_graph_set_memory_budget(ngx_graph* graph, uint64_t bytes);

/*
 * The order in which all-sources runs (opts.sources == NULL, and batch runs) take the sources: clusters of nearby
 * vertices, 32 to a tile (each seed with its lightest unassigned out-neighbours), so that a tile's sources share arc
 * passes. order: n entries (for a batch, each graph's local ids, graph after graph). Per-source outputs are always
 * indexed by vertex. Callers that split an all-sources job into batches get the same tiles by taking contiguous
 * chunks of this order. No reference counterpart (the reference loops over its local vertices in id order,
 * AllPairsShortestPath.h:130-143).
 */
NGX_API int ngx_graph_source_order(const ngx_graph* graph, int64_t* order);

/*
 * Autotuning of a single-graph handle. ngx_graph_autotune times the task (NGX_TASK_APSP, _BRANDES or _GRAD, below) on
 * the first `sample_sources` sources of the graph's all-sources order (0 = one wave: 32 x resident CTAs) for bucket
 * widths (multiples of the mean arc length), block shapes and CTAs per source tile, one parameter at a time, and keeps
 * the fastest (traversed arcs per second) in the handle: later runs of that task use it for every option they leave
 * at 0 (delta, block_threads with ctas_per_sm, tile_ctas). Results never depend on these choices. best (optional)
 * receives the choice. No reference counterpart (the reference has no launch parameters; its delta-stepping takes
 * delta from --apsp-delta, neurograph.cpp:507-515).
 */
typedef enum { NGX_TASK_APSP = 0, NGX_TASK_BRANDES = 1, NGX_TASK_GRAD = 2 } ngx_task;

typedef struct {
    double delta_scale; /* bucket width = delta_scale x the mean arc length */
    int block_threads;  /* threads per CTA */
    int ctas_per_sm;    /* resident CTAs per SM */
    int tile_ctas;      /* CTAs per source tile */
    int trials;         /* configurations timed */
    double gteps;       /* traversed arcs per second of the choice on the sample, in 1e9 */
} ngx_tuning;

NGX_API int ngx_graph_autotune(ngx_graph* graph, int task, int64_t sample_sources, ngx_tuning* best);

/* APSP summaries (and optional histogram / per-source outputs) over the requested sources. */
NGX_API int ngx_apsp(ngx_graph* graph, const ngx_apsp_opts* opts, ngx_apsp_result* result);

/* Full distance rows of the requested sources: rows has num_sources * n entries, +inf where unreachable. */
NGX_API int ngx_sssp_rows(ngx_graph* graph, const ngx_apsp_opts* opts, double* rows);

/*
 * Brandes betweenness (regular metric) of the requested sources: bc (n entries) is overwritten with the sum over
 * sources of the pair dependencies; result (optional) receives the APSP summaries of the same run.
 * opts->mode NGX_MODE_PLAIN runs one source per CTA (the per-source form, for comparison); its dependency sums run
 * in another order than the batched form's, so the two agree to rounding, not bit for bit. The gradient entry
 * points below have the batched form only.
 */
NGX_API int ngx_brandes(ngx_graph* graph, const ngx_apsp_opts* opts, double* bc, ngx_apsp_result* result);

/*
 * Gradient of CPL and of global efficiency (regular metric, over the requested sources) with respect to every arc
 * length |w_e|: dcpl, deff have m entries each; arcs on no shortest path get 0. result (optional) receives the APSP
 * summaries of the same run.
 */
NGX_API int ngx_apsp_grad(ngx_graph* graph, const ngx_apsp_opts* opts, double* dcpl, double* deff, ngx_apsp_result* result);

/*
 * The same runs with the sums left unconverted, for combining the runs of several ranks exactly (the reference reduces
 * its per-rank betweenness vectors, BetweennessCentrality.h:74, reduce_componentwise_sum). Each value is a 128-bit
 * unsigned fixed-point number value * 2^64 in two words (low, high): bc_fixed holds 2 n words, the sum over the
 * requested sources of the pair dependencies; dcpl_fixed and deff_fixed hold 2 m words each, the gradient sums before
 * the division by R (the reached pairs in result) and, for deff, before the sign. The sums of disjoint source sets add
 * as 128-bit integers (modulo 2^128) to the sum of their union, and ngx_fixed_to_double turns a sum into the doubles
 * ngx_brandes / ngx_apsp_grad return: bc = to_double(bc_fixed, 1, +1), dcpl = to_double(dcpl_fixed, R, +1),
 * deff = to_double(deff_fixed, R, -1), with R summed over the same source sets.
 */
NGX_API int ngx_brandes_fixed(ngx_graph* graph, const ngx_apsp_opts* opts, uint64_t* bc_fixed, ngx_apsp_result* result);
NGX_API int ngx_apsp_grad_fixed(ngx_graph* graph, const ngx_apsp_opts* opts, uint64_t* dcpl_fixed, uint64_t* deff_fixed,
                                ngx_apsp_result* result);
/* out[i] = sign * value(words[2i], words[2i+1]) / divisor, as the library converts its own sums. Host-only. */
NGX_API int ngx_fixed_to_double(const uint64_t* words, int64_t count, double divisor, double sign, double* out);

/* ------------------------------------------------------------------------------------------------------------------
 * APSP without device allocation. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they run: a process whose caching allocator already holds
 * nearly all of the GPU (a cudaMalloc there fails or empties the cache), or a loop with a latency bound (cudaFree
 * synchronizes the device). Same inputs and results as ngx_apsp in the batched form, but every device buffer comes
 * from one fixed array of NGX_NOALLOC_SCRATCH_BYTES per device inside the library: no device memory is allocated, and
 * host memory only to build an error message. Differences from ngx_apsp: result must not be NULL; limits, rejected with
 * NGX_INVALID_ARGUMENT: n <= NGX_NOALLOC_MAX_VERTICES, num_sources <= NGX_NOALLOC_MAX_SOURCES, hist_max > 0 whenever
 * hist_bins > 0 (no automatic bound); the plain form is rejected with NGX_UNSUPPORTED; kernel_ms is not measured (0).
 * Every call looks up the array's address (cudaGetSymbolAddress, which may load the library's device code on the
 * first call) and synchronizes the graph's stream, so the call can never be made while that stream is being captured.
 * Calls that overlap on the same device share the array and race: serialize them.
 */
#define NGX_NOALLOC_SCRATCH_BYTES (32u << 20)
#define NGX_NOALLOC_MAX_VERTICES 32768
#define NGX_NOALLOC_MAX_SOURCES 32768

NGX_API int ngx_apsp_noalloc(ngx_graph* graph, const ngx_apsp_opts* opts, ngx_apsp_result* result);

/* ------------------------------------------------------------------------------------------------------------------
 * Batches: many independent graphs of uneven sizes in one handle and one persistent launch, fed by a device queue of
 * (graph, source tile) work items in longest-first order. No reference counterpart: the reference processes one
 * graph per run (neurograph.cpp:139-416); the batch runs that loop's APSP / betweenness for every graph at once.
 */

#define NGX_SIZE_CLASSES 32 /* graphs are grouped by floor(log2(n)) for the tuned bucket widths */

typedef struct {
    int task;               /* ngx_task: APSP summaries; + Brandes betweenness; + CPL / efficiency gradient */
    int metric;             /* ngx_metric (APSP only; betweenness and the gradient use |w|) */
    double delta_scale;     /* bucket width = delta_scale x the graph's mean arc length; <= 0: its size class's tuned
                               scale, or before ngx_batch_autotune has run 2 / sqrt(the graph's mean out-degree),
                               clamped to 0.125-2 */
    int block_threads;      /* 0 = default */
    int64_t hist_bins;      /* distance histogram bins per graph; 0 = none */
    double hist_max;        /* histogram bound, the same for all graphs; must be > 0 when hist_bins > 0 */
    int use_cuda_graph;     /* capture the run (output reset + launch) and replay it while these options are unchanged */
    uint64_t max_iterations;/* cap on phases per source tile; 0 = 4 * n + 64 of the largest graph */
    int tile_ctas;          /* CTAs per source tile, as in ngx_apsp_opts */
} ngx_batch_opts;

/* Validates and uploads `count` CSRs into one handle. Vertex and arc numbering stays per graph in every output. */
NGX_API int ngx_batch_create(const ngx_csr* graphs, int64_t count, int device, ngx_graph** out);

/*
 * All-sources run of every graph of a batch handle. results: `count` entries (per-graph summaries; their optional
 * per-source / histogram pointers are honoured). bc: sum of n entries (graph after graph) or NULL, for NGX_TASK_BRANDES.
 * dcpl, deff: sum of m entries (graph after graph) or NULL, for NGX_TASK_GRAD.
 */
NGX_API int ngx_batch_run(ngx_graph* batch, const ngx_batch_opts* opts, ngx_apsp_result* results, double* bc, double* dcpl, double* deff);

/*
 * Picks the bucket width scale of every size class present in the batch: for each class, the median-size graph's first
 * wave of source tiles runs with scales 1/8 .. 4 and the fastest (traversed arcs per second) is kept in the handle.
 * Then, since one launch runs every graph, one launch shape for the whole batch: block shapes (512 x 2, 384 x 2,
 * 256 x 3, 256 x 4 threads x CTAs per SM) and then 1, 2 or 4 CTAs per source tile, timed on the size class holding
 * most of the batch's work; ngx_batch_run uses it when its options leave block_threads and tile_ctas at 0, and
 * ngx_graph_tuning reads it. class_scales (optional, NGX_SIZE_CLASSES entries) receives the scales (0 for classes
 * without graphs).
 */
NGX_API int ngx_batch_autotune(ngx_graph* batch, int task, double* class_scales);

/* The launch shape and bucket width a handle keeps for `task` (from ngx_graph_autotune or ngx_batch_autotune; all
 * zero if the task was not tuned). */
NGX_API int ngx_graph_tuning(const ngx_graph* graph, int task, ngx_tuning* out);

/*
 * Replaces the weights of a graph or batch handle in place (same arcs, caller order, sum of m entries). A weight may
 * not change between zero and non-zero (that changes the arc set; create a new handle instead).
 */
NGX_API int ngx_graph_update_weights(ngx_graph* graph, const double* w);

/* ------------------------------------------------------------------------------------------------------------------
 * Loading neurograph's network files (host only; no GPU needed until ngx_graph_create_from_network). Replaces
 * DistributedGraph::construct_graph's loading for one process that reads every rank's files
 * (source/graph/DistributedGraph.cpp:68-127 over FileLoader.cpp:96-327 and ArcTransformer.cpp:21-69): vertices per rank
 * from <dir>/positions/rank_<r>_positions.txt, out arcs from <dir>/network/rank_<r><prefix>_out_network.txt (and in
 * arcs from ..._in_network.txt when undirected), the same line rules, repeated arcs summed as int32, the same
 * transforms in the same order, zero weights dropped. Vertex v of rank r gets the global id prefix[r] + v. Each row of
 * the CSR is sorted by target. Files are parsed on `threads` host threads (0 = all).
 */
typedef struct ngx_network ngx_network;

#define NGX_LOAD_REMOVE_SELF_ARCS 1 /* ArcTransformer::remove_self_arcs */
#define NGX_LOAD_UNDIRECTED 2       /* ArcTransformer::synchronize_arcs: out arcs plus reversed in arcs */
#define NGX_LOAD_ONE_WEIGHT 4       /* ArcTransformer::all_weights_one */

NGX_API int ngx_network_load(const char* directory, int32_t number_ranks, const char* file_prefix, int flags, int threads, ngx_network** out);
NGX_API int ngx_network_size(const ngx_network* network, int64_t* n, int64_t* m);
/* row_ptr: n + 1 entries; col, w: m entries (weights as doubles of the summed int32 values). */
NGX_API int ngx_network_csr(const ngx_network* network, int64_t* row_ptr, int32_t* col, double* w);
NGX_API int ngx_graph_create_from_network(const ngx_network* network, int device, ngx_graph** out);
NGX_API void ngx_network_destroy(ngx_network* network);

/* ------------------------------------------------------------------------------------------------------------------
 * Diameter approximation. Replaces DiameterApproximation::compute_approximation
 * (source/metrics/paths/DiameterApproximation.h:54-126; mark_as_centers :154-179, perform_growing_step :204-284,
 * contract :297-): balls of radius r grown around random centres, the graph contracted to its balls (arc weight
 * w + d(u) + d(v), the last arc of a centre pair in CSR order winning), and the exact diameter of the contracted
 * graph, plus 2r. Centres
 * are drawn from std::mt19937 seeded with `seed` through std::uniform_real_distribution<double>(0, 1) (the reference's
 * DefaultRandomNumberGenerator, seeded there with the MPI rank: 0 for one rank), or, when draws != NULL, from
 * draws[0], draws[1], ... (the last one repeating). Weights must be positive integers below 2^31 (zeros are absent
 * arcs), as the reference's 32-bit weights and unsigned distances require; the CSR's arc order is the reference's
 * stored order when the results must agree exactly. ngx_diameter_contract (host only) returns the contracted graph;
 * ngx_diameter_approximation runs its APSP on `device` with the batched kernel.
 */
NGX_API int ngx_diameter_contract(const ngx_csr* csr, uint64_t r, const double* draws, int64_t num_draws, uint32_t seed, ngx_network** contracted);
NGX_API int ngx_diameter_approximation(const ngx_csr* csr, uint64_t r, const double* draws, int64_t num_draws, uint32_t seed, int device,
                                       uint64_t* diameter);

/* Strongly connected components of a single-graph handle, on its device.
 * Replaces StronglyConnectedComponents::compute_strongly_connected_components (source/metrics/connectivity/
 * StronglyConnectedComponents.h:17-36) and its SccResult (number_components, largest_component_size,
 * component_sizes: size -> number of components), which all of the reference's algorithms (Tarjan gathered, forward
 * backward, coloring, multistep) return identically. Weights and self arcs are ignored; a vertex without arcs is a
 * component of its own. component (host int32[n] or NULL) receives each vertex's component, named by its largest
 * vertex; size_histogram (host uint64[n + 1] or NULL) receives the number of components of each size. */
NGX_API int ngx_scc(ngx_graph* graph, int32_t* component, uint64_t* number_components, uint64_t* largest_component, uint64_t* size_histogram);

#ifdef __cplusplus
}
#endif

#endif
