/*
 * C interface over the reference implementation's own shortest-path hot path, compiled from its unmodified
 * sources against the single-rank shims in ref_shim/ (see Makefile). Test infrastructure only: the tests use it
 * to pin the project's CPU restatement (ngx_oracle.c) bit for bit on integer-weight graphs, and to export the
 * reference's one-rank test fixture graphs as CSR. It is never linked into the product library.
 *
 * Entry points it wraps (paths relative to the reference project):
 *   AllPairsShortestPath::compute_apsp / compute_apsp_inverse      source/metrics/paths/AllPairsShortestPath.h:54-79
 *   AllPairsShortestPath::compute_apsp_delta_stepping              source/metrics/paths/AllPairsShortestPath.h:95-98
 *   Dijkstra::compute_sssp                                          source/metrics/paths/Dijkstra.h:55-98
 *   DeltaStepping::compute_shortest_distances                       source/metrics/paths/DeltaStepping.h:36-82
 *   BrandesVariant::accumulate_betweenness                          source/metrics/paths/BetweennessCentralityVariants/BrandesVariant.h:50-74
 *   BetweennessCentrality::compute_average_betweenness_centrality   source/metrics/paths/BetweennessCentrality.h:46-80
 *   DistributedGraph::construct_graph (in memory and from files)   source/graph/DistributedGraph.cpp:46-127
 */

#include "GraphTest.h"
#include "Types.h"

#include "graph/DistributedGraph.h"
#include "graph/GraphTypes.h"
#include "metrics/paths/AllPairsShortestPath.h"
#include "metrics/paths/BetweennessCentrality.h"
#include "metrics/paths/DeltaStepping.h"
#include "metrics/paths/Dijkstra.h"
#include "metrics/paths/BetweennessCentralityVariants/BrandesVariant.h"
#include "metrics/paths/DiameterApproximation.h"
#include "metrics/connectivity/StronglyConnectedComponents.h"
#include "utility/RandomNumberGenerator.h"

#include <mpi-wrapper/MPIWrapper.h>
#include <mpi-wrapper/instrumentation/MPIProgress.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <string>
#include <vector>

namespace {

void ensure_initialised() {
    static const bool initialised = [] {
        int argc = 0;
        char** argv = nullptr;
        mpiPP::MPIWrapper::init(argc, argv);
        mpiPP::MPIProgress::set_disable_status(true);
        return true;
    }();
    static_cast<void>(initialised);
}

thread_local std::string last_error{};

template <typename F>
int guarded(F&& body) {
    try {
        ensure_initialised();
        body();
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return 1;
    }
}

/* Gives access to the reference's protected one-rank fixture builders (tests/GraphTest.h). */
class FixtureAccess : public GraphTest {
public:
    void TestBody() override { }

    static std::vector<std::pair<const char*, std::function<DistributedGraph()>>> all() {
        return {
            { "standard", [] { return get_standard_one_rank_graph(); } },
            { "empty", [] { return get_empty_one_rank_graph(); } },
            { "standard_uu", [] { return get_standard_uu_one_rank_graph(); } },
            { "full", [] { return get_full_one_rank_graph(); } },
            { "negative_weight", [] { return get_negative_weight_one_rank_graph(); } },
            { "standard_four_rank_on_one_rank", [] { return get_standard_four_rank_graph_on_one_rank(); } },
            { "standard_uu_four_rank_on_one_rank", [] { return get_standard_uu_four_rank_graph_on_one_rank(); } },
            { "full_four_rank_on_one_rank", [] { return get_full_four_rank_graph_on_one_rank(); } },
            { "standard_seven_rank_on_one_rank", [] { return get_standard_seven_rank_graph_on_one_rank(); } },
            { "standard_uu_seven_rank_on_one_rank", [] { return get_standard_uu_seven_rank_graph_on_one_rank(); } },
            { "full_seven_rank_on_one_rank", [] { return get_full_seven_rank_graph_on_one_rank(); } },
            { "multi_component_four_rank_on_one_rank", [] { return get_multi_component_four_rank_graph_on_one_rank(); } },
        };
    }
};

struct RefGraph {
    DistributedGraph graph;
};

DistributedGraph build_from_csr(std::int64_t n, const std::int64_t* row_ptr, const std::int32_t* col, const std::int32_t* w) {
    auto nodes = LoadedNodes{};
    nodes.positions.assign(static_cast<std::size_t>(n), Vec3d{ 0.0, 0.0, 0.0 });
    nodes.area_names = { "area" };
    nodes.signal_types = { "ex" };
    nodes.area_names_ind.assign(static_cast<std::size_t>(n), 0U);
    nodes.signal_types_ind.assign(static_cast<std::size_t>(n), 0U);

    auto out_arcs = LoadedArcs(static_cast<std::size_t>(n));
    auto in_arcs = LoadedArcs(static_cast<std::size_t>(n));
    for (std::int64_t u = 0; u < n; ++u) {
        for (auto e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
            const auto v = static_cast<node_id_type>(col[e]);
            /* Duplicate arcs are summed, as the file loader does (source/graph/FileLoader.cpp:248,323). */
            out_arcs[static_cast<std::size_t>(u)][{ 0, v }] += w[e];
            in_arcs[v][{ 0, static_cast<node_id_type>(u) }] += w[e];
        }
    }
    return DistributedGraph::construct_graph(std::move(nodes), in_arcs, out_arcs);
}

/* Writes the out-arc CSR of a one-rank graph in the graph's own stored arc order. */
void export_csr(const DistributedGraph& graph, std::int64_t* n_out, std::int64_t* m_out, std::int64_t* row_ptr, std::int32_t* col, std::int32_t* w,
                std::int64_t capacity) {
    const auto n = static_cast<std::int64_t>(graph.get_number_local_nodes());
    auto m = std::int64_t{ 0 };
    for (std::int64_t u = 0; u < n; ++u) {
        const auto arcs = graph.get_out_arcs(0, static_cast<node_id_type>(u));
        if (row_ptr != nullptr) {
            row_ptr[u] = m;
        }
        for (const auto& arc : arcs) {
            if (col != nullptr && m < capacity) {
                col[m] = static_cast<std::int32_t>(arc.target_id);
                w[m] = arc.weight;
            }
            ++m;
        }
    }
    if (row_ptr != nullptr) {
        row_ptr[n] = m;
    }
    *n_out = n;
    *m_out = m;
}

template <typename d_type>
void write_apsp(const ApspGlobalResult<d_type>& result, double* cpl, double* eff, double* diameter, std::uint64_t* unreachable,
                std::uint64_t* cluster_keys, std::uint64_t* cluster_counts, std::int64_t cluster_capacity, std::int64_t* cluster_len) {
    *cpl = result.average_shortest_path_length;
    *eff = result.average_efficiency;
    *diameter = static_cast<double>(result.diameter);
    *unreachable = result.number_disconnected_pairs;
    auto i = std::int64_t{ 0 };
    for (const auto& [key, count] : result.cluster_sizes) {
        if (i < cluster_capacity) {
            cluster_keys[i] = key;
            cluster_counts[i] = count;
        }
        ++i;
    }
    *cluster_len = i;
}

} // namespace

extern "C" {

const char* ngxref_last_error() { return last_error.c_str(); }

int ngxref_fixture_count() { return static_cast<int>(FixtureAccess::all().size()); }

const char* ngxref_fixture_name(int index) {
    static auto fixtures = FixtureAccess::all();
    if (index < 0 || index >= static_cast<int>(fixtures.size())) {
        return nullptr;
    }
    return fixtures[static_cast<std::size_t>(index)].first;
}

/* Two-call protocol: first with col == nullptr to learn n and m, then with buffers of n + 1 and m entries. */
int ngxref_fixture_csr(int index, std::int64_t* n, std::int64_t* m, std::int64_t* row_ptr, std::int32_t* col, std::int32_t* w, std::int64_t capacity) {
    return guarded([&] {
        const auto fixtures = FixtureAccess::all();
        utility::Exception::check(index >= 0 && index < static_cast<int>(fixtures.size()), "fixture index {} out of range", index);
        const auto graph = fixtures[static_cast<std::size_t>(index)].second();
        export_csr(graph, n, m, row_ptr, col, w, capacity);
    });
}

/* Loads per-rank text files with the reference's file loader and load-time transforms (one rank). */
int ngxref_load_csr(const char* path, int remove_self_arcs, int undirected, int one_weight, std::int64_t* n, std::int64_t* m, std::int64_t* row_ptr,
                    std::int32_t* col, std::int32_t* w, std::int64_t capacity) {
    return guarded([&] {
        const auto graph = DistributedGraph::construct_graph(std::filesystem::path{ path }, remove_self_arcs != 0, undirected != 0, one_weight != 0, "");
        export_csr(graph, n, m, row_ptr, col, w, capacity);
    });
}

int ngxref_graph_create(std::int64_t n, const std::int64_t* row_ptr, const std::int32_t* col, const std::int32_t* w, void** out) {
    return guarded([&] { *out = new RefGraph{ build_from_csr(n, row_ptr, col, w) }; });
}

int ngxref_fixture_graph(int index, void** out) {
    return guarded([&] {
        const auto fixtures = FixtureAccess::all();
        utility::Exception::check(index >= 0 && index < static_cast<int>(fixtures.size()), "fixture index {} out of range", index);
        *out = new RefGraph{ fixtures[static_cast<std::size_t>(index)].second() };
    });
}

void ngxref_graph_destroy(void* graph) { delete static_cast<RefGraph*>(graph); }

/* The out-arc CSR of a graph in the reference's stored arc order (duplicates merged, zero weights dropped). */
int ngxref_graph_csr(void* handle, std::int64_t* n, std::int64_t* m, std::int64_t* row_ptr, std::int32_t* col, std::int32_t* w, std::int64_t capacity) {
    return guarded([&] { export_csr(static_cast<RefGraph*>(handle)->graph, n, m, row_ptr, col, w, capacity); });
}

/* queue: 0 PriorityQueue, 1 FibonacciHeap, 2 BucketQueue (source/Types.h:47-51). */
int ngxref_apsp(void* handle, int inverse, int queue, double* cpl, double* eff, double* diameter, std::uint64_t* unreachable, std::uint64_t* cluster_keys,
                std::uint64_t* cluster_counts, std::int64_t cluster_capacity, std::int64_t* cluster_len) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        const auto queue_type = static_cast<DijkstraQueueType>(queue);
        if (inverse != 0) {
            write_apsp(AllPairsShortestPath::compute_apsp_inverse(graph, queue_type), cpl, eff, diameter, unreachable, cluster_keys, cluster_counts,
                       cluster_capacity, cluster_len);
        } else {
            write_apsp(AllPairsShortestPath::compute_apsp(graph, queue_type), cpl, eff, diameter, unreachable, cluster_keys, cluster_counts,
                       cluster_capacity, cluster_len);
        }
    });
}

/* epoch: 0 PushBruteForce, 1 PushCheck, 2 PushShortLong, 3 PushInnerShort, 4 PullModel (source/Types.h:36-42). */
int ngxref_apsp_delta_stepping(void* handle, std::uint64_t delta, int epoch, double* cpl, double* eff, double* diameter, std::uint64_t* unreachable,
                               std::uint64_t* cluster_keys, std::uint64_t* cluster_counts, std::int64_t cluster_capacity, std::int64_t* cluster_len) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        write_apsp(AllPairsShortestPath::compute_apsp_delta_stepping(graph, delta, static_cast<DeltaSteppingEpochType>(epoch)), cpl, eff, diameter,
                   unreachable, cluster_keys, cluster_counts, cluster_capacity, cluster_len);
    });
}

/*
 * Full distance rows for the given sources through Dijkstra::compute_sssp, plus its per-source summary.
 * rows: k * n entries, as uint64 (regular metric, unreachable = UINT64_MAX) or double (inverse metric, unreachable = DBL_MAX);
 * summary: k * 4 doubles (sum of distances, maximum finite distance, sum of efficiencies, number unreachable).
 */
int ngxref_sssp_rows(void* handle, int inverse, int queue, const std::int64_t* sources, std::int64_t k, void* rows, double* summary) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        const auto n = static_cast<std::size_t>(graph.get_number_local_nodes());
        const auto prefix = std::vector<global_node_id_type>{ 0, n };
        const auto queue_type = static_cast<DijkstraQueueType>(queue);
        for (std::int64_t i = 0; i < k; ++i) {
            const auto source = static_cast<node_id_type>(sources[i]);
            if (inverse != 0) {
                auto distances = std::vector<inverse_distance_type>(n);
                const auto r = Dijkstra::compute_sssp<inverse_distance_type>(graph, source, prefix, distances, queue_type);
                if (rows != nullptr) {
                    std::memcpy(static_cast<double*>(rows) + i * static_cast<std::int64_t>(n), distances.data(), n * sizeof(double));
                }
                summary[4 * i + 0] = r.sum_shortest_paths;
                summary[4 * i + 1] = r.maximum_finite_distance;
                summary[4 * i + 2] = r.sum_efficiency;
                summary[4 * i + 3] = static_cast<double>(r.number_unreachable_nodes);
            } else {
                auto distances = std::vector<distance_type>(n);
                const auto r = Dijkstra::compute_sssp<distance_type>(graph, source, prefix, distances, queue_type);
                if (rows != nullptr) {
                    std::memcpy(static_cast<std::uint64_t*>(rows) + i * static_cast<std::int64_t>(n), distances.data(), n * sizeof(std::uint64_t));
                }
                summary[4 * i + 0] = static_cast<double>(r.sum_shortest_paths);
                summary[4 * i + 1] = static_cast<double>(r.maximum_finite_distance);
                summary[4 * i + 2] = r.sum_efficiency;
                summary[4 * i + 3] = static_cast<double>(r.number_unreachable_nodes);
            }
        }
    });
}

/* Per-source summary through DeltaStepping::compute_shortest_distances (4 doubles per source, as above). */
int ngxref_delta_stepping(void* handle, std::uint64_t delta, int epoch, const std::int64_t* sources, std::int64_t k, double* summary) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        for (std::int64_t i = 0; i < k; ++i) {
            const auto r = DeltaStepping::compute_shortest_distances(graph, NodeIdentifier{ 0, static_cast<node_id_type>(sources[i]) }, delta,
                                                                     static_cast<DeltaSteppingEpochType>(epoch));
            summary[4 * i + 0] = static_cast<double>(r.sum_shortest_paths);
            summary[4 * i + 1] = static_cast<double>(r.maximum_finite_distance);
            summary[4 * i + 2] = r.sum_efficiency;
            summary[4 * i + 3] = static_cast<double>(r.number_unreachable_nodes);
        }
    });
}

/* Per-node betweenness of all sources (BrandesVariant) and the average (BetweennessCentrality, algorithm 0 Brandes / 1 PathEnumeration). */
namespace {
// Replays a fixed list of draws (the last one repeating), for the constant and single-centre generators of the
// reference's own diameter tests.
class ReplayRandomNumberGenerator : public RandomNumberGenerator {
public:
    ReplayRandomNumberGenerator(const double* draws, std::int64_t count)
        : values(draws, draws + count) { }
    [[nodiscard]] double draw() override {
        const auto v = values[next < values.size() ? next : values.size() - 1];
        ++next;
        return v;
    }

private:
    std::vector<double> values;
    std::size_t next{ 0 };
};
} // namespace

/* DiameterApproximation::compute_approximation (metrics/paths/DiameterApproximation.h) with the default generator
 * (std::mt19937 seeded with `seed`) or, when draws != NULL, the replayed draws. */
int ngxref_diameter_approximation(void* handle, std::uint64_t r, const double* draws, std::int64_t num_draws, unsigned int seed, std::uint64_t* out) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        if (draws != nullptr && num_draws > 0) {
            auto generator = ReplayRandomNumberGenerator{ draws, num_draws };
            *out = DiameterApproximation::compute_approximation(graph, r, generator);
        } else {
            auto generator = DefaultRandomNumberGenerator{ seed };
            *out = DiameterApproximation::compute_approximation(graph, r, generator);
        }
    });
}

// StronglyConnectedComponents::compute_strongly_connected_components; sizes (n + 1 entries) receives component_sizes.
int ngxref_scc(void* handle, int algorithm, std::uint64_t tail_threshold, std::uint64_t* number_components, std::uint64_t* largest, std::uint64_t* sizes,
               std::int64_t capacity) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        const auto result = StronglyConnectedComponents::compute_strongly_connected_components(graph, static_cast<SccAlgorithm>(algorithm), tail_threshold);
        *number_components = result.number_components;
        *largest = result.largest_component_size;
        std::fill(sizes, sizes + capacity, std::uint64_t{ 0 });
        for (const auto& [size, count] : result.component_sizes) {
            if (static_cast<std::int64_t>(size) >= capacity) {
                throw std::runtime_error("ngxref_scc: a component size beyond the output");
            }
            sizes[size] = count;
        }
    });
}

int ngxref_betweenness(void* handle, int algorithm, double* per_node, double* average) {
    return guarded([&] {
        const auto& graph = static_cast<RefGraph*>(handle)->graph;
        const auto n = static_cast<std::size_t>(graph.get_number_local_nodes());
        if (per_node != nullptr) {
            const auto prefix = std::vector<global_node_id_type>{ 0, n };
            auto bc = std::vector<double>(n, 0.0);
            auto status = mpiPP::MPIProgress{ n, "Betweenness Centrality" };
            BrandesVariant::accumulate_betweenness(graph, prefix, bc, status);
            std::memcpy(per_node, bc.data(), n * sizeof(double));
        }
        if (average != nullptr) {
            *average = BetweennessCentrality::compute_average_betweenness_centrality(graph, static_cast<BetweennessCentralityAlgorithm>(algorithm));
        }
    });
}

} // extern "C"
