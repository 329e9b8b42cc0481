// C++20 host-side adapter between neurograph's DistributedGraph / metric classes and the neurograph-b200 C ABI.
//
// Header-only; a maintainer includes it from the reference's metric headers, where the new GPU enum values are
// dispatched (AllPairsShortestPath::compute_apsp_impl, BetweennessCentrality::compute_average_betweenness_centrality).
// It mirrors the reference's own interfaces:
//   compute_apsp_gpu<distance_type>          AllPairsShortestPath::compute_apsp           (AllPairsShortestPath.h:54-57)
//   compute_apsp_gpu<inverse_distance_type>  AllPairsShortestPath::compute_apsp_inverse   (AllPairsShortestPath.h:76-79)
//   compute_average_betweenness_gpu          BetweennessCentrality::compute_average_betweenness_centrality
//                                            (BetweennessCentrality.h:46-80)
// with the same argument meaning, the same result types (ApspGlobalResult, source/Types.h:237-244) and the same error
// behaviour: a failure throws utility::Exception (external/cpp-utility/Exception.hpp), as Dijkstra::compute_sssp does
// for invalid input (Dijkstra.h:66-75).
#pragma once

#include "ngx_b200.h"

#include "Types.h"
#include "graph/DistributedGraph.h"

#include <cpp-utility/Exception.hpp>

#include <mpi-wrapper/core/MPIInfo.h>

#include <cmath>
#include <cstdint>
#include <span>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace ngx_neurograph {

inline void check(const int status) {
    if (status != NGX_OK) {
        utility::Exception::fail("neurograph-b200: {} ({})", ngx_status_string(status), ngx_last_error());
    }
}

// Global out-arc CSR of a one-rank graph, in the graph's stored arc order (DistributedGraph::get_out_arcs,
// DistributedGraph.h:275-311; global id = prefix_distribution[rank] + local id, AllPairsShortestPath.h:115-117).
struct HostCsr {
    std::int64_t n = 0;
    std::vector<std::int64_t> row_ptr{};
    std::vector<std::int32_t> col{};
    std::vector<double> w{};
};

[[nodiscard]] inline HostCsr build_csr(const DistributedGraph& graph) {
    utility::Exception::check(mpiPP::MPIInfo::get_number_ranks() == 1, "neurograph-b200: the GPU path runs on one rank (one GPU)");
    const auto n = graph.get_number_local_nodes();
    auto csr = HostCsr{};
    csr.n = static_cast<std::int64_t>(n);
    csr.row_ptr.reserve(static_cast<std::size_t>(n) + 1);
    csr.row_ptr.push_back(0);
    for (auto u = node_id_type{ 0 }; u < n; ++u) {
        for (const auto& [target_rank, target_id, weight] : graph.get_out_arcs(0, u)) {
            csr.col.push_back(static_cast<std::int32_t>(target_id));
            csr.w.push_back(static_cast<double>(weight));  // the library takes |w| (or 1/|w|), DijkstraCommon.h:36-54
        }
        csr.row_ptr.push_back(static_cast<std::int64_t>(csr.col.size()));
    }
    return csr;
}

// Owns one device-resident graph (CSR + reverse CSR).
class GpuGraph {
public:
    explicit GpuGraph(const DistributedGraph& graph, const int device = 0)
        : csr_(build_csr(graph)) {
        const auto view = ngx_csr{ csr_.n, static_cast<std::int64_t>(csr_.col.size()), csr_.row_ptr.data(), csr_.col.data(), csr_.w.data() };
        check(ngx_graph_create(&view, device, &handle_));
    }
    GpuGraph(const GpuGraph&) = delete;
    GpuGraph& operator=(const GpuGraph&) = delete;
    ~GpuGraph() { ngx_graph_destroy(handle_); }

    [[nodiscard]] ngx_graph* get() const noexcept { return handle_; }
    [[nodiscard]] std::int64_t number_nodes() const noexcept { return csr_.n; }

private:
    HostCsr csr_;
    ngx_graph* handle_ = nullptr;
};

struct GpuOptions {
    double delta = 0.0;  // bucket width; 0 picks one from the arc lengths (--apsp-delta maps here for gpu-batched)
    std::int64_t histogram_bins = 0;
    double histogram_max = 0.0;
};

// AllPairsShortestPath::compute_apsp / compute_apsp_inverse on the GPU (all sources). d_type selects the metric as in
// the reference: distance_type uses |w|, inverse_distance_type uses 1/|w|.
template <typename d_type>
[[nodiscard]] ApspGlobalResult<d_type> compute_apsp_gpu(const DistributedGraph& graph, const GpuOptions& options = {},
                                                        std::vector<std::uint64_t>* histogram = nullptr) {
    static_assert(std::is_same_v<d_type, distance_type> || std::is_same_v<d_type, inverse_distance_type>);
    const auto gpu = GpuGraph{ graph };
    const auto n = static_cast<std::size_t>(gpu.number_nodes());
    auto unreachable = std::vector<std::uint64_t>(n);
    auto opts = ngx_apsp_opts{};
    opts.metric = std::is_same_v<d_type, distance_type> ? NGX_METRIC_REGULAR : NGX_METRIC_INVERSE;
    opts.mode = NGX_MODE_BATCHED;
    opts.delta = options.delta;
    opts.hist_bins = options.histogram_bins;
    opts.hist_max = options.histogram_max;
    auto result = ngx_apsp_result{};
    result.src_unreachable = unreachable.data();
    if (histogram != nullptr && options.histogram_bins > 0) {
        histogram->assign(static_cast<std::size_t>(options.histogram_bins), 0);
        result.hist = histogram->data();
    }
    check(ngx_apsp(gpu.get(), &opts, &result));

    auto out = ApspGlobalResult<d_type>{};
    out.average_shortest_path_length = result.cpl;
    out.average_efficiency = result.efficiency;
    if constexpr (std::is_same_v<d_type, distance_type>) {
        out.diameter = static_cast<distance_type>(result.diameter);  // integer-valued: exact below 2^53
    } else {
        out.diameter = result.diameter;
    }
    out.number_disconnected_pairs = result.unreachable;
    for (const auto u : unreachable) {
        ++out.cluster_sizes[static_cast<global_node_id_type>(n) - u];  // AllPairsShortestPath.h:139-140
    }
    return out;
}

// BetweennessCentrality::compute_average_betweenness_centrality on the GPU (Brandes, all sources).
[[nodiscard]] inline double compute_average_betweenness_gpu(const DistributedGraph& graph, std::vector<double>* per_node = nullptr,
                                                             const GpuOptions& options = {}) {
    const auto gpu = GpuGraph{ graph };
    auto bc = std::vector<double>(static_cast<std::size_t>(gpu.number_nodes()));
    auto opts = ngx_apsp_opts{};
    opts.metric = NGX_METRIC_REGULAR;
    opts.mode = NGX_MODE_BATCHED;
    opts.delta = options.delta;
    check(ngx_brandes(gpu.get(), &opts, bc.data(), nullptr));
    auto sum = 0.0;
    for (const auto value : bc) {
        sum += value;
    }
    if (per_node != nullptr) {
        *per_node = std::move(bc);
    }
    return sum / static_cast<double>(gpu.number_nodes());  // BetweennessCentrality.h:76-79
}

// StronglyConnectedComponents::compute_strongly_connected_components on the GPU (any SccAlgorithm gives this result).
[[nodiscard]] inline SccResult compute_scc_gpu(const DistributedGraph& graph) {
    const auto gpu = GpuGraph{ graph };
    const auto n = static_cast<std::size_t>(gpu.number_nodes());
    auto histogram = std::vector<std::uint64_t>(n + 1);
    auto number = std::uint64_t{};
    auto largest = std::uint64_t{};
    check(ngx_scc(gpu.get(), nullptr, &number, &largest, histogram.data()));
    auto out = SccResult{};
    out.number_components = number;
    out.largest_component_size = largest;
    for (std::size_t size = 1; size <= n; ++size) {
        if (histogram[size] != 0) {
            out.component_sizes[size] = histogram[size];
        }
    }
    return out;
}

}  // namespace ngx_neurograph
