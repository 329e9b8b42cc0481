/*
 * Integration check (test infrastructure): the reference's own one-rank fixture graphs, built by its own fixture
 * code, go through the reference's AllPairsShortestPath / BetweennessCentrality and through the C++20 adapter
 * neurograph_b200/host/ngx_neurograph.h that a maintainer would call from those classes. The results
 * must agree: CPL, diameter, unreachable pairs and cluster sizes exactly, efficiency within the reference's rounding,
 * average betweenness within 1e-12 relative, strongly connected components exactly. Exit code 0 when every fixture agrees. Needs a B200.
 */
#include "GraphTest.h"
#include "Types.h"

#include "metrics/paths/AllPairsShortestPath.h"
#include "metrics/paths/BetweennessCentrality.h"
#include "metrics/connectivity/StronglyConnectedComponents.h"

#include "ngx_neurograph.h"

#include <mpi-wrapper/MPIWrapper.h>
#include <mpi-wrapper/instrumentation/MPIProgress.h>

#include <cmath>
#include <cstdio>
#include <functional>
#include <utility>
#include <vector>

namespace {
class Fixtures : public GraphTest {
public:
    void TestBody() override { }
    static std::vector<std::pair<const char*, std::function<DistributedGraph()>>> all() {
        return {
            { "standard", [] { return get_standard_one_rank_graph(); } },
            { "standard_uu", [] { return get_standard_uu_one_rank_graph(); } },
            { "full", [] { return get_full_one_rank_graph(); } },
            { "negative_weight", [] { return get_negative_weight_one_rank_graph(); } },
            { "standard_four_rank_on_one_rank", [] { return get_standard_four_rank_graph_on_one_rank(); } },
            { "standard_seven_rank_on_one_rank", [] { return get_standard_seven_rank_graph_on_one_rank(); } },
            { "standard_uu_seven_rank_on_one_rank", [] { return get_standard_uu_seven_rank_graph_on_one_rank(); } },
            { "multi_component_four_rank_on_one_rank", [] { return get_multi_component_four_rank_graph_on_one_rank(); } },
        };
    }
};

template <typename R>
bool same_apsp(const R& a, const R& b, double eff_rel) {
    return a.average_shortest_path_length == b.average_shortest_path_length && a.diameter == b.diameter &&
           a.number_disconnected_pairs == b.number_disconnected_pairs && a.cluster_sizes == b.cluster_sizes &&
           std::fabs(a.average_efficiency - b.average_efficiency) <= eff_rel * std::fabs(b.average_efficiency);
}
}  // namespace

int main(int argc, char** argv) {
    mpiPP::MPIWrapper::init(argc, argv);
    mpiPP::MPIProgress::set_disable_status(true);
    int failures = 0;
    for (const auto& [name, make] : Fixtures::all()) {
        const auto graph = make();
        const auto ref = AllPairsShortestPath::compute_apsp(graph);
        const auto gpu = ngx_neurograph::compute_apsp_gpu<distance_type>(graph);
        const auto ref_inv = AllPairsShortestPath::compute_apsp_inverse(graph);
        const auto gpu_inv = ngx_neurograph::compute_apsp_gpu<inverse_distance_type>(graph);
        const bool apsp_ok = same_apsp(gpu, ref, 1e-13);
        const bool inv_ok = std::fabs(gpu_inv.average_shortest_path_length - ref_inv.average_shortest_path_length) <=
                                1e-13 * std::fabs(ref_inv.average_shortest_path_length) &&
                            gpu_inv.diameter == ref_inv.diameter && gpu_inv.cluster_sizes == ref_inv.cluster_sizes &&
                            std::fabs(gpu_inv.average_efficiency - ref_inv.average_efficiency) <= 1e-13 * std::fabs(ref_inv.average_efficiency);
        const auto bc_ref = BetweennessCentrality::compute_average_betweenness_centrality(graph);
        const auto bc_gpu = ngx_neurograph::compute_average_betweenness_gpu(graph);
        const bool bc_ok = std::fabs(bc_gpu - bc_ref) <= 1e-12 * std::fmax(1.0, std::fabs(bc_ref));
        const auto scc_ref = StronglyConnectedComponents::compute_strongly_connected_components(graph);
        const auto scc_gpu = ngx_neurograph::compute_scc_gpu(graph);
        const bool scc_ok = scc_gpu.number_components == scc_ref.number_components && scc_gpu.largest_component_size == scc_ref.largest_component_size &&
                            scc_gpu.component_sizes == scc_ref.component_sizes;
        std::printf("%-40s apsp %s  inverse %s  betweenness %s (%.17g vs %.17g)  scc %s\n", name, apsp_ok ? "ok" : "MISMATCH", inv_ok ? "ok" : "MISMATCH",
                    bc_ok ? "ok" : "MISMATCH", bc_gpu, bc_ref, scc_ok ? "ok" : "MISMATCH");
        if (!apsp_ok || !inv_ok) {
            std::printf("  regular: gpu cpl %.17g eff %.17g dia %llu unreach %llu clusters %zu | ref cpl %.17g eff %.17g dia %llu unreach %llu clusters %zu\n",
                        gpu.average_shortest_path_length, gpu.average_efficiency, static_cast<unsigned long long>(gpu.diameter),
                        static_cast<unsigned long long>(gpu.number_disconnected_pairs), gpu.cluster_sizes.size(), ref.average_shortest_path_length,
                        ref.average_efficiency, static_cast<unsigned long long>(ref.diameter), static_cast<unsigned long long>(ref.number_disconnected_pairs),
                        ref.cluster_sizes.size());
            std::printf("  inverse: gpu cpl %.17g eff %.17g dia %.17g | ref cpl %.17g eff %.17g dia %.17g\n", gpu_inv.average_shortest_path_length,
                        gpu_inv.average_efficiency, gpu_inv.diameter, ref_inv.average_shortest_path_length, ref_inv.average_efficiency, ref_inv.diameter);
        }
        failures += apsp_ok && inv_ok && bc_ok && scc_ok ? 0 : 1;
    }
    mpiPP::MPIWrapper::finalize();
    return failures == 0 ? 0 : 1;
}
