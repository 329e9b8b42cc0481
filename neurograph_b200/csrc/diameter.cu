// Diameter approximation: balls grown around random centres, the graph contracted to its balls, and the exact
// diameter of the (much smaller) contracted graph computed by the batched APSP kernel.
//
// Restates DiameterApproximation::compute_approximation (source/metrics/paths/DiameterApproximation.h) for one
// process: centres are drawn per iteration with probability 2^iteration / n from std::mt19937 through
// std::uniform_real_distribution<double> (utility/RandomNumberGenerator.h:40-52; the same library types, so the same
// numbers) or from caller-given draws; a growing step repeats rounds in which every vertex with a centre offers its
// centre along each arc of weight <= 2r to non-stable neighbours still within (iteration - generation + 1) * 2r, and
// each vertex keeps the first offer with the smallest distance (the reference answers the questions of a round in the
// order they were generated: vertices ascending, arcs in CSR order); reached vertices become stable; the iterations
// stop when every vertex is stable. The contracted graph has one vertex per centre (numbered in vertex order) and,
// per arc u -> v, the arc centre(u) -> centre(v) of weight w + d(u) + d(v), the last arc in CSR order winning when
// several map to the same pair. Its exact diameter plus 2r is the approximation.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_network.h"


namespace ngx {
namespace {

constexpr uint64_t kNoDistance = std::numeric_limits<uint64_t>::max();
constexpr uint64_t kNoGeneration = std::numeric_limits<uint64_t>::max();

struct Draws {
    const double* values;
    int64_t count;
    int64_t next = 0;
    std::mt19937 prng;
    std::uniform_real_distribution<double> dist{ 0.0, 1.0 };
    Draws(const double* v, int64_t c, uint32_t seed) : values(v), count(c), prng(seed) {}
    double draw() {
        if (values != nullptr && count > 0) {
            const double x = values[next < count ? next : count - 1];
            ++next;
            return x;
        }
        return dist(prng);
    }
};

struct Offer {
    int64_t target;
    int64_t center;
    uint64_t distance;
    uint64_t generation;
};

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_diameter_contract(const ngx_csr* csr, uint64_t r, const double* draws, int64_t num_draws, uint32_t seed, ngx_network** out) {
    return guard_host("ngx_diameter_contract", [&]() -> int {
        if (csr == nullptr || out == nullptr || csr->n < 0 || csr->m < 0 || (csr->n > 0 && csr->row_ptr == nullptr) ||
            (csr->m > 0 && (csr->col == nullptr || csr->w == nullptr))) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_contract: invalid CSR or NULL out");
        }
        *out = nullptr;
        const int64_t n = csr->n;
        if (n == 0) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_contract: the graph has no vertices");
        }
        // weights: positive integers of the reference's weight type (its distances are unsigned integers)
        for (int64_t e = 0; e < csr->m; ++e) {
            const double x = csr->w[e];
            if (x != 0.0 && !(x >= 1.0 && x <= 2147483647.0 && std::floor(x) == x)) {
                return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_contract: weights must be positive integers below 2^31 (arc " + std::to_string(e) + ")");
            }
            if (csr->col[e] < 0 || csr->col[e] >= n) {
                return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_contract: arc target out of range");
            }
        }
        std::vector<int64_t> center(static_cast<size_t>(n), -1);
        std::vector<uint64_t> distance(static_cast<size_t>(n), kNoDistance);
        std::vector<uint64_t> generation(static_cast<size_t>(n), kNoGeneration);
        std::vector<uint8_t> stable(static_cast<size_t>(n), 0);
        Draws rng(draws, num_draws, seed);
        const uint64_t two_r = 2 * r;
        const auto last_iteration = static_cast<uint64_t>(std::ceil(std::log2(static_cast<double>(n))));
        std::vector<Offer> offers;
        std::vector<int64_t> changed_list;                               // vertices changed by the last round
        std::vector<uint64_t> changed_mark(static_cast<size_t>(n), 0);  // == stamp: already in changed_list
        uint64_t stamp = 1;
        for (uint64_t iteration = 0; iteration < last_iteration; ++iteration) {
            // mark_as_centers
            const double threshold = std::pow(2.0, static_cast<double>(iteration)) / static_cast<double>(n);
            bool has_center = false;
            for (int64_t v = 0; v < n; ++v) {
                if (center[static_cast<size_t>(v)] >= 0) {
                    has_center = true;
                    continue;
                }
                if (rng.draw() >= threshold) {
                    continue;
                }
                center[static_cast<size_t>(v)] = v;
                distance[static_cast<size_t>(v)] = 0;
                generation[static_cast<size_t>(v)] = iteration;
                stable[static_cast<size_t>(v)] = 1;
                has_center = true;
            }
            if (!has_center) {
                continue;
            }
            // perform_growing_step: rounds of offers built from the round's starting state, then applied in order. The
            // first round of an iteration hears every vertex with a centre (the distance bound grows with the iteration);
            // a later round only the vertices changed by the round before: an unchanged vertex's offers were rejected, or
            // accepted and so no longer smaller, and target distances only decrease, so none of them could be accepted.
            // The offers keep their order (vertices ascending, arcs in CSR order), so the results are the same.
            bool first_round = true;
            changed_list.clear();
            for (;;) {
                offers.clear();
                const int64_t heard = first_round ? n : static_cast<int64_t>(changed_list.size());
                for (int64_t h = 0; h < heard; ++h) {
                    const int64_t u = first_round ? h : changed_list[static_cast<size_t>(h)];
                    if (center[static_cast<size_t>(u)] < 0) {
                        continue;
                    }
                    const uint64_t du = distance[static_cast<size_t>(u)];
                    const uint64_t gu = generation[static_cast<size_t>(u)];
                    for (int64_t e = csr->row_ptr[u]; e < csr->row_ptr[u + 1]; ++e) {
                        if (csr->w[e] == 0.0) {
                            continue;  // not stored by the reference
                        }
                        const uint64_t we = static_cast<uint64_t>(csr->w[e]);
                        const int64_t v = csr->col[e];
                        if (we > two_r || stable[static_cast<size_t>(v)] == 1) {
                            continue;
                        }
                        const uint64_t nd = du + we;
                        if ((iteration - gu + 1) * two_r < nd) {
                            continue;
                        }
                        if (nd >= distance[static_cast<size_t>(v)]) {
                            continue;
                        }
                        offers.push_back(Offer{ v, center[static_cast<size_t>(u)], nd, gu });
                    }
                }
                first_round = false;
                changed_list.clear();
                for (const Offer& o : offers) {
                    if (distance[static_cast<size_t>(o.target)] <= o.distance) {
                        continue;
                    }
                    center[static_cast<size_t>(o.target)] = o.center;
                    distance[static_cast<size_t>(o.target)] = o.distance;
                    generation[static_cast<size_t>(o.target)] = o.generation;
                    stable[static_cast<size_t>(o.target)] = 0;
                    if (changed_mark[static_cast<size_t>(o.target)] != stamp) {
                        changed_mark[static_cast<size_t>(o.target)] = stamp;
                        changed_list.push_back(o.target);
                    }
                }
                if (changed_list.empty()) {
                    break;
                }
                std::sort(changed_list.begin(), changed_list.end());  // heard in vertex order
                ++stamp;
            }
            // stabilize_nodes, check_all_stable
            bool all_stable = true;
            for (int64_t v = 0; v < n; ++v) {
                if (center[static_cast<size_t>(v)] >= 0) {
                    stable[static_cast<size_t>(v)] = 1;
                }
                all_stable = all_stable && stable[static_cast<size_t>(v)] == 1;
            }
            if (all_stable) {
                break;
            }
        }
        // contract: centres numbered in vertex order; every vertex mapped to its centre's new id
        std::vector<int64_t> new_id(static_cast<size_t>(n), -1);
        int64_t centers = 0;
        for (int64_t v = 0; v < n; ++v) {
            if (center[static_cast<size_t>(v)] < 0) {
                return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_contract: vertex " + std::to_string(v) + " was not reached by any centre");
            }
            if (center[static_cast<size_t>(v)] == v) {
                new_id[static_cast<size_t>(v)] = centers++;
            }
        }
        std::vector<std::map<int64_t, uint64_t>> rows(static_cast<size_t>(centers));
        for (int64_t u = 0; u < n; ++u) {
            const int64_t cu = new_id[static_cast<size_t>(center[static_cast<size_t>(u)])];
            for (int64_t e = csr->row_ptr[u]; e < csr->row_ptr[u + 1]; ++e) {
                if (csr->w[e] == 0.0) {
                    continue;
                }
                const int64_t v = csr->col[e];
                const int64_t cv = new_id[static_cast<size_t>(center[static_cast<size_t>(v)])];
                const uint64_t weight = static_cast<uint64_t>(csr->w[e]) + distance[static_cast<size_t>(u)] + distance[static_cast<size_t>(v)];
                if (weight > 2147483647ull) {
                    return fail(NGX_UNSUPPORTED, "ngx_diameter_contract: a contracted arc weight exceeds the reference's 32-bit weights");
                }
                rows[static_cast<size_t>(cu)][cv] = weight;  // the last arc in CSR order wins
            }
        }
        auto net = new ngx_network();
        net->n = centers;
        net->rank_nodes.assign(1, centers);
        net->row_ptr.assign(static_cast<size_t>(centers) + 1, 0);
        for (int64_t c = 0; c < centers; ++c) {
            for (const auto& [target, weight] : rows[static_cast<size_t>(c)]) {
                net->col.push_back(static_cast<int32_t>(target));
                net->w.push_back(static_cast<double>(weight));
            }
            net->row_ptr[static_cast<size_t>(c + 1)] = static_cast<int64_t>(net->col.size());
        }
        *out = net;
        return NGX_OK;
    });
}

int ngx_diameter_approximation(const ngx_csr* csr, uint64_t r, const double* draws, int64_t num_draws, uint32_t seed, int device, uint64_t* diameter) {
    return guard_host("ngx_diameter_approximation", [&]() -> int {
        if (diameter == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_diameter_approximation: diameter is NULL");
        }
        ngx_network* net = nullptr;
        int rc = ngx_diameter_contract(csr, r, draws, num_draws, seed, &net);
        if (rc != NGX_OK) {
            return rc;
        }
        // the exact diameter of the contracted graph (integer weights: exact in FP64)
        ngx_graph* g = nullptr;
        rc = ngx_graph_create_from_network(net, device, &g);
        if (rc == NGX_OK) {
            ngx_apsp_opts opts{};
            opts.metric = NGX_METRIC_REGULAR;
            opts.mode = NGX_MODE_BATCHED;
            ngx_apsp_result result{};
            rc = ngx_apsp(g, &opts, &result);
            if (rc == NGX_OK) {
                *diameter = static_cast<uint64_t>(result.diameter) + 2 * r;
            }
            ngx_graph_destroy(g);
        }
        delete net;
        return rc;
    });
}

}  // extern "C"
