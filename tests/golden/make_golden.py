"""Generates the committed golden fixtures under tests/golden/ from the reference implementation itself.

Run here, where the reference sources exist (the GPU machine has no copy of them):

    python tests/golden/make_golden.py

It builds oracle/_ref (the reference's own sources against single-rank shims, see oracle/Makefile), then writes

* ``reference_fixtures.npz``  the reference's one-rank test fixture graphs (tests/GraphTestOneRank.cpp,
  GraphTestFourRanks.cpp, GraphTestSevenRanks.cpp, GraphTestMultiComponent.cpp, built by the reference's own
  fixture code), seeded random integer-weight graphs, and the reference's sample input
  input/rank_1_nodes_5000_arcs_6 loaded through its FileLoader; each with the reference's outputs: APSP and
  inverse-APSP scalars, per-source summaries for every source, Brandes betweenness per node, and full distance
  rows of a few sources.
* ``reference_expectations.json``  golden values transcribed from the reference's own test files, with the
  file:line each one comes from.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

# the reference project's source tree: $NGX_REFERENCE_DIR, or where this machine keeps it
REFERENCE_DIR = oracle.REFERENCE_SOURCES or os.environ.get("NGX_REFERENCE_DIR", "/root/reference")
SAMPLE_INPUT = os.path.join(REFERENCE_DIR, "input", "rank_1_nodes_5000_arcs_6")

# Golden values from the reference's test suite (paths relative to the reference project).
EXPECTATIONS = {
    "apsp": [
        {"fixture": "standard", "cpl": 3.1, "eff": 0.4222486772486772, "eff_tol": 1e-6, "diameter": 7, "unreachable": 0,
         "cluster_sizes": {"10": 10}, "cite": "tests/apsp/test_apsp.cpp:67-84"},
        {"fixture": "standard_uu", "cpl": 1.6, "cpl_tol": 1e-6, "eff": 0.7222222222222222, "eff_tol": 1e-6, "diameter": 3,
         "unreachable": 0, "cluster_sizes": {"10": 10}, "cite": "tests/apsp/test_apsp.cpp:110-127"},
        {"fixture": "full", "cpl": 1.0, "eff": 1.0, "diameter": 1, "unreachable": 0, "cluster_sizes": {"10": 10},
         "cite": "tests/apsp/test_apsp.cpp:129-146"},
        {"fixture": "standard_four_rank_on_one_rank", "cpl": 19.784615384615385, "eff": 0.13387777556694200, "eff_tol": 1e-6,
         "diameter": 40, "unreachable": 0, "cluster_sizes": {"40": 40}, "cite": "tests/apsp/test_apsp.cpp:148-165"},
        {"fixture": "standard_uu_four_rank_on_one_rank", "cpl": 2.5025641025641026, "cpl_tol": 1e-6, "eff": 0.48384615384615381,
         "eff_tol": 1e-6, "diameter": 5, "unreachable": 0, "cluster_sizes": {"40": 40}, "cite": "tests/apsp/test_apsp.cpp:167-184"},
        {"fixture": "full_four_rank_on_one_rank", "cpl": 1.0, "eff": 1.0, "eff_tol": 1e-6, "diameter": 1, "unreachable": 0,
         "cluster_sizes": {"36": 36}, "cite": "tests/apsp/test_apsp.cpp:186-203"},
        {"fixture": "standard_seven_rank_on_one_rank", "cpl": 17.587448559670783, "eff": 0.15517143563687033, "eff_tol": 1e-6,
         "diameter": 40, "unreachable": 2886, "cluster_sizes": {"1": 6, "2": 4, "20": 20, "40": 40},
         "cite": "tests/apsp/test_apsp.cpp:461-483"},
        {"fixture": "standard_uu_seven_rank_on_one_rank", "cpl": 2.4061538461538463, "cpl_tol": 1e-6, "eff": 0.50605128205128700,
         "eff_tol": 1e-6, "diameter": 5, "unreachable": 2880, "cluster_sizes": {"1": 3, "2": 4, "3": 3, "20": 20, "40": 40},
         "cite": "tests/apsp/test_apsp.cpp:485-508"},
        {"fixture": "full_seven_rank_on_one_rank", "cpl": 1.0, "eff": 1.0, "eff_tol": 1e-6, "diameter": 1, "unreachable": 0,
         "cluster_sizes": {"63": 63}, "cite": "tests/apsp/test_apsp.cpp:510-528"},
        {"fixture": "disconnected", "cpl": 1.5, "eff": 0.75, "eff_tol": 1e-6, "diameter": 2, "unreachable": 6,
         "cluster_sizes": {"3": 3, "1": 1}, "cite": "tests/apsp/test_apsp.cpp:31-64, :86-108"},
    ],
    "apsp_inverse": [
        {"fixture": "standard", "cpl": 1.7043209876543211, "cpl_tol": 1e-6, "eff": 0.89050315072273489, "eff_tol": 1e-6,
         "diameter": 4.5, "unreachable": 0, "cluster_sizes": {"10": 10}, "cite": "tests/apsp/test_apsp.cpp:274-291"},
        {"fixture": "standard_uu", "cpl": 1.6, "cpl_tol": 1e-6, "eff": 0.7222222222222222, "eff_tol": 1e-6, "diameter": 3,
         "unreachable": 0, "cluster_sizes": {"10": 10}, "cite": "tests/apsp/test_apsp.cpp:293-310"},
        {"fixture": "full", "cpl": 1.0, "eff": 1.0, "diameter": 1, "unreachable": 0, "cluster_sizes": {"10": 10},
         "cite": "tests/apsp/test_apsp.cpp:312-329"},
        {"fixture": "standard_four_rank_on_one_rank", "cpl": 1.7130795130795136, "cpl_tol": 1e-6, "eff": 1.2097533633823983,
         "eff_tol": 1e-6, "diameter": 4.7727272727272725, "diameter_tol": 1e-6, "unreachable": 0, "cluster_sizes": {"40": 40},
         "cite": "tests/apsp/test_apsp.cpp:331-348"},
        {"fixture": "standard_seven_rank_on_one_rank", "cpl": 1.7007328947915260, "cpl_tol": 1e-6, "eff": 1.2430679013912713,
         "eff_tol": 1e-6, "diameter": 4.7727272727272725, "diameter_tol": 1e-6, "unreachable": 2886,
         "cluster_sizes": {"1": 6, "2": 4, "20": 20, "40": 40}, "cite": "tests/apsp/test_apsp.cpp:603-624"},
    ],
    "brandes_average": [
        {"fixture": "standard", "value": 13.583333333333332, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:23-34"},
        {"fixture": "standard_uu", "value": 5.4, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:36-47"},
        {"fixture": "full", "value": 0.0, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:49-60"},
        {"fixture": "standard_four_rank_on_one_rank", "value": 112.12194180319423, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:62-73"},
        {"fixture": "standard_uu_four_rank_on_one_rank", "value": 58.6, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:75-86"},
        {"fixture": "full_four_rank_on_one_rank", "value": 0.0, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:88-99"},
        {"fixture": "standard_seven_rank_on_one_rank", "value": 74.447050803480930, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:146-158"},
        {"fixture": "standard_uu_seven_rank_on_one_rank", "value": 39.171428571428571, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:160-171"},
        {"fixture": "full_seven_rank_on_one_rank", "value": 0.0, "tol": 1e-6, "cite": "tests/centrality/test_brandes.cpp:173-185"},
    ],
    # Per-source summaries of the standard graphs for every delta (tests/delta_stepping/test_push_check.cpp:25-67).
    "per_source": [
        {"fixture": "standard", "sum": [25, 31, 24, 22, 20, 45, 32, 31, 23, 26], "max": [5, 6, 4, 4, 4, 7, 6, 5, 4, 5],
         "eff": [4.3666666, 3.4833333, 4.0, 4.6666666, 4.9166666, 2.1023809, 3.2833333, 3.3166666, 4.0833333, 3.7833333],
         "eff_tol": 1e-6, "unreachable": 0, "cite": "tests/delta_stepping/test_push_check.cpp:27-48"},
        {"fixture": "standard_uu", "sum": [16, 13, 16, 13, 13, 15, 13, 17, 14, 14], "max": [3, 2, 3, 2, 2, 2, 2, 3, 2, 3],
         "eff": [6.1666666, 7.0, 5.8333333, 7.0, 7.0, 6.0, 7.0, 5.6666666, 6.5, 6.8333333],
         "eff_tol": 1e-6, "unreachable": 0, "cite": "tests/delta_stepping/test_push_check.cpp:50-72"},
    ],
}


def _disconnected():
    """tests/apsp/test_apsp.cpp:31-64: 0 -> 1 -> 2 -> 0 and an isolated node 3, unit weights."""
    return 4, np.array([0, 1, 2, 3, 3], np.int64), np.array([1, 2, 0], np.int32), np.array([1, 1, 1], np.int32)


def _random_graph(rng, n, mean_degree, wmax, negative=False):
    degrees = rng.poisson(mean_degree, size=n)
    row_ptr = np.zeros(n + 1, np.int64)
    row_ptr[1:] = np.cumsum(degrees)
    col = rng.integers(0, n, size=int(row_ptr[-1])).astype(np.int32)
    w = rng.integers(1, wmax + 1, size=col.size).astype(np.int32)
    if negative:
        w *= rng.choice(np.array([-1, 1], np.int32), size=w.size)
    return n, row_ptr, col, w


def _record(ref: oracle.Reference, prefix: str, graph: oracle.RefGraph, out: dict, rows_for=4, brandes=True) -> None:
    n, row_ptr, col, w = graph.csr()
    out[f"{prefix}/row_ptr"] = row_ptr
    out[f"{prefix}/col"] = col
    out[f"{prefix}/w"] = w
    for metric, inverse in (("regular", False), ("inverse", True)):
        a = graph.apsp(inverse=inverse)
        keys = np.array(sorted(a["cluster_sizes"]), np.uint64)
        out[f"{prefix}/{metric}/scalars"] = np.array([a["cpl"], a["efficiency"], a["diameter"], float(a["unreachable"])])
        out[f"{prefix}/{metric}/cluster_keys"] = keys
        out[f"{prefix}/{metric}/cluster_counts"] = np.array([a["cluster_sizes"][int(k)] for k in keys], np.uint64)
        if n > 0:
            rows, summary = graph.sssp_rows(np.arange(n), inverse=inverse)
            out[f"{prefix}/{metric}/per_source"] = summary
            pick = np.unique(np.linspace(0, n - 1, num=min(rows_for, n)).astype(np.int64))
            out[f"{prefix}/{metric}/row_sources"] = pick
            out[f"{prefix}/{metric}/rows"] = rows[pick]
    if brandes and n > 0:
        bc, avg = graph.betweenness()
        out[f"{prefix}/brandes/bc"] = bc
        out[f"{prefix}/brandes/average"] = np.array([avg])


def main() -> None:
    oracle.build(reference_dir=REFERENCE_DIR)
    ref = oracle.Reference()
    out: dict[str, np.ndarray] = {}
    names = []
    for i, name in enumerate(ref.fixture_names()):
        _record(ref, name, ref.fixture_graph(i), out, rows_for=64)
        names.append(name)
    ref_graph = ref.graph(*_disconnected())
    _record(ref, "disconnected", ref_graph, out, rows_for=4)
    names.append("disconnected")

    rng = np.random.default_rng(20261203)
    shapes = [(300, 4.0, 10, False), (800, 3.0, 3, False), (500, 6.0, 1, False), (200, 2.0, 5, True)]
    for j, (n, deg, wmax, neg) in enumerate(shapes):
        name = f"random_{j}"
        _record(ref, name, ref.graph(*_random_graph(rng, n, deg, wmax, neg)), out, rows_for=8)
        names.append(name)

    if os.path.isdir(SAMPLE_INPUT):
        n, row_ptr, col, w = ref.load_csr(SAMPLE_INPUT)
        sample = ref.graph(n, row_ptr, col, w)
        _record(ref, "sample_5000", sample, out, rows_for=8)
        names.append("sample_5000")

    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **out)
    with open(os.path.join(HERE, "reference_expectations.json"), "w") as f:
        json.dump(EXPECTATIONS, f, indent=1)
    print(f"wrote {len(names)} graphs: {', '.join(names)}")


if __name__ == "__main__":
    main()
