"""Parity of the CUDA APSP path (through the C ABI) with the oracle and with the reference's own outputs.

Bit-exact: distances, per-source exact sums, maxima, unreachable counts, cluster sizes, histogram counts, CPL (the
exactly rounded sum of distances over R). Efficiency: bit-exact against the oracle's exactly rounded sum, and within
the reference's own rounding bound (terms * eps * sum) against the reference's sequential sum.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps
MODES = ["batched", "plain"]


def gpu_graph(n, row_ptr, col, w):
    return ngx.Graph(n, row_ptr, col, w)


def check_against_oracle(g_gpu, csr, restatement, metric="regular", mode="batched", sources=None, bins=0, hist_max=0.0, delta=0.0):
    m = oracle.METRIC_INVERSE if metric == "inverse" else oracle.METRIC_REGULAR
    want = restatement.apsp(csr, sources=sources, metric=m, bins=bins, hist_max=hist_max)
    got = g_gpu.apsp(sources=sources, metric=metric, mode=mode, per_source=True, hist_bins=bins, hist_max=hist_max, delta=delta)
    ps, ws = got.per_source, want["per_source"]
    assert np.array_equal(ps["sum"], ws["sum"])
    assert np.array_equal(ps["sum_inv"], ws["sum_inv"])
    assert np.array_equal(ps["max"], ws["max"])
    assert np.array_equal(ps["unreachable"], ws["unreachable"])
    assert np.array_equal(ps["arcs"], ws["arcs"])
    assert got.sum_distances == want["sum_distances"]
    assert got.sum_inverse == want["sum_inverse"]
    assert got.diameter == want["diameter"]
    assert got.unreachable == want["unreachable"]
    assert got.reached_pairs == want["reached_pairs"]
    assert got.traversed_arcs == want["traversed_arcs"]
    assert got.cluster_sizes == want["cluster_sizes"]
    if want["reached_pairs"] > 0:
        assert got.cpl == want["cpl"] and got.efficiency == want["efficiency"]
    if bins:
        assert np.array_equal(got.hist, want["hist"])
        assert got.hist_overflow == want["hist_overflow"]
    return got, want


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("metric", ["regular", "inverse"])
def test_reference_fixtures(golden, restatement, mode, metric):
    """Every reference fixture graph (the reference's own fixture builders) and its APSP outputs."""
    for name, g in golden.items():
        if g.n == 0:
            continue
        with gpu_graph(g.n, g.row_ptr, g.col, g.w) as gg:
            got, want = check_against_oracle(gg, g.csr(), restatement, metric=metric, mode=mode, bins=64, hist_max=64.0)
            ref = g.apsp(metric)
            assert got.diameter == ref["diameter"], name
            assert got.unreachable == ref["unreachable"], name
            assert got.cluster_sizes == ref["cluster_sizes"], name
            if metric == "regular":
                assert got.cpl == ref["cpl"], name  # integer distances: exact sum, same rounding as the reference
            else:
                assert math.isclose(got.cpl, ref["cpl"], rel_tol=g.n * g.n * EPS), name
            bound = got.reached_pairs * EPS * 4
            assert math.isclose(got.efficiency, ref["efficiency"], rel_tol=bound), name


@pytest.mark.parametrize("mode", MODES)
def test_reference_fixture_rows(golden, mode):
    for name, g in golden.items():
        if g.n == 0:
            continue
        for metric in ("regular", "inverse"):
            srcs = g.get(f"{metric}/row_sources")
            rows = g.get(f"{metric}/rows")
            with gpu_graph(g.n, g.row_ptr, g.col, g.w) as gg:
                got = gg.sssp_rows(srcs, metric=metric, mode=mode)
            if metric == "regular":
                want = np.where(rows == np.iinfo(np.uint64).max, np.inf, rows.astype(np.float64))
            else:
                want = np.where(rows == np.finfo(np.float64).max, np.inf, rows)
            assert np.array_equal(got, want), (name, metric)


@pytest.mark.parametrize("mode", MODES)
def test_sample_input_all_sources(golden, restatement, mode):
    """The reference's sample input (5000 vertices, read by its FileLoader), all sources."""
    g = golden["sample_5000"]
    with gpu_graph(g.n, g.row_ptr, g.col, g.w) as gg:
        got, _ = check_against_oracle(gg, g.csr(), restatement, mode=mode, bins=1024, hist_max=float(g.apsp()["diameter"]) + 1)
    ref = g.apsp()
    assert got.cpl == ref["cpl"] and got.diameter == ref["diameter"] and got.cluster_sizes == ref["cluster_sizes"]


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("weights", ["lognormal", "int", "unit"])
def test_synthetic_connectomes(restatement, seed, weights):
    c = synth.connectome(1500, 12, 0.15, weights=weights, seed=seed, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with gpu_graph(c.n, c.row_ptr, c.col, c.w) as gg:
        got, want = check_against_oracle(gg, csr, restatement, bins=1024, hist_max=0.0 + 40.0)
        srcs = np.array([0, 7, 999, 1499])
        rows = gg.sssp_rows(srcs)
        for s, row in zip(srcs, rows):
            assert np.array_equal(row, restatement.sssp(csr, int(s)))
        plain, _ = check_against_oracle(gg, csr, restatement, mode="plain", sources=np.arange(0, 1500, 7))


def test_delta_does_not_change_results(restatement):
    c = synth.connectome(800, 10, 0.2, weights="lognormal", seed=5, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with gpu_graph(c.n, c.row_ptr, c.col, c.w) as gg:
        for delta in (1e-3, 0.05, 1.0, 1e9):
            for mode in MODES:
                check_against_oracle(gg, csr, restatement, mode=mode, delta=delta)


def test_source_subsets_duplicates_and_ragged_tiles(restatement):
    c = synth.random_graph(700, 4, weights="lognormal", seed=9)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with gpu_graph(c.n, c.row_ptr, c.col, c.w) as gg:
        for srcs in ([5], [3, 3, 3], list(range(33)), list(range(699, 0, -13)), [0] * 70):
            for mode in MODES:
                check_against_oracle(gg, csr, restatement, mode=mode, sources=np.array(srcs))


def test_edge_cases(restatement):
    # single vertex, no arcs
    with gpu_graph(1, [0, 0], [], []) as gg:
        r = gg.apsp(per_source=True)
        assert r.reached_pairs == 0 and math.isnan(r.cpl) and r.cluster_sizes == {1: 1}
    # zero-weight arcs are absent; self loops never shorten anything; negative weights count by absolute value
    n, row_ptr, col, w = 4, [0, 3, 4, 5, 5], [1, 0, 2, 2, 3], [0.0, 2.0, -3.0, 1.5, -0.5]
    csr = oracle.Csr.from_arrays(n, row_ptr, col, w)
    with gpu_graph(n, row_ptr, col, w) as gg:
        for mode in MODES:
            for metric in ("regular", "inverse"):
                check_against_oracle(gg, csr, restatement, mode=mode, metric=metric)
    # empty graph
    with gpu_graph(0, [0], [], []) as gg:
        r = gg.apsp()
        assert r.reached_pairs == 0


def test_errors_leave_the_context_usable(restatement):
    c = synth.random_graph(400, 5, weights="lognormal", seed=2)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with gpu_graph(c.n, c.row_ptr, c.col, c.w) as gg:
        with pytest.raises(ngx.NgxError) as e:
            gg.apsp(sources=[400])
        assert e.value.status == 1
        with pytest.raises(ngx.NgxError) as e:
            gg.apsp(max_iterations=1, delta=1e-6)
        assert e.value.status == 4  # TIMEOUT: the iteration cap stops the kernel, it reports instead of spinning
        check_against_oracle(gg, csr, restatement)


def test_source_order_is_a_permutation_and_runs_agree():
    """All-sources runs take the sources in the graph's locality order; the order is a permutation, per-source outputs
    still come back by vertex, and running contiguous chunks of the order gives the same totals as one run."""
    c = synth.connectome(2000, 12, 0.15, weights="lognormal", seed=5, use_gpu=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        order = g.source_order()
        assert np.array_equal(np.sort(order), np.arange(c.n))
        whole = g.apsp(per_source=True)
        by_vertex = g.apsp(sources=np.arange(c.n), per_source=True)
        for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
            assert np.array_equal(whole.per_source[k], by_vertex.per_source[k]), k
        assert whole.sum_distances == by_vertex.sum_distances and whole.cluster_sizes == by_vertex.cluster_sizes
        digits = np.zeros((2, ngx.ACC_DIGITS), np.uint64)
        for chunk in np.array_split(order, 5):
            digits += g.apsp(sources=chunk, exact=True).acc_digits
        assert ngx.exact_round(digits[0]) == whole.sum_distances
        assert ngx.exact_round(digits[1]) == whole.sum_inverse
    small = synth.connectome(40, 4, 0.3, weights="int", seed=6, use_gpu=False)
    graphs = [(c.n, c.row_ptr, c.col, c.w), (small.n, small.row_ptr, small.col, small.w)]
    with ngx.Batch(graphs) as b:
        results, _ = b.run("apsp", per_source=True)
    assert np.array_equal(results[0].per_source["sum"], whole.per_source["sum"])


def test_graph_from_network_files(tmp_path, restatement):
    """ngx_network_load + ngx_graph_create_from_network: a graph built straight from per-rank network files runs the
    same APSP as one built from the loaded CSR, and matches the oracle on that CSR."""
    from test_loader import write_network

    write_network(str(tmp_path), 500, 2, np.random.default_rng(3))
    with ngx.Graph.from_network(str(tmp_path), 2, remove_self_arcs=True) as g:
        got = g.apsp(per_source=True, hist_bins=64, hist_max=40.0)
        csr = oracle.Csr.from_arrays(g.n, g.row_ptr, g.col, g.w)
    want = restatement.apsp(csr, bins=64, hist_max=40.0)
    assert got.sum_distances == want["sum_distances"] and got.unreachable == want["unreachable"]
    assert got.cluster_sizes == want["cluster_sizes"] and np.array_equal(got.hist, want["hist"])
    n, rp, c, w = ngx.load_network(str(tmp_path), 2, remove_self_arcs=True)
    with ngx.Graph(n, rp, c, w) as g2:
        again = g2.apsp()
    assert again.sum_distances == got.sum_distances and again.diameter == got.diameter


@pytest.mark.parametrize("kind", ["signed_and_zero", "heavy", "self_and_repeated", "components"])
def test_graph_families_against_oracle(restatement, kind):
    """The families the oracle is pinned on against the live reference (tests/test_oracle.py): signed and zero weights,
    weights up to the int32 limit, self and repeated arcs, many small components; both metrics, both forms, and
    betweenness."""
    import zlib

    from test_oracle import _family

    rng = np.random.default_rng(zlib.crc32(kind.encode()) + 1)
    for _ in range(2):
        n, row_ptr, col, w = _family(kind, rng)
        w = w.astype(np.float64)
        csr = oracle.Csr.from_arrays(n, row_ptr, col, w)
        with gpu_graph(n, row_ptr, col, w) as gg:
            for metric in ("regular", "inverse"):
                for mode in MODES:
                    check_against_oracle(gg, csr, restatement, metric=metric, mode=mode, bins=32, hist_max=4.0e9 if kind == "heavy" else 64.0)
            bc, _ = gg.brandes()
        want = restatement.brandes(csr)
        assert np.allclose(bc, want, rtol=1e-12, atol=1e-12 * max(1.0, float(np.abs(want).mean()))), kind
