"""The oracle (the C restatement of the reference's hot path) against the reference's own outputs and golden values.

CPU only. The golden fixtures were produced by the reference implementation itself (tests/golden/make_golden.py);
where its sources and the shim build are present (oracle/_ref), the live reference is compared too.
"""

from __future__ import annotations

import math
import zlib

import numpy as np
import pytest

import oracle

UINT64_MAX = np.iinfo(np.uint64).max


def _ref_rows_as_float(rows):
    return np.where(rows == UINT64_MAX, np.inf, rows.astype(np.float64))


def test_exact_sum_is_correctly_rounded(restatement):
    rng = np.random.default_rng(7)
    cases = [
        rng.lognormal(0, 1, 10000),
        rng.random(1000) * 1e-300,                      # subnormal territory
        np.array([1e307, 5e307, 1e-320]),                 # near overflow
        np.array([1.0, 2.0 ** -53, 2.0 ** -53]),          # exact tie handling
        np.array([1.0, 2.0 ** -53]),
        np.array([1.0, 2.0 ** -53, 2.0 ** -105]),
        1.0 / np.arange(1, 20000, dtype=np.float64),
        np.zeros(3),
        np.array([5e-324]),
    ]
    for x in cases:
        assert restatement.exact_sum(x) == math.fsum(x), x[:4]


@pytest.mark.parametrize("metric", ["regular", "inverse"])
def test_restatement_matches_reference_outputs(golden, restatement, metric):
    """Scalars, cluster sizes and per-source summaries: bit-exact with the reference's own code on every fixture."""
    m = oracle.METRIC_INVERSE if metric == "inverse" else oracle.METRIC_REGULAR
    for name, g in golden.items():
        ref = g.apsp(metric)
        got = restatement.apsp(g.csr(), metric=m)
        r = got["reached_pairs"]
        if g.n == 0:
            continue
        # the reference accumulates in its own order; the restatement reproduces that order exactly
        assert got["sum_distances_sequential"] / r == ref["cpl"] or (math.isnan(ref["cpl"]) and r == 0), name
        assert got["sum_inverse_sequential"] / r == ref["efficiency"], name
        assert got["diameter"] == ref["diameter"], name
        assert got["unreachable"] == ref["unreachable"], name
        assert got["cluster_sizes"] == ref["cluster_sizes"], name
        per = g.get(f"{metric}/per_source")
        ps = got["per_source"]
        assert np.array_equal(ps["max"], per[:, 1]), name
        assert np.array_equal(ps["sum_inv_seq"], per[:, 2]), name
        assert np.array_equal(ps["unreachable"].astype(np.float64), per[:, 3]), name
        if metric == "regular":
            assert np.array_equal(ps["sum"], per[:, 0]), name  # integer sums are exact either way


@pytest.mark.parametrize("metric", ["regular", "inverse"])
def test_restatement_rows_match_reference(golden, restatement, metric):
    m = oracle.METRIC_INVERSE if metric == "inverse" else oracle.METRIC_REGULAR
    for name, g in golden.items():
        if g.n == 0:
            continue
        srcs = g.get(f"{metric}/row_sources")
        rows = g.get(f"{metric}/rows")
        for s, row in zip(srcs, rows):
            want = _ref_rows_as_float(row) if metric == "regular" else np.where(row == np.finfo(np.float64).max, np.inf, row)
            assert np.array_equal(restatement.sssp(g.csr(), int(s), m), want), (name, s)


def test_restatement_brandes_matches_reference(golden, restatement):
    """Per-node betweenness: bit-exact (same settle order, same summation order as BrandesVariant)."""
    for name, g in golden.items():
        bc_ref = g.get("brandes/bc")
        if bc_ref is None:
            continue
        bc = restatement.brandes(g.csr())
        assert np.array_equal(bc, bc_ref), name
        avg = g.get("brandes/average")[0]
        assert math.isclose(bc.sum() / g.n, avg, rel_tol=1e-12, abs_tol=1e-12), name


def test_restatement_reproduces_reference_test_expectations(golden, restatement, expectations):
    """The golden values written in the reference's own test files (file:line in the JSON)."""
    for case in expectations["apsp"] + [dict(c, inverse=True) for c in expectations["apsp_inverse"]]:
        g = golden[case["fixture"]]
        got = restatement.apsp(g.csr(), metric=oracle.METRIC_INVERSE if case.get("inverse") else oracle.METRIC_REGULAR)
        r = got["reached_pairs"]
        cpl = got["sum_distances_sequential"] / r
        eff = got["sum_inverse_sequential"] / r
        assert abs(cpl - case["cpl"]) <= case.get("cpl_tol", 0.0), case["cite"]
        assert abs(eff - case["eff"]) <= case.get("eff_tol", 0.0), case["cite"]
        assert abs(got["diameter"] - case["diameter"]) <= case.get("diameter_tol", 0.0), case["cite"]
        assert got["unreachable"] == case["unreachable"], case["cite"]
        assert got["cluster_sizes"] == {int(k): v for k, v in case["cluster_sizes"].items()}, case["cite"]
    for case in expectations["brandes_average"]:
        g = golden[case["fixture"]]
        assert abs(restatement.brandes(g.csr()).sum() / g.n - case["value"]) <= case["tol"], case["cite"]
    for case in expectations["per_source"]:
        g = golden[case["fixture"]]
        ps = restatement.apsp(g.csr())["per_source"]
        assert list(ps["sum"]) == case["sum"], case["cite"]
        assert list(ps["max"]) == case["max"], case["cite"]
        assert np.allclose(ps["sum_inv_seq"], case["eff"], atol=case["eff_tol"], rtol=0), case["cite"]
        assert (ps["unreachable"] == case["unreachable"]).all(), case["cite"]


def test_histogram_bin_rule(restatement):
    """floor(d / (H / bins)) clamped to the last bin; d >= H counted as overflow; t == s excluded."""
    g = oracle.Csr.from_arrays(3, [0, 1, 2, 2], [1, 2], [0.25, 0.75])
    got = restatement.apsp(g, sources=[0], bins=4, hist_max=1.0)
    # d(0,1) = 0.25 -> bin 1, d(0,2) = 1.0 -> overflow
    assert list(got["hist"]) == [0, 1, 0, 0]
    assert got["hist_overflow"] == 1


def _fd_grad(restatement, g, arcs, h_rel=1e-6):
    """Central differences of the per-pair sums: numerator sum(d+ - d-) formed pair by pair (no cancellation)."""
    out = []
    r = None
    for e in arcs:
        rows = {}
        for sign in (+1, -1):
            w = g.w.copy()
            h = h_rel * w[e]
            w[e] += sign * h
            gg = oracle.Csr.from_arrays(g.n, g.row_ptr, g.col, w)
            rows[sign] = np.array([restatement.sssp(gg, s) for s in range(g.n)])
        dp, dm = rows[+1], rows[-1]
        fin = np.isfinite(dp) & (dp > 0)
        h = h_rel * g.w[e]
        dcpl = float(np.sum(dp[fin] - dm[fin])) / (2 * h)
        deff = float(np.sum(1.0 / dp[fin] - 1.0 / dm[fin])) / (2 * h)
        r = int(fin.sum())
        out.append((dcpl / r, deff / r))
    return out


def test_gradient_matches_finite_differences(restatement):
    from neurograph_b200 import synth

    c = synth.connectome(120, 5, 0.2, weights="lognormal", sigma=0.5, seed=3, use_gpu=False)
    g = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    dcpl, deff, tot = restatement.apsp_grad(g)
    rng = np.random.default_rng(0)
    arcs = rng.choice(g.m, size=12, replace=False)
    for e, (fc, fe) in zip(arcs, _fd_grad(restatement, g, arcs)):
        assert math.isclose(dcpl[e], fc, rel_tol=1e-6, abs_tol=1e-12), e
        assert math.isclose(deff[e], fe, rel_tol=1e-6, abs_tol=1e-12), e
    plain = restatement.apsp(g)
    assert tot["cpl"] == plain["cpl"] and tot["efficiency"] == plain["efficiency"]


@pytest.mark.skipif(not oracle.Reference.available(), reason="reference shim build not present")
def test_restatement_matches_live_reference_on_random_graphs(restatement):
    ref = oracle.Reference()
    rng = np.random.default_rng(11)
    for n, deg, wmax in [(150, 3.0, 4), (400, 5.0, 10), (300, 1.5, 2)]:
        degrees = rng.poisson(deg, n)
        row_ptr = np.concatenate([[0], np.cumsum(degrees)]).astype(np.int64)
        col = rng.integers(0, n, row_ptr[-1]).astype(np.int32)
        w = rng.integers(1, wmax + 1, row_ptr[-1]).astype(np.int32)
        rg = ref.graph(n, row_ptr, col, w)
        n2, rp2, col2, w2 = rg.csr()
        g = oracle.Csr.from_arrays(n2, rp2, col2, w2.astype(np.float64))
        ra = rg.apsp()
        oa = restatement.apsp(g)
        assert ra["cpl"] == oa["sum_distances_sequential"] / oa["reached_pairs"]
        assert ra["efficiency"] == oa["sum_inverse_sequential"] / oa["reached_pairs"]
        assert ra["cluster_sizes"] == oa["cluster_sizes"] and ra["diameter"] == oa["diameter"]
        bc_ref, _ = rg.betweenness()
        assert np.array_equal(bc_ref, restatement.brandes(g))
        for epoch in range(4):  # PushBruteForce, PushCheck, PushShortLong, PushInnerShort
            da = rg.apsp_delta_stepping(3, epoch)
            assert da["cpl"] == ra["cpl"] and da["diameter"] == ra["diameter"]


def _family(kind, rng):
    """Random integer graphs with what the reference's loader and Dijkstra must handle."""
    n = 220
    degrees = rng.poisson(4.0, n)
    row_ptr = np.concatenate([[0], np.cumsum(degrees)]).astype(np.int64)
    m = int(row_ptr[-1])
    col = rng.integers(0, n, m).astype(np.int32)
    if kind == "signed_and_zero":  # lengths are |w|; zero weights are absent arcs
        w = rng.integers(-6, 7, m)
    elif kind == "heavy":  # weights up to the int32 limit: sums far above 2^32, still exact in FP64 here
        w = rng.integers(1, 2**31 - 1, m)
    elif kind == "self_and_repeated":  # self arcs, and arcs repeated within a row
        src = np.repeat(np.arange(n), degrees)
        col = np.where(rng.random(m) < 0.1, src, col).astype(np.int32)
        dup = np.nonzero(np.diff(row_ptr) >= 2)[0]
        col[row_ptr[dup] + 1] = col[row_ptr[dup]]
        w = rng.integers(1, 9, m)
    else:  # "components": arcs only inside blocks of 11 vertices
        src = np.repeat(np.arange(n), degrees)
        col = ((src // 11) * 11 + rng.integers(0, 11, m)).clip(0, n - 1).astype(np.int32)
        w = rng.integers(1, 9, m)
    return n, row_ptr, col, w.astype(np.int32)


@pytest.mark.skipif(not oracle.Reference.available(), reason="reference shim build not present")
@pytest.mark.parametrize("kind", ["signed_and_zero", "heavy", "self_and_repeated", "components"])
def test_restatement_matches_live_reference_on_graph_families(restatement, kind):
    ref = oracle.Reference()
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    for _ in range(2):
        n, row_ptr, col, w = _family(kind, rng)
        rg = ref.graph(n, row_ptr, col, w)
        n2, rp2, col2, w2 = rg.csr()  # the reference's stored arcs (zero weights dropped) in its order
        g = oracle.Csr.from_arrays(n2, rp2, col2, w2.astype(np.float64))
        for inverse in (False, True):
            ra = rg.apsp(inverse=inverse)
            oa = restatement.apsp(g, metric=oracle.METRIC_INVERSE if inverse else oracle.METRIC_REGULAR)
            assert ra["cpl"] == oa["sum_distances_sequential"] / oa["reached_pairs"], (kind, inverse)
            assert ra["efficiency"] == oa["sum_inverse_sequential"] / oa["reached_pairs"], (kind, inverse)
            assert ra["diameter"] == oa["diameter"] and ra["cluster_sizes"] == oa["cluster_sizes"], (kind, inverse)
            assert ra["unreachable"] == oa["unreachable"], (kind, inverse)
        bc_ref, _ = rg.betweenness()
        bc = restatement.brandes(g)
        assert np.allclose(bc, bc_ref, rtol=1e-12, atol=1e-12 * max(1.0, float(np.abs(bc_ref).mean()))), kind


@pytest.mark.skipif(not oracle.Reference.available(), reason="reference shim build not present")
def test_reference_pull_model_misses_shortest_paths():
    """A finding, kept as a test: the reference's PullModel epoch (DeltaSteppingVariants/PullModelVariant.h) returns
    distances longer than Dijkstra's on this random integer graph with delta = 3 and arcs heavier than delta, so its
    APSP differs from compute_apsp. The other four epochs agree with Dijkstra, as tests/apsp/test_apsp_delta_stepping.cpp
    requires; the GPU delta-stepping returns Dijkstra's fixed point."""
    ref = oracle.Reference()
    rng = np.random.default_rng(11)
    n, deg, wmax = 150, 3.0, 4
    degrees = rng.poisson(deg, n)
    row_ptr = np.concatenate([[0], np.cumsum(degrees)]).astype(np.int64)
    col = rng.integers(0, n, row_ptr[-1]).astype(np.int32)
    w = rng.integers(1, wmax + 1, row_ptr[-1]).astype(np.int32)
    rg = ref.graph(n, row_ptr, col, w)
    dijkstra = rg.apsp()
    pull = rg.apsp_delta_stepping(3, 4)
    assert pull["cpl"] > dijkstra["cpl"]
    assert rg.apsp_delta_stepping(1000, 4)["cpl"] == dijkstra["cpl"]  # no heavy arcs: agrees


@pytest.mark.skipif(not __import__("os").path.exists(oracle.REFERENCE_GTESTS), reason="reference gtests not built")
def test_reference_own_hot_path_tests_pass_under_the_shim():
    """The reference's own tests/apsp, tests/dijkstra, tests/delta_stepping and tests/centrality files, compiled from
    its sources against the single-rank shims, pass: the shim build runs the reference faithfully."""
    import subprocess

    out = subprocess.run([oracle.REFERENCE_GTESTS], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "0 failed" in out.stdout
