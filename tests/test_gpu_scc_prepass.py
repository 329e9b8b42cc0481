"""The strongly-connected-components pre-pass of the APSP runs (through the C ABI).

On a graph of several strongly connected components a single-graph handle computes its components once (ngx_scc),
keeps each component's sources together in its all-sources order, and lets every source tile keep a list of the
vertices it reached, so that the bucket steps and the APSP epilogue visit those instead of all n vertices
(StronglyConnectedComponents.h:34-35 in the reference is the component computation this reuses). None of it may change
a result: APSP summaries, per-source outputs and histograms bit for bit, betweenness within 1e-12, against the oracle,
on the SCC test families and on many disjoint small components; with groups of CTAs per tile too; and the order must
hold each component's sources together.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth
from test_scc import scc_family

pytestmark = pytest.mark.gpu

REL = 1e-12


def many_components(n_blocks=400, size=25, seed=0):
    """Disjoint connectomes of `size` vertices (one component each, or a few), plus one-way arcs between some."""
    rng = np.random.default_rng(seed)
    rows, cols, ws = [], [], []
    n = n_blocks * size
    for b in range(n_blocks):
        c = synth.connectome(size, 3, 0.3, weights="lognormal", seed=seed * 1000 + b, use_gpu=False)
        for u in range(size):
            for e in range(c.row_ptr[u], c.row_ptr[u + 1]):
                rows.append(b * size + u)
                cols.append(b * size + int(c.col[e]))
                ws.append(float(c.w[e]))
    for _ in range(n_blocks // 4):  # arcs from a block to a later one: components reach others, not back
        a = int(rng.integers(0, n_blocks - 1))
        bb = int(rng.integers(a + 1, n_blocks))
        rows.append(a * size + int(rng.integers(0, size)))
        cols.append(bb * size + int(rng.integers(0, size)))
        ws.append(float(rng.lognormal()))
    order = np.argsort(np.asarray(rows), kind="stable")
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, np.asarray(rows) + 1, 1)
    return n, np.cumsum(row_ptr), np.asarray(cols, np.int32)[order], np.asarray(ws)[order]


CASES = {
    "sparse": lambda: scc_family("sparse", 6000, 11),
    "cycles_dag": lambda: scc_family("cycles_dag", 6000, 12),
    "zero_weights": lambda: scc_family("zero_weights", 5000, 13),
    "isolated": lambda: scc_family("isolated", 5000, 14),
    "many_components": lambda: many_components(),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("tile_ctas", [1, 4])
def test_results_with_the_prepass_match_the_oracle(restatement, name, tile_ctas):
    n, rp, col, w = CASES[name]()
    csr = oracle.Csr.from_arrays(n, rp, col, w)
    want = restatement.apsp(csr, bins=128, hist_max=60.0)
    with ngx.Graph(n, rp, col, w) as g:
        comps = g.scc()
        assert comps["number_components"] > 1
        got = g.apsp(per_source=True, hist_bins=128, hist_max=60.0, tile_ctas=tile_ctas)
        subset = np.arange(0, n, max(1, n // 40))
        rows = g.sssp_rows(subset, tile_ctas=tile_ctas)
        bc, _ = g.brandes(tile_ctas=tile_ctas)
        order = g.source_order()
    for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), (name, k)
    assert got.sum_distances == want["sum_distances"] and got.unreachable == want["unreachable"]
    assert got.diameter == want["diameter"] and got.cluster_sizes == want["cluster_sizes"]
    assert np.array_equal(got.hist, want["hist"]) and got.hist_overflow == want["hist_overflow"]
    for i, s in enumerate(subset):
        assert np.array_equal(rows[i], restatement.sssp(csr, int(s))), (name, s)
    want_bc = restatement.brandes(csr)
    floor = REL * max(1.0, float(np.abs(want_bc).mean()))
    assert np.all(np.abs(bc - want_bc) <= np.maximum(REL * np.abs(want_bc), floor)), name
    # each component's sources are contiguous in the all-sources order
    comp_of = comps["component"][order]
    changes = np.count_nonzero(comp_of[1:] != comp_of[:-1])
    assert changes == comps["number_components"] - 1, name
    assert np.array_equal(np.sort(order), np.arange(n))


def test_long_chain_runs_without_the_prepass(restatement):
    """A graph whose components need more passes than the pre-pass allows (a long path) runs without it."""
    n, rp, col, w = scc_family("path", 12000, 3)
    csr = oracle.Csr.from_arrays(n, rp, col, w)
    sources = np.arange(0, n, 97)
    with ngx.Graph(n, rp, col, w) as g:
        got = g.apsp(sources=sources, per_source=True)
    want = restatement.apsp(csr, sources=sources)
    for k in ("sum", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), k
