"""Diameter approximation (host part, no GPU): the contracted graph of ngx_diameter_contract, whose exact diameter
(computed here by the oracle) plus 2r is the approximation.

Pinned by the golden values written in the reference's own tests (tests/diameter_approximation/
test_diameter_approximation.cpp: all centres give the exact diameter + 2r, a single centre on node 0 collapses the
standard graphs) and, where the reference build is here, by the reference's DiameterApproximation itself on its
fixture graphs and on random integer-weight connectomes, with replayed draws and with std::mt19937 seeds. Exact
equality: the approximation is an integer.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

# (fixture, r, draws, value, test_diameter_approximation.cpp line)
GOLDEN = [
    ("standard", 2, [0.0], 11, 70), ("standard_uu", 1, [0.0], 5, 85), ("full", 2, [0.0], 5, 100),
    ("standard_four_rank_on_one_rank", 2, [0.0], 44, 115), ("standard_uu_four_rank_on_one_rank", 2, [0.0], 9, 130),
    ("full_four_rank_on_one_rank", 2, [0.0], 5, 145), ("standard", 2, [0.0, 1.0], 4, 160),
    ("standard_uu", 1, [0.0, 1.0], 2, 175), ("standard_seven_rank_on_one_rank", 2, [0.0], 44, 270),
]


def approximation(restatement, n, row_ptr, col, w, r, draws=None, seed=0):
    cn, crp, cc, cw = ngx.diameter_contract(n, row_ptr, col, w, r, draws=draws, seed=seed)
    return int(restatement.apsp(oracle.Csr.from_arrays(cn, crp, cc, cw))["diameter"]) + 2 * r


@pytest.mark.parametrize("name,r,draws,value,line", GOLDEN, ids=[f"{g[0]}-r{g[1]}-{len(g[2])}" for g in GOLDEN])
def test_reference_golden_values(golden, restatement, name, r, draws, value, line):
    g = golden[name]
    assert approximation(restatement, g.n, g.row_ptr, g.col, g.w, r, draws=draws) == value, f"test_diameter_approximation.cpp:{line}"


def test_all_centres_is_the_exact_diameter(restatement):
    c = synth.connectome(300, 5, 0.2, weights="int", seed=4, use_gpu=False)
    exact = int(restatement.apsp(oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w))["diameter"])
    cn, crp, cc, cw = ngx.diameter_contract(c.n, c.row_ptr, c.col, c.w, 3, draws=[0.0])
    assert cn == c.n  # every vertex its own centre: the contracted graph is the graph
    assert approximation(restatement, c.n, c.row_ptr, c.col, c.w, 3, draws=[0.0]) == exact + 6


def test_invalid_inputs():
    with pytest.raises(ngx.NgxError, match="positive integers"):
        ngx.diameter_contract(2, [0, 1, 1], [1], [1.5], 1)
    with pytest.raises(ngx.NgxError, match="no vertices"):
        ngx.diameter_contract(0, [0], [], [], 1)
    with pytest.raises(ngx.NgxError, match="not reached"):  # one vertex: no iteration draws a centre
        ngx.diameter_contract(1, [0, 0], [], [], 1)


def _agree(restatement, g, n, rp, c, w, r, draws, seed):
    """The reference's approximation, or its failure (a vertex no centre reached), must be ours too."""
    try:
        want = g.diameter_approximation(r, draws=draws, seed=seed)
    except Exception:  # noqa: BLE001
        with pytest.raises(ngx.NgxError):
            approximation(restatement, n, rp, c, w, r, draws=draws, seed=seed)
        return 0
    assert approximation(restatement, n, rp, c, w, r, draws=draws, seed=seed) == want, (r, draws, seed)
    return 1


def test_against_the_reference(restatement):
    if not oracle.Reference.available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    ref = oracle.Reference()
    names = ref.fixture_names()
    for i, name in enumerate(names):
        if name in ("empty", "negative_weight"):  # the reference loops without end on 0 vertices; negative weights throw
            continue
        g = ref.fixture_graph(i)
        n, rp, c, w = g.csr()
        for r in (1, 2, 3):
            for draws, seed in (([0.0], 0), ([0.0, 1.0], 0), (None, 0), (None, 7)):
                _agree(restatement, g, n, rp, c, w.astype(np.float64), r, draws, seed)
    agreed_values = 0
    for s in range(6):
        n, rp, c, w = symmetric_graph(200 + 40 * s, 4 + s, seed=50 + s)
        g = ref.graph(n, rp, c, w.astype(np.int32))
        n, rp, c, w = g.csr()  # the reference's stored arc order: the last arc of a centre pair wins
        for r in (1, 2, 4):
            for seed in (0, 3):
                agreed_values += _agree(restatement, g, n, rp, c, w.astype(np.float64), r, None, seed)
    assert agreed_values >= 24  # most cases reach every vertex, so values (not just failures) are compared


def test_against_the_reference_on_larger_graphs(restatement):
    """Thousands of vertices: growing steps of many rounds, where the rounds after the first hear only the vertices the
    round before changed."""
    if not oracle.Reference.available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    ref = oracle.Reference()
    agreed_values = 0
    for n, degree, seed in ((3000, 4, 5), (6000, 8, 3)):
        n, rp, c, w = symmetric_graph(n, degree, seed=seed)
        g = ref.graph(n, rp, c, w.astype(np.int32))
        n, rp, c, w = g.csr()
        for r in (1, 2, 3):
            for s in (1, 2, 3):
                agreed_values += _agree(restatement, g, n, rp, c, w.astype(np.float64), r, None, s)
    assert agreed_values >= 12


def symmetric_graph(n, degree, seed):
    """A connectome with every arc mirrored and weights 1..3, so that balls can reach every vertex."""
    cg = synth.connectome(n, degree, 0.2, weights="int", seed=seed, use_gpu=False)
    u = np.repeat(np.arange(cg.n), np.diff(cg.row_ptr))
    src = np.concatenate([u, cg.col.astype(np.int64)])
    dst = np.concatenate([cg.col.astype(np.int64), u])
    key, first = np.unique(src * n + dst, return_index=True)
    w = 1 + (np.concatenate([cg.w, cg.w]).astype(np.int64)[first] % 3)
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, key // n + 1, 1)
    return n, np.cumsum(row_ptr), (key % n).astype(np.int32), w.astype(np.float64)
