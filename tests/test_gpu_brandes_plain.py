"""The plain per-source Brandes form (one source per CTA, ``mode="plain"``) against the reference fixtures and the
oracle.

It is the baseline the batched form is compared with, so it must compute the same outputs: the same betweenness
(1e-12 relative, with an absolute floor of 1e-12 x the mean for (near) zero values; its dependency sums run in
another fixed order than the batched form's) and the same fused APSP summaries and histogram, bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

REL = 1e-12


def assert_bc_close(got, want, label=""):
    floor = REL * max(1.0, float(np.abs(want).mean()) if want.size else 1.0)
    err = np.abs(got - want)
    bad = err > np.maximum(REL * np.abs(want), floor)
    assert not bad.any(), (label, np.nonzero(bad)[0][:5], got[bad][:5], want[bad][:5])


def test_reference_fixtures(golden):
    for name, g in golden.items():
        bc_ref = g.get("brandes/bc")
        if bc_ref is None:
            continue
        with ngx.Graph(g.n, g.row_ptr, g.col, g.w) as gg:
            bc, res = gg.brandes(mode="plain", hist_bins=64, hist_max=64.0)
            _, batched = gg.brandes(hist_bins=64, hist_max=64.0)
        assert_bc_close(bc, bc_ref, name)
        assert res.cpl == batched.cpl and res.efficiency == batched.efficiency and res.diameter == batched.diameter, name
        assert np.array_equal(res.hist, batched.hist), name


@pytest.mark.parametrize("weights,seed", [("int", 21), ("lognormal", 22), ("unit", 23)])
def test_synthetic_against_oracle_and_batched(restatement, weights, seed):
    c = synth.connectome(800, 9, 0.2, weights=weights, seed=seed, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    subset = np.arange(3, 800, 7)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, res = gg.brandes(mode="plain")
        bc2, _ = gg.brandes(mode="plain")
        bc_batched, res_batched = gg.brandes()
        bc_sub, _ = gg.brandes(sources=subset, mode="plain", per_source=True)
    assert_bc_close(bc, restatement.brandes(csr), weights)
    assert_bc_close(bc, bc_batched, "plain vs batched")
    assert np.array_equal(bc, bc2)  # deterministic
    assert res.cpl == res_batched.cpl and res.efficiency == res_batched.efficiency
    assert res.traversed_arcs == res_batched.traversed_arcs and res.reached_pairs == res_batched.reached_pairs
    assert_bc_close(bc_sub, restatement.brandes(csr, sources=subset), "subset")


def test_ties_and_unreachable(restatement):
    """Unit weights on a sparse random graph: equal-length paths (sigma > 1) and unreachable pairs."""
    c = synth.random_graph(500, 1.8, weights="unit", seed=31)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, res = gg.brandes(mode="plain")
    assert_bc_close(bc, restatement.brandes(csr), "ties")
    assert res.unreachable > 0


def test_dense_ties(restatement):
    c = synth.random_graph(250, 30, weights="unit", seed=32)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, _ = gg.brandes(mode="plain")
    assert_bc_close(bc, restatement.brandes(csr), "dense ties")


def test_edge_cases():
    # one vertex, no arcs
    with ngx.Graph(1, np.zeros(2, np.int64), np.zeros(0, np.int32), np.zeros(0)) as gg:
        bc, res = gg.brandes(mode="plain")
    assert bc.tolist() == [0.0] and res.reached_pairs == 0
    # a path 0 -> 1 -> 2: only the middle vertex lies between a pair
    with ngx.Graph(3, np.array([0, 1, 2, 2], np.int64), np.array([1, 2], np.int32), np.array([1.0, 2.0])) as gg:
        bc, _ = gg.brandes(mode="plain")
    assert bc.tolist() == [0.0, 1.0, 0.0]
