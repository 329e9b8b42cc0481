"""Brandes betweenness on the GPU (through the C ABI) against the reference's per-node values and the oracle.

Tolerance: 1e-12 relative per vertex, with an absolute floor of 1e-12 x the mean betweenness for vertices whose
value is (near) zero. The GPU sums in a different (fixed, deterministic) order than the reference's heap order.
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


def test_reference_fixtures(golden, expectations):
    for name, g in golden.items():
        bc_ref = g.get("brandes/bc")
        if bc_ref is None:
            continue
        with ngx.Graph(g.n, g.row_ptr, g.col, g.w) as gg:
            bc, res = gg.brandes()
            apsp = gg.apsp()
        assert_bc_close(bc, bc_ref, name)
        avg_ref = g.get("brandes/average")[0]
        assert abs(bc.sum() / g.n - avg_ref) <= REL * max(1.0, abs(avg_ref)), name
        # the fused APSP summaries of the Brandes run are the APSP run's, bit for bit
        assert res.cpl == apsp.cpl and res.efficiency == apsp.efficiency and res.diameter == apsp.diameter, name
    for case in expectations["brandes_average"]:
        g = golden[case["fixture"]]
        with ngx.Graph(g.n, g.row_ptr, g.col, g.w) as gg:
            bc, _ = gg.brandes()
        assert abs(bc.sum() / g.n - case["value"]) <= case["tol"], case["cite"]


def test_sample_input_all_sources(golden):
    g = golden["sample_5000"]
    with ngx.Graph(g.n, g.row_ptr, g.col, g.w) as gg:
        bc, _ = gg.brandes()
    assert_bc_close(bc, g.get("brandes/bc"), "sample_5000")


@pytest.mark.parametrize("weights,seed", [("int", 1), ("int", 2), ("lognormal", 3), ("unit", 4)])
def test_synthetic_against_oracle(restatement, weights, seed):
    c = synth.connectome(900, 8, 0.2, weights=weights, seed=seed, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    want = restatement.brandes(csr)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, _ = gg.brandes()
        bc2, _ = gg.brandes()
        subset = np.arange(5, 900, 11)
        bc_sub, _ = gg.brandes(sources=subset)
    assert_bc_close(bc, want, weights)
    assert np.array_equal(bc, bc2)  # deterministic: fixed-order sums, order-free fixed-point accumulation
    assert_bc_close(bc_sub, restatement.brandes(csr, sources=subset), "subset")


def test_many_ties_and_unreachable(restatement):
    """Unit weights on a sparse random graph: many equal-length paths (sigma > 1) and many unreachable pairs."""
    c = synth.random_graph(600, 1.6, weights="unit", seed=8)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, res = gg.brandes()
    assert_bc_close(bc, restatement.brandes(csr), "ties")
    assert res.unreachable > 0


def test_inverse_metric_is_rejected():
    c = synth.random_graph(50, 3, seed=1)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        opts, _, _ = gg._opts(None, "inverse", "batched", 0.0, 0, 0.0, 0, 0, 0)
        bc = np.zeros(c.n)
        r = ngx._Result()
        import ctypes as C

        assert ngx.library().ngx_brandes(gg._handle, C.byref(opts), bc.ctypes.data, C.byref(r)) == 6


def test_path_counts_beyond_2_53_use_the_pull_form(restatement):
    """A chain of 70 diamonds has 2^70 shortest paths: the atomic sigma push can no longer be exact, so the run must
    fall back to the order-defined pull form and still agree with the oracle."""
    diamonds = 70
    n = 3 * diamonds + 1
    src, dst = [], []
    for i in range(diamonds):
        hub, a, b, nxt = 3 * i, 3 * i + 1, 3 * i + 2, 3 * i + 3
        src += [hub, hub, a, b]
        dst += [a, b, nxt, nxt]
    order = np.lexsort((dst, src))
    src, dst = np.array(src)[order], np.array(dst)[order]
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, src + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    w = np.ones(src.size)
    csr = oracle.Csr.from_arrays(n, row_ptr, dst, w)
    with ngx.Graph(n, row_ptr, dst, w) as gg:
        bc, _ = gg.brandes()
        bc2, _ = gg.brandes()
    assert_bc_close(bc, restatement.brandes(csr), "diamonds")
    assert np.array_equal(bc, bc2)


def test_dense_ties_use_the_arc_scanning_passes(restatement):
    """Unit weights on a dense graph give many equal-length predecessors: the DAG overflows the successor lists and
    the arc-scanning passes run; results still match the oracle."""
    c = synth.random_graph(300, 40, weights="unit", seed=12)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, res = gg.brandes()
        dcpl, deff, _ = gg.apsp_grad()
    assert res.dag_scan_tiles > 0
    assert_bc_close(bc, restatement.brandes(csr), "dense ties")
    want_cpl, want_eff, _ = restatement.apsp_grad(csr)
    assert np.allclose(dcpl, want_cpl, rtol=1e-12, atol=1e-15) and np.allclose(deff, want_eff, rtol=1e-12, atol=1e-15)


def test_sparse_graphs_use_the_successor_lists(restatement):
    c = synth.connectome(1200, 10, 0.2, weights="lognormal", seed=13, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        bc, res = gg.brandes()
    assert res.dag_scan_tiles == 0
    assert_bc_close(bc, restatement.brandes(csr), "lists")
