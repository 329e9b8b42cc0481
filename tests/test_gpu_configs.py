"""Parity at the sizes of the benchmark configurations, against the oracle (the CPU restatement pinned to the reference).

* Uneven batch (512 connectomes, N ~ U{500..20000}, degree ~ U[5, 60], 45 % integer / 45 % log-normal / 10 % unit
  weights): graphs drawn by the benchmark's own generator, one of each weight kind at small and mid degree and the two
  largest graphs of degree >= 50 (~19,500 vertices), run in one batch handle. Small graphs: every source's summaries
  bit for bit and betweenness within 1e-12 relative against the oracle's all-sources run. Large graphs: 64 seeded
  sources' summaries bit for bit against the oracle; betweenness of the whole graph equal bit for bit to the
  single-graph handle's all-sources run, whose betweenness on the same 64 sources is within 1e-12 of the oracle's.
* Adjoint (N=50,000, out-degree Poisson(40), log-normal(0, 0.5) weights): the gradient of CPL and efficiency over
  1024 seeded sources against central finite differences (h = 1e-6 w_e) on 200 seeded arcs that lie on shortest
  paths plus 50 uniformly drawn arcs, within 1e-6 relative; the numerators are differences of the exact sums of d and
  1/d (so no cancellation), the denominator the exact difference of the perturbed weights. And the full gradient of an
  N=2000 graph of the same generator against the oracle's CPU gradient within 1e-12 relative.
* Large (N=1e6, out-degree Poisson(40), kernel exp(-d/0.05), log-normal(0, 1)): 16 seeded sources' full distance
  rows, summaries and histogram bit for bit, and their betweenness within 1e-12 relative.
"""

from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

import bench
import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

REL = 1e-12


def _free_cache():
    try:
        import torch

        torch.cuda.empty_cache()
    except Exception:  # noqa: BLE001
        pass


def close(got, want, rel, label, floor_scale=None):
    scale = float(np.abs(want).mean()) if floor_scale is None else floor_scale
    floor = rel * max(1e-300, scale)
    bad = np.abs(got - want) > np.maximum(rel * np.abs(want), floor)
    assert not bad.any(), (label, np.nonzero(bad)[0][:5], got[bad][:5], want[bad][:5])


# ------------------------------------------------------------------------------------------------ uneven batch
SMALL = [424, 390, 156, 9, 504, 65]  # (n, degree, kind): int 615/7.7, 640/37.3; lognormal 584/58.8, 529/22.3; unit 899/51.9, 1534/47.2
LARGE = [361, 28]                    # int 19665/50.8, lognormal 19525/58.4


def test_uneven_batch_sample():
    specs = bench.uneven_batch_specs()
    for i in SMALL + LARGE:
        assert specs[i][0] >= 500
    assert all(specs[i][1] >= 50 and specs[i][0] > 19000 for i in LARGE)
    assert {specs[i][2] for i in SMALL} == {"int", "lognormal", "unit"}
    graphs = bench.uneven_batch_graphs(indices=SMALL + LARGE)
    _free_cache()
    hist_max = bench.UNEVEN_BATCH["hist_max"]
    with ngx.Batch(graphs) as b:
        results, bcs = b.run("brandes", hist_bins=1024, hist_max=hist_max, per_source=True)
    check = oracle.ParallelRestatement()
    for j, i in enumerate(SMALL):
        n, rp, col, w = graphs[j]
        csr = oracle.Csr.from_arrays(n, rp, col, w)
        want = check.apsp_sources(csr, np.arange(n), bins=1024, hist_max=hist_max)
        for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
            assert np.array_equal(results[j].per_source[k], want["per_source"][k]), (i, k)
        assert np.array_equal(results[j].hist, want["hist"]), i
        assert results[j].unreachable == want["unreachable"] and results[j].diameter == want["diameter"], i
        close(bcs[j], check.brandes_sources(csr, np.arange(n)), REL, ("bc", i), max(1.0, float(np.abs(bcs[j]).mean())))
    rng = np.random.default_rng(17)
    for j, i in enumerate(LARGE, start=len(SMALL)):
        n, rp, col, w = graphs[j]
        csr = oracle.Csr.from_arrays(n, rp, col, w)
        sample = rng.choice(n, size=64, replace=False)
        want = check.apsp_sources(csr, sample, bins=1024, hist_max=hist_max)
        for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
            assert np.array_equal(results[j].per_source[k][sample], want["per_source"][k]), (i, k)
        with ngx.Graph(n, rp, col, w) as g:
            bc_single, _ = g.brandes()
            bc_sample, _ = g.brandes(sources=sample)
        assert np.array_equal(bcs[j], bc_single), i
        want_bc = check.brandes_sources(csr, sample)
        close(bc_sample, want_bc, REL, ("bc sample", i), max(1.0, float(np.abs(want_bc).mean())))


# ------------------------------------------------------------------------------------------------ adjoint
def _exact_int(digits) -> int:
    """An exact accumulator (NGX_ACC_DIGITS words, word i a multiple of 2^(32 i + NGX_ACC_EXP0)) as an integer number
    of units 2^NGX_ACC_EXP0."""
    return sum(int(d) << (32 * i) for i, d in enumerate(np.asarray(digits, dtype=np.uint64).tolist()))


ACC_UNIT = Fraction(1, 2 ** 1088)  # 2^NGX_ACC_EXP0


@pytest.fixture(scope="module")
def adjoint_graph():
    c = synth.connectome(50_000, 40, 0.08, weights="lognormal", sigma=0.5, seed=2)
    _free_cache()
    return c


def test_adjoint_against_finite_differences(adjoint_graph):
    c = adjoint_graph
    rng = np.random.default_rng(41)
    sources = np.sort(rng.choice(c.n, size=1024, replace=False))
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        dcpl, deff, res = g.apsp_grad(sources=sources)
        on_paths = np.nonzero(dcpl > 0)[0]
        arcs = np.concatenate([rng.choice(on_paths, size=200, replace=False), rng.choice(c.m, size=50, replace=False)])
        fd_cpl = np.zeros(arcs.size)
        fd_eff = np.zeros(arcs.size)
        for j, e in enumerate(arcs):
            h = 1e-6 * c.w[e]
            sums = {}
            w = c.w.copy()
            for sign in (1, -1):
                w[e] = c.w[e] + sign * h
                g.update_weights(w)
                r = g.apsp(sources=sources, exact=True)
                assert r.reached_pairs == res.reached_pairs
                sums[sign] = (_exact_int(r.acc_digits[0]), _exact_int(r.acc_digits[1]), w[e])
            step = Fraction(sums[1][2]) - Fraction(sums[-1][2])  # the exact difference of the perturbed weights
            fd_cpl[j] = float((sums[1][0] - sums[-1][0]) * ACC_UNIT / step / res.reached_pairs)
            fd_eff[j] = float((sums[1][1] - sums[-1][1]) * ACC_UNIT / step / res.reached_pairs)
        g.update_weights(c.w)
    assert on_paths.size > 1000
    scale = float(np.abs(dcpl[arcs[:200]]).mean())
    close(dcpl[arcs], fd_cpl, 1e-6, "dcpl vs FD", scale)
    close(deff[arcs], fd_eff, 1e-6, "deff vs FD", float(np.abs(deff[arcs[:200]]).mean()))


def test_adjoint_against_cpu_gradient_on_2000_vertices():
    c = synth.connectome(2000, 40, 0.08, weights="lognormal", sigma=0.5, seed=3, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    want_cpl, want_eff, reached = oracle.ParallelRestatement().apsp_grad_sources(csr)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        dcpl, deff, res = g.apsp_grad()
    assert res.reached_pairs == reached
    close(dcpl, want_cpl, REL, "dcpl", float(np.abs(want_cpl).max()) * 1e-3)
    close(deff, want_eff, REL, "deff", float(np.abs(want_eff).max()) * 1e-3)


# ------------------------------------------------------------------------------------------------ large
@pytest.fixture(scope="module")
def large_graph():
    c = synth.connectome(1_000_000, 40, 0.05, weights="lognormal", sigma=1.0, seed=2)
    _free_cache()
    return c


def test_large_graph_sources(large_graph):
    c = large_graph
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    sample = np.random.default_rng(5).choice(c.n, size=16, replace=False)
    check = oracle.ParallelRestatement()
    want_rows = check.sssp_rows(csr, sample)
    want = check.apsp_sources(csr, sample, bins=1024, hist_max=4.0)
    want_bc = check.brandes_sources(csr, sample)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        rows = g.sssp_rows(sample)
        got = g.apsp(sources=sample, per_source=True, hist_bins=1024, hist_max=4.0)
        bc, _ = g.brandes(sources=sample)
    assert np.array_equal(rows, want_rows)
    for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), k
    assert np.array_equal(got.hist, want["hist"]) and got.hist_overflow == want["hist_overflow"]
    close(bc, want_bc, REL, "bc", max(1.0, float(np.abs(want_bc).mean())))
