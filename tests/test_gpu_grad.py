"""The adjoint kernel: gradient of CPL and of global efficiency with respect to every arc length.

Checked against the oracle's CPU gradient (1e-12 relative) and against central finite differences of the GPU's own
APSP (1e-6 relative, h = 1e-6 x w_e, numerators formed pair by pair from full distance rows to avoid cancellation),
on tie-free log-normal weights.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu


def close(got, want, rel, label):
    floor = rel * max(1e-300, float(np.abs(want).max()) if want.size else 1.0) * 1e-3
    bad = np.abs(got - want) > np.maximum(rel * np.abs(want), floor)
    assert not bad.any(), (label, np.nonzero(bad)[0][:5], got[bad][:5], want[bad][:5])


@pytest.mark.parametrize("n,deg,seed", [(300, 5, 1), (2000, 6, 2)])
def test_against_cpu_gradient(restatement, n, deg, seed):
    c = synth.connectome(n, deg, 0.15, weights="lognormal", sigma=0.5, seed=seed, use_gpu=False)
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    dcpl_w, deff_w, tot = restatement.apsp_grad(csr)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        dcpl, deff, res = gg.apsp_grad()
        dcpl2, deff2, _ = gg.apsp_grad()
    close(dcpl, dcpl_w, 1e-12, "dcpl")
    close(deff, deff_w, 1e-12, "deff")
    assert res.cpl == tot["cpl"] and res.efficiency == tot["efficiency"]
    assert np.array_equal(dcpl, dcpl2) and np.array_equal(deff, deff2)
    assert (dcpl >= 0).all() and (deff <= 0).all()


def test_against_finite_differences():
    c = synth.connectome(400, 6, 0.2, weights="lognormal", sigma=0.5, seed=7, use_gpu=False)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as gg:
        dcpl, deff, res = gg.apsp_grad()
    rng = np.random.default_rng(0)
    on_dag = np.nonzero(dcpl > 0)[0]
    arcs = rng.choice(on_dag, size=min(20, on_dag.size), replace=False)
    everything = np.arange(c.n)
    for e in arcs:
        h = 1e-6 * c.w[e]
        rows = {}
        for sign in (1, -1):
            w = c.w.copy()
            w[e] += sign * h
            with ngx.Graph(c.n, c.row_ptr, c.col, w) as gp:
                rows[sign] = gp.sssp_rows(everything)
        dp, dm = rows[1], rows[-1]
        fin = np.isfinite(dp) & (dp > 0)
        fd_cpl = float(np.sum(dp[fin] - dm[fin])) / (2 * h) / res.reached_pairs
        fd_eff = float(np.sum(1.0 / dp[fin] - 1.0 / dm[fin])) / (2 * h) / res.reached_pairs
        assert abs(dcpl[e] - fd_cpl) <= 1e-6 * abs(fd_cpl), (e, dcpl[e], fd_cpl)
        assert abs(deff[e] - fd_eff) <= 1e-6 * abs(fd_eff), (e, deff[e], fd_eff)


def test_autograd_function_matches_the_adjoint_and_finite_differences():
    """neurograph_b200.autograd: backward of (CPL, E) equals the adjoint outputs and a central finite difference."""
    import torch

    from neurograph_b200.autograd import apsp_metrics

    c = synth.connectome(300, 6, 0.2, weights="lognormal", seed=13, use_gpu=False)
    w = torch.tensor(c.w, dtype=torch.float64, requires_grad=True)
    out = apsp_metrics(w, c.n, c.row_ptr, c.col)
    (out[0] + 2.0 * out[1]).backward()
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        dcpl, deff, r = g.apsp_grad()
    assert out[0].item() == r.cpl and out[1].item() == r.efficiency
    want = dcpl + 2.0 * deff
    assert np.allclose(w.grad.numpy(), want, rtol=1e-12, atol=0.0)
    rng = np.random.default_rng(2)
    for e in rng.choice(c.m, size=5, replace=False):
        h = 1e-6 * c.w[e]
        vals = []
        for sign in (1.0, -1.0):
            wp = c.w.copy()
            wp[e] += sign * h
            o = apsp_metrics(torch.tensor(wp), c.n, c.row_ptr, c.col)
            vals.append(o[0].item() + 2.0 * o[1].item())
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - want[e]) <= 1e-4 * max(1e-12, abs(want[e])) + 1e-9, (e, fd, want[e])


def test_caller_output_arrays():
    """out= writes the gradients (and, for brandes, the betweenness) into the caller's arrays, page-locked ones
    included, with the same values as freshly allocated outputs; arrays of the wrong kind are refused."""
    import torch

    c = synth.connectome(600, 8, 0.2, weights="lognormal", seed=17, use_gpu=False)
    pinned = [torch.empty(c.m, dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        dcpl, deff, _ = g.apsp_grad()
        for _ in range(2):  # twice: the arrays are reused
            a, b, _ = g.apsp_grad(out=(pinned[0], pinned[1]))
            assert np.array_equal(a, dcpl) and np.array_equal(b, deff)
            assert a.ctypes.data == pinned[0].ctypes.data
        bc, _ = g.brandes()
        bc_out = np.full(c.n, -1.0)
        bc2, _ = g.brandes(out=bc_out)
        assert np.array_equal(bc2, bc) and bc2.ctypes.data == bc_out.ctypes.data
        for bad in (np.zeros(c.m, np.float32), np.zeros(c.m - 1), np.zeros((c.m, 2))[:, 0]):
            with pytest.raises(ValueError):
                g.apsp_grad(out=(bad, pinned[2]))
        with pytest.raises(ValueError):
            g.brandes(out=bc_out, fixed=True)
