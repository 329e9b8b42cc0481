"""Batches of uneven graphs in one handle and one persistent launch (through the C ABI).

Every graph of a batch must give exactly what a single-graph handle and the oracle give: APSP summaries and
per-source outputs bit for bit, histogram counts bit for bit, betweenness and gradients within 1e-12 relative (the
fixed-point sums are order-free, so they also equal the single-graph run's bit for bit). Replays of a captured run,
in-place weight updates and the bucket-width autotuner must not change any result.
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

REL = 1e-12


def uneven_batch(count=18, seed=0):
    """Connectomes and random graphs from 1 to ~1500 vertices, integer, lognormal and unit weights."""
    rng = np.random.default_rng(seed)
    graphs = []
    kinds = ["int", "lognormal", "unit"]
    for i in range(count):
        n = int(rng.choice([1, 2, 7, 40, 150, 333, 700, 1500])) if i > 1 else [1500, 1][i]
        kind = kinds[i % 3]
        if i % 4 == 3:
            c = synth.random_graph(n, 3, weights=kind, seed=seed * 100 + i)
        else:
            c = synth.connectome(n, 6, 0.2, weights=kind, seed=seed * 100 + i, use_gpu=False)
        graphs.append((c.n, c.row_ptr, c.col, c.w))
    return graphs


def close(got, want, label):
    floor = REL * max(1.0, float(np.abs(want).mean()) if want.size else 1.0)
    bad = np.abs(got - want) > np.maximum(REL * np.abs(want), floor)
    assert not bad.any(), (label, np.nonzero(bad)[0][:5], got[bad][:5], want[bad][:5])


def same_summary(a: ngx.ApspResult, b, label):
    if isinstance(b, dict):
        keys = ("sum_distances", "sum_inverse", "diameter", "unreachable", "reached_pairs", "traversed_arcs")
        for k in keys:
            assert getattr(a, k) == b[k], (label, k, getattr(a, k), b[k])
        if b["reached_pairs"] > 0:
            assert a.cpl == b["cpl"] and a.efficiency == b["efficiency"], label
        assert a.cluster_sizes == b["cluster_sizes"], label
    else:
        for k in ("sum_distances", "sum_inverse", "diameter", "unreachable", "reached_pairs", "traversed_arcs", "cpl", "efficiency"):
            x, y = getattr(a, k), getattr(b, k)
            assert x == y or (x != x and y != y), (label, k, x, y)  # a graph without reached pairs has NaN averages


@pytest.mark.parametrize("metric", ["regular", "inverse"])
def test_batch_apsp_matches_oracle(restatement, metric):
    graphs = uneven_batch(18, seed=1)
    m = oracle.METRIC_INVERSE if metric == "inverse" else oracle.METRIC_REGULAR
    with ngx.Batch(graphs) as b:
        results, _ = b.run("apsp", metric=metric, hist_bins=256, hist_max=32.0, per_source=True)
    for i, (n, rp, c, w) in enumerate(graphs):
        want = restatement.apsp(oracle.Csr.from_arrays(n, rp, c, w), metric=m, bins=256, hist_max=32.0)
        got = results[i]
        same_summary(got, want, i)
        ws = want["per_source"]
        for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
            assert np.array_equal(got.per_source[k], ws[k]), (i, k)
        assert np.array_equal(got.hist, want["hist"]), i
        assert got.hist_overflow == want["hist_overflow"], i


def test_batch_equals_single_graph_handles():
    graphs = uneven_batch(12, seed=2)
    with ngx.Batch(graphs) as b:
        results, _ = b.run("apsp")
    for i, (n, rp, c, w) in enumerate(graphs):
        with ngx.Graph(n, rp, c, w) as g:
            same_summary(results[i], g.apsp(), i)


def test_batch_brandes_and_gradient(restatement):
    graphs = uneven_batch(10, seed=3)
    with ngx.Batch(graphs) as b:
        res_b, bcs = b.run("brandes")
        res_g, grads = b.run("grad")
        res_a, _ = b.run("apsp")
    for i, (n, rp, c, w) in enumerate(graphs):
        csr = oracle.Csr.from_arrays(n, rp, c, w)
        close(bcs[i], restatement.brandes(csr), f"bc {i}")
        want_cpl, want_eff = restatement.apsp_grad(csr)[:2]
        close(grads[i][0], want_cpl, f"dcpl {i}")
        close(grads[i][1], want_eff, f"deff {i}")
        same_summary(res_b[i], res_a[i], i)
        same_summary(res_g[i], res_a[i], i)
        with ngx.Graph(n, rp, c, w) as g:
            bc_single, _ = g.brandes()
        assert np.array_equal(bcs[i], bc_single), i  # fixed-point sums: the same bits whatever the tile schedule


def test_cuda_graph_replay_is_identical():
    graphs = uneven_batch(14, seed=4)
    with ngx.Batch(graphs) as b:
        base, _ = b.run("apsp", hist_bins=64, hist_max=16.0, per_source=True)
        for _ in range(3):  # first call launches and captures, the next ones replay
            again, _ = b.run("apsp", hist_bins=64, hist_max=16.0, per_source=True, use_cuda_graph=True)
            for i in range(len(graphs)):
                same_summary(again[i], base[i], i)
                assert np.array_equal(again[i].hist, base[i].hist)
                assert np.array_equal(again[i].per_source["sum"], base[i].per_source["sum"])
        bc0, bcs0 = b.run("brandes")
        for _ in range(2):
            bc1, bcs1 = b.run("brandes", use_cuda_graph=True)
            for i in range(len(graphs)):
                assert np.array_equal(bcs1[i], bcs0[i]), i


def test_update_weights_equals_a_fresh_handle(restatement):
    graphs = uneven_batch(8, seed=5)
    rng = np.random.default_rng(7)
    new_w = []
    for n, rp, c, w in graphs:
        nw = np.where(w != 0, rng.integers(1, 50, size=w.size).astype(np.float64), 0.0)
        new_w.append(nw)
    with ngx.Batch(graphs) as b:
        b.run("apsp", use_cuda_graph=True)
        b.update_weights(new_w)
        got, _ = b.run("apsp", use_cuda_graph=True)  # the captured run reads the arcs in place
        got_bc, bcs = b.run("brandes")
    fresh = [(n, rp, c, nw) for (n, rp, c, _), nw in zip(graphs, new_w)]
    with ngx.Batch(fresh) as f:
        want, _ = f.run("apsp")
        _, want_bcs = f.run("brandes")
    for i in range(len(graphs)):
        same_summary(got[i], want[i], i)
        assert np.array_equal(bcs[i], want_bcs[i]), i
    # a zero weight may not become non-zero (that would change the arc set)
    n, rp, c, w = graphs[0]
    bad = [x.copy() for x in new_w]
    if (w == 0).any():
        bad[0][np.nonzero(w == 0)[0][0]] = 1.0
    else:
        bad[0][0] = 0.0
    with ngx.Batch(graphs) as b:
        with pytest.raises(ngx.NgxError):
            b.update_weights(bad)


def test_single_graph_update_weights(restatement):
    c = synth.connectome(600, 8, 0.2, weights="lognormal", seed=11, use_gpu=False)
    w2 = c.w * np.random.default_rng(3).uniform(0.5, 2.0, size=c.w.size)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        g.apsp()
        g.update_weights(w2)
        got = g.apsp(per_source=True)
        dcpl, deff, _ = g.apsp_grad()
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, w2)
    want = restatement.apsp(csr)
    same_summary(got, want, "updated")
    want_cpl, want_eff = restatement.apsp_grad(csr)[:2]
    close(dcpl, want_cpl, "dcpl")
    close(deff, want_eff, "deff")


def test_autotune_keeps_results():
    graphs = uneven_batch(16, seed=6)
    with ngx.Batch(graphs) as b:
        before, _ = b.run("apsp")
        scales = b.autotune("apsp")
        shape = b.tuning("apsp")
        after, _ = b.run("apsp")
    # one launch shape for the whole batch
    assert (shape["block_threads"], shape["ctas_per_sm"]) in ((512, 2), (384, 2), (256, 3), (256, 4)), shape
    # 0: the library's own group rule won the trials
    assert shape["tile_ctas"] in (0, 1, 2, 4) and shape["trials"] == 7 and shape["gteps"] > 0, shape
    classes = {int(np.floor(np.log2(n))) for n, *_ in graphs if n > 0}
    for c in range(ngx.SIZE_CLASSES):
        if c in classes:
            # a fixed multiple of the mean arc length, or the class's default width (2 / sqrt(mean out-degree))
            assert 0.125 <= scales[c] <= 4.0, (c, scales[c])
        else:
            assert scales[c] == 0.0
    for i in range(len(graphs)):
        same_summary(after[i], before[i], i)


def test_single_graph_entry_points_reject_batches():
    graphs = uneven_batch(3, seed=8)
    with ngx.Batch(graphs) as b:
        g = ngx.Graph.__new__(ngx.Graph)
        g._handle, g.n, g.m = b._handle, sum(b.ns), sum(b.ms)
        with pytest.raises(ngx.NgxError):
            g.apsp()
        g._handle = None
