"""Source tiles worked by groups of CTAs (opts.tile_ctas) must give exactly what one CTA per tile gives.

Every output is exact or order-free (integer counts, exactly rounded sums, fixed-point betweenness and gradients,
distances as the unique fixed point), so for every group size the APSP summaries, per-source outputs, histogram,
distance rows, betweenness and both gradients must equal the single-CTA run bit for bit; one case is also checked
against the oracle. Group sizes cover 2, odd sizes, sizes that do not divide the resident CTA count, and groups
larger than the number of tiles; the batch path (one cooperative launch over many graphs, replayed from a captured CUDA
graph) and the abort flag are checked with groups too.
"""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

GROUPS = [2, 3, 7, 37, 148]


def same_result(a, b, label):
    for k in ("sum_distances", "sum_inverse", "diameter", "unreachable", "reached_pairs", "traversed_arcs", "hist_overflow"):
        x, y = getattr(a, k), getattr(b, k)
        assert x == y, (label, k, x, y)
    if b.hist is not None:
        assert np.array_equal(a.hist, b.hist), label
    if b.per_source is not None:
        for k, v in b.per_source.items():
            assert np.array_equal(a.per_source[k], v), (label, k)


@pytest.fixture(scope="module")
def graphs():
    return {
        "lognormal": synth.connectome(6000, 20, 0.1, weights="lognormal", seed=51, use_gpu=False),
        "int": synth.connectome(4000, 12, 0.12, weights="int", seed=52, use_gpu=False),
        "sparse": synth.random_graph(5000, 1.2, weights="lognormal", seed=53),
    }


@pytest.mark.parametrize("kind", ["lognormal", "int", "sparse"])
def test_apsp_rows_and_summaries_with_groups(graphs, kind):
    c = graphs[kind]
    sources = np.random.default_rng(1).choice(c.n, size=700, replace=False)
    kw = dict(sources=sources, per_source=True, hist_bins=512, hist_max=40.0)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        want = g.apsp(tile_ctas=1, **kw)
        want_rows = g.sssp_rows(sources[:70], tile_ctas=1)
        for gs in GROUPS:
            same_result(g.apsp(tile_ctas=gs, **kw), want, (kind, gs))
            assert np.array_equal(g.sssp_rows(sources[:70], tile_ctas=gs), want_rows), (kind, gs)
        inv = g.apsp(metric="inverse", tile_ctas=1, **kw)
        same_result(g.apsp(metric="inverse", tile_ctas=5, **kw), inv, (kind, "inverse"))


@pytest.mark.parametrize("kind", ["lognormal", "int"])
def test_betweenness_and_gradients_with_groups(graphs, kind):
    c = graphs[kind]
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        bc1, r1 = g.brandes(tile_ctas=1, per_source=True)
        dcpl1, deff1, _ = g.apsp_grad(tile_ctas=1)
        for gs in (2, 7, 37):
            bc, r = g.brandes(tile_ctas=gs, per_source=True)
            assert np.array_equal(bc, bc1), (kind, gs)
            same_result(r, r1, (kind, "brandes", gs))
            dcpl, deff, _ = g.apsp_grad(tile_ctas=gs)
            assert np.array_equal(dcpl, dcpl1) and np.array_equal(deff, deff1), (kind, gs)


def test_groups_against_the_oracle(graphs, restatement):
    c = graphs["lognormal"]
    csr = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    sources = np.arange(0, c.n, 37)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        got = g.apsp(sources=sources, per_source=True, hist_bins=256, hist_max=30.0, tile_ctas=11)
        bc, _ = g.brandes(sources=sources, tile_ctas=11)
    want = restatement.apsp(csr, sources=sources, bins=256, hist_max=30.0)
    for k in ("sum", "sum_inv", "max", "unreachable", "arcs"):
        assert np.array_equal(got.per_source[k], want["per_source"][k]), k
    assert np.array_equal(got.hist, want["hist"])
    want_bc = restatement.brandes(csr, sources=sources)
    floor = 1e-12 * max(1.0, float(np.abs(want_bc).mean()))
    assert np.all(np.abs(bc - want_bc) <= np.maximum(1e-12 * np.abs(want_bc), floor))


def test_batch_with_groups_and_replay():
    rng = np.random.default_rng(4)
    gl = []
    for i in range(9):
        n = int(rng.choice([1, 40, 333, 1500]))
        c = synth.connectome(n, 6, 0.2, weights=["int", "lognormal", "unit"][i % 3], seed=60 + i, use_gpu=False)
        gl.append((c.n, c.row_ptr, c.col, c.w))
    with ngx.Batch(gl) as b:
        want, want_bc = b.run("brandes", hist_bins=128, hist_max=40.0, per_source=True, tile_ctas=1)
        for _ in range(2):  # capture, then replay
            got, got_bc = b.run("brandes", hist_bins=128, hist_max=40.0, per_source=True, tile_ctas=6, use_cuda_graph=True)
            for i in range(len(gl)):
                same_result(got[i], want[i], ("batch", i))
                assert np.array_equal(got_bc[i], want_bc[i]), i


def test_abort_with_groups():
    c = synth.connectome(30000, 30, 0.08, weights="lognormal", seed=54)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        box = {}

        def run():
            try:
                g.apsp(tile_ctas=8)
                box["error"] = None
            except ngx.NgxError as e:
                box["error"] = e

        th = threading.Thread(target=run)
        th.start()
        time.sleep(0.02)
        while th.is_alive():
            g.request_abort()
            th.join(0.005)
        assert box["error"] is not None and box["error"].status == 5  # NGX_ABORTED
        sources = np.arange(64)
        same_result(g.apsp(sources=sources, per_source=True, tile_ctas=8), g.apsp(sources=sources, per_source=True, tile_ctas=1), "after abort")


def test_tile_ctas_out_of_range_is_rejected(graphs):
    c = graphs["int"]
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        with pytest.raises(ngx.NgxError):
            g.apsp(tile_ctas=513)
        with pytest.raises(ngx.NgxError):
            g.apsp(tile_ctas=-1)
