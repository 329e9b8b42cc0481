"""ngx_graph_autotune on a single-graph handle: the tuned bucket width, block shape and CTAs per tile are valid, are
used by later runs that leave those options at 0, and change no result (distances are the unique fixed point, sums are
exact, betweenness and gradients are fixed-point sums): every output equals the untuned run bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu

SHAPES = ((512, 2), (384, 2), (256, 3), (256, 4))


@pytest.fixture(scope="module")
def graph():
    return synth.connectome(8000, 30, 0.1, weights="lognormal", seed=71, use_gpu=False)


def test_autotune_apsp_keeps_results(graph):
    c = graph
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        before = g.apsp(per_source=True, hist_bins=256, hist_max=20.0)
        t = g.autotune("apsp", sample_sources=2048)
        after = g.apsp(per_source=True, hist_bins=256, hist_max=20.0)
        g_arcs = int(g.layout()["row_ptr"][-1])  # stored arcs
    # a fixed multiple of the mean arc length, or the graph's default width 2 / sqrt(mean out-degree)
    default_scale = min(2.0, max(0.125, 2.0 / np.sqrt(max(1.0, g_arcs / c.n))))
    assert t["delta_scale"] in (0.125, 0.25, 0.5, 1.0, 2.0) or abs(t["delta_scale"] - default_scale) < 1e-12, t
    assert (t["block_threads"], t["ctas_per_sm"]) in SHAPES, t
    assert t["tile_ctas"] >= 0 and t["trials"] >= 8 and t["gteps"] > 0, t  # 0: the library's own choice
    for k in ("sum_distances", "sum_inverse", "diameter", "unreachable", "reached_pairs", "traversed_arcs", "hist_overflow"):
        assert getattr(before, k) == getattr(after, k), k
    assert np.array_equal(before.hist, after.hist)
    for k, v in before.per_source.items():
        assert np.array_equal(v, after.per_source[k]), k


def test_autotune_brandes_and_gradient_keep_results(graph):
    c = graph
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        bc0, _ = g.brandes()
        d0, e0, _ = g.apsp_grad()
        tb = g.autotune("brandes", sample_sources=1024)
        tg = g.autotune("grad", sample_sources=1024)
        bc1, _ = g.brandes()
        d1, e1, _ = g.apsp_grad()
    assert (tb["block_threads"], tb["ctas_per_sm"]) in SHAPES and (tg["block_threads"], tg["ctas_per_sm"]) in SHAPES
    assert np.array_equal(bc0, bc1)
    assert np.array_equal(d0, d1) and np.array_equal(e0, e1)
