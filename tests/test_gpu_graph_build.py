"""The device build of a graph handle against the host build (through the C ABI).

ngx_graph_create builds a single graph's CSR and reverse CSR with device kernels (checks, zero weights dropped, both
arc lengths, a stable device sort by target); ngx_graph_create_ex(NGX_BUILD_ON_HOST) builds them on host threads.
Every device array must be identical bit for bit (the same stored order, lengths, in-arc order within a target), the
mean lengths that set the default bucket widths too, and so must every result and every error message. Cases: the
benchmark's connectome family, signed / zero / repeated / self arcs, empty rows, isolated vertices, one vertex, no
arcs, and bad arcs (out-of-range target, NaN, infinite weight).
"""

from __future__ import annotations

import numpy as np
import pytest

import neurograph_b200 as ngx
from neurograph_b200 import synth

pytestmark = pytest.mark.gpu


def _signed_mixed(seed):
    rng = np.random.default_rng(seed)
    c = synth.random_graph(3000, 6, weights="int", seed=seed, self_loops=True)
    w = c.w * rng.choice([-1.0, 1.0], size=c.m)
    w[rng.random(c.m) < 0.1] = 0.0  # zero weights: absent arcs
    # repeated arcs: duplicate a few rows' first arc (the caller's CSR may hold them)
    rows = [c.col[c.row_ptr[u]:c.row_ptr[u + 1]].tolist() for u in range(c.n)]
    ws = [w[c.row_ptr[u]:c.row_ptr[u + 1]].tolist() for u in range(c.n)]
    for u in range(0, c.n, 97):
        if rows[u]:
            rows[u].append(rows[u][0])
            ws[u].append(ws[u][0] + 1.0)
    rows[5], ws[5] = [], []  # an empty row
    row_ptr = np.zeros(c.n + 1, np.int64)
    row_ptr[1:] = np.cumsum([len(r) for r in rows])
    return c.n, row_ptr, np.array([x for r in rows for x in r], np.int32), np.array([x for r in ws for x in r], np.float64)


CASES = {
    "connectome": lambda: (lambda c: (c.n, c.row_ptr, c.col, c.w))(synth.connectome(20000, 40, 0.08, weights="lognormal", seed=3)),
    "signed zero repeated self": lambda: _signed_mixed(4),
    "isolated vertices": lambda: (lambda c: (c.n, c.row_ptr, c.col, c.w))(synth.random_graph(5000, 0.3, weights="lognormal", seed=5)),
    "one vertex with a self arc": lambda: (1, np.array([0, 1], np.int64), np.array([0], np.int32), np.array([2.5])),
    "no arcs": lambda: (7, np.zeros(8, np.int64), np.zeros(0, np.int32), np.zeros(0)),
    "all zero weights": lambda: (3, np.array([0, 2, 3, 3], np.int64), np.array([1, 2, 0], np.int32), np.zeros(3)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_build_equals_host_build(name):
    n, rp, col, w = CASES[name]()
    with ngx.Graph(n, rp, col, w, build="device") as gd, ngx.Graph(n, rp, col, w, build="host") as gh:
        a, b = gd.layout(), gh.layout()
        for k in ("row_ptr", "rrow_ptr", "arc_src", "mean_lengths"):
            assert np.array_equal(a[k], b[k]), (name, k)
        for k in ("arcs", "arcs_inverse", "rarcs"):
            assert a[k].tobytes() == b[k].tobytes(), (name, k)
        if n > 1 and a["arcs"].size:
            ra, rb = gd.apsp(per_source=True), gh.apsp(per_source=True)
            assert ra.sum_distances == rb.sum_distances and ra.diameter == rb.diameter
            assert np.array_equal(gd.source_order(), gh.source_order())
            bca, _ = gd.brandes()
            bcb, _ = gh.brandes()
            assert np.array_equal(bca, bcb)
    # the in-arcs of each target in ascending source order, each arc once
    m = a["arcs"].size
    assert np.array_equal(np.sort(a["rarcs"]["id"]), np.arange(m))
    for v in range(0, n, max(1, n // 200)):
        seg = a["rarcs"][a["rrow_ptr"][v]:a["rrow_ptr"][v + 1]]
        assert np.all(np.diff(seg["id"]) > 0)
        assert np.all(a["arcs"]["col"][seg["id"]] == v)


@pytest.mark.parametrize("bad", ["target", "negative target", "nan", "inf"])
def test_bad_arcs_give_the_same_error(bad):
    c = synth.random_graph(500, 4, weights="lognormal", seed=6)
    col, w = c.col.copy(), c.w.copy()
    at = c.m // 2
    if bad == "target":
        col[at] = c.n
    elif bad == "negative target":
        col[at] = -3
    elif bad == "nan":
        w[at] = np.nan
    else:
        w[at] = np.inf
    w[at + 5] = np.nan  # a later bad arc: the first one is reported
    messages = []
    for build in ("device", "host"):
        with pytest.raises(ngx.NgxError) as e:
            ngx.Graph(c.n, c.row_ptr, col, w, build=build)
        messages.append(str(e.value))
    assert messages[0] == messages[1]
    assert f"arc {at} " in messages[0]


def test_update_weights_on_a_device_built_handle():
    c = synth.connectome(3000, 10, 0.15, weights="lognormal", seed=7, use_gpu=False)
    w2 = c.w * np.random.default_rng(1).uniform(0.5, 2.0, c.m)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g, ngx.Graph(c.n, c.row_ptr, c.col, w2, build="host") as want:
        g.update_weights(w2)
        a, b = g.apsp(per_source=True), want.apsp(per_source=True)
        assert a.sum_distances == b.sum_distances
        for k, v in b.per_source.items():
            assert np.array_equal(a.per_source[k], v), k
