"""Sharded all-sources runs through the C ABI: two ranks (gloo for the exchange, both on cuda:0, each with its own
graph handle and disjoint source shard; no rank's kernel waits for another's) must reproduce the single-run results
bit for bit: APSP (exact sums merged word by word, counts, histogram, diameter, cluster sizes), betweenness and both
gradients (128-bit fixed-point words merged, then converted once)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import neurograph_b200 as ngx
from neurograph_b200 import sharded, synth

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(kind):
    return synth.connectome(3000, 8, 0.15, weights=kind, seed=91, use_gpu=False)


def _rank(rank, world, port, kind, out_dir):
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        c = _graph(kind)
        with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
            merged = sharded.apsp_sharded(g, dist, hist_bins=128, hist_max=40.0)
        if rank == 0:
            np.save(os.path.join(out_dir, "merged.npy"), np.array([merged], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["lognormal", "int"])
def test_two_shards_equal_one_run(tmp_path, kind):
    mp.spawn(_rank, args=(2, _free_port(), kind, str(tmp_path)), nprocs=2, join=True)
    merged = np.load(tmp_path / "merged.npy", allow_pickle=True)[0]
    c = _graph(kind)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        want = g.apsp(hist_bins=128, hist_max=40.0, per_source=True)
    for k in ("sum_distances", "sum_inverse", "cpl", "efficiency", "diameter", "unreachable", "reached_pairs", "traversed_arcs",
              "hist_overflow", "cluster_sizes"):
        assert merged[k] == getattr(want, k), (k, merged[k], getattr(want, k))
    assert np.array_equal(merged["hist"], want.hist)


def _dag_rank(rank, world, port, kind, out_dir):
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        c = _graph(kind)
        with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
            bc = sharded.brandes_sharded(g, dist)
            dcpl, deff, reached = sharded.grad_sharded(g, dist)
        if rank == 0:
            np.savez(os.path.join(out_dir, "dag.npz"), bc=bc, dcpl=dcpl, deff=deff, reached=reached)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["lognormal", "int"])
def test_two_shards_of_betweenness_and_gradients_equal_one_run(tmp_path, kind):
    mp.spawn(_dag_rank, args=(2, _free_port(), kind, str(tmp_path)), nprocs=2, join=True)
    got = np.load(tmp_path / "dag.npz")
    c = _graph(kind)
    with ngx.Graph(c.n, c.row_ptr, c.col, c.w) as g:
        bc, _ = g.brandes()
        dcpl, deff, r = g.apsp_grad()
    assert int(got["reached"]) == r.reached_pairs
    assert np.array_equal(got["bc"], bc)
    assert np.array_equal(got["dcpl"], dcpl) and np.array_equal(got["deff"], deff)
