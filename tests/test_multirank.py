"""The multi-rank path on CPU: two gloo ranks, no GPU.

Covers what a sharded run exchanges and how the benchmark shards: exact accumulators merged word by word round to the
bits of a single sum (math.fsum), a whole-graph APSP assembled from two disjoint source shards equals the oracle's
all-sources run bit for bit, shard bounds are tile-aligned and cover every vertex once, and the benchmark's per-rank
source batches are disjoint with max / sum timing reductions.
"""

from __future__ import annotations

import math
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import neurograph_b200 as ngx
import oracle
from neurograph_b200 import sharded, synth

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(rank, world, port, body):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        body(rank, world)
    finally:
        dist.destroy_process_group()


def _spawn(body):
    mp.spawn(_run, args=(WORLD, _free_port(), body), nprocs=WORLD, join=True)


def _values(rank):
    rng = np.random.default_rng(100 + rank)
    return np.concatenate([rng.lognormal(0.0, 4.0, 20000), rng.random(5000) * 1e-300, [0.0, 1e300, 5e-324]])


def _exact_merge(rank, world):
    digits = ngx.exact_accumulate(_values(rank))
    merged = sharded.merge_exact(digits, dist)
    everything = np.concatenate([_values(r) for r in range(world)])
    assert ngx.exact_round(merged) == math.fsum(everything)


def test_exact_accumulators_merge_over_ranks():
    _spawn(_exact_merge)


def _graph():
    c = synth.connectome(400, 5, 0.2, weights="lognormal", seed=77, use_gpu=False)
    return c, oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)


def _shard_partial(restatement, csr, sources, bins, hist_max):
    """This rank's partial result in the shape the GPU returns it (exact=True), computed on the CPU by the oracle."""
    part = restatement.apsp(csr, sources=sources, bins=bins, hist_max=hist_max)
    digits = np.zeros((2, ngx.ACC_DIGITS), np.uint64)
    for s in sources:
        row = restatement.sssp(csr, int(s))
        finite = row[np.isfinite(row)]
        ngx.exact_accumulate(finite, digits[0])
        ngx.exact_accumulate(1.0 / finite[finite != 0.0], digits[1])
    return SimpleNamespace(acc_digits=digits, unreachable=part["unreachable"], reached_pairs=part["reached_pairs"],
                           traversed_arcs=part["traversed_arcs"], hist_overflow=part["hist_overflow"], diameter=part["diameter"],
                           hist=part["hist"], cluster_sizes=part["cluster_sizes"])


def _apsp_merge(rank, world):
    oracle.build()
    restatement = oracle.Restatement()
    c, csr = _graph()
    sources = sharded.shard_sources(c.n, rank, world)
    merged = sharded.merge_apsp(_shard_partial(restatement, csr, sources, 64, 12.0), dist)
    want = restatement.apsp(csr, bins=64, hist_max=12.0)
    for k in ("sum_distances", "sum_inverse", "cpl", "efficiency", "diameter", "unreachable", "reached_pairs", "traversed_arcs",
              "hist_overflow", "cluster_sizes"):
        assert merged[k] == want[k], (k, merged[k], want[k])
    assert np.array_equal(merged["hist"], want["hist"])


def test_sharded_apsp_equals_single_run():
    _spawn(_apsp_merge)


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 1000, 100000])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_are_tile_aligned_and_cover_once(n, world):
    parts = [sharded.shard_sources(n, r, world) for r in range(world)]
    allv = np.concatenate(parts) if parts else np.zeros(0, np.int64)
    assert np.array_equal(np.sort(allv), np.arange(n))
    for p in parts[:-1]:
        if p.size:
            assert p[0] % 32 == 0 and (p[-1] + 1) % 32 == 0
    sizes = [p.size for p in parts]
    assert max(sizes) - min(sizes) <= 32


def _bench_helpers(rank, world):
    import bench

    batches = bench.source_batches(100000, 9472, 4, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, [b.tolist() for b in batches])
    for step in range(4):
        a, b = set(gathered[0][step]), set(gathered[1][step])
        assert not (a & b)
    assert bench.reduce_over_ranks(dist, 1.5 + rank, "max", "cpu") == 1.5 + world - 1
    assert bench.reduce_over_ranks(dist, 1.5 + rank, "sum", "cpu") == sum(1.5 + r for r in range(world))


def test_bench_sharding_and_timing_reductions():
    _spawn(_bench_helpers)
