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


def _fixed_words(values) -> list[int]:
    """The library's 128-bit fixed point of non-negative doubles (value * 2^64, fraction truncated), as Python ints."""
    out = []
    for x in values:
        x = float(x)
        if not x > 0.0:
            out.append(0)
            continue
        whole = math.floor(x)
        out.append((int(whole) << 64) + int(math.ldexp(x - whole, 64)))
    return out


def _pack(ints) -> np.ndarray:
    mask = (1 << 64) - 1
    return np.array([[v & mask, (v >> 64) & mask] for v in ints], dtype=np.uint64).reshape(-1, 2)


def _random_words(rank, count=3000):
    rng = np.random.default_rng(200 + rank)
    words = rng.integers(0, 1 << 63, size=(count, 2), dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    words[:10] = np.uint64(0xFFFFFFFFFFFFFFFF)  # carries through every limb, and the modulo-2^128 wrap
    words[10:20, 1] = 0
    return words


def _fixed_merge(rank, world):
    merged = sharded.merge_fixed(_random_words(rank), dist)
    want = [0] * merged.shape[0]
    for r in range(world):
        for i, (lo, hi) in enumerate(_random_words(r).tolist()):
            want[i] = (want[i] + lo + (hi << 64)) % (1 << 128)
    assert np.array_equal(merged, _pack(want))


def test_fixed_point_sums_merge_over_ranks():
    _spawn(_fixed_merge)


def _brandes_merge(rank, world):
    """Each rank's betweenness words, as the library forms them (per-source dependencies truncated to fixed point and
    summed exactly), from the oracle's per-source dependencies; the merged words equal the all-sources words."""
    oracle.build()
    restatement = oracle.Restatement()
    c, csr = _graph()
    per_source = [restatement.brandes(csr, sources=[s]) for s in range(c.n)]

    def words_of(sources):
        total = [0] * c.n
        for s in sources:
            for v, x in enumerate(_fixed_words(per_source[s])):
                total[v] += x
        return total

    mine = sharded.shard_sources(c.n, rank, world)
    merged = sharded.merge_fixed(_pack(words_of(mine)), dist)
    whole = words_of(range(c.n))
    assert np.array_equal(merged, _pack(whole))
    bc = ngx.fixed_to_double(merged)
    want = restatement.brandes(csr)
    assert np.all(np.abs(bc - want) <= 1e-12 * np.maximum(np.abs(want), 1.0))


def test_sharded_betweenness_words_equal_the_single_run():
    _spawn(_brandes_merge)


def test_bench_sharding_and_timing_reductions():
    _spawn(_bench_helpers)
