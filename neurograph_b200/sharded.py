"""All-sources APSP over several ranks (one process per GPU): sources sharded, graph replicated, one exact exchange.

The reference shards sources over MPI ranks and combines the per-rank results at the end
(source/metrics/paths/AllPairsShortestPath.h:130-158: each rank loops over its local sources, then the sums, the
unreachable count and the cluster sizes are reduced). Here every rank runs the batched kernel on its contiguous,
tile-aligned slice of the vertices, and `merge_apsp` is the only exchange: the exact digit accumulators of the sums of
d and 1/d are summed word by word (so the merged sums round once, to the same bits as a single-GPU run), counts and
histograms are summed, the diameter is the maximum, and cluster sizes are merged. torch.distributed carries the
exchange (NCCL between GPUs, gloo on CPU).
"""

from __future__ import annotations

import numpy as np

from . import ACC_DIGITS, exact_round


def shard_sources(n: int, rank: int, world: int, tile: int = 32) -> np.ndarray:
    """Rank `rank`'s sources: a contiguous slice of 0..n-1 whose bounds are multiples of the source tile width, so no
    tile straddles two ranks and the slices differ by at most one tile."""
    tiles = (n + tile - 1) // tile
    first = tiles * rank // world
    last = tiles * (rank + 1) // world
    return np.arange(first * tile, min(last * tile, n), dtype=np.int64)


def _device(dist, group):
    backend = dist.get_backend(group)
    return "cuda" if backend == "nccl" else "cpu"


def merge_exact(digits, dist, group=None) -> np.ndarray:
    """Sum of every rank's normalized accumulators (any leading shape, last axis ACC_DIGITS), word by word."""
    import torch

    d = np.asarray(digits, dtype=np.uint64)
    if d.shape[-1] != ACC_DIGITS or int(d.max(initial=0)) >= 1 << 32:
        raise ValueError("expected normalized accumulators (every word below 2^32)")
    t = torch.from_numpy(d.astype(np.int64)).to(_device(dist, group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().astype(np.uint64)


def merge_apsp(result, dist, group=None) -> dict:
    """Combines the per-rank ApspResult of disjoint source sets (run with exact=True). Returns the whole-graph values:
    sum_distances, sum_inverse (exactly rounded), cpl, efficiency, diameter, unreachable, reached_pairs,
    traversed_arcs, hist_overflow, hist (if every rank has one) and cluster_sizes."""
    import torch

    if result.acc_digits is None:
        raise ValueError("run the shards with exact=True")
    dev = _device(dist, group)
    digits = merge_exact(result.acc_digits, dist, group)
    counts = torch.tensor([result.unreachable, result.reached_pairs, result.traversed_arcs, result.hist_overflow],
                          dtype=torch.int64, device=dev)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    diameter = torch.tensor([result.diameter], dtype=torch.float64, device=dev)
    dist.all_reduce(diameter, op=dist.ReduceOp.MAX, group=group)
    hist = None
    if result.hist is not None:
        h = torch.from_numpy(result.hist.astype(np.int64)).to(dev)
        dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
        hist = h.cpu().numpy().astype(np.uint64)
    world = dist.get_world_size(group)
    sizes = [None] * world
    dist.all_gather_object(sizes, dict(result.cluster_sizes), group=group)
    cluster_sizes: dict[int, int] = {}
    for part in sizes:
        for k, v in part.items():
            cluster_sizes[int(k)] = cluster_sizes.get(int(k), 0) + int(v)
    unreachable, reached, traversed, overflow = (int(x) for x in counts.cpu().tolist())
    sum_d = exact_round(digits[0])
    sum_inv = exact_round(digits[1])
    return {
        "sum_distances": sum_d, "sum_inverse": sum_inv,
        "cpl": sum_d / reached if reached else float("nan"), "efficiency": sum_inv / reached if reached else float("nan"),
        "diameter": float(diameter.item()), "unreachable": unreachable, "reached_pairs": reached,
        "traversed_arcs": traversed, "hist_overflow": overflow, "hist": hist, "cluster_sizes": cluster_sizes,
    }


def apsp_sharded(graph, dist, group=None, **apsp_kwargs) -> dict:
    """This rank's share of an all-sources APSP on `graph` (the same graph on every rank), merged over the group."""
    if apsp_kwargs.get("hist_bins", 0) > 0 and not apsp_kwargs.get("hist_max", 0.0) > 0.0:
        raise ValueError("a sharded histogram needs an explicit hist_max (the same bins on every rank)")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    sources = shard_sources(graph.n, rank, world)
    kw = dict(apsp_kwargs)
    kw["per_source"] = True  # cluster sizes need the per-source unreachable counts
    r = graph.apsp(sources=sources, exact=True, **kw)
    return merge_apsp(r, dist, group)
