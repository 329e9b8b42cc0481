"""All-sources APSP over several ranks (one process per GPU): sources sharded, graph replicated, one exact exchange.

The reference shards sources over MPI ranks and combines the per-rank results at the end
(source/metrics/paths/AllPairsShortestPath.h:130-158: each rank loops over its local sources, then the sums, the
unreachable count and the cluster sizes are reduced; BetweennessCentrality.h:74 sums the per-rank betweenness vectors
with reduce_componentwise_sum). Here every rank runs the batched kernel on its contiguous, tile-aligned slice of the
sources, and one exchange merges the results exactly:

* `merge_apsp`: the exact digit accumulators of the sums of d and 1/d are summed word by word (so the merged sums
  round once, to the same bits as a single-GPU run), counts and histograms are summed, the diameter is the maximum,
  and cluster sizes are merged;
* `merge_fixed`: per-vertex betweenness and per-arc gradient sums, which the library keeps as 128-bit fixed-point
  integers, are split into 32-bit limbs, summed, and carried back into 128-bit words, so the merged betweenness and
  gradients convert to the bits of a single run.

torch.distributed carries the exchange (NCCL between GPUs, gloo on CPU).
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


def merge_fixed(words, dist, group=None) -> np.ndarray:
    """Sum over the ranks of (count, 2) 128-bit fixed-point words (low, high), modulo 2^128 like the library's own
    sums: each word is split into 32-bit limbs, the limbs are summed with one all-reduce (below 2^63 for up to 2^31
    ranks), and the carries are propagated on the host."""
    import torch

    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1, 2)
    mask = np.uint64(0xFFFFFFFF)
    limbs = np.stack([w[:, 0] & mask, w[:, 0] >> np.uint64(32), w[:, 1] & mask, w[:, 1] >> np.uint64(32)], axis=1)
    t = torch.from_numpy(limbs.astype(np.int64)).to(_device(dist, group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    s = t.cpu().numpy().astype(np.uint64)
    out = np.zeros_like(s)
    carry = np.zeros(s.shape[0], np.uint64)
    for i in range(4):
        v = s[:, i] + carry
        out[:, i] = v & mask
        carry = v >> np.uint64(32)
    # limbs back into (low, high); the carry out of the top limb is the modulo-2^128 wrap
    return np.stack([out[:, 0] | (out[:, 1] << np.uint64(32)), out[:, 2] | (out[:, 3] << np.uint64(32))], axis=1)


def shard_order(graph, rank: int, world: int, tile: int = 32) -> np.ndarray:
    """Rank `rank`'s sources for a betweenness or gradient run: a tile-aligned contiguous chunk of the graph's own
    all-sources order (tiles of nearby vertices), so the sharded run takes the same tiles as a single run."""
    order = graph.source_order()
    bounds = shard_sources(order.size, rank, world, tile)
    return order[bounds] if bounds.size else np.zeros(0, np.int64)


def brandes_sharded(graph, dist, group=None, **kwargs) -> np.ndarray:
    """This rank's share of an all-sources Brandes run on `graph` (the same graph on every rank), merged over the
    group: the per-vertex betweenness of the whole graph, the bits of a single run."""
    from . import fixed_to_double

    sources = shard_order(graph, dist.get_rank(group), dist.get_world_size(group))
    words, _ = graph.brandes(sources=sources, fixed=True, **kwargs)
    return fixed_to_double(merge_fixed(words, dist, group), 1.0, 1.0)


def grad_sharded(graph, dist, group=None, **kwargs):
    """This rank's share of an all-sources gradient run, merged over the group: (dcpl, deff, reached_pairs) of the
    whole graph, the bits of a single run (the sums are merged first, then divided once by the merged R)."""
    import torch

    from . import fixed_to_double

    sources = shard_order(graph, dist.get_rank(group), dist.get_world_size(group))
    dcpl_w, deff_w, r = graph.apsp_grad(sources=sources, fixed=True, **kwargs)
    both = merge_fixed(np.concatenate([dcpl_w, deff_w]), dist, group)
    reached = torch.tensor([r.reached_pairs], dtype=torch.int64, device=_device(dist, group))
    dist.all_reduce(reached, op=dist.ReduceOp.SUM, group=group)
    total = int(reached.item())
    m = dcpl_w.shape[0]
    return fixed_to_double(both[:m], float(total), 1.0), fixed_to_double(both[m:], float(total), -1.0), total
