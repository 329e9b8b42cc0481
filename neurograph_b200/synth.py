"""Seeded synthetic connectomes of the shapes neurograph is benchmarked on.

N vertices uniform in the unit cube (FP64 positions), 8 areas by octant, 80/20 excitatory/inhibitory types,
out-degree ~ Poisson(lambda), each target drawn (with replacement, no self-loops) with probability proportional to
exp(-||x_u - x_v|| / length_scale); repeated targets are merged by summing their weights, as the reference's file
loader does (source/graph/FileLoader.cpp:248,323). Weights: integer U{1..10}, log-normal(mu, sigma), or unit.

The dense sampler evaluates the kernel against every vertex (exact), on the GPU through torch when one is present and
the graph is large, else with numpy. It is input generation for tests and benchmarks, not part of the timed path.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Connectome:
    n: int
    row_ptr: np.ndarray  # int64, n + 1
    col: np.ndarray      # int32, m
    w: np.ndarray        # float64, m
    positions: np.ndarray
    area: np.ndarray     # octant index 0..7
    excitatory: np.ndarray

    @property
    def m(self) -> int:
        return int(self.col.size)


def _weights(rng: np.random.Generator, count: int, kind: str, mu: float, sigma: float) -> np.ndarray:
    if kind == "int":
        return rng.integers(1, 11, size=count).astype(np.float64)
    if kind == "lognormal":
        return rng.lognormal(mean=mu, sigma=sigma, size=count)
    if kind == "unit":
        return np.ones(count, np.float64)
    raise ValueError(f"unknown weight kind {kind!r}")


def _targets_numpy(rng, pos, degrees, length_scale, chunk=512):
    n = pos.shape[0]
    sources, targets = [], []
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        d = np.sqrt(((pos[c0:c1, None, :] - pos[None, :, :]) ** 2).sum(-1))
        k = np.exp(-d / length_scale)
        k[np.arange(c1 - c0), np.arange(c0, c1)] = 0.0
        cum = np.cumsum(k, axis=1)
        for i in range(c1 - c0):
            deg = int(degrees[c0 + i])
            if deg == 0 or cum[i, -1] <= 0.0:
                continue
            r = rng.random(deg) * cum[i, -1]
            t = np.minimum(np.searchsorted(cum[i], r, side="right"), n - 1)
            sources.append(np.full(deg, c0 + i, np.int64))
            targets.append(t.astype(np.int64))
    if not sources:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(sources), np.concatenate(targets)


def _targets_torch(seed, pos, degrees, length_scale, chunk=2048):
    import torch

    dev = torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    p = torch.as_tensor(pos, dtype=torch.float32, device=dev)
    deg = torch.as_tensor(degrees, dtype=torch.int64, device=dev)
    n = p.shape[0]
    sources, targets = [], []
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        kmax = int(deg[c0:c1].max().item()) if c1 > c0 else 0
        if kmax == 0:
            continue
        k = torch.exp(-torch.cdist(p[c0:c1], p) / length_scale)
        k[torch.arange(c1 - c0, device=dev), torch.arange(c0, c1, device=dev)] = 0.0
        t = torch.multinomial(k, kmax, replacement=True, generator=gen)
        keep = torch.arange(kmax, device=dev)[None, :] < deg[c0:c1, None]
        rows = torch.arange(c0, c1, device=dev)[:, None].expand(-1, kmax)
        sources.append(rows[keep].cpu().numpy())
        targets.append(t[keep].cpu().numpy())
        del k
    return np.concatenate(sources).astype(np.int64), np.concatenate(targets).astype(np.int64)


def connectome(n: int, mean_degree: float, length_scale: float = 0.1, weights: str = "int", mu: float = 0.0, sigma: float = 1.0,
               seed: int = 0, use_gpu: bool | None = None) -> Connectome:
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3))
    area = ((pos[:, 0] >= 0.5).astype(np.int64) | ((pos[:, 1] >= 0.5).astype(np.int64) << 1) | ((pos[:, 2] >= 0.5).astype(np.int64) << 2))
    excitatory = rng.random(n) < 0.8
    degrees = rng.poisson(mean_degree, size=n) if n > 1 else np.zeros(n, np.int64)
    if use_gpu is None:
        use_gpu = n > 20000
        if use_gpu:
            try:
                import torch

                use_gpu = torch.cuda.is_available()
            except Exception:  # noqa: BLE001
                use_gpu = False
    if use_gpu:
        src, dst = _targets_torch(seed, pos, degrees, length_scale)
    else:
        src, dst = _targets_numpy(rng, pos, degrees, length_scale)
    w = _weights(rng, src.size, weights, mu, sigma)
    # merge repeated (u, v) by summing weights; arcs of a vertex sorted by target
    key = src * n + dst
    order = np.argsort(key, kind="stable")
    key, w = key[order], w[order]
    uniq, start = np.unique(key, return_index=True)
    merged_w = np.add.reduceat(w, start) if w.size else w
    u = (uniq // n).astype(np.int64)
    v = (uniq % n).astype(np.int32)
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, u + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    return Connectome(n, row_ptr, v, merged_w.astype(np.float64), pos, area, excitatory)


def random_graph(n: int, mean_degree: float, weights: str = "int", seed: int = 0, mu: float = 0.0, sigma: float = 1.0,
                 self_loops: bool = False) -> Connectome:
    """Uniform random targets (no spatial kernel): quick test graphs with many ties (int) or none (lognormal)."""
    rng = np.random.default_rng(seed)
    degrees = rng.poisson(mean_degree, size=n)
    src = np.repeat(np.arange(n, dtype=np.int64), degrees)
    dst = rng.integers(0, max(n, 1), size=src.size).astype(np.int64)
    if not self_loops and n > 1:
        same = dst == src
        dst[same] = (dst[same] + 1) % n
    w = _weights(rng, src.size, weights, mu, sigma)
    key = src * n + dst
    order = np.argsort(key, kind="stable")
    key, w = key[order], w[order]
    uniq, start = np.unique(key, return_index=True)
    merged_w = np.add.reduceat(w, start) if w.size else w
    u = (uniq // max(n, 1)).astype(np.int64)
    v = (uniq % max(n, 1)).astype(np.int32)
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, u + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    z = np.zeros(n)
    return Connectome(n, row_ptr, v, merged_w.astype(np.float64), np.zeros((n, 3)), z.astype(np.int64), z.astype(bool))
