"""Benchmark: all-sources APSP + Brandes throughput (GTEPS) on B200, batched form, with the reference CPU path beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ngx|reference]

Workload (the batched single-graph configuration): a synthetic connectome with N = 100,000 vertices in the unit cube,
out-degree Poisson(100) (about 1e7 arcs after merging repeated targets), spatial kernel exp(-d / 0.08), log-normal(0, 1)
FP64 weights, generated from a fixed seed. One step = one batch of sources (a contiguous chunk of the library's
all-sources order, ngx_graph_source_order, consumed batch after batch) run through ngx_brandes: distances by batched delta-stepping, the fused APSP
summaries (exact sums of d and 1/d, diameter, unreachable count, 1024-bin distance histogram, per-source outputs) and
Brandes betweenness, in one persistent launch. GTEPS = traversed arcs (sum over sources of the out-degrees of the
vertices they reach) / seconds.

Timing: W untimed steps, then K steps between a barrier + synchronize on both sides; device time from CUDA events on
the stream the library runs on (handed to it with ngx_graph_set_stream); max over ranks. The graph (320 MB of CSR and
reverse CSR) and the per-CTA workspaces (GBs) are larger than L2, so no flush is needed between steps.
e2e: the same metric through the C ABI from host buffers, for the K-step job as a user runs it: the graph is created
from the pinned host CSR once (H2D, inside the timed region), every step passes its source list from the host and
copies its results (betweenness, per-source summaries, histogram) back (D2H); wall clock, synchronized.
Under torchrun (N > 1) every rank runs its own disjoint batches (weak scaling); only the timing scalars are reduced.

--impl reference: the reference's algorithm on the host cores. The reference's own build (oracle/_ref) reads int32
weights only, so for this FP64-weight workload the CPU restatement of its Dijkstra and Brandes (oracle/ngx_oracle.c,
bit-exact with the reference on integer weights) runs in one process per host core on disjoint sources.
"""

from __future__ import annotations

import argparse
import contextlib
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "batched single graph: synthetic connectome N=100000, out-degree Poisson(100), kernel exp(-d/0.08), "
                "log-normal(0,1) FP64 weights; APSP summaries + 1024-bin histogram + Brandes per source batch",
    "n": 100000, "mean_degree": 100.0, "length_scale": 0.08, "weights": "lognormal(0,1)", "seed": 2,
}
# The plain small configuration: the one the reference itself can load (integer weights), all sources per step.
WORKLOAD_C1 = {
    "workload": "plain small graph: synthetic connectome N=5000, out-degree Poisson(6), kernel exp(-d/0.1), integer weights "
                "U{1..10} stored FP64; all-sources APSP summaries + 1024-bin histogram + Brandes per step",
    "n": 5000, "mean_degree": 6.0, "length_scale": 0.1, "weights": "int U{1..10}", "seed": 1,
}
HIST_BINS = 1024
L2_BYTES = 126 << 20
SLOTS_PER_WAVE = 296  # 148 SMs x 2 resident CTAs
DEFAULT_SOURCES_PER_STEP = SLOTS_PER_WAVE * 32


def pause_gc():
    """Collects now and pauses Python's cyclic garbage collector for a timed region (as timeit does): a full
    collection over the interpreter's objects takes tens of milliseconds and would otherwise land in a random step."""
    gc.collect()
    gc.disable()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ngx", "reference"], default="ngx")
    ap.add_argument("--sources-per-step", type=int, default=DEFAULT_SOURCES_PER_STEP)
    ap.add_argument("--n", "--vertices", dest="n", type=int, default=WORKLOAD["n"],
                    help="vertices of the connectome (--vertices also passes through torchrun, whose own options --n abbreviates)")
    ap.add_argument("--degree", type=float, default=WORKLOAD["mean_degree"])
    ap.add_argument("--length-scale", type=float, default=WORKLOAD["length_scale"])
    ap.add_argument("--sigma", type=float, default=1.0, help="log-normal sigma of the weights")
    ap.add_argument("--workload", choices=["single", "uneven-batch", "scc", "c1"], default="single",
                    help="single: one connectome (the headline); uneven-batch: 512 connectomes of 500-20000 vertices in one "
                         "handle; scc: strongly connected components of the connectome (ngx_scc) beside the reference's SCC; "
                         "c1: the plain small integer-weight connectome (N=5000), all sources per step, beside the reference "
                         "itself built from source")
    ap.add_argument("--delta", type=float, default=0.0,
                    help="bucket width; 0 = the library's default (2/sqrt(mean out-degree) x the mean arc length)")
    ap.add_argument("--mode", choices=["brandes", "apsp", "grad", "plain"], default="brandes",
                    help="what one step runs: APSP+Brandes (the headline), APSP only, APSP+gradient, or the plain per-source form")
    ap.add_argument("--block-threads", type=int, default=0, help="tile kernel block size (0 = the library default)")
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="resident tile CTAs per SM (0 = as many as fit)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the plain/batched APSP comparison runs")
    ap.add_argument("--autotune", action="store_true",
                    help="run the library's autotuner for the mode before the warm-up (outside the timed region) and use its "
                         "bucket width and block shape for every step, the e2e job included")
    args = ap.parse_args()
    if args.workload == "c1":
        # every step is the whole all-sources job of the small graph; the bucket width follows the integer weights
        args.n, args.degree, args.length_scale = WORKLOAD_C1["n"], WORKLOAD_C1["mean_degree"], WORKLOAD_C1["length_scale"]
        args.sources_per_step = WORKLOAD_C1["n"]
    return args


def make_graph(n, degree, length_scale=WORKLOAD["length_scale"], sigma=1.0, workload="single"):
    from neurograph_b200 import synth

    if workload == "c1":
        return synth.connectome(WORKLOAD_C1["n"], WORKLOAD_C1["mean_degree"], WORKLOAD_C1["length_scale"], weights="int",
                                seed=WORKLOAD_C1["seed"], use_gpu=False)
    return synth.connectome(n, degree, length_scale, weights="lognormal", mu=0.0, sigma=sigma, seed=WORKLOAD["seed"])


def workload_overrides(args):
    """Config keys that differ from the default connectome (other generator parameters on the same code path)."""
    if args.workload == "c1":
        return {k: v for k, v in WORKLOAD_C1.items() if k != "n"}  # n comes from the generated graph
    if (args.n, args.degree, args.length_scale, args.sigma) == (WORKLOAD["n"], WORKLOAD["mean_degree"], WORKLOAD["length_scale"], 1.0):
        return {}
    return {"workload": f"single graph: synthetic connectome N={args.n}, out-degree Poisson({args.degree:g}), kernel "
                        f"exp(-d/{args.length_scale:g}), log-normal(0,{args.sigma:g}) FP64 weights; mode {args.mode}",
            "mean_degree": args.degree, "length_scale": args.length_scale, "weights": f"lognormal(0,{args.sigma:g})"}


def reduce_over_ranks(dist, x, op, device):
    """Max or sum of a timing scalar over the ranks (the only collective of the benchmark: sources are sharded, the
    data path exchanges nothing). dist is torch.distributed or None for one process."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def source_batches(n, per_step, count, rank, world, order=None):
    """Step i of rank r takes the (i * world + r)-th chunk of `per_step` sources of `order` (wrapping around): the
    library's all-sources order (ngx_graph_source_order) for the GPU arm, a seeded permutation otherwise."""
    perm = np.random.default_rng(12345).permutation(n) if order is None else np.asarray(order, dtype=np.int64)
    out = []
    for i in range(count):
        start = ((i * world + rank) * per_step) % n
        idx = (start + np.arange(per_step)) % n
        out.append(np.ascontiguousarray(perm[idx], dtype=np.int64))
    return out


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.proc = None
        self.device_index = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                                          "-i", str(self.device_index)], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def wait_first_sample(self, timeout_s=10.0):
        """nvidia-smi's start-up (NVML initialisation) can stall the GPU's host interface; wait for its first sample so
        that this happens before the timed region, not inside it."""
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < timeout_s:
            self.file.flush()
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)
        time.sleep(0.3)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, sm_max, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                sm_max.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.strip().lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(sm_max), "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def peak_label(kind):
    """How the roofline's peak was obtained: the measured copy bandwidth, or the fallback figure."""
    return "measured hbm_gbs (MEASURED_PEAKS.json)" if kind == "measured" else "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic_per_arc(mode):
    """DRAM bytes per traversed arc of the mode's tile kernel on this workload, from the committed ncu summary (or None)."""
    path = os.path.join(ROOT, "profiles", f"tile_kernel_{mode}_connectome_n100k.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_traversed_arc:"):
                return float(line.split(":", 1)[1])
    return None


_WORKER = {}


def cpu_worker_init(directory, count=1):
    """Maps the CSRs (graph 0 .. count-1) read-only (shared page cache across the worker processes)."""
    sys.path.insert(0, ROOT)
    import oracle

    _WORKER["graphs"] = []
    for i in range(count):
        row_ptr, col, w = (np.load(os.path.join(directory, f"g{i}_{name}.npy"), mmap_mode="r") for name in ("row_ptr", "col", "w"))
        _WORKER["graphs"].append(oracle.Csr(int(row_ptr.size - 1), row_ptr, col, w))
    _WORKER["oracle"] = oracle.Restatement()


def cpu_worker(task):
    """task: sources of graph 0, or (graph index, sources)."""
    gi, sources = task if isinstance(task, tuple) else (0, task)
    g, r = _WORKER["graphs"][gi], _WORKER["oracle"]
    t0 = time.perf_counter()
    a = r.apsp(g, sources=sources, bins=HIST_BINS, hist_max=64.0)
    r.brandes(g, sources=sources)
    return int(a["traversed_arcs"]), time.perf_counter() - t0


def save_graphs(directory, graphs):
    for i, (_, row_ptr, col, w) in enumerate(graphs):
        for name, arr in (("row_ptr", row_ptr), ("col", col), ("w", w)):
            np.save(os.path.join(directory, f"g{i}_{name}.npy"), arr)


def remove_graphs(directory, count):
    for i in range(count):
        for name in ("row_ptr", "col", "w"):
            os.unlink(os.path.join(directory, f"g{i}_{name}.npy"))
    os.rmdir(directory)


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def time_reference_pool(args, directory, count, tasks_per_step):
    """W + K steps of the restatement over a spawned process pool (one process per host core); each step maps one
    task per process. Returns (timed seconds, traversed arcs) of the K timed steps."""
    import multiprocessing as mp

    cores = host_cores()
    ctx = mp.get_context("spawn")
    times, arcs = [], []
    with ctx.Pool(cores, initializer=cpu_worker_init, initargs=(directory, count)) as pool:
        pool.map(cpu_worker, [(0, np.zeros(0, np.int64))] * cores)  # start every worker and map the graphs before timing
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(cpu_worker, tasks_per_step(i), chunksize=1)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
                arcs.append(sum(r[0] for r in res))
    return sum(times), sum(arcs)


def reference_line(args, metric, unit, value, total_s, config, cores, kind, sample):
    return {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if unit == "GTEPS" else "int32", "data": "synthetic", "config": config,
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, rank, world):
    """The reference arm on the host cores (rank 0 only): the reference's algorithm for the selected workload."""
    if rank != 0:
        return
    if args.workload == "scc":
        run_reference_scc(args)
        return
    if args.workload == "uneven-batch":
        run_reference_uneven_batch(args)
        return
    if args.workload == "c1":
        run_reference_c1(args)
        return
    c = make_graph(args.n, args.degree, args.length_scale, args.sigma)
    cores = host_cores()
    directory = tempfile.mkdtemp(prefix="ngx_ref_")
    save_graphs(directory, [(c.n, c.row_ptr, c.col, c.w)])
    batches = source_batches(c.n, cores, args.warmup + args.steps, 0, 1)
    total, arcs = time_reference_pool(args, directory, 1, lambda i: [(0, batches[i][j:j + 1]) for j in range(len(batches[i]))])
    remove_graphs(directory, 1)
    value = arcs / total / 1e9
    line = reference_line(args, "APSP+Brandes GTEPS (batched single graph)", "GTEPS", value, total,
                          dict(WORKLOAD, **workload_overrides(args), n=c.n, arcs=int(c.m), sources_per_step=cores,
                               parallelism=f"{cores} host processes x 1 thread"), cores, "port",
                          f"{cores} sources per step (one per process), APSP summaries + histogram + Brandes, CPU restatement "
                          "of the reference Dijkstra/Brandes (the reference build reads int32 weights only)")
    print(json.dumps(line), flush=True)


def run_reference_uneven_batch(args, sample_graphs=8):
    """The uneven batch on the host cores: every step four sources per process, round-robin over a seeded sample of the
    batch's graphs (the CPU rate per traversed arc hardly depends on the graph, and generating all 512 graphs on the
    host takes over half an hour)."""
    indices = list(range(0, UNEVEN_BATCH["graphs"], UNEVEN_BATCH["graphs"] // sample_graphs))[:sample_graphs]
    graphs = uneven_batch_graphs(indices=indices)
    cores = host_cores()
    directory = tempfile.mkdtemp(prefix="ngx_ref_")
    save_graphs(directory, graphs)
    rng = np.random.default_rng(12345)

    per_step = 4 * cores

    def tasks(i):
        out = []
        for j in range(per_step):
            gi = (i * per_step + j) % len(graphs)
            out.append((gi, np.array([int(rng.integers(0, graphs[gi][0]))], np.int64)))
        return out

    total, arcs = time_reference_pool(args, directory, len(graphs), tasks)
    remove_graphs(directory, len(graphs))
    value = arcs / total / 1e9
    line = reference_line(args, "APSP+Brandes GTEPS (uneven multi-graph batch)", "GTEPS", value, total,
                          dict(UNEVEN_BATCH, workload="uneven batch: 512 connectomes, N ~ U{500..20000}, out-degree ~ U[5,60]; "
                               f"host arm on graphs {indices}", parallelism=f"{cores} host processes x 1 thread"), cores, "port",
                          f"{per_step} sources per step ({per_step // cores} per process) over {len(graphs)} of the batch's graphs, APSP summaries + "
                          "histogram + Brandes, CPU restatement of the reference Dijkstra/Brandes")
    print(json.dumps(line), flush=True)


def run_reference_scc(args):
    """The reference's own StronglyConnectedComponents (Multistep, its default) built from source, once per step."""
    import oracle

    config = {**WORKLOAD, **workload_overrides(args), "workload": "strongly connected components of the synthetic connectome "
              f"N={args.n} (reference StronglyConnectedComponents, Multistep, one rank)"}
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build (oracle/_ref) is not present; build it with "
                          "__graft_entry__.build() where the reference sources are", "config": config}), flush=True)
        return
    c = make_graph(args.n, args.degree, args.length_scale, args.sigma)
    ref = oracle.Reference()
    with stdout_to_stderr():
        rg = ref.graph(c.n, c.row_ptr, c.col, np.ones(c.m, np.int32))  # SCC ignores the weights
        total = 0.0
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            rg.scc(3)
            if i >= args.warmup:
                total += time.perf_counter() - t0
    value = c.m * args.steps / total / 1e9
    line = reference_line(args, "SCC arcs per second (strongly connected components of one graph)", "G arcs/s", value, total,
                          dict(config, n=c.n, arcs=int(c.m)), 1, "reference",
                          "the whole graph once per step, reference StronglyConnectedComponents (Multistep) built from source, "
                          "one rank x one thread")
    print(json.dumps(line), flush=True)


_REF_WORKER = {}


def ref_worker_init(directory):
    """One reference graph per worker process, built by the reference's own in-memory DistributedGraph construction
    from the saved integer CSR; what the reference prints goes to stderr."""
    sys.path.insert(0, ROOT)
    import oracle

    os.dup2(2, 1)
    n = int(np.load(os.path.join(directory, "g0_row_ptr.npy")).size - 1)
    row_ptr, col, w = (np.load(os.path.join(directory, f"g0_{name}.npy")) for name in ("row_ptr", "col", "w"))
    _REF_WORKER["graph"] = oracle.Reference().graph(n, row_ptr, col, w.astype(np.int32))


def ref_worker(_):
    """One whole all-sources job in the reference: AllPairsShortestPath::compute_apsp with PriorityQueue Dijkstra
    (AllPairsShortestPath.h:54-57) and BrandesVariant::accumulate_betweenness (BrandesVariant.h:50-74)."""
    g = _REF_WORKER["graph"]
    t0 = time.perf_counter()
    g.apsp(inverse=False, queue=0)
    g.betweenness(0)
    return time.perf_counter() - t0


def c1_traversed_arcs(c):
    """Traversed arcs of one all-sources pass (sum over sources of the out-degrees of the reached vertices)."""
    import oracle

    return int(oracle.Restatement().apsp(oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w))["traversed_arcs"])


def run_reference_c1(args):
    """The plain small configuration on the host cores through the reference itself (built from source against
    single-rank shims): each step runs one whole all-sources APSP + Brandes job in every host process at once (the
    reference's hot path is single-threaded per rank and this one-rank build cannot split sources across processes)."""
    import multiprocessing as mp

    import oracle

    config = dict(WORKLOAD_C1)
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build (oracle/_ref) is not present; build it with "
                          "__graft_entry__.build() where the reference sources are", "config": config}), flush=True)
        return
    c = make_graph(0, 0, workload="c1")
    arcs_per_job = c1_traversed_arcs(c)
    cores = host_cores()
    directory = tempfile.mkdtemp(prefix="ngx_ref_")
    save_graphs(directory, [(c.n, c.row_ptr, c.col, c.w)])
    total = 0.0
    with mp.get_context("spawn").Pool(cores, initializer=ref_worker_init, initargs=(directory,)) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            pool.map(ref_worker, range(cores), chunksize=1)
            if i >= args.warmup:
                total += time.perf_counter() - t0
    remove_graphs(directory, 1)
    value = cores * arcs_per_job * args.steps / total / 1e9
    line = reference_line(args, "APSP+Brandes GTEPS (plain small graph, all sources)", "GTEPS", value, total,
                          dict(config, n=c.n, arcs=int(c.m), sources_per_step=c.n * cores,
                               parallelism=f"{cores} host processes x 1 rank x 1 thread, one whole job each per step"),
                          cores, "reference",
                          f"every step {cores} concurrent whole jobs (all {c.n} sources: compute_apsp with PriorityQueue Dijkstra + "
                          "BrandesVariant::accumulate_betweenness), the reference built from source, 1 rank x 1 thread each")
    print(json.dumps(line), flush=True)


def reference_single_core_c1(c):
    """The reference itself on one core: one whole all-sources APSP + Brandes job of the plain small graph."""
    import oracle

    if not oracle.Reference.available():
        return None
    arcs = c1_traversed_arcs(c)
    with stdout_to_stderr():
        g = oracle.Reference().graph(c.n, c.row_ptr, c.col, c.w.astype(np.int32))
        t0 = time.perf_counter()
        g.apsp(inverse=False, queue=0)
        g.betweenness(0)
        dt = time.perf_counter() - t0
    return {"value": arcs / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "reference",
            "sample": f"one whole all-sources job ({c.n} sources, APSP with PriorityQueue Dijkstra + Brandes), {dt:.2f} s, "
                      "the reference built from source, 1 rank x 1 thread"}


def cpu_baseline_single_core(c, sources, budget_s=12.0):
    """The CPU restatement on one core, source after source, until about `budget_s` seconds of work are done."""
    import oracle

    g = oracle.Csr.from_arrays(c.n, c.row_ptr, c.col, c.w)
    r = oracle.Restatement()
    arcs, done = 0, 0
    t0 = time.perf_counter()
    for s in sources:
        one = np.array([s], dtype=np.int64)
        a = r.apsp(g, sources=one, bins=HIST_BINS, hist_max=64.0)
        r.brandes(g, sources=one)
        arcs += a["traversed_arcs"]
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": arcs / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
            "sample": f"{done} sources of the same graph, APSP summaries + histogram + Brandes, {dt:.1f} s, single thread; "
                      "CPU restatement of the reference Dijkstra/Brandes (bit-exact with the reference on integer weights)"}


UNEVEN_BATCH = {"graphs": 512, "n_min": 500, "n_max": 20000, "degree_min": 5.0, "degree_max": 60.0, "length_scale": 0.1,
                "weights": "45% integer U{1..10}, 45% log-normal(0,1), 10% unit", "seed": 3, "hist_max": 200.0}


def uneven_batch_specs():
    """(n, mean degree, weight kind) of each of the uneven batch's 512 seeded connectomes."""
    cfg = UNEVEN_BATCH
    rng = np.random.default_rng(cfg["seed"])
    specs = []
    for i in range(cfg["graphs"]):
        n = int(rng.integers(cfg["n_min"], cfg["n_max"] + 1))
        deg = float(rng.uniform(cfg["degree_min"], cfg["degree_max"]))
        u = rng.random()
        kind = "int" if u < 0.45 else ("lognormal" if u < 0.9 else "unit")
        specs.append((n, deg, kind))
    return specs


def uneven_batch_graphs(rank=0, world=1, indices=None):
    """The uneven-batch workload: 512 seeded connectomes (rank r builds graphs r, r + world, ...; or only `indices`)."""
    from neurograph_b200 import synth

    cfg = UNEVEN_BATCH
    specs = uneven_batch_specs()
    graphs = []
    use_gpu = True
    if indices is not None:
        import torch

        use_gpu = torch.cuda.is_available()  # a sample for the host arm: the CPU sampler where there is no GPU
    for i in (range(rank, cfg["graphs"], world) if indices is None else indices):
        n, deg, kind = specs[i]
        # the dense sampler on the GPU: its O(n^2) CPU form takes over half an hour for the 512 graphs
        c = synth.connectome(n, deg, cfg["length_scale"], weights=kind, seed=10_000 + i, use_gpu=use_gpu)
        graphs.append((c.n, c.row_ptr, c.col, c.w))
    return graphs


def run_uneven_batch(args, ngx, torch, rank, world, barrier, max_over_ranks, sum_over_ranks, local_rank):
    """All sources of every graph of the batch per step (APSP summaries + histogram + Brandes), one persistent launch,
    replayed from a captured CUDA graph after the first step."""
    t0 = time.perf_counter()
    graphs = uneven_batch_graphs(rank, world)
    m_total = sum(int(g[2].size) for g in graphs)
    log(f"[bench] {len(graphs)} graphs, {m_total} arcs generated in {time.perf_counter() - t0:.1f}s")
    torch.cuda.empty_cache()
    stream = torch.cuda.Stream()
    b = ngx.Batch(graphs, device=local_rank)
    b.set_stream(stream.cuda_stream)
    run = dict(task="brandes", hist_bins=HIST_BINS, hist_max=UNEVEN_BATCH["hist_max"], use_cuda_graph=True)
    for _ in range(args.warmup):
        b.run(**run)
    clocks = ClockSampler(local_rank)
    pause_gc()
    clocks.start()
    clocks.wait_first_sample()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    arcs, kernel_ms = 0, 0.0
    for _ in range(args.steps):
        results, _ = b.run(**run)
        arcs += sum(r.traversed_arcs for r in results)
        kernel_ms += results[0].kernel_ms if results else 0.0
    ev1.record(stream)
    barrier()
    clock_info = clocks.stop()
    gc.enable()
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    value = sum_over_ranks(float(arcs)) / elapsed / 1e9
    reached = 0
    for (n, rp, c, w), r in zip(graphs, results):
        reached += r.reached_pairs + n
    per_arc, per_vertex = 76.0, 56.0
    alg = (per_arc * arcs + per_vertex * reached * args.steps) / args.steps
    peak, peak_kind = measured_peaks()
    achieved = alg / (kernel_ms / args.steps / 1e3) / 1e9
    # the e2e job builds its own handle: release this one's graphs and workspaces first
    b.close()
    torch.cuda.synchronize()
    e2e = None
    if not args.no_e2e:
        pinned = [(n, torch.from_numpy(rp).pin_memory().numpy(), torch.from_numpy(c).pin_memory().numpy(),
                   torch.from_numpy(w).pin_memory().numpy()) for n, rp, c, w in graphs]
        h2d = sum(rp.nbytes + c.nbytes + w.nbytes for _, rp, c, w in pinned)
        barrier()
        pause_gc()
        t1 = time.perf_counter()
        with ngx.Batch(pinned, device=local_rank) as be:
            res, extra = be.run(task="brandes", hist_bins=HIST_BINS, hist_max=UNEVEN_BATCH["hist_max"])
        barrier()
        e2e_elapsed = max_over_ranks(time.perf_counter() - t1)
        gc.enable()
        d2h = sum(x.nbytes for x in extra) + sum(r.hist.nbytes for r in res)
        e2e = {"value": sum_over_ranks(float(sum(r.traversed_arcs for r in res))) / e2e_elapsed / 1e9, "unit": "GTEPS",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "timing": "wall clock, synchronized; batch created from pinned host CSRs, one all-sources run, results to host"}
    if rank != 0:
        return
    line = {
        "metric": "APSP+Brandes GTEPS (uneven multi-graph batch)", "value": value, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(UNEVEN_BATCH, workload="uneven batch: 512 connectomes, N ~ U{500..20000}, out-degree ~ U[5,60], "
                       "kernel exp(-d/0.1), mixed weights; all-source APSP + 1024-bin histogram + Brandes per graph, one "
                       "persistent launch replayed from a CUDA graph", arcs=m_total, graphs_on_rank0=len(graphs),
                       l2="workspaces (GBs) exceed the 126 MB L2; no flush needed"),
        "gpu_launches": args.steps * 2,
        "clocks": clock_info,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_label(peak_kind), "traffic": None,
                     "algorithmic_bytes_per_launch": alg, "kernel": "tile_kernel<Brandes> (ngx_batch_run)"},
        "e2e": e2e,
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


@contextlib.contextmanager
def stdout_to_stderr():
    """Sends what native code prints on fd 1 (the reference's timer reports) to stderr, keeping stdout to the one
    JSON line."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def run_scc(args, ngx, torch, rank, world, barrier, max_over_ranks, sum_over_ranks, local_rank):
    """Strongly connected components of the connectome per step (ngx_scc: trim, colour and peel passes), every rank
    on its own replica; the reference's StronglyConnectedComponents (Multistep, its default, and TarjanGathered) on the
    host beside it."""
    t0 = time.perf_counter()
    c = make_graph(args.n, args.degree, args.length_scale, args.sigma, args.workload)
    log(f"[bench] graph n={c.n} m={c.m} generated in {time.perf_counter() - t0:.1f}s")
    # a graph whose CSR + reverse CSR fit in L2 is timed step by step with L2 flushed between the steps (outside the
    # timed intervals); larger graphs and their workspaces exceed L2 by themselves
    graph_bytes = 2 * 16 * c.m + 2 * 8 * (c.n + 1)
    flush = graph_bytes < L2_BYTES
    flush_buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=f"cuda:{local_rank}") if flush else None
    torch.cuda.empty_cache()
    stream = torch.cuda.Stream()
    g = ngx.Graph(c.n, c.row_ptr, c.col, c.w, device=local_rank)
    g.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        first = g.scc()
    clocks = ClockSampler(local_rank)
    pause_gc()
    clocks.start()
    clocks.wait_first_sample()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        out = g.scc()
    ev1.record(stream)
    barrier()
    clock_info = clocks.stop()
    gc.enable()
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    arcs = int(c.m)
    value = sum_over_ranks(float(arcs * args.steps)) / elapsed / 1e9
    assert out["number_components"] == first["number_components"]
    # compulsory bytes of one call: both CSRs read once (4 B target per arc and direction, 8 B row offset per vertex
    # and direction) and the component array written once
    alg = 2 * (4 * arcs + 8 * c.n) + 4 * c.n
    peak, peak_kind = measured_peaks()
    achieved = alg / (elapsed / args.steps) / 1e9
    # the e2e job builds its own handle: release this one's graph and workspaces first (on the largest graphs the two
    # would not fit on the device together)
    g.close()
    torch.cuda.synchronize()
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(x).pin_memory().numpy() for x in (c.row_ptr, c.col, c.w)]
        barrier()
        pause_gc()
        t1 = time.perf_counter()
        with ngx.Graph(c.n, *pinned, device=local_rank) as ge:
            res = ge.scc()
        barrier()
        e2e_elapsed = max_over_ranks(time.perf_counter() - t1)
        gc.enable()
        e2e = {"value": sum_over_ranks(float(arcs)) / e2e_elapsed / 1e9, "unit": "G arcs/s",
               "h2d_bytes_per_step": int(sum(x.nbytes for x in pinned)), "d2h_bytes_per_step": int(res["component"].nbytes + 8 * (c.n + 3)),
               "timing": "wall clock, synchronized; graph handle created from pinned host CSR arrays, one ngx_scc call, "
                         "components and size histogram to host"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        if oracle.Reference.available():
            ref = oracle.Reference()
            with stdout_to_stderr():
                rg = ref.graph(c.n, c.row_ptr, c.col, np.ones(c.m, np.int32))  # SCC ignores the weights
                timings = {}
                for name, algorithm in (("multistep", 3), ("tarjan_gathered", 0)):
                    t1 = time.perf_counter()
                    got = rg.scc(algorithm)
                    timings[name] = time.perf_counter() - t1
                    if got["component_sizes"] != out["component_sizes"]:
                        raise RuntimeError(f"the reference's {name} SCC differs from ngx_scc")
            best = min(timings, key=timings.get)
            cpu = {"value": arcs / timings[best] / 1e9, "unit": "G arcs/s", "cores": 1, "kind": "reference",
                   "sample": f"the whole graph once per algorithm, reference StronglyConnectedComponents built from source "
                             f"(one rank): multistep {timings['multistep']:.3f} s, tarjan_gathered {timings['tarjan_gathered']:.3f} s; "
                             f"value from the faster ({best}); same component sizes as ngx_scc"}
    if rank != 0:
        return
    line = {
        "metric": "SCC arcs per second (strongly connected components of one graph)", "value": value, "unit": "G arcs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {**WORKLOAD, **workload_overrides(args), "workload": f"strongly connected components of the synthetic connectome "
                   f"N={c.n}, {c.m} arcs (ngx_scc per step, every rank on its own replica)", "n": c.n, "arcs": int(c.m),
                   "components": out["number_components"], "largest": out["largest_component_size"],
                   "l2": "graph arrays (both CSRs, ~16 B per arc each) exceed the 126 MB L2 at this size; no flush"},
        "gpu_launches": None,
        "clocks": clock_info,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_label(peak_kind), "traffic": None,
                     "algorithmic_bytes_per_launch": alg,
                     "kernel": "the whole ngx_scc call (trim, colour, peel passes with host-read change flags); bytes: "
                               "both CSRs read once + components written once"},
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    import neurograph_b200 as ngx

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_over_ranks(dist, x, "max", "cuda")

    def sum_over_ranks(x):
        return reduce_over_ranks(dist, x, "sum", "cuda")

    if args.workload in ("uneven-batch", "scc"):
        run = run_uneven_batch if args.workload == "uneven-batch" else run_scc
        run(args, ngx, torch, rank, world, barrier, max_over_ranks, sum_over_ranks, local_rank)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    t0 = time.perf_counter()
    c = make_graph(args.n, args.degree, args.length_scale, args.sigma, args.workload)
    log(f"[bench] graph n={c.n} m={c.m} generated in {time.perf_counter() - t0:.1f}s")
    # a graph whose CSR + reverse CSR fit in L2 is timed step by step with L2 flushed between the steps (outside the
    # timed intervals); larger graphs and their workspaces exceed L2 by themselves
    graph_bytes = 2 * 16 * c.m + 2 * 8 * (c.n + 1)
    flush = graph_bytes < L2_BYTES
    flush_buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=f"cuda:{local_rank}") if flush else None
    torch.cuda.empty_cache()  # the generator's cached blocks would otherwise shrink the library's workspace budget
    stream = torch.cuda.Stream()
    g = ngx.Graph(c.n, c.row_ptr, c.col, c.w, device=local_rank)
    g.set_stream(stream.cuda_stream)
    # one step = one wave of the all-sources job in the library's order (tiles of nearby sources)
    batches = source_batches(c.n, args.sources_per_step, args.warmup + args.steps, rank, world, order=g.source_order())
    tuning = None
    if args.autotune and args.mode in ("apsp", "brandes", "grad"):
        # the tuned width is passed on as an explicit delta, so that the e2e job's fresh handle runs with it too
        tuning = g.autotune(args.mode)
        args.delta = float(tuning["delta_scale"] * g.layout()["mean_lengths"][0])
        if (tuning["block_threads"], tuning["ctas_per_sm"]) != (512, 2):
            args.block_threads, args.ctas_per_sm = int(tuning["block_threads"]), int(tuning["ctas_per_sm"])
        log(f"[bench] autotune: {tuning} -> delta {args.delta:.6g}")

    # page-locked result arrays, allocated once and reused by every step (the device writes them directly, with no
    # staging copy and no first-touch page faults on freshly allocated host memory)
    def pinned(size):
        return torch.empty(max(size, 1), dtype=torch.float64).pin_memory().numpy()

    bc_out = pinned(c.n) if args.mode == "brandes" else None
    grad_out = (pinned(g.m), pinned(g.m)) if args.mode == "grad" else None

    def step(graph, sources, hist_max):
        """One step of the selected mode; returns (result, host outputs)."""
        if args.mode == "brandes":
            bc, r = graph.brandes(sources=sources, delta=args.delta, hist_bins=HIST_BINS, hist_max=hist_max, per_source=True,
                                  block_threads=args.block_threads, ctas_per_sm=args.ctas_per_sm, out=bc_out)
            return r, [bc]
        if args.mode == "grad":
            dcpl, deff, r = graph.apsp_grad(sources=sources, delta=args.delta, block_threads=args.block_threads, ctas_per_sm=args.ctas_per_sm,
                                            out=grad_out)
            return r, [dcpl, deff]
        mode = "plain" if args.mode == "plain" else "batched"
        r = graph.apsp(sources=sources, mode=mode, delta=args.delta if mode == "batched" else 0.1, hist_bins=HIST_BINS, hist_max=hist_max,
                       per_source=True, block_threads=args.block_threads, ctas_per_sm=args.ctas_per_sm)
        return r, []

    # histogram bound: sampled eccentricity x 1.5 from the first warm-up step, fixed for the timed steps
    hist_max = 0.0
    launches = 0       # tile-kernel launches (the roofline's unit)
    gpu_launches = 0   # all of the library's kernels in the timed region
    for i in range(args.warmup):
        r, _ = step(g, batches[i], hist_max)
        hist_max = r.hist_max if r.hist_max > 0 else hist_max
    clocks = ClockSampler(local_rank)
    pause_gc()
    clocks.start()
    clocks.wait_first_sample()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    arcs = 0
    reached = 0
    kernel_ms = 0.0
    step_events = []
    step_kernel_ms = []
    step_starts = []
    for i in range(args.warmup, args.warmup + args.steps):
        if flush:
            with torch.cuda.stream(stream):
                flush_buf.fill_(i)  # writes twice the L2 capacity
            step_starts.append(torch.cuda.Event(enable_timing=True))
            step_starts[-1].record(stream)
        t_host = time.perf_counter()
        r, _ = step(g, batches[i], hist_max)
        log(f"[bench] host call {1e3 * (time.perf_counter() - t_host):.1f} ms")
        arcs += r.traversed_arcs
        reached += r.reached_pairs + len(batches[i])
        kernel_ms += r.kernel_ms
        step_kernel_ms.append(r.kernel_ms)
        log(f"[bench] counters: phases {r.phases} expansions {r.expansions} lane_expansions {r.lane_expansions} "
            f"dag_levels {r.dag_levels} dag_entries {r.dag_entries} dag_scan_tiles {r.dag_scan_tiles} phase_cycles {list(r.phase_cycles)}")
        launches += 1
        gpu_launches += {"apsp": 1, "plain": 1, "brandes": 2, "grad": 3}[args.mode]  # + fixed-point conversions
        step_events.append(torch.cuda.Event(enable_timing=True))
        step_events[-1].record(stream)
    ev1.record(stream)
    barrier()
    clock_info = clocks.stop()
    gc.enable()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    prev = ev0
    for k, (e, kms) in enumerate(zip(step_events, step_kernel_ms)):
        log(f"[bench] step {k}: {prev.elapsed_time(e):.1f} ms, kernel {kms:.1f} ms")
        prev = e
    if flush:
        # the timed region is the steps alone: the flushes between them are not counted
        elapsed = sum(a.elapsed_time(b) for a, b in zip(step_starts, step_events)) / 1e3
    elapsed_max = max_over_ranks(elapsed)
    arcs_total = sum_over_ranks(float(arcs))
    value = arcs_total / elapsed_max / 1e9

    # roofline of the dominant kernel (the Brandes tile kernel), algorithmic bytes: SSSP 20 B per traversed arc
    # + 24 B per reached vertex; Brandes adds 56 B per arc + 32 B per vertex; the adjoint adds 84 B + 56 B
    per_arc, per_vertex = {"brandes": (76.0, 56.0), "grad": (104.0, 80.0), "apsp": (20.0, 24.0), "plain": (20.0, 24.0)}[args.mode]
    alg_bytes = per_arc * arcs + per_vertex * reached
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    traffic_per_arc = profiled_traffic_per_arc(args.mode)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_label(peak_kind),
                "traffic": None if traffic_per_arc is None else traffic_per_arc * arcs / launches,
                "algorithmic_bytes_per_launch": alg_bytes / launches,
                "kernel": {"brandes": "tile_kernel<Brandes> (ngx_brandes)", "grad": "tile_kernel<Grad> (ngx_apsp_grad)",
                           "apsp": "tile_kernel<Apsp> (ngx_apsp)", "plain": "sssp_plain_kernel (ngx_apsp, plain form)"}[args.mode]}

    # forms on the same graph: the plain per-source GPU form (one source per CTA) against the batched one, for APSP
    # and for APSP + histogram + Brandes (the same outputs as the timed steps)
    forms = {}
    if rank == 0 and not args.no_forms:
        sample = batches[0][: SLOTS_PER_WAVE * 4]
        rp = g.apsp(sources=sample, mode="plain", delta=0.1)
        rpb = g.brandes(sources=sample, mode="plain", delta=0.1, hist_bins=HIST_BINS, hist_max=hist_max)[1]
        rb = g.apsp(sources=batches[0], delta=args.delta, hist_bins=HIST_BINS, hist_max=hist_max)
        forms = {"plain_apsp_gteps": rp.gteps, "batched_apsp_gteps": rb.gteps, "plain_apsp_brandes_gteps": rpb.gteps,
                 "batched_apsp_brandes_gteps": arcs / (kernel_ms / 1e3) / 1e9,
                 "plain_sources": int(len(sample)), "batched_sources": int(len(batches[0]))}

    # e2e through the C ABI from host buffers: the job of K steps as a user runs it, all inside the timed region: the
    # graph is created from the pinned host CSR (uploaded once for the job), then every step passes its host source
    # list and reads its results (betweenness / gradients, per-source summaries, histogram) back, then the graph is
    # destroyed. The graph upload is counted in the per-step H2D bytes as its share over the K steps.
    # the e2e job builds its own handle: release this one's graph and workspaces first (on the largest graphs the two
    # would not fit on the device together)
    g.close()
    torch.cuda.synchronize()
    e2e = None
    if not args.no_e2e:
        pinned = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in (("row_ptr", c.row_ptr), ("col", c.col), ("w", c.w))}
        graph_bytes = pinned["row_ptr"].nbytes + pinned["col"].nbytes + pinned["w"].nbytes
        h2d = graph_bytes / args.steps + batches[0].nbytes
        d2h = 0
        barrier()
        pause_gc()
        t1 = time.perf_counter()
        e2e_arcs = 0
        with ngx.Graph(c.n, pinned["row_ptr"], pinned["col"], pinned["w"], device=local_rank) as ge:
            for i in range(args.warmup, args.warmup + args.steps):
                r, outs = step(ge, batches[i], hist_max)
                e2e_arcs += r.traversed_arcs
                d2h = sum(a.nbytes for a in outs) + (r.hist.nbytes if r.hist is not None else 0) + \
                    sum(a.nbytes for a in (r.per_source or {}).values())
        barrier()
        e2e_elapsed = max_over_ranks(time.perf_counter() - t1)
        gc.enable()
        e2e = {"value": sum_over_ranks(float(e2e_arcs)) / e2e_elapsed / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "timing": f"wall clock, synchronized; graph created from the pinned host CSR once for the {args.steps}-step job, "
                         "every step's sources from the host and results to the host"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = reference_single_core_c1(c) if args.workload == "c1" else cpu_baseline_single_core(c, batches[0])

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    metric = {"brandes": "APSP+Brandes GTEPS (batched single graph)", "apsp": "APSP GTEPS (batched single graph)",
              "grad": "APSP+gradient GTEPS (batched single graph)", "plain": "APSP GTEPS (plain per-source form)"}[args.mode]
    if args.workload == "c1":
        metric = metric.replace("batched single graph", "plain small graph, all sources")
    line = {
        "metric": metric, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(WORKLOAD, **workload_overrides(args), n=c.n, arcs=c.m, mode=args.mode, sources_per_step=args.sources_per_step, delta=args.delta,
                       **({"autotune": tuning} if tuning is not None else {}), hist_bins=HIST_BINS,
                       hist_max=hist_max, parallelism=f"sources sharded over {world} GPU(s), no data-path collective",
                       l2=(f"graph ({graph_bytes / 1e6:.1f} MB CSR + reverse CSR) fits in L2: L2 flushed between steps by a "
                           f"{2 * L2_BYTES >> 20} MiB write outside the timed intervals") if flush else
                          (f"graph ({graph_bytes / 1e6:.0f} MB CSR + reverse CSR) and workspaces (GBs) exceed the 126 MB L2; "
                           "no flush needed")),
        "gpu_launches": gpu_launches,
        "clocks": clock_info,
        "roofline": roofline,
        "forms": forms,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
