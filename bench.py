"""Benchmark: classic label propagation, GTEPS per iteration, R-MAT scale 24.

Workload (the reference's headline configuration for this path): R-MAT
scale 24 (16.8M vertices), edge factor 16, a/b/c/d = .57/.19/.19/.05,
seed 2, symmetrised, self loops and duplicates removed, degree-descending
relabel, int32 CSR; classic LP (method 1), labels = vertex ids at the start,
20 synchronous iterations.  A bench "step" is one such 20-iteration run over
the device-resident graph.  GTEPS = CSR entries x iterations / seconds.

* value: device time (CUDA events on the launching stream) of K steps with
  the graph already in HBM; the CSR (~1.9 GB) is larger than L2, so no
  explicit flush is done between steps.
* e2e: the same metric through the public API with host buffers: every step
  copies the CSR from pinned host memory (glp_graph_create), runs, and reads
  the labels back into a pinned host buffer.
* roofline: the dominant kernel group in the steps that count every vertex
  of the group (full-count steps; the other steps recount only majority
  failures or the neighbours of changed vertices), algorithmic bytes
  8*m_t + 12*n_t per launch over its CUDA-event launch time, against the
  measured HBM copy peak.  Tier times come from PROFILE_RUNS further runs
  after the timed region, with the step's kernels on one stream so that each
  tier's events bracket only its own kernels (the timed runs overlap tiers on
  three streams).  whole_step_roofline: 8m + 12n + 4 bytes per iteration over
  the mean iteration time of the timed runs.
* cpu_baseline: the reference's own OpenMP CPU path (tutorial/CPUlp.cuh,
  compiled from source into oracle/_ref) on the same graph: all iterations of
  one run from label = id, the same run --impl reference times.
* parity: the headline run's final labels against the CPU oracle.

Multi-GPU: each rank runs an independent replica (the path does not shard
across GPUs); value = total edges*iterations of all ranks / max rank time.

--impl reference times the reference's own CPU implementation instead
(rank 0 only): one step = one LP iteration, the steps being the iterations of
one run on the same graph, which it builds on the host without the engine.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

ITERS = 20
PROFILE_RUNS = 3  # untimed runs with per-tier CUDA events (roofline, tier times)
TIER_NAMES = ("tiny", "group16", "group32", "mid", "big", "hub", "aux", "majority")
TIER_PLAN_KEYS = {0: "tiny", 1: "group16", 2: "group32", 3: "mid", 4: "big", 5: "hub"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="glp", choices=["glp", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--iters", type=int, default=ITERS)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="classic",
                    choices=["classic", "batched", "served", "layered", "weighted", "slpa"],
                    help="classic: the R-MAT headline line (with a batched summary unless --no-batched); "
                         "batched / served: that workload alone; layered / weighted / slpa: one run of that path "
                         "on R-MAT --scale (SLPA: the overlapping planted graph of 2M vertices), for profiling")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the layered / weighted / SLPA measurements")
    ap.add_argument("--requests", type=int, default=300, help="served workload: requests per arrival rate")
    ap.add_argument("--rates", default="50,200", help="served workload: Poisson arrival rates (req/s)")
    ap.add_argument("--serve-seed", type=int, default=6)
    ap.add_argument("--graphs", type=int, default=4096, help="batched workload: number of graphs")
    ap.add_argument("--batch-seed", type=int, default=5)
    ap.add_argument("--plain-sample", type=int, default=256,
                    help="batched workload: graphs timed through the one-graph-at-a-time engine")
    return ap.parse_args()


# ----------------------------------------------------------------- distributed
def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(ws, x: float, op) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist
    # NCCL reduces device tensors; the gloo backend (CPU tests) host ones
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(ws, x: float) -> float:
    """The slowest rank's time: every multi-GPU figure is timed this way."""
    import torch.distributed as dist
    return _reduce(ws, x, dist.ReduceOp.MAX if ws > 1 else None)


def sum_over_ranks(ws, x: float) -> float:
    """Work done by all ranks together (weak scaling: each rank a replica)."""
    import torch.distributed as dist
    return _reduce(ws, x, dist.ReduceOp.SUM if ws > 1 else None)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.proc = None
        self.lines: list[str] = []
        try:
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            ident = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
        except Exception:
            ident = str(device)
        self.cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                    "-i", ident]

    def start(self):
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch per kernel tier from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


# ----------------------------------------------------------------- workload
def make_graph(scale: int, seed: int, device):
    from glp_b200 import graphs
    on_gpu = torch.device(device).type == "cuda"
    if on_gpu:
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = graphs.rmat(scale, 16, seed=seed, device=device)
    if on_gpu:
        torch.cuda.synchronize()
    return g, time.perf_counter() - t0


def workload_config(args, n: int, m: int) -> dict:
    """The workload's config object, identical in both arms."""
    return {"workload": f"rmat{args.scale}-ef16-seed{args.seed}-classic-{args.iters}it", "n": int(n), "m": int(m),
            "iterations_per_run": args.iters,
            "l2": "inputs larger than L2 (CSR %.2f GB); no flush" % ((4 * (n + 1 + m)) / 1e9)}


def write_csr(path: str, off: np.ndarray, cols: np.ndarray):
    with open(path, "wb") as f:
        np.array([len(off) - 1, len(cols)], dtype=np.int64).tofile(f)
        off.astype(np.int32).tofile(f)
        cols.astype(np.int32).tofile(f)


def cpu_threads() -> int:
    """Threads of the reference CPU path: CPUlp.cuh:50 hard-codes
    num_threads(20); OMP_THREAD_LIMIT caps it at the host's CPUs so that it is
    not oversubscribed (it cannot use more than 20 without editing it)."""
    return max(1, min(20, os.cpu_count() or 1))


def ref_cpulp_run(csr_path: str, niter: int, threads: int):
    """Run the reference CPUlp::sync_run_1 (oracle/_ref/ref_cpulp) for niter
    iterations from label = id; returns (per-iteration seconds as printed by
    the reference, final labels)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_cpulp")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    env = dict(os.environ)
    env["OMP_THREAD_LIMIT"] = str(threads)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "l.bin")
        r = subprocess.run([exe, "sync-csr", csr_path, str(niter), out], capture_output=True, text=True, env=env,
                           check=True)
        labels = np.fromfile(out, dtype=np.int32)
    return [float(x) for x in re.findall(r"t1: ([0-9.eE+-]+)", r.stdout)], labels


def cpu_reference_leg(args, off: np.ndarray, cols: np.ndarray, niter: int) -> dict:
    """The reference's own OpenMP CPU path (tutorial/CPUlp.cuh sync_run_1,
    compiled from source into oracle/_ref) on the workload graph: one run of
    niter iterations from label = id, iteration 0 included, timed by the
    reference's own per-iteration timer."""
    n, m = len(off) - 1, len(cols)
    threads = cpu_threads()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.csr")
        write_csr(path, off, cols)
        times, _ = ref_cpulp_run(path, niter, threads)
    t = sum(times)
    return {"value": round(m * len(times) / t / 1e9, 4), "unit": "GTEPS", "cores": threads, "kind": "reference",
            "iterations": len(times), "seconds": round(t, 2), "host_cpus": os.cpu_count(),
            "sample": f"reference CPUlp::sync_run_1 (tutorial/CPUlp.cuh, built from source), all {len(times)} "
                      f"iterations of one run from label = id on the full graph (n={n}, m={m}), {t:.1f} s; "
                      f"OMP_THREAD_LIMIT={threads} on a host with {os.cpu_count()} cpus"}


# ----------------------------------------------------------------- arms
def run_reference(args, ws, rank):
    """The reference's own CPU implementation of the path (no engine code: the
    graph is built on the host by the oracle's restatement of the sampler)."""
    if rank != 0:
        return
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_cpulp")):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_cpulp was not built"}))
        return
    from oracle import oracle as O
    t0 = time.perf_counter()
    off, cols = O.rmat_csr(args.scale, 16, seed=args.seed)
    gen_s = time.perf_counter() - t0
    n, m = len(off) - 1, len(cols)
    # one step = one CPU iteration; the steps are the first --steps iterations
    # (at most the workload's own count) of one run, iteration 0 included
    leg = cpu_reference_leg(args, off, cols, max(1, min(args.steps, args.iters)))
    steps = leg["iterations"]
    t = leg["seconds"]
    line = {
        "metric": f"classic LP GTEPS per iteration, R-MAT scale {args.scale}", "value": leg["value"],
        "unit": "GTEPS", "n_gpus": args.gpus, "steps": steps, "warmup": 0,
        "ms_per_step": round(1000 * t / max(steps, 1), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic R-MAT (seeded), generated on the host",
        "config": workload_config(args, n, m),
        "step": "one reference CPU iteration; the steps are iterations 0..%d of one run from label = id "
                "(a CPU iteration needs no warm-up, so --warmup %d is not applied)" % (steps - 1, args.warmup),
        "graph_gen_s": round(gen_s, 2),
        "impl": "reference",
        "cpu_baseline": {k: leg[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": leg["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# the engine's default step-mode thresholds (glp_params majority_permille /
# frontier_permille left at 0): a step after the first counts every vertex
# only when the previous step changed at least this many labels per 1000
# vertices (the rule of k_step_mode)
MAJORITY_PERMILLE = 500


def full_count_roofline(plan: dict, runs: list, n: int, peak: float,
                        majority_permille: int = MAJORITY_PERMILLE) -> dict:
    """Roofline of the dominant kernel group over the steps that count every
    vertex of the group.  A classic step after the first runs in full mode
    unless the previous step changed fewer than majority_permille labels per
    1000 vertices (then only the vertices that fail a majority test, or in
    frontier steps only the neighbours of changed vertices, are recounted);
    the first step of a graph with ascending rows is a closed form and
    launches no tier kernel.  Bytes per launch are the group's algorithmic
    bytes, 8 per CSR entry (column + neighbour label) and 12 per vertex
    (offsets, own label, written label)."""
    per = {}
    full_steps = 0
    for r in runs:
        ch = r.changed
        st = r.step_tier_ms
        if st is None:
            continue
        for it in range(1, len(ch)):
            if int(ch[it - 1]) * 1000 < majority_permille * n:
                continue
            full_steps += 1
            for t, key in TIER_PLAN_KEYS.items():
                per.setdefault(key, 0.0)
                per[key] += float(st[it][t])
    if not per or full_steps == 0:
        return {}
    key = max(per, key=per.get)
    n_t, m_t = plan[f"v_{key}"], plan[f"e_{key}"]
    bytes_launch = 8 * m_t + 12 * n_t
    avg_ms = per[key] / full_steps
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    groups = {}
    for k, ms in per.items():
        if ms <= 0:
            continue
        b = 8 * plan[f"e_{k}"] + 12 * plan[f"v_{k}"]
        a = b / (ms / full_steps / 1e3) / 1e9
        groups[k] = {"avg_ms": round(ms / full_steps, 4), "bytes_per_launch": int(b), "achieved_gbs": round(a, 1),
                     "frac": round(a / peak, 4)}
    return {"kernel": f"k_{key}", "bytes_per_launch": int(bytes_launch), "avg_launch_ms": round(avg_ms, 4),
            "achieved": round(achieved, 1), "frac": round(achieved / peak, 4), "full_count_launches": full_steps,
            "groups": groups}


def run_glp(args, ws, rank, local):
    from glp_b200 import _lib
    from glp_b200.engine import Graph, make_params
    from glp_b200.graphs import CSR

    dev = torch.device("cuda", local if ws > 1 else 0)
    g, gen_s = make_graph(args.scale, args.seed, dev)
    n, m = g.n, g.m
    # every iteration's step runs inside the timed region; the engine's
    # default stop at a two-step cycle (exact, fewer steps) is timed apart
    params = make_params(cycle_stop=-1)
    handle = Graph(g)
    plan = handle.plan(params)
    labels_dev = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    for _ in range(args.warmup):
        handle.run(_lib.METHOD_CLASSIC, args.iters, params, labels_out=labels_dev, stream=sp)
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(dev.index)
    clocks.start()
    tier_ms = np.zeros(8)
    launches = 0
    barrier(ws)
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        r = handle.run(_lib.METHOD_CLASSIC, args.iters, params, labels_out=labels_dev, stream=sp)
        launches += r.launches
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    # per-tier kernel times, outside the timed region: the same run with every
    # kernel of a step on one stream (serial_step), so that a tier's CUDA-event
    # time is its kernels' own duration, not a span shared with the tiers
    # running beside it
    prof_params = make_params(serial_step=1, cycle_stop=-1)
    prof_runs = []
    for _ in range(PROFILE_RUNS):
        r = handle.run(_lib.METHOD_CLASSIC, args.iters, prof_params, labels_out=labels_dev, stream=sp, profile=True)
        tier_ms += r.tier_ms
        prof_runs.append(r)
    torch.cuda.synchronize(dev)
    # the engine's default parameters: a run stops stepping once a step ends
    # in a two-step cycle (the later labelings are the last two in turn)
    dflt = make_params()
    for _ in range(args.warmup):
        handle.run(_lib.METHOD_CLASSIC, args.iters, dflt, labels_out=labels_dev, stream=sp)
    barrier(ws)
    torch.cuda.synchronize(dev)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    cyc_launches = 0
    for _ in range(args.steps):
        r = handle.run(_lib.METHOD_CLASSIC, args.iters, dflt, labels_out=labels_dev, stream=sp)
        cyc_launches += r.launches
    c1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    cyc_ms = max_over_ranks(ws, c0.elapsed_time(c1))
    cyc_value = sum_over_ranks(ws, float(m) * args.iters * args.steps) / (cyc_ms / 1e3) / 1e9
    ms_max = max_over_ranks(ws, ms)
    edges_total = sum_over_ranks(ws, float(m) * args.iters * args.steps)
    value = edges_total / (ms_max / 1e3) / 1e9

    # end to end through the public API with host buffers
    off_h = g.offsets.cpu().pin_memory()
    cols_h = g.cols.cpu().pin_memory()
    host_csr = CSR(off_h, cols_h, None, g.symmetric)
    lab_pin = torch.empty(n, dtype=torch.int32).pin_memory()  # the client's result buffer
    for _ in range(1):  # warm the host path once
        h2 = Graph(host_csr)
        h2.run(_lib.METHOD_CLASSIC, args.iters, params, labels_out=lab_pin)
        h2.close()
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    parts = {"create_ms": 0.0, "run_ms": 0.0, "destroy_ms": 0.0}
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        h2 = Graph(host_csr)
        t1 = time.perf_counter()
        h2.run(_lib.METHOD_CLASSIC, args.iters, params, labels_out=lab_pin)
        t2 = time.perf_counter()
        h2.close()
        t3 = time.perf_counter()
        parts["create_ms"] += (t1 - t0) * 1e3 / args.e2e_steps
        parts["run_ms"] += (t2 - t1) * 1e3 / args.e2e_steps
        parts["destroy_ms"] += (t3 - t2) * 1e3 / args.e2e_steps
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(ws, e0.elapsed_time(e1))
    e2e_edges = sum_over_ranks(ws, float(m) * args.iters * args.e2e_steps)
    e2e_value = e2e_edges / (e2e_ms / 1e3) / 1e9
    dev_labels = labels_dev.cpu().numpy()
    same = bool(np.array_equal(lab_pin.numpy(), dev_labels))

    # roofline of the dominant kernel group, over the steps that count every
    # vertex of the group (full-count steps)
    peak, peak_kind = measured_peak()
    launches_per_tier = PROFILE_RUNS * args.iters
    roof = full_count_roofline(plan, prof_runs, n, peak)
    key = roof["kernel"][2:] if roof else "big"
    traffic = profiled_traffic().get("full_count_launch", {}).get(key)
    total_bytes_iter = 8 * m + 12 * n + 4
    iter_ms = ms / (args.steps * args.iters)

    cpu, parity, refgpu = None, None, None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        off_np, cols_np = off_h.numpy(), cols_h.numpy()
        try:
            cpu = cpu_reference_leg(args, off_np, cols_np, args.iters)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GTEPS", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}
        # the reference's own GPU kernels (header/kernel.cuh's five classic bin
        # kernels, driven by oracle/_ref/ref_gpu_lp with a correct plan) on
        # the same graph and GPU: device time of the same 20 iterations
        refgpu = None
        exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_lp")
        if os.path.exists(exe):
            try:
                with tempfile.TemporaryDirectory() as d:
                    path, lab_path = os.path.join(d, "g.csr"), os.path.join(d, "l.bin")
                    write_csr(path, off_np, cols_np)
                    r = subprocess.run([exe, "classic-time", path, str(args.iters), "-", lab_path],
                                       capture_output=True, text=True, check=True, timeout=900)
                    total = float(re.search(r"total_ms ([0-9.eE+-]+)", r.stdout).group(1))
                    ref_lab = np.fromfile(lab_path, dtype=np.int32)
                refgpu = {"value": round(m * args.iters / (total / 1e3) / 1e9, 3), "unit": "GTEPS",
                          "ms_per_run": round(total, 3),
                          "labels_differing_from_this_engine": int(np.count_nonzero(ref_lab != dev_labels)),
                          "what": "the reference's own classic bin kernels (header/kernel.cuh l_*_labelload, "
                                  "its thresholds and launch shapes) on this GPU, one run of the same iterations, "
                                  "CUDA events per step; labels differ where its medium/big lanes break ties "
                                  "differently"}
            except Exception as e:
                refgpu = {"value": None, "what": f"failed: {e}"}
        # parity of the headline run's final labels with the oracle (the
        # synchronous rule restated on the CPU), outside every timed region
        try:
            from oracle import oracle as O
            t0 = time.perf_counter()
            ref = O.classic_run(off_np, cols_np, args.iters)
            parity = {"labels_equal_oracle": bool(np.array_equal(ref, dev_labels)),
                      "mismatches": int(np.count_nonzero(ref != dev_labels)),
                      "oracle_s": round(time.perf_counter() - t0, 1),
                      "what": f"final labels after {args.iters} iterations vs the CPU oracle's synchronous rule"}
        except Exception as e:
            parity = {"labels_equal_oracle": None, "what": f"oracle failed: {e}"}

    if rank == 0:
        line = {
            "metric": f"classic LP GTEPS per iteration, R-MAT scale {args.scale}",
            "value": round(value, 3), "unit": "GTEPS", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic R-MAT (seeded), generated on the GPU",
            "config": workload_config(args, n, m),
            "step": f"one {args.iters}-iteration run over the device-resident graph, every iteration's step run",
            "parallelism": f"replicas{ws}", "graph_gen_s": round(gen_s, 2),
            "e2e": {"value": round(e2e_value, 3), "unit": "GTEPS", "h2d_bytes_per_step": int(4 * (n + 1 + m)),
                    "d2h_bytes_per_step": int(4 * n), "steps": args.e2e_steps, "labels_match_device_run": same,
                    "host_clock_parts": {k: round(v, 2) for k, v in parts.items()}},
            "gpu_launches": int(launches),
            "with_cycle_stop": {"value": round(cyc_value, 3),
                                "ms_per_step": round(cyc_ms / args.steps, 3),
                                "launches_per_run": int(cyc_launches // max(args.steps, 1)),
                                "launches_per_run_every_step": int(launches // max(args.steps, 1)),
                                "how": "the engine's default parameters: a run stops stepping once a step ends in "
                                       "a two-step cycle; the same final labels"},
            "roofline": {"bound": "hbm", "achieved": roof.get("achieved"), "peak": peak, "unit": "GB/s",
                         "frac": roof.get("frac"), "traffic": traffic, "kernel": roof.get("kernel"),
                         "peak_kind": peak_kind, "bytes_per_launch": roof.get("bytes_per_launch"),
                         "avg_launch_ms": roof.get("avg_launch_ms"),
                         "launches": roof.get("full_count_launches"),
                         "how": "full-count steps only (every vertex of the group counted), serialised "
                                "per-tier CUDA events of %d untimed runs" % PROFILE_RUNS,
                         "groups": roof.get("groups")},
            "whole_step_roofline": {"bytes_per_iter": int(total_bytes_iter), "iter_ms": round(iter_ms, 4),
                                    "achieved_gbs": round(total_bytes_iter / (iter_ms / 1e3) / 1e9, 1),
                                    "frac": round(total_bytes_iter / (iter_ms / 1e3) / 1e9 / peak, 4)},
            "tier_ms_per_iter": {TIER_NAMES[i]: round(tier_ms[i] / launches_per_tier, 4) for i in TIER_PLAN_KEYS},
            "plan": plan,
            "clocks": clk,
            "cpu_baseline": cpu,
            "reference_gpu_kernels": refgpu,
            "parity": parity,
        }
    handle.close()
    del handle, labels_dev, g
    torch.cuda.empty_cache()
    if not args.no_batched:
        bl = run_batched(args, ws, rank, local)
        if rank == 0:
            line["batched"] = {k: bl[k] for k in ("metric", "value", "unit", "ms_per_step", "config", "plain",
                                                 "vs_plain", "e2e", "roofline", "cpu_baseline")}
    if not args.no_served:
        sv = run_served(args, ws, rank, local)
        if rank == 0:
            line["served"] = sv
    if not args.no_suite:
        su = run_suite(args, ws, rank, local)
        if rank == 0:
            line["suite"] = su
    if rank == 0:
        print(json.dumps(_with_summary(line)))


# ----------------------------------------------------------------- suite
def run_suite(args, ws, rank, local):
    """The other paths at scale, device time per run with the graph resident:
    layered LP (5 layers x 10 iterations, gamma 1..1/16 -> dstar 2,3,5,9,17)
    and classic LP, unweighted and with integer weights in [1, 16], on R-MAT
    scale 24 (seed 2) and on a planted partition of 10M vertices in 1,000
    communities (mean intra-degree 18, inter-degree 2, seed 3); SLPA (T = 20,
    r = 0.1, 20 iterations) on the overlapping planted graph of 2M vertices
    (2,000 communities, overlap 0.1, mean degree 24, seed 4).  Roofline bytes
    per iteration: classic 8m+12n+4, weighted +4m, layered 8m+16n+4 (+4m
    weighted), SLPA step 8m+16n+4."""
    from glp_b200 import _lib, graphs
    from glp_b200.engine import Graph, make_params

    dev = torch.device("cuda", local if ws > 1 else 0)
    peak, peak_kind = measured_peak()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    out = []

    def measure(name, g, method, niter, params, per_iter_bytes, iters_per_run):
        n, m = g.n, g.m
        with Graph(g) as h:
            lab = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            h.run(method, niter, params, labels_out=lab, stream=sp)  # warm-up
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 2
            e0.record(stream)
            for _ in range(reps):
                h.run(method, niter, params, labels_out=lab, stream=sp)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / reps
        it_ms = ms / iters_per_run
        gbs = per_iter_bytes / (it_ms / 1e3) / 1e9
        out.append({"workload": name, "n": n, "m": m, "ms_per_run": round(ms, 3), "iterations": iters_per_run,
                    "gteps_per_iter": round(m / (it_ms / 1e3) / 1e9, 2), "achieved_gbs": round(gbs, 1),
                    "frac": round(gbs / peak, 4), "bytes_per_iter": int(per_iter_bytes)})

    gammas = make_params(dstar=[2, 3, 5, 9, 17])
    for gname, builder in (("rmat24-seed2", lambda w: graphs.rmat(24, 16, seed=2, device=dev, weighted=w)),
                           ("planted10M-k1000-seed3",
                            lambda w: graphs.planted(10_000_000, 1000, 18.0, 2.0, seed=3, device=dev, weighted=w))):
        for weighted in (False, True):
            g = builder(weighted)
            n, m = g.n, g.m
            wb = 4 * m if weighted else 0
            tag = f"{gname}{'-weighted' if weighted else ''}"
            measure(f"classic-{tag}-20it", g, _lib.METHOD_CLASSIC, 20, make_params(cycle_stop=-1),
                    8 * m + 12 * n + 4 + wb, 20)
            measure(f"layered-{tag}-5x10it", g, _lib.METHOD_LAYERED, 10, gammas, 8 * m + 16 * n + 4 + wb, 50)
            del g
            torch.cuda.empty_cache()
    g = graphs.overlapping(2_000_000, 2000, 0.1, 24.0, seed=4, device=dev)
    measure("slpa-overlap2M-k2000-seed4-T20", g, _lib.METHOD_SLPA, 20,
            make_params(slpa_T=20, slpa_r=0.1, seed=4), 8 * g.m + 16 * g.n + 4, 20)
    del g
    torch.cuda.empty_cache()
    return {"peak_gbs": peak, "peak_kind": peak_kind, "runs": out,
            "how": "device time (CUDA events) of 2 runs after 1 warm-up run, graph resident, labels on the device; "
                   "classic runs run every iteration's step (no stop at a two-step cycle)"}


def run_one_path(args, ws, rank, local):
    """One path of the suite on its own (profiling): layered LP (5 layers x 3
    iterations, dstar 2,3,5,9,17) or weighted classic LP (20 iterations) on
    R-MAT --scale, or SLPA (T = 20, 20 iterations) on the overlapping planted
    graph of 2M vertices; --warmup runs, then --steps runs timed with CUDA
    events."""
    from glp_b200 import _lib, graphs
    from glp_b200.engine import Graph, make_params

    dev = torch.device("cuda", local if ws > 1 else 0)
    if args.workload == "slpa":
        g = graphs.overlapping(2_000_000, 2000, 0.1, 24.0, seed=4, device=dev)
        method, niter, params, per_iter = _lib.METHOD_SLPA, 20, make_params(slpa_T=20, slpa_r=0.1, seed=4), 20
    elif args.workload == "layered":
        g = graphs.rmat(args.scale, 16, seed=args.seed, device=dev)
        method, niter, params, per_iter = _lib.METHOD_LAYERED, 3, make_params(dstar=[2, 3, 5, 9, 17]), 15
    else:
        g = graphs.rmat(args.scale, 16, seed=args.seed, device=dev, weighted=True)
        method, niter, params, per_iter = _lib.METHOD_CLASSIC, args.iters, make_params(), args.iters
    stream = torch.cuda.current_stream(dev)
    with Graph(g) as h:
        lab = torch.empty(g.n, dtype=torch.int32, device=dev)
        for _ in range(max(args.warmup, 1)):
            h.run(method, niter, params, labels_out=lab, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            h.run(method, niter, params, labels_out=lab, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    return {"workload": args.workload, "n": g.n, "m": g.m, "ms_per_run": round(ms, 3),
            "gteps_per_iter": round(g.m * per_iter / (ms / 1e3) / 1e9, 2)}


# ----------------------------------------------------------------- served
def served_requests(count: int, seed: int, device):
    """The served workload (seed 6): a pool of graphs (24 planted-partition
    graphs of 10k-100k vertices, R-MAT scales 20-23) and `count` requests
    over it: 80 % planted / 20 % R-MAT, methods 60 % classic, 25 % layered
    (3 layers, dstar 2/3/5), 15 % SLPA (T = niter, r = 0.1), niter 10 or 20.
    Counter based: request i depends only on (seed, i)."""
    from glp_b200 import graphs
    from glp_b200.engine import make_params
    from glp_b200.graphs import _splitmix64

    specs = graphs.batch_specs(24, seed, n_range=(10000, 100000))
    pool_p = [graphs.planted(s["n"], s["k"], s["intra"], s["inter"], s["seed"], device=device).to("cpu")
              for s in specs]
    pool_r = [graphs.rmat(sc, 16, seed=seed * 100 + sc, device=device).to("cpu") for sc in (20, 21, 22, 23)]
    torch.cuda.empty_cache()
    pool = pool_p + pool_r
    reqs = []
    for i in range(count):
        u = [_splitmix64(_splitmix64(seed ^ 0xABCDEF) ^ (i * 8 + j)) / 2.0 ** 64 for j in range(6)]
        g = pool_p[int(u[1] * len(pool_p))] if u[0] < 0.8 else pool_r[int(u[1] * len(pool_r))]
        niter = 10 if u[3] < 0.5 else 20
        if u[2] < 0.60:
            method, params = 1, None
        elif u[2] < 0.85:
            method, params = 2, make_params(dstar=[2, 3, 5])
        else:
            method, params = 3, make_params(slpa_T=niter, slpa_r=0.1, seed=seed)
        reqs.append({"g": g, "gi": next(k for k, x in enumerate(pool) if x is g), "method": method, "niter": niter,
                     "params": params, "u_gap": u[4]})
    return reqs, pool


def _with_summary(line: dict) -> dict:
    """The line with a compact "summary" right after "config": the figures of
    the long objects at its end (baselines, parity, batched, served, suite)
    in a few hundred bytes, so that a reader of a truncated line sees them."""
    sm = {}
    cpu, ref = line.get("cpu_baseline"), line.get("reference_gpu_kernels")
    if isinstance(cpu, dict):
        sm["cpu_baseline_gteps"] = cpu.get("value")
    if isinstance(ref, dict):
        sm["reference_gpu_kernels_gteps"] = ref.get("value")
    if "parity" in line:
        sm["parity"] = line["parity"].get("labels_equal_oracle") if isinstance(line["parity"], dict) else None
    rf = line.get("roofline")
    if isinstance(rf, dict):
        sm["roofline_frac"] = rf.get("frac")
    cs = line.get("with_cycle_stop")
    if isinstance(cs, dict):
        sm["with_cycle_stop_gteps"] = cs.get("value")
    b = line.get("batched")
    if isinstance(b, dict):
        sm["batched_graphs_per_s"] = b.get("value")
        sm["batched_vs_plain"] = b.get("vs_plain")
    sv = line.get("served")
    if isinstance(sv, dict):
        sm["served"] = [{"rate": r["rate"], "throughput": r["served"]["throughput"],
                         "sequential_throughput": r["sequential"]["throughput"],
                         "vs_sequential": r["throughput_vs_sequential"], "p50_ms": r["served"]["p50_ms"],
                         "sequential_p50_ms": r["sequential"]["p50_ms"]} for r in sv.get("rates", [])]
    su = line.get("suite")
    if isinstance(su, dict):
        sm["suite_gteps"] = {r["workload"]: r["gteps_per_iter"] for r in su.get("runs", [])}
    out = {}
    for k, v in line.items():
        out[k] = v
        if k == "config":
            out["summary"] = sm
    return out


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def run_served(args, ws, rank, local):
    """Open-loop Poisson arrivals at each rate; the native server (continuous
    batching into the persistent kernel + overlapping one-graph solves)
    against a sequential one-request-at-a-time engine on the same schedule.
    Latency = completion - scheduled arrival."""
    from glp_b200.engine import Graph
    from glp_b200.server import Server

    dev = torch.device("cuda", local if ws > 1 else 0)
    t0 = time.time()
    reqs, pool = served_requests(args.requests, args.serve_seed, dev)
    gen_s = time.time() - t0
    rates = [float(x) for x in args.rates.split(",") if x]
    out = []
    for rate in rates:
        arrivals = np.cumsum([-np.log(max(1e-12, 1.0 - r["u_gap"])) / rate for r in reqs])
        arrivals -= arrivals[0]
        # served: the pool is resident (uploaded before the stream starts);
        # one unpaced pass over the requests warms the server (its workers'
        # cached handles, per-method buffers and batch buffers), as the
        # sequential engine below is warmed
        with Server() as srv:
            gids = [srv.add_graph(g) for g in pool]
            warm = [srv.submit_graph(gids[r["gi"]], r["method"], r["niter"], r["params"]) for r in reqs]
            for h in warm:
                srv.wait(h)
            rounds0 = srv.info()["rounds"]
            handles, lags = [], []
            start = time.perf_counter()
            for r, at in zip(reqs, arrivals):
                wait = start + at - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                lags.append(time.perf_counter() - (start + at))
                handles.append(srv.submit_graph(gids[r["gi"]], r["method"], r["niter"], r["params"]))
            stats = [srv.wait(h) for h in handles]
            rounds = srv.info()["rounds"] - rounds0
        lat = [(st["done_s"] - st["submit_s"] + lag) * 1e3 for st, lag in zip(stats, lags)]
        span = max(st["done_s"] for st in stats) - min(st["submit_s"] for st in stats)
        served = {"throughput": round(len(reqs) / span, 1), "p50_ms": round(_pct(lat, 50), 2),
                  "p99_ms": round(_pct(lat, 99), 2), "rounds": int(rounds),
                  "batched_frac": round(sum(st["path"] == 1 for st in stats) / len(stats), 3)}
        # sequential one-request-at-a-time engine, same schedule, the same
        # graphs resident (one handle each, created before the stream)
        lat_s, same, service = [], True, []
        resident = [Graph(g) for g in pool]
        for r in reqs:  # the same unpaced warm-up pass
            resident[r["gi"]].run(r["method"], r["niter"], r["params"])
        start = time.perf_counter()
        for r, at, h in zip(reqs, arrivals, handles):
            wait = start + at - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            t_run = time.perf_counter()
            lab = resident[r["gi"]].run(r["method"], r["niter"], r["params"]).labels
            service.append(time.perf_counter() - t_run)
            lat_s.append((time.perf_counter() - (start + at)) * 1e3)
            same = same and bool(np.array_equal(lab, h.labels))
        span_s = (time.perf_counter() - start)
        for gh in resident:
            gh.close()
        seq = {"throughput": round(len(reqs) / span_s, 1), "p50_ms": round(_pct(lat_s, 50), 2),
               "p99_ms": round(_pct(lat_s, 99), 2)}
        # where the sequential engine's time goes, per request class: the
        # served speed-up this mix can reach is bounded by the classes that
        # batching does not shorten
        classes = {}
        for r, t in zip(reqs, service):
            key = ("planted" if r["g"].n <= 100000 else "rmat") + "-" + {1: "classic", 2: "layered", 3: "slpa"}[
                r["method"]]
            c = classes.setdefault(key, {"requests": 0, "service_s": 0.0})
            c["requests"] += 1
            c["service_s"] += t
        total_s = sum(service)
        for c in classes.values():
            c["mean_ms"] = round(1e3 * c["service_s"] / c["requests"], 3)
            c["share"] = round(c["service_s"] / total_s, 4)
            c["service_s"] = round(c["service_s"], 3)
        unbatched = sum(c["service_s"] for k, c in classes.items() if k != "planted-classic")
        # latency percentiles per class, served and sequential: where the
        # served path gains or loses against one request at a time
        by_class = {}
        for r, ls, lq in zip(reqs, lat, lat_s):
            key = ("planted" if r["g"].n <= 100000 else "rmat") + "-" + {1: "classic", 2: "layered", 3: "slpa"}[
                r["method"]]
            c = by_class.setdefault(key, {"served": [], "sequential": []})
            c["served"].append(ls)
            c["sequential"].append(lq)
        latency_by_class = {k: {"requests": len(v["served"]), "served_p50_ms": round(_pct(v["served"], 50), 2),
                                "served_p99_ms": round(_pct(v["served"], 99), 2),
                                "sequential_p50_ms": round(_pct(v["sequential"], 50), 2),
                                "sequential_p99_ms": round(_pct(v["sequential"], 99), 2)}
                            for k, v in by_class.items()}
        out.append({"rate": rate, "served": served, "sequential": seq, "latency_by_class": latency_by_class,
                    "throughput_vs_sequential": round(served["throughput"] / seq["throughput"], 2),
                    "labels_match_alone": same, "sequential_service_by_class": classes,
                    "bound_if_batched_classes_were_free": round(total_s / max(unbatched, 1e-9), 2)})
    mix = {"planted": round(sum(r["g"].n <= 100000 for r in reqs) / len(reqs), 3),
           "classic": round(sum(r["method"] == 1 for r in reqs) / len(reqs), 3),
           "layered": round(sum(r["method"] == 2 for r in reqs) / len(reqs), 3),
           "slpa": round(sum(r["method"] == 3 for r in reqs) / len(reqs), 3)}
    return {"metric": "served LP throughput (req/s) and p50/p99 latency, open-loop Poisson arrivals",
            "unit": "req/s", "requests": len(reqs), "seed": args.serve_seed, "mix": mix, "rates": out,
            "graph_gen_s": round(gen_s, 2),
            "how": "native server, graph pool resident: FIFO admission by a 150 GB HBM budget, small classic "
                   "requests in rounds of the persistent batched kernel (grids sized to the round), one-graph "
                   "requests expected below 20 ms on a short-job worker, the rest on one one-graph worker (shortest "
                   "job first) with cached handles; sequential = one request at a time through glp_run on resident "
                   "handles; both warmed by one unpaced pass over the requests before the timed stream"}


# ----------------------------------------------------------------- batched
def run_batched(args, ws, rank, local, embed=False):
    """The batched workload: `args.graphs` planted-partition graphs (vertex
    counts log-uniform in [1k, 200k], 4-64 communities, mean degree
    log-uniform in [4, 64], seed --batch-seed), 20 classic iterations each,
    all of them in one persistent launch per step (CUDA-graph replay, labels
    left on the device).  Against the one-graph-at-a-time engine on a
    systematic sample of the same graphs (handles resident, labels on the
    device), and, end to end, against packing from host buffers + a run with
    labels back to the host."""
    from glp_b200 import _lib, graphs
    from glp_b200.batch import Batch
    from glp_b200.engine import Graph, make_params

    dev = torch.device("cuda", local if ws > 1 else 0)
    t0 = time.time()
    gs = graphs.batch_planted(args.graphs, args.batch_seed, device=dev)
    torch.cuda.synchronize(dev)
    gen_s = time.time() - t0
    n = sum(g.n for g in gs)
    m = sum(g.m for g in gs)
    b = Batch(gs)
    t0 = time.time()
    best, cand_ms = b.tune(3)
    tune_s = time.time() - t0
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    out = torch.empty(max(b.n, 1), dtype=torch.int32, device=dev)
    pg = make_params(use_graph=1)
    for _ in range(args.warmup):
        b.run(args.iters, pg, labels_out=out, stream=sp, changed=False)
    torch.cuda.synchronize(dev)
    barrier(ws)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        b.run(args.iters, pg, labels_out=out, stream=sp, changed=False)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    ms = max_over_ranks(ws, ev0.elapsed_time(ev1))
    total_graphs = sum_over_ranks(ws, float(args.graphs * args.steps))
    value = total_graphs / (ms / 1e3)
    labels = out[:b.n].cpu().numpy()

    # plain engine: a systematic sample, handles resident, labels on the device
    idx = list(range(0, args.graphs, max(1, args.graphs // max(1, args.plain_sample))))
    hs = [Graph(gs[i]) for i in idx]
    outs = [torch.empty(max(h.n, 1), dtype=torch.int32, device=dev) for h in hs]
    for h, o in zip(hs[:4], outs[:4]):
        h.run(_lib.METHOD_CLASSIC, args.iters, labels_out=o, stream=sp)
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    for h, o in zip(hs, outs):
        h.run(_lib.METHOD_CLASSIC, args.iters, labels_out=o, stream=sp)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = ev0.elapsed_time(ev1)
    mismatch = sum(int(not np.array_equal(o[:h.n].cpu().numpy(), labels[b.vbase[i]:b.vbase[i + 1]]))
                   for i, h, o in zip(idx, hs, outs))
    for h in hs:
        h.close()
    del hs, outs
    plain_value = len(idx) / (plain_ms / 1e3)

    # end to end: host buffers in, packing + run + labels out, every step
    host = [graphs.CSR(g.offsets.cpu().pin_memory(), g.cols.cpu().pin_memory(), None, g.symmetric) for g in gs]
    h2d = int(sum(4 * (g.n + 1 + g.m) for g in gs))
    e2e_steps = max(1, min(args.e2e_steps, 2))
    torch.cuda.synchronize(dev)
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    same = True
    for _ in range(e2e_steps):
        with Batch(host) as bh:
            lab_h, _ = bh.run(args.iters, changed=False)
        same = same and bool(np.array_equal(lab_h, labels))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(ws, e0.elapsed_time(e1))
    e2e_value = sum_over_ranks(ws, float(args.graphs * e2e_steps)) / (e2e_ms / 1e3)
    del host

    # roofline: 8 B per CSR entry (column + gathered label), 8 B offset +
    # 4 B own label + 4 B written label per vertex, per iteration
    bytes_iter = 8 * m + 16 * n + 8
    iter_ms = ms / (args.steps * args.iters)
    peak, peak_kind = measured_peak()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            k = 4
            times = []
            with tempfile.TemporaryDirectory() as d:
                for g in gs[:k]:
                    path = os.path.join(d, "g.csr")
                    write_csr(path, g.offsets.cpu().numpy(), g.cols.cpu().numpy())
                    times.append(sum(ref_cpulp_run(path, args.iters, cpu_threads())[0]))
            cpu = {"value": round(k / sum(times), 3), "unit": "graphs/s", "cores": cpu_threads(),
                   "kind": "reference",
                   "sample": f"reference CPUlp::sync_run_1 (tutorial/CPUlp.cuh, built from source), first {k} graphs "
                             f"of the batch x {args.iters} iterations, {sum(times):.2f} s"}
        except Exception as e:
            cpu = {"value": None, "unit": "graphs/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    res = {
        "metric": f"batched classic LP graphs/s ({args.graphs} planted-partition graphs, {args.iters} iterations)",
        "value": round(value, 1), "unit": "graphs/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic planted-partition batch (seeded), generated on the GPU",
        "config": {"workload": f"batch{args.graphs}-planted-seed{args.batch_seed}-classic-{args.iters}it",
                   "graphs": args.graphs, "n": n, "m": m, "parallelism": f"replicas{ws}",
                   "l2": "inputs larger than L2 (CSR %.1f GB); no flush" % (4 * (n + 1 + m) / 1e9),
                   "launch": "one persistent cooperative launch per step, CUDA-graph replay",
                   "tuned": {"threads": best.batch_threads, "thread_tier_max": best.tiny_max,
                             "warp_tier_max": best.mid_max},
                   "tune_s": round(tune_s, 2), "graph_gen_s": round(gen_s, 2)},
        "plain": {"value": round(plain_value, 1), "unit": "graphs/s", "sample_graphs": len(idx),
                  "sample_vertex_frac": round(sum(gs[i].n for i in idx) / n, 4),
                  "labels_match_batch": mismatch == 0,
                  "how": "glp_run method 1 per graph, handles resident, labels on the device"},
        "vs_plain": round(value / plain_value, 2),
        "e2e": {"value": round(e2e_value, 1), "unit": "graphs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(4 * n), "steps": e2e_steps, "labels_match_device_run": same},
        "gpu_launches": int(args.steps),
        "roofline": {"bound": "hbm", "achieved": round(bytes_iter / (iter_ms / 1e3) / 1e9, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(bytes_iter / (iter_ms / 1e3) / 1e9 / peak, 4), "traffic": None,
                     "kernel": "k_batch", "peak_kind": peak_kind, "bytes_per_iter": int(bytes_iter),
                     "iter_ms": round(iter_ms, 4)},
        "cpu_baseline": cpu,
    }
    b.close()
    del gs
    torch.cuda.empty_cache()
    return res


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.workload == "batched":
        res = run_batched(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(res))
    elif args.workload == "served":
        res = run_served(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(res))
    elif args.workload in ("layered", "weighted", "slpa"):
        res = run_one_path(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(res))
    else:
        run_glp(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
