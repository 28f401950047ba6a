"""Benchmark of the BFS hot path on B200.

Default workload (the headline configuration): direction-optimising
single-source BFS on an undirected Graph500-style R-MAT graph, scale 24,
edge factor 16 (a=.57 b=.19 c=.19), self loops and duplicates removed, ids
permuted, generated on the GPU from a seed. One step = one BFS from each of
64 seeded non-isolated sources (the reference runs 64 sources per call,
bfs_gpu_opt.cuh:370). GTEPS follows the reference's convention: directed CSR
entries of the reached vertices (report(), validate.h:115-123) per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 runs under torchrun, one process per GPU. Sources are
independent, so every rank runs its own 64-source set on its own replica of
the graph (weak scaling, no data-path collective); timing is the max over ranks.
--impl reference times the CPU BFS (the oracle port: the reference has no CPU
BFS of its own, validate.h holds only a spot check) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RMAT = dict(a=0.57, b=0.19, c=0.19)
METRIC = "GTEPS, R-MAT s24 ef16; batched-vs-single-source GTEPS; p50/p99 query latency"


def graph_seed(scale):
    return 0x5EED0000 + scale


def source_seed(scale, rank=0):
    return 0x50C0000 + scale + 1000 * rank


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """Samples SM clock and throttle reasons with nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name: str):
    """Per-BFS DRAM bytes from the committed ncu summary (profiles/<name>)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith("dram_bytes_per_bfs:"):
                    return float(ln.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# --------------------------------------------------------------- ours -----
def run_ours(args, rank, world, dist):
    import torch
    import enterprise_b200 as eb

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    t0 = time.time()
    g = eb.Graph.rmat(args.scale, args.ef, seed=graph_seed(args.scale), gpu=local, **RMAT)
    gen_s = time.time() - t0
    V, E = g.vert_count, g.edge_count
    beg = np.empty(V + 1, dtype=np.int64)
    csr_h = None
    srcs = None
    # sources need the degree array; download offsets only
    full = g.download() if (rank == 0 and world == 1) else None
    if full is not None:
        beg, csr_h = full.beg_pos, full.csr
    else:
        beg = g.download().beg_pos
    srcs = eb.pick_sources(beg, source_seed(args.scale, rank), args.sources)

    stream = torch.cuda.Stream(device=local)
    sptr = stream.cuda_stream
    depth = torch.empty(V, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > L2 (126 MB)

    # per-source edges / levels (first pass also builds the workspace and the CUDA graph)
    stats = [g.bfs_device(int(s), depth.data_ptr(), 0, sptr) for s in srcs]
    m_c = np.array([st.traversed_edges for st in stats], dtype=np.float64)
    n_c = np.array([st.reached_vertices for st in stats], dtype=np.float64)
    levels = np.array([st.levels for st in stats])
    b_alg = 4 * m_c + 8 * n_c + 4 * V  # algorithmic bytes per BFS

    n = len(srcs)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]

    def step(timed: bool):
        flush.fill_(1)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for i, s in enumerate(srcs):
                ev[i][0].record(stream)
                g.bfs_device(int(s), depth.data_ptr(), 0, sptr, stats=False)
                ev[i][1].record(stream)
        stream.synchronize()
        return [ev[i][0].elapsed_time(ev[i][1]) for i in range(n)], ev[0][0].elapsed_time(ev[n - 1][1])

    for _ in range(args.warmup):
        step(False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    per_bfs = []
    step_ms = []
    for _ in range(args.steps):
        t_each, t_step = step(True)
        per_bfs.append(t_each)
        step_ms.append(t_step)
    clocks = clk.stop()
    if dist:
        dist.barrier()
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    edges_per_step = float(m_c.sum())
    value = world * edges_per_step * args.steps / (total_ms * 1e-3) / 1e9
    per = np.array(per_bfs)  # steps x sources (ms)
    mean_per_src = per.mean(axis=0)
    gteps_src = m_c / (mean_per_src * 1e-3) / 1e9
    hmean = len(gteps_src) / float(np.sum(1.0 / gteps_src))
    amean = float(np.mean(gteps_src))
    peak, peak_kind = measured_peak()
    achieved = float(b_alg.mean() / (mean_per_src.mean() * 1e-3) / 1e9)
    traffic = profiled_traffic("bfs_s24_rmat_traffic.txt")

    # ------------------------------------------------ e2e through the C ABI
    host_depth = np.empty(V, dtype=np.int32)
    try:
        eb.host_register(host_depth)
        pinned = True
    except Exception:
        pinned = False
    e2e_steps = max(1, min(args.steps, 3))
    for s in srcs[:4]:
        g.bfs(int(s), depth_out=host_depth)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for s in srcs:
            g.bfs(int(s), depth_out=host_depth)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * edges_per_step * e2e_steps / e2e_s / 1e9
    if pinned:
        eb.host_unregister(host_depth)

    # ------------------------------------------- CPU baseline (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(beg, csr_h, srcs, args, g, depth)

    launches = int(args.steps * np.sum(1 + 2 * levels)) * world
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic: seeded Graph500-parameter R-MAT generated on the GPU (no dataset)",
        "config": {
            "workload": f"direction-optimizing single-source BFS, R-MAT scale {args.scale} edge factor {args.ef}, "
                        f"{args.sources} seeded sources per step",
            "graph": {"vertices": V, "directed_entries": E, "generator_seed": graph_seed(args.scale)},
            "parallelism": f"replicas x{world} (sources independent, no collective on the data path)",
            "l2": "inputs larger than L2 (CSR %.2f GB) and a 256 MB L2 flush before every step" % (4 * E / 1e9),
            "graph_gen_s": round(gen_s, 2),
        },
        "gteps_harmonic_mean": round(hmean, 3),
        "gteps_arithmetic_mean": round(amean, 3),
        "gteps_graph500": round(value / 2, 3),
        "ms_per_bfs_median": round(float(np.median(mean_per_src)), 4),
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind,
            "traffic": traffic,
            "unit_of_work": "one BFS (one CUDA-graph launch: reset + [expand, inspect] x levels); "
                            "algorithmic bytes 4*m_c + 8*n_c + 4*V",
        },
        "e2e": {"value": round(e2e_value, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * len(srcs),
                "d2h_bytes_per_step": 4 * V * len(srcs), "api": "ent_bfs (C ABI) with host depth buffer",
                "host_buffer_pinned": pinned},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    return line


def cpu_baseline(beg, csr, srcs, args, g, depth):
    """Oracle port timed on the host cores over a bounded sample of sources;
    also checks the GPU depths of those sources bit-exact (checker use)."""
    import oracle
    threads = oracle.max_threads()
    budget_s = args.cpu_budget
    t_tot, e_tot, ran, ok = 0.0, 0.0, 0, True
    t1_tot, e1_tot = 0.0, 0.0
    for s in srcs:
        t0 = time.perf_counter()
        d = oracle.bfs_omp_do(beg, csr, int(s), threads=threads)
        dt = time.perf_counter() - t0
        e, _ = oracle.report(beg, d)
        t_tot += dt
        e_tot += e
        ran += 1
        gd = np.empty(len(beg) - 1, dtype=np.int32)
        g.bfs(int(s), depth_out=gd)
        ok = ok and bool(np.array_equal(gd, d))
        if ran == 1:  # one single-thread serial run for scale
            t0 = time.perf_counter()
            oracle.bfs(beg, csr, int(s))
            t1_tot = time.perf_counter() - t0
            e1_tot = e
        if t_tot + t1_tot > budget_s:
            break
    return {"value": round(e_tot / t_tot / 1e9, 4), "unit": "GTEPS", "cores": threads, "kind": "port",
            "sample": f"{ran} of the {len(srcs)} sources, direction-optimizing OpenMP CPU BFS on {threads} threads",
            "single_thread_serial_gteps": round(e1_tot / t1_tot / 1e9, 4) if t1_tot else None,
            "gpu_depths_bit_exact_on_sample": ok}


# ----------------------------------------------------------- reference ----
def run_reference(args, rank, world):
    """CPU BFS (oracle port; the reference has no CPU BFS) on all host threads,
    same graph and sources; each step is a bounded sample (one source)."""
    if rank != 0:
        return None
    import enterprise_b200 as eb
    import oracle
    t0 = time.time()
    csr = eb.Csr.rmat(args.scale, args.ef, seed=graph_seed(args.scale), **RMAT)
    gen_s = time.time() - t0
    srcs = eb.pick_sources(csr.beg_pos, source_seed(args.scale), args.sources)
    threads = oracle.max_threads()
    def one(i):
        s = int(srcs[i % len(srcs)])
        t = time.perf_counter()
        d = oracle.bfs_omp_do(csr.beg_pos, csr.csr, s, threads=threads)
        dt = time.perf_counter() - t
        return oracle.report(csr.beg_pos, d)[0], dt
    for i in range(args.warmup):
        one(i)
    edges, secs = 0.0, 0.0
    for i in range(args.steps):
        e, dt = one(args.warmup + i)
        edges += e
        secs += dt
    value = edges / secs / 1e9
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * secs / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic: seeded Graph500-parameter R-MAT built on the host (same CSR as the GPU arm)",
        "config": {"workload": f"direction-optimizing single-source BFS, R-MAT scale {args.scale} edge factor "
                               f"{args.ef}, {args.sources} seeded sources",
                   "graph": {"vertices": csr.vert_count, "directed_entries": csr.edge_count},
                   "graph_gen_s": round(gen_s, 2)},
        "cpu_baseline": {"value": round(value, 4), "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"one source per step ({args.steps} timed, {args.warmup} warm-up), "
                                   "direction-optimizing OpenMP CPU BFS (oracle port; the reference has no CPU BFS)"},
        "e2e": {"value": round(value, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":
        import torch
        import torch.distributed as tdist
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                 timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_ours(args, rank, world, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
