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


# Seed of rank `rank`'s source set (enterprise_b200.replicas.source_seed, kept
# here as well so that the CPU arm imports no product code; a test keeps the
# two equal).
SOURCE_SEED_BASE = 0x50C0000


def source_seed(scale, rank=0):
    return SOURCE_SEED_BASE + scale + 1000 * rank


def headline_config(args, V, E):
    """The workload both arms run, named the same way in both JSON lines."""
    return {
        "workload": f"direction-optimizing single-source BFS, R-MAT scale {args.scale} edge factor {args.ef}, "
                    f"{args.sources} seeded sources per step",
        "graph": {"vertices": int(V), "directed_entries": int(E), "generator_seed": graph_seed(args.scale),
                  "source_seed": source_seed(args.scale)},
        "l2": "inputs larger than L2 (CSR %.2f GB)" % (4 * E / 1e9),
    }


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


def profiled_traffic(name: str, key: str = "dram_bytes_per_bfs"):
    """A `key: value` figure from a committed ncu summary (profiles/<name>)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith(key + ":"):
                    return float(ln.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def profiled_options(name: str):
    """The traversal options an ncu summary was captured with (its `options:` line)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith("options:"):
                    return json.loads(ln.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


TRAFFIC_PROFILE = "bfs_rmat_s22_traffic.md"


def headline_traffic(run_opts: dict, E: int):
    """(DRAM bytes per traversal, basis) for the headline's roofline: the ncu
    capture's bytes scaled to this graph by directed entries, and only when
    this run traverses with the options the capture used."""
    want = profiled_options(TRAFFIC_PROFILE)
    per, e_prof = profiled_traffic(TRAFFIC_PROFILE), profiled_traffic(TRAFFIC_PROFILE, "directed_entries")
    if not want or not per or not e_prof:
        return None, f"no capture summary (profiles/{TRAFFIC_PROFILE})"
    differ = {k: (v, run_opts.get(k)) for k, v in want.items() if run_opts.get(k) != v}
    if differ:
        return None, f"this run's options differ from the capture's: {differ}"
    return per * E / e_prof, (f"ncu DRAM bytes per traversal (profiles/{TRAFFIC_PROFILE}, R-MAT s22, same "
                              f"options) x {E / e_prof:.3f} directed entries")


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
    tuned = None
    if not args.no_tune:
        from enterprise_b200 import tune
        t0 = time.time()
        tune_srcs = eb.pick_sources(beg, source_seed(args.scale, rank) + 0x7E57, 16)  # disjoint from the timed set
        cache = tune.TuneCache()
        key = tune.TuneCache.key(tune.gpu_name(local), tune.graph_class(V, E, "rmat"), "single")
        where = cache.source(key)
        opts, ms, hit = tune.autotune(g, tune_srcs, "single", reps=2, label="rmat", device=local, cache=cache)
        tuned = {"opts": {k: v for k, v in vars(opts).items() if k != "fault_inject"}, "cached": hit,
                 "cache": {"user": "this machine's tuning cache", "shipped": "the package's shipped results of an "
                           "earlier search on this GPU model (enterprise_b200/tuned/b200.json)"}.get(where, "searched now"),
                 "search_s": round(time.time() - t0, 2)}

    if args.opts:  # explicit traversal options (on top of the tuner's or the defaults)
        o = g.opts
        for k, v in json.loads(args.opts).items():
            setattr(o, k, type(getattr(o, k))(v))
        g.opts = o
    if args.loop != "graph":
        o = g.opts
        o.loop = eb.LOOP[args.loop]
        g.opts = o
    run_opts = {k: v for k, v in vars(g.opts).items() if k not in ("fault_inject", "loop")}

    stream = torch.cuda.Stream(device=local)
    sptr = stream.cuda_stream
    depth = torch.empty(V, dtype=torch.int32, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > L2 (126 MB)

    # per-source edges / levels (first pass also builds the workspace and the CUDA graph)
    stats = [g.bfs_device(int(s), depth.data_ptr(), 0, sptr) for s in srcs]
    m_c = np.array([st.traversed_edges for st in stats], dtype=np.float64)
    n_c = np.array([st.reached_vertices for st in stats], dtype=np.float64)
    levels = np.array([st.levels for st in stats])
    launches_per_step = int(sum(st.launches for st in stats))  # reset, level kernels, cluster kernel
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
    depth_ref_last = depth.cpu().numpy()  # the last source's depths from the device-timed run
    if dist:
        dist.barrier()
    from enterprise_b200 import replicas
    dev = f"cuda:{local}"
    edges_per_step = float(m_c.sum())
    job_edges, job_s, rate = replicas.job_rate(edges_per_step * args.steps, float(sum(step_ms)) * 1e-3, dist, dev)
    total_ms = job_s * 1e3
    value = rate / 1e9
    per = np.array(per_bfs)  # steps x sources (ms)
    mean_per_src = per.mean(axis=0)
    gteps_src = m_c / (mean_per_src * 1e-3) / 1e9
    hmean = len(gteps_src) / float(np.sum(1.0 / gteps_src))
    amean = float(np.mean(gteps_src))
    # the reference's own average: arithmetic, over sources whose traversal has
    # more than 2 levels (bfs_gpu_opt.cuh:411-431)
    deep = levels > 2
    amean_ref = float(np.mean(gteps_src[deep])) if deep.any() else None
    peak, peak_kind = measured_peak()
    achieved = float(b_alg.mean() / (mean_per_src.mean() * 1e-3) / 1e9)
    traffic, traffic_basis = headline_traffic(run_opts, E)  # DRAM bytes per traversal (ncu) or None
    physical = traffic / (mean_per_src.mean() * 1e-3) / 1e9 if traffic else None  # GB/s

    # ------------------------------------------------ e2e through the C ABI
    # The reference's per-source loop (traverse, copy the depths to the host)
    # as one call: ent_bfs_many_u8 returns the reference's own depth type (one
    # byte per vertex, 255 = unreached); ent_bfs_many returns int32 depths.
    # Each source's depths land in their own pinned host row; the copy of one
    # source overlaps the next traversal.
    src_list = [int(s) for s in srcs]
    e2e_steps = args.steps  # the same number of steps as the device-timed figure

    def e2e_run(dtype):
        rows = len(src_list)
        try:
            import psutil
            if psutil.virtual_memory().available < 3 * rows * V * np.dtype(dtype).itemsize:
                rows = 2  # not enough host memory for a row per source: alternate two rows
        except Exception:
            rows = 2
        host = np.empty((rows, V), dtype=dtype)
        try:
            eb.host_register(host)
            pinned = True
        except Exception:
            pinned = False
        outs = [host[i % rows] for i in range(len(src_list))]
        g.bfs_many(src_list[:4], outs[:4])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            st_many = g.bfs_many(src_list, outs)
        el = time.perf_counter() - t0
        _, _, rate = replicas.job_rate(edges_per_step * e2e_steps, el, dist, dev)
        # the same call's traversals alone (CUDA events around each, last step)
        trav_ms = sum(x.device_ms for x in st_many)
        trav_rate = sum(x.traversed_edges for x in st_many) / (trav_ms * 1e-3) if trav_ms > 0 else 0.0
        want = depth_ref_last if dtype == np.int32 else np.where(depth_ref_last < 0, 255, depth_ref_last).astype(np.uint8)
        ok = bool(np.array_equal(outs[-1], want))
        if pinned:
            eb.host_unregister(host)
        return rate / 1e9, rows, pinned, ok, trav_rate / 1e9

    e2e_value, e2e_rows, pinned, e2e_ok, trav_u8 = e2e_run(np.uint8)
    e2e_i32, _, _, e2e_ok32, _ = e2e_run(np.int32)

    # ------------------------------------------- CPU baseline (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(beg, csr_h, srcs, args, g, depth)

    launches = args.steps * launches_per_step * world
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
        "config": headline_config(args, V, E),
        "parallelism": f"replicas x{world} (sources independent, no collective on the data path)",
        "l2_flush": "a 256 MB buffer written before every step, besides inputs larger than L2",
        "graph_gen_s": round(gen_s, 2),
        "gteps_harmonic_mean": round(hmean, 3),
        "gteps_reference_convention": {
            "value": round(amean_ref, 3) if amean_ref is not None else None,
            "rule": "arithmetic mean over sources with more than 2 levels",
            "time": "includes the on-device depth/status reset (the reference times without it); the reset "
                    "(k_reset) is about 2% of kernel time per the committed s24 launch list"},
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
            "traffic": round(traffic) if traffic else None,
            "traffic_basis": traffic_basis,
            "physical_gbs": round(physical, 1) if physical else None,
            "physical_frac": round(physical / peak, 4) if physical else None,
            "unit_of_work": "one BFS (one CUDA-graph launch: reset + [expand, inspect] x levels); "
                            "algorithmic bytes 4*m_c + 8*n_c + 4*V; physical = ncu DRAM bytes per traversal "
                            "over the same mean traversal time",
        },
        "e2e": {"value": round(e2e_value, 3), "unit": "GTEPS", "h2d_bytes_per_step": 4 * len(srcs),
                "d2h_bytes_per_step": V * len(srcs),
                "api": "ent_bfs_many_u8 (C ABI): every source's depths, in the reference's byte depth "
                       "type, copied to a host row, the copy overlapping the next traversal",
                "host_rows": e2e_rows, "host_buffer_pinned": pinned, "last_row_matches_device_run": e2e_ok,
                "traversal_device_gteps": round(trav_u8, 3),
                "traversal_device_rule": "the call's traversals alone, CUDA events around each (last step): "
                                         "the byte-depth traversal writes the reference's depth type itself",
                "int32_depths": {"value": round(e2e_i32, 3), "api": "ent_bfs_many",
                                 "d2h_bytes_per_step": 4 * V * len(srcs), "last_row_matches_device_run": e2e_ok32}},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if tuned:
        line["autotuned"] = tuned
    if world == 1 and not args.no_extras:
        g.close()
        del depth, flush
        torch.cuda.empty_cache()
        line["batched"] = run_batched(args)
        line["high_diameter_and_uniform"] = run_deep(args)
        line["ingest"] = run_ingest(args)
        line["serving"] = run_serving(args)
        if args.burst_seconds > 0:
            line["serving_rmat_queued"] = run_burst(args)
    elif not args.no_extras:
        g.close()
        del depth, flush
        torch.cuda.empty_cache()
        extras = run_extras_multi(args, rank, world, dist)
        if rank == 0:
            line.update(extras)
    return line


def run_extras_multi(args, rank, world, dist):
    """The batched and serving legs with one replica per rank (weak scaling:
    every rank runs the single-GPU leg's work on its own GPU with its own
    seeded sources or query stream). Each rank computes its leg without any
    collective, then one all_gather_object on every rank, failed or not,
    brings the results to rank 0, which sums the work and takes the slowest
    rank's time."""
    local = {}
    for name, fn in (("batched", lambda: run_batched(args, rank, no_multi=True)),
                     ("serving", lambda: run_serving(args, rank, seconds=args.serve_seconds_multi, raw=True))):
        try:
            local[name] = fn()
        except Exception as e:  # noqa: BLE001 - reported in the line, the collective below still runs
            local[name] = {"error": f"{type(e).__name__}: {e}"}
    every = [None] * world
    dist.all_gather_object(every, local)
    if rank != 0:
        return {}
    out = {}
    errs = [e["batched"]["error"] for e in every if "error" in e["batched"]]
    if errs:
        out["batched"] = {"error": errs[0], "ranks": world}
    else:
        b = {"ranks": world, "graph": every[0]["batched"]["graph"],
             "kind": "replicas: every rank runs each batch width on its own seeded sources"}
        for key in [k for k in every[0]["batched"] if k.startswith("batch_") and isinstance(every[0]["batched"][k], dict)
                    and "edges" in every[0]["batched"][k]]:
            ms = max(e["batched"][key]["ms"] for e in every)
            edges = sum(e["batched"][key]["edges"] for e in every)
            b[key] = {"ms_max_over_ranks": ms, "gteps_aggregate": round(edges / ms / 1e6, 2),
                      "oracle_mismatches": sum(len(e["batched"][key]["oracle_mismatches"]) for e in every)}
        out["batched"] = b
    errs = [e["serving"]["error"] for e in every if "error" in e["serving"]]
    if errs:
        out["serving"] = {"error": errs[0], "ranks": world}
    else:
        lat = np.concatenate([np.asarray(e["serving"].pop("latencies_ms")) for e in every])
        s = {"ranks": world, "kind": "one server per rank, each with its own seeded Poisson stream",
             "completed": sum(e["serving"]["completed"] for e in every),
             "throughput_qps": round(sum(e["serving"]["throughput_qps"] for e in every), 1),
             "gteps": round(sum(e["serving"]["gteps"] for e in every), 2),
             "p50_ms": round(float(np.percentile(lat, 50)), 3) if len(lat) else None,
             "p99_ms": round(float(np.percentile(lat, 99)), 3) if len(lat) else None,
             "p999_ms": round(float(np.percentile(lat, 99.9)), 3) if len(lat) else None,
             "sampled_exact": all(e["serving"]["sampled_exact"] for e in every),
             "per_rank": [{k: e["serving"][k] for k in ("completed", "throughput_qps", "mean_batch", "p99_ms")}
                          for e in every]}
        out["serving"] = s
    return out


def run_batched(args, rank=0, no_multi=False):
    """Bitwise multi-source BFS on R-MAT s22 ef16: batches of 64/256/1024
    sources against 256 sequential single-source runs of the same sources,
    plus 48 R-MAT graphs of scales 12-20, edge factors 8-32, in one launch."""
    import torch
    import enterprise_b200 as eb
    scale = args.batch_scale
    g = eb.Graph.rmat(scale, 16, seed=graph_seed(scale), **RMAT)
    host = g.download()  # the CSR the oracle checks rows against
    beg = host.beg_pos
    srcs = eb.pick_sources(beg, source_seed(scale, rank), 1024)
    tune_srcs = eb.pick_sources(beg, source_seed(scale, rank) + 0x7E57, 1024)  # disjoint from the timed sources
    V = g.vert_count
    tuned = {}
    if not args.no_tune:
        # the sequential baseline runs with single-source options tuned for this graph too
        from enterprise_b200 import tune
        o1, _, hit = tune.autotune(g, tune_srcs[:16], "single", reps=2, label="rmat")
        tuned["single"] = {"alpha": o1.alpha, "beta": o1.beta, "small_max": o1.small_max,
                           "large_min": o1.large_min, "chunk_edges": o1.chunk_edges, "cached": hit}
    d1 = torch.empty(V, dtype=torch.int32, device="cuda")
    st = [g.bfs_device(int(s), d1.data_ptr()) for s in srcs[:256]]
    m = np.array([x.traversed_edges for x in st], dtype=np.float64)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    strm = torch.cuda.Stream()
    seq = []
    for _ in range(3):
        torch.cuda.synchronize()
        s0.record(strm)
        for s in srcs[:256]:
            g.bfs_device(int(s), d1.data_ptr(), 0, strm.cuda_stream, stats=False)
        s1.record(strm)
        torch.cuda.synchronize()
        seq.append(s0.elapsed_time(s1))
    seq_ms = min(seq)
    out = {"graph": f"rmat s{scale} ef16", "vertices": V, "directed_entries": g.edge_count,
           "sequential_256": {"ms": round(seq_ms, 3), "gteps": round(m.sum() / seq_ms / 1e6, 2),
                              "kind": "256 direction-optimizing single-source runs, back to back"}}
    for n in [int(x) for x in args.batch_sizes.split(",")]:
        if not args.no_tune:
            # each batch width gets its own search, on sources disjoint from the timed ones
            ob, _, hit = tune.autotune(g, tune_srcs[:n], "batch", reps=1, label=f"rmat-batch{n}")
            tuned[f"batch_{n}"] = {"batch_alpha": ob.batch_alpha, "batch_small_max": ob.batch_small_max,
                                   "batch_large_min": ob.batch_large_min, "batch_heavy": ob.batch_heavy,
                                   "cached": hit}
        dd = torch.empty((n, V), dtype=torch.int32, device="cuda")
        times, edges = [], 0
        for rep in range(4):
            if args.batch_loop == "host":  # same kernels, launched per level (for profilers)
                rows = g.trace_batch([int(x) for x in srcs[:n]], dd.data_ptr())
                if rep:
                    times.append(sum(r["expand_ms"] + r["inspect_ms"] for r in rows))
                stb = g.bfs_batch_device(srcs[:n], dd.data_ptr()) if rep == 3 else None
            else:
                stb = g.bfs_batch_device(srcs[:n], dd.data_ptr())
                if rep:
                    times.append(stb[0].device_ms)
            if stb:
                edges = sum(x.traversed_edges for x in stb)
        ms = min(times)
        # rows against the CPU oracle: every row of the 256-source batch, 16 spread rows of the others
        check = range(n) if n == 256 else sorted(set(np.linspace(0, n - 1, 16).astype(int).tolist()))
        bad = oracle_rows(host, [int(srcs[i]) for i in check], lambda j, _c=list(check): dd[_c[j]].cpu().numpy())
        out[f"batch_{n}"] = {"ms": round(ms, 3), "gteps": round(edges / ms / 1e6, 2), "edges": int(edges),
                            "oracle_checked": len(check), "oracle_mismatches": bad,
                            "levels": stb[0].td_levels + stb[0].bu_levels}
        del dd
        torch.cuda.empty_cache()
    if tuned:
        out["autotuned"] = tuned
    if "batch_256" in out:
        out["batch_256_vs_sequential_256"] = round(out["sequential_256"]["ms"] / out["batch_256"]["ms"], 3)
        # roofline of the batch from ncu-measured DRAM bytes (algorithmic sums would count the
        # shared CSR reads once per source), scaled from the profiled graph by directed entries
        prof = "bfs_batch_rmat_s21_256_graph.md"
        tb, e_prof = profiled_traffic(prof, "dram_bytes_per_batch"), profiled_traffic(prof, "directed_entries")
        if tb and e_prof:
            traffic = tb * g.edge_count / e_prof
            peak, peak_kind = measured_peak()
            gbs = traffic / (out["batch_256"]["ms"] * 1e-3) / 1e9
            # in-run lower bound: the output rows written once plus one read of the CSR
            min_bytes = 4.0 * 256 * V + 4.0 * g.edge_count + 8.0 * V
            min_gbs = min_bytes / (out["batch_256"]["ms"] * 1e-3) / 1e9
            out["batch_256_roofline"] = {
                "bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                "frac": round(gbs / peak, 4), "peak_kind": peak_kind, "traffic": round(traffic),
                "basis": f"scaled estimate: ncu DRAM bytes of whole 256-source batches on R-MAT s21 "
                         f"(profiles/{prof}), scaled to this graph by directed entries",
                "min_bytes": round(min_bytes), "min_bytes_gbs": round(min_gbs, 1),
                "min_bytes_frac": round(min_gbs / peak, 4),
                "min_bytes_rule": "in-run lower bound: 4*n_src*V of int32 rows written + 4*E + 8*V of CSR read once"}
        # the same batch writing the reference's byte depths (a quarter of the row bytes)
        if not args.no_tune:
            tune.autotune(g, tune_srcs[:256], "batch", reps=1, label="rmat-batch256")  # its options again
        d8 = torch.empty((256, V), dtype=torch.uint8, device="cuda")
        t8 = []
        for rep in range(4):
            st8 = g.bfs_batch_device_u8(srcs[:256], d8.data_ptr())
            if rep:
                t8.append(st8[0].device_ms)
        chk8 = [0, 128, 255]
        bad8 = oracle_rows(host, [int(srcs[i]) for i in chk8], lambda j: d8[chk8[j]].cpu().numpy(), as_bytes=True)
        out["batch_256_byte_rows"] = {"ms": round(min(t8), 3), "oracle_checked": len(chk8),
                                      "oracle_mismatches": bad8}
        del d8
    g.close()
    if args.no_multi or no_multi:
        torch.cuda.empty_cache()
        return out
    out["multi_graph_48"] = run_multi(args)
    return out


def run_multi(args):
    """48 R-MAT graphs of uneven sizes (scales 12-20, edge factors 8-32), 64
    seeded sources each, as one multi-graph plan: one CUDA-graph launch, one
    batched traversal over the disjoint union of the graphs. The first and
    last row of every graph are compared with the oracle. With --batch-loop
    host the plan also runs once through its host-driven trace (the same
    kernels launched per level, which profilers can see) and reports it."""
    import torch
    import enterprise_b200 as eb
    rng = np.random.default_rng(0x48)
    graphs, sources, hosts, total_v = [], [], [], 0
    for k in range(48):
        sc = int(rng.integers(12, 21))
        ef = int(rng.choice([8, 16, 32]))
        gk = eb.Graph.rmat(sc, ef, seed=0xC4000 + k, **RMAT)
        hk = gk.download()
        graphs.append(gk)
        hosts.append(hk)
        sources.append(eb.pick_sources(hk.beg_pos, 0xC4100 + k, 64))
        total_v += gk.vert_count
    plan = eb.MultiPlan(graphs, sources)
    mts = [plan.run() for _ in range(4)][1:]
    ms = min(mts)
    edges = 0
    for gk, sk in zip(graphs, sources):
        # per-source edges (report() convention) from a separate batched run
        dd = torch.empty((len(sk), gk.vert_count), dtype=torch.int32, device="cuda")
        edges += sum(x.traversed_edges for x in gk.bfs_batch_device(sk, dd.data_ptr()))
        del dd
    trace = None
    if args.batch_loop == "host":
        rows = plan.trace(0)
        trace = [{"level": r["level"], "direction": r["direction"],
                  "ms": round(r["expand_ms"] + r["inspect_ms"], 4)} for r in rows]
    # the first and the last row of every graph against the CPU oracle
    bad = []
    for k in range(48):
        dk = plan.depths(k)
        bad += [dict(m, graph=k) for m in
                oracle_rows(hosts[k], [int(sources[k][0]), int(sources[k][63])], lambda j: dk[0 if j == 0 else 63])]
    out = {"ms": round(ms, 3), "graphs": 48, "sources_per_graph": 64, "vertices_total": total_v,
           "gteps": round(edges / ms / 1e6, 2), "oracle_checked": 96, "oracle_mismatches": bad,
           "launches": "one CUDA graph launch: one batched traversal over the disjoint union of "
                       "the graphs (one width class, shared source slots)"}
    if trace is not None:
        out["host_driven_trace"] = trace
    plan.close()
    for gk in graphs:
        gk.close()
    torch.cuda.empty_cache()
    return out


def run_deep(args):
    """High-diameter and low-skew graphs, 32 seeded sources each: a 4096^2
    4-neighbour grid with 10% of edges dropped (thousands of levels, tiny
    frontiers: the small-frontier cluster kernel) and an Erdos-Renyi graph
    with 2^24 vertices and mean degree 32. Each source's depths are compared
    with the same traversal on the grid-wide path alone (mode off)."""
    import torch
    import enterprise_b200 as eb
    out = {}
    specs = [("grid_4096x4096", lambda: eb.Graph.grid(4096, 4096, 0.1, seed=0x6E1D4096)),
             ("er_2^24_d32", lambda: eb.Graph.er(1 << 24, 32.0, seed=0xE12424))]
    specs = [sp for sp in specs if sp[0].split("_")[0] in args.deep_graphs.split(",")]
    for name, make in specs:
        g = make()
        if args.loop != "graph":
            o = g.opts
            o.loop = eb.LOOP[args.loop]
            g.opts = o
        beg = g.download().beg_pos
        srcs = eb.pick_sources(beg, 0x50C0C3 + len(name), args.deep_sources)
        tuned = None
        if name.startswith("er") and not args.no_tune:  # the grid runs in the small-frontier mode throughout
            from enterprise_b200 import tune
            t0 = time.time()
            tsrc = eb.pick_sources(beg, 0x50C0C3 + len(name) + 0x7E57, 8)
            opts, _, hit = tune.autotune(g, tsrc, "single", reps=1, label="er")
            tuned = {"opts": {k: v for k, v in vars(opts).items() if k != "fault_inject"}, "cached": hit,
                     "search_s": round(time.time() - t0, 2)}
        V = g.vert_count
        depth = torch.empty(V, dtype=torch.int32, device="cuda")
        strm = torch.cuda.Stream()
        sp = strm.cuda_stream
        st = [g.bfs_device(int(s), depth.data_ptr(), 0, sp) for s in srcs]
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in srcs]
        with torch.cuda.stream(strm):
            for i, s in enumerate(srcs):
                ev[i][0].record(strm)
                g.bfs_device(int(s), depth.data_ptr(), 0, sp, stats=False)
                ev[i][1].record(strm)
        strm.synchronize()
        ms = np.array([a.elapsed_time(b) for a, b in ev])
        m = np.array([x.traversed_edges for x in st], dtype=np.float64)
        lv = np.array([x.levels for x in st])
        nl = np.array([x.narrow_levels for x in st])
        # two sources against the CPU oracle, one of them also against the grid-wide path alone
        rows = [g.bfs(int(s))[0] for s in srcs[:2]]
        batch = None
        if name.startswith("grid"):
            # the same sources as one batch call (on a deep graph: concurrent single-source
            # lanes, one cluster each) against their single-source traversals back to back
            nb = len(srcs)
            brows = torch.empty((nb, V), dtype=torch.int32, device="cuda")
            stb = g.bfs_batch_device([int(s) for s in srcs], brows.data_ptr())  # probe, build, warm
            tb = [g.bfs_batch_device([int(s) for s in srcs], brows.data_ptr())[0].device_ms for _ in range(2)]
            brow = [brows[i].cpu().numpy() for i in (0, nb - 1)]
            del brows
            batch = {"sources": nb, "ms": round(min(tb), 3), "single_source_total_ms": round(float(ms.sum()), 3),
                     "speedup_vs_single": round(float(ms.sum()) / min(tb), 2),
                     "mode": "concurrent single-source lanes" if stb[0].narrow_levels > 0 else "bitwise",
                     "rows_oracle_checked": 2}
        o = g.opts
        o.narrow_max_frontier = 0
        g.opts = o
        off = g.bfs(int(srcs[0]))[0]
        on = rows[0]
        host = g.download()
        g.close()
        bad = oracle_rows(host, [int(s) for s in srcs[:2]], lambda j: rows[j])
        if batch is not None:
            batch["oracle_mismatches"] = oracle_rows(host, [int(srcs[0]), int(srcs[-1])], lambda j: brow[j])
        del host
        out[name] = {"vertices": V, "sources": len(srcs), "ms_per_bfs_mean": round(float(ms.mean()), 3),
                     "gteps_harmonic": round(len(m) / float(np.sum(ms * 1e-3 / m)) / 1e9, 3),
                     "gteps_total": round(float(m.sum() / ms.sum() / 1e6), 3),
                     "levels_mean": round(float(lv.mean()), 1),
                     "small_frontier_levels_mean": round(float(nl.mean()), 1),
                     "us_per_level": round(float((ms / lv).mean() * 1e3), 3),
                     "same_depths_with_small_frontier_mode_off": bool(np.array_equal(on, off)),
                     "oracle_checked": 2, "oracle_mismatches": bad,
                     "autotuned": tuned}
        if batch is not None:
            out[name]["batched"] = batch
        del depth
        torch.cuda.empty_cache()
    return out


def run_ingest(args):
    """Loading the reference's binary format (int64 beg_pos.bin and csr.bin,
    R-MAT at --ingest-scale) into a device graph: the host path (read + narrow
    on the host, then upload) against the streamed loader (chunks read in
    parallel into pinned buffers, narrowed on the GPU). The files are written
    first, so both reads come from the page cache; the best of two runs."""
    import tempfile
    import torch
    import enterprise_b200 as eb
    sc = args.ingest_scale
    g = eb.Graph.rmat(sc, 16, seed=graph_seed(sc), **RMAT)
    host = g.download()
    g.close()
    out = {"graph": f"rmat s{sc} ef16", "vertices": host.vert_count, "directed_entries": host.edge_count}
    with tempfile.TemporaryDirectory() as d:
        b, c = os.path.join(d, "g_beg_pos.bin"), os.path.join(d, "g_csr.bin")
        host.save(b, c)
        nbytes = os.path.getsize(b) + os.path.getsize(c)
        out["file_bytes"] = nbytes

        def timed(fn):
            best, res = None, None
            for _ in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = fn()
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
                if _ == 0:
                    res.close()
            return best, res

        t_host, g1 = timed(lambda: eb.Graph.from_csr(eb.Csr.load(b, c)))
        t_dev, g2 = timed(lambda: eb.Graph.load(b, c))
        same = bool(np.array_equal(g1.download().csr, g2.download().csr))
        g1.close()
        g2.close()
        torch.cuda.empty_cache()
        # the drop-in command line end to end on the same files: load, the
        # reference's 64 glibc rand() sources, validation, its stdout lines
        cli = {}
        for name, extra in (("streamed_gpu_certified", []), ("host_load_gpu_certified", ["--host-load"])):
            t0 = time.perf_counter()
            r = subprocess.run([eb.CLI_PATH, b, c] + extra, capture_output=True, text=True, timeout=900)
            wall = time.perf_counter() - t0
            line = [x for x in r.stdout.splitlines() if x.startswith("Final Average TEPS (Billion):")]
            cli[name] = {"wall_s": round(wall, 3), "exit": r.returncode,
                         "correct": r.stdout.count("BFS result validation: CORRECT"),
                         "wrong": r.stdout.count("WRONG"),
                         "final_average_teps": float(line[0].split(":")[1]) if line else None}
        out["cli_64_sources"] = cli
    del host
    torch.cuda.empty_cache()
    out.update({"host_path_s": round(t_host, 3), "host_path_gbs": round(nbytes / t_host / 1e9, 2),
                "streamed_s": round(t_dev, 3), "streamed_gbs": round(nbytes / t_dev / 1e9, 2),
                "speedup": round(t_host / t_dev, 2), "same_csr": same,
                "note": "includes building the traversal structures (degree-ordered rows, lead arrays)"})
    return out


def run_serving(args, rank=0, seconds=None, raw=False, rate=None, rmat_only=False, join=1):
    """Poisson stream of BFS queries against 16 device-resident graphs (12
    R-MAT s14-22 ef16, 4 grids 1024^2..2048^2 with 10% of edges dropped):
    continuous batching, admission by HBM depth rows, latency percentiles.
    rank > 0 draws its own query stream (replicas); raw adds the latencies;
    rmat_only serves the 12 R-MAT graphs alone (the load point where queries
    queue and the batched slots take them)."""
    import torch
    import enterprise_b200 as eb
    rmat_scales = [14, 15, 16, 17, 18, 18, 19, 19, 20, 20, 21, 22]
    graphs, begs, hosts = [], [], []
    for k, sc in enumerate(rmat_scales):
        graphs.append(eb.Graph.rmat(sc, 16, seed=0xC5000 + k, **RMAT))
    for k, w in enumerate([] if rmat_only else [1024, 1448, 1774, 2048]):
        graphs.append(eb.Graph.grid(w, w, 0.1, seed=0xC5100 + k))
    for gk in graphs:
        hosts.append(gk.download())  # for the oracle's check of the sampled queries
        begs.append(hosts[-1].beg_pos)
    pools = [eb.pick_sources(b, 0xC5200 + k + 1000 * rank, 512) for k, b in enumerate(begs)]
    rng = np.random.default_rng(0xC5 + 1000 * rank + (7 if rmat_only else 0))
    duration = args.serve_seconds if seconds is None else seconds
    rate = args.serve_rate if rate is None else rate
    n_q = int(rng.poisson(rate * duration))
    arrivals = np.sort(rng.uniform(0, duration, n_q))
    which = rng.integers(0, len(graphs), n_q)
    pick = rng.integers(0, 512, n_q)
    lat, qwait, edges, done = [], [], 0, 0
    lat_cls = {"rmat": [], "grid": []}
    sample_every = max(1, n_q // 40)
    checks, bad_status, mismatches, samples = 0, 0, [], []
    graph_of = {}
    with eb.Server(graphs, max_batch=args.serve_batch, slots_per_graph=args.serve_slots,
                   single_cluster=args.serve_cluster, join=join) as srv:
        t0 = time.perf_counter()
        i = 0
        while done < n_q:
            now = time.perf_counter() - t0
            while i < n_q and arrivals[i] <= now:
                q = srv.submit(int(which[i]), int(pools[which[i]][pick[i]]))
                graph_of[q] = (int(which[i]), int(pools[which[i]][pick[i]]), i % sample_every == 0)
                i += 1
            for r in srv.poll(wait_us=200):
                done += 1
                lat.append(r["latency_ms"])
                qwait.append(r["queue_ms"])
                edges += r["traversed_edges"]
                gi, src, sample = graph_of.pop(r["query_id"])
                lat_cls["grid" if gi >= len(rmat_scales) else "rmat"].append(r["latency_ms"])
                if r["status"] != 0:
                    bad_status += 1
                if sample and r["status"] == 0:
                    samples.append((gi, src, srv.depth(r["query_id"])))  # checked after the run
                srv.release(r["query_id"])
            if time.perf_counter() - t0 > duration * 3 + 60:
                break
        wall = time.perf_counter() - t0
        c = srv.counters()
    for gk in graphs:
        gk.close()
    torch.cuda.empty_cache()
    for gi, src, d in samples:
        mismatches += [dict(m, graph=gi) for m in oracle_rows(hosts[gi], [src], lambda j: d)]
    checks = len(samples)
    lat = np.array(lat)
    extra = {"latencies_ms": [float(x) for x in lat]} if raw else {}
    return {**extra, "graphs": "12 R-MAT s14-22 ef16" + ("" if rmat_only else
                                                           " + 4 grids 1024^2,1448^2,1774^2,2048^2 (10% edges dropped)"),
            "arrival": f"Poisson {rate}/s for {duration} s ({n_q} queries, seeded)",
            "completed": int(done), "wall_s": round(wall, 2), "throughput_qps": round(done / wall, 1),
            "gteps": round(edges / wall / 1e9, 2),
            "p50_ms": round(float(np.percentile(lat, 50)), 3) if len(lat) else None,
            "p99_ms": round(float(np.percentile(lat, 99)), 3) if len(lat) else None,
            "p999_ms": round(float(np.percentile(lat, 99.9)), 3) if len(lat) else None,
            "queue_p50_ms": round(float(np.percentile(qwait, 50)), 3) if len(qwait) else None,
            "batches": c["batches"], "mean_batch": round(c["launched"] / max(1, c["batches"]), 2),
            "max_batch_seen": c["max_batch_seen"], "joined_running_batches": c["joined"],
            "fast_slot_queries": c["fast_launches"], "oracle_checked": checks,
            "sampled_exact": not mismatches and bad_status == 0, "bad_status": bad_status,
            "mismatches": mismatches[:5], "max_batch": args.serve_batch, "slots_per_graph": args.serve_slots, "single_cluster": args.serve_cluster,
            "single_source_graphs": c["single_graphs"],
            "by_class": {k: {"queries": len(v),
                             "p50_ms": round(float(np.percentile(v, 50)), 3) if v else None,
                             "p99_ms": round(float(np.percentile(v, 99)), 3) if v else None}
                         for k, v in lat_cls.items()}}


def run_burst(args):
    """The second serving point: the 12 R-MAT graphs alone at a rate where
    queries queue, so that batches form and waiting queries join running
    batches at level boundaries; then the same stream with joining off."""
    out = run_serving(args, seconds=args.burst_seconds, rate=args.burst_rate, rmat_only=True)
    off = run_serving(args, seconds=args.burst_seconds, rate=args.burst_rate, rmat_only=True, join=0)
    out["join_off"] = {k: off[k] for k in ("completed", "throughput_qps", "gteps", "p50_ms", "p99_ms", "p999_ms",
                                           "queue_p50_ms", "mean_batch", "batches", "sampled_exact")}
    return out


def oracle_rows(host, srcs, get_row, as_bytes=False):
    """Checker for the extra legs (outside every timed region): the depth rows
    the GPU produced for `srcs` (get_row(j) -> row j, host numpy) against the
    CPU oracle's direction-optimising BFS on all host threads. Returns the
    mismatches (at most 5 described), empty when every row is bit-exact."""
    import oracle
    bad = []
    for j, s in enumerate(srcs):
        exp = oracle.bfs_omp_do(host.beg_pos, host.csr, int(s))
        if as_bytes:
            exp = np.where(exp < 0, 255, exp).astype(np.uint8)
        got = np.asarray(get_row(j))
        if not np.array_equal(got, exp):
            diff = np.flatnonzero(got != exp)
            if len(bad) < 5:
                bad.append({"src": int(s), "n_diff": int(len(diff)), "at": int(diff[0]) if len(diff) else -1})
            else:
                bad.append({"src": int(s)})
    return bad


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
    """The CPU arm: the oracle's direction-optimising OpenMP BFS (the reference
    has no CPU BFS of its own; validate.h holds only a spot check) on all host
    threads, over the GPU arm's workload: the same seeded R-MAT, rebuilt on the
    host by the oracle's generator (the same CSR, bit for bit), and the same
    seeded sources, all of them in every step. Loads no product code."""
    if rank != 0:
        return None
    import oracle
    t0 = time.time()
    beg, adj = oracle.gen_rmat(args.scale, args.ef, seed=graph_seed(args.scale), **RMAT)
    gen_s = time.time() - t0
    srcs = [int(s) for s in oracle.pick_sources(beg, source_seed(args.scale), args.sources)]
    threads = oracle.max_threads()

    def step():
        edges, secs = 0.0, 0.0
        for s in srcs:
            t = time.perf_counter()
            d = oracle.bfs_omp_do(beg, adj, s, threads=threads)
            secs += time.perf_counter() - t
            edges += oracle.report(beg, d)[0]
        return edges, secs

    for _ in range(args.warmup):
        step()
    edges, secs = 0.0, 0.0
    for _ in range(args.steps):
        e, dt = step()
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
        "data": "synthetic: seeded Graph500-parameter R-MAT built on the host by the oracle's generator "
                "(the GPU arm's CSR, bit for bit)",
        "config": headline_config(args, len(beg) - 1, len(adj)),
        "parallelism": f"{threads} host threads (OpenMP)",
        "graph_gen_s": round(gen_s, 2),
        "cpu_baseline": {"value": round(value, 4), "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"all {len(srcs)} sources in every step ({args.steps} timed, {args.warmup} "
                                   "warm-up), direction-optimizing OpenMP CPU BFS (oracle port; the reference "
                                   "has no CPU BFS)"},
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
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner")
    ap.add_argument("--opts", default="",
                    help="JSON object of traversal options (BfsOpts fields) applied to the headline graph")
    ap.add_argument("--loop", choices=["graph", "host"], default="graph",
                    help="level loop driver; host launches each kernel (profilers can see them)")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and serving measurements")
    ap.add_argument("--batch-scale", type=int, default=22)
    ap.add_argument("--batch-sizes", default="64,256,1024", help="sources per batch in the batched leg")
    ap.add_argument("--no-multi", action="store_true", help="skip the 48-graph launch of the batched leg")
    ap.add_argument("--batch-loop", choices=["graph", "host"], default="graph",
                    help="host: drive each batch level by level from the host (kernels visible to ncu)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving run length (the configuration's 60 s)")
    ap.add_argument("--burst-rate", type=float, default=40000.0,
                    help="second serving point: R-MAT graphs only, at a rate where queries queue")
    ap.add_argument("--burst-seconds", type=float, default=10.0, help="its length (0: skip it)")
    ap.add_argument("--serve-seconds-multi", type=float, default=20.0,
                    help="serving run length per rank when --gpus N > 1 (replicas, one stream each)")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-batch", type=int, default=64)
    ap.add_argument("--serve-slots", type=int, default=1)
    ap.add_argument("--serve-cluster", type=int, default=8,
                    help="CTAs per small-frontier cluster of the deep graphs' single-source slots")
    ap.add_argument("--deep-graphs", default="grid,er", help="graphs of the high-diameter/uniform leg")
    ap.add_argument("--deep-sources", type=int, default=32)
    ap.add_argument("--ingest-scale", type=int, default=24)
    ap.add_argument("--only", choices=["batch", "multi", "serve", "deep", "ingest", "burst"], default=None,
                    help="run only one of the extra measurements and print it")
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
        if args.only:
            line = {"batch": run_batched, "multi": run_multi, "serve": run_serving, "deep": run_deep,
                    "ingest": run_ingest, "burst": run_burst
                    }[args.only](args)
        elif args.impl == "reference":
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
