"""World-size-2 tests of the replicated (N > 1) path on CPU with gloo.

A job on N GPUs is N independent replicas (enterprise_b200/replicas.py):
per-rank seeded sources, no collective on the data path, the work summed and
the time maxed over ranks. These tests run that bookkeeping as two gloo ranks
with the oracle standing in for each rank's traversal, check the reductions
and that a rank which dies is detected by the survivor through a short
process-group timeout (no GPU involved), and run bench.py's reference arm under
torchrun with two ranks.
"""
from __future__ import annotations

import datetime
import json
import os
import socket
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s=60):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _replica_worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import enterprise_b200 as eb
    from enterprise_b200 import replicas
    import oracle
    dist = _init(rank, world, port)
    try:
        csr = eb.Csr.rmat(11, 8, seed=0x5EED000B)
        srcs = replicas.rank_sources(csr.beg_pos, 11, rank, 8)
        dist.barrier()
        t0 = time.perf_counter()
        edges = 0.0
        for s in srcs:
            d, _ = oracle.bfs(csr.beg_pos, csr.csr, int(s))
            edges += oracle.report(csr.beg_pos, d)[0]
        secs = time.perf_counter() - t0 + 0.01 * (rank + 1)  # distinct per-rank times
        dist.barrier()
        units, job_s, rate = replicas.job_rate(edges, secs, dist, "cpu")
        every = [None] * world
        dist.all_gather_object(every, {"srcs": [int(x) for x in srcs], "edges": edges, "secs": secs})
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"units": units, "job_s": job_s, "rate": rate, "every": every}, f)
    finally:
        dist.destroy_process_group()


def _shard_worker(rank, world, port, out_dir):
    """One shared source list sharded over the ranks by the product's plan;
    each rank computes its chunks' rows (the oracle stands in for the GPU
    batch, which needs a device) and rank 0 assembles them in input order."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import enterprise_b200 as eb
    from enterprise_b200 import replicas
    import oracle
    dist = _init(rank, world, port)
    try:
        csr = eb.Csr.rmat(10, 8, seed=0x5EED000A)
        srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 0x5A4D, 37)]
        mine = replicas.rank_chunks(len(srcs), world, rank, max_batch=8)
        local = []
        for b, e in mine:
            rows = np.stack([oracle.bfs(csr.beg_pos, csr.csr, s)[0] for s in srcs[b:e]])
            local.append(((b, e), rows))
        full = replicas.gather_rows(local, len(srcs), dist)
        res = {"chunks": mine}
        if rank == 0:
            exp = np.stack([oracle.bfs(csr.beg_pos, csr.csr, s)[0] for s in srcs])
            res["in_order"] = bool(np.array_equal(full, exp))
        else:
            res["in_order"] = full is None
        with open(os.path.join(out_dir, f"shard{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_shard_rows_world2_gloo(tmp_path):
    codes = _spawn(_shard_worker, 2, tmp_path)
    assert codes == [0, 0]
    r0 = json.load(open(tmp_path / "shard0.json"))
    r1 = json.load(open(tmp_path / "shard1.json"))
    assert r0["in_order"] and r1["in_order"]
    got = sorted(tuple(c) for c in r0["chunks"] + r1["chunks"])
    assert got[0][0] == 0 and got[-1][1] == 37
    assert all(a[1] == b[0] for a, b in zip(got, got[1:]))  # contiguous, no overlap
    assert r0["chunks"] and r1["chunks"]  # both ranks got work


def test_replicas_plan_rules():
    sys.path.insert(0, ROOT)
    import enterprise_b200 as eb
    for n, reps, mb in [(1000, 2, 256), (5, 8, 1024), (1, 1, 1), (2048, 3, 2048), (4097, 4, 1024), (0, 2, 4)]:
        chunks = eb.replicas_plan(n, reps, mb)
        assert sum(e - b for b, e in chunks) == n
        assert all(0 < e - b <= mb for b, e in chunks)
        assert all(a[1] == b[0] for a, b in zip(chunks, chunks[1:]))
        assert (not chunks) or (chunks[0][0] == 0 and chunks[-1][1] == n)
        if n >= reps:
            assert len(chunks) >= min(reps, n)  # every replica can get work
    with pytest.raises(Exception):
        eb.replicas_plan(10, 0, 4)
    from enterprise_b200 import replicas
    allc = [c for r in range(3) for c in replicas.rank_chunks(100, 3, r, 16)]
    assert sorted(allc) == eb.replicas_plan(100, 3, 16)


def _dying_worker(rank, world, port, out_dir):
    dist = _init(rank, world, port, timeout_s=3)
    if rank == 1:
        os._exit(0)  # leaves between steps, without telling anyone
    t0 = time.perf_counter()
    err = None
    try:
        dist.barrier()
    except Exception as e:  # noqa: BLE001 - any error is the detection
        err = type(e).__name__
    with open(os.path.join(out_dir, "rank0.json"), "w") as f:
        json.dump({"error": err, "waited_s": time.perf_counter() - t0}, f)
    os._exit(0)


def _spawn(fn, world, out_dir):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=fn, args=(r, world, port, str(out_dir))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            raise AssertionError("rank did not finish")
    return [p.exitcode for p in procs]


def test_replicas_single_process():
    from enterprise_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(2.0) == 2.0
    assert replicas.job_rate(10.0, 2.0) == (10.0, 2.0, 5.0)
    with pytest.raises(ValueError):
        replicas.job_rate(1.0, 0.0)
    assert replicas.source_seed(24, 0) != replicas.source_seed(24, 1)


def test_replicas_world2_gloo(tmp_path):
    codes = _spawn(_replica_worker, 2, tmp_path)
    assert codes == [0, 0]
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    # every rank agrees on the job figures
    assert r0["units"] == r1["units"] and r0["job_s"] == r1["job_s"]
    every = r0["every"]
    assert r0["units"] == pytest.approx(sum(e["edges"] for e in every))
    assert r0["job_s"] == pytest.approx(max(e["secs"] for e in every))
    assert r0["rate"] == pytest.approx(r0["units"] / r0["job_s"])
    # ranks draw their own, different source sets
    assert every[0]["srcs"] != every[1]["srcs"]
    assert all(len(set(e["srcs"])) == len(e["srcs"]) for e in every)


def test_dead_rank_detected_by_timeout(tmp_path):
    _spawn(_dying_worker, 2, tmp_path)
    r0 = json.load(open(tmp_path / "rank0.json"))
    assert r0["error"] is not None
    assert r0["waited_s"] < 60


def test_bench_reference_arm_torchrun_world2():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--gpus", "2", "--impl", "reference", "--scale", "12", "--ef", "8", "--steps", "3", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["unit"] == "GTEPS"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"
    # the rest of the line's contract
    assert line["metric"].startswith("GTEPS, R-MAT s24 ef16") and line["higher_is_better"] is True
    assert (line["steps"], line["warmup"], line["scaling"]) == (3, 3, "weak")
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["sample"]
    assert "workload" in line["config"] and line["dtype"] == "int32"
