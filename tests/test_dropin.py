"""The reference's own command line as a maintainer would switch it over.

oracle/Makefile compiles the reference's unmodified main.cu (with its own
graph.h, graph.hpp and wtime.h, where they lie) against this repository's
include/bfs_gpu_opt.cuh and links it to libenterprise_b200.so, giving
oracle/_ref/dropin_enterprise.bin. Its call bfs_gpu_coalescing_mem<int,int>
(main.cu:80-86) instantiates the drop-in template (bfs_gpu_opt.cuh:293-300),
its loader is the reference's graph<long,long,double,int,int,double>
(graph.hpp:33-118) and its 64 sources are the reference's glibc rand() draw
(main.cu:55-78). The files read are the golden fixtures, which are in the
reference's int64 format.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin_enterprise.bin")
GOLDEN = os.path.join(ROOT, "tests", "golden")
BANNER = "Input format: ./exe beg_pos(binary, signed long) csr_file(binary, signed long)"

needs_dropin = pytest.mark.skipif(not os.path.exists(DROPIN),
                                  reason="drop-in build needs the reference sources (oracle/Makefile REF_DIR)")


def _files(name):
    return os.path.join(GOLDEN, f"{name}_beg_pos.bin"), os.path.join(GOLDEN, f"{name}_csr.bin")


def _blocks(out):
    """(source, traversed vertices, traversed edges or None, verdict or None) per 'Test n' block."""
    rows = []
    for blk in out.split("Test ")[1:]:
        src = int(re.search(r"Started from: (\d+)", blk).group(1))
        tv = re.search(r"Traversed vertices: (\d+)\s+Traversed edges: (\d+)", blk)
        verdict = re.search(r"BFS result validation: (\w+)", blk)
        rows.append((src, int(tv.group(1)) if tv else None, int(tv.group(2)) if tv else None,
                     verdict.group(1) if verdict else None))
    return rows


@needs_dropin
def test_dropin_wrong_input_as_reference():
    r = subprocess.run([DROPIN], capture_output=True, text=True, timeout=60)
    assert r.stdout.splitlines() == [BANNER, "Wrong input"]
    assert r.returncode == 255  # main.cu:45 returns -1


@needs_dropin
def test_dropin_uses_reference_loader():
    b, c = _files("rmat_s10_ef16")
    r = subprocess.run([DROPIN, b, c], capture_output=True, text=True, timeout=300)
    lines = r.stdout.splitlines()
    E = os.path.getsize(c) // 8
    V = os.path.getsize(b) // 8 - 1
    assert lines[0] == BANNER
    assert lines[1] == f"Possible edge count: {E}"
    assert lines[2] == "Weight file cannot open"
    assert lines[3].startswith(f"Graph load (success): {V} verts, {E} edges")


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("name", ["rmat_s10_ef16", "rmat_s12_ef8"])
def test_dropin_runs_reference_main_on_gpu(eb, orc, name):
    b, c = _files(name)
    r = subprocess.run([DROPIN, b, c], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = r.stdout
    lines = out.splitlines()
    assert lines[0] == BANNER
    for key in ("Weight file cannot open", "GPU alloc space: ", "CPU alloc space: ", "In gpu bfs"):
        assert any(ln.startswith(key) for ln in lines), key
    assert out.index("CPU alloc space") < out.index("In gpu bfs") < out.index("Test 1\n")
    rows = _blocks(out)
    assert len(rows) == 64
    assert [f"Test {i}" for i in range(1, 65)] == re.findall(r"^Test \d+", out, flags=re.M)
    # the same glibc rand() sources as this repository's own command line draws
    ours = subprocess.run([eb.CLI_PATH, b, c, "--host-load"], capture_output=True, text=True, timeout=600)
    assert ours.returncode == 0, ours.stdout[-2000:]
    assert [s for s, *_ in _blocks(ours.stdout)] == [s for s, *_ in rows]
    assert len(set(s for s, *_ in rows)) == 64
    csr = eb.Csr.load(b, c)
    validated = 0
    for src, tv, te, verdict in rows:
        d, _ = orc.bfs(csr.beg_pos, csr.csr, src)
        if d.max() + 1 > 2:  # the reference validates and reports sources deeper than 2 levels
            validated += 1
            assert verdict == "CORRECT", src
            assert (te, tv) == orc.report(csr.beg_pos, d), src
        else:
            assert verdict is None and f"Traverse depth is {d.max() + 1}" in out
    assert validated > 0
    assert "WRONG" not in out
    m = re.search(r"^Final Average TEPS \(Billion\): ([0-9.eE+-]+)$", out, flags=re.M)
    assert m and float(m.group(1)) > 0
