"""CPU tests of the C ABI library itself: it loads, exports every function
include/enterprise_b200.h declares, and fails with status codes (never a
crash or exit) when no GPU is usable. No compute call needs a GPU here."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ent_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(eb):
    out = subprocess.run(["nm", "-D", "--defined-only", eb.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(ent_[a-z0-9_]+)$", out.stdout, flags=re.M))
    declared = _declared("enterprise_b200.h")
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in declared:
        getattr(eb.lib(), s)


def test_abi_version_and_defaults(eb):
    assert eb.lib().ent_abi_version() == 5
    o = eb.BfsOpts()
    import ctypes
    c = eb._Opts()
    eb.lib().ent_bfs_opts_default(ctypes.byref(c))
    assert eb.BfsOpts._from_c(c) == o


def test_struct_layout_matches_header(eb):
    import ctypes
    assert ctypes.sizeof(eb._Opts) == 4 + 4 + 8 * 3 + 4 * 5 + 4 + 8 + 4 * 12
    assert ctypes.sizeof(eb._Stats) == 8 + 8 + 4 * 4 + 8 + 4 * 2
    assert ctypes.sizeof(eb._ServerOpts) == 4 * 4 + 8 + 4 * 6
    assert ctypes.sizeof(eb._ServerCounters) == 8 * 9 + 4 * 2 + 8 * 2


def test_server_option_defaults(eb):
    import ctypes
    c = eb._ServerOpts()
    eb.lib().ent_server_opts_default(ctypes.byref(c))
    assert (c.max_batch, c.slots_per_graph, c.single_source_levels, c.single_slots) == (64, 2, 64, 8)
    assert (c.fast_slots, c.fast_max_waiting, c.single_cluster) == (2, 2, 8)


def test_invalid_arguments_return_status(eb):
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.rmat(0, 16)
    assert ei.value.code == 1
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.from_edges([0, 5], [1, 2], 3)
    assert ei.value.code == 5


def test_cli_wrong_input():
    cli = os.path.join(ROOT, "enterprise_b200", "lib", "enterprise.bin")
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.stdout.startswith("Input format: ./exe beg_pos(binary, signed long) csr_file(binary, signed long)")
    assert "Wrong input" in r.stdout
    assert r.returncode == 255  # main returns -1 (main.cu:43-47)


def test_cli_reports_load_failure(tmp_path):
    cli = os.path.join(ROOT, "enterprise_b200", "lib", "enterprise.bin")
    r = subprocess.run([cli, str(tmp_path / "nope_beg"), str(tmp_path / "nope_csr")], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Graph load failed" in r.stdout


def test_no_cpu_fallback_without_gpu(eb):
    """On a machine without a GPU the device path errors out; nothing computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = eb.Csr.rmat(6, 4, seed=1)
    with pytest.raises(eb.EntError) as ei:
        eb.Graph.from_csr(g)
    assert ei.value.code == 2


def test_device_alloc_without_a_gpu_is_a_status(eb):
    """ent_device_alloc reports a missing GPU as a status, not a crash."""
    import ctypes
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = ctypes.c_void_p(1)
    rc = eb.lib().ent_device_alloc(0, 1024, ctypes.byref(p))
    assert rc != 0 and not p.value
    assert eb.lib().ent_device_free(None) == 0
