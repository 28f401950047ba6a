"""Host-side pieces of bench.py that need no GPU: the figures it reads from
the committed ncu summaries (the roofline `traffic` of the headline and the
measured bytes of a batch) parse to the values the summaries state."""
import os
import sys

import pytest

ROOT =os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_profile_figures_parse():
    import bench
    assert bench.profiled_traffic(bench.TRAFFIC_PROFILE) == 168.5e6
    assert bench.profiled_traffic(bench.TRAFFIC_PROFILE, "directed_entries") == 128311084
    assert bench.profiled_traffic("bfs_batch_rmat_s21_256_graph.md", "dram_bytes_per_batch") == 4.890e9
    assert bench.profiled_traffic("bfs_batch_rmat_s21_256_graph.md", "directed_entries") == 63536952
    assert bench.profiled_traffic("no_such_summary.md") is None


def test_headline_traffic_only_for_the_captured_options():
    """The roofline's DRAM figure is used only when the run traverses with the
    options the ncu capture used; otherwise it is withheld with the reason."""
    import bench
    want = bench.profiled_options(bench.TRAFFIC_PROFILE)
    assert want and want["alpha"] == 48.0
    run = dict(want, policy=0, batch_alpha=4.0)
    t, basis = bench.headline_traffic(run, 520772318)
    assert t == pytest.approx(168.5e6 * 520772318 / 128311084) and "same options" in basis
    t, basis = bench.headline_traffic(dict(run, alpha=24.0), 520772318)
    assert t is None and "differ" in basis


def test_bench_source_seed_matches_replicas():
    import bench
    from enterprise_b200 import replicas
    for scale in (12, 22, 24):
        for rank in (0, 1, 7):
            assert bench.source_seed(scale, rank) == replicas.source_seed(scale, rank)


_REF_ARM = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
class A: pass
a = A()
a.scale, a.ef, a.sources, a.steps, a.warmup = 12, 8, 16, 1, 3
line = bench.run_reference(a, 0, 1)
maps = open("/proc/self/maps").read()
print(json.dumps({{"line": line, "product_imported": "enterprise_b200" in sys.modules,
                   "product_mapped": "libenterprise_b200" in maps, "oracle_mapped": "liboracle" in maps}}))
"""


def test_reference_arm_loads_no_product_code():
    """The CPU arm builds its graph and sources with the oracle alone; its
    workload description is the GPU arm's (same graph, same sources)."""
    import subprocess
    import json
    import bench
    r = subprocess.run([sys.executable, "-c", _REF_ARM.format(root=ROOT)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["product_imported"] and not out["product_mapped"] and out["oracle_mapped"]
    line = out["line"]
    assert line["impl"] == "reference" and line["value"] > 0

    class A:
        scale, ef, sources = 12, 8, 16
    import enterprise_b200 as eb
    csr = eb.Csr.rmat(12, 8, seed=bench.graph_seed(12), **bench.RMAT)
    assert line["config"] == bench.headline_config(A, csr.vert_count, csr.edge_count)


def test_measured_peak_is_a_bandwidth():
    import bench
    peak, kind = bench.measured_peak()
    assert kind in ("measured", "fallback") and 1000 < peak < 10000  # GB/s
