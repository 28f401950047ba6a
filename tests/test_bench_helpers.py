"""Host-side pieces of bench.py that need no GPU: the figures it reads from
the committed ncu summaries (the roofline `traffic` of the headline and the
measured bytes of a batch) parse to the values the summaries state."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_profile_figures_parse():
    import bench
    assert bench.profiled_traffic("bfs_rmat_s24_traffic.txt") == 0.835e9
    assert bench.profiled_traffic("bfs_batch_rmat_s21_256_graph.md", "dram_bytes_per_batch") == 4.882e9
    assert bench.profiled_traffic("bfs_batch_rmat_s21_256_graph.md", "directed_entries") == 63536952
    assert bench.profiled_traffic("no_such_summary.md") is None


def test_measured_peak_is_a_bandwidth():
    import bench
    peak, kind = bench.measured_peak()
    assert kind in ("measured", "fallback") and 1000 < peak < 10000  # GB/s
