"""Generates the golden vectors under tests/golden/ from the reference itself.

Phase 1 (any machine, CPU):
    python tests/golden/make_golden.py graphs <dir>
writes each fixture graph in the reference's binary format (int64
<name>_beg_pos.bin and <name>_csr.bin, graph.hpp:33-118) plus <name>_sources.txt.

Phase 2 (a GPU machine, with oracle/_ref/ref_bfs_dump built from the reference's
sources by oracle/Makefile):
    python tests/golden/make_golden.py reference <dir>
runs the reference's own GPU BFS (bfs_tdbu_clfy_sort, via ref_bfs_dump) on every
graph and writes <name>_ref_depth.bin: one uint8 depth array per source, as the
reference stores depths (depth_t = unsigned char, 0xFF = unreached, comm.h:69,131).

The committed fixtures are phase 1 + phase 2 outputs for the graphs below.
Every graph's depth never exceeds 254, the reference's representable range.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def fixture_graphs():
    import enterprise_b200 as eb
    out = {}
    out["rmat_s10_ef16"] = eb.Csr.rmat(10, 16, seed=0x601D0010)
    out["rmat_s12_ef8"] = eb.Csr.rmat(12, 8, seed=0x601D0012)
    out["er_2000_d10"] = eb.Csr.er(2000, 10.0, seed=0x601DE12)
    out["grid_40x30"] = eb.Csr.grid(40, 30, 0.1, seed=0x601D6)
    e = np.array([(0, 1), (1, 2), (2, 3), (5, 6), (6, 7), (7, 5), (8, 9), (3, 10), (10, 11)])
    out["hand_components"] = eb.Csr.from_edges(e[:, 0], e[:, 1], 14)  # 4, 12, 13 isolated
    star = np.array([(0, i) for i in range(1, 40)] + [(i, i + 1) for i in range(40, 79)] + [(39, 40)])
    out["hand_star_path"] = eb.Csr.from_edges(star[:, 0], star[:, 1], 80)
    return out


def sources_for(name, csr):
    import enterprise_b200 as eb
    if name.startswith("hand_"):
        return list(range(csr.vert_count))  # every vertex, isolated ones included
    return [int(s) for s in eb.pick_sources(csr.beg_pos, 0x601D5 + len(name), 16)]


def write_graphs(d: str) -> None:
    os.makedirs(d, exist_ok=True)
    for name, csr in fixture_graphs().items():
        csr.save(os.path.join(d, f"{name}_beg_pos.bin"), os.path.join(d, f"{name}_csr.bin"))
        with open(os.path.join(d, f"{name}_sources.txt"), "w") as f:
            f.write("\n".join(str(s) for s in sources_for(name, csr)) + "\n")
        print("wrote", name, csr.vert_count, csr.edge_count)


def run_reference(d: str) -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bfs_dump")
    names = sorted(f[: -len("_sources.txt")] for f in os.listdir(d) if f.endswith("_sources.txt"))
    for name in names:
        p = lambda s: os.path.join(d, name + s)  # noqa: E731
        r = subprocess.run([exe, p("_beg_pos.bin"), p("_csr.bin"), p("_sources.txt"), p("_ref_depth.bin")],
                           capture_output=True, text=True, timeout=120)
        if r.returncode != 0:
            raise SystemExit(f"reference run failed on {name}: {r.stdout[-500:]} {r.stderr[-500:]}")
        print("reference depths", name, os.path.getsize(p("_ref_depth.bin")))


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] not in ("graphs", "reference"):
        raise SystemExit(__doc__)
    (write_graphs if sys.argv[1] == "graphs" else run_reference)(sys.argv[2])
