"""GPU parity at the benchmark's full sizes, through properties that do not
need the CPU oracle to finish: every traversal's depths and parents pass the
Graph500-style certificates (ent_validate: every vertex and every edge, the
same rules as the oracle's check_depths / check_parents), its statistics agree
with its depth array, and batched rows equal single-source results. Sizes are
those of the benchmark configurations: R-MAT scale 24 edge factor 16, the
4096 x 4096 grid with 10% of edges dropped, Erdos-Renyi with 2^24 vertices and
mean degree 32, and a 256-source batch on R-MAT scale 22."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _certify(eb, g, srcs, parents=True):
    import torch
    V = g.vert_count
    depth = torch.empty(V, dtype=torch.int32, device="cuda")
    parent = torch.empty(V, dtype=torch.int32, device="cuda") if parents else None
    for s in srcs:
        st = g.bfs_device(int(s), depth.data_ptr(), parent.data_ptr() if parents else 0)
        (dc, db), pres = g.validate_device(int(s), depth.data_ptr(), parent.data_ptr() if parents else 0)
        assert (dc, db) == (0, -1), f"depth certificate broken: rule {dc} at vertex {db} (source {s})"
        if parents:
            assert pres == (0, -1), f"parent certificate broken: {pres} (source {s})"
        reached = depth >= 0
        assert st.reached_vertices == int(reached.sum())
        assert st.levels == int(depth.max()) + 1
        assert st.status == 0


def test_rmat_s24_headline_config(eb):
    with eb.Graph.rmat(24, 16, seed=0x5EED0000 + 24, a=0.57, b=0.19, c=0.19) as g:
        _certify(eb, g, eb.pick_sources(g.download().beg_pos, 0x50C0000 + 24, 4))


def test_grid_4096_config(eb):
    with eb.Graph.grid(4096, 4096, 0.1, seed=0x6E1D4096) as g:
        _certify(eb, g, eb.pick_sources(g.download().beg_pos, 0x50C0400, 2))


def test_er_2_24_config(eb):
    with eb.Graph.er(1 << 24, 32.0, seed=0xE12424) as g:
        _certify(eb, g, eb.pick_sources(g.download().beg_pos, 0x50C0E24, 2))


def test_batched_s22_256_rows(eb):
    import torch
    with eb.Graph.rmat(22, 16, seed=0x5EED0000 + 22, a=0.57, b=0.19, c=0.19) as g:
        V = g.vert_count
        srcs = [int(s) for s in eb.pick_sources(g.download().beg_pos, 0x50C0000 + 22, 256)]
        rows = torch.empty((256, V), dtype=torch.int32, device="cuda")
        stats = g.bfs_batch_device(srcs, rows.data_ptr())
        one = torch.empty(V, dtype=torch.int32, device="cuda")
        for k in (0, 1, 77, 128, 200, 255):
            (dc, db), _ = g.validate_device(srcs[k], rows[k].data_ptr())
            assert (dc, db) == (0, -1), f"row {k}: depth certificate rule {dc} at {db}"
            g.bfs_device(srcs[k], one.data_ptr())
            assert torch.equal(rows[k], one), f"row {k} differs from the single-source traversal"
            assert stats[k].reached_vertices == int((rows[k] >= 0).sum())
            assert stats[k].levels == int(rows[k].max()) + 1
