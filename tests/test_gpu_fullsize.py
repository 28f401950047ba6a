"""GPU parity at the benchmark's full sizes. Every sampled traversal is
compared bit for bit with the CPU oracle (the OpenMP direction-optimising BFS
on all host threads, or the serial queue BFS on the deep grid, where a
level-synchronous CPU BFS would pay thousands of barriers), and it also passes
the Graph500-style certificates on the GPU (ent_validate: every vertex and
every edge, the oracle's check_depths / check_parents rules) with statistics
that agree with its depth array. Sizes are those of the benchmark
configurations: R-MAT scale 24 edge factor 16, the 4096 x 4096 grid with 10%
of edges dropped, Erdos-Renyi with 2^24 vertices and mean degree 32, batches
of 256 and 1024 sources on R-MAT scale 22, and graphs of the 48-graph
multi-graph launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_depths(orc, csr, src, serial=False):
    if serial:
        return orc.bfs(csr.beg_pos, csr.csr, int(src))[0]
    return orc.bfs_omp_do(csr.beg_pos, csr.csr, int(src))


def _certify(eb, orc, g, srcs, parents=True, serial=False):
    import torch
    V = g.vert_count
    csr = g.download()
    depth = torch.empty(V, dtype=torch.int32, device="cuda")
    parent = torch.empty(V, dtype=torch.int32, device="cuda") if parents else None
    for s in srcs:
        st = g.bfs_device(int(s), depth.data_ptr(), parent.data_ptr() if parents else 0)
        (dc, db), pres = g.validate_device(int(s), depth.data_ptr(), parent.data_ptr() if parents else 0)
        assert (dc, db) == (0, -1), f"depth certificate broken: rule {dc} at vertex {db} (source {s})"
        if parents:
            assert pres == (0, -1), f"parent certificate broken: {pres} (source {s})"
        got = depth.cpu().numpy()
        exp = _oracle_depths(orc, csr, s, serial)
        np.testing.assert_array_equal(got, exp, err_msg=f"source {s} differs from the CPU oracle")
        assert (st.traversed_edges, st.reached_vertices) == orc.report(csr.beg_pos, exp)
        assert st.levels == int(exp.max()) + 1
        assert st.status == 0


def test_rmat_s24_headline_config(eb, orc):
    with eb.Graph.rmat(24, 16, seed=0x5EED0000 + 24, a=0.57, b=0.19, c=0.19) as g:
        _certify(eb, orc, g, eb.pick_sources(g.download().beg_pos, 0x50C0000 + 24, 4))


def test_grid_4096_config(eb, orc):
    with eb.Graph.grid(4096, 4096, 0.1, seed=0x6E1D4096) as g:
        _certify(eb, orc, g, eb.pick_sources(g.download().beg_pos, 0x50C0400, 2), serial=True)


def test_er_2_24_config(eb, orc):
    with eb.Graph.er(1 << 24, 32.0, seed=0xE12424) as g:
        _certify(eb, orc, g, eb.pick_sources(g.download().beg_pos, 0x50C0E24, 2))


def _batch_rows_vs_oracle(eb, orc, g, srcs, rows_to_check):
    import torch
    V = g.vert_count
    csr = g.download()
    rows = torch.empty((len(srcs), V), dtype=torch.int32, device="cuda")
    stats = g.bfs_batch_device(srcs, rows.data_ptr())
    for k in rows_to_check:
        got = rows[k].cpu().numpy()
        exp = _oracle_depths(orc, csr, srcs[k])
        np.testing.assert_array_equal(got, exp, err_msg=f"row {k} (source {srcs[k]}) differs from the oracle")
        assert (stats[k].traversed_edges, stats[k].reached_vertices) == orc.report(csr.beg_pos, exp)
        assert stats[k].levels == int(exp.max()) + 1
    (dc, db), _ = g.validate_device(srcs[rows_to_check[0]], rows[rows_to_check[0]].data_ptr())
    assert (dc, db) == (0, -1)


def test_batched_s22_256_rows(eb, orc):
    """Every row of the 256-source batch the benchmark times."""
    with eb.Graph.rmat(22, 16, seed=0x5EED0000 + 22, a=0.57, b=0.19, c=0.19) as g:
        srcs = [int(s) for s in eb.pick_sources(g.download().beg_pos, 0x50C0000 + 22, 256)]
        _batch_rows_vs_oracle(eb, orc, g, srcs, list(range(256)))


def test_batched_s22_1024_sampled_rows(eb, orc):
    with eb.Graph.rmat(22, 16, seed=0x5EED0000 + 22, a=0.57, b=0.19, c=0.19) as g:
        srcs = [int(s) for s in eb.pick_sources(g.download().beg_pos, 0x50C0000 + 22, 1024)]
        _batch_rows_vs_oracle(eb, orc, g, srcs, [0, 1, 63, 64, 511, 512, 1000, 1023])


def test_multi_graph_plan_rows(eb, orc):
    """A few graphs of the benchmark's 48-graph plan (the same scales, edge
    factors and seeds), launched together; one row of each against the oracle."""
    rng = np.random.default_rng(0x48)
    specs = [(int(rng.integers(12, 21)), int(rng.choice([8, 16, 32]))) for _ in range(48)]
    pick = [0, 7, 23, 47]
    graphs = [eb.Graph.rmat(specs[k][0], specs[k][1], seed=0xC4000 + k, a=0.57, b=0.19, c=0.19) for k in pick]
    try:
        csrs = [g.download() for g in graphs]
        sources = [eb.pick_sources(c.beg_pos, 0xC4100 + k, 64) for c, k in zip(csrs, pick)]
        plan = eb.MultiPlan(graphs, sources)
        try:
            plan.run()
            for j in range(len(pick)):
                d = plan.depths(j)
                for r in (0, 63):
                    exp = _oracle_depths(orc, csrs[j], sources[j][r])
                    np.testing.assert_array_equal(d[r], exp, err_msg=f"plan graph {pick[j]} row {r}")
        finally:
            plan.close()
    finally:
        for g in graphs:
            g.close()
