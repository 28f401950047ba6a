"""GPU parity tests of the bitwise multi-source traversal: every source's
int32 depth row is bit-exact against a single-source CPU BFS (the oracle),
and per-source statistics follow the reference's report() convention."""
import numpy as np
import pytest

from conftest import hand_graphs, tier_graph

pytestmark = pytest.mark.gpu


def _check_rows(eb, orc, csr, depth, stats, srcs):
    assert depth.shape == (len(srcs), csr.vert_count)
    for i, s in enumerate(srcs):
        exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(s))
        np.testing.assert_array_equal(depth[i], exp, err_msg=f"row {i} (source {s})")
        e, v = orc.report(csr.beg_pos, exp)
        assert (stats[i].traversed_edges, stats[i].reached_vertices) == (e, v), f"stats row {i}"
        assert stats[i].levels == int(exp.max()) + 1


def test_hand_graphs_every_vertex_as_source(eb, orc):
    for name, V, edges in hand_graphs():
        e = np.array(edges, dtype=np.int64)
        csr = eb.Csr.from_edges(e[:, 0], e[:, 1], V)
        with eb.Graph.from_csr(csr) as g:
            srcs = list(range(V))
            depth, stats = g.bfs_batch(srcs)
            _check_rows(eb, orc, csr, depth, stats, srcs)


@pytest.mark.parametrize("n", [1, 63, 64, 65, 128, 200, 256, 511, 1024])
def test_widths_rmat(eb, orc, n):
    """n sources -> 1..16 words per vertex (thread and lane-group bottom-up)."""
    csr = eb.Csr.rmat(12, 16, seed=100 + n)
    srcs = eb.pick_sources(csr.beg_pos, n, min(n, 1500))
    with eb.Graph.from_csr(csr) as g:
        depth, stats = g.bfs_batch(srcs)
        check = srcs if n <= 128 else srcs[:: max(1, n // 96)]
        idx = [list(srcs).index(s) for s in check]
        for i in idx:
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(srcs[i]))
            np.testing.assert_array_equal(depth[i], exp, err_msg=f"row {i}")
            assert stats[i].reached_vertices == (exp >= 0).sum()


def test_duplicate_and_isolated_sources(eb, orc):
    csr = eb.Csr.from_edges([0, 1, 2, 3], [1, 2, 3, 4], 8)  # 5..7 isolated
    with eb.Graph.from_csr(csr) as g:
        srcs = [2, 2, 0, 7, 4, 2, 6]
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)


def _mode(g, deep):
    o = g.opts
    o.batch_deep = deep
    g.opts = o


@pytest.mark.parametrize("deep", [0, 2])
def test_tier_graph_deep_levels(eb, orc, deep):
    """~1000 levels: the bitwise batch's level log wraps through many flush
    windows; as concurrent single-source lanes, each source runs on its own."""
    V, s, d = tier_graph()
    csr = eb.Csr.from_edges(s, d, V)
    srcs = [0, 1, 3000, 3041, 4999, 5999, 5500, 2, 2]
    with eb.Graph.from_csr(csr) as g:
        _mode(g, deep)
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)


@pytest.mark.parametrize("deep", [0, 1, 2])
def test_grid_batch(eb, orc, deep):
    csr = eb.Csr.grid(48, 40, 0.1, seed=4)
    srcs = eb.pick_sources(csr.beg_pos, 3, 100)
    with eb.Graph.from_csr(csr) as g:
        _mode(g, deep)
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)


@pytest.mark.parametrize("n", [1, 7, 64, 65, 300])
def test_deep_batch_lanes_on_a_grid(eb, orc, n):
    """A batch on a deep grid runs as concurrent single-source lanes, forced and
    in auto mode (the probe finds the grid deep), with at most 3 lanes and with
    as many as fit: every row against the oracle; each source's statistics are
    its own traversal's (small-frontier levels included)."""
    csr = eb.Csr.grid(160, 120, 0.1, seed=33 + n)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 900 + n, n)]
    with eb.Graph.from_csr(csr) as g:
        for deep, lanes in ((2, 3), (1, 0)):
            o = g.opts
            o.batch_deep, o.batch_deep_lanes = deep, lanes
            g.opts = o
            depth, stats = g.bfs_batch(srcs)
            _check_rows(eb, orc, csr, depth, stats, srcs)
            assert all(st.narrow_levels > 0 for st in stats)


def test_deep_batch_lanes_device_rows_and_streams(eb, orc):
    """Device rows through a caller's stream: the call returns before the lanes
    finish, and work queued on that stream after it sees complete rows."""
    import torch
    csr = eb.Csr.grid(200, 90, 0.1, seed=8)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 81, 40)]
    with eb.Graph.from_csr(csr) as g:
        _mode(g, 2)
        rows = torch.full((len(srcs), g.vert_count), 7, dtype=torch.int32, device="cuda")
        strm = torch.cuda.Stream()
        with torch.cuda.stream(strm):
            g.bfs_batch_device(srcs, rows.data_ptr(), stream=strm.cuda_stream, stats=False)
            total = rows.sum(dim=1)  # queued behind the batch on the same stream
        strm.synchronize()
        host = rows.cpu().numpy()
        for i in (0, 13, 39):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, srcs[i])
            np.testing.assert_array_equal(host[i], exp)
        assert total.cpu().tolist() == host.sum(axis=1).tolist()


def test_deep_batch_lanes_on_shallow_and_small_graphs(eb, orc):
    """Forced onto R-MAT (hubs of thousands of edges, a few levels) and onto a
    graph with repeated, isolated and small-component sources: the same rows.
    Auto mode leaves R-MAT to the bitwise batch."""
    csr = eb.Csr.rmat(13, 16, seed=4242)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 4243, 100)]
    with eb.Graph.from_csr(csr) as g:
        _mode(g, 2)
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)
        _mode(g, 1)
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)
        assert all(st.narrow_levels == 0 for st in stats)  # the bitwise batch ran
    csr = eb.Csr.from_edges([0, 1, 2, 3, 9], [1, 2, 3, 4, 10], 12)  # 5..8, 11 isolated
    with eb.Graph.from_csr(csr) as g:
        _mode(g, 2)
        srcs = [2, 2, 0, 7, 4, 2, 6, 9, 11, 10]
        depth, stats = g.bfs_batch(srcs)
        _check_rows(eb, orc, csr, depth, stats, srcs)

def test_batch_matches_single_and_repeats(eb, orc):
    csr = eb.Csr.rmat(14, 16, seed=77)
    srcs = eb.pick_sources(csr.beg_pos, 9, 256)
    with eb.Graph.from_csr(csr) as g:
        d1, _ = g.bfs_batch(srcs)
        d2, _ = g.bfs_batch(srcs[::-1])
        np.testing.assert_array_equal(d1, d2[::-1])
        for i in range(0, 256, 37):
            np.testing.assert_array_equal(d1[i], g.bfs(int(srcs[i]))[0])


def test_batch_device_output(eb, orc):
    import torch
    csr = eb.Csr.rmat(13, 8, seed=5)
    srcs = eb.pick_sources(csr.beg_pos, 2, 70)
    with eb.Graph.from_csr(csr) as g:
        out = torch.empty((len(srcs), g.vert_count), dtype=torch.int32, device="cuda")
        stats = g.bfs_batch_device(srcs, out.data_ptr())
        host = out.cpu().numpy()
        for i in range(0, len(srcs), 7):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(srcs[i]))
            np.testing.assert_array_equal(host[i], exp)
        assert len(stats) == len(srcs)


def test_multi_graph_one_launch(eb, orc):
    """Graphs of uneven sizes and widths, each with its own sources, in one launch."""
    specs = [(9, 8, 3), (11, 16, 70), (12, 32, 130), (10, 8, 1), (13, 16, 64)]
    csrs = [eb.Csr.rmat(s, ef, seed=500 + i) for i, (s, ef, _) in enumerate(specs)]
    graphs = [eb.Graph.from_csr(c) for c in csrs]
    srcs = [eb.pick_sources(c.beg_pos, 600 + i, n) for i, (c, (_, _, n)) in enumerate(zip(csrs, specs))]
    outs = eb.bfs_multi(graphs, srcs)
    for c, s, d in zip(csrs, srcs, outs):
        for i in range(0, len(s), max(1, len(s) // 8)):
            exp, _ = orc.bfs(c.beg_pos, c.csr, int(s[i]))
            np.testing.assert_array_equal(d[i], exp)
    plan = eb.MultiPlan(graphs, srcs)
    for _ in range(2):
        plan.run()
        for k, (c, s) in enumerate(zip(csrs, srcs)):
            d = plan.depths(k)
            exp, _ = orc.bfs(c.beg_pos, c.csr, int(s[-1]))
            np.testing.assert_array_equal(d[-1], exp)
    plan.close()
    for g in graphs:
        g.close()


def test_multi_graph_union_every_row(eb, orc):
    """The plan runs each width class as one traversal over the disjoint union
    of its graphs. One class mixes a deep grid (many flush windows), R-MAT
    graphs with 1 and 64 sources (padded slots), a source on an isolated
    vertex and one graph listed twice with other sources; a second class holds
    a 100-source request. Every row of every graph against the oracle, twice,
    and the plan still answers after its graphs are closed."""
    grid = eb.Csr.grid(60, 50, 0.1, seed=0x6E1D77)
    r1 = eb.Csr.rmat(11, 8, seed=0x5EED0101)
    r2 = eb.Csr.rmat(12, 16, seed=0x5EED0102)
    iso_s = np.array([0, 1, 2], dtype=np.int64)
    iso = eb.Csr.from_edges(iso_s, iso_s + 1, 6)  # path 0-1-2-3, vertices 4 and 5 isolated
    csrs = [grid, r1, r2, iso, r2, r1]
    graphs = [eb.Graph.from_csr(c) for c in csrs[:4]]
    handles = graphs + [graphs[2], graphs[1]]
    srcs = [eb.pick_sources(grid.beg_pos, 700, 5),
            eb.pick_sources(r1.beg_pos, 701, 1),
            eb.pick_sources(r2.beg_pos, 702, 64),
            np.array([5, 0, 3], dtype=np.int32),
            eb.pick_sources(r2.beg_pos, 703, 7),
            eb.pick_sources(r1.beg_pos, 704, 100)]
    plan = eb.MultiPlan(handles, srcs)
    try:
        for _ in range(2):
            plan.run()
            for k, (c, s) in enumerate(zip(csrs, srcs)):
                d = plan.depths(k)
                assert d.shape == (len(s), c.vert_count)
                for i, v in enumerate(s):
                    exp, _ = orc.bfs(c.beg_pos, c.csr, int(v))
                    np.testing.assert_array_equal(d[i], exp, err_msg=f"graph {k} row {i}")
        for g in graphs:
            g.close()
        plan.run()
        exp, _ = orc.bfs(grid.beg_pos, grid.csr, int(srcs[0][4]))
        np.testing.assert_array_equal(plan.depths(0)[4], exp)
    finally:
        plan.close()
        for g in graphs:
            g.close()


def test_multi_graph_trace(eb, orc):
    """A plan's per-level trace of one width class: a row per level up to the
    deepest graph of the union, the final flush last, and the rows of the
    traced run readable afterwards; the other class keeps its own rows."""
    r1 = eb.Csr.rmat(12, 16, seed=0x5EED0201)
    grid = eb.Csr.grid(40, 30, 0.0, seed=1)
    csrs = [r1, grid, r1]
    graphs = [eb.Graph.from_csr(r1), eb.Graph.from_csr(grid)]
    srcs = [eb.pick_sources(r1.beg_pos, 801, 20), np.array([0, 1199], dtype=np.int32),
            eb.pick_sources(r1.beg_pos, 802, 200)]
    with eb.MultiPlan([graphs[0], graphs[1], graphs[0]], srcs) as plan:
        plan.run()
        rows = plan.trace(1)
        assert rows[-1]["level"] == -1
        assert [r["level"] for r in rows[:-1]] == list(range(len(rows) - 1))
        deepest = max(int(orc.bfs(c.beg_pos, c.csr, int(v))[0].max()) for c, s in zip(csrs[:2], srcs[:2]) for v in s)
        assert len(rows) - 1 == deepest + 1  # the level that finds nothing ends the run
        assert all(r["direction"] in (0, 1) for r in rows[:-1])
        for k, (c, s) in enumerate(zip(csrs, srcs)):
            d = plan.depths(k)
            for i in (0, len(s) - 1):
                exp, _ = orc.bfs(c.beg_pos, c.csr, int(s[i]))
                np.testing.assert_array_equal(d[i], exp, err_msg=f"graph {k} row {i}")
        with pytest.raises(eb.EntError):
            plan.trace(3)
    for g in graphs:
        g.close()


@pytest.mark.parametrize("n", [40, 130, 600])
def test_sources_in_small_components(eb, orc, n):
    """Sources of small components mixed with giant-component sources. Once a
    small component's frontier is empty its source is no longer active, so the
    giant component's vertices stop needing its bit and are marked done in
    every bottom-up tier (light, mid, large); rows stay exact."""
    base = eb.Csr.rmat(13, 16, seed=4242)
    V0 = base.vert_count
    s = np.repeat(np.arange(V0, dtype=np.int64), np.diff(base.beg_pos))
    d = base.csr.astype(np.int64)
    # appended components: a 30-vertex path, three pairs, one isolated vertex
    path = np.arange(V0, V0 + 30, dtype=np.int64)
    pairs = np.array([[V0 + 30, V0 + 31], [V0 + 32, V0 + 33], [V0 + 34, V0 + 35]], dtype=np.int64)
    s = np.concatenate([s, path[:-1], pairs[:, 0]])
    d = np.concatenate([d, path[1:], pairs[:, 1]])
    csr = eb.Csr.from_edges(s, d, V0 + 37)
    hub = int(np.argmax(np.diff(csr.beg_pos)))
    reach, _ = orc.bfs(csr.beg_pos, csr.csr, hub)
    deg = np.diff(csr.beg_pos)
    small = [int(v) for v in np.nonzero((reach < 0) & (deg > 0))[0]][: max(4, n // 8)]
    small += [V0, V0 + 29, V0 + 31, V0 + 36]
    giant = eb.pick_sources(csr.beg_pos, 31 + n, n - len(small))
    srcs = [int(x) for x in giant] + small
    rng = np.random.default_rng(n)
    rng.shuffle(srcs)
    with eb.Graph.from_csr(csr) as g:
        o = g.opts
        o.batch_alpha = 4.0
        o.batch_small_max = 8
        o.batch_large_min = 64
        g.opts = o
        depth, stats = g.bfs_batch(srcs)
        check = [i for i, x in enumerate(srcs) if x in small or reach[x] < 0] + list(range(0, n, max(1, n // 24)))
        for i in sorted(set(check)):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(srcs[i]))
            np.testing.assert_array_equal(depth[i], exp, err_msg=f"row {i} (source {srcs[i]})")
            assert stats[i].reached_vertices == (exp >= 0).sum()
            assert stats[i].levels == int(exp.max()) + 1


@pytest.mark.parametrize("n", [5, 70, 300])
def test_byte_rows_match_int32_rows(eb, orc, n):
    """ent_bfs_batch_u8: the reference's byte depths equal the int32 rows with
    -1 read as 255, for 1, 2 and 8 words per vertex; the device variant too."""
    import torch
    csr = eb.Csr.rmat(13, 16, seed=700 + n)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 701 + n, n)]
    with eb.Graph.from_csr(csr) as g:
        d32, st32 = g.bfs_batch(srcs)
        d8, st8 = g.bfs_batch_u8(srcs)
        np.testing.assert_array_equal(d8, np.where(d32 < 0, 255, d32).astype(np.uint8))
        assert [s.traversed_edges for s in st8] == [s.traversed_edges for s in st32]
        dev = torch.empty((n, g.vert_count), dtype=torch.uint8, device="cuda")
        g.bfs_batch_device_u8(srcs, dev.data_ptr())
        np.testing.assert_array_equal(dev.cpu().numpy(), d8)
        for i in range(0, n, max(1, n // 6)):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, srcs[i])
            np.testing.assert_array_equal(d8[i], np.where(exp < 0, 255, exp).astype(np.uint8))


@pytest.mark.parametrize("deep", [0, 2])
def test_byte_rows_refuse_depths_above_254(eb, orc, deep):
    """A 300-vertex path (depths up to 299, several flush windows): the call
    reports ENT_ERR_UNSUPPORTED; the row of a source whose depths stay below
    255 is still complete."""
    n = 300
    csr = eb.Csr.from_edges(np.arange(n - 1), np.arange(1, n), n)
    with eb.Graph.from_csr(csr) as g:
        _mode(g, deep)
        out = np.zeros((2, n), dtype=np.uint8)
        with pytest.raises(eb.EntError, match="byte depths") as ei:
            g.bfs_batch_u8([150, 0], depth_out=out)
        assert ei.value.code == 8
        exp, _ = orc.bfs(csr.beg_pos, csr.csr, 150)
        np.testing.assert_array_equal(out[0], exp.astype(np.uint8))


def test_widest_batch_and_one_more(eb, orc):
    """2048 sources (32 words per vertex, the most one launch takes): eight
    lanes share a neighbour's words in the heavy tiers and the flush walks
    eight column groups; every tier is forced with small thresholds. 2049
    sources are refused."""
    csr = eb.Csr.rmat(12, 16, seed=2048)
    base = [int(s) for s in eb.pick_sources(csr.beg_pos, 2049, 1500)]
    srcs = (base * 2)[:2048]  # repeats are allowed and give the same rows
    with eb.Graph.from_csr(csr) as g:
        o = g.opts
        o.batch_small_max = 8
        o.batch_large_min = 64
        g.opts = o
        depth, stats = g.bfs_batch(srcs)
        for i in list(range(0, 2048, 97)) + [2047]:
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, srcs[i])
            np.testing.assert_array_equal(depth[i], exp, err_msg=f"row {i}")
            assert stats[i].traversed_edges == orc.report(csr.beg_pos, exp)[0]
        np.testing.assert_array_equal(depth[0], depth[len(base)])  # the same source twice
        with pytest.raises(eb.EntError) as ei:
            g.bfs_batch(srcs + [srcs[0]])
        assert ei.value.code == 8
