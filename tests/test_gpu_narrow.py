"""GPU tests of the small-frontier mode of the single-source traversal: one
thread-block cluster that runs many top-down levels per launch. Checked like
every other path: bit-exact depths against the CPU oracle, Graph500 parent
checks and report() statistics, through the C ABI; plus the hand-over in both
directions, the shared-memory overflow (spill) path, every cluster size, both
loop drivers and the launch accounting."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(eb, csr, **opts):
    g = eb.Graph.from_csr(csr)
    o = g.opts
    for k, v in opts.items():
        setattr(o, k, eb.POLICY[v] if k == "policy" else (eb.LOOP[v] if k == "loop" else v))
    g.opts = o
    return g


def _check(orc, csr, g, src):
    d, p, st = g.bfs(int(src), parents=True)
    exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(src))
    np.testing.assert_array_equal(d, exp, err_msg=f"depth mismatch from source {src}")
    rc, bad = orc.check_parents(csr.beg_pos, csr.csr, int(src), d, p)
    assert rc == 0, f"parent check {rc} at vertex {bad}"
    e, v = orc.report(csr.beg_pos, exp)
    assert (st.traversed_edges, st.reached_vertices) == (e, v)
    assert st.levels == int(exp.max()) + 1
    assert st.status == 0
    assert st.narrow_levels <= st.td_levels
    assert st.td_levels + st.bu_levels == st.levels
    return st


def broom(n_leaves=9000, n_paths=50, path_len=30):
    """A hub (vertex 0) with n_leaves leaves; leaves 1..n_paths each start a
    path of path_len vertices. Returns (V, src, dst, end of the first path)."""
    edges = [(0, i) for i in range(1, n_leaves + 1)]
    nxt = n_leaves + 1
    ends = []
    for leaf in range(1, n_paths + 1):
        prev = leaf
        for _ in range(path_len):
            edges.append((prev, nxt))
            prev = nxt
            nxt += 1
        ends.append(prev)
    e = np.array(edges, dtype=np.int64)
    return nxt, e[:, 0], e[:, 1], ends[0]


@pytest.fixture(scope="module")
def grid(eb):
    return eb.Csr.grid(300, 200, 0.1, seed=0x6E1D)


@pytest.mark.parametrize("loop", ["graph", "host"])
@pytest.mark.parametrize("policy", ["beamer", "reference", "td"])
def test_grid_runs_in_small_frontier_mode(eb, orc, grid, loop, policy):
    with _graph(eb, grid, loop=loop, policy=policy) as g:
        for src in eb.pick_sources(grid.beg_pos, 11, 6):
            st = _check(orc, grid, g, src)
            assert st.narrow_levels >= st.levels - 2  # all but the first level(s)
            assert st.launches < st.levels  # far fewer launches than two per level


def test_grid_same_depths_with_mode_off(eb, orc, grid):
    srcs = eb.pick_sources(grid.beg_pos, 12, 4)
    with _graph(eb, grid) as on, _graph(eb, grid, narrow_max_frontier=0) as off:
        for s in srcs:
            d_on, _, st_on = on.bfs(int(s))
            d_off, _, st_off = off.bfs(int(s))
            np.testing.assert_array_equal(d_on, d_off)
            assert st_off.narrow_levels == 0
            # reset, then expand + inspect per level; the graph loop runs its body in pairs,
            # so an odd level count adds one pair that finds the traversal done
            assert st_off.launches == 1 + 2 * (st_off.levels + st_off.levels % 2)
            assert (st_on.levels, st_on.reached_vertices, st_on.traversed_edges) == \
                   (st_off.levels, st_off.reached_vertices, st_off.traversed_edges)


@pytest.mark.parametrize("nc", [1, 2, 4, 8, 16])
def test_every_cluster_size(eb, orc, grid, nc):
    with _graph(eb, grid, narrow_cluster=nc) as g:
        for src in eb.pick_sources(grid.beg_pos, 13, 3):
            assert _check(orc, grid, g, src).narrow_levels > 0


def test_hand_over_when_the_frontier_grows(eb, orc, grid):
    """Entry at <= 64 vertices, exit above 128: a grid frontier outgrows the
    mode, the grid-wide levels take over, and the mode comes back when the
    frontier shrinks again."""
    with _graph(eb, grid, narrow_max_frontier=64) as g:
        for src in eb.pick_sources(grid.beg_pos, 14, 4):
            st = _check(orc, grid, g, src)
            assert 0 < st.narrow_levels < st.levels - 1


def test_spill_past_shared_memory(eb, orc):
    """One CTA (4096 entries per buffer) meets a hub with 9000 new neighbours:
    the rest spills to global memory and the run hands over; afterwards the
    49 remaining paths run in the mode again (top-down policy: the mode only
    takes top-down levels)."""
    V, s, d, end = broom()
    csr = eb.Csr.from_edges(s, d, V)
    with _graph(eb, csr, policy="td", narrow_cluster=1, narrow_max_frontier=2048, narrow_max_degree=1 << 20,
                narrow_max_edges=1 << 30) as g:
        for src in (end, 1, 0, V - 1):
            st = _check(orc, csr, g, src)
            assert st.narrow_levels > 0


def test_heavy_vertex_leaves_the_mode(eb, orc):
    """With the default degree limit the hub is expanded by the grid-wide
    tiers, and the paths before and after it by the cluster."""
    V, s, d, end = broom()
    csr = eb.Csr.from_edges(s, d, V)
    with _graph(eb, csr) as g:
        st = _check(orc, csr, g, end)
        assert 0 < st.narrow_levels < st.levels


@pytest.mark.parametrize("loop", ["graph", "host"])
def test_directed_path_ending_in_an_empty_row(eb, orc, loop):
    """A directed CSR (top-down policy: it follows out-edges only) whose last
    vertex, reached at the last level, has an empty row starting at E, one past
    the adjacency array: the cluster claims it without touching that address."""
    n = 400
    beg = np.concatenate([np.arange(n, dtype=np.int64), [n - 1]])
    adj = np.arange(1, n, dtype=np.int32)
    csr = eb.Csr(beg, adj)
    with _graph(eb, csr, loop=loop, policy="td") as g:
        d, _, st = g.bfs(0)
        exp, _ = orc.bfs(csr.beg_pos, csr.csr, 0)
        np.testing.assert_array_equal(d, exp)
        assert d[n - 1] == n - 1 and st.narrow_levels > 0


def test_trace_shows_cluster_runs(eb, orc, grid):
    src = int(eb.pick_sources(grid.beg_pos, 15, 1)[0])
    with _graph(eb, grid) as g:
        rows, st = g.trace(src)
        assert any(r["direction"] == 2 for r in rows)
        d, _, _ = g.bfs(src)
        exp, _ = orc.bfs(grid.beg_pos, grid.csr, src)
        np.testing.assert_array_equal(d, exp)


def test_rmat_tail_levels(eb, orc):
    """Skewed graph: the mode may only take small tail levels (degree limit)."""
    csr = eb.Csr.rmat(14, 16, seed=0x5EED000E)
    with _graph(eb, csr) as g:
        for src in eb.pick_sources(csr.beg_pos, 16, 8):
            _check(orc, csr, g, src)


def test_device_api_on_a_stream(eb, orc, grid):
    import torch
    with _graph(eb, grid) as g:
        depth = torch.empty(g.vert_count, dtype=torch.int32, device="cuda")
        stream = torch.cuda.Stream()
        for src in eb.pick_sources(grid.beg_pos, 17, 3):
            st = g.bfs_device(int(src), depth.data_ptr(), 0, stream.cuda_stream)
            exp, _ = orc.bfs(grid.beg_pos, grid.csr, int(src))
            np.testing.assert_array_equal(depth.cpu().numpy(), exp)
            assert st.narrow_levels > 0


@pytest.mark.parametrize("bad", [dict(narrow_max_frontier=16385), dict(narrow_max_frontier=-1),
                                 dict(narrow_cluster=17), dict(narrow_max_degree=0),
                                 dict(narrow_max_edges=-5), dict(narrow_max_degree=(1 << 20) + 1)])
def test_invalid_options_rejected(eb, grid, bad):
    with eb.Graph.from_csr(grid) as g:
        o = g.opts
        for k, v in bad.items():
            setattr(o, k, v)
        with pytest.raises(eb.EntError):
            g.opts = o
