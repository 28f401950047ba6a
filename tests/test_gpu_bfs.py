"""GPU parity tests of the single-source traversal: bit-exact int32 depths
against the CPU oracle, Graph500 parent checks, statistics equal to the
reference's report() convention. Every call goes through the C ABI."""
import numpy as np
import pytest

from conftest import hand_graphs, tier_graph

pytestmark = pytest.mark.gpu

POLICIES = ["beamer", "reference", "td", "bu"]


def _graph(eb, csr, **opts):
    g = eb.Graph.from_csr(csr)
    if opts:
        o = g.opts
        for k, v in opts.items():
            setattr(o, k, eb.POLICY[v] if k == "policy" else (eb.LOOP[v] if k == "loop" else v))
        g.opts = o
    return g


def _check(eb, orc, csr, g, src, parents=True):
    d, p, st = g.bfs(int(src), parents=parents)
    exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(src))
    np.testing.assert_array_equal(d, exp, err_msg=f"depth mismatch from source {src}")
    if parents:
        rc, bad = orc.check_parents(csr.beg_pos, csr.csr, int(src), d, p)
        assert rc == 0, f"parent check {rc} at vertex {bad}"
    e, v = orc.report(csr.beg_pos, exp)
    assert (st.traversed_edges, st.reached_vertices) == (e, v)
    assert st.levels == int(exp.max()) + 1
    assert st.status == 0
    return st


# narrow: the small-frontier cluster kernel on (default) or off (every level
# through the grid-wide expander and inspector)
@pytest.mark.parametrize("narrow", [8192, 0])
@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("loop", ["graph", "host"])
def test_hand_graphs_all_sources(eb, orc, policy, loop, narrow):
    for name, V, edges in hand_graphs():
        e = np.array(edges, dtype=np.int64)
        csr = eb.Csr.from_edges(e[:, 0], e[:, 1], V)
        with _graph(eb, csr, policy=policy, loop=loop, narrow_max_frontier=narrow) as g:
            for s in range(V):
                _check(eb, orc, csr, g, s)


@pytest.mark.parametrize("narrow", [8192, 0])
@pytest.mark.parametrize("policy", POLICIES)
def test_tier_graph_every_tier_and_many_levels(eb, orc, policy, narrow):
    V, s, d = tier_graph()
    csr = eb.Csr.from_edges(s, d, V)
    with _graph(eb, csr, policy=policy, narrow_max_frontier=narrow) as g:
        for src in [0, 1, 3000, 3041, 4999, 5999, 5500]:
            _check(eb, orc, csr, g, src)


@pytest.mark.parametrize("opts", [
    dict(hub_slots=0),
    dict(hub_slots=4096),
    dict(small_max=4, large_min=8, chunk_edges=32),
    dict(small_max=64, large_min=64),
    dict(blocks_per_sm=1),
    dict(policy="reference", ref_ratio=0.01),
    dict(alpha=1e9, beta=1e-9),
    dict(alpha=0.01, beta=2.0),
])
def test_option_variants(eb, orc, opts):
    csr = eb.Csr.rmat(13, 16, seed=21)
    with _graph(eb, csr, narrow_max_frontier=0, **opts) as g:
        for src in eb.pick_sources(csr.beg_pos, 4, 6):
            _check(eb, orc, csr, g, src)


@pytest.mark.parametrize("loop", ["graph", "host"])
@pytest.mark.parametrize("alpha,beta", [(2.0, 4.0), (8.0, 16.0), (48.0, 1024.0), (4.0, 1e6)])
def test_bottom_up_to_top_down_from_the_list(eb, orc, alpha, beta, loop):
    """A bottom-up level on a shrinking frontier also lists what it finds, and
    a switch to top-down after it classifies that list instead of scanning the
    frontier bitmap; a CTA that finds more than it can list sends the switch
    back to the bitmap. Small graphs give each CTA few status words, so both
    happen across these direction thresholds (beta 1e6 switches back only for
    tiny frontiers)."""
    for csr in (eb.Csr.rmat(14, 16, seed=0x7157), eb.Csr.er(30000, 8.0, seed=0x7158)):
        with _graph(eb, csr, loop=loop, alpha=alpha, beta=beta, narrow_max_frontier=0) as g:
            for src in eb.pick_sources(csr.beg_pos, 19, 6):
                st = _check(eb, orc, csr, g, src)
                assert st.td_levels + st.bu_levels == st.levels


@pytest.mark.parametrize("hub", [0, 4096])
@pytest.mark.parametrize("policy", ["beamer", "reference", "bu"])
def test_bottom_up_levels_in_a_row(eb, orc, policy, hub):
    """Runs of bottom-up levels (the bottom-up-only policy makes every level
    one), with and without the hub table, through both loop drivers: depths
    against the oracle, parents, the same statistics. Launch counts: the
    CUDA-graph loop launches expand, inspector and the small-frontier kernel
    (which leaves at once unless chosen) in every loop body, and runs its
    bodies in pairs (one more body than the host loop's iterations where
    their count is odd); the host-driven loop launches the small-frontier
    kernel only where it runs."""
    for csr in (eb.Csr.rmat(15, 16, seed=0x7159), eb.Csr.er(40000, 12.0, seed=0x715A)):
        with _graph(eb, csr, policy=policy, hub_slots=hub) as gg, \
                _graph(eb, csr, policy=policy, hub_slots=hub, loop="host") as gh:
            for src in eb.pick_sources(csr.beg_pos, 23, 5):
                sg = _check(eb, orc, csr, gg, src)
                sh = _check(eb, orc, csr, gh, src)
                assert (sg.levels, sg.td_levels, sg.bu_levels, sg.narrow_levels) == \
                       (sh.levels, sh.td_levels, sh.bu_levels, sh.narrow_levels)
                it, rem = divmod(sg.launches - 1, 3)
                assert rem == 0 and it % 2 == 0, sg.launches
                assert any(0 <= sh.launches - 1 - 2 * h <= h for h in (it - 1, it)), (sg.launches, sh.launches)
                if policy == "bu":
                    assert sg.bu_levels == sg.levels >= 3


def test_source_entry_in_every_part_of_the_fill(eb, orc):
    """The reset kernel writes the source's own entries (depth 0, parent itself)
    inside its fills: in the scalar head of an output that is not 16-byte
    aligned, in a 16-byte vector (any lane) and in the scalar tail (V = 1031 is
    not a multiple of 4 or 16). int32 depths and parents at element offsets
    0..3 of a device buffer, and byte depths through the many-source call."""
    import torch
    csr = eb.Csr.er(1031, 6.0, seed=0x51F1)
    V = csr.vert_count
    srcs = [0, 1, 2, 3, 4, 5, 6, 7, 15, 16, 17, 18, 19, 1019, 1020, 1023, 1024, 1027, 1028, 1029, 1030]
    exps = {s: orc.bfs(csr.beg_pos, csr.csr, s)[0] for s in srcs}
    with eb.Graph.from_csr(csr) as g:
        for off in range(4):
            depth = torch.empty(V + 4, dtype=torch.int32, device="cuda")
            parent = torch.empty(V + 4, dtype=torch.int32, device="cuda")
            for s in srcs:
                g.bfs_device(s, depth.data_ptr() + 4 * off, parent.data_ptr() + 4 * off)
                d = depth[off:off + V].cpu().numpy()
                p = parent[off:off + V].cpu().numpy()
                np.testing.assert_array_equal(d, exps[s], err_msg=f"offset {off}, source {s}")
                assert orc.check_parents(csr.beg_pos, csr.csr, s, d, p)[0] == 0, (off, s)
        rows = [np.empty(V, dtype=np.uint8) for _ in srcs]
        g.bfs_many(srcs, rows)
        for s, r in zip(srcs, rows):
            np.testing.assert_array_equal(r, np.where(exps[s] < 0, 255, exps[s]).astype(np.uint8), err_msg=f"bytes {s}")


def test_rmat_s16_64_sources_bit_exact(eb, orc):
    """R-MAT scale 16, edge factor 16, 64 seeded non-isolated sources."""
    host = eb.Csr.rmat(16, 16, seed=0x5EED0016)
    with eb.Graph.rmat(16, 16, seed=0x5EED0016) as g:
        dev = g.download()
        assert np.array_equal(dev.beg_pos, host.beg_pos) and np.array_equal(dev.csr, host.csr)
        for src in eb.pick_sources(host.beg_pos, 0x50C0016, 64):
            _check(eb, orc, host, g, src)


@pytest.mark.parametrize("kind", ["grid", "er"])
def test_grid_and_er_small(eb, orc, kind):
    if kind == "grid":
        host = eb.Csr.grid(96, 80, 0.1, seed=31)
        g = eb.Graph.grid(96, 80, 0.1, seed=31)
    else:
        host = eb.Csr.er(20000, 32.0, seed=32)
        g = eb.Graph.er(20000, 32.0, seed=32)
    with g:
        dev = g.download()
        assert np.array_equal(dev.beg_pos, host.beg_pos) and np.array_equal(dev.csr, host.csr)
        for src in eb.pick_sources(host.beg_pos, 7, 8):
            _check(eb, orc, host, g, src)


def test_isolated_and_boundary_sources(eb, orc):
    csr = eb.Csr.from_edges([0, 1], [1, 2], 6)
    with eb.Graph.from_csr(csr) as g:
        d, p, st = g.bfs(4, parents=True)
        assert d.tolist() == [-1, -1, -1, -1, 0, -1]
        assert p.tolist() == [-1, -1, -1, -1, 4, -1]
        assert st.levels == 1 and st.reached_vertices == 1 and st.traversed_edges == 0
        with pytest.raises(eb.EntError):
            g.bfs(6)
        with pytest.raises(eb.EntError):
            g.bfs(-1)


def test_device_api_matches_host_api(eb, orc):
    import torch
    csr = eb.Csr.rmat(14, 16, seed=5)
    with eb.Graph.from_csr(csr) as g:
        depth = torch.empty(g.vert_count, dtype=torch.int32, device="cuda")
        parent = torch.empty(g.vert_count, dtype=torch.int32, device="cuda")
        for src in eb.pick_sources(csr.beg_pos, 3, 4):
            st = g.bfs_device(int(src), depth.data_ptr(), parent.data_ptr())
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(src))
            np.testing.assert_array_equal(depth.cpu().numpy(), exp)
            assert orc.check_parents(csr.beg_pos, csr.csr, int(src), exp, parent.cpu().numpy())[0] == 0
            assert st.reached_vertices == (exp >= 0).sum()


@pytest.mark.parametrize("loop", ["graph", "host"])
def test_many_sources_pipelined_to_host(eb, orc, loop):
    """ent_bfs_many: every source's host array equals the oracle and the
    single-call result; stats match; NULL entries skip the copy; a repeated
    array holds the later source; pinned and pageable arrays both work."""
    csr = eb.Csr.rmat(14, 16, seed=21)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 22, 9)]
    V = csr.vert_count
    with _graph(eb, csr, loop=loop) as g:
        outs = [np.full(V, 7, dtype=np.int32) for _ in srcs]
        pinned = outs[1]
        eb.host_register(pinned)
        try:
            stats = g.bfs_many(srcs, outs)
        finally:
            eb.host_unregister(pinned)
        for s, d, st in zip(srcs, outs, stats):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, s)
            np.testing.assert_array_equal(d, exp, err_msg=f"source {s}")
            e, v = orc.report(csr.beg_pos, exp)
            assert (st.traversed_edges, st.reached_vertices, st.status) == (e, v, 0)
            assert st.levels == int(exp.max()) + 1
            one = g.bfs(s)[2]
            assert (one.traversed_edges, one.levels) == (st.traversed_edges, st.levels)
        shared = np.full(V, 7, dtype=np.int32)
        skipped = np.full(V, 7, dtype=np.int32)
        g.bfs_many(srcs[:3], [shared, None, shared])
        np.testing.assert_array_equal(shared, orc.bfs(csr.beg_pos, csr.csr, srcs[2])[0])
        assert (skipped == 7).all()
        assert g.bfs_many([], []) == []
        with pytest.raises(eb.EntError):
            g.bfs_many([srcs[0], V], [None, None])


@pytest.mark.parametrize("loop", ["graph", "host"])
def test_many_sources_byte_depths(eb, orc, loop):
    """ent_bfs_many_u8: the traversal writes the reference's byte depths (255 =
    unreached) itself, equal to the oracle's depths, on an R-MAT graph and on a
    grid that runs in the small-frontier kernel (under 255 levels); a
    traversal deeper than 254 levels is refused while the other sources' rows
    are still written."""
    rm = eb.Csr.rmat(13, 8, seed=23)  # isolated vertices give 255 entries
    grid = eb.Csr.grid(90, 70, 0.1, seed=25)
    for csr, n_src in ((rm, 5), (grid, 3)):
        srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 24, n_src)]
        V = csr.vert_count
        with _graph(eb, csr, loop=loop) as g:
            outs = [np.zeros(V, dtype=np.uint8) for _ in srcs]
            stats = g.bfs_many(srcs, outs)
            for s, d, st in zip(srcs, outs, stats):
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, s)
                assert exp.max() < 255
                np.testing.assert_array_equal(d, np.where(exp < 0, 255, exp).astype(np.uint8))
                assert st.reached_vertices == (exp >= 0).sum()
                if csr is grid:
                    assert st.narrow_levels > 0
            # int32 rows from the same graph afterwards (the other instantiation)
            d32 = [np.zeros(V, dtype=np.int32) for _ in srcs]
            g.bfs_many(srcs, d32)
            for s, d in zip(srcs, d32):
                np.testing.assert_array_equal(d, orc.bfs(csr.beg_pos, csr.csr, s)[0])
    n = 300  # a path: depths up to 299
    path = eb.Csr.from_edges(np.arange(n - 1), np.arange(1, n), n)
    with eb.Graph.from_csr(path) as g:
        near, far = np.zeros(n, dtype=np.uint8), np.zeros(n, dtype=np.uint8)
        with pytest.raises(eb.EntError, match="byte depths"):
            g.bfs_many([150, 0], [near, far])
        exp, _ = orc.bfs(path.beg_pos, path.csr, 150)
        np.testing.assert_array_equal(near, exp.astype(np.uint8))


def test_repeated_traversals_are_independent(eb, orc):
    """State from one traversal never leaks into the next (bitmaps, queues, hubs)."""
    csr = eb.Csr.rmat(12, 16, seed=8)
    srcs = eb.pick_sources(csr.beg_pos, 12, 16)
    with eb.Graph.from_csr(csr) as g:
        first = [g.bfs(int(s))[0].copy() for s in srcs]
        for s, d0 in zip(reversed(srcs), reversed(first)):
            d1 = g.bfs(int(s))[0]
            np.testing.assert_array_equal(d0, d1)


def test_cli_end_to_end(eb, orc, tmp_path):
    """enterprise.bin on the reference's files: the default route (files
    streamed to the GPU, every result certified there), the reference's route
    (--host-load: host CSR, then upload) and --batch in both give the
    same per-source reach, edges and levels, all validated."""
    import json
    import subprocess
    csr = eb.Csr.rmat(12, 16, seed=99)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    csr.save(bp, cp)
    runs = {}
    for name, extra in (("gpu", []), ("host", ["--host-load"]), ("gpu_batch", ["--batch", "3"]),
                        ("host_batch", ["--host-load", "--batch", "3"])):
        js = tmp_path / f"{name}.jsonl"
        r = subprocess.run([eb.CLI_PATH, bp, cp, "--sources", "8", "--json", str(js)] + extra,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, name + ": " + r.stdout + r.stderr
        assert "Final Average TEPS (Billion):" in r.stdout and "WRONG" not in r.stdout, name
        assert r.stdout.count("BFS result validation: CORRECT") + r.stdout.count("Traverse depth is") == 8, name
        lines = [json.loads(x) for x in js.read_text().splitlines()]
        assert all(x["check"] == 0 for x in lines) and all(x["batched"] == ("batch" in name) for x in lines)
        runs[name] = [(x["source"], x["edges"], x["reached"], x["levels"]) for x in lines]
    assert runs["gpu"] == runs["host"] == runs["gpu_batch"] == runs["host_batch"]
    for src, edges, reached, levels in runs["gpu"]:
        exp, _ = orc.bfs(csr.beg_pos, csr.csr, src)
        assert (edges, reached) == orc.report(csr.beg_pos, exp) and levels == int(exp.max()) + 1

@pytest.mark.parametrize("policy", POLICIES)
def test_raw_csr_with_duplicates_and_self_loops(eb, orc, policy):
    """Files from the reference's own edge-list converter keep duplicate edges
    and self loops and need not sort rows. Such a (symmetric) CSR taken as it
    is: depths equal the oracle's on the same arrays, report() counts every
    listed entry, and the batched path and the GPU certificates agree."""
    import torch
    base = eb.Csr.rmat(12, 8, seed=888)
    V = base.vert_count
    rng = np.random.default_rng(889)
    rows = []
    for v in range(V):
        r = list(base.csr[base.beg_pos[v]:base.beg_pos[v + 1]])
        if r and rng.random() < 0.3:
            r += r[: max(1, len(r) // 3)]          # duplicates (each mirrored below)
        if rng.random() < 0.1:
            r.append(v)                            # self loop
        rows.append(r)
    # keep the adjacency symmetric: mirror every duplicate
    extra = [[] for _ in range(V)]
    for v, r in enumerate(rows):
        seen = {}
        for u in r:
            seen[u] = seen.get(u, 0) + 1
        for u, k in seen.items():
            if u != v and k > 1:
                extra[u] += [v] * (k - 1)
    adj_rows = [np.array(r + e, dtype=np.int32) for r, e in zip(rows, extra)]
    for r in adj_rows:
        rng.shuffle(r)
    beg = np.zeros(V + 1, dtype=np.int64)
    beg[1:] = np.cumsum([len(r) for r in adj_rows])
    adj = np.concatenate(adj_rows).astype(np.int32)
    srcs = [int(s) for s in eb.pick_sources(beg, 890, 6)]
    with _graph(eb, eb.Csr(beg, adj), policy=policy) as g:
        for s in srcs:
            exp, _ = orc.bfs(beg, adj, s)
            d, p, st = g.bfs(s, parents=True)
            np.testing.assert_array_equal(d, exp)
            assert (st.traversed_edges, st.reached_vertices) == orc.report(beg, exp)
            (dc, db), (pc, pb) = g.validate(s, d, p)
            assert (dc, pc) == (0, 0), (dc, db, pc, pb)
        rows_b, _ = g.bfs_batch(srcs)
        for i, s in enumerate(srcs):
            np.testing.assert_array_equal(rows_b[i], orc.bfs(beg, adj, s)[0])


@pytest.mark.parametrize("V", [1, 5, 37])
def test_edgeless_graphs(eb, orc, V):
    """No edges at all (and a single vertex): every entry point returns the
    source at depth 0 and -1 (255 in bytes) elsewhere, with exact statistics."""
    empty = np.zeros(0, dtype=np.int64)
    csr = eb.Csr.from_edges(empty, empty, V)
    assert csr.edge_count == 0
    srcs = [0, V - 1]
    with eb.Graph.from_csr(csr) as g:
        for s in srcs:
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, s)
            d, p, st = g.bfs(s, parents=True)
            np.testing.assert_array_equal(d, exp)
            assert (st.reached_vertices, st.traversed_edges, st.levels) == (1, 0, 1)
            assert p[s] == s and (p >= 0).sum() == 1
            (dc, _), (pc, _) = g.validate(s, d, p)
            assert (dc, pc) == (0, 0)
        rows, stats = g.bfs_batch(srcs)
        for i, s in enumerate(srcs):
            np.testing.assert_array_equal(rows[i], orc.bfs(csr.beg_pos, csr.csr, s)[0])
            assert stats[i].reached_vertices == 1
        outs = [np.zeros(V, dtype=np.uint8) for _ in srcs]
        g.bfs_many(srcs, outs)
        for s, o in zip(srcs, outs):
            np.testing.assert_array_equal(o, np.where(np.arange(V) == s, 0, 255).astype(np.uint8))
        # a multi-graph plan whose union starts and ends with this edgeless graph
        other = eb.Csr.rmat(8, 4, seed=0xED6E + V)
        parts = [(csr, srcs), (other, [0, 5, 9]), (csr, [V - 1])]
        with eb.Graph.from_csr(other) as go, eb.MultiPlan([g, go, g], [s for _, s in parts]) as plan:
            plan.run()
            for k, (c, ss) in enumerate(parts):
                d = plan.depths(k)
                for i, s in enumerate(ss):
                    np.testing.assert_array_equal(d[i], orc.bfs(c.beg_pos, c.csr, s)[0], err_msg=f"part {k} row {i}")
