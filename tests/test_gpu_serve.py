"""GPU tests of the serving loop: every query's depths are identical to the
same BFS run alone (ent_bfs), whatever else shares its batch, its slot or the
device; admission by memory throttles and resumes; the queue refuses when full."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _drain(srv, want, timeout_polls=20000):
    done = []
    polls = 0
    while len(done) < want and polls < timeout_polls:
        done += srv.poll(wait_us=2000)
        polls += 1
    assert len(done) == want, f"only {len(done)} of {want} queries completed"
    return done


def test_results_same_alone_and_in_the_mix(eb, orc):
    csrs = [eb.Csr.rmat(12, 16, seed=61), eb.Csr.grid(60, 50, 0.1, seed=62), eb.Csr.er(5000, 12, seed=63),
            eb.Csr.rmat(10, 8, seed=64)]
    graphs = [eb.Graph.from_csr(c) for c in csrs]
    rng = np.random.default_rng(7)
    alone = {}
    with eb.Server(graphs, max_batch=16, slots_per_graph=2) as srv:
        qs = {}
        for _ in range(300):
            gi = int(rng.integers(len(graphs)))
            src = int(eb.pick_sources(csrs[gi].beg_pos, int(rng.integers(1 << 30)), 1)[0])
            qs[srv.submit(gi, src)] = (gi, src)
        res = _drain(srv, len(qs))
        assert srv.counters()["batches"] >= 2
        for r in res:
            gi, src = qs[r["query_id"]]
            assert (r["graph"], r["src"], r["status"]) == (gi, src, 0)
            got = srv.depth(r["query_id"])
            key = (gi, src)
            if key not in alone:
                alone[key] = graphs[gi].bfs(src)[0]
            np.testing.assert_array_equal(got, alone[key])
            e, v = orc.report(csrs[gi].beg_pos, got)
            assert (r["traversed_edges"], r["reached_vertices"]) == (e, v)
            assert r["latency_ms"] >= r["queue_ms"] >= 0
            srv.release(r["query_id"])
        c = srv.counters()
        assert c["completed"] == c["released"] == 300 and c["rows_free"] == c["rows_total"]
    for g in graphs:
        g.close()


def test_admission_by_memory_throttles_and_resumes(eb):
    """5 depth rows: 5 queries run, the rest wait until results are released."""
    csr = eb.Csr.rmat(11, 8, seed=71)
    g = eb.Graph.from_csr(csr)
    srcs = eb.pick_sources(csr.beg_pos, 3, 40)
    with eb.Server([g], max_batch=8, slots_per_graph=2, rows_per_graph=5) as srv:
        ids = [srv.submit(0, int(s)) for s in srcs]
        done = []
        for _ in range(500):
            done += srv.poll(wait_us=2000)
            if len(done) >= 5:
                break
        done += srv.poll(wait_us=50000)  # nothing else can run: every row is held
        assert len(done) == 5
        c = srv.counters()
        assert c["rows_free"] == 0 and c["pending"] == len(ids) - 5
        released = 0
        for _ in range(5000):
            while released < len(done):
                srv.release(done[released]["query_id"])
                released += 1
            if released == len(ids):
                break
            done += srv.poll(wait_us=2000)
        assert released == len(ids)
        assert srv.counters()["completed"] == len(ids)
    g.close()


def test_queue_limit_refuses(eb):
    csr = eb.Csr.rmat(10, 8, seed=81)
    g = eb.Graph.from_csr(csr)
    with eb.Server([g], max_batch=4, slots_per_graph=1, rows_per_graph=1, max_pending=3) as srv:
        src = int(eb.pick_sources(csr.beg_pos, 1, 1)[0])
        accepted, refused = 0, 0
        for _ in range(20):
            try:
                srv.submit(0, src)
                accepted += 1
            except eb.EntError as e:
                assert e.code == 9
                refused += 1
        assert refused > 0 and accepted >= 3
        assert srv.counters()["rejected"] == refused
    g.close()


def test_submissions_from_threads(eb):
    csr = eb.Csr.rmat(12, 8, seed=91)
    g = eb.Graph.from_csr(csr)
    srcs = eb.pick_sources(csr.beg_pos, 5, 64)
    ref = {int(s): g.bfs(int(s))[0] for s in srcs}
    with eb.Server([g], max_batch=32, slots_per_graph=3) as srv:
        ids = {}
        lock = threading.Lock()

        def worker(part):
            for s in part:
                q = srv.submit(0, int(s))
                with lock:
                    ids[q] = int(s)

        ts = [threading.Thread(target=worker, args=(srcs[i::4],)) for i in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for r in _drain(srv, len(srcs)):
            np.testing.assert_array_equal(srv.depth(r["query_id"]), ref[ids[r["query_id"]]])
            srv.release(r["query_id"])
    g.close()


def test_fresh_graph_traversals_while_serving(eb, orc):
    """First traversals of new graphs (workspace set-up included) run while the
    server keeps other streams busy; their results must not depend on timing."""
    load = [eb.Graph.grid(400, 400, 0.1, seed=101), eb.Graph.rmat(16, 16, seed=102)]
    pools = [eb.pick_sources(g.download().beg_pos, 9, 64) for g in load]
    with eb.Server(load, max_batch=64, slots_per_graph=2) as srv:
        ids = [srv.submit(k % 2, int(pools[k % 2][k % 64])) for k in range(400)]
        for seed in range(4):
            csr = eb.Csr.rmat(14, 16, seed=200 + seed)
            with eb.Graph.from_csr(csr) as g:
                for src in eb.pick_sources(csr.beg_pos, seed, 3):
                    d, _, st = g.bfs(int(src))
                    exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(src))
                    np.testing.assert_array_equal(d, exp)
                    db, _ = g.bfs_batch([int(src)])
                    np.testing.assert_array_equal(db[0], exp)
        for r in _drain(srv, len(ids)):
            srv.release(r["query_id"])
    for g in load:
        g.close()


def test_deep_graphs_served_one_source_per_launch(eb, orc):
    """A grid (hundreds of levels) gets single-source slots, an R-MAT graph
    keeps bitwise batches; every result equals the traversal run alone."""
    csrs = [eb.Csr.grid(150, 120, 0.1, seed=81), eb.Csr.rmat(12, 16, seed=82)]
    graphs = [eb.Graph.from_csr(c) for c in csrs]
    rng = np.random.default_rng(8)
    with eb.Server(graphs, max_batch=32, slots_per_graph=2, single_slots=4) as srv:
        assert srv.counters()["single_graphs"] == 1
        qs = {}
        for _ in range(120):
            gi = int(rng.integers(2))
            src = int(eb.pick_sources(csrs[gi].beg_pos, int(rng.integers(1 << 30)), 1)[0])
            qs[srv.submit(gi, src)] = (gi, src)
        for r in _drain(srv, len(qs)):
            gi, src = qs[r["query_id"]]
            assert (r["graph"], r["src"], r["status"]) == (gi, src, 0)
            exp, _ = orc.bfs(csrs[gi].beg_pos, csrs[gi].csr, src)
            np.testing.assert_array_equal(srv.depth(r["query_id"]), exp)
            e, v = orc.report(csrs[gi].beg_pos, exp)
            assert (r["traversed_edges"], r["reached_vertices"], r["levels"]) == (e, v, int(exp.max()) + 1)
            srv.release(r["query_id"])
        c = srv.counters()
        assert c["completed"] == c["released"] == 120 and c["max_batch_seen"] > 1
    for g in graphs:
        g.close()


def test_single_source_mode_off_keeps_batches(eb, orc):
    csr = eb.Csr.grid(80, 60, 0.1, seed=83)
    g = eb.Graph.from_csr(csr)
    srcs = eb.pick_sources(csr.beg_pos, 5, 20)
    with eb.Server([g], max_batch=16, slots_per_graph=1, single_source_levels=0) as srv:
        assert srv.counters()["single_graphs"] == 0
        ids = {srv.submit(0, int(s)): int(s) for s in srcs}
        for r in _drain(srv, len(ids)):
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, ids[r["query_id"]])
            np.testing.assert_array_equal(srv.depth(r["query_id"]), exp)
            srv.release(r["query_id"])
        assert srv.counters()["max_batch_seen"] > 1
    g.close()


def test_single_source_slots_admission_by_memory(eb, orc):
    """3 depth rows on a deep graph: at most 3 queries hold rows; the rest
    wait for releases, then complete with the same depths."""
    csr = eb.Csr.grid(100, 100, 0.1, seed=84)
    g = eb.Graph.from_csr(csr)
    srcs = eb.pick_sources(csr.beg_pos, 6, 12)
    with eb.Server([g], rows_per_graph=3, single_slots=8) as srv:
        assert srv.counters()["single_graphs"] == 1
        ids = {srv.submit(0, int(s)): int(s) for s in srcs}
        got = 0
        for _ in range(200):
            res = srv.poll(wait_us=20000)
            assert srv.counters()["rows_free"] >= 0
            for r in res:
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, ids[r["query_id"]])
                np.testing.assert_array_equal(srv.depth(r["query_id"]), exp)
                srv.release(r["query_id"])
                got += 1
            if got == len(ids):
                break
        assert got == len(ids)
    g.close()


def test_fast_slots_take_lone_queries(eb, orc):
    """On a shallow graph, queries that arrive one at a time run on the fast
    single-source slots; a burst goes to the batched slots; the depths are the
    same either way, and with fast_slots=0 every query is batched."""
    csr = eb.Csr.rmat(12, 16, seed=91)
    g = eb.Graph.from_csr(csr)
    srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 92, 24)]
    for fast in (2, 0):
        with eb.Server([g], max_batch=16, slots_per_graph=1, fast_slots=fast, fast_max_waiting=2) as srv:
            for s in srcs[:6]:  # one at a time
                q = srv.submit(0, s)
                (r,) = _drain(srv, 1)
                assert r["query_id"] == q and r["status"] == 0
                np.testing.assert_array_equal(srv.depth(q), orc.bfs(csr.beg_pos, csr.csr, s)[0])
                srv.release(q)
            ids = {srv.submit(0, s): s for s in srcs[6:]}  # a burst
            for r in _drain(srv, len(ids)):
                np.testing.assert_array_equal(srv.depth(r["query_id"]),
                                              orc.bfs(csr.beg_pos, csr.csr, ids[r["query_id"]])[0])
                srv.release(r["query_id"])
            c = srv.counters()
            if fast:
                assert c["fast_launches"] >= 6 and c["max_batch_seen"] > 1
            else:
                assert c["fast_launches"] == 0
    g.close()


def test_queries_join_a_running_batch(eb, orc):
    """Continuous batching at level boundaries. On a graph whose batches run
    about a thousand levels, served by bitwise batches alone (no single-source
    slots, one batched slot), queries submitted while a batch runs join it in
    its free source positions at its next level boundary. Every result, joined
    or not, equals the oracle's depths from its own source."""
    import time
    from conftest import tier_graph
    V, s, d = tier_graph()
    csr = eb.Csr.from_edges(s, d, V)
    g = eb.Graph.from_csr(csr)
    srcs = [int(x) for x in eb.pick_sources(csr.beg_pos, 5, 60)]
    srcs[:2] = [5999, 5500]  # deep in the tail: the first batch runs ~1000 levels
    try:
        # joining allowed at any level here, so that queries submitted milliseconds into the batch join it
        with eb.Server([g], max_batch=64, slots_per_graph=1, single_source_levels=0, fast_slots=0,
                       join=1 << 30) as srv:
            qs = {srv.submit(0, srcs[0]): srcs[0], srv.submit(0, srcs[1]): srcs[1]}
            time.sleep(0.003)
            for x in srcs[2:]:
                qs[srv.submit(0, x)] = x
                time.sleep(0.0002)
            res = _drain(srv, len(qs))
            c = srv.counters()
            assert c["joined"] > 0, c
            for r in res:
                src = qs[r["query_id"]]
                assert r["status"] == 0
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, src)
                np.testing.assert_array_equal(srv.depth(r["query_id"]), exp, err_msg=f"source {src}")
                assert (r["traversed_edges"], r["reached_vertices"]) == orc.report(csr.beg_pos, exp)
                assert r["levels"] == int(exp.max()) + 1
                srv.release(r["query_id"])
            c = srv.counters()
            assert c["completed"] == c["released"] == len(qs) and c["rows_free"] == c["rows_total"]
            assert c["batches"] < len(qs)
    finally:
        g.close()


@pytest.mark.parametrize("join", [0, 1])
def test_join_off_keeps_waiting_queries_for_the_next_batch(eb, orc, join):
    """With joining off, queries that arrive while the batch runs wait for the
    slot; with the default limit (level 1), they arrive too late to join this
    batch of a thousand levels and wait as well. Results are the same."""
    import time
    from conftest import tier_graph
    V, s, d = tier_graph()
    csr = eb.Csr.from_edges(s, d, V)
    g = eb.Graph.from_csr(csr)
    srcs = [5999, 5500] + [int(x) for x in eb.pick_sources(csr.beg_pos, 6, 20)]
    try:
        with eb.Server([g], max_batch=64, slots_per_graph=1, single_source_levels=0, fast_slots=0,
                       join=join) as srv:
            qs = {srv.submit(0, srcs[0]): srcs[0], srv.submit(0, srcs[1]): srcs[1]}
            time.sleep(0.003)
            for x in srcs[2:]:
                qs[srv.submit(0, x)] = x
            res = _drain(srv, len(qs))
            assert srv.counters()["joined"] == 0
            for r in res:
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, qs[r["query_id"]])
                np.testing.assert_array_equal(srv.depth(r["query_id"]), exp)
                srv.release(r["query_id"])
    finally:
        g.close()
