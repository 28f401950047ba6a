"""A seeded sweep of small graphs of every kind (R-MAT, Erdős–Rényi, grids,
sparse random edge lists with isolated vertices) through every traversal
entry point, all against the CPU oracle: single sources through both loop
drivers under a random direction policy (parents checked), a batch with
duplicate and isolated sources (int32 and byte rows, per-source statistics),
and one multi-graph plan over the whole sweep."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_CASES = 96


def _case(eb, seed):
    rng = np.random.default_rng(0x5EE9 + seed)
    kind = seed % 4
    if kind == 0:
        csr = eb.Csr.rmat(int(rng.integers(8, 13)), int(rng.choice([4, 8, 16])), seed=int(rng.integers(1 << 30)))
    elif kind == 1:
        csr = eb.Csr.er(int(rng.integers(500, 5000)), float(rng.uniform(1.0, 12.0)), seed=int(rng.integers(1 << 30)))
    elif kind == 2:
        csr = eb.Csr.grid(int(rng.integers(10, 60)), int(rng.integers(10, 60)), float(rng.uniform(0.0, 0.3)),
                          seed=int(rng.integers(1 << 30)))
    else:
        V = int(rng.integers(100, 3000))
        m = int(rng.integers(V // 4, 3 * V))
        s, d = rng.integers(0, V, m), rng.integers(0, V, m)
        csr = eb.Csr.from_edges(s, d, V)
    return rng, csr


def _opts(eb, g, rng):
    o = g.opts
    o.policy = eb.POLICY[str(rng.choice(["beamer", "reference", "td", "bu"]))]
    o.alpha = float(rng.choice([2.0, 14.0, 48.0]))
    o.beta = float(rng.choice([4.0, 24.0, 1024.0]))
    o.batch_alpha = float(rng.choice([1.0, 4.0, 16.0]))
    o.batch_small_max = int(rng.choice([4, 32, 64]))
    o.batch_large_min = int(rng.choice([64, 1024]))
    g.opts = o


@pytest.fixture(scope="module")
def sweep(eb):
    cases = [_case(eb, k) for k in range(N_CASES)]
    yield cases


@pytest.mark.parametrize("k", range(N_CASES))
def test_sweep_case(eb, orc, sweep, k):
    rng, csr = sweep[k]
    V = csr.vert_count
    exp_of = {}

    def exp(s):
        if s not in exp_of:
            exp_of[s] = orc.bfs(csr.beg_pos, csr.csr, int(s))[0]
        return exp_of[s]

    with eb.Graph.from_csr(csr) as g, eb.Graph.from_csr(csr) as gh:
        _opts(eb, g, rng)
        o = gh.opts
        o.policy, o.loop = g.opts.policy, eb.LOOP["host"]
        gh.opts = o
        for s in rng.integers(0, V, 4):
            for gg in (g, gh):
                d, p, st = gg.bfs(int(s), parents=True)
                np.testing.assert_array_equal(d, exp(s), err_msg=f"case {k} source {s}")
                assert orc.check_parents(csr.beg_pos, csr.csr, int(s), d, p)[0] == 0
                assert (st.traversed_edges, st.reached_vertices) == orc.report(csr.beg_pos, exp(s))
        n = int(rng.integers(1, 150))
        srcs = rng.integers(0, V, n)
        srcs[n // 2] = srcs[0]  # a duplicate
        rows, sts = g.bfs_batch(srcs)
        for i, s in enumerate(srcs):
            np.testing.assert_array_equal(rows[i], exp(s), err_msg=f"case {k} batch row {i}")
            assert (sts[i].traversed_edges, sts[i].reached_vertices) == orc.report(csr.beg_pos, exp(s))
        if max(int(exp(s).max()) for s in srcs) <= 254:
            rows8, _ = g.bfs_batch_u8(srcs)
            for i, s in enumerate(srcs):
                np.testing.assert_array_equal(rows8[i], np.where(exp(s) < 0, 255, exp(s)).astype(np.uint8))


def test_sweep_as_one_plan(eb, orc, sweep):
    """Every graph of the sweep in one multi-graph plan (several width
    classes), the first and last row of each against the oracle."""
    graphs, srcs = [], []
    try:
        for k, (_, csr) in enumerate(sweep):
            rng = np.random.default_rng(0xA11 + k)
            graphs.append(eb.Graph.from_csr(csr))
            srcs.append(rng.integers(0, csr.vert_count, int(rng.integers(1, 140))).astype(np.int32))
        with eb.MultiPlan(graphs, srcs) as plan:
            plan.run()
            for k, (_, csr) in enumerate(sweep):
                d = plan.depths(k)
                for i in (0, len(srcs[k]) - 1):
                    exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(srcs[k][i]))
                    np.testing.assert_array_equal(d[i], exp, err_msg=f"plan graph {k} row {i}")
    finally:
        for g in graphs:
            g.close()
