"""CPU tests of the oracle: hand-made graphs, agreement of its three BFS
variants, planted mistakes caught by the certificates, and agreement with the
reference's own validate()/report() compiled from its sources."""
import numpy as np
import pytest

from conftest import hand_graphs, tier_graph


def _expected_depths(V, edges, src):
    """Pure-Python BFS, small cases only (independent of the C oracle)."""
    adj = [[] for _ in range(V)]
    for u, v in edges:
        if u != v:
            adj[u].append(v)
            adj[v].append(u)
    d = [-1] * V
    d[src] = 0
    frontier = [src]
    while frontier:
        nxt = []
        for u in frontier:
            for v in adj[u]:
                if d[v] == -1:
                    d[v] = d[u] + 1
                    nxt.append(v)
        frontier = nxt
    return np.array(d, dtype=np.int32)


@pytest.mark.parametrize("name,V,edges", hand_graphs())
def test_oracle_hand_graphs(eb, orc, name, V, edges):
    e = np.array(edges, dtype=np.int64)
    g = eb.Csr.from_edges(e[:, 0], e[:, 1], V)
    for src in range(V):
        exp = _expected_depths(V, edges, src)
        d0, p0 = orc.bfs(g.beg_pos, g.csr, src, parents=True)
        d1, p1 = orc.bfs_omp(g.beg_pos, g.csr, src, threads=3, parents=True)
        d2 = orc.bfs_omp_do(g.beg_pos, g.csr, src, threads=2)
        np.testing.assert_array_equal(d0, exp)
        np.testing.assert_array_equal(d1, exp)
        np.testing.assert_array_equal(d2, exp)
        assert orc.check_depths(g.beg_pos, g.csr, src, d0)[0] == 0
        assert orc.check_parents(g.beg_pos, g.csr, src, d0, p0)[0] == 0
        assert orc.check_parents(g.beg_pos, g.csr, src, d1, p1)[0] == 0


def test_oracle_known_answers(eb, orc):
    # path 0-1-...-7 from 3: depths |i-3|
    e = np.array([(i, i + 1) for i in range(7)])
    g = eb.Csr.from_edges(e[:, 0], e[:, 1], 8)
    d, _ = orc.bfs(g.beg_pos, g.csr, 3)
    assert d.tolist() == [3, 2, 1, 0, 1, 2, 3, 4]
    # two components: the other side is unreached (-1)
    e = np.array([(0, 1), (1, 2), (3, 4)])
    g = eb.Csr.from_edges(e[:, 0], e[:, 1], 6)
    d, p = orc.bfs(g.beg_pos, g.csr, 0, parents=True)
    assert d.tolist() == [0, 1, 2, -1, -1, -1]
    assert p.tolist() == [0, 0, 1, -1, -1, -1]
    assert orc.report(g.beg_pos, d) == (4, 3)


@pytest.mark.parametrize("scale,ef,abc,seed", [(10, 16, (0.57, 0.19, 0.19), 1), (14, 16, (0.57, 0.19, 0.19), 0x5EED000E),
                                               (13, 8, (0.45, 0.15, 0.15), 77)])
def test_oracle_generator_is_the_products(eb, orc, scale, ef, abc, seed):
    """The benchmark's CPU arm rebuilds the GPU arm's graph and sources with the
    oracle's own generator: same CSR and same seeded sources, bit for bit."""
    a, b, c = abc
    beg, adj = orc.gen_rmat(scale, ef, a, b, c, seed=seed)
    csr = eb.Csr.rmat(scale, ef, a=a, b=b, c=c, seed=seed)
    np.testing.assert_array_equal(beg, csr.beg_pos)
    np.testing.assert_array_equal(adj, csr.csr)
    for s in (0, 5, 0x50C0018):
        np.testing.assert_array_equal(orc.pick_sources(beg, s, 64), eb.pick_sources(csr.beg_pos, s, 64))


def test_oracle_variants_agree_rmat(eb, orc):
    g = eb.Csr.rmat(12, 16, seed=11)
    for s in eb.pick_sources(g.beg_pos, 5, 8):
        d0, _ = orc.bfs(g.beg_pos, g.csr, s)
        np.testing.assert_array_equal(orc.bfs_omp(g.beg_pos, g.csr, s)[0], d0)
        np.testing.assert_array_equal(orc.bfs_omp_do(g.beg_pos, g.csr, s), d0)


def test_oracle_tier_graph_many_levels(eb, orc):
    V, s, d = tier_graph()
    g = eb.Csr.from_edges(s, d, V)
    d0, p0 = orc.bfs(g.beg_pos, g.csr, 0, parents=True)
    assert d0.max() > 900
    np.testing.assert_array_equal(orc.bfs_omp_do(g.beg_pos, g.csr, 0), d0)
    assert orc.check_parents(g.beg_pos, g.csr, 0, d0, p0)[0] == 0


def test_certificates_catch_planted_mistakes(eb, orc):
    """Mistakes are planted in a copy of the oracle's output, on the CPU."""
    g = eb.Csr.rmat(10, 8, seed=3)
    src = int(eb.pick_sources(g.beg_pos, 1, 1)[0])
    d, p = orc.bfs(g.beg_pos, g.csr, src, parents=True)
    reached = np.flatnonzero(d > 0)
    v = int(reached[len(reached) // 2])
    bad = d.copy(); bad[v] += 1
    assert orc.check_depths(g.beg_pos, g.csr, src, bad)[0] != 0
    bad = d.copy(); bad[v] = -1
    assert orc.check_depths(g.beg_pos, g.csr, src, bad)[0] != 0
    bad = d.copy(); bad[src] = 1
    assert orc.check_depths(g.beg_pos, g.csr, src, bad)[0] != 0
    badp = p.copy(); badp[v] = v
    assert orc.check_parents(g.beg_pos, g.csr, src, d, badp)[0] != 0
    badp = p.copy(); badp[src] = -1
    assert orc.check_parents(g.beg_pos, g.csr, src, d, badp)[0] != 0
    # a parent one level up that is not adjacent
    same_level_up = np.flatnonzero(d == d[v] - 1)
    nbrs = set(g.csr[g.beg_pos[v]:g.beg_pos[v + 1]].tolist())
    non_adj = [u for u in same_level_up.tolist() if u not in nbrs]
    if non_adj:
        badp = p.copy(); badp[v] = non_adj[0]
        assert orc.check_parents(g.beg_pos, g.csr, src, d, badp)[0] == -5


def test_reference_validate_and_report_agree(eb, orc):
    """The reference's own validate()/report() (validate.h:34-127), compiled
    unmodified from its sources, accept the oracle's depths and count the
    same edges and vertices."""
    if orc.ref() is None:
        pytest.skip("reference validate() not built (reference sources absent)")
    g = eb.Csr.rmat(14, 16, seed=0x5EED)
    for s in eb.pick_sources(g.beg_pos, 9, 6):
        d, _ = orc.bfs(g.beg_pos, g.csr, s)
        assert d.max() < 255
        assert orc.ref_validate(g.beg_pos, g.csr, d, times=2000) == 0
        assert orc.ref_report(g.beg_pos, d) == orc.report(g.beg_pos, d)
    # and reject a planted mistake: every reached vertex shifted on one side
    d, _ = orc.bfs(g.beg_pos, g.csr, int(s))
    bad = d.copy()
    bad[d == 2] = 4
    assert orc.ref_validate(g.beg_pos, g.csr, bad, times=20000) != 0
