"""GPU tests of ent_validate (Graph500-style certificates on the device):
on correct results it accepts, and on damaged results it reports exactly the
rule and vertex the CPU oracle reports (check_depths / check_parents). The
damage is planted in the host arrays handed to the validator (valid memory,
wrong values), never in a kernel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _both(orc, csr, g, src, depth, parent):
    (dc, db), pres = g.validate(src, depth, parent)
    exp_d = orc.check_depths(csr.beg_pos, csr.csr, src, depth)
    assert (dc, db) == exp_d
    if parent is not None:
        exp_p = orc.check_parents(csr.beg_pos, csr.csr, src, depth, parent)
        assert pres == exp_p
    return (dc, db), pres


@pytest.mark.parametrize("kind", ["rmat", "grid", "er"])
def test_correct_results_pass(eb, orc, kind):
    csr = {"rmat": lambda: eb.Csr.rmat(13, 16, seed=41), "grid": lambda: eb.Csr.grid(90, 70, 0.1, seed=42),
           "er": lambda: eb.Csr.er(6000, 10.0, seed=43)}[kind]()
    with eb.Graph.from_csr(csr) as g:
        for src in eb.pick_sources(csr.beg_pos, 5, 6):
            d, p, _ = g.bfs(int(src), parents=True)
            assert _both(orc, csr, g, int(src), d, p) == ((0, -1), (0, -1))


def test_damaged_results_match_the_oracle(eb, orc):
    csr = eb.Csr.rmat(12, 8, seed=44)
    rng = np.random.default_rng(9)
    with eb.Graph.from_csr(csr) as g:
        src = int(eb.pick_sources(csr.beg_pos, 6, 1)[0])
        d0, p0, _ = g.bfs(src, parents=True)
        reached = np.flatnonzero(d0 > 0)
        unreached = np.flatnonzero(d0 < 0)
        cases = []
        for _ in range(12):
            d, p = d0.copy(), p0.copy()
            kind = rng.integers(9)
            v = int(rng.choice(reached))
            if kind == 0:
                d[v] += 1                      # depth too deep (-5 or -6 somewhere)
            elif kind == 1:
                d[v] -= 1                      # depth too shallow
            elif kind == 2:
                d[v] = -7                      # below -1
            elif kind == 3 and len(unreached):
                u = int(rng.choice(unreached)); p[u] = v   # unreached vertex with a parent
            elif kind == 4:
                p[v] = csr.vert_count + 5      # parent out of range
            elif kind == 5:
                p[v] = int(rng.choice(np.flatnonzero(d0 == d0[v])))  # same depth: never a parent
            elif kind == 6:
                d[src] = 1                     # source not at depth 0
            elif kind == 7:
                p[src] = v                     # source's parent not itself
            else:
                d[v] = 0                       # a second depth-0 vertex
            cases.append((d, p))
        for d, p in cases:
            (dc, _), (pc, _) = _both(orc, csr, g, src, d, p)
            assert dc != 0 or pc != 0


def test_unsorted_rows_from_a_caller_csr(eb, orc):
    """A caller's CSR may list a row's neighbours in any order: the parent
    certificate sorts a copy for its edge search."""
    csr = eb.Csr.rmat(11, 8, seed=45)
    beg, adj = csr.beg_pos.copy(), csr.csr.copy()
    rng = np.random.default_rng(3)
    for v in range(csr.vert_count):
        rng.shuffle(adj[beg[v]:beg[v + 1]])
    shuffled = eb.Csr(beg, adj)
    with eb.Graph.from_arrays(beg, adj) as g:
        src = int(eb.pick_sources(beg, 7, 1)[0])
        d, p, _ = g.bfs(src, parents=True)
        assert _both(orc, shuffled, g, src, d, p) == ((0, -1), (0, -1))
        p2 = p.copy()
        v = int(np.flatnonzero(d == 2)[0])
        p2[v] = int(np.flatnonzero(d == 1)[-1]) if p[v] != np.flatnonzero(d == 1)[-1] else int(np.flatnonzero(d == 1)[0])
        _both(orc, shuffled, g, src, d, p2)


def test_validate_without_parents(eb, orc):
    csr = eb.Csr.grid(40, 40, 0.1, seed=46)
    with eb.Graph.from_csr(csr) as g:
        d, _, _ = g.bfs(0)
        (dc, db), pres = g.validate(0, d)
        assert (dc, db) == (0, -1) and pres is None
