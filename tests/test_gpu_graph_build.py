"""GPU tests of the device-side graph builder for a caller's edge list: it
gives the same canonical CSR as the host builder (both directions, self loops
and duplicates dropped, rows ascending), traversals on it match the oracle,
and bad input fails with a status."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("V,n,seed", [(1, 0, 1), (10, 0, 2), (50, 400, 3), (3000, 20000, 4), (1 << 17, 1 << 20, 5)])
def test_edge_list_same_csr_as_host(eb, V, n, seed):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, V, n)
    dst = rng.integers(0, V, n)
    if n:
        k = n // 10
        src[:k] = dst[:k]                                    # self loops
        src[k:2 * k], dst[k:2 * k] = src[3 * k:4 * k], dst[3 * k:4 * k]          # duplicates
        src[2 * k:3 * k], dst[2 * k:3 * k] = dst[4 * k:5 * k], src[4 * k:5 * k]  # reversed duplicates
    host = eb.Csr.from_edges(src, dst, V)
    with eb.Graph.from_edges(src, dst, V) as g:
        assert (g.vert_count, g.edge_count) == (host.vert_count, host.edge_count)
        dev = g.download()
        np.testing.assert_array_equal(dev.beg_pos, host.beg_pos)
        np.testing.assert_array_equal(dev.csr, host.csr)


def test_edge_list_traversal_matches_oracle(eb, orc):
    rng = np.random.default_rng(6)
    V = 5000
    src, dst = rng.integers(0, V, 30000), rng.integers(0, V, 30000)
    host = eb.Csr.from_edges(src, dst, V)
    with eb.Graph.from_edges(src, dst, V) as g:
        for s in eb.pick_sources(host.beg_pos, 8, 4):
            d, _, _ = g.bfs(int(s))
            np.testing.assert_array_equal(d, orc.bfs(host.beg_pos, host.csr, int(s))[0])


@pytest.mark.parametrize("bad_src,bad_dst", [(-1, 0), (0, 100), (100, 100)])
def test_edge_list_out_of_range(eb, bad_src, bad_dst):
    src = np.array([0, 1, bad_src, 2])
    dst = np.array([1, 2, bad_dst, 3])
    with pytest.raises(eb.EntError) as ei:
        eb.Graph.from_edges(src, dst, 100)
    assert ei.value.code == 5 and "edge 2" in str(ei.value)
