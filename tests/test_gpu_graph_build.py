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


def _write(tmp_path, beg, adj, width=8, name="g"):
    b, c = tmp_path / f"{name}_beg_pos.bin", tmp_path / f"{name}_csr.bin"
    np.asarray(beg, dtype=np.int64).tofile(b)
    np.asarray(adj, dtype=np.int64 if width == 8 else np.int32).tofile(c)
    return str(b), str(c)


@pytest.mark.parametrize("width", [8, 4])
def test_load_streams_the_same_csr(eb, tmp_path, width):
    host = eb.Csr.rmat(15, 16, seed=91)
    b, c = _write(tmp_path, host.beg_pos, host.csr, width)
    with eb.Graph.load(b, c) as g:
        dev = g.download()
        np.testing.assert_array_equal(dev.beg_pos, host.beg_pos)
        np.testing.assert_array_equal(dev.csr, host.csr)
        src = int(eb.pick_sources(host.beg_pos, 3, 1)[0])
        np.testing.assert_array_equal(g.bfs(src)[0], eb.Graph.from_csr(host).bfs(src)[0])


def test_load_many_chunks(eb, tmp_path):
    """More than two 64 MB chunks of int64 ids: the pinned buffers take turns."""
    host = eb.Csr.rmat(20, 16, seed=92)
    assert host.edge_count * 8 > 3 * (64 << 20)
    b, c = _write(tmp_path, host.beg_pos, host.csr, 8)
    with eb.Graph.load(b, c) as g:
        dev = g.download()
        np.testing.assert_array_equal(dev.beg_pos, host.beg_pos)
        np.testing.assert_array_equal(dev.csr, host.csr)


def _broken_files(tmp_path):
    beg = np.array([0, 2, 3, 5, 6], dtype=np.int64)
    adj = np.array([1, 2, 0, 0, 3, 2], dtype=np.int64)
    cases = {}
    cases["id_out_of_range"] = _write(tmp_path, beg, [1, 2, 0, 0, 9, 2], 8, "a")
    cases["id_negative_int32"] = _write(tmp_path, beg, [1, -2, 0, 0, 3, 2], 4, "b")
    cases["not_monotone"] = _write(tmp_path, [0, 2, 1, 5, 6], adj, 8, "c")
    cases["first_not_zero"] = _write(tmp_path, [1, 2, 3, 5, 6], adj, 8, "d")
    cases["csr_size_mismatch"] = _write(tmp_path, beg, adj[:5], 8, "e")
    b, c = _write(tmp_path, beg, adj, 8, "f")
    with open(b, "ab") as f:
        f.write(b"\x00\x01\x02")  # not a multiple of 8 bytes
    cases["beg_size"] = (b, c)
    cases["missing"] = (str(tmp_path / "nope_beg_pos.bin"), c)
    return cases


def test_load_errors_match_the_host_loader(eb, tmp_path):
    for name, (b, c) in _broken_files(tmp_path).items():
        with pytest.raises(eb.EntError) as host:
            eb.Csr.load(b, c)
        with pytest.raises(eb.EntError) as dev:
            eb.Graph.load(b, c)
        assert (dev.value.code, str(dev.value)) == (host.value.code, str(host.value)), name
