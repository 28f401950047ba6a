"""CPU tests of the graph boundary: the reference's binary CSR format
(graph.hpp:33-118), the canonical builder and the seeded generators."""
import ctypes
import os

import numpy as np
import pytest

from conftest import hand_graphs


def _canonical(g):
    V = g.vert_count
    rows = np.repeat(np.arange(V, dtype=np.int64), np.diff(g.beg_pos))
    return rows, g.csr.astype(np.int64)


@pytest.mark.parametrize("kind", ["rmat", "grid", "er"])
def test_generators_canonical(eb, kind):
    if kind == "rmat":
        g = eb.Csr.rmat(12, 16, seed=1)
    elif kind == "grid":
        g = eb.Csr.grid(50, 40, 0.1, seed=2)
    else:
        g = eb.Csr.er(3000, 10.0, seed=3)
    rows, cols = _canonical(g)
    V = g.vert_count
    assert g.beg_pos[0] == 0 and g.beg_pos[-1] == g.edge_count
    assert np.all(np.diff(g.beg_pos) >= 0)
    assert np.all((cols >= 0) & (cols < V))
    assert not np.any(rows == cols), "self loop"
    k = rows * V + cols
    assert np.all(np.diff(k) > 0), "rows sorted ascending, no duplicates"
    assert np.array_equal(np.sort(k), np.sort(cols * V + rows)), "symmetric"


def test_generators_deterministic_and_seeded(eb):
    a = eb.Csr.rmat(11, 8, seed=42)
    b = eb.Csr.rmat(11, 8, seed=42)
    c = eb.Csr.rmat(11, 8, seed=43)
    assert np.array_equal(a.beg_pos, b.beg_pos) and np.array_equal(a.csr, b.csr)
    assert not np.array_equal(a.csr, c.csr)


def test_grid_shape(eb):
    w, h = 30, 20
    full = eb.Csr.grid(w, h, 0.0, seed=1)
    assert full.edge_count == 2 * (h * (w - 1) + (h - 1) * w)
    deg = full.degrees()
    assert sorted(np.bincount(deg).nonzero()[0].tolist()) == [2, 3, 4]
    dropped = eb.Csr.grid(w, h, 0.1, seed=1)
    frac = 1 - dropped.edge_count / full.edge_count
    assert 0.03 < frac < 0.2


def test_rmat_skew(eb):
    g = eb.Csr.rmat(14, 16, seed=0x5EED0016)
    deg = g.degrees()
    assert deg.max() > 50 * deg.mean()  # heavy tail
    assert (deg == 0).sum() > 0.1 * g.vert_count  # Graph500 R-MAT leaves many isolated vertices


@pytest.mark.parametrize("name,V,edges", hand_graphs())
def test_save_load_roundtrip_int64(eb, tmp_path, name, V, edges):
    e = np.array(edges, dtype=np.int64)
    g = eb.Csr.from_edges(e[:, 0], e[:, 1], V)
    bp, cp = str(tmp_path / "g_beg_pos.bin"), str(tmp_path / "g_csr.bin")
    g.save(bp, cp)
    assert os.path.getsize(bp) == 8 * (V + 1)
    assert os.path.getsize(cp) == 8 * g.edge_count  # reference format: int64 csr
    h = eb.Csr.load(bp, cp)
    assert np.array_equal(h.beg_pos, g.beg_pos) and np.array_equal(h.csr, g.csr)


def test_load_int32_csr_autodetect(eb, tmp_path):
    g = eb.Csr.rmat(8, 4, seed=9)
    bp, cp = tmp_path / "b.bin", tmp_path / "c.bin"
    g.beg_pos.astype(np.int64).tofile(bp)
    g.csr.astype(np.int32).tofile(cp)
    h = eb.Csr.load(str(bp), str(cp))
    assert np.array_equal(h.csr, g.csr)


def test_load_errors_are_status_codes(eb, tmp_path):
    bp, cp = tmp_path / "b.bin", tmp_path / "c.bin"
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.load(str(tmp_path / "missing"), str(cp))
    assert ei.value.code == 4
    np.array([0, 2, 1, 3], dtype=np.int64).tofile(bp)  # not monotone
    np.array([1, 2, 0], dtype=np.int64).tofile(cp)
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.load(str(bp), str(cp))
    assert ei.value.code == 5
    np.array([0, 1, 2, 3], dtype=np.int64).tofile(bp)
    np.array([1, 7, 0], dtype=np.int64).tofile(cp)  # id out of range
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.load(str(bp), str(cp))
    assert ei.value.code == 5
    np.array([1, 2], dtype=np.int64).tofile(cp)  # truncated csr
    with pytest.raises(eb.EntError) as ei:
        eb.Csr.load(str(bp), str(cp))
    assert ei.value.code == 5
    with open(bp, "wb") as f:
        f.write(b"\0" * 12)  # not a multiple of 8
    with pytest.raises(eb.EntError):
        eb.Csr.load(str(bp), str(cp))


def test_pick_sources(eb):
    g = eb.Csr.rmat(10, 4, seed=2)
    s = eb.pick_sources(g.beg_pos, 77, 64)
    assert len(set(s.tolist())) == 64
    assert np.all(g.degrees()[s] > 0)
    assert np.array_equal(s, eb.pick_sources(g.beg_pos, 77, 64))
    with pytest.raises(eb.EntError):
        eb.pick_sources(g.beg_pos, 1, g.vert_count + 1)


def test_pick_sources_compat_matches_glibc_rand(eb):
    """Same draws as main.cu:55-78: rand()%V, reject orphans and repeats."""
    libc = ctypes.CDLL(None)
    g = eb.Csr.rmat(10, 2, seed=5)
    deg = g.degrees()
    libc.srand(1)
    got = eb.pick_sources_compat(g.beg_pos, 64)
    libc.srand(1)
    exp = []
    V = g.vert_count
    while len(exp) < 64:
        s = libc.rand() % V
        if deg[s] == 0 or s in exp:
            continue
        exp.append(s)
    assert got.tolist() == exp


def test_device_load_checks_format_before_any_gpu(eb, tmp_path):
    """The streamed loader rejects malformed files with the host loader's
    status and message before it needs a device."""
    b, c = tmp_path / "x_beg_pos.bin", tmp_path / "x_csr.bin"
    np.array([1, 2, 3], dtype=np.int64).tofile(b)
    np.array([1, 0, 0], dtype=np.int64).tofile(c)
    with pytest.raises(eb.EntError) as host:
        eb.Csr.load(str(b), str(c))
    with pytest.raises(eb.EntError) as dev:
        eb.Graph.load(str(b), str(c))
    assert (dev.value.code, str(dev.value)) == (host.value.code, str(host.value))
