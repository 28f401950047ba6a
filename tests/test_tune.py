"""Autotuner: the cache logic on CPU (with a stand-in search), the native
search on the GPU (chosen options stay within the candidates and depths stay
bit-exact)."""
import numpy as np
import pytest


def test_graph_class_and_key():
    from enterprise_b200.tune import TuneCache, graph_class
    assert graph_class(1 << 24, 520_000_000, "rmat") == "rmat-v2^24-d31"
    assert graph_class(4096, 8192) == "v2^12-d2"
    assert TuneCache.key("B200", "x", "single") == "B200|x|single"


def test_cache_roundtrip_and_reuse(tmp_path, eb):
    from enterprise_b200 import tune

    class FakeGraph:
        vert_count, edge_count = 1 << 16, 1 << 20

        def __init__(self):
            self.applied = None

        @property
        def opts(self):
            return self.applied

        @opts.setter
        def opts(self, o):
            self.applied = o

    calls = []

    def fake_search(graph, sources, mode, reps):
        calls.append(mode)
        o = eb.BfsOpts(small_max=64, alpha=32.0, batch_alpha=8.0)
        return o, 1.25

    cache = tune.TuneCache(str(tmp_path / "t.json"))
    g = FakeGraph()
    o, ms, hit = tune.autotune(g, [1, 2], "single", cache=cache, label="rmat", searcher=fake_search)
    assert (hit, ms, o.small_max) == (False, 1.25, 64)
    again = tune.TuneCache(str(tmp_path / "t.json"))
    o2, ms2, hit2 = tune.autotune(g, [1, 2], "single", cache=again, label="rmat", searcher=fake_search)
    assert hit2 and ms2 is None and o2 == o and g.applied == o
    assert calls == ["single"]
    o3, _, hit3 = tune.autotune(g, [1, 2], "batch", cache=again, label="rmat", searcher=fake_search)
    assert not hit3 and calls == ["single", "batch"]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["single", "batch"])
def test_native_search_keeps_results_exact(eb, orc, mode):
    from enterprise_b200 import tune
    csr = eb.Csr.rmat(13, 16, seed=123)
    srcs = eb.pick_sources(csr.beg_pos, 5, 6 if mode == "single" else 70)
    with eb.Graph.from_csr(csr) as g:
        opts, ms = tune.search(g, srcs, mode, reps=1)
        assert ms > 0
        assert opts.small_max in (16, 32, 64, 128, 256) and opts.batch_small_max in (16, 32, 64)
        assert g.opts == opts
        for s in srcs[:3]:
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(s))
            np.testing.assert_array_equal(g.bfs(int(s))[0], exp)
        d, _ = g.bfs_batch(srcs[:5])
        for i in range(5):
            np.testing.assert_array_equal(d[i], orc.bfs(csr.beg_pos, csr.csr, int(srcs[i]))[0])


def test_shipped_results_cover_the_headline_class(eb, tmp_path):
    """The package ships an earlier B200 search for R-MAT scale 24 edge factor
    16; a fresh cache falls back to it, and the user's own entries win."""
    from dataclasses import asdict
    from enterprise_b200 import tune
    key = tune.TuneCache.key("NVIDIA B200", tune.graph_class(1 << 24, 520772318, "rmat"), "single")
    cache = tune.TuneCache(str(tmp_path / "none.json"))
    assert cache.source(key) == "shipped"
    o = cache.get(key)
    assert (o.alpha, o.beta, o.small_max, o.large_min, o.chunk_edges) == (48.0, 1024.0, 16, 128, 256)
    o.alpha = 12.0
    cache.put(key, o, 1.0)
    again = tune.TuneCache(str(tmp_path / "none.json"))
    assert again.source(key) == "user" and again.get(key).alpha == 12.0
    assert tune.TuneCache(str(tmp_path / "x.json"), shipped=None).source(key) is None
