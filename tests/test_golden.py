"""Golden vectors produced by the reference's own GPU BFS (bfs_tdbu_clfy_sort,
compiled unmodified from its sources for sm_100a and run on a B200 by
tests/golden/make_golden.py). They pin the CPU oracle to the reference
(CPU test) and check this library's CUDA path against the reference directly
(GPU test). Graph files are in the reference's binary format (int64)."""
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(f[: -len("_ref_depth.bin")] for f in os.listdir(HERE) if f.endswith("_ref_depth.bin"))


def _load(eb, name):
    csr = eb.Csr.load(os.path.join(HERE, f"{name}_beg_pos.bin"), os.path.join(HERE, f"{name}_csr.bin"))
    srcs = [int(x) for x in open(os.path.join(HERE, f"{name}_sources.txt")).read().split()]
    raw = np.fromfile(os.path.join(HERE, f"{name}_ref_depth.bin"), dtype=np.uint8)
    raw = raw.reshape(len(srcs), csr.vert_count)
    ref = np.where(raw == 0xFF, -1, raw.astype(np.int32)).astype(np.int32)  # INFTY -> -1
    return csr, srcs, ref


def test_fixture_set_is_complete():
    assert len(NAMES) >= 6
    for n in NAMES:
        for suffix in ("_beg_pos.bin", "_csr.bin", "_sources.txt"):
            assert os.path.exists(os.path.join(HERE, n + suffix))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_gpu_bfs(eb, orc, name):
    csr, srcs, ref = _load(eb, name)
    for i, s in enumerate(srcs):
        d, _ = orc.bfs(csr.beg_pos, csr.csr, s)
        np.testing.assert_array_equal(d, ref[i], err_msg=f"{name} source {s}")
        assert orc.report(csr.beg_pos, d) == orc.report(csr.beg_pos, ref[i])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_path_matches_reference_gpu_bfs(eb, name):
    csr, srcs, ref = _load(eb, name)
    with eb.Graph.from_csr(csr) as g:
        for policy in ("beamer", "reference", "td", "bu"):
            o = g.opts
            o.policy = eb.POLICY[policy]
            g.opts = o
            for i, s in enumerate(srcs):
                np.testing.assert_array_equal(g.bfs(s)[0], ref[i], err_msg=f"{name} {policy} source {s}")
        d, _ = g.bfs_batch(srcs)
        np.testing.assert_array_equal(d, ref)
