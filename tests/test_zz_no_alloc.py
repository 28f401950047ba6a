"""GPU test of ent_bfs_noalloc, the traversal that allocates no GPU memory.

It serves callers that may not allocate when they traverse (latency-critical
paths where cudaMalloc can synchronise the device, plug-ins whose process
memory belongs to another allocator or a fixed budget). The test calls it
through the C ABI, twice in a row on the same device (the second call reuses
the static scratch the first left behind), and checks each result bit-exact
against the existing ent_bfs entry point and the CPU oracle. This file is collected last so a
run that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(eb):
    f = eb.lib().ent_bfs_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]
    return f


def _run(eb, g, src, out):
    beg, adj = g.device_csr()
    rc = _noalloc(eb)(C.c_void_p(beg), C.c_void_p(adj), g.vert_count, int(src), C.c_void_p(out.data_ptr()), None)
    if rc != 0:
        raise eb.EntError(rc, eb.lib().ent_last_error().decode())


@pytest.mark.parametrize("kind", ["rmat", "grid", "hand"])
def test_noalloc_matches_ent_bfs_twice(eb, orc, kind):
    import torch
    if kind == "rmat":
        csr = eb.Csr.rmat(15, 16, seed=404)
    elif kind == "grid":
        csr = eb.Csr.grid(200, 150, 0.1, seed=405)
    else:
        csr = eb.Csr.from_edges([0, 1, 2, 4, 5], [1, 2, 3, 5, 6], 9)
    with eb.Graph.from_csr(csr) as g:
        out = torch.full((g.vert_count,), 7, dtype=torch.int32, device="cuda")
        srcs = eb.pick_sources(csr.beg_pos, 1, 2) if kind != "hand" else [0, 4]
        # two different sources, a repeat, and (hand graph) an isolated source
        order = list(srcs) + [srcs[0]] + ([7] if kind == "hand" else [])
        for src in order:
            _run(eb, g, src, out)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            ref, _, _ = g.bfs(int(src))
            np.testing.assert_array_equal(got, ref)  # the existing entry point
            exp, _ = orc.bfs(csr.beg_pos, csr.csr, int(src))
            np.testing.assert_array_equal(got, exp)  # and the CPU oracle


def test_noalloc_rejects_too_large_and_bad_source(eb):
    import torch
    f = _noalloc(eb)
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = f(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), (1 << 20) + 1, 0,
           C.c_void_p(dummy.data_ptr()), None)
    assert rc == 1 and b"no-allocation limit" in eb.lib().ent_last_error()
    rc = f(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), 4, 9, C.c_void_p(dummy.data_ptr()), None)
    assert rc == 1
