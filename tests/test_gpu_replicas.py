"""GPU tests of the replica set (ent_replicas_*): one graph on several GPUs,
a many-source request spread over them chunk by chunk, rows in input order.
With one GPU visible, the replicas are two handles of the graph on that GPU
(their batches run side by side and wait on nothing of each other); with more,
one replica per GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gpus():
    import torch
    n = torch.cuda.device_count()
    return list(range(n)) if n > 1 else [0, 0]


def test_replicas_rows_in_input_order(eb, orc):
    csr = eb.Csr.rmat(14, 16, seed=0x5EED000E)
    graphs = [eb.Graph.from_csr(csr, gpu=d) for d in _gpus()]
    try:
        srcs = [int(s) for s in eb.pick_sources(csr.beg_pos, 0x2E9, 300)]
        srcs[7] = srcs[3]  # a repeated source
        with eb.Replicas(graphs, max_batch=64) as r:
            rows, stats = r.bfs_batch(srcs)
            ran = r.sources_run()
            assert sum(ran) == len(srcs)
            for i, s in enumerate(srcs):
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, s)
                np.testing.assert_array_equal(rows[i], exp, err_msg=f"row {i} (source {s})")
                assert (stats[i].traversed_edges, stats[i].reached_vertices) == orc.report(csr.beg_pos, exp)
            rows8 = r.bfs_batch_u8(srcs[:70])
            for i in (0, 35, 69):
                exp, _ = orc.bfs(csr.beg_pos, csr.csr, srcs[i])
                np.testing.assert_array_equal(rows8[i], np.where(exp < 0, 255, exp).astype(np.uint8))
    finally:
        for g in graphs:
            g.close()


def test_replicas_reject_mismatched_graphs(eb):
    a = eb.Graph.from_csr(eb.Csr.rmat(10, 8, seed=1))
    b = eb.Graph.from_csr(eb.Csr.rmat(11, 8, seed=1))
    try:
        with pytest.raises(eb.EntError):
            eb.Replicas([a, b])
        with pytest.raises(eb.EntError):
            eb.Replicas([a, a])
        with eb.Replicas([a]) as r:
            with pytest.raises(eb.EntError):
                r.bfs_batch([a.vert_count])  # source out of range
    finally:
        a.close()
        b.close()
