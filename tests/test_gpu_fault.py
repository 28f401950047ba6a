"""Failure detection on the GPU without a GPU fault: the only spin wait of the
traversal (the decoupled look-back of the frontier classification) is
bounded. With the fault_inject hook the first tile of a classification never
publishes its prefix, so the tiles waiting for it run out their spin limit;
the traversal must end with ENT_ERR_TIMEOUT (status read by the host, no trap,
no hang), and the same context must then run exact traversals again."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ENT_ERR_TIMEOUT = 6


@pytest.mark.parametrize("loop", ["graph", "host"])
def test_lookback_wait_runs_out_cleanly(eb, orc, loop):
    csr = eb.Csr.rmat(14, 16, seed=4321)
    src = int(eb.pick_sources(csr.beg_pos, 4322, 1)[0])
    exp, _ = orc.bfs(csr.beg_pos, csr.csr, src)
    with eb.Graph.from_csr(csr) as g:
        o = g.opts
        o.loop = eb.LOOP[loop]
        o.policy = eb.POLICY["td"]       # every level classified by the look-back scan
        o.narrow_max_frontier = 0        # no small-frontier kernel: all levels go through it
        o.fault_inject = 1
        g.opts = o
        t0 = time.time()
        with pytest.raises(eb.EntError) as ei:
            g.bfs(src)
        assert ei.value.code == ENT_ERR_TIMEOUT, str(ei.value)
        assert time.time() - t0 < 120
        o.fault_inject = 0
        g.opts = o
        for _ in range(2):
            d, _, st = g.bfs(src)
            np.testing.assert_array_equal(d, exp)
            assert st.status == 0
