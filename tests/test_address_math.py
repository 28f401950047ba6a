"""CPU checks of the address arithmetic behind every 16-byte vector access in
the batched kernels (bfs_batch.cu), for many graph and batch shapes. A
vector access must start on a 16-byte boundary; these mirror the offsets the
kernels form and assert the alignment the code relies on."""
import itertools

import pytest

WORDS = [1, 2, 4, 8, 16, 32]  # words per vertex (64 sources each)
VERTS = [1, 2, 3, 7, 8, 9, 31, 33, 1000, 1023, 4097]
LOG_BASE_ALIGN = 256  # the log is carved from a 256-byte aligned slab


def wpl_of(W):  # light tier: words per lane
    return min(W, 4)


def cg_of(W):  # flush: columns per pass
    return min(W, 4)


@pytest.mark.parametrize("V,W", list(itertools.product(VERTS, WORDS)))
def test_bottom_up_frontier_gathers(V, W):
    """load_words<WPL>: F + u*W + gl*WPL words, ulonglong2 when WPL >= 2."""
    wpl = wpl_of(W)
    if wpl < 2:
        return
    G = W // wpl
    for slot in range(3):
        slot_off = slot * V * W * 8
        for u in range(min(V, 40)):
            for gl in range(G):
                off = LOG_BASE_ALIGN + slot_off + (u * W + gl * wpl) * 8
                for j in range(0, wpl, 2):
                    assert (off + 8 * j) % 16 == 0


@pytest.mark.parametrize("V,W", list(itertools.product(VERTS, WORDS)))
def test_flush_column_loads(V, W):
    """load_cols<CG>: slot k + (v*W + cg) words, ulonglong2 pairs when CG >= 2."""
    cg_n = cg_of(W)
    if cg_n < 2:
        return
    for k in range(4):
        for v in range(min(V, 40)):
            for cg in range(0, W, cg_n):
                off = LOG_BASE_ALIGN + (k * V * W + v * W + cg) * 8
                for j in range(0, cg_n, 2):
                    assert (off + 8 * j) % 16 == 0


@pytest.mark.parametrize("V,W", list(itertools.product(VERTS, WORDS)))
def test_recycle_vector_path_only_when_aligned(V, W):
    """k_b_recycle uses ulonglong2 only when V*W is even: then every slot base is aligned."""
    vec = (V * W) % 2 == 0
    for k in range(17):
        base = LOG_BASE_ALIGN + k * V * W * 8
        if vec:
            assert base % 16 == 0
        elif k % 2 == 1:
            assert base % 16 != 0  # the case the scalar path exists for


@pytest.mark.parametrize("V", VERTS)
def test_flush_depth_row_stores(V):
    """int4 depth stores only when V % 4 == 0 (row starts s*V*4 bytes apart)."""
    vec_ok = V % 4 == 0
    for s in range(5):
        for q in range(0, min(V, 64) // 4):
            off = (s * V + q * 4) * 4
            if vec_ok:
                assert off % 16 == 0
