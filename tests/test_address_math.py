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
def test_flush_column_loads_and_stores(V, W):
    """load_cols<CG> / store_cols<CG> (the zeroing and the carry into slot 0):
    slot k + (v*W + cg) words, ulonglong2 pairs when CG >= 2."""
    cg_n = cg_of(W)
    if cg_n < 2:
        return
    for k in range(17):
        for v in range(min(V, 40)):
            for cg in range(0, W, cg_n):
                off = LOG_BASE_ALIGN + (k * V * W + v * W + cg) * 8
                for j in range(0, cg_n, 2):
                    assert (off + 8 * j) % 16 == 0


def flush_vec(V, depth_addr, windows, out_bytes):
    """FlushState::vec as k_b_flush forms it."""
    return windows == 0 and V % 4 == 0 and depth_addr % (4 if out_bytes else 16) == 0


@pytest.mark.parametrize("V,out_bytes", list(itertools.product(VERTS + [4096, 1 << 20], [False, True])))
def test_flush_vector_row_stores(V, out_bytes):
    """Vector row stores (int4 for int32 rows, one 32-bit word for byte rows)
    at row * V + v0 + sub + vi, vi a multiple of 4, only when vec holds; the
    span degrees are read as int4 at sub + vi."""
    esz = 1 if out_bytes else 4
    for depth_addr in (0x7f0000000000, 0x7f0000000004, 0x7f0000000008, 0x7f0000000001):
        if not flush_vec(V, depth_addr, 0, out_bytes):
            continue
        for cg_n in (1, 2, 4):
            vs = 1024 // cg_n
            for row in range(6):
                for v0 in range(0, min(V, 3072), 1024):
                    nv = min(1024, V - v0)
                    for sub in range(0, nv, vs):
                        nsub = min(vs, nv - sub)
                        assert nsub % 4 == 0  # whole groups of 4: no tail
                        for vi in range(0, nsub, 4):
                            off = depth_addr + (row * V + v0 + sub + vi) * esz
                            assert off % (4 * esz) == 0
                            assert ((sub + vi) * 4) % 16 == 0  # s_deg int4


def tile_word(cg_n, vi, c):
    if cg_n == 1:
        return vi * 16 + (c ^ (((vi >> 1) ^ (vi >> 5)) & 15))
    return vi * 16 * cg_n + (c ^ ((vi ^ (vi >> 5)) & 31))


@pytest.mark.parametrize("cg_n", [1, 2, 4])
def test_flush_tile_swizzle(cg_n):
    """The tile swizzle is a permutation of each vertex's row; a warp's decode
    stores (32 consecutive vertices) and scalar reads hit 32 banks; the vector
    reads (vertices base + 4l + t, base a multiple of 128) hit 32 banks, or 16
    (two lanes a bank) when CG == 1."""
    vs = 1024 // cg_n
    cols = 16 * cg_n
    for vi in range(vs):
        row = [tile_word(cg_n, vi, c) for c in range(cols)]
        assert sorted(row) == list(range(vi * cols, (vi + 1) * cols))
    for w0 in range(0, vs, 32):
        for c in range(cols):
            banks = {tile_word(cg_n, w0 + l, c) % 32 for l in range(32)}
            assert len(banks) == 32
    for base in range(0, vs, 128):
        for t in range(4):
            for c in range(cols):
                banks = [tile_word(cg_n, base + 4 * l + t, c) % 32 for l in range(32)]
                worst = max(banks.count(b) for b in set(banks))
                assert worst == (2 if cg_n == 1 else 1)


def sext_byte(w, j):
    """prmt.b32 in its default mode with selector j | (8+j) * 0x1110."""
    sel = j | ((8 + j) * 0x1110)
    out = 0
    for i in range(4):
        nib = (sel >> (4 * i)) & 15
        b = (w >> (8 * (nib & 7))) & 0xFF
        if nib & 8:
            b = 0xFF if b & 0x80 else 0
        out |= b << (8 * i)
    return out - (1 << 32) if out & 0x80000000 else out


def test_flush_byte_sign_extension():
    """Tile bytes are a slot index 0..15 or 0xFF (not found): byte j becomes the
    index or -1, and v = d + (rb & ~(d >> 31)) is the depth or -1."""
    import random
    rnd = random.Random(7)
    for _ in range(2000):
        bs = [rnd.choice([0xFF] + list(range(16))) for _ in range(4)]
        w = bs[0] | bs[1] << 8 | bs[2] << 16 | bs[3] << 24
        rb = rnd.randrange(0, 300)
        for j in range(4):
            d = sext_byte(w, j)
            assert d == (-1 if bs[j] == 0xFF else bs[j])
            m = -1 if d < 0 else 0
            v = d + (rb & ~m)
            assert v == (-1 if bs[j] == 0xFF else bs[j] + rb)
            if rb <= 239:  # the byte-row vector path: no depth above 254
                assert v <= 254


def test_flush_stat_sums_fit():
    """The per-lane degree sum (at most 32 vertices below 2^31) split at bit
    16 sums over 32 lanes in 32 bits; a pair of degrees fits 32 bits."""
    lane_max = 32 * (2**31 - 1)
    assert lane_max < 2**36
    assert 32 * (lane_max >> 16) < 2**32
    assert 32 * 0xFFFF < 2**32
    assert 2 * (2**31 - 1) < 2**32


def test_flush_smem_fits():
    """k_b_flush's dynamic shared memory at the largest batch (W = 32)."""
    tile, degs = 64 * 1024, 1024 * 4
    for W in WORDS:
        smem = tile + degs + W * 64 * (4 + 8 + 4) + 16
        assert smem <= 227 * 1024
        # s_edg follows s_cnt (W*64 words of 4 bytes): 8-byte aligned
        assert (tile + degs + W * 64 * 4) % 8 == 0
