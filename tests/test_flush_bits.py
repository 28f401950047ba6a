"""CPU mirror of the batched flush's decode arithmetic (bfs_batch.cu): the slot
fold in groups of four and the bit-block transpose that turns a vertex's found
mask and slot-index planes into tile bytes. Each step is restated as the
kernel forms it and checked against the direct definition (byte = slot index
of the source, 0xFF where not found) on random slot words."""
import random

M32 = 0xFFFFFFFF


def swap_blocks(a, b, s, mask):
    t = ((a >> s) ^ b) & mask
    b ^= t
    a ^= (t << s) & M32
    return a, b


def byte_perm(x, y, sel):
    src = x | (y << 32)
    out = 0
    for i in range(4):
        k = (sel >> (4 * i)) & 7
        out |= ((src >> (8 * k)) & 0xFF) << (8 * i)
    return out


def byte_transpose4(a, b, c, d):
    ab_lo, ab_hi = byte_perm(a, b, 0x5140), byte_perm(a, b, 0x7362)
    cd_lo, cd_hi = byte_perm(c, d, 0x5140), byte_perm(c, d, 0x7362)
    return (byte_perm(ab_lo, cd_lo, 0x5410), byte_perm(ab_lo, cd_lo, 0x7632),
            byte_perm(ab_hi, cd_hi, 0x5410), byte_perm(ab_hi, cd_hi, 0x7632))


def planes_to_tile_words(f, h0, h1, h2, h3):
    nf = ~f & M32
    r = [h0 | nf, h1 | nf, h2 | nf, h3 | nf, nf, nf, nf, nf]
    for (i, j) in ((0, 1), (2, 3), (4, 5), (6, 7)):
        r[i], r[j] = swap_blocks(r[i], r[j], 1, 0x55555555)
    for (i, j) in ((0, 2), (1, 3), (4, 6), (5, 7)):
        r[i], r[j] = swap_blocks(r[i], r[j], 2, 0x33333333)
    for (i, j) in ((0, 4), (1, 5), (2, 6), (3, 7)):
        r[i], r[j] = swap_blocks(r[i], r[j], 4, 0x0F0F0F0F)
    out = [0] * 8
    out[0], out[2], out[4], out[6] = byte_transpose4(r[0], r[1], r[2], r[3])
    out[1], out[3], out[5], out[7] = byte_transpose4(r[4], r[5], r[6], r[7])
    return out


def fold(slots, first, last):
    """The kernel's fold: groups of four slots from 0, pairs (ka, ka+1)."""
    f = p0 = p1 = p2 = p3 = 0
    for k0 in range(0, last + 1, 4):
        for h in range(2):
            ka, kb = k0 + 2 * h, k0 + 2 * h + 1
            wa = slots[ka] if first <= ka <= last else 0
            wb = slots[kb] if first <= kb <= last else 0
            u = wa | wb
            f |= u
            p0 |= wb
            if h:
                p1 |= u
            if k0 & 4:
                p2 |= u
            if k0 & 8:
                p3 |= u
    return f, p0, p1, p2, p3


def random_slots(rnd, n_slots, first):
    """Disjoint 64-bit slot words: each source is found in at most one slot."""
    slots = [0] * 16
    for s in range(64):
        k = rnd.randrange(-1, n_slots)
        if k >= first:
            slots[k] |= 1 << s
    return slots


def test_tile_bytes_match_definition():
    rnd = random.Random(0xF1A5)
    for trial in range(400):
        first = rnd.choice([0, 1])
        last = rnd.randrange(first, 16)
        slots = random_slots(rnd, last + 1, first)
        # a stale word outside [first, last] must be ignored
        if first == 1:
            slots[0] = rnd.getrandbits(64)
        f, p0, p1, p2, p3 = fold(slots, first, last)
        for hw in range(2):
            sh = 32 * hw
            words = planes_to_tile_words((f >> sh) & M32, (p0 >> sh) & M32, (p1 >> sh) & M32,
                                         (p2 >> sh) & M32, (p3 >> sh) & M32)
            for n in range(8):
                for r in range(4):
                    s = sh + 4 * n + r
                    want = 0xFF
                    for k in range(first, last + 1):
                        if (slots[k] >> s) & 1:
                            want = k
                    assert (words[n] >> (8 * r)) & 0xFF == want, (trial, s)


def test_byte_transpose4():
    rnd = random.Random(3)
    for _ in range(200):
        w = [rnd.getrandbits(32) for _ in range(4)]
        t = byte_transpose4(*w)
        for g in range(4):
            for r in range(4):
                assert (t[g] >> (8 * r)) & 0xFF == (w[r] >> (8 * g)) & 0xFF
