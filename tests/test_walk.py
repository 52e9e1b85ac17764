"""The batched stencil's arithmetic walk (ColumnWalk / walk_site in lym_batch.cuh): a numpy
restatement of its integer steps, checked against the traversal of the order tables
(order_table_kernel) and the neighbour half-sites of the site layout (neighbour_h,
MPILattice/LocalLayout.h:34-110 through the oracle's geometry), for every traversal column
the autotuner times; and the exactness of its multiply-high divisions."""
import numpy as np
import pytest

LATTICES = [(8, 8, 8, 8), (4, 8, 12, 16), (10, 6, 14, 4), (24, 24, 24, 48)]


def magic(d):
    return 0 if d == 1 else ((1 << 32) + d - 1) // d


def wdiv(n, m):
    return n if m == 0 else (n * np.uint64(m)) >> np.uint64(32)


def walk(L, by, bz, p, w):
    if by == 0:
        by, bz = L[1], L[2]
    lth, nzb = L[3] // 2, L[2] // bz
    u = w.astype(np.uint64)
    parts = []
    for d in (lth, bz, by, L[0], nzb):
        q = wdiv(u, magic(d))
        parts.append((u - q * np.uint64(d)).astype(np.int64))
        u = q
    th, zi, yi, x, zb = parts
    yb = u.astype(np.int64)
    y, z = yb * by + yi, zb * bz + zi
    t = 2 * th + ((p + x + y + z) & 1)
    sx, sy, sz = lth * L[2] * L[1], lth * L[2], lth
    h = th + sz * z + sy * y + sx * x
    nf = [h + np.where(c + 1 == L[k], -c * s, s) for k, (c, s) in enumerate(((x, sx), (y, sy), (z, sz)))]
    nb = [h + np.where(c == 0, (L[k] - 1) * s, -s) for k, (c, s) in enumerate(((x, sx), (y, sy), (z, sz)))]
    base = h - th
    nf.append(base + (np.where(t + 1 == L[3], 0, t + 1) >> 1))
    nb.append(base + (np.where(t == 0, L[3] - 1, t - 1) >> 1))
    return h, nf, nb


def order(L, by, bz, w):
    if by == 0:
        return w
    lth, u = L[3] // 2, w.copy()
    th = u % lth; u //= lth
    zi = u % bz; u //= bz
    yi = u % by; u //= by
    x = u % L[0]; u //= L[0]
    nzb = L[2] // bz
    zb, yb = u % nzb, u // nzb
    return th + lth * ((zb * bz + zi) + L[2] * ((yb * by + yi) + L[1] * x))


def neighbours(L, p, h):
    s0 = 2 * h
    t0, r = s0 % L[3], s0 // L[3]
    z = r % L[2]; r //= L[2]
    y, x = r % L[1], r // L[1]
    c = [x, y, z, t0 + ((p + x + y + z) & 1)]
    nf, nb = [], []
    for mu in range(4):
        for d, out in ((1, nf), (-1, nb)):
            n = list(c)
            v = n[mu] + d
            n[mu] = np.where(v == L[mu], 0, np.where(v < 0, L[mu] - 1, v))
            out.append((L[3] * (L[2] * (L[1] * n[0] + n[1]) + n[2]) + n[3]) >> 1)
    return nf, nb


def columns(L):
    out = [(0, 0)] + [(by, L[2]) for by in (2, 4, 8, 12)] + [(4, 4), (8, 8)]
    return [(a, b) for a, b in out if a == 0 or (L[1] % a == 0 and L[2] % b == 0 and (a, b) != (L[1], L[2]))]


@pytest.mark.parametrize("L", LATTICES)
def test_walk_matches_tables(L):
    Vh = int(np.prod(L)) // 2
    w = np.arange(Vh, dtype=np.int64)
    for by, bz in columns(L):
        for p in (0, 1):
            h, nf, nb = walk(L, by, bz, p, w)
            assert np.array_equal(h, order(L, by, bz, w))
            assert len(np.unique(h)) == Vh
            rf, rb = neighbours(L, p, h)
            for mu in range(4):
                assert np.array_equal(nf[mu], rf[mu]) and np.array_equal(nb[mu], rb[mu]), (by, bz, p, mu)


def test_multiply_high_division_exact():
    """floor(n / d) = umulhi(n, ceil(2^32 / d)) for d <= 256 and n < 2^24 (the walk's range):
    the error term n (m d - 2^32) / 2^32 stays below 1 / d; checked on the bottom and top of
    the range."""
    ns = np.concatenate([np.arange(1 << 18, dtype=np.uint64),
                         np.arange((1 << 24) - (1 << 18), 1 << 24, dtype=np.uint64)])
    for d in range(2, 257):
        assert np.array_equal(wdiv(ns, magic(d)), ns // np.uint64(d)), d
