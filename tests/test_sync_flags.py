"""The readiness flags between the chain's stages (plan.cpp flag_sync,
cdef.cu cdef_wait_lf, lr.cu lr_wait_cdef): every sample a CDEF item reads
from the loop filter's output lies in a 64x64 tile whose flag the item waits
for; every sample a loop-restoration rectangle reads from CDEF's output lies
in a half superblock whose flag it waits for; and every loop-filter row it
reads outside its stripe lies in a tile that one of those half superblocks
waited for. The wait ranges below restate the kernels' formulas; the reads
are enumerated sample by sample from the kernels' staging rules."""
import random

import pytest


def cdef_waits(pw, ph, sx, sy, sc, y0, R):
    """The tiles cdef_wait_lf waits for (threads 0..47: 4 x 4 per plane)."""
    r0, r1 = max((y0 >> sy) - 2, 0), min(((y0 + R) >> sy) + 1, ph - 1)
    c0, c1 = max(((sc * 64) >> sx) - 8, 0), min(((sc * 64 + 64) >> sx) + 7, pw - 1)
    out = set()
    for dy in range(4):
        for dx in range(4):
            ty, tx = (r0 >> 6) + dy, (c0 >> 6) + dx
            if r0 <= r1 and c0 <= c1 and ty <= (r1 >> 6) and tx <= (c1 >> 6):
                out.add((ty, tx))
    return out


def cdef_reads(pw, ph, sx, sy, sc, y0, R, mi_rows, mi_cols):
    """The loop-filter samples stage_plane loads: rows -2 .. R+1 of the
    plane's part of the superblock, 8 columns either side, inside the
    mode-info area and the plane."""
    xlim, ylim = (mi_cols * 4) >> sx, (mi_rows * 4) >> sy
    px0, py0 = (sc * 64) >> sx, (y0 >> sy) - 2
    for r in range((R >> sy) + 4):
        gy = py0 + r
        if 0 <= gy < min(ylim, ph):
            for gx in range(max(px0 - 8, 0), min(px0 + (64 >> sx) + 8, xlim, pw)):
                yield gy, gx


def lr_waits(sx, sy, y0, y1, xa, xb, sbc):
    """The half superblocks lr_wait_cdef waits for (threads 0..15: 4 x 4)."""
    h0, h1 = (y0 << sy) >> 5, ((y1 << sy) + sy) >> 5
    c0, c1 = (xa << sx) >> 6, min(((xb << sx) + sx) >> 6, sbc - 1)
    return {(h0 + t // 4, c0 + t % 4) for t in range(16) if h0 + t // 4 <= h1 and c0 + t % 4 <= c1}


def check(W, H, sx, sy, half, lr_cols=64):
    mi_cols, mi_rows = 2 * ((W + 7) >> 3), 2 * ((H + 7) >> 3)
    sbr, sbc = (mi_rows + 15) // 16, (mi_cols + 15) // 16
    for p in range(3):
        psx, psy = (sx, sy) if p else (0, 0)
        pw, ph = (W + psx) >> psx, (H + psy) >> psy
        waited = {}  # half superblock -> the tiles its CDEF item waited for
        R = 32 if half else 64
        for sr in range(sbr):
            for sc in range(sbc):
                for a in ((0, 1) if half else (0,)):
                    if half and sr * 16 + a * 8 >= mi_rows:
                        continue  # the planner makes no item past the mode-info area
                    y0 = sr * 64 + a * R
                    w = cdef_waits(pw, ph, psx, psy, sc, y0, R)
                    for gy, gx in cdef_reads(pw, ph, psx, psy, sc, y0, R, mi_rows, mi_cols):
                        assert (gy // 64, gx // 64) in w, (W, H, sx, sy, half, p, sr, sc, a, gy, gx)
                    for hh in ((2 * sr + a,) if half else (2 * sr, 2 * sr + 1)):
                        waited[(hh, sc)] = w
        pex, pey = pw - 1, ph - 1
        for s in range((H + 8 + 63) // 64):
            ss = (-8 + s * 64) >> psy
            se = ss + (64 >> psy) - 1
            y0, y1 = max(ss, 0), min(se, pey)
            if y0 > y1:
                continue
            for x0 in range(0, pex + 1, lr_cols):
                w = min(lr_cols, pex + 1 - x0)
                xa, xb = max(x0 - 3, 0), min(x0 + w + 2, pex)
                got = lr_waits(psx, psy, y0, y1, xa, xb, sbc)
                # the stripe's rows come from CDEF's output
                for y in range(y0, y1 + 1):
                    for x in range(xa, xb + 1):
                        key = ((y << psy) >> 5, (x << psx) >> 6)
                        assert key in got and key in waited, (W, H, sx, sy, p, s, x0, y, x)
                # the 2 rows either side of the stripe from the loop filter's
                lf = set().union(*(waited[k] for k in got))
                for y in list(range(ss - 2, ss)) + list(range(se + 1, se + 3)):
                    yy = max(min(y, pey), 0)
                    if ss <= yy <= se:
                        continue
                    for x in range(xa, xb + 1):
                        assert (yy // 64, x // 64) in lf, (W, H, sx, sy, p, s, x0, yy, x)


SIZES = [(352, 288), (200, 136), (127, 65), (17, 9), (64, 64), (65, 65), (104, 66), (160, 96), (640, 360)]


@pytest.mark.parametrize("W,H", SIZES)
@pytest.mark.parametrize("sx,sy", [(1, 1), (0, 0), (1, 0)])
def test_flags_cover_every_read(W, H, sx, sy):
    for half in (True, False):
        check(W, H, sx, sy, half)


def test_flags_cover_every_read_random_shapes():
    r = random.Random(7)
    for _ in range(6):
        W, H = r.randrange(8, 400), r.randrange(8, 300)
        for sx, sy in ((1, 1), (0, 0), (1, 0)):
            check(W, H, sx, sy, r.random() < 0.5, lr_cols=r.choice((32, 64)))
