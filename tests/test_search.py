"""The oracle's encoder filter searches (encoder/cdef.rs:52-251,
encoder/mod.rs:1457-1506) against independent numpy restatements of their
parts: the unfiltered candidate's block errors (skip flags, the frame crop,
the 64x64 blocks that code an index), the greedy choice recomputed in Python
from the error table, and the loop-filter search's per-scale plane errors;
and the loop-restoration search's Wiener fit (encoder/lr.rs:212-328) against
a pure-Python restatement, window construction included. CPU only."""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O

CASES = {
    "256x144_10b": dict(width=256, height=144, bit_depth=10, seed=3),
    "200x120_8b": dict(width=200, height=120, bit_depth=8, sample_bytes=1, seed=4),
    "136x72_12b_444": dict(width=136, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=5),
    "160x96_10b_422": dict(width=160, height=96, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=6),
    "120x80_10b_mono": dict(width=120, height=80, bit_depth=10, mono=1, seed=7),
}


def host_map(ptr, n, dtype):
    return np.frombuffer((C.c_uint8 * (n * np.dtype(dtype).itemsize)).from_address(ptr), dtype=dtype, count=n)


def skip_map(sf):
    f = sf.f
    mi = host_map(f.maps.mi, f.mi_count * 8, np.uint8).reshape(-1, 8)
    return (mi[:, 3] & 0x80 != 0).reshape(-1, f.maps.mi_stride)


def coding_blocks(sf):
    info, maps = sf.f.info, sf.f.maps
    fbr, fbc = (info.mi_rows + 15) // 16, (info.mi_cols + 15) // 16
    idx = host_map(maps.cdef_idx, fbr * maps.cdef_stride, np.int8).reshape(fbr, maps.cdef_stride)
    return idx, fbr, fbc


def unfiltered_block_sse(sf, cur, src):
    """Per 64x64 block: luma and chroma squared error of the unfiltered
    reconstruction over the non-skip 8x8 blocks, inside the frame."""
    info = sf.f.info
    skip = skip_map(sf)
    idx, fbr, fbc = coding_blocks(sf)
    out = np.zeros((fbr * fbc, 2), np.uint64)
    for fr in range(fbr):
        for fc in range(fbc):
            if idx[fr, fc] < 0:
                continue
            ys = uvs = 0
            for r in range(fr * 16, min(fr * 16 + 16, info.mi_rows), 2):
                for c in range(fc * 16, min(fc * 16 + 16, info.mi_cols), 2):
                    if skip[r, c] and skip[r + 1, c] and skip[r, c + 1] and skip[r + 1, c + 1]:
                        continue
                    for p in range(info.num_planes):
                        sx = info.subsampling_x if p else 0
                        sy = info.subsampling_y if p else 0
                        fw, fh = (info.frame_width + sx) >> sx, (info.frame_height + sy) >> sy
                        x0, y0 = (c * 4) >> sx, (r * 4) >> sy
                        x1, y1 = min(x0 + (8 >> sx), fw), min(y0 + (8 >> sy), fh)
                        if x1 <= x0 or y1 <= y0:
                            continue
                        d = cur.arrays[p][y0:y1, x0:x1].astype(np.int64) - src.arrays[p][y0:y1, x0:x1]
                        e = int((d * d).sum())
                        if p == 0:
                            ys += e
                        else:
                            uvs += e
            out[fr * fbc + fc] = (ys, uvs)
    return out


def greedy(sse, coded, ny, nuv, lam):
    """encoder/cdef.rs:195-240 in plain Python (float totals in block order)."""
    blocks = [b for b in range(len(sse)) if coded[b]]
    ysse = [[int(sse[b, k]) for k in range(ny)] for b in blocks]
    uvsse = [[int(sse[b, ny + k]) for k in range(nuv)] for b in blocks]
    nb = len(blocks)

    def best_for(s):
        total, pick = 0.0, []
        for b in range(nb):
            v = [ysse[b][y] + uvsse[b][u] for y, u in s]
            m = min(v)
            pick.append(v.index(m))
            total += float(m)
        return total, pick

    best, chosen = (float("inf"), None, None), []
    for bits in range(4):
        while len(chosen) < 1 << bits:
            add = (float("inf"), (0, 0))
            for y in range(ny):
                for u in range(nuv):
                    if (y, u) in chosen:
                        continue
                    t, _ = best_for(chosen + [(y, u)])
                    if t < add[0]:
                        add = (t, (y, u))
            chosen.append(add[1])
        t, pick = best_for(chosen)
        cost = t + lam * float(bits) * float(nb)
        if cost < best[0]:
            best = (cost, list(chosen), pick)
    return best[1], best[2], [blocks[i] for i in range(nb)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_unfiltered_candidate_is_plain_block_error(name):
    sf = A.SynthHandle(**CASES[name])
    cur, src = O.search_inputs(sf, 11)
    _, _, sse = O.cdef_search(sf, cur, src, 100, 100.0, False)
    ny, _ = A.CDEF_SEARCH_N[False]
    want = unfiltered_block_sse(sf, cur, src)
    assert np.array_equal(sse[:, 0], want[:, 0]), "luma (0, 0) candidate"
    if sf.f.info.num_planes > 1:
        assert np.array_equal(sse[:, ny], want[:, 1]), "chroma (0, 0) candidate"
    else:
        assert not sse[:, ny:].any()


@pytest.mark.parametrize("thorough", [False, True])
@pytest.mark.parametrize("lam", [0.0, 60.0, 3000.0])
def test_greedy_matches_python_restatement(thorough, lam):
    sf = A.SynthHandle(**CASES["256x144_10b"])
    cur, src = O.search_inputs(sf, 12)
    res, table, sse = O.cdef_search(sf, cur, src, 140, lam, thorough)
    ny, nuv = A.CDEF_SEARCH_N[thorough]
    idx, fbr, fbc = coding_blocks(sf)
    coded = [idx[b // fbc, b % fbc] >= 0 for b in range(fbr * fbc)]
    chosen, pick, blocks = greedy(sse, coded, ny, nuv, lam)
    assert res.bits == len(chosen).bit_length() - 1
    ylist = [(p, s) for p in ([0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15] if thorough else [0, 1, 2, 4, 6, 9, 12])
             for s in range(4)]
    uvlist = [(p, s) for p in ([0, 1, 2, 3, 4, 6, 8, 11] if thorough else [0, 1, 2, 4, 7]) for s in range(3)]
    assert res.pairs() == [ylist[y] + uvlist[u] for y, u in chosen]
    assert res.damping_minus_3 == min(140 >> 6, 3)
    t2 = table.reshape(fbr, -1)
    for b, pk in zip(blocks, pick):
        assert t2[b // fbc, b % fbc] == pk
    assert np.array_equal(t2[idx < 0], idx[idx < 0])


def test_identity_reconstruction_chooses_no_filtering():
    sf = A.SynthHandle(**CASES["256x144_10b"])
    _, src = O.search_inputs(sf, 13)
    res, table, sse = O.cdef_search(sf, src, src, 200, 10.0, False)
    assert res.bits == 0 and res.pairs() == [(0, 0, 0, 0)]
    assert not sse[:, 0].any()
    idx, _, _ = coding_blocks(sf)
    t2 = table.reshape(idx.shape)
    assert np.array_equal(t2[idx >= 0], np.zeros((idx >= 0).sum(), np.int8))


def test_no_coding_block_is_cdef_off():
    sf = A.SynthHandle(**CASES["200x120_8b"])
    idx, fbr, _ = coding_blocks(sf)
    idx[:] = -1  # the synthetic frame's own table, in place
    cur, src = O.search_inputs(sf, 14)
    res, table, sse = O.cdef_search(sf, cur, src, 255, 1.0, True)
    assert (res.damping_minus_3, res.bits, res.pairs()) == (0, 0, [(0, 0, 0, 0)])
    assert (table == -1).all() and not sse.any()


@pytest.mark.parametrize("name", sorted(CASES))
def test_lf_search_scale_zero_is_plain_plane_error(name):
    sf = A.SynthHandle(**CASES[name])
    cur, src = O.search_inputs(sf, 15)
    levels, sse = O.lf_search(sf, cur, src)
    info = sf.f.info
    for p in range(info.num_planes):
        sx = info.subsampling_x if p else 0
        sy = info.subsampling_y if p else 0
        w, h = (info.frame_width + sx) >> sx, (info.frame_height + sy) >> sy
        d = cur.arrays[p][:h, :w].astype(np.int64) - src.arrays[p][:h, :w]
        assert int(sse[0, p]) == int((d * d).sum())
    assert not sse[:, info.num_planes:].any()
    # each plane's level is the first scale with its least error
    start = list(sf.f.params.loop_filter_level)
    lv = [[min(int(np.floor(l * s + 0.5)), 63) for l in start] for s in (0.0, 0.5, 0.75, 1.0, 1.25, 1.5)]
    best = [int(np.argmin(sse[:, p])) for p in range(3)]
    want = [lv[best[0]][0], lv[best[0]][0], lv[best[1]][2], lv[best[2]][3]]
    if info.num_planes == 1:
        want[2] = want[3] = 0
    assert levels == ([0, 0, 0, 0] if want[0] == 0 else want)


def test_searches_thread_count_invariant():
    sf = A.SynthHandle(**CASES["160x96_10b_422"])
    cur, src = O.search_inputs(sf, 16)
    a = O.cdef_search(sf, cur, src, 90, 20.0, True, threads=1)
    b = O.cdef_search(sf, cur, src, 90, 20.0, True, threads=0)
    assert a[0].pairs() == b[0].pairs() and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert O.lf_search(sf, cur, src, threads=1)[0] == O.lf_search(sf, cur, src, threads=0)[0]


# ---------------------------------------------------------------------------
# Loop-restoration search (encoder/lr.rs)
# ---------------------------------------------------------------------------
WIENER_MIN, WIENER_MAX = (-5, -23, -17), (10, 8, 46)


def py_solve(m, v):
    """encoder/lr.rs:212-233 in Python floats (f64, same operation order)."""
    n = len(v)
    m = [list(r) for r in m]
    v = list(v)
    for i in range(n):
        piv = i
        for a in range(i + 1, n):
            if abs(m[a][i]) >= abs(m[piv][i]):
                piv = a
        m[i], m[piv] = m[piv], m[i]
        v[i], v[piv] = v[piv], v[i]
        if abs(m[i][i]) < 1e-9:
            return [0.0] * n
        for r in range(n):
            if r != i:
                f = m[r][i] / m[i][i]
                for c in range(i, n):
                    m[r][c] -= f * m[i][c]
                v[r] -= f * v[i]
    return [v[i] / m[i][i] for i in range(n)]


def rust_round(x):
    return int(np.floor(x + 0.5)) if x >= 0 else -int(np.floor(-x + 0.5))


def py_fit_wiener(plane, rects, src, step):
    """encoder/lr.rs:235-328 on pre-built windows: rects = [(win, y0, h)]."""
    first = 0 if plane == 0 else 1
    hc, vc = [0.0] * 3, [0.0] * 3
    for it in range(3):
        vertical = it % 2 == 0
        m = [[0.0] * 3 for _ in range(3)]
        v = [0.0] * 3
        for win, y0, h, x0, w in rects:
            at = lambda r, c: float(win[r][c])  # noqa: E731
            for i in range(0, h, step):
                for j in range(0, w, step):
                    line = []
                    for t in range(7):
                        r, c = (i + t, j + 3) if vertical else (i + 3, j + t)
                        other = hc if vertical else vc
                        center = at(r, c)
                        s = center
                        for k in range(3):
                            d = 3 - k
                            a, b = (at(r, c - d), at(r, c + d)) if vertical else (at(r - d, c), at(r + d, c))
                            s += other[k] * (a + b - 2.0 * center)
                        line.append(s)
                    target = float(src[y0 + i][x0 + j]) - line[3]
                    d = [line[k] + line[6 - k] - 2.0 * line[3] for k in range(3)]
                    for a in range(first, 3):
                        for b in range(first, 3):
                            m[a][b] += d[a] * d[b]
                        v[a] += d[a] * target
        if first == 0:
            sol = py_solve(m, v)
        else:
            s2 = py_solve([[m[1][1], m[1][2]], [m[2][1], m[2][2]]], [v[1], v[2]])
            sol = [0.0, s2[0], s2[1]]
        if vertical:
            vc = sol
        else:
            hc = sol
    q = lambda c: tuple(0 if k < first else min(max(rust_round(c[k] * 128.0), WIENER_MIN[k]), WIENER_MAX[k])  # noqa
                        for k in range(3))
    return (q(vc), q(hc))


def py_lr_rects(sf, plane, cur, cdef, ur, uc):
    """The unit's stripes as (window, y0, h, x0, w) (postfilter.rs:640-675, 765-777)."""
    info, p = sf.f.info, sf.f.params
    sx = info.subsampling_x if plane else 0
    sy = info.subsampling_y if plane else 0
    pex = ((info.upscaled_width + sx) >> sx) - 1
    pey = ((info.frame_height + sy) >> sy) - 1
    us = p.loop_restoration_size[plane]
    x0 = uc * us
    x1 = pex if uc + 1 == p.lr_unit_cols[plane] else min((uc + 1) * us - 1, pex)
    w = x1 - x0 + 1
    rects = []
    for s in range((info.frame_height + 8 + 63) // 64):
        ss = (-8 + s * 64) >> sy
        se = ss + (64 >> sy) - 1
        y0, y1 = max(ss, 0), min(se, pey)
        if y0 > y1:
            continue
        luma_row = s * 64 - 8 if s * 64 >= 8 else 0
        if min(p.lr_unit_rows[plane] - 1, ((luma_row + 8) >> sy) // us) != ur:
            continue
        h = y1 - y0 + 1
        win = [[0] * (w + 6) for _ in range(h + 6)]
        for r in range(h + 6):
            y = min(max(y0 + r - 3, 0), pey)
            for c in range(w + 6):
                xx = max(min(x0 + c - 3, pex), 0)
                if y < ss:
                    win[r][c] = int(cur.arrays[plane][max(ss - 2, y)][xx])
                elif y > se:
                    win[r][c] = int(cur.arrays[plane][min(se + 2, y)][xx])
                else:
                    win[r][c] = int(cdef.arrays[plane][y][xx])
        rects.append((win, y0, h, x0, w))
    return rects


@pytest.mark.parametrize("effort", [0, 1])
def test_lr_wiener_fit_matches_python_restatement(effort):
    """lambda -1e12 makes every unit take its Wiener filter, exposing each
    fitted coefficient set."""
    sf = A.SynthHandle(width=72, height=40, bit_depth=10, seed=8, enable_lr=1, lr_unit_shift=0, lr_uv_shift=1)
    cur, cdef, src = O.lr_search_inputs(sf, 21)
    ft, units = O.lr_search(sf, cur, cdef, src, -1e12, effort)
    p = sf.f.params
    assert ft == [1, 1, 1]
    for plane in range(3):
        for ur in range(p.lr_unit_rows[plane]):
            for uc in range(p.lr_unit_cols[plane]):
                rects = py_lr_rects(sf, plane, cur, cdef, ur, uc)
                want = py_fit_wiener(plane, rects, src.arrays[plane], 2 if effort == 0 else 1)
                got = units[plane][ur * p.lr_unit_cols[plane] + uc]
                assert got[0] == 1 and got[1] == want, (plane, ur, uc)


def test_lr_search_identity_chooses_none():
    sf = A.SynthHandle(width=256, height=144, bit_depth=10, seed=9, enable_lr=1)
    cur, cdef, src = O.lr_search_inputs(sf, 22)
    ft, units = O.lr_search(sf, cur, src, src, 5.0, 2)
    assert ft == [0, 0, 0] and all(u[0] == 0 for pl in units for u in pl)


def test_lr_search_thread_count_invariant():
    sf = A.SynthHandle(width=200, height=120, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=10, enable_lr=1)
    cur, cdef, src = O.lr_search_inputs(sf, 23)
    assert O.lr_search(sf, cur, cdef, src, 50.0, 1, threads=1) == O.lr_search(sf, cur, cdef, src, 50.0, 1, threads=0)
