"""The CPU oracle against the reference's own known-answer tests for this path
and against the committed regression fixtures (CPU only).

Pins:
- lf.rs:309-353 (`lanes_match_the_process`): the four-lane loop-filter kernel
  equals the one-sample process of 7.14.6 on 20 000 random edges from the
  reference's xorshift seed 0x0bad_5eed_1234_5678.
- cdef.rs:250-311 (`simd_matches_scalar`): the case generator with seed
  0x2545_f491_4f6c_dd1d yields windows whose scalar filter is deterministic and
  respects the filter's clamp (result within the window's available min/max).
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

import av1pf as A
import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

LF_SEED = 0x0BAD5EED12345678
CDEF_SEED = 0x2545F4914F6CDD1D


def lf_cases(n, seed=LF_SEED):
    edges = np.zeros((n, 56), np.int32)
    prm = (A.LfEdgeParams * n)()
    O.lib().oracle_lf_kat_cases(seed, n, edges.ctypes.data, C.addressof(prm))
    return edges, prm


def cdef_cases(n, seed=CDEF_SEED):
    win = np.zeros((3 * n, 144), np.int32)
    taps = (A.CdefTaps * (3 * n))()
    O.lib().oracle_cdef_kat_cases(seed, n, win.ctypes.data, C.addressof(taps))
    return win, taps


def test_lf_lanes_match_one_sample_process():
    n = 20000
    edges, prm = lf_cases(n)
    lanes = edges.copy()
    one = edges.copy()
    O.lib().oracle_lf_filter_lanes(lanes.ctypes.data, C.addressof(prm), n)
    O.lib().oracle_lf_reference(one.ctypes.data, C.addressof(prm), n)
    assert np.array_equal(lanes, one)
    # the cases exercise the filters (not all masked off)
    assert (lanes != edges).any(axis=1).sum() > n // 4


def test_lf_case_generator_matches_reference_distribution():
    edges, prm = lf_cases(300)
    for c in range(300):
        p = prm[c]
        assert p.bit_depth == [8, 10, 12][c % 3]
        assert (p.chroma != 0) == (c % 5 == 0)
        assert 1 <= p.limit <= 9 and 0 <= p.blimit < 130 and 0 <= p.thresh < 4
        assert p.filter_size in ((4, 6, 8) if p.chroma else (4, 6, 8, 16))
        assert edges[c].max() < (1 << p.bit_depth) and edges[c].min() >= 0


def test_cdef_scalar_cases_clamped_and_deterministic():
    n = 4000
    win, taps = cdef_cases(n)
    res = np.zeros((3 * n, 64), np.uint16)
    O.lib().oracle_cdef_filter(win.ctypes.data, C.addressof(taps), res.ctypes.data, 3 * n)
    res2 = np.zeros_like(res)
    O.lib().oracle_cdef_filter(win.ctypes.data, C.addressof(taps), res2.ctypes.data, 3 * n)
    assert np.array_equal(res, res2)
    na = np.iinfo(np.int32).min
    changed = 0
    for e in range(0, 3 * n, 37):
        t = taps[e]
        w = win[e].reshape(12, 12)
        for i in range(t.h):
            for j in range(t.w):
                x = w[i + 2, j + 2]
                v = int(res[e, i * t.w + j])
                blk = w[i:i + 5, j:j + 5]
                avail = blk[blk != na]
                assert avail.min() <= v <= avail.max()
                changed += v != x
    assert changed > 0


def test_oracle_threads_match_serial():
    s = A.SynthHandle(width=200, height=120, bit_depth=10, seed=3, segmentation=1, delta_lf=2)
    r1, f1 = O.chain(s, threads=1)
    r8, f8 = O.chain(s, threads=8)
    assert np.array_equal(f1, f8)
    for a, b in zip(r1.arrays, r8.arrays):
        assert np.array_equal(a, b)


def _digest(ref, fb):
    h = hashlib.sha256()
    for a in ref.arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(fb.tobytes())
    return h.hexdigest()


def test_golden_fixtures():
    """Oracle outputs on the committed synthetic cases are unchanged (the
    fixtures come from tests/golden/make_golden.py)."""
    import make_golden
    with open(os.path.join(GOLDEN, "chain_digests.json")) as fh:
        want = json.load(fh)
    assert set(want) == set(make_golden.CASES)
    for name, kw in make_golden.CASES.items():
        s = A.SynthHandle(**kw)
        ref, fb = O.chain(s, threads=0)
        assert _digest(ref, fb) == want[name], name


def test_golden_small_frame_arrays():
    """The smallest fixture is stored in full: the oracle reproduces it."""
    import make_golden
    z = np.load(os.path.join(GOLDEN, "small_8bit.npz"))
    s = A.SynthHandle(**make_golden.CASES["small_8bit"])
    inp = O.HostPlanes.like_synth(s)
    for p in range(3):
        assert np.array_equal(inp.arrays[p], z[f"in{p}"])
    ref, fb = O.chain(s, threads=1)
    assert np.array_equal(fb, z["frame"])
    for p in range(3):
        assert np.array_equal(ref.arrays[p], z[f"ref{p}"])


@pytest.mark.parametrize("bad", ["bit_depth", "mi_cols", "sample_bytes"])
def test_oracle_rejects_bad_descriptors(bad):
    s = A.SynthHandle(width=64, height=64, bit_depth=8, sample_bytes=1)
    info = A.FrameInfo.from_buffer_copy(s.f.info)
    setattr(info, bad, {"bit_depth": 9, "mi_cols": 3, "sample_bytes": 3}[bad])
    inp = O.HostPlanes.like_synth(s)
    ref = O.HostPlanes.visible(s.f.info)
    rc = O.lib().oracle_chain(C.byref(info), C.byref(s.f.params), C.byref(s.f.maps), inp.c, ref.c, None, 1)
    assert rc == A.ERR_INVALID_INPUT
