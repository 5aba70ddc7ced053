"""The oracle against a second CPU restatement written from the AV1
specification's pseudo-code (oracle/spec_check.py), bit for bit, on small
synthetic frames: CDEF (7.15) and the film-grain output process (7.18.3)
stage by stage, and the whole chain (7.14 loop filter, 7.15 CDEF, 7.16
upscaling, 7.17 loop restoration, 7.18 output).

The oracle and the CUDA kernels were both written from the reference's Rust
code; a misreading of it that they share would pass every GPU parity test.
This restatement shares no code with either, so such a misreading shows up
here. The film-grain cases also vary the parameters the synthetic
generator holds fixed: auto-regression lag 0-3, overlap off, the restricted
range clip (with the identity matrix's chroma limit), chroma scaled from
luma, and luma without grain.
"""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O
import spec_check as S
from conftest import cuda_available

CDEF_CASES = {
    "352x288_8bit_u8": dict(width=352, height=288, bit_depth=8, sample_bytes=1, content=1, seed=1, frame_index=2),
    "10bit_420": dict(width=200, height=136, bit_depth=10, seed=2),
    "12bit_444": dict(width=136, height=96, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=4),
    "10bit_422": dict(width=152, height=88, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=5),
    "8bit_mono": dict(width=120, height=72, bit_depth=8, sample_bytes=1, mono=1, seed=6),
    "big_blocks": dict(width=192, height=128, bit_depth=10, min_block_log2=5, skip_pct=10, seed=17),
    "odd_127x65": dict(width=127, height=65, bit_depth=10, seed=25),
    "tiny_17x9": dict(width=17, height=9, bit_depth=8, sample_bytes=1, seed=24),
}


def _maps(sf):
    f = sf.f
    info, maps = f.info, f.maps
    mi = np.frombuffer((C.c_uint8 * (f.mi_count * 8)).from_address(maps.mi), np.uint8)
    mi = mi.reshape(-1, maps.mi_stride, 8)
    skip = (mi[: info.mi_rows, : info.mi_cols, 3] & 0x80) != 0
    idx = np.frombuffer((C.c_int8 * f.cdef_count).from_address(maps.cdef_idx), np.int8).reshape(-1, maps.cdef_stride)
    return skip, idx


@pytest.mark.parametrize("name", sorted(CDEF_CASES))
def test_cdef_matches_specification(name):
    sf = A.SynthHandle(**CDEF_CASES[name])
    info, p = sf.f.info, sf.f.params
    assert p.cdef_enabled
    cur = O.HostPlanes.like_synth(sf)
    out = O.HostPlanes.zeros_like(cur)
    assert O.lib().oracle_cdef(C.byref(info), C.byref(p), C.byref(sf.f.maps), cur.c, out.c, 1) == 0
    skip, idx = _maps(sf)
    fr = dict(bit_depth=info.bit_depth, ss_x=info.subsampling_x, ss_y=info.subsampling_y, mi_rows=info.mi_rows,
              mi_cols=info.mi_cols, num_planes=info.num_planes)
    strengths = dict(damping=p.cdef_damping, y_pri=list(p.cdef_y_pri_strength), y_sec=list(p.cdef_y_sec_strength),
                     uv_pri=list(p.cdef_uv_pri_strength), uv_sec=list(p.cdef_uv_sec_strength))
    want = S.cdef_frame([a.astype(np.int64) for a in cur.arrays], fr, skip, idx, strengths)
    filtered = 0
    for pl in range(info.num_planes):
        sx = info.subsampling_x if pl else 0
        sy = info.subsampling_y if pl else 0
        h, w = (info.mi_rows * 4) >> sy, (info.mi_cols * 4) >> sx
        got = out.arrays[pl][:h, :w].astype(np.int64)
        bad = np.argwhere(got != want[pl][:h, :w])
        assert not len(bad), f"{name} plane {pl}: {len(bad)} samples differ, first at {tuple(bad[0])}"
        filtered += int(np.count_nonzero(want[pl][:h, :w] != cur.arrays[pl][:h, :w]))
    assert filtered > 0, "the case filtered nothing"


GRAIN_BASE = {
    "10bit_420": dict(width=200, height=136, bit_depth=10, enable_grain=1, seed=10, frame_index=3),
    "8bit_u8_420": dict(width=150, height=98, bit_depth=8, sample_bytes=1, enable_grain=1, seed=11),
    "12bit_444": dict(width=120, height=70, bit_depth=12, subsampling_x=0, subsampling_y=0, enable_grain=1, seed=9,
                      frame_index=7),
    "10bit_422": dict(width=130, height=70, bit_depth=10, subsampling_x=1, subsampling_y=0, enable_grain=1, seed=12),
    # frame_index 0 would give grain_seed 0, which leaves the luma generator at 0 (no luma grain)
    "8bit_mono": dict(width=90, height=50, bit_depth=8, sample_bytes=1, mono=1, enable_grain=1, seed=13, frame_index=5),
    "odd_127x65": dict(width=127, height=65, bit_depth=10, enable_grain=1, seed=25),
}


def _vary(g, how):
    """Parameter changes the generator does not make (all keep the
    format's rules: increasing points, no chroma points with chroma scaled
    from luma)."""
    if how.startswith("lag"):
        g.ar_coeff_lag = int(how[3:])
    elif how == "no_overlap":
        g.overlap_flag = 0
    elif how == "restricted":
        g.clip_to_restricted_range = 1
    elif how == "csfl":
        g.chroma_scaling_from_luma = 1
        g.num_cb_points = 0
        g.num_cr_points = 0
    elif how == "no_luma":
        g.num_y_points = 0


GRAIN_CASES = [(b, v) for b in sorted(GRAIN_BASE) for v in ("as_made",)] + \
    [("10bit_420", v) for v in ("lag0", "lag1", "lag2", "no_overlap", "restricted", "csfl", "no_luma")] + \
    [("12bit_444", v) for v in ("lag1", "csfl", "restricted")] + \
    [("10bit_422", v) for v in ("no_overlap", "no_luma")] + [("8bit_mono", "lag2")]


@pytest.mark.parametrize("base,how", GRAIN_CASES, ids=[f"{b}-{v}" for b, v in GRAIN_CASES])
def test_grain_output_matches_specification(base, how):
    sf = A.SynthHandle(**GRAIN_BASE[base])
    info, p = sf.f.info, A.Params.from_buffer_copy(sf.f.params)
    _vary(p.film_grain, how)
    if how == "restricted" and info.num_planes == 3:
        info = A.FrameInfo.from_buffer_copy(info)
        info.matrix_coefficients = 0  # MC_IDENTITY: chroma clipped to the luma range
    assert p.film_grain.apply
    ref = O.HostPlanes.like_synth(sf)
    got = np.zeros(A.frame_bytes(info), np.uint8)
    assert O.lib().oracle_output(C.byref(info), C.byref(p), ref.c, got.ctypes.data) == 0
    want = S.output_frame(info, p, ref.arrays)
    assert got.shape == want.shape
    bad = np.flatnonzero(got != want)
    assert not len(bad), f"{base} {how}: {len(bad)} bytes differ, first at {bad[0]}"
    # the grain changed the frame
    plain = A.FrameInfo.from_buffer_copy(info)
    q = A.Params.from_buffer_copy(p)
    q.film_grain.apply = 0
    assert not np.array_equal(want, S.output_frame(plain, q, ref.arrays))


def test_specification_random_numbers():
    """7.18.3.2 from a seed: the first values of the 16-bit generator
    stepped by hand."""
    r = S.Random(1)
    # r = 1: bit = 1 ^ 0 ^ 0 ^ 0 = 1 -> r = 0x8000; 11 bits: 0x8000 >> 5 = 1024
    assert r.get(11) == 1024
    # r = 0x8000: bit = 0 -> r = 0x4000 -> 512
    assert r.get(11) == 512


CHAIN_CASES = {
    "8bit_u8_420": dict(width=160, height=96, bit_depth=8, sample_bytes=1, content=1, seed=1, frame_index=2),
    "10bit_420_seg_dlf": dict(width=136, height=104, bit_depth=10, seed=3, segmentation=1, delta_lf=2),
    "10bit_420_dlf1": dict(width=120, height=72, bit_depth=10, seed=33, delta_lf=1, segmentation=1),
    "12bit_444": dict(width=96, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=4),
    "10bit_422": dict(width=104, height=66, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=5),
    "8bit_mono": dict(width=96, height=64, bit_depth=8, sample_bytes=1, mono=1, seed=6),
    "superres_d9": dict(width=144, height=80, bit_depth=10, superres_denom=9, seed=7),
    "superres_d16_grain": dict(width=128, height=70, bit_depth=10, superres_denom=16, enable_grain=1, seed=8,
                               frame_index=4),
    "lr_unit128": dict(width=200, height=140, bit_depth=10, lr_unit_shift=1, seed=14),
    "big_blocks": dict(width=128, height=128, bit_depth=10, min_block_log2=5, skip_pct=10, seed=17),
    "odd_67x45_grain": dict(width=67, height=45, bit_depth=10, enable_grain=1, seed=25, frame_index=1),
    "12bit_422_sr11_grain": dict(width=112, height=64, bit_depth=12, subsampling_x=1, subsampling_y=0,
                                 superres_denom=11, enable_grain=1, seed=41, frame_index=6),
    "8bit_u8_444_grain": dict(width=96, height=64, bit_depth=8, sample_bytes=1, subsampling_x=0, subsampling_y=0,
                              enable_grain=1, seed=42, frame_index=2),
    "lr_unit256_uv_half": dict(width=180, height=104, bit_depth=10, lr_unit_shift=2, lr_uv_shift=1, seed=43),
    "no_cdef": dict(width=120, height=72, bit_depth=10, enable_cdef=0, seed=44),
    "no_lf": dict(width=120, height=72, bit_depth=10, enable_lf=0, seed=45),
    "8bit_u16_samples": dict(width=104, height=64, bit_depth=8, sample_bytes=2, seed=46),
}


@pytest.mark.parametrize("name", sorted(CHAIN_CASES))
def test_chain_matches_specification(name):
    """The whole chain (7.14 loop filter, 7.15 CDEF, 7.16 upscaling, 7.17
    loop restoration, 7.18 output with film grain) restated from the
    specification, against the oracle's chain: the reference frame and the
    packed output frame, bit for bit."""
    sf = A.SynthHandle(**CHAIN_CASES[name])
    ref_cpu, fb_cpu = O.chain(sf, threads=1)
    inp = O.HostPlanes.like_synth(sf)
    vis, fb = S.chain(sf, inp.arrays)
    for p, (g, c) in enumerate(zip(vis, ref_cpu.arrays)):
        bad = np.argwhere(g != c)
        assert not len(bad), f"{name} plane {p}: {len(bad)} samples differ, first at {tuple(bad[0])}"
    assert np.array_equal(fb, fb_cpu), f"{name}: packed frame differs"


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("name", ["10bit_420_seg_dlf", "superres_d16_grain", "12bit_444", "8bit_u8_420"])
def test_gpu_chain_matches_specification(name):
    """The CUDA chain through the C ABI against the specification's
    restatement directly (no oracle in between)."""
    import gpu_util as G
    sf = A.SynthHandle(**CHAIN_CASES[name])
    vis, fb = S.chain(sf, O.HostPlanes.like_synth(sf).arrays)
    ctx = G.Ctx()
    try:
        ref_gpu, fb_gpu = G.gpu_chain(ctx, G.DevFrame(sf))
    finally:
        ctx.close()
    for p, (g, c) in enumerate(zip(ref_gpu, vis)):
        assert np.array_equal(g, c), f"{name} plane {p}"
    assert np.array_equal(fb_gpu, fb), f"{name}: packed frame"
