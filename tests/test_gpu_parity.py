"""Parity of the CUDA path (through the C ABI) with the CPU oracle, bit for bit.

Mirrors the reference's own tests for the path: the loop-filter and CDEF
known-answer cases (lf.rs:309-353, cdef.rs:250-311) run through the device
DSP entry points; whole frames run through each stage and the whole chain at
8, 10 and 12 bits, 4:2:0 / 4:2:2 / 4:4:4 / monochrome, with superres, film
grain, segmentation and delta-lf, odd and tiny sizes.
"""
import ctypes as C
import json
import hashlib
import os

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G
    import torch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctx():
    c = G.Ctx()
    yield c
    c.close()


def assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, label=""):
    for p, (g, c) in enumerate(zip(ref_gpu, ref_cpu.arrays)):
        if not np.array_equal(g, c):
            bad = np.argwhere(g != c)
            y, x = bad[0]
            raise AssertionError(f"{label} plane {p}: {len(bad)} samples differ, first at (y={y}, x={x}): "
                                 f"gpu {g[y, x]} cpu {c[y, x]}")
    if fb_cpu is not None:
        assert np.array_equal(fb_gpu, fb_cpu), f"{label} packed frame differs"


# ---------------------------------------------------------------------------
# DSP known-answer tests
# ---------------------------------------------------------------------------
def test_dsp_lf_matches_oracle(ctx):
    n = 20000
    edges = np.zeros((n, 56), np.int32)
    prm = (A.LfEdgeParams * n)()
    O.lib().oracle_lf_kat_cases(0x0BAD5EED12345678, n, edges.ctypes.data, C.addressof(prm))
    want = edges.copy()
    O.lib().oracle_lf_filter_lanes(want.ctypes.data, C.addressof(prm), n)
    d_edges = torch.from_numpy(edges.copy()).cuda()
    d_prm = G.to_dev(C.addressof(prm), C.sizeof(prm))
    A.check(A.lib().av1pf_dsp_lf_filter(ctx.p, d_edges.data_ptr(), d_prm.data_ptr(), n, None))
    torch.cuda.synchronize()
    got = d_edges.cpu().numpy()
    assert np.array_equal(got, want), f"{(got != want).any(axis=1).sum()} edges differ"


def test_dsp_cdef_matches_oracle(ctx):
    n = 4000
    win = np.zeros((3 * n, 144), np.int32)
    taps = (A.CdefTaps * (3 * n))()
    O.lib().oracle_cdef_kat_cases(0x2545F4914F6CDD1D, n, win.ctypes.data, C.addressof(taps))
    want = np.zeros((3 * n, 64), np.uint16)
    O.lib().oracle_cdef_filter(win.ctypes.data, C.addressof(taps), want.ctypes.data, 3 * n)
    d_win = torch.from_numpy(win).cuda()
    d_taps = G.to_dev(C.addressof(taps), C.sizeof(taps))
    d_res = torch.zeros((3 * n, 64), dtype=torch.int16, device="cuda")
    A.check(A.lib().av1pf_dsp_cdef_filter(ctx.p, d_win.data_ptr(), d_taps.data_ptr(), d_res.data_ptr(), 3 * n, None))
    torch.cuda.synchronize()
    got = d_res.cpu().numpy().view(np.uint16)
    for e in range(3 * n):
        t = taps[e]
        k = t.w * t.h
        assert np.array_equal(got[e, :k], want[e, :k]), f"window {e} ({t.w}x{t.h}) differs"


# ---------------------------------------------------------------------------
# whole chain
# ---------------------------------------------------------------------------
CHAIN_CASES = {
    "c1_352x288_8bit_u8": dict(width=352, height=288, bit_depth=8, sample_bytes=1, content=1, seed=1, frame_index=2),
    "c1_352x288_8bit_u16": dict(width=352, height=288, bit_depth=8, sample_bytes=2, content=1, seed=1),
    "b10_420": dict(width=480, height=270, bit_depth=10, seed=2),
    "b10_420_seg_dlf": dict(width=320, height=200, bit_depth=10, seed=3, segmentation=1, delta_lf=2),
    "b10_420_dlf1": dict(width=200, height=136, bit_depth=10, seed=33, delta_lf=1, segmentation=1),
    "b12_444": dict(width=256, height=160, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=4),
    "b10_422": dict(width=264, height=130, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=5),
    "b8_mono": dict(width=200, height=120, bit_depth=8, sample_bytes=1, mono=1, seed=6),
    "b12_mono": dict(width=150, height=90, bit_depth=12, mono=1, seed=16),
    "b10_superres_d9": dict(width=400, height=200, bit_depth=10, superres_denom=9, seed=7),
    "b10_superres_d16": dict(width=384, height=180, bit_depth=10, superres_denom=16, seed=8),
    "b12_444_superres_grain": dict(width=288, height=150, bit_depth=12, subsampling_x=0, subsampling_y=0,
                                   superres_denom=13, enable_grain=1, seed=9, frame_index=7),
    "b10_grain": dict(width=330, height=210, bit_depth=10, enable_grain=1, seed=10, frame_index=3),
    "b8_grain_u8": dict(width=300, height=170, bit_depth=8, sample_bytes=1, enable_grain=1, seed=11),
    "b10_422_grain": dict(width=260, height=140, bit_depth=10, subsampling_x=1, subsampling_y=0, enable_grain=1,
                          seed=12),
    "b8_mono_grain": dict(width=180, height=100, bit_depth=8, sample_bytes=1, mono=1, enable_grain=1, seed=13),
    "lr_unit128": dict(width=500, height=300, bit_depth=10, lr_unit_shift=1, seed=14),
    "lr_unit256_uv_same": dict(width=600, height=330, bit_depth=8, sample_bytes=1, lr_unit_shift=2, lr_uv_shift=0,
                               seed=15),
    "big_blocks": dict(width=320, height=256, bit_depth=10, min_block_log2=5, skip_pct=10, seed=17),
    "all_skip": dict(width=256, height=128, bit_depth=10, skip_pct=100, seed=18),
    "no_lf": dict(width=240, height=160, bit_depth=10, enable_lf=0, seed=19),
    "no_cdef": dict(width=240, height=160, bit_depth=10, enable_cdef=0, seed=20),
    "no_lr": dict(width=240, height=160, bit_depth=10, enable_lr=0, seed=21),
    "nothing": dict(width=96, height=64, bit_depth=8, sample_bytes=1, enable_lf=0, enable_cdef=0, enable_lr=0,
                    seed=22),
    "tiny_8x8": dict(width=8, height=8, bit_depth=10, seed=23),
    "tiny_17x9": dict(width=17, height=9, bit_depth=8, sample_bytes=1, seed=24),
    "odd_127x65_grain": dict(width=127, height=65, bit_depth=10, enable_grain=1, seed=25),
    "odd_superres": dict(width=123, height=77, bit_depth=8, sample_bytes=1, superres_denom=11, enable_grain=1,
                         seed=26),
}


@pytest.mark.parametrize("name", sorted(CHAIN_CASES))
def test_chain_matches_oracle(ctx, name):
    sf = A.SynthHandle(**CHAIN_CASES[name])
    ref_cpu, fb_cpu = O.chain(sf, threads=0)
    df = G.DevFrame(sf)
    ref_gpu, fb_gpu = G.gpu_chain(ctx, df)
    assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, name)
    # the input planes are left unchanged
    inp = O.HostPlanes.like_synth(sf)
    for p in range(sf.info.num_planes):
        assert np.array_equal(df.inp.host(p), inp.arrays[p])


def test_chain_repeatable_and_stream(ctx):
    sf = A.SynthHandle(width=320, height=180, bit_depth=10, enable_grain=1, superres_denom=12, seed=40)
    df = G.DevFrame(sf)
    r1, f1 = G.gpu_chain(ctx, df)
    s = torch.cuda.Stream()
    r2, f2 = G.gpu_chain(ctx, df, stream=C.c_void_p(s.cuda_stream))
    assert np.array_equal(f1, f2)
    for a, b in zip(r1, r2):
        assert np.array_equal(a, b)


def test_golden_digests_on_gpu(ctx):
    """The GPU chain reproduces the committed oracle fixtures."""
    import make_golden
    with open(os.path.join(GOLDEN, "chain_digests.json")) as fh:
        want = json.load(fh)
    for name, kw in make_golden.CASES.items():
        sf = A.SynthHandle(**kw)
        df = G.DevFrame(sf)
        refs, fb = G.gpu_chain(ctx, df)
        h = hashlib.sha256()
        for a in refs:
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(fb.tobytes())
        assert h.hexdigest() == want[name], name


# ---------------------------------------------------------------------------
# per-stage entry points
# ---------------------------------------------------------------------------
STAGE_CASES = ["b10_420_seg_dlf", "b12_444", "b10_422", "c1_352x288_8bit_u8", "b8_mono", "b10_superres_d9",
               "b12_444_superres_grain", "lr_unit128"]


@pytest.mark.parametrize("name", STAGE_CASES)
def test_stages_match_oracle(ctx, name):
    sf = A.SynthHandle(**CHAIN_CASES[name])
    info, params, maps = sf.f.info, sf.f.params, sf.f.maps
    L, OL = A.lib(), O.lib()
    df = G.DevFrame(sf)
    np_ = info.num_planes
    # loop filter, in place
    cur = O.HostPlanes.like_synth(sf)
    assert OL.oracle_loop_filter(C.byref(info), C.byref(params), C.byref(maps), cur.c, 0) == 0
    d_cur = G.DevPlanes.from_host(info, O.HostPlanes.like_synth(sf))
    A.check(L.av1pf_loop_filter(ctx.p, C.byref(info), C.byref(params), C.byref(df.maps), d_cur.c, None))
    torch.cuda.synchronize()
    mr, mc = info.mi_rows * 4, info.mi_cols * 4
    for p in range(np_):
        sx = info.subsampling_x if p else 0
        sy = info.subsampling_y if p else 0
        assert np.array_equal(d_cur.host(p), cur.arrays[p]), f"loop filter plane {p}"
    # CDEF (compare the mode-info area: the device writes only there)
    cd = O.HostPlanes.zeros_like(cur)
    assert OL.oracle_cdef(C.byref(info), C.byref(params), C.byref(maps), cur.c, cd.c, 0) == 0
    d_cd = G.DevPlanes.from_host(info, O.HostPlanes.zeros_like(cur))
    A.check(L.av1pf_cdef(ctx.p, C.byref(info), C.byref(params), C.byref(df.maps), d_cur.c, d_cd.c, None))
    torch.cuda.synchronize()
    for p in range(np_):
        sx = info.subsampling_x if p else 0
        sy = info.subsampling_y if p else 0
        w, h = mc >> sx, mr >> sy
        assert np.array_equal(d_cd.host(p, w, h), cd.arrays[p][:h, :w]), f"cdef plane {p}"
    # superres of both frames
    if params.use_superres:
        up_c = O.HostPlanes.upscaled(info)
        up_d = O.HostPlanes.upscaled(info)
        assert OL.oracle_superres(C.byref(info), C.byref(params), cur.c, up_c.c) == 0
        assert OL.oracle_superres(C.byref(info), C.byref(params), cd.c, up_d.c) == 0
        d_upc = G.DevPlanes.from_host(info, O.HostPlanes.upscaled(info))
        d_upd = G.DevPlanes.from_host(info, O.HostPlanes.upscaled(info))
        A.check(L.av1pf_superres(ctx.p, C.byref(info), C.byref(params), d_cur.c, d_upc.c, None))
        A.check(L.av1pf_superres(ctx.p, C.byref(info), C.byref(params), d_cd.c, d_upd.c, None))
        torch.cuda.synchronize()
        for p in range(np_):
            w, h = sf.plane_dims(p)
            assert np.array_equal(d_upc.host(p, w, h), up_c.arrays[p][:h, :w]), f"superres cur {p}"
            assert np.array_equal(d_upd.host(p, w, h), up_d.arrays[p][:h, :w]), f"superres cdef {p}"
        src_cur, src_cd, d_src_cur, d_src_cd = up_c, up_d, d_upc, d_upd
    else:
        src_cur, src_cd, d_src_cur, d_src_cd = cur, cd, d_cur, d_cd
    # loop restoration
    lr = O.HostPlanes.visible(info)
    assert OL.oracle_loop_restoration(C.byref(info), C.byref(params), C.byref(maps), src_cur.c, src_cd.c, lr.c, 0) == 0
    d_lr = G.DevPlanes.visible(info)
    A.check(L.av1pf_loop_restoration(ctx.p, C.byref(info), C.byref(params), C.byref(df.maps), d_src_cur.c,
                                     d_src_cd.c, d_lr.c, None))
    torch.cuda.synchronize()
    for p in range(np_):
        assert np.array_equal(d_lr.host(p), lr.arrays[p]), f"loop restoration plane {p}"
    # output (crop + grain + pack)
    fb = np.zeros(A.frame_bytes(info), np.uint8)
    assert OL.oracle_output(C.byref(info), C.byref(params), lr.c, fb.ctypes.data) == 0
    d_fb = G.dev_bytes(A.frame_bytes(info))
    A.check(L.av1pf_output(ctx.p, C.byref(info), C.byref(params), d_lr.c, d_fb.data_ptr(), None))
    torch.cuda.synchronize()
    assert np.array_equal(d_fb[: A.frame_bytes(info)].cpu().numpy(), fb), "output"


# ---------------------------------------------------------------------------
# host-buffer chain, batch
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["c1_352x288_8bit_u8", "b12_444_superres_grain", "b10_422_grain"])
def test_chain_host_matches_oracle(ctx, name):
    sf = A.SynthHandle(**CHAIN_CASES[name])
    ref_cpu, fb_cpu = O.chain(sf, threads=0)
    info = sf.f.info
    inp = O.HostPlanes.like_synth(sf)
    ref = O.HostPlanes.visible(info)
    fb = np.zeros(A.frame_bytes(info), np.uint8)
    A.check(A.lib().av1pf_chain_host(ctx.p, C.byref(info), C.byref(sf.f.params), C.byref(sf.f.maps), inp.c, ref.c,
                                     fb.ctypes.data))
    assert_same(ref.arrays, fb, ref_cpu, fb_cpu, name)


def test_chain_host_many_matches_oracle(ctx):
    """Frames of different shapes through the pipelined host entry point (more
    frames than device slots, so slots are reused across shapes), some with
    pinned and some with pageable buffers, some without a reference download:
    every output equals the oracle's."""
    import torch
    names = ["c1_352x288_8bit_u8", "b12_444_superres_grain", "b10_420", "b10_422_grain", "tiny_17x9",
             "b10_420", "b8_mono_grain"]
    sfs = [A.SynthHandle(**dict(CHAIN_CASES[n], seed=CHAIN_CASES[n]["seed"] + 7 * i)) for i, n in enumerate(names)]
    want = [O.chain(sf, threads=0) for sf in sfs]
    jobs = (A.HostJob * len(sfs))()
    keep = []
    for i, sf in enumerate(sfs):
        info = sf.f.info
        inp = O.HostPlanes.like_synth(sf)
        ref = O.HostPlanes.visible(info) if i % 3 != 1 else None
        if i % 2 == 0:
            fb_t = torch.zeros(A.frame_bytes(info), dtype=torch.uint8).pin_memory()
            fb, fb_ptr = fb_t, fb_t.data_ptr()
        else:
            fb = np.zeros(A.frame_bytes(info), np.uint8)
            fb_ptr = fb.ctypes.data
        keep.append((inp, ref, fb))
        jobs[i].info = C.pointer(info)
        jobs[i].params = C.pointer(sf.f.params)
        jobs[i].maps = C.pointer(sf.f.maps)
        jobs[i].inp = C.cast(inp.c, C.POINTER(A.Plane))
        jobs[i].ref_out = C.cast(ref.c, C.POINTER(A.Plane)) if ref is not None else None
        jobs[i].frame_out = fb_ptr
    A.check(A.lib().av1pf_chain_host_many(ctx.p, len(sfs), jobs), "chain_host_many")
    for i, ((inp, ref, fb), (ref_cpu, fb_cpu)) in enumerate(zip(keep, want)):
        fb_np = fb.numpy() if hasattr(fb, "numpy") else fb
        assert np.array_equal(fb_np, fb_cpu), f"frame {i} ({names[i]}): packed frame"
        if ref is not None:
            for p in range(sfs[i].info.num_planes):
                assert np.array_equal(ref.arrays[p], ref_cpu.arrays[p]), f"frame {i} plane {p}"
    # an invalid job refuses the whole call before anything is queued
    bad = (A.HostJob * 1)()
    bad[0] = jobs[0]
    bad[0].inp = None
    assert A.lib().av1pf_chain_host_many(ctx.p, 1, bad) == A.ERR_INVALID_INPUT
    A.check(A.lib().av1pf_chain_host_many(ctx.p, 0, None))


def test_batch_matches_per_frame(ctx):
    names = ["c1_352x288_8bit_u8", "b10_420", "b12_444_superres_grain", "b10_422_grain", "b8_mono_grain",
             "tiny_17x9", "lr_unit128", "b10_superres_d16"]
    sfs = [A.SynthHandle(**CHAIN_CASES[n]) for n in names]
    dfs = [G.DevFrame(s) for s in sfs]
    outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]
    jobs = (A.Job * len(dfs))()
    for i, (d, (r, fb)) in enumerate(zip(dfs, outs)):
        jobs[i].info = C.pointer(d.info)
        jobs[i].params = C.pointer(d.params)
        jobs[i].maps = C.pointer(d.maps)
        jobs[i].inp = C.cast(d.inp.c, C.POINTER(A.Plane))
        jobs[i].ref_out = C.cast(r.c, C.POINTER(A.Plane))
        jobs[i].frame_out = fb.data_ptr()
    # graph and direct launches; frame groups on parallel branches (2 and 3)
    for flags in (0, A.BATCH_NO_GRAPH, 3 << A.BATCH_GROUPS_SHIFT, A.BATCH_NO_GRAPH | (2 << A.BATCH_GROUPS_SHIFT)):
        for r, fb in outs:
            for t in r.t:
                t.zero_()
            fb.zero_()
        b = C.c_void_p()
        A.check(A.lib().av1pf_batch_create(ctx.p, jobs, len(dfs), flags, C.byref(b)), "batch_create")
        for _ in range(2):
            A.check(A.lib().av1pf_batch_run(b, None), "batch_run")
        torch.cuda.synchronize()
        for i, (sf, (r, fb)) in enumerate(zip(sfs, outs)):
            ref_cpu, fb_cpu = O.chain(sf, threads=0)
            got = [r.host(p) for p in range(sf.info.num_planes)]
            assert_same(got, fb[: A.frame_bytes(sf.info)].cpu().numpy(), ref_cpu, fb_cpu, f"batch[{i}] {names[i]}")
        A.lib().av1pf_batch_destroy(b)


# ---------------------------------------------------------------------------
# full-size frames
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("cfg", [
    dict(width=1920, height=1080, bit_depth=10, seed=101),
    dict(width=3840, height=2160, bit_depth=10, superres_denom=13, enable_grain=1, seed=102, frame_index=4),
    dict(width=3840, height=2160, bit_depth=12, subsampling_x=0, subsampling_y=0, superres_denom=10,
         enable_grain=1, seed=103, frame_index=5),
])
def test_full_size_frames(ctx, cfg):
    sf = A.SynthHandle(**cfg)
    ref_cpu, fb_cpu = O.chain(sf, threads=0)
    df = G.DevFrame(sf)
    ref_gpu, fb_gpu = G.gpu_chain(ctx, df)
    assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, str(cfg))


# ---------------------------------------------------------------------------
# errors
# ---------------------------------------------------------------------------
def test_invalid_inputs_rejected(ctx):
    sf = A.SynthHandle(width=64, height=64, bit_depth=10, seed=1)
    df = G.DevFrame(sf)
    ref = G.DevPlanes.visible(df.info)
    L = A.lib()
    bad = A.FrameInfo.from_buffer_copy(df.info)
    bad.mi_cols += 2
    assert L.av1pf_chain(ctx.p, C.byref(bad), C.byref(df.params), C.byref(df.maps), df.inp.c, ref.c, None,
                         None) == A.ERR_INVALID_INPUT
    bp = A.Params.from_buffer_copy(df.params)
    bp.cdef_damping = 9
    assert L.av1pf_chain(ctx.p, C.byref(df.info), C.byref(bp), C.byref(df.maps), df.inp.c, ref.c, None,
                         None) == A.ERR_INVALID_INPUT
    small = (A.Plane * 3)(*df.inp.c)
    small[0].width = 16
    assert L.av1pf_chain(ctx.p, C.byref(df.info), C.byref(df.params), C.byref(df.maps), small, ref.c, None,
                         None) == A.ERR_INVALID_INPUT
    assert L.av1pf_last_error()


def random_chain_config(seed):
    """A seeded random frame: size, bit depth and storage, subsampling,
    superres, film grain, segmentation and delta-lf, block sizes and skip
    rate, LR unit sizes, each stage on or off."""
    rng = np.random.default_rng(5000 + seed)
    bd = int(rng.choice([8, 10, 12]))
    sub = [(1, 1), (1, 0), (0, 0)][int(rng.integers(0, 3))]
    cfg = dict(width=int(rng.integers(8, 520)), height=int(rng.integers(8, 300)), bit_depth=bd,
               subsampling_x=sub[0], subsampling_y=sub[1], seed=6000 + seed, frame_index=int(rng.integers(0, 8)),
               content=int(rng.integers(0, 2)), noise_sigma=int(rng.integers(0, 12)),
               enable_lf=int(rng.random() < 0.9), enable_cdef=int(rng.random() < 0.9),
               enable_lr=int(rng.random() < 0.9), enable_grain=int(rng.random() < 0.4),
               segmentation=int(rng.random() < 0.3), delta_lf=int(rng.integers(0, 3)),
               min_block_log2=int(rng.integers(2, 6)), skip_pct=int(rng.integers(0, 101)),
               lr_unit_shift=int(rng.integers(0, 3)), lr_uv_shift=int(rng.integers(0, 2)))
    if bd == 8 and rng.random() < 0.5:
        cfg["sample_bytes"] = 1
    if rng.random() < 0.15:
        cfg["mono"] = 1
    if rng.random() < 0.3:
        cfg["superres_denom"] = int(rng.integers(9, 17))
    return cfg


@pytest.mark.parametrize("seed", range(30))
def test_chain_random_configurations(ctx, seed):
    cfg = random_chain_config(seed)
    sf = A.SynthHandle(**cfg)
    ref_cpu, fb_cpu = O.chain(sf, threads=0)
    ref_gpu, fb_gpu = G.gpu_chain(ctx, G.DevFrame(sf))
    assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, f"random {seed}: {cfg}")
