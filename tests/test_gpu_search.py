"""The encoder's filter searches on the GPU (av1pf_cdef_search,
av1pf_lf_search, av1pf_lr_search) against the oracle, bit for bit: the
chosen CDEF strengths, bits and damping, the per-block index table and every
candidate's per-block error; the loop-filter levels and every scale's plane
errors; every restoration unit's choice (type, Wiener coefficients,
self-guided set and weights) and each plane's restoration type. Shapes cover
8/10/12-bit, one- and two-byte samples, 4:2:0, 4:2:2, 4:4:4 and monochrome,
ragged frame edges, full HD, frames with no coding block, and both
candidate lists."""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available
from test_search import CASES, coding_blocks

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G
    import torch

GPU_CASES = dict(CASES)
GPU_CASES["1920x1080_10b"] = dict(width=1920, height=1080, bit_depth=10, seed=21)
GPU_CASES["1000x600_12b_444"] = dict(width=1000, height=600, bit_depth=12, subsampling_x=0, subsampling_y=0,
                                     seed=22)


@pytest.fixture(scope="module")
def ctx():
    c = G.Ctx()
    yield c
    c.close()


def gpu_cdef_search(ctx, sf, df, cur, src, q, lam, thorough):
    info = sf.f.info
    fbr, fbc = (info.mi_rows + 15) // 16, (info.mi_cols + 15) // 16
    ny, nuv = A.CDEF_SEARCH_N[bool(thorough)]
    dcur, dsrc = G.DevPlanes.from_host(info, cur), G.DevPlanes.from_host(info, src)
    res = A.CdefSearchResult()
    table = np.zeros(fbr * df.maps.cdef_stride, np.int8)
    sse = np.zeros((fbr * fbc, ny + nuv), np.uint64)
    A.check(A.lib().av1pf_cdef_search(ctx.p, C.byref(info), C.byref(df.maps), dcur.c, dsrc.c, q, lam,
                                      int(thorough), C.byref(res), table.ctypes.data, sse.ctypes.data, None),
            "av1pf_cdef_search")
    return res, table, sse


def assert_cdef_same(g, o, what):
    (rg, tg, sg), (ro, to, so) = g, o
    assert (rg.damping_minus_3, rg.bits) == (ro.damping_minus_3, ro.bits), what
    assert rg.pairs() == ro.pairs(), what
    assert np.array_equal(sg, so), f"{what}: block errors differ at {np.argwhere(sg != so)[:5]}"
    assert np.array_equal(tg, to), what


@pytest.mark.parametrize("thorough", [False, True], ids=["fast", "thorough"])
@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_cdef_search_matches_oracle(ctx, name, thorough):
    sf = A.SynthHandle(**GPU_CASES[name])
    cur, src = O.search_inputs(sf, 31)
    df = G.DevFrame(sf)
    for q, lam in ((30, 0.0), (140, 40.0), (250, 900.0)):
        o = O.cdef_search(sf, cur, src, q, lam, thorough)
        g = gpu_cdef_search(ctx, sf, df, cur, src, q, lam, thorough)
        assert_cdef_same(g, o, f"{name} q{q} lambda{lam}")


def test_cdef_search_picks_filters_on_noisy_reconstruction(ctx):
    """A reconstruction with strong block noise: the search chooses several
    nonzero strengths, and GPU and oracle agree on them."""
    sf = A.SynthHandle(**GPU_CASES["1920x1080_10b"])
    cur, src = O.search_inputs(sf, 32, amp=24)
    o = O.cdef_search(sf, cur, src, 120, 1.0, False)
    g = gpu_cdef_search(ctx, sf, G.DevFrame(sf), cur, src, 120, 1.0, False)
    assert_cdef_same(g, o, "noisy 1080p")
    assert o[0].bits >= 1 and any(p != (0, 0, 0, 0) for p in o[0].pairs())


def test_cdef_search_without_coding_blocks(ctx):
    sf = A.SynthHandle(**GPU_CASES["200x120_8b"])
    idx, _, _ = coding_blocks(sf)
    idx[:] = -1
    cur, src = O.search_inputs(sf, 33)
    o = O.cdef_search(sf, cur, src, 200, 5.0, True)
    g = gpu_cdef_search(ctx, sf, G.DevFrame(sf), cur, src, 200, 5.0, True)
    assert_cdef_same(g, o, "no coding blocks")
    assert g[0].bits == 0 and g[0].damping_minus_3 == 0


def test_cdef_search_rejects_bad_arguments(ctx):
    sf = A.SynthHandle(**GPU_CASES["256x144_10b"])
    cur, src = O.search_inputs(sf, 34)
    df = G.DevFrame(sf)
    info = sf.f.info
    dcur, dsrc = G.DevPlanes.from_host(info, cur), G.DevPlanes.from_host(info, src)
    res = A.CdefSearchResult()
    L = A.lib()
    for q, lam in ((-1, 1.0), (256, 1.0), (10, float("nan")), (10, -1.0), (10, float("inf"))):
        rc = L.av1pf_cdef_search(ctx.p, C.byref(info), C.byref(df.maps), dcur.c, dsrc.c, q, lam, 0, C.byref(res),
                                 None, None, None)
        assert rc == A.ERR_INVALID_INPUT, (q, lam)
    assert L.av1pf_cdef_search(ctx.p, C.byref(info), C.byref(df.maps), dcur.c, None, 10, 1.0, 0, C.byref(res),
                               None, None, None) == A.ERR_INVALID_INPUT


def gpu_lf_search(ctx, sf, cur, src, params=None):
    info = sf.f.info
    df = G.DevFrame(sf)
    dcur, dsrc = G.DevPlanes.from_host(info, cur), G.DevPlanes.from_host(info, src)
    levels = (C.c_int32 * 4)()
    sse = np.zeros((6, 3), np.uint64)
    A.check(A.lib().av1pf_lf_search(ctx.p, C.byref(info), C.byref(params if params is not None else sf.f.params),
                                    C.byref(df.maps), dcur.c, dsrc.c, levels, sse.ctypes.data, None),
            "av1pf_lf_search")
    torch.cuda.synchronize()
    # the reconstruction is left unfiltered
    for p in range(info.num_planes):
        a = dcur.host(p)
        assert np.array_equal(a, cur.arrays[p]), "av1pf_lf_search changed its input"
    return list(levels), sse


@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_lf_search_matches_oracle(ctx, name):
    sf = A.SynthHandle(**GPU_CASES[name])
    cur, src = O.search_inputs(sf, 35)
    lv_o, sse_o = O.lf_search(sf, cur, src)
    lv_g, sse_g = gpu_lf_search(ctx, sf, cur, src)
    assert np.array_equal(sse_g, sse_o), name
    assert lv_g == lv_o, name


def test_lf_search_picks_levels_on_blocky_reconstruction(ctx):
    """Starting levels with blocking artefacts to remove: a nonzero level is
    chosen and GPU and oracle agree on every scale's errors."""
    sf = A.SynthHandle(**GPU_CASES["256x144_10b"])
    src = O.HostPlanes.like_synth(sf)
    rng = np.random.default_rng(36)
    cur = []
    for a in src.arrays:
        h, w = a.shape
        steps = np.kron(rng.integers(-40, 41, size=((h + 7) // 8, (w + 7) // 8)), np.ones((8, 8), np.int64))[:h, :w]
        cur.append(np.clip(a.astype(np.int64) + steps, 0, 1023).astype(a.dtype))
    cur = O.HostPlanes(cur)
    p = A.Params.from_buffer_copy(sf.f.params)
    for k, v in enumerate((30, 30, 20, 20)):
        p.loop_filter_level[k] = v
    lv_o, sse_o = O.lf_search(sf, cur, src, params=p)
    lv_g, sse_g = gpu_lf_search(ctx, sf, cur, src, params=p)
    assert np.array_equal(sse_g, sse_o) and lv_g == lv_o
    assert lv_o[0] > 0


LR_CASES = {
    "256x144_10b": dict(width=256, height=144, bit_depth=10, seed=41, enable_lr=1),
    "200x120_8b_u8": dict(width=200, height=120, bit_depth=8, sample_bytes=1, seed=42, enable_lr=1, lr_unit_shift=1),
    "136x72_12b_444": dict(width=136, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=43,
                           enable_lr=1),
    "160x96_10b_422": dict(width=160, height=96, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=44,
                           enable_lr=1, lr_unit_shift=2),
    "120x80_10b_mono": dict(width=120, height=80, bit_depth=10, mono=1, seed=45, enable_lr=1),
    "600x300_12b_256units": dict(width=600, height=300, bit_depth=12, seed=46, enable_lr=1, lr_unit_shift=2,
                                 lr_uv_shift=0),
    "1920x1080_10b": dict(width=1920, height=1080, bit_depth=10, seed=47, enable_lr=1),
}


def gpu_lr_search(ctx, sf, cur, cdef, src, lam, effort):
    info, params = sf.f.info, sf.f.params
    dcur, dcdef, dsrc = (G.DevPlanes.from_host(info, x) for x in (cur, cdef, src))
    arrs = O.lr_unit_arrays(params, info.num_planes)
    ptrs = (C.POINTER(A.LrUnit) * 3)(*[C.cast(a, C.POINTER(A.LrUnit)) if a is not None else None for a in arrs])
    ft = (C.c_int32 * 3)()
    A.check(A.lib().av1pf_lr_search(ctx.p, C.byref(info), C.byref(params), dcur.c, dcdef.c, dsrc.c, lam, effort,
                                    ptrs, ft, None), "av1pf_lr_search")
    units = [[O.lr_unit_tuple(u) for u in arrs[p][:params.lr_unit_rows[p] * params.lr_unit_cols[p]]]
             if arrs[p] is not None else [] for p in range(3)]
    return list(ft), units


@pytest.mark.parametrize("effort", [0, 1, 2], ids=["fast", "normal", "thorough"])
@pytest.mark.parametrize("name", sorted(LR_CASES))
def test_lr_search_matches_oracle(ctx, name, effort):
    sf = A.SynthHandle(**LR_CASES[name])
    cur, cdef, src = O.lr_search_inputs(sf, 51)
    # lambda -1e12 makes every unit take its Wiener filter (every fitted
    # coefficient compared); 0 takes the least error (self-guided fits compared)
    for lam in (0.0, 150.0, -1e12):
        o = O.lr_search(sf, cur, cdef, src, lam, effort)
        g = gpu_lr_search(ctx, sf, cur, cdef, src, lam, effort)
        assert g[0] == o[0], f"{name} lambda {lam}: frame types"
        for p in range(3):
            bad = [k for k, (a, b) in enumerate(zip(g[1][p], o[1][p])) if a != b]
            assert not bad, f"{name} lambda {lam} plane {p}: units {bad[:4]} gpu {[g[1][p][k] for k in bad[:2]]} " \
                            f"oracle {[o[1][p][k] for k in bad[:2]]}"


def test_lr_search_identity_and_rejection(ctx):
    sf = A.SynthHandle(**LR_CASES["256x144_10b"])
    cur, cdef, src = O.lr_search_inputs(sf, 52)
    ft, units = gpu_lr_search(ctx, sf, cur, src, src, 5.0, 1)
    assert ft == [0, 0, 0] and all(u[0] == 0 for pl in units for u in pl)
    info, params = sf.f.info, sf.f.params
    d = G.DevPlanes.from_host(info, src)
    arrs = O.lr_unit_arrays(params, info.num_planes)
    ptrs = (C.POINTER(A.LrUnit) * 3)(*[C.cast(a, C.POINTER(A.LrUnit)) for a in arrs])
    ft = (C.c_int32 * 3)()
    L = A.lib()
    for lam, eff in ((float("nan"), 1), (1.0, 3), (1.0, -1)):
        assert L.av1pf_lr_search(ctx.p, C.byref(info), C.byref(params), d.c, d.c, d.c, lam, eff, ptrs, ft,
                                 None) == A.ERR_INVALID_INPUT
    assert L.av1pf_lr_search(ctx.p, C.byref(info), C.byref(params), d.c, None, d.c, 1.0, 1, ptrs, ft,
                             None) == A.ERR_INVALID_INPUT


def test_searches_interleaved_with_chains_on_one_context(ctx):
    """The searches share the context with the chain (its streams, events,
    descriptor buffers and the loop-filter search's planning): chains run
    before, between and after them stay bit-exact, and each search repeats
    its result."""
    sf_chain = A.SynthHandle(width=640, height=360, bit_depth=10, superres_denom=12, enable_grain=1, seed=61)
    ref_cpu, fb_cpu = O.chain(sf_chain, threads=0)
    df_chain = G.DevFrame(sf_chain)

    def chain_ok():
        ref_gpu, fb_gpu = G.gpu_chain(ctx, df_chain)
        assert all(np.array_equal(g, c) for g, c in zip(ref_gpu, ref_cpu.arrays))
        assert np.array_equal(fb_gpu, fb_cpu)

    sf = A.SynthHandle(width=320, height=192, bit_depth=10, seed=62, enable_lr=1)
    cur, src = O.search_inputs(sf, 63)
    lcur, lcdef, lsrc = O.lr_search_inputs(sf, 64)
    df = G.DevFrame(sf)
    want_cdef = O.cdef_search(sf, cur, src, 100, 20.0, False)
    want_lf = O.lf_search(sf, cur, src)
    want_lr = O.lr_search(sf, lcur, lcdef, lsrc, 80.0, 1)
    chain_ok()
    for _ in range(2):
        assert_cdef_same(gpu_cdef_search(ctx, sf, df, cur, src, 100, 20.0, False), want_cdef, "interleaved")
        chain_ok()
        lv, sse = gpu_lf_search(ctx, sf, cur, src)
        assert lv == want_lf[0] and np.array_equal(sse, want_lf[1])
        chain_ok()
        assert gpu_lr_search(ctx, sf, lcur, lcdef, lsrc, 80.0, 1) == want_lr
        chain_ok()


@pytest.mark.parametrize("seed", range(40))
def test_searches_random_configurations(ctx, seed):
    """Seeded random frame shapes and parameters through all three searches,
    GPU against oracle: 8/10/12-bit, u8/u16, every subsampling, sizes from
    8 samples up, both CDEF lists, every LR effort and unit size, lambdas of
    both signs (LR) and zero."""
    rng = np.random.default_rng(1000 + seed)
    bd = int(rng.choice([8, 10, 12]))
    sub = [(1, 1), (1, 0), (0, 0)][int(rng.integers(0, 3))]
    cfg = dict(width=int(rng.integers(8, 400)), height=int(rng.integers(8, 260)), bit_depth=bd,
               subsampling_x=sub[0], subsampling_y=sub[1], seed=2000 + seed, enable_lr=1,
               lr_unit_shift=int(rng.integers(0, 3)), lr_uv_shift=int(rng.integers(0, 2)),
               skip_pct=int(rng.integers(0, 100)))
    if bd == 8 and rng.random() < 0.5:
        cfg["sample_bytes"] = 1
    if rng.random() < 0.15:
        cfg["mono"] = 1
    sf = A.SynthHandle(**cfg)
    amp = int(rng.integers(1, 40)) << (bd - 8)
    cur, src = O.search_inputs(sf, 3000 + seed, amp=amp)
    df = G.DevFrame(sf)
    q, lam, thorough = int(rng.integers(0, 256)), float(rng.choice([0.0, 3.0, 50.0, 2000.0])), bool(rng.random() < 0.5)
    assert_cdef_same(gpu_cdef_search(ctx, sf, df, cur, src, q, lam, thorough),
                     O.cdef_search(sf, cur, src, q, lam, thorough), f"cdef {cfg}")
    lv, sse = gpu_lf_search(ctx, sf, cur, src)
    lv_o, sse_o = O.lf_search(sf, cur, src)
    assert lv == lv_o and np.array_equal(sse, sse_o), f"lf {cfg}"
    lcur, lcdef, lsrc = O.lr_search_inputs(sf, 4000 + seed, amp=amp)
    eff, llam = int(rng.integers(0, 3)), float(rng.choice([0.0, 40.0, 500.0, -1e9]))
    assert gpu_lr_search(ctx, sf, lcur, lcdef, lsrc, llam, eff) == O.lr_search(sf, lcur, lcdef, lsrc, llam, eff), \
        f"lr {cfg} effort {eff} lambda {llam}"


@pytest.mark.parametrize("thorough", [False, True], ids=["fast", "thorough"])
def test_cdef_search_many_matches_per_frame_oracle(ctx, thorough):
    """A batch of frames of different shapes, formats, q and lambda in one
    call: each frame's result, table and block errors equal the oracle's
    per-frame search."""
    cfgs = [dict(width=640, height=360, bit_depth=10, seed=71), dict(width=200, height=120, bit_depth=8,
                                                                      sample_bytes=1, seed=72),
            dict(width=136, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=73),
            dict(width=120, height=80, bit_depth=10, mono=1, seed=74),
            dict(width=72, height=40, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=75),
            dict(width=1920, height=1080, bit_depth=10, seed=76)]
    sfs = [A.SynthHandle(**c) for c in cfgs]
    idx, _, _ = coding_blocks(sfs[4])
    idx[:] = -1  # one frame without coding blocks
    keep, jobs, want = [], (A.CdefSearchJob * len(sfs))(), []
    ny, nuv = A.CDEF_SEARCH_N[thorough]
    for i, sf in enumerate(sfs):
        cur, src = O.search_inputs(sf, 80 + i, amp=8 << (sf.f.info.bit_depth - 8))
        q, lam = 40 * i + 10, [0.0, 5.0, 60.0, 900.0, 2.0, 40.0][i]
        want.append(O.cdef_search(sf, cur, src, q, lam, thorough))
        info = sf.f.info
        df = G.DevFrame(sf)
        dcur, dsrc = G.DevPlanes.from_host(info, cur), G.DevPlanes.from_host(info, src)
        fbr, fbc = (info.mi_rows + 15) // 16, (info.mi_cols + 15) // 16
        res = A.CdefSearchResult()
        table = np.zeros(fbr * df.maps.cdef_stride, np.int8)
        sse = np.zeros((fbr * fbc, ny + nuv), np.uint64)
        keep.append((sf, df, dcur, dsrc, res, table, sse))
        jobs[i].info = C.pointer(info)
        jobs[i].maps = C.pointer(df.maps)
        jobs[i].cur = C.cast(dcur.c, C.POINTER(A.Plane))
        jobs[i].src = C.cast(dsrc.c, C.POINTER(A.Plane))
        jobs[i].base_q_idx = q
        jobs[i].lam = lam
        jobs[i].result = C.pointer(res)
        jobs[i].cdef_idx_out = table.ctypes.data
        jobs[i].block_sse = sse.ctypes.data
    A.check(A.lib().av1pf_cdef_search_many(ctx.p, len(sfs), jobs, int(thorough), None), "av1pf_cdef_search_many")
    for i, (sf, df, dcur, dsrc, res, table, sse) in enumerate(keep):
        assert_cdef_same((res, table, sse), want[i], f"batch frame {i}")


@pytest.mark.parametrize("effort", [0, 1, 2], ids=["fast", "normal", "thorough"])
def test_lr_search_many_matches_per_frame_oracle(ctx, effort):
    """A batch of frames of different shapes, formats, unit sizes and lambdas
    in one call: each frame's units and restoration types equal the oracle's
    per-frame search."""
    cfgs = [dict(width=256, height=144, bit_depth=10, seed=141, enable_lr=1),
            dict(width=200, height=120, bit_depth=8, sample_bytes=1, seed=142, enable_lr=1, lr_unit_shift=1),
            dict(width=136, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=143, enable_lr=1),
            dict(width=120, height=80, bit_depth=10, mono=1, seed=144, enable_lr=1),
            dict(width=600, height=300, bit_depth=12, seed=145, enable_lr=1, lr_unit_shift=2, lr_uv_shift=0)]
    lams = [0.0, 150.0, -1e12, 40.0, 300.0]
    keep, want = [], []
    jobs = (A.LrSearchJob * len(cfgs))()
    for i, cfg in enumerate(cfgs):
        sf = A.SynthHandle(**cfg)
        cur, cdef, src = O.lr_search_inputs(sf, 150 + i)
        want.append(O.lr_search(sf, cur, cdef, src, lams[i], effort))
        info, params = sf.f.info, sf.f.params
        dev = [G.DevPlanes.from_host(info, x) for x in (cur, cdef, src)]
        arrs = O.lr_unit_arrays(params, info.num_planes)
        keep.append((sf, dev, arrs))
        jobs[i].info = C.pointer(info)
        jobs[i].params = C.pointer(params)
        jobs[i].cur = C.cast(dev[0].c, C.POINTER(A.Plane))
        jobs[i].cdef = C.cast(dev[1].c, C.POINTER(A.Plane))
        jobs[i].src = C.cast(dev[2].c, C.POINTER(A.Plane))
        jobs[i].lam = lams[i]
        for p in range(3):
            jobs[i].units_out[p] = C.cast(arrs[p], C.POINTER(A.LrUnit)) if arrs[p] is not None else None
    A.check(A.lib().av1pf_lr_search_many(ctx.p, len(cfgs), jobs, effort, None), "av1pf_lr_search_many")
    for i, (sf, dev, arrs) in enumerate(keep):
        params = sf.f.params
        units = [[O.lr_unit_tuple(u) for u in arrs[p][:params.lr_unit_rows[p] * params.lr_unit_cols[p]]]
                 if arrs[p] is not None else [] for p in range(3)]
        assert (list(jobs[i].frame_type_out), units) == want[i], f"batch frame {i}"


def test_lf_search_many_matches_per_frame_oracle(ctx):
    """A batch of frames of different shapes, formats and starting levels in
    one call: each frame's levels and errors equal the oracle's search."""
    cfgs = [dict(width=256, height=144, bit_depth=10, seed=171), dict(width=200, height=120, bit_depth=8,
                                                                       sample_bytes=1, seed=172),
            dict(width=136, height=72, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=173),
            dict(width=120, height=80, bit_depth=10, mono=1, seed=174),
            dict(width=640, height=360, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=175)]
    keep, want = [], []
    jobs = (A.LfSearchJob * len(cfgs))()
    for i, cfg in enumerate(cfgs):
        sf = A.SynthHandle(**cfg)
        cur, src = O.search_inputs(sf, 180 + i, amp=(10 + 8 * i) << (sf.f.info.bit_depth - 8))
        p = A.Params.from_buffer_copy(sf.f.params)
        for k, v in enumerate(((8, 8, 4, 4), (30, 30, 20, 20), (63, 50, 63, 0), (12, 0, 5, 5), (0, 0, 9, 9))[i]):
            p.loop_filter_level[k] = v
        want.append(O.lf_search(sf, cur, src, params=p))
        info = sf.f.info
        df = G.DevFrame(sf)
        dcur, dsrc = G.DevPlanes.from_host(info, cur), G.DevPlanes.from_host(info, src)
        sse = np.zeros((6, 3), np.uint64)
        keep.append((sf, p, df, dcur, dsrc, sse))
        jobs[i].info = C.pointer(info)
        jobs[i].params = C.pointer(p)
        jobs[i].maps = C.pointer(df.maps)
        jobs[i].cur = C.cast(dcur.c, C.POINTER(A.Plane))
        jobs[i].src = C.cast(dsrc.c, C.POINTER(A.Plane))
        jobs[i].sse_out = sse.ctypes.data
    A.check(A.lib().av1pf_lf_search_many(ctx.p, len(cfgs), jobs, None), "av1pf_lf_search_many")
    for i, (sf, p, df, dcur, dsrc, sse) in enumerate(keep):
        assert list(jobs[i].levels_out) == want[i][0], f"batch frame {i}"
        assert np.array_equal(sse, want[i][1]), f"batch frame {i}"
