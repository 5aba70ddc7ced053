"""Kernel variants and the autotuner: every variant computes the same samples.

The chain runs its loop filter in four ways (edge lists for both
directions; vertical edges per shared-memory tile with a horizontal edge
list; the horizontal edges inside the CDEF kernel; or both directions per
shared-memory tile in one kernel) and restores 64- or
32-column loop-restoration rectangles; each combination is compared with the
CPU oracle bit for bit on the same synthetic frames as the chain tests (the
default, mode 3 with 64-column rectangles, is what test_gpu_parity runs). The autotuner is
checked for its bookkeeping and for leaving results unchanged, including a
batch whose frames end up on different variants.
"""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available
from test_gpu_parity import CHAIN_CASES, assert_same

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G
    import torch

VARIANTS = [(0, 64), (1, 64), (2, 64), (0, 32), (2, 32), (3, 32)]


@pytest.fixture(scope="module")
def ctx():
    c = G.Ctx()
    yield c
    c.close()


def set_tuning(ctx, mode, cols):
    t = A.Tuning(mode, cols)
    A.check(A.lib().av1pf_set_tuning(ctx.p, C.byref(t)), "set_tuning")


@pytest.mark.parametrize("variant", VARIANTS, ids=[f"lf{m}_lr{c}" for m, c in VARIANTS])
@pytest.mark.parametrize("name", sorted(CHAIN_CASES))
def test_chain_variant_matches_oracle(ctx, name, variant):
    set_tuning(ctx, *variant)
    try:
        sf = A.SynthHandle(**CHAIN_CASES[name])
        ref_cpu, fb_cpu = O.chain(sf, threads=0)
        ref_gpu, fb_gpu = G.gpu_chain(ctx, G.DevFrame(sf))
        assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, f"{name} {variant}")
    finally:
        set_tuning(ctx, -1, 0)


@pytest.mark.parametrize("variant", [(0, 64), (1, 64), (2, 64)])
def test_full_hd_variant(ctx, variant):
    set_tuning(ctx, *variant)
    try:
        sf = A.SynthHandle(width=1920, height=1080, bit_depth=10, seed=111)
        ref_cpu, fb_cpu = O.chain(sf, threads=0)
        ref_gpu, fb_gpu = G.gpu_chain(ctx, G.DevFrame(sf))
        assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, f"1080p {variant}")
    finally:
        set_tuning(ctx, -1, 0)


def test_full_superblock_ctas_with_fused_lf(ctx):
    """A 4K frame has more than one wave of CDEF superblocks, so CDEF runs a
    CTA per whole superblock (1080p and smaller frames run halves); with
    loop-filter mode 2 that path also filters the horizontal edges and writes
    the stripe-boundary rows."""
    set_tuning(ctx, 2, 64)
    try:
        sf = A.SynthHandle(width=3840, height=2160, bit_depth=10, seed=113)
        ref_cpu, fb_cpu = O.chain(sf, threads=0)
        ref_gpu, fb_gpu = G.gpu_chain(ctx, G.DevFrame(sf))
        assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, "4K lf_mode 2")
    finally:
        set_tuning(ctx, -1, 0)


def test_tuning_rejects_bad_values(ctx):
    for bad in [(4, 0), (-2, 0), (0, 48), (1, 128)]:
        t = A.Tuning(*bad)
        assert A.lib().av1pf_set_tuning(ctx.p, C.byref(t)) == A.ERR_INVALID_INPUT
    t = A.Tuning()
    A.check(A.lib().av1pf_get_tuning(ctx.p, C.byref(t)))
    assert (t.lf_mode, t.lr_rect_cols) == (-1, 0)


def _jobs(dfs, outs):
    jobs = (A.Job * len(dfs))()
    for i, (d, (r, fb)) in enumerate(zip(dfs, outs)):
        jobs[i].info = C.pointer(d.info)
        jobs[i].params = C.pointer(d.params)
        jobs[i].maps = C.pointer(d.maps)
        jobs[i].inp = C.cast(d.inp.c, C.POINTER(A.Plane))
        jobs[i].ref_out = C.cast(r.c, C.POINTER(A.Plane))
        jobs[i].frame_out = fb.data_ptr()
    return jobs


def test_autotune_records_shapes_and_keeps_results():
    c = G.Ctx()  # a fresh context: nothing recorded yet
    try:
        names = ["b10_420", "b12_444_superres_grain", "no_cdef", "b10_420"]
        sfs = [A.SynthHandle(**dict(CHAIN_CASES[n], seed=CHAIN_CASES[n]["seed"] + 100 * i))
               for i, n in enumerate(names)]
        dfs = [G.DevFrame(s) for s in sfs]
        outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]
        jobs = _jobs(dfs, outs)
        t = A.Tuning()
        ms = C.c_float()
        assert A.lib().av1pf_tuned_choice(c.p, C.byref(dfs[0].info), C.byref(t), C.byref(ms)) == A.ERR_NOT_FOUND
        n = C.c_int32()
        A.check(A.lib().av1pf_autotune(c.p, jobs, len(dfs), 3, C.byref(n)), "autotune")
        assert n.value == 3  # the two b10_420 frames share a shape
        for d in dfs:
            A.check(A.lib().av1pf_tuned_choice(c.p, C.byref(d.info), C.byref(t), C.byref(ms)))
            assert t.lf_mode in (0, 1, 2, 3) and t.lr_rect_cols in (32, 64) and ms.value > 0
        # CDEF off: the horizontal pass inside CDEF does not apply, so mode 2 is never chosen
        A.check(A.lib().av1pf_tuned_choice(c.p, C.byref(dfs[2].info), C.byref(t), C.byref(ms)))
        assert t.lf_mode in (0, 1, 3)
        # the chain and a batch on the recorded choices still match the oracle
        for sf, d in zip(sfs, dfs):
            ref_cpu, fb_cpu = O.chain(sf, threads=0)
            ref_gpu, fb_gpu = G.gpu_chain(c, d)
            assert_same(ref_gpu, fb_gpu, ref_cpu, fb_cpu, "tuned chain")
        for r, fb in outs:
            for x in r.t:
                x.zero_()
            fb.zero_()
        b = C.c_void_p()
        A.check(A.lib().av1pf_batch_create(c.p, jobs, len(dfs), A.BATCH_AUTOTUNE, C.byref(b)), "batch_create")
        A.check(A.lib().av1pf_batch_run(b, None), "batch_run")
        torch.cuda.synchronize()
        for i, (sf, (r, fb)) in enumerate(zip(sfs, outs)):
            ref_cpu, fb_cpu = O.chain(sf, threads=0)
            got = [r.host(p) for p in range(sf.info.num_planes)]
            assert_same(got, fb[: A.frame_bytes(sf.info)].cpu().numpy(), ref_cpu, fb_cpu, f"tuned batch[{i}]")
        A.lib().av1pf_batch_destroy(b)
    finally:
        c.close()


def test_batch_mixing_fused_and_separate_frames(ctx):
    """A batch where some frames take the fused pass and some cannot (CDEF
    off) runs the separate horizontal pass for those alone."""
    set_tuning(ctx, 2, 64)
    try:
        names = ["b10_420", "no_cdef", "b8_grain_u8", "b10_422_grain"]
        sfs = [A.SynthHandle(**CHAIN_CASES[n]) for n in names]
        dfs = [G.DevFrame(s) for s in sfs]
        outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]
        jobs = _jobs(dfs, outs)
        b = C.c_void_p()
        A.check(A.lib().av1pf_batch_create(ctx.p, jobs, len(dfs), 0, C.byref(b)), "batch_create")
        A.check(A.lib().av1pf_batch_run(b, None), "batch_run")
        torch.cuda.synchronize()
        for i, (sf, (r, fb)) in enumerate(zip(sfs, outs)):
            ref_cpu, fb_cpu = O.chain(sf, threads=0)
            got = [r.host(p) for p in range(sf.info.num_planes)]
            assert_same(got, fb[: A.frame_bytes(sf.info)].cpu().numpy(), ref_cpu, fb_cpu, f"mixed batch[{i}]")
        A.lib().av1pf_batch_destroy(b)
    finally:
        set_tuning(ctx, -1, 0)


def test_per_frame_many_shapes(ctx):
    """av1pf_chain replans only the descriptors while the structure repeats
    and uploads them into two buffers in turn: cycle 11 shapes twice,
    interleaved (every call a new structure), and check every result."""
    cfgs = [dict(width=64 + 24 * k, height=48 + 16 * k, bit_depth=(8, 10, 12)[k % 3],
                 sample_bytes=1 if k % 3 == 0 else 2, enable_grain=k % 2, superres_denom=9 + k % 8 if k % 4 == 1 else 8,
                 seed=500 + k) for k in range(11)]
    sfs = [A.SynthHandle(**c) for c in cfgs]
    want = [O.chain(sf, threads=0) for sf in sfs]
    dfs = [G.DevFrame(sf) for sf in sfs]
    launches0 = A.lib().av1pf_launch_count()
    for rnd in range(2):
        for k in list(range(11)) + list(range(10, -1, -1)):
            ref_gpu, fb_gpu = G.gpu_chain(ctx, dfs[k])
            assert_same(ref_gpu, fb_gpu, want[k][0], want[k][1], f"shape {k} round {rnd}")
    # every call launched its kernels
    assert A.lib().av1pf_launch_count() - launches0 >= 2 * 22 * 4
