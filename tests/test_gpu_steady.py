"""The per-frame paths as the benchmark times them: distinct frames of one
shape through back-to-back av1pf_chain calls on one context, with no host
synchronisation between the calls; and av1pf_set_threads, which sets how
many frames the pipelined host entry point keeps in flight.

After the first call of a shape, av1pf_chain rebuilds only the frame
descriptors (the work lists repeat) and uploads them into two descriptor
buffers in turn, so call k's upload overlaps call k-1's kernels. Every
frame's reference planes and packed output are compared with the oracle bit
for bit, which covers the descriptor-only replan and both buffers on frames
whose content differs.
"""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O
import replica as R
from conftest import cuda_available
from test_gpu_parity import assert_same

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G
    import torch


@pytest.fixture(scope="module")
def ctx():
    c = G.Ctx()
    yield c
    c.close()


def _run_back_to_back(ctx, sfs, rounds=2):
    dfs = [G.DevFrame(s) for s in sfs]
    outs = [[(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs] for _ in range(rounds)]
    L = A.lib()
    for rnd in range(rounds):
        for d, (r, fb) in zip(dfs, outs[rnd]):
            A.check(L.av1pf_chain(ctx.p, C.byref(d.info), C.byref(d.params), C.byref(d.maps), d.inp.c, r.c,
                                  fb.data_ptr(), None), "av1pf_chain")
    torch.cuda.synchronize()
    return outs


@pytest.mark.parametrize("grain", [0, 1], ids=["plain", "grain"])
def test_back_to_back_1080p_frames_match_oracle(ctx, grain):
    """8 distinct 1920x1080 10-bit 4:2:0 frames of the benchmark's pool
    generator, twice over, launched back to back."""
    n = 8
    sfs = [A.SynthHandle(width=1920, height=1080, bit_depth=10, enable_grain=grain, frame_index=i,
                         seed=R.frame_seed(0, i)) for i in range(n)]
    outs = _run_back_to_back(ctx, sfs)
    for i, sf in enumerate(sfs):
        ref_cpu, fb_cpu = O.chain(sf, threads=0)
        for rnd, o in enumerate(outs):
            r, fb = o[i]
            got = [r.host(p) for p in range(sf.info.num_planes)]
            assert_same(got, fb[: A.frame_bytes(sf.info)].cpu().numpy(), ref_cpu, fb_cpu,
                        f"frame {i} round {rnd} grain {grain}")


def test_back_to_back_frames_differ(ctx):
    """The pool's frames really differ (a replan that reused one frame's
    descriptors for the next would otherwise go unnoticed)."""
    sfs = [A.SynthHandle(width=640, height=360, bit_depth=10, seed=R.frame_seed(0, i)) for i in range(3)]
    outs = _run_back_to_back(ctx, sfs, rounds=1)[0]
    packed = [fb[: A.frame_bytes(s.info)].cpu().numpy() for s, (r, fb) in zip(sfs, outs)]
    assert not np.array_equal(packed[0], packed[1]) and not np.array_equal(packed[1], packed[2])
    for sf, p in zip(sfs, packed):
        assert np.array_equal(p, O.chain(sf, threads=0)[1])


def _host_jobs(sfs):
    jobs = (A.HostJob * len(sfs))()
    keep = []
    for i, sf in enumerate(sfs):
        info = sf.f.info
        inp = O.HostPlanes.like_synth(sf)
        fb = np.zeros(A.frame_bytes(info), np.uint8)
        keep.append((inp, fb))
        jobs[i].info = C.pointer(info)
        jobs[i].params = C.pointer(sf.f.params)
        jobs[i].maps = C.pointer(sf.f.maps)
        jobs[i].inp = C.cast(inp.c, C.POINTER(A.Plane))
        jobs[i].ref_out = None
        jobs[i].frame_out = fb.ctypes.data
    return jobs, keep


@pytest.mark.parametrize("threads", [1, 2, 5])
def test_set_threads_sets_host_frame_slots(threads):
    """av1pf_set_threads(n) sets how many frames av1pf_chain_host_many keeps
    in flight, one device frame slot each: against a context left at the
    default of 3 slots, the context holds (n - 3) slots' bytes more, and
    every frame still equals the oracle's."""
    sfs = [A.SynthHandle(width=352, height=288, bit_depth=10, seed=40 + i, frame_index=i) for i in range(6)]
    want = [O.chain(sf, threads=0)[1] for sf in sfs]
    held = {}
    for n in (0, threads):  # 0 = the default
        c = G.Ctx()
        try:
            A.check(A.lib().av1pf_set_threads(c.p, n), "set_threads")
            jobs, keep = _host_jobs(sfs)
            A.check(A.lib().av1pf_chain_host_many(c.p, len(sfs), jobs), "chain_host_many")
            for i, (inp, fb) in enumerate(keep):
                assert np.array_equal(fb, want[i]), f"threads {n} frame {i}"
            b = C.c_uint64()
            A.check(A.lib().av1pf_ctx_memory(c.p, C.byref(b)))
            held[n] = b.value
        finally:
            c.close()
    # every slot is sized for the same frames, so the difference is a whole number of slots
    diff = held[threads] - held[0]
    assert (diff > 0) == (threads > 3) and (diff < 0) == (threads < 3)
    slot = abs(diff) // abs(threads - 3)
    assert slot > 0 and abs(diff) == slot * abs(threads - 3)


def test_set_threads_rejects_negative(ctx):
    assert A.lib().av1pf_set_threads(ctx.p, -1) == A.ERR_INVALID_INPUT
    A.check(A.lib().av1pf_set_threads(ctx.p, 64))  # above 8 means 8
    A.check(A.lib().av1pf_set_threads(ctx.p, 0))
