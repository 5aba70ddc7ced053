"""Device reference slots (av1pf_refs_*): the reference frame update process
of 7.20 (decoder/mod.rs:797-806) over frames the chain leaves on the device,
and show_existing_frame (decoder/mod.rs:819-842).

A sequence of frames with different refresh_frame_flags goes through
av1pf_refs_chain; after each call every slot must hold the frame the
reference's update would have put there (tracked here in Python), with its
samples equal bit for bit to the oracle's loop-restoration output of that
frame. Slots that share a frame share its planes, frames no slot holds are
reused, and show_existing_frame outputs a slot's frame as the oracle's
output process does.
"""
import ctypes as C

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G
    import torch


@pytest.fixture(scope="module")
def ctx():
    c = G.Ctx()
    yield c
    c.close()


def packed(info, planes_ptr_array, ctx, params=None):
    """A frame's planes as the packed output frame (film grain off unless
    `params` applies it), read back from the device."""
    if params is None:
        params = A.Params()
    fb = G.dev_bytes(A.frame_bytes(info))
    A.check(A.lib().av1pf_output(ctx.p, C.byref(info), C.byref(params), planes_ptr_array, fb.data_ptr(), None),
            "output")
    torch.cuda.synchronize()
    return fb[: A.frame_bytes(info)].cpu().numpy()


def oracle_ref_packed(sf):
    """The oracle's loop-restoration output of `sf`, packed without grain."""
    ref, _ = O.chain(sf, threads=0)
    info = sf.f.info
    fb = np.zeros(A.frame_bytes(info), np.uint8)
    assert O.lib().oracle_output(C.byref(info), C.byref(A.Params()), ref.c, fb.ctypes.data) == 0
    return fb


def get(refs, slot):
    r = A.RefFrame()
    A.check(A.lib().av1pf_refs_get(refs, slot, C.byref(r)), "refs_get")
    return r


def test_refresh_sequence_matches_the_update_process(ctx):
    L = A.lib()
    refs = C.c_void_p()
    A.check(L.av1pf_refs_create(ctx.p, C.byref(refs)), "refs_create")
    try:
        # key frame (all slots), then inter frames refreshing various slots; the
        # 6th frame changes shape (a larger frame of the same stream)
        flags = [0xFF, 0x01, 0x06, 0x00, 0x81, 0x10, 0x7E]
        cfgs = [dict(width=320, height=200, bit_depth=10, seed=60 + k, frame_index=k) for k in range(len(flags))]
        cfgs[5] = dict(width=400, height=232, bit_depth=10, seed=65, frame_index=5)
        sfs = [A.SynthHandle(**c) for c in cfgs]
        want = [oracle_ref_packed(sf) for sf in sfs]
        held = [None] * 8  # frame index per slot, as the update process leaves it
        peak = 0  # frames the pool needs: the most held at once when a frame is made, plus that one
        for k, (sf, fl) in enumerate(zip(sfs, flags)):
            peak = max(peak, len({h for h in held if h is not None}) + 1)
            df = G.DevFrame(sf)
            fb = G.dev_bytes(A.frame_bytes(sf.info))
            A.check(L.av1pf_refs_chain(refs, C.byref(sf.f.info), C.byref(sf.f.params), C.byref(df.maps), df.inp.c, fl,
                                       100 + k, fb.data_ptr(), None), "refs_chain")
            torch.cuda.synchronize()
            # the packed output is the chain's own
            assert np.array_equal(fb[: A.frame_bytes(sf.info)].cpu().numpy(), O.chain(sf, threads=0)[1])
            for i in range(8):
                if (fl >> i) & 1:
                    held[i] = k
            ptrs = {}
            for i in range(8):
                r = get(refs, i)
                if held[i] is None:
                    assert r.valid == 0
                    continue
                j = held[i]
                assert r.valid == 1 and r.frame_id == j + 1 and r.order_hint == 100 + j, f"after frame {k} slot {i}"
                assert (r.info.upscaled_width, r.info.frame_height) == (sfs[j].info.upscaled_width,
                                                                        sfs[j].info.frame_height)
                got = packed(r.info, r.planes, ctx)
                assert np.array_equal(got, want[j]), f"after frame {k}: slot {i} (frame {j}) samples"
                ptrs.setdefault(j, set()).add(r.planes[0].data)
            # slots holding one frame share its planes
            assert all(len(v) == 1 for v in ptrs.values())
            # a frame no slot holds goes back to the pool and is reused: the
            # table has never made more frames than were held at once plus
            # the one being made
            b, n = C.c_uint64(), C.c_int32()
            A.check(L.av1pf_refs_memory(refs, C.byref(b), C.byref(n)), "refs_memory")
            assert n.value <= peak, f"after frame {k}: {n.value} frames made, {peak} needed"
        # show_existing_frame of slot 1 with film grain: the output process on that frame
        r1 = get(refs, 1)
        sf = sfs[held[1]]
        gp = A.Params.from_buffer_copy(A.SynthHandle(width=320, height=200, bit_depth=10, enable_grain=1, seed=77,
                                                     frame_index=9).f.params)
        fb = G.dev_bytes(A.frame_bytes(r1.info))
        A.check(L.av1pf_refs_show(refs, 1, C.byref(gp), 0, fb.data_ptr(), None), "refs_show")
        torch.cuda.synchronize()
        ref_cpu = O.chain(sf, threads=0)[0]
        want_show = np.zeros(A.frame_bytes(r1.info), np.uint8)
        assert O.lib().oracle_output(C.byref(sf.f.info), C.byref(gp), ref_cpu.c, want_show.ctypes.data) == 0
        assert np.array_equal(fb[: A.frame_bytes(r1.info)].cpu().numpy(), want_show)
        # a shown key frame refreshes every slot with it
        A.check(L.av1pf_refs_show(refs, 1, C.byref(A.Params()), 0xFF, fb.data_ptr(), None), "refs_show key")
        for i in range(8):
            assert get(refs, i).frame_id == r1.frame_id
    finally:
        A.check(L.av1pf_refs_destroy(refs), "refs_destroy")


def test_refs_reject_bad_arguments(ctx):
    L = A.lib()
    refs = C.c_void_p()
    A.check(L.av1pf_refs_create(ctx.p, C.byref(refs)), "refs_create")
    try:
        r = A.RefFrame()
        assert L.av1pf_refs_get(refs, 8, C.byref(r)) == A.ERR_INVALID_INPUT
        A.check(L.av1pf_refs_get(refs, 3, C.byref(r)))
        assert r.valid == 0
        fb = G.dev_bytes(1024)
        # show_existing_frame of an empty slot
        assert L.av1pf_refs_show(refs, 0, C.byref(A.Params()), 0, fb.data_ptr(), None) == A.ERR_INVALID_INPUT
        sf = A.SynthHandle(width=64, height=48, bit_depth=8, sample_bytes=1, seed=3)
        df = G.DevFrame(sf)
        assert L.av1pf_refs_chain(refs, C.byref(sf.f.info), C.byref(sf.f.params), C.byref(df.maps), df.inp.c, 0x100, 0,
                                  None, None) == A.ERR_INVALID_INPUT
    finally:
        A.check(L.av1pf_refs_destroy(refs), "refs_destroy")
