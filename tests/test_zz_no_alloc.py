"""av1pf_output_noalloc: the output stage (film grain + crop + packing) for
callers that cannot let the library allocate device memory — for example a
decoder inside a host whose device memory belongs to another allocator, or a
real-time output path that cannot risk an allocation failing mid-stream.
Its scratch is a fixed array inside the library instead of context memory.

Checked through the C ABI against the regular entry point (av1pf_output) and
the oracle's output process, bit for bit, on calls in a row that reuse the
shared array — including a frame at the array's limit (8192x8192 with film
grain: exactly 65,536 block offsets, and a work list that needs taller
tiles) — and for a clean refusal of frames beyond that limit. A CPU test
checks that the entry point's source calls no allocating routine. This file
is collected last so a failure here leaves every other test already run.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available

if cuda_available():
    import gpu_util as G
    import torch

CASES = [
    dict(width=330, height=210, bit_depth=10, enable_grain=1, seed=10, frame_index=3),
    dict(width=288, height=150, bit_depth=12, subsampling_x=0, subsampling_y=0, superres_denom=13, enable_grain=1,
         seed=9, frame_index=7),
    dict(width=300, height=170, bit_depth=8, sample_bytes=1, enable_grain=0, seed=11),
    dict(width=260, height=140, bit_depth=10, subsampling_x=1, subsampling_y=0, enable_grain=1, seed=12),
    # the limit: ceil(8192/32)^2 = 65,536 block offsets; 12,288 32-row output items exceed the fixed
    # work list, so the tiles are 64 rows tall
    dict(width=8192, height=8192, bit_depth=10, enable_grain=1, enable_lr=0, seed=21, frame_index=2),
]


def _frame(sf):
    """Device reference-frame planes (the synthetic planes stand in for an
    LR frame) and a packed-output buffer."""
    info = sf.f.info
    d_ref = G.DevPlanes.from_host(info, O.HostPlanes.like_synth(sf))
    return d_ref, G.dev_bytes(A.frame_bytes(info))


def _regular_output(ctx, sf, d_ref):
    info = sf.f.info
    fb = G.dev_bytes(A.frame_bytes(info))
    A.check(A.lib().av1pf_output(ctx.p, C.byref(info), C.byref(sf.f.params), d_ref.c, fb.data_ptr(), None))
    torch.cuda.synchronize()
    return fb[: A.frame_bytes(info)].cpu().numpy()


def _oracle_output(sf):
    info = sf.f.info
    fb = np.zeros(A.frame_bytes(info), np.uint8)
    assert O.lib().oracle_output(C.byref(info), C.byref(sf.f.params), O.HostPlanes.like_synth(sf).c,
                                 fb.ctypes.data) == 0
    return fb


def test_no_alloc_source_calls_no_allocator():
    """The entry point's file allocates nothing: no cudaMalloc/cudaFree of
    any kind, no context buffer, no torch."""
    src = open(os.path.join(os.path.dirname(__file__), "..", "rivet-av1_b200", "csrc", "noalloc.cu")).read()
    code = "\n".join(line.split("//")[0] for line in src.splitlines())  # comments may name them
    for pat in (r"cudaMalloc\w*", r"cudaFree\w*", r"\bcuMem\w*", r"\bensure\(", r"\bnew\b", r"\bmalloc\(",
                r"torch"):
        assert not re.search(pat, code), f"noalloc.cu calls {pat}"


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_no_alloc_output_matches_regular_output_on_calls_in_a_row():
    ctx = G.Ctx()
    sfs = [A.SynthHandle(**kw) for kw in CASES]
    frames = [_frame(sf) for sf in sfs]
    want = [_regular_output(ctx, sf, d_ref) for sf, (d_ref, _) in zip(sfs, frames)]
    for i, sf in enumerate(sfs):
        assert np.array_equal(want[i], _oracle_output(sf)), f"case {i}: av1pf_output differs from the oracle"
    L = A.lib()
    free_after_first = None
    # two passes over all cases: every call after the first reuses the array
    for rnd in range(2):
        for i, (sf, (d_ref, fb)) in enumerate(zip(sfs, frames)):
            fb.fill_(0xAB)
            rc = L.av1pf_output_noalloc(C.byref(sf.f.info), C.byref(sf.f.params), d_ref.c, fb.data_ptr(), None)
            assert rc == A.OK, L.av1pf_last_error()
            torch.cuda.synchronize()
            got = fb[: A.frame_bytes(sf.f.info)].cpu().numpy()
            assert np.array_equal(got, want[i]), f"round {rnd} case {i}: differs from av1pf_output"
            free = torch.cuda.mem_get_info()[0]
            if free_after_first is None:
                free_after_first = free
            else:
                assert free == free_after_first, "device memory changed across no-allocation calls"
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_no_alloc_refuses_frames_beyond_its_limit():
    sf = A.SynthHandle(width=64, height=64, bit_depth=10, enable_grain=1, enable_lr=0, seed=3)
    d_ref, fb = _frame(sf)
    info = A.FrameInfo.from_buffer_copy(sf.f.info)
    info.upscaled_width = info.frame_width = 16384
    info.frame_height = 16384
    info.mi_cols = 2 * ((16384 + 7) >> 3)
    info.mi_rows = 2 * ((16384 + 7) >> 3)
    rc = A.lib().av1pf_output_noalloc(C.byref(info), C.byref(sf.f.params), d_ref.c, fb.data_ptr(), None)
    assert rc == A.ERR_UNSUPPORTED
    assert b"too large" in A.lib().av1pf_last_error()
