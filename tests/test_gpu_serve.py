"""The serving loop (continuous batching over many streams) through the C
ABI: every result equals the oracle's, a frame gives the same bytes alone and
in a mix of streams, admission refuses streams beyond the HBM cap, and bad
requests are rejected without touching the device."""
import ctypes as C
import threading

import numpy as np
import pytest

import av1pf as A
import oracle as O
from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

if cuda_available():
    import gpu_util as G

L = A.lib


def open_server(ctx, cap=40 << 30, max_batch=16, inflight=2):
    cfg = A.ServeConfig(cap, max_batch, inflight, 100)
    s = C.c_void_p()
    A.check(L().av1pf_serve_open(ctx.p, C.byref(cfg), C.byref(s)), "serve_open")
    return s


def request(sf, keep):
    inp = O.HostPlanes.like_synth(sf)
    keep.append(inp)
    r = A.Request()
    r.info = C.pointer(sf.f.info)
    r.params = C.pointer(sf.f.params)
    r.maps = C.pointer(sf.f.maps)
    r.inp = C.cast(inp.c, C.POINTER(A.Plane))
    return r


STREAMS = [dict(width=320, height=180, bit_depth=8, sample_bytes=1),
           dict(width=480, height=270, bit_depth=10),
           dict(width=256, height=144, bit_depth=12, subsampling_x=0, subsampling_y=0, superres_denom=12,
                enable_grain=1),
           dict(width=200, height=120, bit_depth=10, subsampling_x=1, subsampling_y=0, enable_grain=1)]


def test_serve_results_match_oracle_and_alone_equals_mix():
    ctx = G.Ctx()
    frames = {i: [A.SynthHandle(**cfg, seed=100 + 10 * i + k, frame_index=k) for k in range(3)]
              for i, cfg in enumerate(STREAMS)}
    want = {(i, k): O.chain(sf, threads=0)[1] for i in frames for k, sf in enumerate(frames[i])}
    keep = []
    # alone: one stream, one frame at a time
    srv = open_server(ctx)
    sid = C.c_int32()
    A.check(L().av1pf_serve_open_stream(srv, C.byref(frames[2][0].f.info), C.byref(sid)))
    t = C.c_uint64()
    A.check(L().av1pf_serve_submit(srv, sid.value, C.byref(request(frames[2][0], keep)), C.byref(t)))
    out_alone = np.zeros(A.frame_bytes(frames[2][0].f.info), np.uint8)
    lat = C.c_double()
    A.check(L().av1pf_serve_poll(srv, t.value, 10000, out_alone.ctypes.data, C.byref(lat)))
    A.check(L().av1pf_serve_close(srv))
    assert np.array_equal(out_alone, want[(2, 0)])
    # the mix: every stream, frames submitted from several threads at once
    srv = open_server(ctx, max_batch=8)
    sids = {}
    for i in frames:
        s = C.c_int32()
        A.check(L().av1pf_serve_open_stream(srv, C.byref(frames[i][0].f.info), C.byref(s)))
        sids[i] = s.value
    tickets = {}
    lock = threading.Lock()

    def submit(i):
        for rep in range(2):
            for k, sf in enumerate(frames[i]):
                tk = C.c_uint64()
                rq = request(sf, keep)
                A.check(L().av1pf_serve_submit(srv, sids[i], C.byref(rq), C.byref(tk)))
                with lock:
                    tickets[tk.value] = (i, k)
    th = [threading.Thread(target=submit, args=(i,)) for i in frames]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for tk, (i, k) in tickets.items():
        out = np.zeros(A.frame_bytes(frames[i][k].f.info), np.uint8)
        A.check(L().av1pf_serve_poll(srv, tk, 20000, out.ctypes.data, None), "poll")
        assert np.array_equal(out, want[(i, k)]), (i, k)
    st = A.ServeStats()
    A.check(L().av1pf_serve_stats_get(srv, C.byref(st)))
    assert st.completed == st.submitted == len(tickets)
    assert st.p99_ms >= st.p50_ms > 0
    assert st.batches >= 1 and st.mean_batch_frames >= 1
    A.check(L().av1pf_serve_close(srv))
    ctx.close()


def test_serve_admission_and_errors():
    ctx = G.Ctx()
    sf = A.SynthHandle(width=640, height=360, bit_depth=10, seed=3)
    srv = open_server(ctx, cap=4 << 20)  # 4 MiB: too small for one 360p stream's slots
    sid = C.c_int32()
    assert L().av1pf_serve_open_stream(srv, C.byref(sf.f.info), C.byref(sid)) == A.ERR_ADMISSION
    st = A.ServeStats()
    A.check(L().av1pf_serve_stats_get(srv, C.byref(st)))
    assert st.refused == 1
    A.check(L().av1pf_serve_close(srv))
    srv = open_server(ctx)
    A.check(L().av1pf_serve_open_stream(srv, C.byref(sf.f.info), C.byref(sid)))
    other = A.SynthHandle(width=320, height=180, bit_depth=10, seed=4)
    keep = []
    t = C.c_uint64()
    # geometry differing from the stream's
    assert L().av1pf_serve_submit(srv, sid.value, C.byref(request(other, keep)), C.byref(t)) == A.ERR_INVALID_INPUT
    assert L().av1pf_serve_submit(srv, 999, C.byref(request(sf, keep)), C.byref(t)) == A.ERR_NOT_FOUND
    assert L().av1pf_serve_poll(srv, 12345, 0, None, None) == A.ERR_NOT_FOUND
    A.check(L().av1pf_serve_submit(srv, sid.value, C.byref(request(sf, keep)), C.byref(t)))
    A.check(L().av1pf_serve_poll(srv, t.value, 10000, None, None))
    A.check(L().av1pf_serve_close_stream(srv, sid.value))
    assert L().av1pf_serve_close_stream(srv, sid.value) == A.ERR_NOT_FOUND
    A.check(L().av1pf_serve_close(srv))
    ctx.close()


def test_serve_close_stream_drops_unpolled_results():
    """A host request that completed but was not polled when its stream
    closed reports ERR_NOT_FOUND at poll instead of reading freed buffers;
    polls before the close still return the frame."""
    import time
    ctx = G.Ctx()
    srv = open_server(ctx)
    sf = A.SynthHandle(**STREAMS[0], seed=41)
    want = O.chain(sf, threads=0)[1]
    sid = C.c_int32()
    A.check(L().av1pf_serve_open_stream(srv, C.byref(sf.f.info), C.byref(sid)))
    keep = []
    t1, t2 = C.c_uint64(), C.c_uint64()
    A.check(L().av1pf_serve_submit(srv, sid.value, C.byref(request(sf, keep)), C.byref(t1)))
    A.check(L().av1pf_serve_submit(srv, sid.value, C.byref(request(sf, keep)), C.byref(t2)))
    out = np.zeros(A.frame_bytes(sf.f.info), np.uint8)
    A.check(L().av1pf_serve_poll(srv, t1.value, 10000, out.ctypes.data, None))
    assert np.array_equal(out, want)
    st = A.ServeStats()
    deadline = time.time() + 10
    while time.time() < deadline:
        A.check(L().av1pf_serve_stats_get(srv, C.byref(st)))
        if st.completed == 2:
            break
        time.sleep(0.01)
    assert st.completed == 2
    A.check(L().av1pf_serve_close_stream(srv, sid.value))
    assert L().av1pf_serve_poll(srv, t2.value, 0, out.ctypes.data, None) == A.ERR_NOT_FOUND
    A.check(L().av1pf_serve_close(srv))
    ctx.close()


def test_serve_device_resident_requests():
    """Frames already on the device (as a GPU decoder leaves them) are served
    in place into the caller's device outputs, bit-exact with the oracle."""
    import torch
    ctx = G.Ctx()
    srv = open_server(ctx)
    cases = [A.SynthHandle(**STREAMS[1], seed=70 + k, frame_index=k) for k in range(3)] + \
            [A.SynthHandle(**STREAMS[2], seed=80 + k, frame_index=k) for k in range(2)]
    sids = {}
    for sf in cases:
        key = (sf.info.upscaled_width, sf.info.bit_depth)
        if key not in sids:
            s = C.c_int32()
            A.check(L().av1pf_serve_open_stream(srv, C.byref(sf.f.info), C.byref(s)))
            sids[key] = s.value
    keep, tickets = [], []
    for sf in cases:
        df = G.DevFrame(sf)
        ref = G.DevPlanes.visible(sf.f.info)
        fb = G.dev_bytes(A.frame_bytes(sf.f.info))
        r = A.Request()
        r.info, r.params, r.maps = C.pointer(df.info), C.pointer(df.params), C.pointer(df.maps)
        r.inp = C.cast(df.inp.c, C.POINTER(A.Plane))
        r.device = 1
        r.ref_out = C.cast(ref.c, C.POINTER(A.Plane))
        r.frame_out = fb.data_ptr()
        keep.append((df, ref, fb, r))
        t = C.c_uint64()
        A.check(L().av1pf_serve_submit(srv, sids[(sf.info.upscaled_width, sf.info.bit_depth)], C.byref(r), C.byref(t)))
        tickets.append(t.value)
    for tk in tickets:
        A.check(L().av1pf_serve_poll(srv, tk, 20000, None, None))
    torch.cuda.synchronize()
    for sf, (df, ref, fb, r) in zip(cases, keep):
        ref_cpu, fb_cpu = O.chain(sf, threads=0)
        assert np.array_equal(fb[: A.frame_bytes(sf.f.info)].cpu().numpy(), fb_cpu)
        for p in range(sf.info.num_planes):
            assert np.array_equal(ref.host(p), ref_cpu.arrays[p])
    A.check(L().av1pf_serve_close(srv))
    ctx.close()


def test_serve_submit_many_group():
    """A group of frames queued at once (av1pf_serve_submit_many) comes back
    equal to the oracle, with 4 slots per stream letting ticks batch several
    frames of one stream; a group with one bad request queues nothing."""
    ctx = G.Ctx()
    frames = {i: [A.SynthHandle(**cfg, seed=300 + 10 * i + k, frame_index=k) for k in range(3)]
              for i, cfg in enumerate(STREAMS)}
    want = {(i, k): O.chain(sf, threads=0)[1] for i in frames for k, sf in enumerate(frames[i])}
    keep = []
    cfg = A.ServeConfig(40 << 30, 32, 2, 100, 4)
    srv = C.c_void_p()
    A.check(L().av1pf_serve_open(ctx.p, C.byref(cfg), C.byref(srv)), "serve_open")
    sids = {}
    for i in frames:
        s = C.c_int32()
        A.check(L().av1pf_serve_open_stream(srv, C.byref(frames[i][0].f.info), C.byref(s)))
        sids[i] = s.value
    order = [(i, k) for rep in range(2) for k in range(3) for i in frames]
    n = len(order)
    ids = (C.c_int32 * n)(*[sids[i] for i, _ in order])
    reqs = (A.Request * n)(*[request(frames[i][k], keep) for i, k in order])
    tks = (C.c_uint64 * n)()
    A.check(L().av1pf_serve_submit_many(srv, n, ids, reqs, tks), "submit_many")
    assert len(set(tks)) == n
    for t, (i, k) in zip(tks, order):
        out = np.zeros(A.frame_bytes(frames[i][k].f.info), np.uint8)
        A.check(L().av1pf_serve_poll(srv, t, 20000, out.ctypes.data, None), "poll")
        assert np.array_equal(out, want[(i, k)]), (i, k)
    st = A.ServeStats()
    A.check(L().av1pf_serve_stats_get(srv, C.byref(st)))
    assert st.completed == st.submitted == n
    # all or nothing: an unknown stream in the group refuses the whole group
    bad = (C.c_int32 * 2)(sids[0], 999)
    reqs2 = (A.Request * 2)(request(frames[0][0], keep), request(frames[0][1], keep))
    tks2 = (C.c_uint64 * 2)()
    assert L().av1pf_serve_submit_many(srv, 2, bad, reqs2, tks2) == A.ERR_NOT_FOUND
    A.check(L().av1pf_serve_stats_get(srv, C.byref(st)))
    assert st.submitted == n
    A.check(L().av1pf_serve_close(srv))
    ctx.close()
