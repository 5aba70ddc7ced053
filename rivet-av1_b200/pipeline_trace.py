"""Trace of the pipelined host-buffer entry point (a profiling aid).

Loads the tracing build of the library (`make -C rivet-av1_b200 trace`
makes libav1pf_trace.so, in which av1pf_chain_host_many records CUDA events
around each frame's upload, chain, download and descriptor upload, and host
timestamps of its enqueue steps), runs `--frames` frames of one workload
from pinned host memory in one av1pf_chain_host_many call after a warm-up,
and prints per frame when each step ran on its stream (us from frame 0's
upload start) and when the host queued it, then the mean step times over
the frames past the pipeline's fill.

    python rivet-av1_b200/pipeline_trace.py [--width 1920 --height 1080 --bit-depth 10] [--frames 64]
"""
import argparse
import ctypes as C
import os
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
sys.path[:0] = [PKG, os.path.join(ROOT, "tests")]

import av1pf as A  # noqa: E402


def pinned_planes(torch, sf):
    """Pinned copies of a synthetic frame's pre-filter planes, as av1pf_plane."""
    f = sf.f
    sb = 2 if f.info.sample_bytes == 2 else 1
    keep, planes = [], (A.Plane * 3)()
    for p in range(f.info.num_planes):
        pl = f.planes[p]
        n = pl.height * pl.stride * sb
        t = torch.frombuffer((C.c_uint8 * n).from_address(pl.data), dtype=torch.uint8).clone().pin_memory()
        keep.append(t)
        planes[p].data = t.data_ptr()
        planes[p].stride, planes[p].width, planes[p].height = pl.stride, pl.width, pl.height
    return planes, keep


def pinned_maps(torch, sf):
    """Pinned copies of a synthetic frame's maps."""
    f = sf.f
    keep = []

    def pin(ptr, n):
        t = torch.frombuffer((C.c_uint8 * n).from_address(ptr), dtype=torch.uint8).clone().pin_memory()
        keep.append(t)
        return t.data_ptr()
    m = A.Maps()
    m.mi_stride, m.cdef_stride = f.maps.mi_stride, f.maps.cdef_stride
    m.mi = pin(f.maps.mi, f.mi_count * 8)
    for p in range(3):
        if f.maps.lf_tx_size[p]:
            m.lf_tx_size[p] = pin(f.maps.lf_tx_size[p], f.tx_count[p])
        if f.maps.lr_units[p] and f.lr_count[p]:
            m.lr_units[p] = pin(f.maps.lr_units[p], f.lr_count[p] * C.sizeof(A.LrUnit))
    m.cdef_idx = pin(f.maps.cdef_idx, f.cdef_count)
    return m, keep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--bit-depth", type=int, default=10)
    ap.add_argument("--frames", type=int, default=64)
    args = ap.parse_args()
    lib_path = os.path.join(PKG, "libav1pf_trace.so")
    if not os.path.exists(lib_path):
        sys.exit("libav1pf_trace.so is missing: make -C rivet-av1_b200 trace")
    A.LIB_PATH = lib_path
    import torch
    import gpu_util as G
    L = A.lib()
    L.av1pf_trace_pipeline.restype = C.c_int
    L.av1pf_trace_pipeline.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_double), C.c_int]
    cfg = dict(width=args.width, height=args.height, bit_depth=args.bit_depth)
    if args.bit_depth == 8:
        cfg["sample_bytes"] = 1
    ctx = G.Ctx(0)
    pool = 16
    sfs = [A.SynthHandle(**cfg, seed=100 + i) for i in range(pool)]
    hosts = []
    for sf in sfs:
        planes, k1 = pinned_planes(torch, sf)
        maps, k2 = pinned_maps(torch, sf)
        fb = torch.empty(A.frame_bytes(sf.f.info), dtype=torch.uint8).pin_memory()
        hosts.append((sf, planes, maps, fb, k1 + k2))
    n = args.frames
    jobs = (A.HostJob * n)()
    for i in range(n):
        sf, planes, maps, fb, _ = hosts[i % pool]
        jobs[i].info = C.pointer(sf.f.info)
        jobs[i].params = C.pointer(sf.f.params)
        jobs[i].maps = C.pointer(maps)
        jobs[i].inp = C.cast(planes, C.POINTER(A.Plane))
        jobs[i].ref_out = None
        jobs[i].frame_out = fb.data_ptr()
    for _ in range(3):
        A.check(L.av1pf_chain_host_many(ctx.p, n, jobs), "chain_host_many")
    dev = (C.c_float * (8 * n))()
    host = (C.c_double * (4 * n))()
    m = L.av1pf_trace_pipeline(dev, host, n)
    print(f"{m} frames of {args.width}x{args.height} {args.bit_depth}-bit through av1pf_chain_host_many")
    print("frame | upload | chain | download | descriptors (us on their streams) | host: begun, upload, chain, "
          "download queued (us)")
    for k in range(m):
        d = [dev[8 * k + j] for j in range(8)]
        h = [host[4 * k + j] for j in range(4)]
        print(f"{k:3d} | {d[0]:8.1f}-{d[1]:8.1f} | {d[2]:8.1f}-{d[3]:8.1f} | {d[4]:8.1f}-{d[5]:8.1f} | "
              f"{d[6]:8.1f}-{d[7]:8.1f} | " + " ".join(f"{x:8.1f}" for x in h))
    past = range(min(8, m - 1), m)
    mean = lambda a, b: sum(dev[8 * k + b] - dev[8 * k + a] for k in past) / len(past)  # noqa: E731
    period = (dev[8 * (m - 1)] - dev[8 * past[0]]) / max(1, m - 1 - past[0])
    print(f"frames {past[0]}..{m - 1}: upload {mean(0, 1):.1f} us, chain {mean(2, 3):.1f} us (from its stream "
          f"waits), download {mean(4, 5):.1f} us, descriptors {mean(6, 7):.1f} us; upload starts "
          f"{period:.1f} us apart")
    ctx.close()


if __name__ == "__main__":
    main()
