"""Per-CTA timeline of back-to-back chain calls (a profiling aid).

Loads the tracing build of the library (`make -C rivet-av1_b200 trace` makes
libav1pf_trace.so: the stage kernels record each CTA's start and end by
%globaltimer, its SM and block), runs `--frames` chains of one workload back
to back on distinct frames after a warm-up, and prints:
  - per frame, each stage kernel's first CTA start, last CTA end (us, from
    the first frame's start), its CTA count and median CTA duration;
  - the frame period over the middle frames;
  - the CTAs resident per stage in 2-us bins across one frame.

    python rivet-av1_b200/timeline.py [--width 1920 --height 1080 --bit-depth 10] [--grain] [--frames 12]
"""
import argparse
import ctypes as C
import os
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
sys.path[:0] = [PKG, os.path.join(ROOT, "tests")]

import av1pf as A  # noqa: E402

KERNELS = {1: "loop_filter", 2: "cdef", 3: "loop_restoration", 4: "output", 5: "superres", 6: "grain_templates"}
CAP = 65536


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--bit-depth", type=int, default=10)
    ap.add_argument("--grain", action="store_true")
    ap.add_argument("--frames", type=int, default=12)
    args = ap.parse_args()
    lib_path = os.path.join(PKG, "libav1pf_trace.so")
    if not os.path.exists(lib_path):
        sys.exit("libav1pf_trace.so is missing: make -C rivet-av1_b200 trace")
    A.LIB_PATH = lib_path
    import torch
    import gpu_util as G
    L = A.lib()
    L.av1pf_trace_read.restype = C.c_int
    L.av1pf_trace_read.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_uint)]
    cfg = dict(width=args.width, height=args.height, bit_depth=args.bit_depth, enable_grain=int(args.grain))
    if args.bit_depth == 8:
        cfg["sample_bytes"] = 1
    ctx = G.Ctx(0)
    pool = 8
    sfs = [A.SynthHandle(**cfg, seed=40 + i, frame_index=3 + i) for i in range(pool)]
    dfs = [G.DevFrame(s) for s in sfs]
    outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]

    def run(i):
        d = dfs[i % pool]
        r, fb = outs[i % pool]
        A.check(L.av1pf_chain(ctx.p, C.byref(d.info), C.byref(d.params), C.byref(d.maps), d.inp.c, r.c,
                              fb.data_ptr(), None))

    buf = (C.c_ulonglong * (3 * CAP))()
    n = C.c_uint()
    for i in range(30):
        run(i)
    torch.cuda.synchronize()
    L.av1pf_trace_read(buf, C.byref(n))  # clears the warm-up's records
    nf = args.frames
    for i in range(nf):
        run(i)
    torch.cuda.synchronize()
    A.check(L.av1pf_trace_read(buf, C.byref(n)), "trace read")
    m = min(n.value, CAP)
    recs = [(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2] >> 40) for i in range(m)]
    t0 = min(r[0] for r in recs)
    by_kernel = {}
    for r in recs:
        by_kernel.setdefault(r[2], []).append(r)
    spans = [dict() for _ in range(nf)]
    for k, rs in by_kernel.items():
        rs.sort(key=lambda r: r[0])
        per = len(rs) // nf
        for f in range(nf):
            ch = rs[f * per:(f + 1) * per]
            durs = sorted(r[1] - r[0] for r in ch)
            spans[f][KERNELS.get(k, str(k))] = (min(r[0] for r in ch) - t0, max(r[1] for r in ch) - t0, per,
                                                durs[len(durs) // 2])
    print(f"{m} CTA records, {nf} frames of {args.width}x{args.height} {args.bit_depth}-bit"
          f"{' with film grain' if args.grain else ''}")
    print("frame | stage: first start - last end (us), CTAs, median CTA us")
    for f in range(nf):
        parts = [f"{k}: {v[0] / 1e3:.1f}-{v[1] / 1e3:.1f}, {v[2]}, {v[3] / 1e3:.2f}"
                 for k, v in sorted(spans[f].items(), key=lambda x: x[1][0])]
        print(f"{f} | " + " | ".join(parts))
    first = min(spans[0], key=lambda k: spans[0][k][0])
    lo, hi = spans[2][first][0], spans[nf - 2][first][0]
    print(f"frame period over frames 2..{nf - 2}: {(hi - lo) / (nf - 4) / 1e3:.2f} us")
    # resident CTAs per stage in 2-us bins across frame 3
    a, b = spans[3][first][0], spans[4][first][0]
    bins = {}
    for r in recs:
        s0, s1 = max(r[0] - t0, a), min(r[1] - t0, b)
        for u in range(int((s0 - a) // 2000), int((s1 - a) // 2000) + 1):
            if 0 <= u * 2000 < b - a:
                name = KERNELS.get(r[2], str(r[2]))
                bins.setdefault(u, {}).setdefault(name, 0)
                bins[u][name] += 1
    print("us from frame 3's start | resident CTAs per stage (touching the 2-us bin)")
    for u in sorted(bins):
        print(f"{2 * u:4d} | " + ", ".join(f"{k} {v}" for k, v in sorted(bins[u].items())))
    ctx.close()


if __name__ == "__main__":
    main()
