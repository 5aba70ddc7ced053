#!/usr/bin/env python3
"""Benchmark of the B200 AV1 post-filter chain (loop filter -> CDEF ->
superres -> loop restoration -> film grain / output packing).

Metric: bit-exact post-filtered Mpx/s (luma pixels upscaled_width x
frame_height per frame, the reference's decbench convention,
examples/av1_decbench.rs:38-50).

Headline workload (one step = one frame through the chain): a single
1920x1080 10-bit 4:2:0 frame of seeded synthetic filter-stage input (low-
frequency field + steps on the transform grid + noise sigma 8; random
partitions, transform sizes, loop-filter levels U[0,63], sharpness U[0,7],
8 CDEF presets, 64x64 LR units of Wiener / self-guided). Steps rotate over
a pool of distinct frames whose inputs total more than twice the 126 MB L2,
so no step starts with its input in L2.

The same run reports, beside the headline:
  e2e          the same metric through the host-buffer entry point from
               pinned host memory (input planes + maps up, packed frame down,
               per step): av1pf_chain_host_many, 64 frames per call (16 pinned
               frames in turn), whose copies overlap the chains; the single-frame synchronous
               av1pf_chain_host latency beside it;
  stages       per-stage device time (CUDA events on the chain's stream);
  roofline     the dominant stage's algorithmic bytes / its event time;
  mix          the batched path (one launch per stage for 64 mixed frames,
               replayed from a CUDA graph) against the per-frame GPU path
               on the same frames, outputs compared bit for bit;
  c3_4k        4K chains with superres + film grain (10-bit 4:2:0, 12-bit 4:4:4);
  serve        continuous-batching server: 32 streams, p50/p99 latency;
  search       the encoder's filter searches (CDEF strengths, fast and
               thorough lists; loop-filter levels) per 1080p / 4K frame,
               against the oracle's time for the same call;
  cpu_baseline the CPU oracle (this repo's C++ restatement of the reference's
               filters, all host threads) on a bounded sample.

Multi-GPU (torchrun): replicas only — each rank runs its own frames, no
collective on the data path; value = all ranks' pixels / max-over-ranks time.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "rivet-av1_b200"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import av1pf as A  # noqa: E402

METRIC = "bit-exact post-filtered Mpx/s"
HEADLINE = dict(width=1920, height=1080, bit_depth=10)
L2_BYTES = 126 * 2**20
HEADLINE_WORKLOAD = "1920x1080 10-bit 4:2:0 single-frame post-filter chain (LF+CDEF+LR+pack)"
# Per launch of each stage's kernels on the headline workload, from one ncu capture of the headline
# bench (profiles/metrics_1080p10_chain.md gives the command): DRAM bytes read and written
# (dram__bytes_read.sum, dram__bytes_write.sum) and warp-instructions executed
# (smsp__inst_executed.sum). ncu flushes the caches before a captured launch, so the reads are cold;
# a frame's 6-19 MB of writes stay in the 126 MB L2 when the launch ends, so the writes read near 0
# (they reach DRAM later, during the next launches). The headline frames have no film grain: the
# loop-restoration kernel packs them and no output kernel runs.
NCU_HEADLINE = {
    "loop_filter": {"dram_read": 8345344, "dram_write": 0, "warp_inst": 10128792},  # lf_fused_kernel (mode 3)
    "cdef": {"dram_read": 6999808, "dram_write": 0, "warp_inst": 16245271},
    "loop_restoration": {"dram_read": 8367872, "dram_write": 13312, "warp_inst": 14475086},
}
B200_SMS, ISSUE_PER_SM_CLK = 148, 4  # four schedulers per SM, one warp-instruction each per clock


def traffic_of(stage):
    n = NCU_HEADLINE.get(stage)
    return None if n is None else n["dram_read"] + n["dram_write"]


def issue_fractions(stage_ms, frame_ms, clocks):
    """The bound that binds this path: warp-instructions issued per stage
    (ncu, per launch) over what the SMs can issue in the stage's measured
    time at the sampled SM clock (148 SMs x 4 per clock)."""
    mhz = clocks.get("sm_mhz") or 1965.0
    per_ms = B200_SMS * ISSUE_PER_SM_CLK * mhz * 1e3  # warp-instructions per ms
    out = {"sm_mhz": mhz, "source": "smsp__inst_executed.sum per launch (ncu) / (148 x 4 x SM clock x time)"}
    total = 0
    for stage, n in NCU_HEADLINE.items():
        total += n["warp_inst"]
        if stage_ms.get(stage):
            out[stage] = round(n["warp_inst"] / (per_ms * stage_ms[stage]), 4)
    out["chain"] = round(total / (per_ms * frame_ms), 4)
    out["warp_inst_per_frame"] = total
    return out


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def plane_set_bytes(info, upscaled=True):
    """S: visible plane-set bytes at the native sample width."""
    w = info.upscaled_width if upscaled else info.frame_width
    n = 0
    for p in range(info.num_planes):
        sx = info.subsampling_x if p else 0
        sy = info.subsampling_y if p else 0
        n += ((w + sx) >> sx) * ((info.frame_height + sy) >> sy)
    return n * (2 if info.bit_depth > 8 else 1)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


# ---------------------------------------------------------------------------
# reference arm: the CPU implementation of the path (the oracle port)
# ---------------------------------------------------------------------------
def cpu_rate(cfgs, budget_s, threads=0):
    """Mpx/s of the CPU oracle over the frames of `cfgs` (cycled) for about
    budget_s seconds of work; returns (Mpx/s, frames, seconds, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sfs = [A.SynthHandle(**c) for c in cfgs]
    cores = os.cpu_count() if threads == 0 else threads
    t0 = time.perf_counter()
    px = 0
    n = 0
    while True:
        sf = sfs[n % len(sfs)]
        O.chain(sf, threads=threads)
        px += sf.info.upscaled_width * sf.info.frame_height
        n += 1
        el = time.perf_counter() - t0
        if (el >= budget_s and n >= 2) or el > 3 * budget_s:
            break
    return px / el / 1e6, n, el, cores


CPU_SEEDS = [1000 + i for i in range(4)]  # the CPU legs' frames (both arms time the same sample)


def headline_config(world):
    """The workload's `config`, identical in both arms' lines."""
    probe = A.SynthHandle(**HEADLINE, seed=1)
    in_bytes = sum(probe.f.plane_bytes[p] for p in range(3))
    pool_n = max(8, int(2 * L2_BYTES / in_bytes) + 1)
    return {"workload": HEADLINE_WORKLOAD, "frames_per_step": 1, "pool_frames": pool_n,
            "l2": f"inputs rotate over {pool_n} distinct frames ({pool_n * in_bytes / 2**20:.0f} MiB > 2x L2)",
            "parallelism": f"replicas x{world}"}, pool_n, in_bytes


def reference_arm(args):
    """The reference's CPU implementation of the path (the oracle port, all
    host threads) on the headline workload: rank 0 alone; the other ranks
    exit without work. The sample is time-bounded like the cpu_baseline leg
    of the GPU arm (at least args.cpu_seconds of frames, rotating over the
    same 4 seeded frames), after the warm-up frames."""
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    config, _, _ = headline_config(world)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sfs = [A.SynthHandle(**HEADLINE, seed=s) for s in CPU_SEEDS]
    for i in range(args.warmup):
        O.chain(sfs[i % len(sfs)], threads=0)
    budget = max(args.cpu_seconds, 1.0)
    rate, n, el, cores = cpu_rate([dict(HEADLINE, seed=s) for s in CPU_SEEDS], budget)
    ms_frame = 1e3 * el / n
    line = {
        "impl": "reference", "metric": METRIC, "value": round(rate, 3), "unit": "Mpx/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_frame, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": config,
        "cpu_baseline": {"value": round(rate, 3), "unit": "Mpx/s", "cores": cores, "kind": "port",
                         "sample": f"{n} frames of the workload in {el:.1f} s (4 seeded frames in turn) after "
                                   f"{args.warmup} warm-up frames, CPU oracle on all host threads"},
        "e2e": {"value": round(rate, 3), "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def main_gpu(args):
    import torch
    import gpu_util as G
    import replica as R
    ranks = R.Ranks()
    rank, world, local = ranks.rank, ranks.world, ranks.local
    torch.cuda.set_device(local)
    if args.only:
        ctx = G.Ctx(local)
        fn = {"mix": lambda: bench_mix(args, ctx, rank, torch.cuda.synchronize, lambda v: v),
              "c3": lambda: bench_4k(args, ctx, torch.cuda.synchronize, lambda v: v),
              "grain": lambda: bench_4k(args, ctx, torch.cuda.synchronize, lambda v: v, GRAIN_CASES),
              "serve": lambda: bench_serve(args, ctx, rank),
              "search": lambda: bench_search(args, ctx, rank, world)}[args.only]
        print(json.dumps({args.only: fn()}), flush=True)
        ctx.close()
        ranks.close()
        return 0
    L = A.lib()
    ctx = G.Ctx(local)
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    # ---- headline pool: distinct frames whose inputs exceed 2x L2 ----
    config, pool_n, in_bytes = headline_config(world)
    sfs = [A.SynthHandle(**HEADLINE, seed=R.frame_seed(rank, i)) for i in range(pool_n)]
    dfs = [G.DevFrame(s) for s in sfs]
    outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]

    def step(i):
        d = dfs[i % pool_n]
        r, fb = outs[i % pool_n]
        rc = L.av1pf_chain(ctx.p, C.byref(d.info), C.byref(d.params), C.byref(d.maps), d.inp.c, r.c,
                           fb.data_ptr(), None)
        if rc:
            A.check(rc, "av1pf_chain")

    # bit-exactness of the measured path: one pool frame against the oracle
    exact = None
    if rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        ref_cpu, fb_cpu = O.chain(sfs[0], threads=0)
        step(0)
        torch.cuda.synchronize()
        exact = bool(np.array_equal(outs[0][1][: A.frame_bytes(dfs[0].info)].cpu().numpy(), fb_cpu) and all(
            np.array_equal(outs[0][0].host(p), ref_cpu.arrays[p]) for p in range(3)))

    for i in range(args.warmup):
        step(i)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.5)  # let nvidia-smi start sampling before the timed region
    barrier()
    launches0 = L.av1pf_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step(args.warmup + i)
    e1.record()
    barrier()
    launches = L.av1pf_launch_count() - launches0
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    ms_max = max_over_ranks(ms)
    # stage times from a separate profiled pass (profiled calls launch stage by
    # stage with events between stages, not from the per-frame graph)
    L.av1pf_set_profiling(ctx.p, 1)
    ms5 = (C.c_float * 5)()
    calls = C.c_uint32()
    L.av1pf_stage_times(ctx.p, ms5, C.byref(calls))  # reset
    for i in range(min(args.steps, 400)):
        step(i)
    torch.cuda.synchronize()
    L.av1pf_stage_times(ctx.p, ms5, C.byref(calls))
    L.av1pf_set_profiling(ctx.p, 0)
    px_frame = 1920 * 1080
    value = R.aggregate_rate(world * args.steps * px_frame, ms_max) / 1e6
    stage_names = ["loop_filter", "cdef", "superres", "loop_restoration", "output"]
    stage_ms = {n: float(ms5[k]) / max(1, calls.value) for k, n in enumerate(stage_names)}

    # ---- roofline of the dominant stage ----
    info = dfs[0].info
    S = plane_set_bytes(info)
    # loop restoration reads the CDEF output and writes the reference frame
    # and (no film grain here) the packed frame
    algo = {"loop_filter": 2 * S, "cdef": 2 * S, "superres": 2 * S,
            "loop_restoration": 2 * S + A.frame_bytes(info), "output": 2 * S}
    dom = max(stage_ms, key=stage_ms.get)
    peak, peak_kind = peaks()
    achieved = algo[dom] / (stage_ms[dom] / 1e3) / 1e9
    chain_bytes = S + S + plane_set_bytes(info)  # input + reference frame + packed output
    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpx/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": config,
        "bit_exact_vs_oracle": exact,
        "gpu_launches": int(launches),
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "algorithmic_bytes": int(algo[dom]), "traffic": traffic_of(dom),
                     "traffic_note": "ncu dram read+write of one cold-cache launch; the launch's writes are "
                                     "still in L2 when it ends, so they are not counted",
                     "chain_frac": round(chain_bytes / (ms_max / args.steps / 1e3) / 1e9 / peak, 4),
                     "issue": issue_fractions(stage_ms, ms_max / args.steps, clocks)},
        "clocks": clocks,
    }

    # ---- e2e through the host-buffer entry point (pinned host memory) ----
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    hosts = []
    for s in sfs[: min(pool_n, 16)]:
        hp = O.HostPlanes.like_synth(s)
        pinned = [torch.from_numpy(a.view(np.uint8).reshape(-1)).pin_memory() for a in hp.arrays]
        planes = (A.Plane * 3)()
        for p, (a, t) in enumerate(zip(hp.arrays, pinned)):
            planes[p].data = t.data_ptr()
            planes[p].stride = a.shape[1]
            planes[p].width = a.shape[1]
            planes[p].height = a.shape[0]
        f = s.f
        m = A.Maps()
        m.mi_stride, m.cdef_stride = f.maps.mi_stride, f.maps.cdef_stride
        keep = []

        def pin(ptr, n):
            t = torch.from_numpy(np.frombuffer((C.c_uint8 * n).from_address(ptr), np.uint8).copy()).pin_memory()
            keep.append(t)
            return t.data_ptr()
        m.mi = pin(f.maps.mi, f.mi_count * 8)
        for p in range(3):
            if f.maps.lf_tx_size[p]:
                m.lf_tx_size[p] = pin(f.maps.lf_tx_size[p], f.tx_count[p])
            if f.maps.lr_units[p] and f.lr_count[p]:
                m.lr_units[p] = pin(f.maps.lr_units[p], f.lr_count[p] * 12)
        m.cdef_idx = pin(f.maps.cdef_idx, f.cdef_count)
        fb = torch.empty(A.frame_bytes(f.info), dtype=torch.uint8).pin_memory()
        hosts.append((s, pinned, planes, m, keep, fb))
    mi_rows = info.mi_rows
    h2d = sum(hosts[0][0].f.plane_bytes[p] for p in range(3)) + mi_rows * hosts[0][3].mi_stride * 8 + \
        sum((mi_rows >> (1 if p else 0)) * hosts[0][3].mi_stride for p in range(3)) + \
        ((mi_rows + 15) // 16) * hosts[0][3].cdef_stride + sum(hosts[0][0].f.lr_count[p] * 12 for p in range(3))
    d2h = A.frame_bytes(info)

    # the pipelined host entry point: each call takes 64 frames, the pinned
    # frames in turn (a call's pipeline fills and drains once, so longer
    # lists amortise that), and every frame's upload, chain and download
    # happen inside it
    group = 4 * len(hosts)
    hjobs = (A.HostJob * group)()
    for i in range(group):
        s, pinned, planes, m, keep, fb = hosts[i % len(hosts)]
        hjobs[i].info = C.pointer(s.f.info)
        hjobs[i].params = C.pointer(s.f.params)
        hjobs[i].maps = C.pointer(m)
        hjobs[i].inp = C.cast(planes, C.POINTER(A.Plane))
        hjobs[i].ref_out = None
        hjobs[i].frame_out = fb.data_ptr()

    def e2e_call():
        A.check(L.av1pf_chain_host_many(ctx.p, group, hjobs), "chain_host_many")

    e2e_calls = max(1, min(args.steps, 1000) // group)
    for i in range(max(1, args.warmup // group + 1)):
        e2e_call()
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_calls):
        e2e_call()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_steps = e2e_calls * group
    # the host path returns the same bytes as the device path
    e2e_exact = bool(np.array_equal(hosts[0][5].numpy(), outs[0][1][: A.frame_bytes(info)].cpu().numpy()))

    # one frame per synchronous av1pf_chain_host call: the latency of the drop-in
    def single_call(i):
        s, pinned, planes, m, keep, fb = hosts[i % len(hosts)]
        A.check(L.av1pf_chain_host(ctx.p, C.byref(s.f.info), C.byref(s.f.params), C.byref(m), planes, None,
                                   fb.data_ptr()), "chain_host")

    single_n = min(args.steps, 200)
    for i in range(args.warmup):
        single_call(i)
    t1 = time.perf_counter()
    for i in range(single_n):
        single_call(i)
    single_s = time.perf_counter() - t1
    result["e2e"] = {"value": round(world * e2e_steps * px_frame / e2e_s / 1e6, 2), "unit": "Mpx/s",
                     "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                     "ms_per_step": round(1e3 * e2e_s / e2e_steps, 3), "bit_exact_vs_device_path": e2e_exact,
                     "api": f"av1pf_chain_host_many, {group} frames per call ({len(hosts)} pinned frames in turn)",
                     "single_call": {"api": "av1pf_chain_host, one frame per call",
                                     "ms_per_frame": round(1e3 * single_s / single_n, 3),
                                     "mpx_s": round(single_n * px_frame / single_s / 1e6, 2)}}
    del hosts, hjobs

    # ---- batched vs per-frame on the mixed-resolution batch ----
    if not args.skip_extras:
        result["mix"] = bench_mix(args, ctx, rank, barrier, max_over_ranks)
        result["c3_4k"] = bench_4k(args, ctx, barrier, max_over_ranks)
        grain = bench_4k(args, ctx, barrier, max_over_ranks, GRAIN_CASES)
        for v in grain.values():
            v["vs_grain_free_headline"] = round(v["ms_per_frame"] / (ms_max / args.steps), 3)
        result["grain_1080p"] = grain
        result["serve"] = bench_serve(args, ctx, rank)
        result["search"] = bench_search(args, ctx, rank, world)

    # ---- CPU baseline (rank 0, N = 1) ----
    if rank == 0 and world == 1:
        rate, n, el, cores = cpu_rate([dict(HEADLINE, seed=s) for s in CPU_SEEDS], args.cpu_seconds)
        result["cpu_baseline"] = {"value": round(rate, 3), "unit": "Mpx/s", "cores": cores, "kind": "port",
                                  "sample": f"{n} frames of the headline workload in {el:.1f} s (4 seeded frames "
                                            f"in turn), CPU oracle on all host threads"}
    ctx.close()
    ranks.close()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


MIX = [(16, dict(width=640, height=360, bit_depth=8, sample_bytes=1)),
       (16, dict(width=960, height=540, bit_depth=8, sample_bytes=1)),
       (16, dict(width=1280, height=720, bit_depth=8, sample_bytes=1)),
       (12, dict(width=1920, height=1080, bit_depth=10)),
       (4, dict(width=3840, height=2160, bit_depth=10, subsampling_x=0, subsampling_y=0))]


def bench_mix(args, ctx, rank, barrier, max_over_ranks):
    """64 mixed frames: per-frame chain calls vs one batch replayed from a graph."""
    import torch
    import gpu_util as G
    L = A.lib()
    sfs = []
    k = 0
    for count, cfg in MIX:
        for _ in range(count):
            sfs.append(A.SynthHandle(**cfg, seed=5000 + 100 * rank + k, frame_index=k))
            k += 1
    dfs = [G.DevFrame(s) for s in sfs]
    out_a = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]
    out_b = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]
    px = sum(s.info.upscaled_width * s.info.frame_height for s in sfs)

    def per_frame():
        for d, (r, fb) in zip(dfs, out_a):
            A.check(L.av1pf_chain(ctx.p, C.byref(d.info), C.byref(d.params), C.byref(d.maps), d.inp.c, r.c,
                                  fb.data_ptr(), None))

    jobs = (A.Job * len(dfs))()
    for i, (d, (r, fb)) in enumerate(zip(dfs, out_b)):
        jobs[i].info = C.pointer(d.info)
        jobs[i].params = C.pointer(d.params)
        jobs[i].maps = C.pointer(d.maps)
        jobs[i].inp = C.cast(d.inp.c, C.POINTER(A.Plane))
        jobs[i].ref_out = C.cast(r.c, C.POINTER(A.Plane))
        jobs[i].frame_out = fb.data_ptr()
    # the autotuner picks the loop-filter mode and LR rectangle width per shape;
    # the per-frame calls and the batch both run on its choices
    n_shapes = C.c_int32()
    A.check(L.av1pf_autotune(ctx.p, jobs, len(dfs), 5, C.byref(n_shapes)), "autotune")
    tuned, seen = [], set()
    for d in dfs:
        i = d.info
        key = (i.upscaled_width, i.frame_height, i.bit_depth, i.subsampling_x, i.subsampling_y)
        if key in seen:
            continue
        seen.add(key)
        t, ms = A.Tuning(), C.c_float()
        A.check(L.av1pf_tuned_choice(ctx.p, C.byref(i), C.byref(t), C.byref(ms)), "tuned_choice")
        sub = "4:4:4" if not i.subsampling_x else ("4:2:2" if not i.subsampling_y else "4:2:0")
        tuned.append({"shape": f"{i.upscaled_width}x{i.frame_height} {i.bit_depth}-bit {sub}",
                      "lf_mode": t.lf_mode, "lr_rect_cols": t.lr_rect_cols, "frame_ms": round(ms.value, 4)})
    # the batch is tuned as a whole: each variant on every frame, and the per-shape choices
    b = C.c_void_p()
    A.check(L.av1pf_batch_create(ctx.p, jobs, len(dfs), A.BATCH_AUTOTUNE, C.byref(b)), "batch_create")

    def timed(fn, reps):
        for _ in range(max(1, args.warmup)):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)) / reps

    reps = max(3, min(20, args.steps // 4))
    t_pf = timed(per_frame, reps)
    t_b = timed(lambda: A.check(L.av1pf_batch_run(b, None)), reps)
    exact = all(np.array_equal(ra.host(p), rb.host(p)) and bool(torch.equal(fa, fb))
                for (ra, fa), (rb, fb), d in zip(out_a, out_b, dfs) for p in range(d.info.num_planes))
    A.lib().av1pf_batch_destroy(b)
    return {"frames": len(dfs), "mpx_per_batch": round(px / 1e6, 3),
            "per_frame_mpx_s": round(px / (t_pf / 1e3) / 1e6, 1), "batched_mpx_s": round(px / (t_b / 1e3) / 1e6, 1),
            "speedup": round(t_pf / t_b, 3), "per_frame_ms": round(t_pf, 3), "batched_ms": round(t_b, 3),
            "bit_exact_batched_vs_per_frame": bool(exact), "autotune": tuned}


C3_CASES = [("10bit_420_superres_grain", 3, dict(width=3840, height=2160, bit_depth=10, superres_denom=13,
                                                  enable_grain=1, seed=77, frame_index=3)),
            ("12bit_444_superres_grain", 3, dict(width=3840, height=2160, bit_depth=12, subsampling_x=0,
                                                  subsampling_y=0, superres_denom=10, enable_grain=1, seed=78,
                                                  frame_index=4))]
# the headline's shape with film grain: its inputs rotate over 20 frames (124 MB of input, plus outputs), so
# the comparison with the grain-free headline is not flattered by L2
GRAIN_CASES = [("1080p_10bit_420_grain", 20, dict(width=1920, height=1080, bit_depth=10, enable_grain=1, seed=79,
                                                  frame_index=5))]


def bench_4k(args, ctx, barrier, max_over_ranks, cases=C3_CASES):
    """Per-frame chains of `cases` (name, distinct frames, synthesis
    arguments): by default config 3's 4K chains with superres (denominator
    13 / 10) and film grain."""
    import torch
    import gpu_util as G
    L = A.lib()
    res = {}
    for name, pool, cfg in cases:
        sfs = [A.SynthHandle(**dict(cfg, seed=cfg["seed"] + i, frame_index=cfg["frame_index"] + i))
               for i in range(pool)]
        dfs = [G.DevFrame(s) for s in sfs]
        outs = [(G.DevPlanes.visible(d.info), G.dev_bytes(A.frame_bytes(d.info))) for d in dfs]

        def run(i):
            d = dfs[i % pool]
            r, fb = outs[i % pool]
            A.check(L.av1pf_chain(ctx.p, C.byref(d.info), C.byref(d.params), C.byref(d.maps), d.inp.c, r.c,
                                  fb.data_ptr(), None))
        for i in range(args.warmup):
            run(i)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(3, min(60, args.steps // 2))
        e0.record()
        for i in range(reps):
            run(i)
        e1.record()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1)) / reps
        # stage times from a profiled pass (stage by stage, events between)
        L.av1pf_set_profiling(ctx.p, 1)
        ms5 = (C.c_float * 5)()
        calls = C.c_uint32()
        L.av1pf_stage_times(ctx.p, ms5, C.byref(calls))
        for i in range(reps):
            run(i)
        torch.cuda.synchronize()
        L.av1pf_stage_times(ctx.p, ms5, C.byref(calls))
        L.av1pf_set_profiling(ctx.p, 0)
        info = dfs[0].info
        chain_bytes = plane_set_bytes(info, upscaled=False) + 2 * plane_set_bytes(info)
        peak, _ = peaks()
        res[name] = {"ms_per_frame": round(ms, 4), "frames": pool,
                     "mpx_s": round(info.upscaled_width * info.frame_height / (ms / 1e3) / 1e6, 1),
                     "chain_hbm_frac": round(chain_bytes / (ms / 1e3) / 1e9 / peak, 4),
                     "stages_ms": {n: round(float(ms5[k]) / max(1, calls.value), 4)
                                   for k, n in enumerate(["loop_filter", "cdef", "superres", "loop_restoration",
                                                          "output"])}}
    return res


def search_cpu(sf, cur, src, thorough, q, lam):
    """The oracle's CDEF and loop-filter searches on all host threads: the
    CPU leg of the search section (one call each; returns their ms and
    results)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    hc, hs = O.HostPlanes(cur), O.HostPlanes(src)
    t = time.perf_counter()
    res, table, _ = O.cdef_search(sf, hc, hs, q, lam, thorough)
    cdef_ms = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    levels, _ = O.lf_search(sf, hc, hs)
    lf_ms = (time.perf_counter() - t) * 1e3
    return cdef_ms, lf_ms, (res.pairs(), res.bits, table), levels


def bench_search(args, ctx, rank, world):
    """The encoder's filter searches (encoder/cdef.rs:52-251,
    encoder/mod.rs:1457-1506) on one frame per call: CDEF strength search
    with the fast and thorough candidate lists and the loop-filter level
    search, device-resident planes, host clock around each synchronous
    call; the oracle's time for the same call beside it (rank 0, N = 1)."""
    import gpu_util as G
    L = A.lib()
    res = {}
    q, lam = 120, 40.0
    for name, cfg in [("1080p_10bit", dict(width=1920, height=1080, bit_depth=10, seed=501)),
                      ("4k_10bit", dict(width=3840, height=2160, bit_depth=10, seed=502))]:
        sf = A.SynthHandle(**cfg)
        cur, src = A.synth_search_planes(sf, 7, amp=24)
        info = sf.f.info
        df = G.DevFrame(sf)
        dcur, dsrc = G.DevPlanes(info, [(a.shape[1], a.shape[0]) for a in cur], [a.shape[1] for a in cur]), \
            G.DevPlanes(info, [(a.shape[1], a.shape[0]) for a in src], [a.shape[1] for a in src])
        import torch
        for p in range(info.num_planes):
            dcur.t[p].copy_(torch.from_numpy(cur[p].view(np.uint8).reshape(-1)))
            dsrc.t[p].copy_(torch.from_numpy(src[p].view(np.uint8).reshape(-1)))
        fbr = (info.mi_rows + 15) // 16
        out = {}
        choice = {}
        for th in (0, 1):
            r = A.CdefSearchResult()
            table = np.zeros(fbr * df.maps.cdef_stride, np.int8)

            def run():
                A.check(L.av1pf_cdef_search(ctx.p, C.byref(info), C.byref(df.maps), dcur.c, dsrc.c, q, lam, th,
                                            C.byref(r), table.ctypes.data, None, None), "av1pf_cdef_search")
            for _ in range(max(3, args.warmup)):
                run()
            reps = 30
            t = time.perf_counter()
            for _ in range(reps):
                run()
            out["cdef_thorough_ms" if th else "cdef_fast_ms"] = round((time.perf_counter() - t) / reps * 1e3, 4)
            choice[th] = (r.pairs(), r.bits, table.copy())
        lv = (C.c_int32 * 4)()

        def runl():
            A.check(L.av1pf_lf_search(ctx.p, C.byref(info), C.byref(sf.f.params), C.byref(df.maps), dcur.c, dsrc.c,
                                      lv, None, None), "av1pf_lf_search")
        for _ in range(max(3, args.warmup)):
            runl()
        reps = 30
        t = time.perf_counter()
        for _ in range(reps):
            runl()
        out["lf_ms"] = round((time.perf_counter() - t) / reps * 1e3, 4)
        out["chosen"] = {"cdef_fast": {"bits": choice[0][1], "pairs": choice[0][0]}, "lf_levels": list(lv)}
        if rank == 0 and world == 1 and args.cpu_seconds > 0:
            exact = True
            for th in (0, 1):
                cms, lms, (pairs, bits, table), levels = search_cpu(sf, cur, src, bool(th), q, lam)
                exact &= pairs == choice[th][0] and bits == choice[th][1] and np.array_equal(table, choice[th][2])
                exact &= levels == list(lv)
                key = "cdef_thorough" if th else "cdef_fast"
                out.setdefault("cpu_oracle_ms", {})[key] = round(cms, 1)
                out["cpu_oracle_ms"]["lf"] = round(lms, 1)
            out["cpu_threads"] = os.cpu_count()
            out["same_choice_as_oracle"] = bool(exact)
            out["speedup_vs_oracle"] = {k: round(out["cpu_oracle_ms"][k] / out[k + "_ms"], 1)
                                        for k in ("cdef_fast", "cdef_thorough", "lf")}
        res[name] = out
    res["lr_1080p_10bit"] = bench_lr_search(args, ctx, rank, world)
    res["cdef_batch_640x360_x16"] = bench_cdef_search_batch(args, ctx)
    res["inputs"] = (f"seeded synthetic frames; reconstruction = source + seeded 4x4-block noise (+-24) and "
                     f"per-sample noise; base_q_idx {q}, lambda {lam}")
    return res


def bench_cdef_search_batch(args, ctx, n=16, w=640, h=360):
    """The CDEF search (fast lists) over n small frames: n per-frame calls
    against one av1pf_cdef_search_many call (host clock around each
    synchronous call; the results are the same by construction and by the
    parity tests)."""
    import gpu_util as G
    import torch
    L = A.lib()
    keep = []
    jobs = (A.CdefSearchJob * n)()
    for i in range(n):
        sf = A.SynthHandle(width=w, height=h, bit_depth=10, seed=600 + i)
        cur, src = A.synth_search_planes(sf, 700 + i, amp=24)
        info = sf.f.info
        df = G.DevFrame(sf)
        planes = []
        for arrs in (cur, src):
            d = G.DevPlanes(info, [(a.shape[1], a.shape[0]) for a in arrs], [a.shape[1] for a in arrs])
            for p in range(info.num_planes):
                d.t[p].copy_(torch.from_numpy(arrs[p].view(np.uint8).reshape(-1)))
            planes.append(d)
        res = A.CdefSearchResult()
        keep.append((sf, df, planes, res))
        jobs[i].info = C.pointer(sf.f.info)
        jobs[i].maps = C.pointer(df.maps)
        jobs[i].cur = C.cast(planes[0].c, C.POINTER(A.Plane))
        jobs[i].src = C.cast(planes[1].c, C.POINTER(A.Plane))
        jobs[i].base_q_idx = 120
        jobs[i].lam = 40.0
        jobs[i].result = C.pointer(res)

    def per_frame():
        for k in range(n):
            A.check(L.av1pf_cdef_search_many(ctx.p, 1, C.byref(jobs[k]), 0, None), "cdef_search_many")

    def batched():
        A.check(L.av1pf_cdef_search_many(ctx.p, n, jobs, 0, None), "cdef_search_many")
    out = {}
    for name, fn in (("per_frame_ms", per_frame), ("batched_ms", batched)):
        for _ in range(max(2, args.warmup)):
            fn()
        reps = 10
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        out[name] = round((time.perf_counter() - t) / reps * 1e3, 3)
    out["batched_vs_per_frame"] = round(out["per_frame_ms"] / out["batched_ms"], 2)
    return out


def bench_lr_search(args, ctx, rank, world, lam=150.0):
    """The loop-restoration search (encoder/lr.rs:64-210) on a 1080p 10-bit
    frame with 64x64 luma / 32x32 chroma units, each effort (fast: 2
    self-guided sets on every other sample; normal: 6; thorough: 16), one
    synchronous call per frame; the oracle's time beside it (rank 0, N = 1)."""
    import gpu_util as G
    import torch
    L = A.lib()
    sf = A.SynthHandle(width=1920, height=1080, bit_depth=10, seed=503, enable_lr=1)
    info, params = sf.f.info, sf.f.params
    cdef, src = A.synth_search_planes(sf, 8)
    cur, _ = A.synth_search_planes(sf, 1008)
    dev = []
    for planes in (cur, cdef, src):
        d = G.DevPlanes(info, [(a.shape[1], a.shape[0]) for a in planes], [a.shape[1] for a in planes])
        for p in range(info.num_planes):
            d.t[p].copy_(torch.from_numpy(planes[p].view(np.uint8).reshape(-1)))
        dev.append(d)
    arrs = [(A.LrUnit * (params.lr_unit_rows[p] * params.lr_unit_cols[p]))() for p in range(info.num_planes)]
    ptrs = (C.POINTER(A.LrUnit) * 3)(*[C.cast(a, C.POINTER(A.LrUnit)) for a in arrs])
    ft = (C.c_int32 * 3)()
    out = {"units": [params.lr_unit_rows[p] * params.lr_unit_cols[p] for p in range(info.num_planes)]}
    for eff, name in enumerate(("fast", "normal", "thorough")):
        def run():
            A.check(L.av1pf_lr_search(ctx.p, C.byref(info), C.byref(params), dev[0].c, dev[1].c, dev[2].c, lam, eff,
                                      ptrs, ft, None), "av1pf_lr_search")
        for _ in range(max(2, args.warmup)):
            run()
        reps = 10
        t = time.perf_counter()
        for _ in range(reps):
            run()
        out[name + "_ms"] = round((time.perf_counter() - t) / reps * 1e3, 3)
        if rank == 0 and world == 1 and args.cpu_seconds > 0:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            t = time.perf_counter()
            ft_o, units_o = O.lr_search(sf, O.HostPlanes(cur), O.HostPlanes(cdef), O.HostPlanes(src), lam, eff)
            cms = (time.perf_counter() - t) * 1e3
            same = ft_o == list(ft) and all(O.lr_unit_tuple(u) == units_o[p][k] for p in range(info.num_planes)
                                            for k, u in enumerate(arrs[p]))
            out.setdefault("cpu_oracle_ms", {})[name] = round(cms, 1)
            out.setdefault("same_choice_as_oracle", {})[name] = bool(same)
            out.setdefault("speedup_vs_oracle", {})[name] = round(cms / out[name + "_ms"], 1)
    out["frame_types"] = list(ft)[:info.num_planes]
    return out


SERVE_MIX = [(8, dict(width=640, height=360, bit_depth=8, sample_bytes=1)),
             (8, dict(width=960, height=540, bit_depth=8, sample_bytes=1)),
             (8, dict(width=1280, height=720, bit_depth=8, sample_bytes=1)),
             (6, dict(width=1920, height=1080, bit_depth=10)),
             (2, dict(width=3840, height=2160, bit_depth=10, subsampling_x=0, subsampling_y=0))]


def bench_serve(args, ctx, rank, duration_s=1.0):
    """Config 5: 32 streams (config 4's resolution mix) at 24-60 fps each,
    seeded Poisson arrivals over `duration_s`. Two feeds are measured through
    the serving loop: frames arriving in host memory (uploaded by the server)
    and frames already resident on the device (as a GPU decoder leaves them).
    Each is compared with the plain per-frame path on the same frame sequence
    (av1pf_chain_host / av1pf_chain, one call per frame), and the serving loop
    is also run saturated (every frame of the sequence queued as one
    av1pf_serve_submit_many group). The per-frame device path's throughput is
    timed with its calls queued back to back, its latency with a synchronize
    after each call.
    Latency is submit -> completion of the batch that carried the frame."""
    import threading
    import torch
    import gpu_util as G
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    L = A.lib()
    rng = np.random.default_rng(2024 + rank)
    streams = []
    k = 0
    for count, cfg in SERVE_MIX:
        for _ in range(count):
            frames = [A.SynthHandle(**cfg, seed=9000 + 100 * rank + 10 * k + j, frame_index=j) for j in range(2)]
            host = [O.HostPlanes.like_synth(sf) for sf in frames]
            dev = [G.DevFrame(sf) for sf in frames]
            outs = [(G.DevPlanes.visible(sf.f.info), G.dev_bytes(A.frame_bytes(sf.f.info))) for sf in frames]
            hreq, dreq = [], []
            for sf, hp, df, (r_out, f_out) in zip(frames, host, dev, outs):
                r = A.Request()
                r.info, r.params, r.maps = C.pointer(sf.f.info), C.pointer(sf.f.params), C.pointer(sf.f.maps)
                r.inp = C.cast(hp.c, C.POINTER(A.Plane))
                hreq.append(r)
                d = A.Request()
                d.info, d.params, d.maps = C.pointer(df.info), C.pointer(df.params), C.pointer(df.maps)
                d.inp = C.cast(df.inp.c, C.POINTER(A.Plane))
                d.device = 1
                d.ref_out = C.cast(r_out.c, C.POINTER(A.Plane))
                d.frame_out = f_out.data_ptr()
                dreq.append(d)
            streams.append({"frames": frames, "host": host, "dev": dev, "outs": outs, "hreq": hreq, "dreq": dreq,
                            "fps": float(rng.uniform(24, 60))})
            k += 1
    arrivals = []
    for si, st in enumerate(streams):
        t, j = float(rng.exponential(1.0 / st["fps"])), 0
        while t < duration_s:
            arrivals.append((t, si, j % 2))
            t += float(rng.exponential(1.0 / st["fps"]))
            j += 1
    arrivals.sort()
    n = len(arrivals)
    px = sum(streams[si]["frames"][j].info.upscaled_width * streams[si]["frames"][j].info.frame_height
             for (_, si, j) in arrivals)
    cfg = A.ServeConfig(40 << 30, 64, 2, 50, 4)  # 40 GB cap, <= 64 frames a batch, 2 in flight, 4 slots a stream
    srv = C.c_void_p()
    A.check(L.av1pf_serve_open(ctx.p, C.byref(cfg), C.byref(srv)), "serve_open")
    for st in streams:
        sid = C.c_int32()
        A.check(L.av1pf_serve_open_stream(srv, C.byref(st["frames"][0].f.info), C.byref(sid)), "open_stream")
        st["sid"] = sid.value

    def run(kind, paced, keep_out=None):
        """Submits the arrival sequence (paced by arrival time or all at once)
        while a second thread polls completions in order."""
        import queue as Q
        pending = Q.Queue()
        lats = []

        def poller():
            while True:
                item = pending.get()
                if item is None:
                    return
                tk, si, j = item
                fb = None
                if kind == "hreq":
                    fb = np.empty(A.frame_bytes(streams[si]["frames"][j].f.info), np.uint8)
                lat = C.c_double()
                A.check(L.av1pf_serve_poll(srv, tk, 120000, fb.ctypes.data if fb is not None else None,
                                           C.byref(lat)), "poll")
                lats.append(lat.value)
                if keep_out is not None and fb is not None:
                    keep_out.setdefault((si, j), fb)
        th = threading.Thread(target=poller)
        if not paced:
            # saturated: the whole sequence in one group, queued at once
            ids = (C.c_int32 * n)(*[streams[si]["sid"] for (_, si, _) in arrivals])
            reqs = (A.Request * n)(*[streams[si][kind][j] for (_, si, j) in arrivals])
            tks = (C.c_uint64 * n)()
        th.start()
        t0 = time.perf_counter()
        if not paced:
            A.check(L.av1pf_serve_submit_many(srv, n, ids, reqs, tks), "submit_many")
            for k, (_, si, j) in enumerate(arrivals):
                pending.put((tks[k], si, j))
        for (ta, si, j) in (arrivals if paced else []):
            while time.perf_counter() - t0 < ta:
                time.sleep(0.0001)
            tk = C.c_uint64()
            A.check(L.av1pf_serve_submit(srv, streams[si]["sid"], C.byref(streams[si][kind][j]), C.byref(tk)),
                    "submit")
            pending.put((tk.value, si, j))
        pending.put(None)
        th.join()
        wall = time.perf_counter() - t0
        return wall, lats

    run("hreq", False)  # warm-up: pinned pools, scratch
    run("dreq", False)
    b0 = A.ServeStats()
    A.check(L.av1pf_serve_stats_get(srv, C.byref(b0)))
    outs = {}
    w_h, lat_h = run("hreq", True, outs)
    b1 = A.ServeStats()
    A.check(L.av1pf_serve_stats_get(srv, C.byref(b1)))
    w_d, lat_d = run("dreq", True)
    s_h, _ = run("hreq", False)
    s_d, _ = run("dreq", False)
    b2 = A.ServeStats()
    A.check(L.av1pf_serve_stats_get(srv, C.byref(b2)))
    A.check(L.av1pf_serve_close(srv))
    # the plain per-frame paths on the same sequence
    pf_h, pf_d, exact = [], [], True
    t0 = time.perf_counter()
    for (ta, si, j) in arrivals:
        sf = streams[si]["frames"][j]
        fb = np.empty(A.frame_bytes(sf.f.info), np.uint8)
        a = time.perf_counter()
        A.check(L.av1pf_chain_host(ctx.p, C.byref(sf.f.info), C.byref(sf.f.params), C.byref(sf.f.maps),
                                   streams[si]["host"][j].c, None, fb.ctypes.data), "chain_host")
        pf_h.append(1e3 * (time.perf_counter() - a))
        if exact and (si, j) in outs:
            exact = bool(np.array_equal(fb, outs[(si, j)]))
    t_pfh = time.perf_counter() - t0
    torch.cuda.synchronize()
    # per-frame device path: throughput with the calls queued back to back
    # (one synchronize at the end), then latency with a synchronize per call
    t0 = time.perf_counter()
    for (ta, si, j) in arrivals:
        df = streams[si]["dev"][j]
        r_out, f_out = streams[si]["outs"][j]
        A.check(L.av1pf_chain(ctx.p, C.byref(df.info), C.byref(df.params), C.byref(df.maps), df.inp.c, r_out.c,
                              f_out.data_ptr(), None), "chain")
    torch.cuda.synchronize()
    t_pfd = time.perf_counter() - t0
    for (ta, si, j) in arrivals:
        df = streams[si]["dev"][j]
        r_out, f_out = streams[si]["outs"][j]
        a = time.perf_counter()
        A.check(L.av1pf_chain(ctx.p, C.byref(df.info), C.byref(df.params), C.byref(df.maps), df.inp.c, r_out.c,
                              f_out.data_ptr(), None), "chain")
        torch.cuda.synchronize()
        pf_d.append(1e3 * (time.perf_counter() - a))

    def pct(v, q):
        return round(float(np.percentile(v, q)), 3)
    return {"streams": len(streams), "frames": n, "mpx": round(px / 1e6, 2), "duration_s": duration_s,
            "offered_fps": round(n / duration_s, 1),
            "host_feed": {"served_fps": round(n / w_h, 1), "p50_ms": pct(lat_h, 50), "p99_ms": pct(lat_h, 99),
                          "mean_batch_frames": round((b1.completed - b0.completed) / max(1, b1.batches - b0.batches), 2),
                          "saturated_fps": round(n / s_h, 1), "saturated_mpx_s": round(px / s_h / 1e6, 1),
                          "per_frame_fps": round(n / t_pfh, 1), "per_frame_mpx_s": round(px / t_pfh / 1e6, 1),
                          "per_frame_p50_ms": pct(pf_h, 50), "per_frame_p99_ms": pct(pf_h, 99),
                          "saturated_vs_per_frame": round(t_pfh / s_h, 3)},
            "device_feed": {"served_fps": round(n / w_d, 1), "p50_ms": pct(lat_d, 50), "p99_ms": pct(lat_d, 99),
                            "saturated_fps": round(n / s_d, 1), "saturated_mpx_s": round(px / s_d / 1e6, 1),
                            "per_frame_fps": round(n / t_pfd, 1), "per_frame_mpx_s": round(px / t_pfd / 1e6, 1),
                            "per_frame_p50_ms": pct(pf_d, 50), "per_frame_p99_ms": pct(pf_d, 99),
                            "saturated_vs_per_frame": round(t_pfd / s_d, 3)},
            "mean_batch_frames_all": round(b2.mean_batch_frames, 2),
            "bit_exact_serve_vs_per_frame": exact}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--skip-extras", action="store_true")
    ap.add_argument("--only", choices=["mix", "c3", "grain", "serve", "search"], default=None,
                    help="run one extra section alone (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return main_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
