#!/usr/bin/env python3
"""Generates the oracle regression fixtures in this folder.

The reference (Rust) cannot run here and ships no pre/post-filter plane
dumps, so these fixtures hold the CPU oracle's own outputs on small seeded
synthetic frames: they pin the oracle against regressions and give the GPU
parity tests fixed expected values. `chain_digests.json` holds SHA-256
digests of (reference-frame planes, packed output frame) per case;
`small_8bit.npz` holds the smallest case in full.

Usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rivet-av1_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = {
    "small_8bit": dict(width=96, height=72, bit_depth=8, sample_bytes=1, content=1, seed=11),
    "c1_352x288_8bit_f3": dict(width=352, height=288, bit_depth=8, sample_bytes=1, content=1, seed=1,
                               frame_index=3),
    "b10_420_seg_dlf": dict(width=240, height=136, bit_depth=10, seed=5, segmentation=1, delta_lf=2),
    "b12_444": dict(width=160, height=96, bit_depth=12, subsampling_x=0, subsampling_y=0, seed=7),
    "b10_422": dict(width=168, height=100, bit_depth=10, subsampling_x=1, subsampling_y=0, seed=8),
    "b8_mono_u16": dict(width=130, height=70, bit_depth=8, sample_bytes=2, mono=1, seed=9),
    "b10_superres_grain": dict(width=256, height=144, bit_depth=10, superres_denom=13, enable_grain=1,
                               seed=12, frame_index=5),
    "b12_444_superres_grain": dict(width=200, height=90, bit_depth=12, subsampling_x=0, subsampling_y=0,
                                   superres_denom=9, enable_grain=1, seed=13, lr_unit_shift=1),
    "b8_grain_unit256": dict(width=300, height=180, bit_depth=8, sample_bytes=1, enable_grain=1,
                             lr_unit_shift=2, seed=14),
}


def digest(ref, fb):
    h = hashlib.sha256()
    for a in ref.arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(fb.tobytes())
    return h.hexdigest()


def main():
    import av1pf as A
    import oracle as O
    out = {}
    for name, kw in CASES.items():
        s = A.SynthHandle(**kw)
        ref, fb = O.chain(s, threads=0)
        out[name] = digest(ref, fb)
        if name == "small_8bit":
            inp = O.HostPlanes.like_synth(s)
            arrs = {f"in{p}": inp.arrays[p] for p in range(3)}
            arrs.update({f"ref{p}": ref.arrays[p] for p in range(3)})
            arrs["frame"] = fb
            np.savez_compressed(os.path.join(HERE, "small_8bit.npz"), **arrs)
    with open(os.path.join(HERE, "chain_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(f"wrote {len(out)} digests")


if __name__ == "__main__":
    main()
