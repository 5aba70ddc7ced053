"""av1pf_frame_md5 / av1pf_md5 (host): RFC 1321's test suite, messages of
every length around the padding boundaries against Python's hashlib, and
the conformance hash of packed frames (the packed bytes, plus two neutral
chroma planes for a monochrome frame, tests/common/mod.rs:101-119)."""
import ctypes as C
import hashlib

import numpy as np
import pytest

import av1pf as A


def md5(data):
    out = C.create_string_buffer(33)
    buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data if data else b"\0")
    A.check(A.lib().av1pf_md5(buf, len(data), out), "av1pf_md5")
    return out.value.decode()


# RFC 1321 appendix A.5 test suite
RFC_SUITE = [
    (b"", "d41d8cd98f00b204e9800998ecf8427e"),
    (b"a", "0cc175b9c0f1b6a831c399e269772661"),
    (b"abc", "900150983cd24fb0d6963f7d28e17f72"),
    (b"message digest", "f96b697d7cb7938d525a2f31aaf161d0"),
    (b"abcdefghijklmnopqrstuvwxyz", "c3fcd3d76192e4007dfb496cca67e13b"),
    (b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789", "d174ab98d277d9f5a5611c2c9f419d9f"),
    (b"1234567890" * 8, "57edf4a22be3c955ac49da2e2107b67a"),
]


@pytest.mark.parametrize("msg,want", RFC_SUITE)
def test_rfc1321_suite(msg, want):
    assert md5(msg) == want


def test_lengths_around_block_boundaries():
    rng = np.random.default_rng(3)
    for n in list(range(0, 200)) + [1000, 4095, 4096, 4097, 65535, 100003]:
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert md5(data) == hashlib.md5(data).hexdigest(), n


@pytest.mark.parametrize("cfg", [dict(width=64, height=48, bit_depth=8, sample_bytes=1),
                                 dict(width=67, height=35, bit_depth=10),
                                 dict(width=50, height=30, bit_depth=12, subsampling_x=0, subsampling_y=0),
                                 dict(width=65, height=33, bit_depth=10, mono=1),
                                 dict(width=64, height=32, bit_depth=8, sample_bytes=1, mono=1)])
def test_frame_md5(cfg):
    sf = A.SynthHandle(seed=4, **cfg)
    info = sf.f.info
    rng = np.random.default_rng(5)
    frame = rng.integers(0, 256, A.frame_bytes(info), dtype=np.uint8)
    h = hashlib.md5(frame.tobytes())
    if info.num_planes == 1:
        cw, ch = (info.upscaled_width + 1) // 2, (info.frame_height + 1) // 2
        mid = 1 << (info.bit_depth - 1)
        plane = (np.full(cw * ch, mid, "<u2").tobytes() if info.bit_depth > 8
                 else np.full(cw * ch, mid, np.uint8).tobytes())
        h.update(plane)
        h.update(plane)
    assert A.frame_md5(info, frame) == h.hexdigest()
