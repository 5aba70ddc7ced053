"""The synthetic input generator makes conformant, deterministic frames with
the configured distributions (CPU only)."""
import ctypes as C

import numpy as np
import pytest

import av1pf as A

TX_W = [4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64]
TX_H = [4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16]


def arr(ptr, n, dtype):
    return np.frombuffer((C.c_uint8 * (n * np.dtype(dtype).itemsize)).from_address(ptr), dtype=dtype)


def test_deterministic():
    a = A.SynthHandle(width=320, height=180, bit_depth=10, seed=9)
    b = A.SynthHandle(width=320, height=180, bit_depth=10, seed=9)
    for p in range(3):
        n = a.f.plane_bytes[p]
        assert np.array_equal(arr(a.f.planes[p].data, n, np.uint8), arr(b.f.planes[p].data, n, np.uint8))
    assert np.array_equal(arr(a.f.maps.mi, a.f.mi_count * 8, np.uint8), arr(b.f.maps.mi, b.f.mi_count * 8, np.uint8))
    c = A.SynthHandle(width=320, height=180, bit_depth=10, seed=10)
    assert not np.array_equal(arr(a.f.planes[0].data, 1000, np.uint8), arr(c.f.planes[0].data, 1000, np.uint8))


@pytest.mark.parametrize("ss", [(1, 1), (1, 0), (0, 0)])
def test_transform_blocks_tile_each_plane(ss):
    """Every transform block starts at a multiple of its size and covers
    exactly its 4x4s: the property in-place edge filtering relies on."""
    s = A.SynthHandle(width=256, height=192, bit_depth=10, subsampling_x=ss[0], subsampling_y=ss[1], seed=3)
    f = s.f
    ms = f.maps.mi_stride
    for p in range(3):
        sx = ss[0] if p else 0
        sy = ss[1] if p else 0
        gw, gh = f.info.mi_cols >> sx, f.info.mi_rows >> sy
        tx = arr(f.maps.lf_tx_size[p], f.tx_count[p], np.uint8).reshape(-1, ms)
        for y in range(gh):
            for x in range(gw):
                t = tx[y, x]
                w4, h4 = TX_W[t] // 4, TX_H[t] // 4
                x0, y0 = x - x % w4, y - y % h4
                assert (tx[y0:y0 + h4, x0:x0 + w4] == t).all(), (p, y, x)


def test_config_distributions():
    s = A.SynthHandle(width=1920, height=1080, bit_depth=10, seed=1)
    p = s.f.params
    assert all(0 <= p.loop_filter_level[k] <= 63 for k in range(4))
    assert 0 <= p.loop_filter_sharpness <= 7
    assert p.cdef_enabled and 3 <= p.cdef_damping <= 6 and p.cdef_bits == 3
    assert all(p.cdef_y_sec_strength[k] in (0, 1, 2, 4) for k in range(8))
    assert p.uses_lr and p.loop_restoration_size[0] == 64
    units = arr(s.f.maps.lr_units[0], s.f.lr_count[0] * 12, np.uint8).reshape(-1, 12)
    types = set(units[:, 0].tolist())
    assert types == {0, 1, 2}
    luma = arr(s.f.planes[0].data, s.f.plane_bytes[0] // 2, np.uint16)
    assert luma.max() <= 1023
    cdef = arr(s.f.maps.cdef_idx, s.f.cdef_count, np.int8)
    assert cdef.max() <= 7 and cdef.min() >= -1


def test_superres_geometry():
    s = A.SynthHandle(width=3840, height=2160, bit_depth=10, superres_denom=13)
    i = s.f.info
    assert i.upscaled_width == 3840 and i.frame_width == (3840 * 8 + 6) // 13
    assert i.mi_cols == 2 * ((i.frame_width + 7) >> 3)
    assert s.f.params.use_superres == 1
