"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the product path. The
oracle restates rivet-av1's post-filter chain on the CPU; see oracle.h for
what pins it.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "rivet-av1_b200"))
import av1pf as A  # noqa: E402  (structure definitions only)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p

        def sig(name, res, *args):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = list(args)

        sig("oracle_loop_filter", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Maps), P(A.Plane), C.c_int)
        sig("oracle_cdef", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Maps), P(A.Plane), P(A.Plane), C.c_int)
        sig("oracle_superres", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Plane), P(A.Plane))
        sig("oracle_loop_restoration", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Maps), P(A.Plane), P(A.Plane),
            P(A.Plane), C.c_int)
        sig("oracle_output", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Plane), vp)
        sig("oracle_chain", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Maps), P(A.Plane), P(A.Plane), vp, C.c_int)
        sig("oracle_lf_filter_lanes", None, vp, vp, C.c_int)
        sig("oracle_lf_reference", None, vp, vp, C.c_int)
        sig("oracle_lf_kat_cases", None, C.c_uint64, C.c_int, vp, vp)
        sig("oracle_cdef_filter", None, vp, vp, vp, C.c_int)
        sig("oracle_cdef_kat_cases", None, C.c_uint64, C.c_int, vp, vp)
        sig("oracle_cdef_search", C.c_int, P(A.FrameInfo), P(A.Maps), P(A.Plane), P(A.Plane), C.c_int32, C.c_double,
            C.c_int32, P(A.CdefSearchResult), vp, vp, C.c_int)
        sig("oracle_lr_search", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Plane), P(A.Plane), P(A.Plane),
            C.c_double, C.c_int32, P(C.POINTER(A.LrUnit)), P(C.c_int32), C.c_int)
        sig("oracle_lf_search", C.c_int, P(A.FrameInfo), P(A.Params), P(A.Maps), P(A.Plane), P(A.Plane),
            P(C.c_int32), vp, C.c_int)
        _lib = L
    return _lib


def dtype_of(info):
    return np.uint8 if info.sample_bytes == 1 else np.uint16


class HostPlanes:
    """numpy-backed planes (one per plane) exposed as an av1pf_plane array."""

    def __init__(self, arrays):
        self.arrays = [np.ascontiguousarray(a) for a in arrays]
        self.c = (A.Plane * 3)()
        for i, a in enumerate(self.arrays):
            self.c[i].data = a.ctypes.data
            self.c[i].stride = a.shape[1]
            self.c[i].width = a.shape[1]
            self.c[i].height = a.shape[0]

    @staticmethod
    def visible(info):
        """Zeroed planes of the visible (upscaled) area."""
        arrs = []
        for p in range(info.num_planes):
            sx = info.subsampling_x if p else 0
            sy = info.subsampling_y if p else 0
            arrs.append(np.zeros(((info.frame_height + sy) >> sy, (info.upscaled_width + sx) >> sx), dtype_of(info)))
        return HostPlanes(arrs)

    @staticmethod
    def like_synth(sf):
        """Copies of a synthetic frame's pre-filter planes (allocated layout)."""
        f = sf.f
        arrs = []
        for p in range(f.info.num_planes):
            pl = f.planes[p]
            dt = dtype_of(f.info)
            n = pl.height * pl.stride
            buf = (C.c_uint8 * (n * np.dtype(dt).itemsize)).from_address(pl.data)
            arrs.append(np.frombuffer(buf, dtype=dt).reshape(pl.height, pl.stride).copy())
        return HostPlanes(arrs)

    @staticmethod
    def zeros_like(other):
        return HostPlanes([np.zeros_like(a) for a in other.arrays])

    @staticmethod
    def upscaled(info):
        """Zeroed planes of the upscaled allocation (superres output)."""
        arrs = []
        mh = info.mi_rows * 4
        ah = (mh + 127) & ~127
        for p in range(info.num_planes):
            sx = info.subsampling_x if p else 0
            sy = info.subsampling_y if p else 0
            w = ((info.upscaled_width + sx) >> sx) + 32
            arrs.append(np.zeros(((ah >> sy) + 32, w), dtype_of(info)))
        return HostPlanes(arrs)


def chain(sf, threads=0, want_frame=True):
    """(ref planes, packed frame bytes) of the oracle chain on a SynthHandle."""
    info, params, maps = sf.f.info, sf.f.params, sf.f.maps
    inp = HostPlanes.like_synth(sf)
    ref = HostPlanes.visible(info)
    fb = np.zeros(A.frame_bytes(info), np.uint8) if want_frame else None
    rc = lib().oracle_chain(C.byref(info), C.byref(params), C.byref(maps), inp.c, ref.c,
                            fb.ctypes.data if want_frame else None, threads)
    if rc != 0:
        raise RuntimeError(f"oracle_chain: {rc}")
    return ref, fb


def search_inputs(sf, seed, amp=None):
    """(cur, src) HostPlanes of av1pf.synth_search_planes."""
    cur, src = A.synth_search_planes(sf, seed, amp)
    return HostPlanes(cur), HostPlanes(src)


def cdef_search(sf, cur, src, q, lam, thorough, threads=0):
    """(result, cdef_idx table, block_sse [blocks, ny + nuv]) of the oracle's
    CDEF search."""
    info, maps = sf.f.info, sf.f.maps
    fbr, fbc = (info.mi_rows + 15) // 16, (info.mi_cols + 15) // 16
    ny, nuv = A.CDEF_SEARCH_N[bool(thorough)]
    res = A.CdefSearchResult()
    table = np.zeros(fbr * maps.cdef_stride, np.int8)
    sse = np.zeros((fbr * fbc, ny + nuv), np.uint64)
    rc = lib().oracle_cdef_search(C.byref(info), C.byref(maps), cur.c, src.c, q, lam, int(thorough), C.byref(res),
                                  table.ctypes.data, sse.ctypes.data, threads)
    if rc != 0:
        raise RuntimeError(f"oracle_cdef_search: {rc}")
    return res, table, sse


def lf_search(sf, cur, src, threads=0, params=None):
    """(levels[4], sse[6, 3]) of the oracle's loop-filter level search."""
    info, maps = sf.f.info, sf.f.maps
    levels = (C.c_int32 * 4)()
    sse = np.zeros((6, 3), np.uint64)
    rc = lib().oracle_lf_search(C.byref(info), C.byref(params if params is not None else sf.f.params),
                                C.byref(maps), cur.c, src.c, levels, sse.ctypes.data, threads)
    if rc != 0:
        raise RuntimeError(f"oracle_lf_search: {rc}")
    return list(levels), sse


def lr_unit_tuple(u):
    """(type, wiener ((v0, v1, v2), (h0, h1, h2)), set, xqd) of an av1pf_lr_unit."""
    return (u.type, (tuple(u.wiener[0]), tuple(u.wiener[1])), u.sgr_set, tuple(u.sgr_xqd))


def lr_unit_arrays(params, num_planes):
    return [(A.LrUnit * max(1, params.lr_unit_rows[p] * params.lr_unit_cols[p]))() if p < num_planes else None
            for p in range(3)]


def lr_search(sf, cur, cdef, src, lam, effort, threads=0):
    """(frame types[3], per-plane lists of unit tuples) of the oracle's LR search."""
    info, params = sf.f.info, sf.f.params
    arrs = lr_unit_arrays(params, info.num_planes)
    ptrs = (C.POINTER(A.LrUnit) * 3)(*[C.cast(a, C.POINTER(A.LrUnit)) if a is not None else None for a in arrs])
    ft = (C.c_int32 * 3)()
    rc = lib().oracle_lr_search(C.byref(info), C.byref(params), cur.c, cdef.c, src.c, lam, effort, ptrs, ft, threads)
    if rc != 0:
        raise RuntimeError(f"oracle_lr_search: {rc}")
    units = [[lr_unit_tuple(u) for u in arrs[p][:params.lr_unit_rows[p] * params.lr_unit_cols[p]]]
             if arrs[p] is not None else [] for p in range(3)]
    return list(ft), units


def lr_search_inputs(sf, seed, amp=None):
    """(cur, cdef, src) HostPlanes for the LR search: the source is the
    synthetic frame's planes, the CDEF output the source plus seeded noise,
    and the deblocked frame (read at stripe boundaries) the source plus other
    noise."""
    cdef, src = A.synth_search_planes(sf, seed, amp)
    cur, _ = A.synth_search_planes(sf, seed + 1000, amp)
    return HostPlanes(cur), HostPlanes(cdef), HostPlanes(src)
