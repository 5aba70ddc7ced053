"""ctypes bindings of the av1pf C ABI (include/av1pf.h) and of the synthetic
input generator (synth/synth.h).

The structures mirror the header field for field. The library is the
in-tree ``libav1pf.so`` built by ``make -C rivet-av1_b200``; loading fails
loudly if it is missing, since there is no other implementation.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libav1pf.so")
SYNTH_PATH = os.path.join(HERE, "libav1pf_synth.so")

OK = 0
ERR_INVALID_INPUT = 1
ERR_UNSUPPORTED = 2
ERR_OOM = 3
ERR_ADMISSION = 4
ERR_TIMEOUT = 5
ERR_CUDA = 6
ERR_NOT_FOUND = 7
MI_SKIP = 0x80
RESTORE_NONE, RESTORE_WIENER, RESTORE_SGRPROJ = 0, 1, 2
BATCH_NO_GRAPH = 1
BATCH_AUTOTUNE = 2
BATCH_GROUPS_SHIFT = 8


class Plane(C.Structure):
    _fields_ = [("data", C.c_void_p), ("stride", C.c_int64), ("width", C.c_int32), ("height", C.c_int32)]


class FrameInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "bit_depth", "sample_bytes", "subsampling_x", "subsampling_y", "num_planes", "frame_width",
        "frame_height", "upscaled_width", "mi_rows", "mi_cols", "matrix_coefficients")]


class Mi(C.Structure):
    _fields_ = [("mi_size", C.c_uint8), ("y_mode", C.c_uint8), ("ref_frame0", C.c_int8),
                ("skip_segment", C.c_uint8), ("delta_lf", C.c_int8 * 4)]


class LrUnit(C.Structure):
    _fields_ = [("type", C.c_uint8), ("sgr_set", C.c_uint8), ("sgr_xqd", C.c_int8 * 2),
                ("wiener", (C.c_int8 * 3) * 2), ("_pad", C.c_uint8 * 2)]


class Maps(C.Structure):
    _fields_ = [("mi", C.c_void_p), ("mi_stride", C.c_int32), ("cdef_stride", C.c_int32),
                ("lf_tx_size", C.c_void_p * 3), ("cdef_idx", C.c_void_p), ("lr_units", C.c_void_p * 3)]


class FilmGrain(C.Structure):
    _fields_ = [
        ("apply", C.c_int32), ("grain_seed", C.c_int32), ("num_y_points", C.c_int32),
        ("point_y_value", C.c_int32 * 16), ("point_y_scaling", C.c_int32 * 16),
        ("chroma_scaling_from_luma", C.c_int32), ("num_cb_points", C.c_int32),
        ("point_cb_value", C.c_int32 * 16), ("point_cb_scaling", C.c_int32 * 16),
        ("num_cr_points", C.c_int32), ("point_cr_value", C.c_int32 * 16), ("point_cr_scaling", C.c_int32 * 16),
        ("grain_scaling_minus_8", C.c_int32), ("ar_coeff_lag", C.c_int32),
        ("ar_coeffs_y_plus_128", C.c_int32 * 24), ("ar_coeffs_cb_plus_128", C.c_int32 * 25),
        ("ar_coeffs_cr_plus_128", C.c_int32 * 25), ("ar_coeff_shift_minus_6", C.c_int32),
        ("grain_scale_shift", C.c_int32), ("cb_mult", C.c_int32), ("cb_luma_mult", C.c_int32),
        ("cb_offset", C.c_int32), ("cr_mult", C.c_int32), ("cr_luma_mult", C.c_int32), ("cr_offset", C.c_int32),
        ("overlap_flag", C.c_int32), ("clip_to_restricted_range", C.c_int32)]


class Params(C.Structure):
    _fields_ = [
        ("loop_filter_level", C.c_int32 * 4), ("loop_filter_sharpness", C.c_int32),
        ("loop_filter_delta_enabled", C.c_int32), ("loop_filter_ref_deltas", C.c_int32 * 8),
        ("loop_filter_mode_deltas", C.c_int32 * 2), ("delta_lf_multi", C.c_int32),
        ("segmentation_enabled", C.c_int32), ("feature_enabled", (C.c_uint8 * 8) * 8),
        ("feature_data", (C.c_int32 * 8) * 8),
        ("cdef_enabled", C.c_int32), ("cdef_damping", C.c_int32), ("cdef_bits", C.c_int32),
        ("cdef_y_pri_strength", C.c_int32 * 8), ("cdef_y_sec_strength", C.c_int32 * 8),
        ("cdef_uv_pri_strength", C.c_int32 * 8), ("cdef_uv_sec_strength", C.c_int32 * 8),
        ("use_superres", C.c_int32), ("uses_lr", C.c_int32), ("frame_restoration_type", C.c_int32 * 3),
        ("loop_restoration_size", C.c_int32 * 3), ("lr_unit_rows", C.c_int32 * 3), ("lr_unit_cols", C.c_int32 * 3),
        ("film_grain", FilmGrain)]


class RefFrame(C.Structure):
    """av1pf_ref_frame: what a device reference slot holds."""
    _fields_ = [("valid", C.c_int32), ("info", FrameInfo), ("order_hint", C.c_uint32), ("frame_id", C.c_uint64),
                ("planes", Plane * 3)]


class Job(C.Structure):
    _fields_ = [("info", C.POINTER(FrameInfo)), ("params", C.POINTER(Params)), ("maps", C.POINTER(Maps)),
                ("inp", C.POINTER(Plane)), ("ref_out", C.POINTER(Plane)), ("frame_out", C.c_void_p)]


class HostJob(C.Structure):
    """av1pf_host_job: one frame of av1pf_chain_host_many (host pointers)."""
    _fields_ = [("info", C.POINTER(FrameInfo)), ("params", C.POINTER(Params)), ("maps", C.POINTER(Maps)),
                ("inp", C.POINTER(Plane)), ("ref_out", C.POINTER(Plane)), ("frame_out", C.c_void_p)]


class Tuning(C.Structure):
    _fields_ = [("lf_mode", C.c_int32), ("lr_rect_cols", C.c_int32)]


class ServeConfig(C.Structure):
    _fields_ = [("hbm_cap_bytes", C.c_uint64), ("max_batch_frames", C.c_int32),
                ("inflight_batches", C.c_int32), ("tick_us", C.c_int32), ("slots_per_stream", C.c_int32)]


class Request(C.Structure):
    _fields_ = [("info", C.POINTER(FrameInfo)), ("params", C.POINTER(Params)), ("maps", C.POINTER(Maps)),
                ("inp", C.POINTER(Plane)), ("device", C.c_int32), ("ref_out", C.POINTER(Plane)),
                ("frame_out", C.c_void_p)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("refused", C.c_uint64),
                ("batches", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_batch_frames", C.c_double), ("resident_bytes", C.c_uint64)]


class CdefSearchResult(C.Structure):
    _fields_ = [("damping_minus_3", C.c_int32), ("bits", C.c_int32), ("y_pri", C.c_int32 * 8),
                ("y_sec", C.c_int32 * 8), ("uv_pri", C.c_int32 * 8), ("uv_sec", C.c_int32 * 8)]

    def pairs(self):
        """[(y_pri, y_sec, uv_pri, uv_sec)] per index (secondaries as coded)."""
        return [(self.y_pri[i], self.y_sec[i], self.uv_pri[i], self.uv_sec[i]) for i in range(1 << self.bits)]


CDEF_SEARCH_N = {False: (28, 15), True: (44, 24)}  # (luma, chroma) candidate pairs


class CdefSearchJob(C.Structure):
    _fields_ = [("info", C.POINTER(FrameInfo)), ("maps", C.POINTER(Maps)), ("cur", C.POINTER(Plane)),
                ("src", C.POINTER(Plane)), ("base_q_idx", C.c_int32), ("lam", C.c_double),
                ("result", C.POINTER(CdefSearchResult)), ("cdef_idx_out", C.c_void_p), ("block_sse", C.c_void_p)]


class LfSearchJob(C.Structure):
    _fields_ = [("info", C.POINTER(FrameInfo)), ("params", C.POINTER(Params)), ("maps", C.POINTER(Maps)),
                ("cur", C.POINTER(Plane)), ("src", C.POINTER(Plane)), ("levels_out", C.c_int32 * 4),
                ("sse_out", C.c_void_p)]


class LrSearchJob(C.Structure):
    _fields_ = [("info", C.POINTER(FrameInfo)), ("params", C.POINTER(Params)), ("cur", C.POINTER(Plane)),
                ("cdef", C.POINTER(Plane)), ("src", C.POINTER(Plane)), ("lam", C.c_double),
                ("units_out", C.POINTER(LrUnit) * 3), ("frame_type_out", C.c_int32 * 3)]


class LfEdgeParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("limit", "blimit", "thresh", "filter_size", "chroma", "bit_depth")]


class CdefTaps(C.Structure):
    _fields_ = [("pri_str", C.c_int32), ("sec_str", C.c_int32), ("pri_adj", C.c_int32), ("sec_adj", C.c_int32),
                ("pri_taps", C.c_int32 * 2), ("sec_taps", C.c_int32 * 2), ("pri_off", C.c_int32 * 2),
                ("sec_off", (C.c_int32 * 2) * 2), ("w", C.c_int32), ("h", C.c_int32)]


# ---------------------------------------------------------------------------
# synthetic inputs (synth/synth.h)
# ---------------------------------------------------------------------------
CONTENT_FIELD, CONTENT_MOVING = 0, 1


class SynthConfig(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("bit_depth", C.c_int32), ("sample_bytes", C.c_int32),
                ("subsampling_x", C.c_int32), ("subsampling_y", C.c_int32), ("mono", C.c_int32),
                ("superres_denom", C.c_int32), ("content", C.c_int32), ("noise_sigma", C.c_int32),
                ("frame_index", C.c_int32), ("seed", C.c_uint64), ("enable_lf", C.c_int32),
                ("enable_cdef", C.c_int32), ("enable_lr", C.c_int32), ("enable_grain", C.c_int32),
                ("lr_unit_shift", C.c_int32), ("lr_uv_shift", C.c_int32), ("segmentation", C.c_int32),
                ("delta_lf", C.c_int32), ("min_block_log2", C.c_int32), ("skip_pct", C.c_int32)]


class SynthFrame(C.Structure):
    _fields_ = [("info", FrameInfo), ("params", Params), ("maps", Maps), ("planes", Plane * 3),
                ("mi_count", C.c_int64), ("tx_count", C.c_int64 * 3), ("cdef_count", C.c_int64),
                ("lr_count", C.c_int64 * 3), ("plane_bytes", C.c_int64 * 3)]


_lib = None
_synth = None


def _sig(lib, name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)


def lib():
    """The product library. Raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C rivet-av1_b200` (no fallback exists)")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        _sig(L, "av1pf_ctx_create", C.c_int, C.c_int, C.c_uint64, P(vp))
        _sig(L, "av1pf_ctx_destroy", C.c_int, vp)
        _sig(L, "av1pf_set_threads", C.c_int, vp, C.c_int)
        _sig(L, "av1pf_ctx_memory", C.c_int, vp, P(C.c_uint64))
        _sig(L, "av1pf_validate", C.c_int, P(FrameInfo), P(Params), P(Plane))
        _sig(L, "av1pf_loop_filter", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), vp)
        _sig(L, "av1pf_cdef", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), P(Plane), vp)
        _sig(L, "av1pf_superres", C.c_int, vp, P(FrameInfo), P(Params), P(Plane), P(Plane), vp)
        _sig(L, "av1pf_loop_restoration", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), P(Plane),
             P(Plane), vp)
        _sig(L, "av1pf_output", C.c_int, vp, P(FrameInfo), P(Params), P(Plane), vp, vp)
        _sig(L, "av1pf_frame_bytes", C.c_size_t, P(FrameInfo))
        _sig(L, "av1pf_frame_md5", C.c_int, P(FrameInfo), vp, C.c_char_p)
        _sig(L, "av1pf_md5", C.c_int, vp, C.c_size_t, C.c_char_p)
        _sig(L, "av1pf_output_noalloc", C.c_int, P(FrameInfo), P(Params), P(Plane), vp, vp)
        _sig(L, "av1pf_chain", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), P(Plane), vp, vp)
        _sig(L, "av1pf_chain_host", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), P(Plane), vp)
        _sig(L, "av1pf_chain_host_many", C.c_int, vp, C.c_int, P(HostJob))
        _sig(L, "av1pf_refs_create", C.c_int, vp, P(vp))
        _sig(L, "av1pf_refs_destroy", C.c_int, vp)
        _sig(L, "av1pf_refs_chain", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), C.c_uint32, C.c_uint32,
             vp, vp)
        _sig(L, "av1pf_refs_get", C.c_int, vp, C.c_int, P(RefFrame))
        _sig(L, "av1pf_refs_show", C.c_int, vp, C.c_int, P(Params), C.c_uint32, vp, vp)
        _sig(L, "av1pf_refs_memory", C.c_int, vp, P(C.c_uint64), P(C.c_int32))
        _sig(L, "av1pf_batch_create", C.c_int, vp, P(Job), C.c_int, C.c_uint32, P(vp))
        _sig(L, "av1pf_batch_run", C.c_int, vp, vp)
        _sig(L, "av1pf_batch_destroy", C.c_int, vp)
        _sig(L, "av1pf_set_tuning", C.c_int, vp, P(Tuning))
        _sig(L, "av1pf_get_tuning", C.c_int, vp, P(Tuning))
        _sig(L, "av1pf_autotune", C.c_int, vp, P(Job), C.c_int, C.c_int32, P(C.c_int32))
        _sig(L, "av1pf_tuned_choice", C.c_int, vp, P(FrameInfo), P(Tuning), P(C.c_float))
        _sig(L, "av1pf_serve_open", C.c_int, vp, P(ServeConfig), P(vp))
        _sig(L, "av1pf_serve_open_stream", C.c_int, vp, P(FrameInfo), P(C.c_int32))
        _sig(L, "av1pf_serve_close_stream", C.c_int, vp, C.c_int32)
        _sig(L, "av1pf_serve_submit", C.c_int, vp, C.c_int32, P(Request), P(C.c_uint64))
        _sig(L, "av1pf_serve_submit_many", C.c_int, vp, C.c_int32, P(C.c_int32), P(Request), P(C.c_uint64))
        _sig(L, "av1pf_serve_poll", C.c_int, vp, C.c_uint64, C.c_int32, vp, P(C.c_double))
        _sig(L, "av1pf_serve_stats_get", C.c_int, vp, P(ServeStats))
        _sig(L, "av1pf_serve_close", C.c_int, vp)
        _sig(L, "av1pf_cdef_search", C.c_int, vp, P(FrameInfo), P(Maps), P(Plane), P(Plane), C.c_int32, C.c_double,
             C.c_int32, P(CdefSearchResult), vp, vp, vp)
        _sig(L, "av1pf_cdef_search_many", C.c_int, vp, C.c_int, P(CdefSearchJob), C.c_int32, vp)
        _sig(L, "av1pf_lr_search", C.c_int, vp, P(FrameInfo), P(Params), P(Plane), P(Plane), P(Plane), C.c_double,
             C.c_int32, P(P(LrUnit)), P(C.c_int32), vp)
        _sig(L, "av1pf_lf_search_many", C.c_int, vp, C.c_int, P(LfSearchJob), vp)
        _sig(L, "av1pf_lr_search_many", C.c_int, vp, C.c_int, P(LrSearchJob), C.c_int32, vp)
        _sig(L, "av1pf_lf_search", C.c_int, vp, P(FrameInfo), P(Params), P(Maps), P(Plane), P(Plane),
             P(C.c_int32), vp, vp)
        _sig(L, "av1pf_dsp_lf_filter", C.c_int, vp, vp, vp, C.c_int, vp)
        _sig(L, "av1pf_dsp_cdef_filter", C.c_int, vp, vp, vp, vp, C.c_int, vp)
        _sig(L, "av1pf_set_profiling", C.c_int, vp, C.c_int)
        _sig(L, "av1pf_stage_times", C.c_int, vp, P(C.c_float), P(C.c_uint32))
        _sig(L, "av1pf_last_error", C.c_char_p)
        _sig(L, "av1pf_launch_count", C.c_uint64)
        _lib = L
    return _lib


def synth():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError(f"{SYNTH_PATH} is missing: run `make -C rivet-av1_b200`")
        S = C.CDLL(SYNTH_PATH)
        _sig(S, "synth_default_config", None, C.POINTER(SynthConfig))
        _sig(S, "synth_create", C.c_int, C.POINTER(SynthConfig), C.POINTER(C.POINTER(SynthFrame)))
        _sig(S, "synth_destroy", None, C.POINTER(SynthFrame))
        _synth = S
    return _synth


def synth_config(**kw):
    cfg = SynthConfig()
    synth().synth_default_config(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


class SynthHandle:
    """Owns one synthetic frame (host memory) until closed."""

    def __init__(self, **kw):
        self.cfg = synth_config(**kw)
        p = C.POINTER(SynthFrame)()
        rc = synth().synth_create(C.byref(self.cfg), C.byref(p))
        if rc != OK:
            raise ValueError(f"synth_create failed: {rc}")
        self._p = p
        self.f = p.contents

    def close(self):
        if self._p:
            synth().synth_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()

    # geometry helpers
    @property
    def info(self):
        return self.f.info

    def plane_dims(self, p, visible=True):
        i = self.f.info
        sx = i.subsampling_x if p else 0
        sy = i.subsampling_y if p else 0
        return ((i.upscaled_width + sx) >> sx, (i.frame_height + sy) >> sy)


def synth_planes(sf):
    """Copies of a synthetic frame's planes (allocated layout) as numpy arrays."""
    import numpy as np
    f = sf.f
    dt = np.uint8 if f.info.sample_bytes == 1 else np.uint16
    out = []
    for p in range(f.info.num_planes):
        pl = f.planes[p]
        n = pl.height * pl.stride
        buf = (C.c_uint8 * (n * np.dtype(dt).itemsize)).from_address(pl.data)
        out.append(np.frombuffer(buf, dtype=dt).reshape(pl.height, pl.stride).copy())
    return out


def synth_search_planes(sf, seed, amp=None):
    """(reconstruction, source) plane lists for the encoder searches on a
    SynthHandle: the source is the synthetic frame's planes, the
    reconstruction the source plus seeded noise of +-amp (default
    3 << (bit_depth - 8)) in 4x4 blocks and +-amp/2 per sample, clipped to
    the sample range."""
    import numpy as np
    info = sf.f.info
    src = synth_planes(sf)
    rng = np.random.default_rng(seed)
    a = (3 << (info.bit_depth - 8)) if amp is None else amp
    hi = (1 << info.bit_depth) - 1
    cur = []
    for arr in src:
        h, w = arr.shape
        blk = rng.integers(-a, a + 1, size=((h + 3) // 4, (w + 3) // 4))
        fine = rng.integers(-(a // 2), a // 2 + 1, size=(h, w))
        noise = np.kron(blk, np.ones((4, 4), np.int64))[:h, :w] + fine
        cur.append(np.clip(arr.astype(np.int64) + noise, 0, hi).astype(arr.dtype))
    return cur, src


def frame_md5(info, frame):
    """av1pf_frame_md5 of a packed frame (numpy uint8 array)."""
    out = C.create_string_buffer(33)
    check(lib().av1pf_frame_md5(C.byref(info), frame.ctypes.data, out), "av1pf_frame_md5")
    return out.value.decode()


def frame_bytes(info):
    """Bytes of the packed output Frame (frame.rs:135-158) — computed here
    without the library so CPU-only code can size buffers."""
    bps = 2 if info.bit_depth > 8 else 1
    w, h = info.upscaled_width, info.frame_height
    n = w * h
    if info.num_planes > 1:
        sx, sy = info.subsampling_x, info.subsampling_y
        n += 2 * ((w + sx) >> sx) * ((h + sy) >> sy)
    return n * bps


def check(rc, what="av1pf"):
    if rc != OK:
        err = None
        try:
            err = lib().av1pf_last_error()
        except Exception:  # pragma: no cover
            pass
        raise RuntimeError(f"{what} failed with status {rc}: {err.decode() if err else ''}")
