"""Device-side helpers of the GPU tests: upload a synthetic frame with torch
(device memory only — every computation goes through libav1pf's C ABI) and
read results back as numpy arrays."""
import ctypes as C

import numpy as np

import av1pf as A


def torch():
    import torch as T
    return T


def dev_bytes(n):
    T = torch()
    return T.empty(max(int(n), 1), dtype=T.uint8, device="cuda")


def to_dev(host_ptr, nbytes):
    """Copies nbytes at a host address into a new device byte tensor."""
    T = torch()
    buf = (C.c_uint8 * max(int(nbytes), 1)).from_address(host_ptr) if nbytes else (C.c_uint8 * 1)()
    arr = np.frombuffer(buf, dtype=np.uint8, count=int(nbytes))
    t = dev_bytes(nbytes)
    if nbytes:
        t[: int(nbytes)].copy_(T.from_numpy(arr.copy()))
    return t


def np_dtype(info):
    return np.uint8 if info.sample_bytes == 1 else np.uint16


class DevPlanes:
    """Device planes (one byte tensor per plane) as an av1pf_plane[3]."""

    def __init__(self, info, dims, strides=None):
        self.info = info
        sb = info.sample_bytes
        self.t = []
        self.c = (A.Plane * 3)()
        for p, (w, h) in enumerate(dims):
            stride = strides[p] if strides else (w + 63) // 64 * 64
            t = dev_bytes(stride * h * sb)
            t.zero_()
            self.t.append(t)
            self.c[p].data = t.data_ptr()
            self.c[p].stride = stride
            self.c[p].width = w
            self.c[p].height = h

    @staticmethod
    def visible(info):
        dims = []
        for p in range(info.num_planes):
            sx = info.subsampling_x if p else 0
            sy = info.subsampling_y if p else 0
            dims.append(((info.upscaled_width + sx) >> sx, (info.frame_height + sy) >> sy))
        return DevPlanes(info, dims)

    @staticmethod
    def from_host(info, host_planes):
        """Uploads HostPlanes (oracle.HostPlanes) keeping their geometry."""
        T = torch()
        dims = [(a.shape[1], a.shape[0]) for a in host_planes.arrays]
        d = DevPlanes(info, dims, strides=[a.shape[1] for a in host_planes.arrays])
        for p, a in enumerate(host_planes.arrays):
            d.t[p].copy_(T.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)))
        return d

    def host(self, p, w=None, h=None):
        """Plane p as a (h, w) numpy array (default: its width/height)."""
        pl = self.c[p]
        w = pl.width if w is None else w
        h = pl.height if h is None else h
        a = self.t[p].cpu().numpy().view(np_dtype(self.info)).reshape(pl.height, pl.stride)
        return a[:h, :w].copy()


class DevFrame:
    """A synthetic frame on the device: planes and maps."""

    def __init__(self, sf):
        self.sf = sf
        f = sf.f
        self.info = f.info
        self.params = f.params
        self.keep = []
        m = A.Maps()
        hm = f.maps
        m.mi_stride = hm.mi_stride
        m.cdef_stride = hm.cdef_stride
        t = to_dev(hm.mi, f.mi_count * 8)
        self.keep.append(t)
        m.mi = t.data_ptr()
        for p in range(3):
            if hm.lf_tx_size[p] and f.tx_count[p]:
                t = to_dev(hm.lf_tx_size[p], f.tx_count[p])
                self.keep.append(t)
                m.lf_tx_size[p] = t.data_ptr()
            if hm.lr_units[p] and f.lr_count[p]:
                t = to_dev(hm.lr_units[p], f.lr_count[p] * C.sizeof(A.LrUnit))
                self.keep.append(t)
                m.lr_units[p] = t.data_ptr()
        t = to_dev(hm.cdef_idx, f.cdef_count)
        self.keep.append(t)
        m.cdef_idx = t.data_ptr()
        self.maps = m
        # input planes in the synthetic (reference) layout
        self.inp = DevPlanes(self.info, [(f.planes[p].width, f.planes[p].height) for p in range(self.info.num_planes)],
                             strides=[f.planes[p].stride for p in range(self.info.num_planes)])
        T = torch()
        for p in range(self.info.num_planes):
            n = f.plane_bytes[p]
            src = np.frombuffer((C.c_uint8 * n).from_address(f.planes[p].data), dtype=np.uint8)
            self.inp.t[p].copy_(T.from_numpy(src.copy()))


class Ctx:
    def __init__(self, device=0, cap=0):
        self.p = C.c_void_p()
        A.check(A.lib().av1pf_ctx_create(device, cap, C.byref(self.p)), "ctx_create")

    def close(self):
        if self.p:
            A.lib().av1pf_ctx_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gpu_chain(ctx, df, want_frame=True, stream=None):
    """Runs av1pf_chain; returns (list of ref planes, packed frame bytes)."""
    T = torch()
    info = df.info
    ref = DevPlanes.visible(info)
    fb = dev_bytes(A.frame_bytes(info)) if want_frame else None
    rc = A.lib().av1pf_chain(ctx.p, C.byref(info), C.byref(df.params), C.byref(df.maps), df.inp.c, ref.c,
                             fb.data_ptr() if want_frame else None, stream)
    A.check(rc, "av1pf_chain")
    T.cuda.synchronize()
    refs = [ref.host(p) for p in range(info.num_planes)]
    return refs, (fb[: A.frame_bytes(info)].cpu().numpy() if want_frame else None)
