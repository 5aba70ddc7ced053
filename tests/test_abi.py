"""The C ABI library loads and exports every entry point include/*.h declares,
and its host-side validation (no device needed) behaves like the reference's
limits. CPU only."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import av1pf as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(av1pf_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", A.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_and_binds_every_symbol():
    L = A.lib()  # ctypes resolves every declared function; raises if one is missing
    for name in declared_functions():
        assert hasattr(L, name)


def test_struct_sizes_match_header():
    assert C.sizeof(A.Mi) == 8
    assert C.sizeof(A.LrUnit) == 12
    assert C.sizeof(A.Plane) == 24


def test_struct_layouts_match_the_compiled_header(tmp_path):
    """sizeof and field offsets of the ABI structs, as gcc lays them out
    from include/av1pf.h, equal the Python bindings'."""
    structs = {"av1pf_frame_info": (A.FrameInfo, []), "av1pf_params": (A.Params, ["film_grain"]),
               "av1pf_film_grain": (A.FilmGrain, ["ar_coeff_shift_minus_6", "clip_to_restricted_range"]),
               "av1pf_maps": (A.Maps, ["cdef_idx", "lr_units"]), "av1pf_plane": (A.Plane, ["height"]),
               "av1pf_host_job": (A.HostJob, ["frame_out"]), "av1pf_job": (A.Job, ["frame_out"]),
               "av1pf_ref_frame": (A.RefFrame, ["info", "order_hint", "frame_id", "planes"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "av1pf.h"', "int main(void) {"]
    for name, (_, fields) in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fld in fields:
            lines.append(f'  printf("{name}.{fld} %zu\\n", offsetof({name}, {fld}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for name, (cls, fields) in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fld in fields:
            assert int(got[f"{name}.{fld}"]) == getattr(cls, fld).offset, f"{name}.{fld}"


def test_validate_accepts_synthetic_frames():
    for kw in [dict(width=1920, height=1080, bit_depth=10), dict(width=352, height=288, bit_depth=8, sample_bytes=1),
               dict(width=640, height=360, bit_depth=12, subsampling_x=0, subsampling_y=0, superres_denom=12,
                    enable_grain=1)]:
        s = A.SynthHandle(**kw)
        assert A.lib().av1pf_validate(C.byref(s.f.info), C.byref(s.f.params), s.f.planes) == A.OK


@pytest.mark.parametrize("field,value", [("bit_depth", 9), ("num_planes", 2), ("mi_rows", 3), ("sample_bytes", 1),
                                         ("upscaled_width", 10)])
def test_validate_rejects_bad_info(field, value):
    s = A.SynthHandle(width=128, height=64, bit_depth=10)
    info = A.FrameInfo.from_buffer_copy(s.f.info)
    setattr(info, field, value)
    assert A.lib().av1pf_validate(C.byref(info), C.byref(s.f.params), s.f.planes) == A.ERR_INVALID_INPUT


def test_validate_rejects_bad_params_and_planes():
    s = A.SynthHandle(width=128, height=64, bit_depth=10, enable_grain=1)
    L = A.lib()
    for mutate in [lambda p: setattr(p, "cdef_damping", 7),
                   lambda p: p.loop_filter_level.__setitem__(0, 64),
                   lambda p: p.lr_unit_cols.__setitem__(0, 99),
                   lambda p: p.loop_restoration_size.__setitem__(0, 48),
                   lambda p: setattr(p.film_grain, "ar_coeff_lag", 4),
                   lambda p: p.film_grain.point_y_value.__setitem__(1, 0)]:
        p = A.Params.from_buffer_copy(s.f.params)
        mutate(p)
        assert L.av1pf_validate(C.byref(s.f.info), C.byref(p), s.f.planes) == A.ERR_INVALID_INPUT
    planes = (A.Plane * 3)(*s.f.planes)
    planes[0].width = 64  # smaller than the mode-info area + 8
    assert L.av1pf_validate(C.byref(s.f.info), C.byref(s.f.params), planes) == A.ERR_INVALID_INPUT
    planes = (A.Plane * 3)(*s.f.planes)
    planes[1].data = planes[1].data + 2  # misaligned
    assert L.av1pf_validate(C.byref(s.f.info), C.byref(s.f.params), planes) == A.ERR_INVALID_INPUT
    # 4:4:0 is not an AV1 format
    info = A.FrameInfo.from_buffer_copy(s.f.info)
    info.subsampling_x = 0
    assert L.av1pf_validate(C.byref(info), None, None) == A.ERR_UNSUPPORTED


def test_frame_bytes_matches_frame_layout():
    s = A.SynthHandle(width=127, height=65, bit_depth=10)
    # frame.rs:135-158: Y w*h, chroma ((w+1)/2)*((h+1)/2) each, 2 bytes at >8 bits
    assert A.lib().av1pf_frame_bytes(C.byref(s.f.info)) == (127 * 65 + 2 * 64 * 33) * 2
    assert A.frame_bytes(s.f.info) == A.lib().av1pf_frame_bytes(C.byref(s.f.info))


def test_ctx_create_without_gpu_fails_cleanly():
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a device is present")
    p = C.c_void_p()
    rc = A.lib().av1pf_ctx_create(0, 0, C.byref(p))
    assert rc != A.OK and not p.value
