#!/usr/bin/env python3
"""Extracts the AV1 specification tables the post-filter chain needs from the
reference's ``src/tables.rs`` into ``av1_tables.h`` (committed beside this
script, so builds need no reference tree).

The tables are specification data (AV1 Bitstream & Decoding Process
Specification, section 9.3 and the filter sections), which the reference
transcribes under the specification's names; nothing else of the reference
is read. Each table becomes an initializer macro ``AV1T_<NAME>`` plus its
dimensions, so host code (``static const``) and device code (``__constant__``)
build from the same data.

Usage: python gen_tables.py <path of the reference's src/tables.rs>
"""
import os
import re
import sys

# name -> C element type. Only tables the post-filter chain or the synthetic
# input generator read.
WANTED = {
    "CDEF_DIRECTIONS": "int8_t",
    "CDEF_PRI_TAPS": "int8_t",
    "CDEF_SEC_TAPS": "int8_t",
    "CDEF_UV_DIR": "uint8_t",
    "DIV_TABLE": "int32_t",
    "GAUSSIAN_SEQUENCE": "int16_t",
    "SGR_PARAMS": "int32_t",
    "SGRPROJ_XQD_MIN": "int32_t",
    "SGRPROJ_XQD_MAX": "int32_t",
    "SGRPROJ_XQD_MID": "int32_t",
    "SUBSAMPLED_SIZE": "uint8_t",
    "TX_WIDTH": "uint8_t",
    "TX_HEIGHT": "uint8_t",
    "UPSCALE_FILTER": "int16_t",
    "WIENER_TAPS_MIN": "int32_t",
    "WIENER_TAPS_MAX": "int32_t",
    "WIENER_TAPS_MID": "int32_t",
    "WIENER_TAPS_K": "int32_t",
    "NUM_4X4_BLOCKS_WIDE": "uint8_t",
    "NUM_4X4_BLOCKS_HIGH": "uint8_t",
    "MAX_TX_SIZE_RECT": "uint8_t",
    "SPLIT_TX_SIZE": "uint8_t",
    "REMAP_LR_TYPE": "uint8_t",
}

DECL = re.compile(r"^pub\(crate\) static (\w+): (.+?) = (\[.*\]);\s*$")


def dims_of(rust_type):
    """``[[i32; 2]; 8]`` -> [8, 2] (outermost first)."""
    dims = []
    t = rust_type.strip()
    while t.startswith("["):
        inner = t[1:t.rindex("]")]
        elem, n = inner.rsplit(";", 1)
        dims.append(int(n.strip()))
        t = elem.strip()
    return dims


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: gen_tables.py <path of the reference's src/tables.rs>")
    src = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    out_path = os.path.join(here, "av1_tables.h")
    found = {}
    with open(src) as f:
        for line in f:
            m = DECL.match(line)
            if m and m.group(1) in WANTED:
                found[m.group(1)] = (dims_of(m.group(2)), m.group(3))
    missing = sorted(set(WANTED) - set(found))
    if missing:
        raise SystemExit(f"tables not found: {missing}")
    lines = [
        "/* Generated by gen_tables.py from the AV1 specification tables (as",
        " * transcribed in the reference's src/tables.rs). Do not edit. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
    ]
    for name in sorted(found):
        dims, lit = found[name]
        init = lit.replace("[", "{").replace("]", "}")
        dim_txt = "".join(f"[{d}]" for d in dims)
        lines.append(f"/* {name}{dim_txt}, element {WANTED[name]} */")
        lines.append(f"#define AV1T_{name}_TYPE {WANTED[name]}")
        lines.append(f"#define AV1T_{name}_DIMS {dim_txt}")
        lines.append(f"#define AV1T_{name} {init}")
        lines.append("")
    with open(out_path, "w") as f:
        f.write("\n".join(lines))
    print(f"wrote {out_path} ({len(found)} tables)")


if __name__ == "__main__":
    main()
