"""A second CPU restatement of two post-filter processes, written from the AV1
Bitstream & Decoding Process Specification's pseudo-code rather than from the
reference's Rust code or from oracle.cpp:

  - 7.15 CDEF process (cdef_block, 7.15.1 cdef_direction, 7.15.2
    cdef_filter with cdef_get_at / is_inside_filter_region / constrain);
  - 7.18.3 film grain synthesis (7.18.3.2 random numbers, 7.18.3.3 grain
    generation, 7.18.3.4 scaling lookup, 7.18.3.5 noise stripes, noise image
    and blending), followed by the packing of the output frame.

TEST INFRASTRUCTURE ONLY: tests/test_spec_check.py compares it with the
oracle's cdef and output processes on small synthetic frames. The oracle and
the CUDA kernels were both written from the reference's Rust code; this file
was written from the specification alone, so a misreading of the reference
that the oracle and the kernels share would show up here as a difference.
It does not pin parity to the reference's binary.

Plain Python and numpy: the per-sample loops are vectorised over 8x8 blocks
(CDEF) and whole planes (grain blending), and the grain templates run as
the specification's scalar loops, so a 352x288 frame takes a few seconds.
Only the specification's constant tables are taken from the library's table
header (av1_tables.h: Cdef_Uv_Dir, Div_Table, Cdef_Directions,
Gaussian_Sequence).
"""
import ctypes as C
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_TABLES = os.path.join(_HERE, "..", "rivet-av1_b200", "csrc", "av1_tables.h")

MI_SIZE = 4
MI_SIZE_LOG2 = 2
CDEF_PRI_TAPS = ((4, 2), (3, 3))
CDEF_SEC_TAPS = ((2, 1), (2, 1))
MC_IDENTITY = 0


def _table(name):
    """A table of av1_tables.h as a numpy array (dims from its _DIMS macro)."""
    txt = open(_TABLES).read()
    dims = [int(d) for d in re.findall(r"\[(\d+)\]", re.search(rf"#define AV1T_{name}_DIMS (.*)", txt).group(1))]
    body = re.search(rf"#define AV1T_{name} (.*)", txt).group(1)
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    return np.array(vals, dtype=np.int64).reshape(dims)


_T = {}


def table(name):
    if name not in _T:
        _T[name] = _table(name)
    return _T[name]


def floor_log2(x):
    return int(x).bit_length() - 1


def round2(x, n):
    """Round2 of the specification (4.7), on ints or int64 arrays."""
    if n == 0:
        return x
    return (x + (1 << (n - 1))) >> n


# ---------------------------------------------------------------------------
# 7.15 CDEF
# ---------------------------------------------------------------------------
def cdef_direction(cur_y, bit_depth, r, c):
    """7.15.1: (yDir, var) of the 8x8 luma block at mode-info (r, c)."""
    div = table("DIV_TABLE")
    x0, y0 = c << MI_SIZE_LOG2, r << MI_SIZE_LOG2
    blk = (cur_y[y0:y0 + 8, x0:x0 + 8].astype(np.int64) >> (bit_depth - 8)) - 128
    partial = np.zeros((8, 15), np.int64)
    for i in range(8):
        for j in range(8):
            x = int(blk[i, j])
            partial[0][i + j] += x
            partial[1][i + j // 2] += x
            partial[2][i] += x
            partial[3][3 + i - j // 2] += x
            partial[4][7 + i - j] += x
            partial[5][3 - i // 2 + j] += x
            partial[6][j] += x
            partial[7][i // 2 + j] += x
    cost = [0] * 8
    for i in range(8):
        cost[2] += int(partial[2][i]) ** 2
        cost[6] += int(partial[6][i]) ** 2
    cost[2] *= int(div[8])
    cost[6] *= int(div[8])
    for i in range(7):
        cost[0] += (int(partial[0][i]) ** 2 + int(partial[0][14 - i]) ** 2) * int(div[i + 1])
        cost[4] += (int(partial[4][i]) ** 2 + int(partial[4][14 - i]) ** 2) * int(div[i + 1])
    cost[0] += int(partial[0][7]) ** 2 * int(div[8])
    cost[4] += int(partial[4][7]) ** 2 * int(div[8])
    for i in range(1, 8, 2):
        for j in range(4 + 1):
            cost[i] += int(partial[i][3 + j]) ** 2
        cost[i] *= int(div[8])
        for j in range(4 - 1):
            cost[i] += (int(partial[i][j]) ** 2 + int(partial[i][10 - j]) ** 2) * int(div[2 * j + 2])
    best_cost, y_dir = 0, 0
    for i in range(8):
        if cost[i] > best_cost:
            best_cost, y_dir = cost[i], i
    var = (best_cost - cost[(y_dir + 4) & 7]) >> 10
    return y_dir, var


def constrain(diff, threshold, damping):
    """constrain() of 7.15.2, vectorised over diff."""
    if not threshold:
        return np.zeros_like(diff)
    adj = max(0, damping - floor_log2(threshold))
    a = np.abs(diff)
    val = np.minimum(a, np.maximum(0, threshold - (a >> adj)))
    return np.sign(diff) * val


def cdef_filter(cur, out, plane, r, c, pri_str, sec_str, damping, direction, fr):
    """7.15.2 on one 8x8 (luma) block's samples of `plane`, vectorised over
    the block: cdef_get_at with is_inside_filter_region per tap."""
    dirs = table("CDEF_DIRECTIONS")
    coeff_shift = fr["bit_depth"] - 8
    sub_x = fr["ss_x"] if plane else 0
    sub_y = fr["ss_y"] if plane else 0
    x0 = (c * MI_SIZE) >> sub_x
    y0 = (r * MI_SIZE) >> sub_y
    w, h = 8 >> sub_x, 8 >> sub_y
    ii, jj = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    src = cur[plane]
    x = src[y0:y0 + h, x0:x0 + w].astype(np.int64)
    total = np.zeros_like(x)
    mx, mn = x.copy(), x.copy()
    pri_tap = CDEF_PRI_TAPS[(pri_str >> coeff_shift) & 1]
    sec_tap = CDEF_SEC_TAPS[(pri_str >> coeff_shift) & 1]

    def get_at(di, dj):
        yy, xx = y0 + ii + di, x0 + jj + dj
        cand_r = (yy << sub_y) >> MI_SIZE_LOG2
        cand_c = (xx << sub_x) >> MI_SIZE_LOG2
        avail = (cand_c >= 0) & (cand_c < fr["mi_cols"]) & (cand_r >= 0) & (cand_r < fr["mi_rows"])
        v = np.zeros_like(x)
        v[avail] = src[yy[avail], xx[avail]]
        return v, avail

    for k in range(2):
        for sign in (-1, 1):
            p, av = get_at(sign * int(dirs[direction][k][0]), sign * int(dirs[direction][k][1]))
            total += np.where(av, pri_tap[k] * constrain(p - x, pri_str, damping), 0)
            mx = np.where(av, np.maximum(p, mx), mx)
            mn = np.where(av, np.minimum(p, mn), mn)
            for off in (-2, 2):
                d2 = (direction + off) & 7
                s, av = get_at(sign * int(dirs[d2][k][0]), sign * int(dirs[d2][k][1]))
                total += np.where(av, sec_tap[k] * constrain(s - x, sec_str, damping), 0)
                mx = np.where(av, np.maximum(s, mx), mx)
                mn = np.where(av, np.minimum(s, mn), mn)
    res = np.clip(x + ((8 + total - (total < 0)) >> 4), mn, mx)
    out[plane][y0:y0 + h, x0:x0 + w] = res


def cdef_frame(cur, fr, skip, cdef_idx, strengths):
    """7.15: CdefFrame from CurrFrame (`cur`, a list of int64 planes) over
    the mode-info area. `skip[r][c]` is the skip flag per mode-info unit,
    `cdef_idx[r >> 4][c >> 4]` the index per 64x64 (-1: not filtered),
    `strengths` holds cdef_damping and the y/uv primary and secondary
    strengths (secondary 3 already read as 4)."""
    out = [p.copy() for p in cur]
    bd = fr["bit_depth"]
    coeff_shift = bd - 8
    uv_dir = table("CDEF_UV_DIR")
    for r in range(0, fr["mi_rows"], 2):
        for c in range(0, fr["mi_cols"], 2):
            idx = int(cdef_idx[r >> 4][c >> 4])
            if idx == -1:
                continue
            if skip[r][c] and skip[r + 1][c] and skip[r][c + 1] and skip[r + 1][c + 1]:
                continue
            y_dir, var = cdef_direction(cur[0], bd, r, c)
            pri = strengths["y_pri"][idx] << coeff_shift
            sec = strengths["y_sec"][idx] << coeff_shift
            direction = 0 if pri == 0 else y_dir
            var_str = min(floor_log2(var >> 6), 12) if (var >> 6) else 0
            pri = ((pri * (4 + var_str) + 8) >> 4) if var else 0
            damping = strengths["damping"] + coeff_shift
            cdef_filter(cur, out, 0, r, c, pri, sec, damping, direction, fr)
            if fr["num_planes"] == 1:
                continue
            pri = strengths["uv_pri"][idx] << coeff_shift
            sec = strengths["uv_sec"][idx] << coeff_shift
            direction = 0 if pri == 0 else int(uv_dir[fr["ss_x"]][fr["ss_y"]][y_dir])
            damping = strengths["damping"] + coeff_shift - 1
            cdef_filter(cur, out, 1, r, c, pri, sec, damping, direction, fr)
            cdef_filter(cur, out, 2, r, c, pri, sec, damping, direction, fr)
    return out


# ---------------------------------------------------------------------------
# 7.18.3 film grain synthesis
# ---------------------------------------------------------------------------
class Random:
    """7.18.3.2: the 16-bit random number generator."""

    def __init__(self, seed):
        self.r = seed & 0xffff

    def get(self, bits):
        r = self.r
        bit = ((r >> 0) ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1
        r = (r >> 1) | (bit << 15)
        self.r = r
        return (r >> (16 - bits)) & ((1 << bits) - 1)


def generate_grain(g, bit_depth, mono, sub_x, sub_y):
    """7.18.3.3: LumaGrain, CbGrain, CrGrain."""
    gauss = table("GAUSSIAN_SEQUENCE")
    grain_min = -(128 << (bit_depth - 8))
    grain_max = (256 << (bit_depth - 8)) - 1 - (128 << (bit_depth - 8))
    shift = 12 - bit_depth + g["grain_scale_shift"]
    rng = Random(g["grain_seed"])
    luma = [[0] * 82 for _ in range(73)]
    for y in range(73):
        for x in range(82):
            gv = int(gauss[rng.get(11)]) if g["num_y_points"] > 0 else 0
            luma[y][x] = round2(gv, shift)
    lag = g["ar_coeff_lag"]
    ar_shift = g["ar_coeff_shift_minus_6"] + 6
    for y in range(3, 73):
        for x in range(3, 82 - 3):
            s, pos = 0, 0
            done = False
            for dr in range(-lag, 1):
                for dc in range(-lag, lag + 1):
                    if dr == 0 and dc == 0:
                        done = True
                        break
                    s += luma[y + dr][x + dc] * (g["ar_coeffs_y_plus_128"][pos] - 128)
                    pos += 1
                if done:
                    break
            luma[y][x] = min(grain_max, max(grain_min, luma[y][x] + round2(s, ar_shift)))
    cb = [[0] * 82 for _ in range(73)]
    cr = [[0] * 82 for _ in range(73)]
    if not mono:
        chroma_w = 44 if sub_x else 82
        chroma_h = 38 if sub_y else 73
        for seed_xor, arr, npts in ((0xb524, cb, g["num_cb_points"]), (0x49d8, cr, g["num_cr_points"])):
            rng = Random(g["grain_seed"] ^ seed_xor)
            for y in range(chroma_h):
                for x in range(chroma_w):
                    gv = int(gauss[rng.get(11)]) if (npts > 0 or g["chroma_scaling_from_luma"]) else 0
                    arr[y][x] = round2(gv, shift)
        for y in range(3, chroma_h):
            for x in range(3, chroma_w - 3):
                s0 = s1 = pos = 0
                done = False
                for dr in range(-lag, 1):
                    for dc in range(-lag, lag + 1):
                        c0 = g["ar_coeffs_cb_plus_128"][pos] - 128
                        c1 = g["ar_coeffs_cr_plus_128"][pos] - 128
                        if dr == 0 and dc == 0:
                            if g["num_y_points"] > 0:
                                lv = 0
                                lx = ((x - 3) << sub_x) + 3
                                ly = ((y - 3) << sub_y) + 3
                                for i in range(sub_y + 1):
                                    for j in range(sub_x + 1):
                                        lv += luma[ly + i][lx + j]
                                lv = round2(lv, sub_x + sub_y)
                                s0 += lv * c0
                                s1 += lv * c1
                            done = True
                            break
                        s0 += cb[y + dr][x + dc] * c0
                        s1 += cr[y + dr][x + dc] * c1
                        pos += 1
                    if done:
                        break
                cb[y][x] = min(grain_max, max(grain_min, cb[y][x] + round2(s0, ar_shift)))
                cr[y][x] = min(grain_max, max(grain_min, cr[y][x] + round2(s1, ar_shift)))
    return (np.array(luma, np.int64), np.array(cb, np.int64), np.array(cr, np.int64))


def scaling_lookup(g, num_planes):
    """7.18.3.4: ScalingLut[plane][0..255]."""
    lut = np.zeros((3, 256), np.int64)
    for plane in range(num_planes):
        if plane == 0 or g["chroma_scaling_from_luma"]:
            n, xs, ys = g["num_y_points"], g["point_y_value"], g["point_y_scaling"]
        elif plane == 1:
            n, xs, ys = g["num_cb_points"], g["point_cb_value"], g["point_cb_scaling"]
        else:
            n, xs, ys = g["num_cr_points"], g["point_cr_value"], g["point_cr_scaling"]
        if n == 0:
            continue
        for x in range(xs[0]):
            lut[plane][x] = ys[0]
        for i in range(n - 1):
            dy = ys[i + 1] - ys[i]
            dx = xs[i + 1] - xs[i]
            delta = dy * ((65536 + (dx >> 1)) // dx)
            for x in range(dx):
                lut[plane][xs[i] + x] = ys[i] + ((x * delta + 32768) >> 16)
        for x in range(xs[n - 1], 256):
            lut[plane][x] = ys[n - 1]
    return lut


def add_noise(planes, g, bit_depth, mono, sub_x, sub_y, w, h, matrix_coefficients):
    """7.18.3.5 on the output planes (int64 arrays, cropped to the visible
    area; modified and returned)."""
    num_planes = 1 if mono else 3
    grains = generate_grain(g, bit_depth, mono, sub_x, sub_y)
    lut = scaling_lookup(g, num_planes)
    grain_min = -(128 << (bit_depth - 8))
    grain_max = (256 << (bit_depth - 8)) - 1 - (128 << (bit_depth - 8))
    overlap = g["overlap_flag"]
    # noise stripes: [stripe][plane] -> (34 >> sub_y rows, wide enough) arrays
    stripes = []
    luma_num = 0
    for y in range(0, (h + 1) // 2, 16):
        rng = Random(g["grain_seed"])
        rng.r ^= ((luma_num * 37 + 178) & 255) << 8
        rng.r ^= (luma_num * 173 + 105) & 255
        st = []
        for plane in range(num_planes):
            psx = sub_x if plane else 0
            psy = sub_y if plane else 0
            st.append(np.zeros((34 >> psy, (((w + 1) // 2 + 16) * 2 >> psx) + 34), np.int64))
        for x in range(0, (w + 1) // 2, 16):
            rand = rng.get(8)
            off_x, off_y = rand >> 4, rand & 15
            for plane in range(num_planes):
                psx = sub_x if plane else 0
                psy = sub_y if plane else 0
                pox = 6 + off_x if psx else 9 + off_x * 2
                poy = 6 + off_y if psy else 9 + off_y * 2
                gr = grains[plane]
                ns = st[plane]
                for i in range(34 >> psy):
                    for j in range(34 >> psx):
                        gv = int(gr[poy + i][pox + j])
                        if psx == 0:
                            if j < 2 and overlap and x > 0:
                                old = int(ns[i][x * 2 + j])
                                gv = old * 27 + gv * 17 if j == 0 else old * 17 + gv * 27
                                gv = min(grain_max, max(grain_min, round2(gv, 5)))
                            ns[i][x * 2 + j] = gv
                        else:
                            if j == 0 and overlap and x > 0:
                                old = int(ns[i][x + j])
                                gv = old * 23 + gv * 22
                                gv = min(grain_max, max(grain_min, round2(gv, 5)))
                            ns[i][x + j] = gv
        stripes.append(st)
        luma_num += 1
    # noise image
    noise = []
    for plane in range(num_planes):
        psx = sub_x if plane else 0
        psy = sub_y if plane else 0
        ph, pw = (h + psy) >> psy, (w + psx) >> psx
        img = np.zeros((ph, pw), np.int64)
        for y in range(ph):
            ln = y >> (5 - psy)
            i = y - (ln << (5 - psy))
            row = stripes[ln][plane][i][:pw].copy()
            if psy == 0:
                if i < 2 and ln > 0 and overlap:
                    old = stripes[ln - 1][plane][i + 32][:pw]
                    row = old * 27 + row * 17 if i == 0 else old * 17 + row * 27
                    row = np.clip(round2(row, 5), grain_min, grain_max)
            else:
                if i < 1 and ln > 0 and overlap:
                    old = stripes[ln - 1][plane][i + 16][:pw]
                    row = np.clip(round2(old * 23 + row * 22, 5), grain_min, grain_max)
            img[y] = row
        noise.append(img)

    def scale_lut(plane, index):
        shift = bit_depth - 8
        x = index >> shift
        rem = index - (x << shift)
        start = lut[plane][x]
        if bit_depth == 8:
            return start
        end = lut[plane][np.minimum(x + 1, 255)]
        return np.where(x == 255, start, start + round2((end - start) * rem, shift))

    if g["clip_to_restricted_range"]:
        min_value = 16 << (bit_depth - 8)
        max_luma = 235 << (bit_depth - 8)
        max_chroma = max_luma if matrix_coefficients == MC_IDENTITY else 240 << (bit_depth - 8)
    else:
        min_value = 0
        max_luma = max_chroma = (256 << (bit_depth - 8)) - 1
    scaling_shift = g["grain_scaling_minus_8"] + 8
    out_y = planes[0]
    if not mono:
        ph, pw = (h + sub_y) >> sub_y, (w + sub_x) >> sub_x
        yy, xx = np.meshgrid(np.arange(ph), np.arange(pw), indexing="ij")
        lx, ly = xx << sub_x, yy << sub_y
        lnx = np.minimum(lx + 1, w - 1)
        avg = round2(out_y[ly, lx] + out_y[ly, lnx], 1) if sub_x else out_y[ly, lx]
        for plane, npts, mult, lmult, offset in ((1, g["num_cb_points"], g["cb_mult"], g["cb_luma_mult"],
                                                  g["cb_offset"]),
                                                 (2, g["num_cr_points"], g["cr_mult"], g["cr_luma_mult"],
                                                  g["cr_offset"])):
            if not (npts > 0 or g["chroma_scaling_from_luma"]):
                continue
            orig = planes[plane]
            if g["chroma_scaling_from_luma"]:
                merged = avg
            else:
                combined = avg * (lmult - 128) + orig * (mult - 128)
                merged = np.clip((combined >> 6) + ((offset - 256) << (bit_depth - 8)), 0, (1 << bit_depth) - 1)
            nz = round2(scale_lut(plane, merged) * noise[plane], scaling_shift)
            planes[plane] = np.clip(orig + nz, min_value, max_chroma)
    if g["num_y_points"] > 0:
        nz = round2(scale_lut(0, out_y) * noise[0], scaling_shift)
        planes[0] = np.clip(out_y + nz, min_value, max_luma)
    return planes


def grain_params(fg):
    """The av1pf_film_grain struct as a dict of ints / lists."""
    d = {}
    for name, _ in fg._fields_:
        v = getattr(fg, name)
        d[name] = list(v) if isinstance(v, C.Array) else int(v)
    return d


def output_frame(info, params, ref_planes):
    """Decoder::output's result from the reference frame: the visible area of
    each plane, film grain (7.18.3) when applied, packed Y, U, V with
    stride = width, u8 at 8-bit and little-endian u16 above."""
    w, h = info.upscaled_width, info.frame_height
    mono = info.num_planes == 1
    planes = []
    for p in range(info.num_planes):
        sx = info.subsampling_x if p else 0
        sy = info.subsampling_y if p else 0
        planes.append(ref_planes[p][:(h + sy) >> sy, :(w + sx) >> sx].astype(np.int64))
    if params.film_grain.apply:
        planes = add_noise(planes, grain_params(params.film_grain), info.bit_depth, mono, info.subsampling_x,
                           info.subsampling_y, w, h, info.matrix_coefficients)
    dt = np.uint8 if info.bit_depth == 8 else np.dtype("<u2")
    return np.concatenate([p.astype(dt).reshape(-1).view(np.uint8) for p in planes])
