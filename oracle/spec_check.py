"""A second CPU restatement of the post-filter processes, written from the
AV1 Bitstream & Decoding Process Specification's pseudo-code rather than from
the reference's Rust code or from oracle.cpp:

  - 7.14 loop filter (edge loop filter, filter size, adaptive filter
    strength and its level selection, filter masks, narrow and wide filters);
  - 7.15 CDEF process (cdef_block, 7.15.1 cdef_direction, 7.15.2
    cdef_filter with cdef_get_at / is_inside_filter_region / constrain);
  - 7.16 super-resolution (upscaling of the CDEF and the pre-CDEF frames);
  - 7.17 loop restoration (per 4x4 block: stripes, units and the source
    sample rule, the Wiener filter with its rounding variables, the
    self-guided box filters and projection);
  - 7.18.3 film grain synthesis (7.18.3.2 random numbers, 7.18.3.3 grain
    generation, 7.18.3.4 scaling lookup, 7.18.3.5 noise stripes, noise image
    and blending), followed by the packing of the output frame;
  - the chain in decode_frame_wrapup's order.

TEST INFRASTRUCTURE ONLY: tests/test_spec_check.py compares it with the
oracle's per-stage and whole-chain processes on small synthetic frames. The
oracle and the CUDA kernels were both written from the reference's Rust
code; this file was written from the specification alone, so a misreading of
the reference that the oracle and the kernels share would show up here as a
difference. It does not pin parity to the reference's binary.

Plain Python and numpy, at the specification's granularity (per edge lane,
per 8x8 CDEF block, per 4x4 restoration block), so frames of a few hundred
samples a side take seconds. Only the specification's constant tables are
taken from the library's table header (av1_tables.h).
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


# ---------------------------------------------------------------------------
# Inputs of the other processes: the ABI's maps and parameters as arrays
# ---------------------------------------------------------------------------
# YMode numbering of av1pf_mi.y_mode (the reference's: UV_CFL_PRED 13 shares
# the intra range, NEARESTMV 14 .. NEW_NEWMV 25)
NEARESTMV, GLOBALMV, GLOBAL_GLOBALMV = 14, 16, 24
RESTORE_NONE, RESTORE_WIENER, RESTORE_SGRPROJ = 0, 1, 2


class Frame:
    """The frame-level inputs of the post-filter processes, read from an
    av1pf_frame_info / av1pf_params / av1pf_maps triple of host pointers."""

    def __init__(self, info, params, maps, f_counts):
        self.info, self.p = info, params
        self.bd = info.bit_depth
        self.ssx, self.ssy = info.subsampling_x, info.subsampling_y
        self.np = info.num_planes
        self.mi_rows, self.mi_cols = info.mi_rows, info.mi_cols
        self.fw, self.fh, self.uw = info.frame_width, info.frame_height, info.upscaled_width
        ms = maps.mi_stride
        self.ms = ms
        mi_count, tx_count, cdef_count, lr_count = f_counts
        raw = np.frombuffer((C.c_uint8 * (mi_count * 8)).from_address(maps.mi), np.uint8).reshape(-1, ms, 8)
        self.mi_size = raw[:, :, 0].astype(np.int64)
        self.y_mode = raw[:, :, 1].astype(np.int64)
        self.ref0 = raw[:, :, 2].view(np.int8).astype(np.int64)
        self.skip = (raw[:, :, 3] & 0x80) != 0
        self.seg = (raw[:, :, 3] & 7).astype(np.int64)
        self.delta_lf = raw[:, :, 4:8].view(np.int8).astype(np.int64)
        self.tx = []
        for k in range(3):
            if maps.lf_tx_size[k] and tx_count[k]:
                a = np.frombuffer((C.c_uint8 * tx_count[k]).from_address(maps.lf_tx_size[k]), np.uint8)
                self.tx.append(a.reshape(-1, ms).astype(np.int64))
            else:
                self.tx.append(None)
        self.cdef_idx = np.frombuffer((C.c_int8 * cdef_count).from_address(maps.cdef_idx),
                                      np.int8).reshape(-1, maps.cdef_stride)
        self.lru = []
        for k in range(3):
            if maps.lr_units[k] and lr_count[k]:
                u = np.frombuffer((C.c_uint8 * (lr_count[k] * 12)).from_address(maps.lr_units[k]),
                                  np.uint8).reshape(-1, 12)
                self.lru.append(u)
            else:
                self.lru.append(None)


def frame_of(sf):
    f = sf.f
    return Frame(f.info, f.params, f.maps, (f.mi_count, list(f.tx_count), f.cdef_count, list(f.lr_count)))


# ---------------------------------------------------------------------------
# 7.14 loop filter
# ---------------------------------------------------------------------------
def filter_strength(fr, row, col, plane, pass_):
    """7.14.4 adaptive_filter_strength with 7.14.5's level selection:
    (lvl, limit, blimit, thresh) of mode-info position (row, col)."""
    p = fr.p
    segment = int(fr.seg[row][col])
    ref = int(fr.ref0[row][col])
    mode = int(fr.y_mode[row][col])
    mode_type = 1 if (mode >= NEARESTMV and mode != GLOBALMV and mode != GLOBAL_GLOBALMV) else 0
    i = pass_ if plane == 0 else plane + 1
    delta_lf = int(fr.delta_lf[row][col][0 if not p.delta_lf_multi else i])
    lvl = min(63, max(0, delta_lf + p.loop_filter_level[i]))
    feature = 1 + i  # SEG_LVL_ALT_LF_Y_V + i
    if p.segmentation_enabled and p.feature_enabled[segment][feature]:
        lvl = min(63, max(0, p.feature_data[segment][feature] + lvl))
    if p.loop_filter_delta_enabled:
        n_shift = lvl >> 5
        if ref <= 0:  # INTRA_FRAME
            lvl += p.loop_filter_ref_deltas[0] << n_shift
        else:
            lvl += (p.loop_filter_ref_deltas[ref] << n_shift) + (p.loop_filter_mode_deltas[mode_type] << n_shift)
        lvl = min(63, max(0, lvl))
    sharp = p.loop_filter_sharpness
    shift = 2 if sharp > 4 else (1 if sharp > 0 else 0)
    limit = min(9 - sharp, max(1, lvl >> shift)) if sharp > 0 else max(1, lvl >> shift)
    blimit = 2 * (lvl + 2) + limit
    thresh = lvl >> 4
    return lvl, limit, blimit, thresh


def sample_filtering(pl, x, y, plane, limit, blimit, thresh, dx, dy, filter_size, bd):
    """7.14.6 on the sample (x, y) of plane array `pl` (int64, in place)."""
    def at(k):
        return int(pl[y + k * dy][x + k * dx])
    shift = bd - 8
    q = [at(k) for k in range(7)] if filter_size >= 16 else [at(k) for k in range(4)]
    pp = [at(-1 - k) for k in range(7)] if filter_size >= 16 else [at(-1 - k) for k in range(4)]
    # 7.14.6.2 filter mask process
    hev = abs(pp[1] - pp[0]) > (thresh << shift) or abs(q[1] - q[0]) > (thresh << shift)
    flen = 4 if filter_size == 4 else (6 if plane else (8 if filter_size == 8 else 16))
    lim, blim = limit << shift, blimit << shift
    mask = abs(pp[1] - pp[0]) <= lim and abs(q[1] - q[0]) <= lim and abs(pp[0] - q[0]) * 2 + abs(pp[1] - q[1]) // 2 <= blim
    if flen >= 6:
        mask = mask and abs(pp[2] - pp[1]) <= lim and abs(q[2] - q[1]) <= lim
    if flen >= 8:
        mask = mask and abs(pp[3] - pp[2]) <= lim and abs(q[3] - q[2]) <= lim
    t = 1 << shift
    flat = False
    if filter_size >= 8:
        flat = abs(pp[1] - pp[0]) <= t and abs(q[1] - q[0]) <= t and abs(pp[2] - pp[0]) <= t and abs(q[2] - q[0]) <= t
        if flen >= 8:
            flat = flat and abs(pp[3] - pp[0]) <= t and abs(q[3] - q[0]) <= t
    flat2 = False
    if filter_size >= 16:
        flat2 = all(abs(pp[k] - pp[0]) <= t and abs(q[k] - q[0]) <= t for k in (6, 5, 4))
    if not mask:
        return
    if filter_size == 4 or not flat:
        # 7.14.6.3 narrow filter
        lo, hi = -(1 << (bd - 1)), (1 << (bd - 1)) - 1

        def c4(v):
            return min(hi, max(lo, v))
        off = 0x80 << shift
        ps1, ps0, qs0, qs1 = pp[1] - off, pp[0] - off, q[0] - off, q[1] - off
        fl = c4(ps1 - qs1) if hev else 0
        fl = c4(fl + 3 * (qs0 - ps0))
        f1 = c4(fl + 4) >> 3
        f2 = c4(fl + 3) >> 3
        pl[y][x] = c4(qs0 - f1) + off
        pl[y - dy][x - dx] = c4(ps0 + f2) + off
        if not hev:
            fr_ = round2(f1, 1)
            pl[y + dy][x + dx] = c4(qs1 - fr_) + off
            pl[y - 2 * dy][x - 2 * dx] = c4(ps1 + fr_) + off
        return
    # 7.14.6.4 wide filter
    log2 = 3 if (filter_size == 8 or not flat2) else 4
    n = 6 if log2 == 4 else (3 if plane == 0 else 2)
    n2 = 0 if (log2 == 3 and plane == 0) else 1
    src = {k: at(k) for k in range(-(n + 1), n + 1)}
    out = {}
    for i in range(-n, n):
        tot = 0
        for j in range(-n, n + 1):
            pos = min(n, max(-(n + 1), i + j))
            tot += src[pos] * (2 if abs(j) <= n2 else 1)
        out[i] = round2(tot, log2)
    for i, v in out.items():
        pl[y + i * dy][x + i * dx] = v


def loop_filter(planes, fr):
    """7.14.1: both passes over every plane whose level is set, in place,
    in raster order (vertical edges of the plane first)."""
    sub = table("SUBSAMPLED_SIZE")
    n4w, n4h = table("NUM_4X4_BLOCKS_WIDE"), table("NUM_4X4_BLOCKS_HIGH")
    txw, txh = table("TX_WIDTH"), table("TX_HEIGHT")
    p = fr.p
    if not (p.loop_filter_level[0] or p.loop_filter_level[1]):
        return planes
    for plane in range(fr.np):
        if plane and not p.loop_filter_level[1 + plane]:
            continue
        sx = fr.ssx if plane else 0
        sy = fr.ssy if plane else 0
        pl = planes[plane]
        for pass_ in range(2):
            dx, dy = (1, 0) if pass_ == 0 else (0, 1)
            for row0 in range(0, fr.mi_rows, 1 << sy):
                for col0 in range(0, fr.mi_cols, 1 << sx):
                    x, y = col0 * 4, row0 * 4
                    if x >= fr.fw or y >= fr.fh or (pass_ == 0 and x == 0) or (pass_ == 1 and y == 0):
                        continue
                    xp, yp = x >> sx, y >> sy
                    row, col = row0 | sy, col0 | sx
                    prev_row, prev_col = row - (dy << sy), col - (dx << sx)
                    plane_size = int(sub[fr.mi_size[row][col]][sx][sy])
                    tx_sz = int(fr.tx[plane][row >> sy][col >> sx])
                    prev_tx = int(fr.tx[plane][prev_row >> sy][prev_col >> sx])
                    skip = bool(fr.skip[row][col])
                    is_intra = fr.ref0[row][col] <= 0
                    if pass_ == 0:
                        block_edge = xp % (4 * int(n4w[plane_size])) == 0
                        tx_edge = xp % int(txw[tx_sz]) == 0
                        base = min(int(txw[prev_tx]), int(txw[tx_sz]))
                    else:
                        block_edge = yp % (4 * int(n4h[plane_size])) == 0
                        tx_edge = yp % int(txh[tx_sz]) == 0
                        base = min(int(txh[prev_tx]), int(txh[tx_sz]))
                    apply = tx_edge and (block_edge or not skip or is_intra)
                    size = min(16 if plane == 0 else 8, base)
                    lvl, limit, blimit, thresh = filter_strength(fr, row, col, plane, pass_)
                    if lvl == 0:
                        lvl, limit, blimit, thresh = filter_strength(fr, prev_row, prev_col, plane, pass_)
                    if not apply or lvl == 0:
                        continue
                    for i in range(4):
                        sample_filtering(pl, xp + dy * i, yp + dx * i, plane, limit, blimit, thresh, dx, dy, size,
                                         fr.bd)
    return planes


# ---------------------------------------------------------------------------
# 7.16 super-resolution
# ---------------------------------------------------------------------------
def _div_trunc(a, b):
    """Integer division truncating toward zero (the specification's /)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def upscale(planes, fr):
    """7.16: the upscaled planes (frame_width -> upscaled_width)."""
    flt = table("UPSCALE_FILTER")
    out = []
    for plane in range(fr.np):
        sx = fr.ssx if plane else 0
        sy = fr.ssy if plane else 0
        down_w = round2(fr.fw, sx)
        up_w = round2(fr.uw, sx)
        ph = round2(fr.fh, sy)
        step = _div_trunc((down_w << 14) + up_w // 2, up_w)
        err = up_w * step - (down_w << 14)
        init = _div_trunc(-((up_w - down_w) << 13) + up_w // 2, up_w) + (1 << 7) - _div_trunc(err, 2)
        init &= (1 << 14) - 1
        max_x = (fr.mi_cols >> sx) * 4 - 1
        src = planes[plane]
        xs = np.arange(up_w, dtype=np.int64)
        src_x = -(1 << 14) + init + xs * step
        px = src_x >> 14
        phase = (src_x & ((1 << 14) - 1)) >> 8
        res = np.zeros((ph, up_w), np.int64)
        for k in range(8):
            sxk = np.clip(px + k - 3, 0, max_x)
            res += src[:ph, sxk] * flt[phase, k][None, :]
        dst = np.zeros((src.shape[0], max(up_w, src.shape[1])), np.int64)
        dst[:ph, :up_w] = np.clip(round2(res, 7), 0, (1 << fr.bd) - 1)
        out.append(dst)
    return out


# ---------------------------------------------------------------------------
# 7.17 loop restoration
# ---------------------------------------------------------------------------
def count_units(unit_size, frame_size):
    return max((frame_size + (unit_size >> 1)) // unit_size, 1)


def loop_restoration(cdef_up, cur_up, fr):
    """7.17: LrFrame from UpscaledCdefFrame (`cdef_up`) with the stripe
    boundary rows taken from UpscaledCurrFrame (`cur_up`), block by block."""
    p = fr.p
    lr = [a.copy() for a in cdef_up]
    if not p.uses_lr:
        return lr
    sgr = table("SGR_PARAMS")
    bd = fr.bd
    maxv = (1 << bd) - 1
    for plane in range(fr.np):
        if p.frame_restoration_type[plane] == RESTORE_NONE:
            continue
        sx = fr.ssx if plane else 0
        sy = fr.ssy if plane else 0
        unit_size = p.loop_restoration_size[plane]
        unit_rows = count_units(unit_size, round2(fr.fh, sy))
        unit_cols = count_units(unit_size, round2(fr.uw, sx))
        pex, pey = round2(fr.uw, sx) - 1, round2(fr.fh, sy) - 1
        units = fr.lru[plane]
        cd, cu = cdef_up[plane], cur_up[plane]
        for y_l in range(0, fr.fh, 4):
            row = y_l >> 2
            stripe = (row * 4 + 8) // 64
            ss = (-8 + stripe * 64) >> sy
            se = ss + (64 >> sy) - 1
            unit_row = min(unit_rows - 1, ((row * 4 + 8) >> sy) // unit_size)
            y = (row * 4) >> sy
            h = min(4 >> sy, pey - y + 1)
            if h <= 0:
                continue
            # the rows this block reads (3 above and below, the stripe rule per row)
            src_rows = {}
            for yy in range(y - 4, y + h + 4):
                yc = min(pey, max(0, yy))
                if yc < ss:
                    src_rows[yy] = cu[max(ss - 2, yc)]
                elif yc > se:
                    src_rows[yy] = cu[min(se + 2, yc)]
                else:
                    src_rows[yy] = cd[yc]
            for x_l in range(0, fr.uw, 4):
                col = x_l >> 2
                unit_col = min(unit_cols - 1, ((col * 4) >> sx) // unit_size)
                x = (col * 4) >> sx
                w = min(4 >> sx, pex - x + 1)
                if w <= 0:
                    continue
                u = units[unit_row * unit_cols + unit_col]
                rtype = int(u[0])
                cols = np.clip(np.arange(x - 4, x + w + 4), 0, pex)

                def window(r0, r1):
                    """Source samples of rows y+r0 .. y+r1-1, columns x-4 .. x+w+3."""
                    return np.array([src_rows[y + r][cols] for r in range(r0, r1)], np.int64)
                if rtype == RESTORE_WIENER:
                    coef = u[4:10].view(np.int8).astype(np.int64).reshape(2, 3)  # [0] vertical, [1] horizontal

                    def filt(c3):
                        f = np.zeros(7, np.int64)
                        f[3] = 128
                        for i in range(3):
                            f[i] = f[6 - i] = c3[i]
                            f[3] -= 2 * c3[i]
                        return f
                    vf, hf = filt(coef[0]), filt(coef[1])
                    r0 = 5 if bd == 12 else 3
                    r1 = 9 if bd == 12 else 11
                    offset = 1 << (bd + 7 - r0 - 1)
                    limit = (1 << (bd + 1 + 7 - r0)) - 1
                    win = window(-3, h + 3)  # h + 6 rows
                    inter = np.zeros((h + 6, w), np.int64)
                    for c in range(w):
                        s = sum(hf[t] * win[:, c + 4 + t - 3] for t in range(7))
                        inter[:, c] = np.clip(round2(s, r0), -offset, limit - offset)
                    out = np.zeros((h, w), np.int64)
                    for r in range(h):
                        s = sum(vf[t] * inter[r + t] for t in range(7))
                        out[r] = np.clip(round2(s, r1), 0, maxv)
                    lr[plane][y:y + h, x:x + w] = out
                elif rtype == RESTORE_SGRPROJ:
                    st = int(u[1]) & 15
                    xqd = u[2:4].view(np.int8).astype(np.int64)
                    win = window(-4, h + 4)  # rows y-4 .. y+h+3, cols x-4 .. x+w+3

                    def box_filter(pass_):
                        r = int(sgr[st][2 * pass_])
                        eps = int(sgr[st][2 * pass_ + 1])
                        n = (2 * r + 1) ** 2
                        n2e = n * n * eps
                        s = ((1 << 20) + n2e // 2) // n2e
                        one_over_n = ((1 << 12) + n // 2) // n
                        A = np.zeros((h + 2, w + 2), np.int64)
                        B = np.zeros((h + 2, w + 2), np.int64)
                        for i in range(-1, h + 1):
                            for j in range(-1, w + 1):
                                blk = win[4 + i - r:4 + i + r + 1, 4 + j - r:4 + j + r + 1]
                                a = round2(int((blk * blk).sum()), 2 * (bd - 8))
                                b = int(blk.sum())
                                d = round2(b, bd - 8)
                                pp = max(0, a * n - d * d)
                                z = round2(pp * s, 20)
                                if z >= 255:
                                    a2 = 256
                                elif z == 0:
                                    a2 = 1
                                else:
                                    a2 = ((z << 8) + z // 2) // (z + 1)
                                A[i + 1][j + 1] = a2
                                B[i + 1][j + 1] = round2((256 - a2) * b * one_over_n, 12)
                        F = np.zeros((h, w), np.int64)
                        for i in range(h):
                            shift = 4 if (pass_ == 0 and (i & 1)) else 5
                            for j in range(w):
                                a = b = 0
                                for ddy in (-1, 0, 1):
                                    for ddx in (-1, 0, 1):
                                        if pass_ == 0:
                                            wt = (6 if ddx == 0 else 5) if ((i + ddy) & 1) else 0
                                        else:
                                            wt = 4 if (ddx == 0 or ddy == 0) else 3
                                        a += wt * int(A[i + 1 + ddy][j + 1 + ddx])
                                        b += wt * int(B[i + 1 + ddy][j + 1 + ddx])
                                v = a * int(cd[y + i][x + j]) + b
                                F[i][j] = round2(v, 8 + shift - 4)
                        return F
                    rr0, rr1 = int(sgr[st][0]), int(sgr[st][2])
                    flt0 = box_filter(0) if rr0 else None
                    flt1 = box_filter(1) if rr1 else None
                    w0, w1 = int(xqd[0]), int(xqd[1])
                    w2 = (1 << 7) - w0 - w1
                    uu = cd[y:y + h, x:x + w] << 4
                    v = w1 * uu
                    v = v + (w0 * flt0 if rr0 else w0 * uu)
                    v = v + (w2 * flt1 if rr1 else w2 * uu)
                    lr[plane][y:y + h, x:x + w] = np.clip(round2(v, 11), 0, maxv)
    return lr


# ---------------------------------------------------------------------------
# The whole chain (decode_frame_wrapup's order) and the output process
# ---------------------------------------------------------------------------
def chain(sf, in_planes):
    """The chain from the pre-filter planes (int64 arrays in the frame's
    allocated layout): loop filter, CDEF, upscaling of the CDEF and the
    pre-CDEF frames, loop restoration; returns (LR frame planes cropped to
    the visible area, packed output frame)."""
    fr = frame_of(sf)
    p = fr.p
    cur = loop_filter([a.astype(np.int64).copy() for a in in_planes], fr)
    if p.cdef_enabled:
        skip = fr.skip[: fr.mi_rows, : fr.mi_cols]
        strengths = dict(damping=p.cdef_damping, y_pri=list(p.cdef_y_pri_strength),
                         y_sec=list(p.cdef_y_sec_strength), uv_pri=list(p.cdef_uv_pri_strength),
                         uv_sec=list(p.cdef_uv_sec_strength))
        frd = dict(bit_depth=fr.bd, ss_x=fr.ssx, ss_y=fr.ssy, mi_rows=fr.mi_rows, mi_cols=fr.mi_cols,
                   num_planes=fr.np)
        cdef = cdef_frame(cur, frd, skip, fr.cdef_idx, strengths)
    else:
        cdef = cur
    if p.use_superres and fr.uw != fr.fw:
        cdef_up, cur_up = upscale(cdef, fr), upscale(cur, fr)
    else:
        cdef_up, cur_up = cdef, cur
    lr = loop_restoration(cdef_up, cur_up, fr)
    vis = []
    for plane in range(fr.np):
        sx = fr.ssx if plane else 0
        sy = fr.ssy if plane else 0
        vis.append(lr[plane][: round2(fr.fh, sy), : round2(fr.uw, sx)].copy())
    return vis, output_frame(sf.f.info, p, vis)
