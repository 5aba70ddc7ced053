/*
 * synth.cpp — seeded synthetic inputs for the post-filter chain.
 *
 * Shapes and value distributions follow the measured configurations: a
 * random partition of each 64x64 superblock into valid blocks, a transform
 * tree per block that tiles it (lf_tx_size per plane, chroma from the block
 * that has chroma, as residual.rs:160-170 writes it), random skip / intra /
 * inter / segment / delta-lf per block, loop-filter levels U[0,63], sharpness
 * U[0,7], 8 CDEF presets (pri 0..15, sec {0,1,2,4}, damping 3..6) with one
 * preset per 64x64 (-1 where the 64x64 is all skip, as tile.rs:1013-1040
 * leaves it), LR units of one type each (none / Wiener with taps in the
 * specification ranges, chroma outer tap 0 / self-guided set 0..15 with the
 * radius-0 xqd rule of tile.rs:429-452), optional superres and film grain.
 * Integer arithmetic only, so every host produces identical frames.
 */
#include "synth.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <unordered_map>
#include <vector>

#include "../csrc/av1_tables.h"

namespace {

const uint8_t SUBSAMPLED_SIZE AV1T_SUBSAMPLED_SIZE_DIMS = AV1T_SUBSAMPLED_SIZE;
const uint8_t TX_WIDTH AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH;
const uint8_t TX_HEIGHT AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT;
const uint8_t NUM_4X4_BLOCKS_WIDE AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE;
const uint8_t NUM_4X4_BLOCKS_HIGH AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH;
const uint8_t MAX_TX_SIZE_RECT AV1T_MAX_TX_SIZE_RECT_DIMS = AV1T_MAX_TX_SIZE_RECT;
const uint8_t SPLIT_TX_SIZE AV1T_SPLIT_TX_SIZE_DIMS = AV1T_SPLIT_TX_SIZE;
const int32_t SGR_PARAMS AV1T_SGR_PARAMS_DIMS = AV1T_SGR_PARAMS;
const int32_t SGRPROJ_XQD_MIN AV1T_SGRPROJ_XQD_MIN_DIMS = AV1T_SGRPROJ_XQD_MIN;
const int32_t SGRPROJ_XQD_MAX AV1T_SGRPROJ_XQD_MAX_DIMS = AV1T_SGRPROJ_XQD_MAX;
const int32_t WIENER_TAPS_MIN AV1T_WIENER_TAPS_MIN_DIMS = AV1T_WIENER_TAPS_MIN;
const int32_t WIENER_TAPS_MAX AV1T_WIENER_TAPS_MAX_DIMS = AV1T_WIENER_TAPS_MAX;

constexpr int BLOCK_INVALID = 22;

// Block size from log2 width/height in samples (BLOCK_* of consts.rs:117-140).
int block_of(int wl, int hl) {
  static const int8_t t[5][5] = {
      // h:  4   8  16  32  64
      {0, 1, 16, -1, -1},   // w 4
      {2, 3, 4, 18, -1},    // w 8
      {17, 5, 6, 7, 20},    // w 16
      {-1, 19, 8, 9, 10},   // w 32
      {-1, -1, 21, 11, 12}, // w 64
  };
  if (wl < 2 || hl < 2 || wl > 6 || hl > 6) return -1;
  return t[wl - 2][hl - 2];
}

struct Rng {  // splitmix64
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  int32_t uni(int32_t lo, int32_t hi) {  // inclusive
    return lo + int32_t(next() % uint64_t(hi - lo + 1));
  }
  bool pct(int p) { return int(next() % 100) < p; }
};

// Irwin-Hall (12 uniforms) approximation of N(0, 1), scaled by 256.
struct GaussTable {
  int16_t v[4096];
  GaussTable() {
    Rng r{0x5eedull};
    for (auto& x : v) {
      int64_t s = 0;
      for (int i = 0; i < 12; i++) s += int64_t(r.next() & 0xffff);
      // sum has mean 6*65536 and sd 65536 (sd of U[0,N) is N/sqrt(12)).
      x = int16_t(((s - 6 * 65536) * 256) / 65536);
    }
  }
};
const GaussTable GAUSS;

struct Owned;
std::mutex g_owned_mu;
std::unordered_map<synth_frame*, Owned*> g_owned;

struct Owned {
  synth_frame f;
  std::vector<av1pf_mi> mi;
  std::vector<uint8_t> tx[3];
  std::vector<int8_t> cdef;
  std::vector<av1pf_lr_unit> lr[3];
  std::vector<uint8_t> planes[3];
  std::vector<int16_t> tx_offset[3];  // per plane 4x4: DC step of its tx block
};

int count_units_in_frame(int unit_size, int frame_size) {  // decoder/mod.rs:1229-1231
  return std::max((frame_size + (unit_size >> 1)) / unit_size, 1);
}

struct Gen {
  const synth_config& c;
  Owned& o;
  Rng rng;
  int mi_rows, mi_cols, ms, ssx, ssy, np;
  int step_amp;

  Gen(const synth_config& cfg, Owned& own, int mr, int mc)
      : c(cfg), o(own), rng{cfg.seed * 0x100000001b3ull + uint64_t(cfg.frame_index) * 0x9e37ull + 1},
        mi_rows(mr), mi_cols(mc), ms(mc + 32), ssx(cfg.subsampling_x), ssy(cfg.subsampling_y),
        np(cfg.mono ? 1 : 3) {
    step_amp = 12 << (cfg.bit_depth - 8);
  }

  void fill_tx(int plane, int x4, int y4, int w4, int h4, int tx) {
    int rows = mi_rows + 32;
    int16_t off = int16_t(rng.uni(-step_amp, step_amp));
    for (int y = y4; y < y4 + h4; y++)
      for (int x = x4; x < x4 + w4; x++)
        if (y < rows && x < ms) {
          o.tx[plane][size_t(y) * size_t(ms) + size_t(x)] = uint8_t(tx);
          o.tx_offset[plane][size_t(y) * size_t(ms) + size_t(x)] = off;
        }
  }

  // A transform tree over a region (in 4x4 units of the plane).
  void tx_tree(int plane, int x4, int y4, int w4, int h4, int tx, int depth, bool uniform, int udepth) {
    bool split;
    if (uniform)
      split = depth < udepth && tx != 0;
    else
      split = depth < 2 && tx != 0 && rng.pct(35);
    if (!split) {
      fill_tx(plane, x4, y4, w4, h4, tx);
      return;
    }
    int sub = SPLIT_TX_SIZE[tx];
    int sw = TX_WIDTH[sub] / 4, sh = TX_HEIGHT[sub] / 4;
    for (int y = y4; y < y4 + h4; y += sh)
      for (int x = x4; x < x4 + w4; x += sw) tx_tree(plane, x, y, sw, sh, sub, depth + 1, uniform, udepth);
  }

  void emit_block(int r, int c_, int wl, int hl) {
    int bsize = block_of(wl, hl);
    int w4 = 1 << (wl - 2), h4 = 1 << (hl - 2);
    bool skip = rng.pct(c.skip_pct);
    bool inter = rng.pct(50);
    av1pf_mi m{};
    m.mi_size = uint8_t(bsize);
    if (inter) {
      m.ref_frame0 = int8_t(rng.uni(1, 7));
      m.y_mode = uint8_t(rng.uni(14, 25));  // NEARESTMV (14) .. NEW_NEWMV (25)
    } else {
      m.ref_frame0 = 0;
      m.y_mode = uint8_t(rng.uni(0, 12));
    }
    uint8_t seg = c.segmentation ? uint8_t(rng.uni(0, 7)) : 0;
    m.skip_segment = uint8_t((skip ? AV1PF_MI_SKIP : 0) | seg);
    if (c.delta_lf) {
      for (int k = 0; k < 4; k++) m.delta_lf[k] = int8_t(rng.uni(-24, 24));
    }
    int rows = mi_rows + 32;
    for (int y = r; y < r + h4; y++)
      for (int x = c_; x < c_ + w4; x++)
        if (y < rows && x < ms) o.mi[size_t(y) * size_t(ms) + size_t(x)] = m;
    // luma transform tree: intra blocks use one size, inter ones a tree
    int tx = MAX_TX_SIZE_RECT[bsize];
    tx_tree(0, c_, r, w4, h4, tx, 0, !inter, rng.uni(0, 2));
    // chroma: only the block that "has chroma" writes it
    if (np > 1) {
      bool has_chroma = !((ssy && h4 == 1 && (r & 1) == 0) || (ssx && w4 == 1 && (c_ & 1) == 0));
      if (has_chroma) {
        int cb = SUBSAMPLED_SIZE[bsize][ssx][ssy];
        int uv_tx = MAX_TX_SIZE_RECT[cb];
        if (TX_WIDTH[uv_tx] == 64 || TX_HEIGHT[uv_tx] == 64) {  // residual.rs:211-225
          if (TX_WIDTH[uv_tx] == 16)
            uv_tx = 9;  // TX_16X32
          else if (TX_HEIGHT[uv_tx] == 16)
            uv_tx = 10;  // TX_32X16
          else
            uv_tx = 3;  // TX_32X32
        }
        int cw4 = NUM_4X4_BLOCKS_WIDE[cb], ch4 = NUM_4X4_BLOCKS_HIGH[cb];
        int cx = c_ >> ssx, cy = r >> ssy;
        for (int p = 1; p < 3; p++) {
          int tw = TX_WIDTH[uv_tx] / 4, th = TX_HEIGHT[uv_tx] / 4;
          for (int y = cy; y < cy + ch4; y += th)
            for (int x = cx; x < cx + cw4; x += tw) fill_tx(p, x, y, std::min(tw, cx + cw4 - x), std::min(th, cy + ch4 - y), uv_tx);
        }
      }
    }
  }

  bool valid_block(int wl, int hl) {
    int b = block_of(wl, hl);
    if (b < 0) return false;
    if (np > 1 && SUBSAMPLED_SIZE[b][ssx][ssy] == BLOCK_INVALID) return false;
    return true;
  }

  // Partition of a square of 2^sl samples at MI (r, c).
  void partition(int r, int c_, int sl) {
    if (r >= mi_rows || c_ >= mi_cols) return;
    int minl = std::max(2, std::min(6, c.min_block_log2));
    int choice = sl <= minl ? 0 : int(rng.next() % 100);
    int half = 1 << (sl - 3);  // half size in MI units
    int q = 1 << (sl - 4 >= 0 ? sl - 4 : 0);
    // 0..24 NONE, 25..59 SPLIT, 60..71 HORZ, 72..83 VERT, 84..91 HORZ_4, 92..99 VERT_4
    if (choice < 25) {
      emit_block(r, c_, sl, sl);
    } else if (choice < 60) {
      partition(r, c_, sl - 1);
      partition(r, c_ + half, sl - 1);
      partition(r + half, c_, sl - 1);
      partition(r + half, c_ + half, sl - 1);
    } else if (choice < 72 && valid_block(sl, sl - 1)) {
      emit_block(r, c_, sl, sl - 1);
      emit_block(r + half, c_, sl, sl - 1);
    } else if (choice < 84 && valid_block(sl - 1, sl)) {
      emit_block(r, c_, sl - 1, sl);
      emit_block(r, c_ + half, sl - 1, sl);
    } else if (choice < 92 && sl >= 4 && valid_block(sl, sl - 2)) {
      for (int i = 0; i < 4; i++) emit_block(r + i * q, c_, sl, sl - 2);
    } else if (sl >= 4 && valid_block(sl - 2, sl)) {
      for (int i = 0; i < 4; i++) emit_block(r, c_ + i * q, sl - 2, sl);
    } else {
      emit_block(r, c_, sl, sl);
    }
  }
};

// Smooth field: bilinear interpolation of a coarse random grid (cell = 2^cl).
struct Field {
  int gw, gh, cl;
  std::vector<int32_t> g;
  Field(Rng& r, int w, int h, int cell_log2, int lo, int hi) : cl(cell_log2) {
    gw = (w >> cl) + 2;
    gh = (h >> cl) + 2;
    g.resize(size_t(gw) * size_t(gh));
    for (auto& v : g) v = r.uni(lo, hi);
  }
  int32_t at(int x, int y) const {
    int gx = x >> cl, gy = y >> cl;
    int fx = x & ((1 << cl) - 1), fy = y & ((1 << cl) - 1);
    int s = 1 << cl;
    int64_t a = g[size_t(gy) * size_t(gw) + size_t(gx)], b = g[size_t(gy) * size_t(gw) + size_t(gx + 1)];
    int64_t cc = g[size_t(gy + 1) * size_t(gw) + size_t(gx)], d = g[size_t(gy + 1) * size_t(gw) + size_t(gx + 1)];
    int64_t top = a * (s - fx) + b * fx, bot = cc * (s - fx) + d * fx;
    return int32_t((top * (s - fy) + bot * fy) >> (2 * cl));
  }
};

void make_planes(const synth_config& c, Owned& o, Rng& rng, int mi_rows, int mi_cols) {
  av1pf_frame_info& info = o.f.info;
  int bd = c.bit_depth;
  int maxv = (1 << bd) - 1;
  int ms = mi_cols + 32;
  int sigma = c.noise_sigma >= 0 ? c.noise_sigma : (c.content == SYNTH_CONTENT_MOVING ? 4 : 8);
  // sigma is stated in 10-bit units for the field content (config: sigma 8
  // at 10 bits) and in 8-bit units for the moving content (sigma 4 at 8 bits).
  int sig_scaled = c.content == SYNTH_CONTENT_MOVING ? (sigma << (bd - 8)) : ((sigma << bd) >> 10);
  if (sig_scaled < 1 && sigma > 0) sig_scaled = 1;
  int aw = (mi_cols * 4 + 127) & ~127, ah = (mi_rows * 4 + 127) & ~127;
  for (int p = 0; p < info.num_planes; p++) {
    int sx = p ? c.subsampling_x : 0, sy = p ? c.subsampling_y : 0;
    int pw = (aw >> sx) + 32, ph = (ah >> sy) + 32;
    size_t sb = size_t(c.sample_bytes);
    o.planes[p].assign(size_t(pw) * size_t(ph) * sb, 0);
    av1pf_plane& pl = o.f.planes[p];
    pl.data = o.planes[p].data();
    pl.stride = pw;
    pl.width = pw;
    pl.height = ph;
    o.f.plane_bytes[p] = int64_t(o.planes[p].size());
    int mid = 1 << (bd - 1);
    Field field(rng, pw, ph, p ? 5 : 6, mid - (mid >> 1), mid + (mid >> 1));
    // moving rectangles (config 1): 4 boxes that move 2 px per frame
    struct Box { int x, y, w, h, v, dx, dy; } boxes[4];
    for (auto& b : boxes) {
      b.w = rng.uni(24, 96) >> sx;
      b.h = rng.uni(24, 96) >> sy;
      b.x = rng.uni(0, std::max(1, (c.width >> sx) - b.w));
      b.y = rng.uni(0, std::max(1, (c.height >> sy) - b.h));
      b.v = rng.uni(0, maxv);
      b.dx = rng.pct(50) ? 2 : -2;
      b.dy = rng.pct(50) ? 2 : -2;
    }
    int gx = rng.uni(1, 4), gy = rng.uni(1, 4);
    for (int y = 0; y < ph; y++) {
      for (int x = 0; x < pw; x++) {
        int32_t v;
        if (c.content == SYNTH_CONTENT_MOVING) {
          v = (maxv / 4) + ((x * gx * (maxv / 2)) / std::max(1, pw * 4)) + ((y * gy * (maxv / 2)) / std::max(1, ph * 4));
          for (auto& b : boxes) {
            int bx = b.x + ((b.dx * c.frame_index) >> sx), by = b.y + ((b.dy * c.frame_index) >> sy);
            if (x >= bx && x < bx + b.w && y >= by && y < by + b.h) v = b.v;
          }
        } else {
          v = field.at(x, y);
          int m4x = x >> 2, m4y = y >> 2;
          if (m4y < mi_rows + 32 && m4x < ms) v += o.tx_offset[p][size_t(m4y) * size_t(ms) + size_t(m4x)];
        }
        v += (int32_t(GAUSS.v[rng.next() & 4095]) * sig_scaled) / 256;
        v = std::max(0, std::min(maxv, v));
        size_t i = size_t(y) * size_t(pw) + size_t(x);
        if (sb == 1)
          o.planes[p][i] = uint8_t(v);
        else
          reinterpret_cast<uint16_t*>(o.planes[p].data())[i] = uint16_t(v);
      }
    }
  }
}

void make_grain(const synth_config& c, av1pf_film_grain& g, Rng& rng, bool mono) {
  std::memset(&g, 0, sizeof(g));
  g.apply = 1;
  g.grain_seed = c.frame_index & 0xffff;
  auto points = [&](int n, int32_t* xs, int32_t* ys) {
    // n distinct increasing values in [0, 255]
    int base = 0;
    for (int i = 0; i < n; i++) {
      int room = 255 - base - (n - 1 - i);
      int step = rng.uni(1, std::max(1, room / (n - i)));
      if (i == 0) step = rng.uni(0, std::max(0, room / n));
      base += step;
      xs[i] = base;
      ys[i] = rng.uni(0, 255);
    }
  };
  g.num_y_points = 14;
  points(14, g.point_y_value, g.point_y_scaling);
  if (!mono) {
    g.num_cb_points = 10;
    points(10, g.point_cb_value, g.point_cb_scaling);
    g.num_cr_points = 10;
    points(10, g.point_cr_value, g.point_cr_scaling);
  }
  g.grain_scaling_minus_8 = rng.uni(0, 3);
  g.ar_coeff_lag = 3;
  for (int i = 0; i < 24; i++) g.ar_coeffs_y_plus_128[i] = rng.uni(0, 255);
  for (int i = 0; i < 25; i++) {
    g.ar_coeffs_cb_plus_128[i] = rng.uni(0, 255);
    g.ar_coeffs_cr_plus_128[i] = rng.uni(0, 255);
  }
  g.ar_coeff_shift_minus_6 = rng.uni(0, 3);
  g.grain_scale_shift = rng.uni(0, 3);
  if (!mono) {
    g.cb_mult = rng.uni(0, 255);
    g.cb_luma_mult = rng.uni(0, 255);
    g.cb_offset = rng.uni(0, 511);
    g.cr_mult = rng.uni(0, 255);
    g.cr_luma_mult = rng.uni(0, 255);
    g.cr_offset = rng.uni(0, 511);
  }
  g.overlap_flag = 1;
  g.clip_to_restricted_range = rng.pct(50);
}

}  // namespace

extern "C" {

void synth_default_config(synth_config* cfg) {
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->width = 1920;
  cfg->height = 1080;
  cfg->bit_depth = 10;
  cfg->sample_bytes = 2;
  cfg->subsampling_x = 1;
  cfg->subsampling_y = 1;
  cfg->superres_denom = 8;
  cfg->content = SYNTH_CONTENT_FIELD;
  cfg->noise_sigma = -1;
  cfg->seed = 1;
  cfg->enable_lf = 1;
  cfg->enable_cdef = 1;
  cfg->enable_lr = 1;
  cfg->enable_grain = 0;
  cfg->lr_unit_shift = 0;
  cfg->lr_uv_shift = 1;
  cfg->min_block_log2 = 2;
  cfg->skip_pct = 30;
}

int synth_create(const synth_config* cfg, synth_frame** out) {
  if (!cfg || !out) return AV1PF_ERR_INVALID_INPUT;
  const synth_config& c = *cfg;
  if (c.width <= 0 || c.height <= 0 || c.width > 16384 || c.height > 16384) return AV1PF_ERR_INVALID_INPUT;
  if (c.bit_depth != 8 && c.bit_depth != 10 && c.bit_depth != 12) return AV1PF_ERR_INVALID_INPUT;
  if (c.sample_bytes != 2 && !(c.sample_bytes == 1 && c.bit_depth == 8)) return AV1PF_ERR_INVALID_INPUT;
  if (c.superres_denom < 8 || c.superres_denom > 16) return AV1PF_ERR_INVALID_INPUT;
  if (c.subsampling_x < 0 || c.subsampling_x > 1 || c.subsampling_y < 0 || c.subsampling_y > 1 ||
      (c.subsampling_y && !c.subsampling_x))
    return AV1PF_ERR_INVALID_INPUT;
  Owned* o = new (std::nothrow) Owned();
  if (!o) return AV1PF_ERR_OOM;
  std::memset(&o->f, 0, sizeof(o->f));
  Rng rng{c.seed * 0x2545f4914f6cdd1dull + uint64_t(c.frame_index) + 7};
  av1pf_frame_info& info = o->f.info;
  info.bit_depth = c.bit_depth;
  info.sample_bytes = c.sample_bytes;
  info.subsampling_x = c.mono ? 1 : c.subsampling_x;
  info.subsampling_y = c.mono ? 1 : c.subsampling_y;
  info.num_planes = c.mono ? 1 : 3;
  info.upscaled_width = c.width;
  // header.rs:718-723: the coded width after superres downscaling
  info.frame_width = c.superres_denom > 8 ? int32_t((uint32_t(c.width) * 8 + uint32_t(c.superres_denom) / 2) / uint32_t(c.superres_denom)) : c.width;
  info.frame_height = c.height;
  info.mi_cols = 2 * ((info.frame_width + 7) >> 3);
  info.mi_rows = 2 * ((info.frame_height + 7) >> 3);
  info.matrix_coefficients = 1;
  int mi_rows = info.mi_rows, mi_cols = info.mi_cols;
  int ms = mi_cols + 32;
  size_t n = size_t(mi_rows + 32) * size_t(ms);
  o->mi.assign(n, av1pf_mi{});
  for (int p = 0; p < 3; p++) {
    o->tx[p].assign(n, 0);
    o->tx_offset[p].assign(n, 0);
  }
  int cdef_stride = (mi_cols >> 4) + 2;
  o->cdef.assign(size_t(cdef_stride) * size_t((mi_rows >> 4) + 2), -1);

  // maps: partition every 64x64 superblock
  synth_config cc = c;
  cc.subsampling_x = info.subsampling_x;
  cc.subsampling_y = info.subsampling_y;
  Gen gen(cc, *o, mi_rows, mi_cols);
  for (int r = 0; r < mi_rows; r += 16)
    for (int col = 0; col < mi_cols; col += 16) gen.partition(r, col, 6);

  av1pf_params& p = o->f.params;
  std::memset(&p, 0, sizeof(p));
  // loop filter (header.rs:938-971)
  if (c.enable_lf) {
    p.loop_filter_level[0] = rng.uni(0, 63);
    p.loop_filter_level[1] = rng.uni(0, 63);
    if (p.loop_filter_level[0] == 0 && p.loop_filter_level[1] == 0) p.loop_filter_level[0] = 1;
    if (info.num_planes > 1) {
      p.loop_filter_level[2] = rng.uni(0, 63);
      p.loop_filter_level[3] = rng.uni(0, 63);
    }
  }
  p.loop_filter_sharpness = rng.uni(0, 7);
  p.loop_filter_delta_enabled = rng.pct(50);
  const int32_t def_ref[8] = {1, 0, 0, 0, -1, 0, -1, -1};  // header.rs:200
  for (int i = 0; i < 8; i++) p.loop_filter_ref_deltas[i] = def_ref[i];
  if (p.loop_filter_delta_enabled && rng.pct(50)) {
    for (int i = 0; i < 8; i++) p.loop_filter_ref_deltas[i] = rng.uni(-12, 12);
    for (int i = 0; i < 2; i++) p.loop_filter_mode_deltas[i] = rng.uni(-12, 12);
  }
  p.delta_lf_multi = c.delta_lf == 2;
  if (c.segmentation) {
    p.segmentation_enabled = 1;
    for (int s = 0; s < 8; s++)
      for (int k = 1; k <= 4; k++) {
        p.feature_enabled[s][k] = rng.pct(50);
        p.feature_data[s][k] = p.feature_enabled[s][k] ? rng.uni(-63, 63) : 0;
      }
  }
  // CDEF (header.rs:972-1002)
  if (c.enable_cdef) {
    p.cdef_enabled = 1;
    p.cdef_damping = rng.uni(3, 6);
    p.cdef_bits = 3;
    const int secs[4] = {0, 1, 2, 4};
    for (int i = 0; i < 8; i++) {
      p.cdef_y_pri_strength[i] = rng.uni(0, 15);
      p.cdef_y_sec_strength[i] = secs[rng.uni(0, 3)];
      if (info.num_planes > 1) {
        p.cdef_uv_pri_strength[i] = rng.uni(0, 15);
        p.cdef_uv_sec_strength[i] = secs[rng.uni(0, 3)];
      }
    }
    // one preset per 64x64, -1 where every block of it is skip
    for (int r = 0; r < mi_rows; r += 16)
      for (int col = 0; col < mi_cols; col += 16) {
        bool all_skip = true;
        for (int y = r; y < std::min(r + 16, mi_rows) && all_skip; y++)
          for (int x = col; x < std::min(col + 16, mi_cols); x++)
            if (!(o->mi[size_t(y) * size_t(ms) + size_t(x)].skip_segment & AV1PF_MI_SKIP)) {
              all_skip = false;
              break;
            }
        o->cdef[size_t(r >> 4) * size_t(cdef_stride) + size_t(col >> 4)] =
            all_skip ? int8_t(-1) : int8_t(rng.uni(0, 7));
      }
  } else {
    p.cdef_damping = 3;
  }
  // superres
  p.use_superres = c.superres_denom > 8;
  // loop restoration (header.rs:1004-1046)
  if (c.enable_lr) {
    p.uses_lr = 1;
    int s0 = 64 << std::max(0, std::min(2, c.lr_unit_shift));
    int uv_shift = (info.subsampling_x && info.subsampling_y) ? (c.lr_uv_shift ? 1 : 0) : 0;
    for (int pl = 0; pl < info.num_planes; pl++) {
      p.frame_restoration_type[pl] = 3;  // RESTORE_SWITCHABLE: per-unit types
      p.loop_restoration_size[pl] = pl ? (s0 >> uv_shift) : s0;
      int sx = pl ? info.subsampling_x : 0, sy = pl ? info.subsampling_y : 0;
      int us = p.loop_restoration_size[pl];
      p.lr_unit_rows[pl] = count_units_in_frame(us, (info.frame_height + sy) >> sy);
      p.lr_unit_cols[pl] = count_units_in_frame(us, (info.upscaled_width + sx) >> sx);
      size_t units = size_t(p.lr_unit_rows[pl]) * size_t(p.lr_unit_cols[pl]);
      o->lr[pl].assign(units, av1pf_lr_unit{});
      for (auto& u : o->lr[pl]) {
        int t = rng.uni(0, 2);
        u.type = uint8_t(t);
        if (t == AV1PF_RESTORE_WIENER) {
          for (int pass = 0; pass < 2; pass++)
            for (int j = 0; j < 3; j++)
              u.wiener[pass][j] = (pl != 0 && j == 0) ? 0 : int8_t(rng.uni(WIENER_TAPS_MIN[j], WIENER_TAPS_MAX[j]));
        } else if (t == AV1PF_RESTORE_SGRPROJ) {
          int set = rng.uni(0, 15);
          u.sgr_set = uint8_t(set);
          int x0 = SGR_PARAMS[set][0] != 0 ? rng.uni(SGRPROJ_XQD_MIN[0], SGRPROJ_XQD_MAX[0]) : 0;
          int x1;
          if (SGR_PARAMS[set][2] != 0)
            x1 = rng.uni(SGRPROJ_XQD_MIN[1], SGRPROJ_XQD_MAX[1]);
          else
            x1 = std::max(SGRPROJ_XQD_MIN[1], std::min(SGRPROJ_XQD_MAX[1], 128 - x0));
          u.sgr_xqd[0] = int8_t(x0);
          u.sgr_xqd[1] = int8_t(x1);
        }
      }
    }
  }
  if (c.enable_grain) make_grain(c, p.film_grain, rng, info.num_planes == 1);

  make_planes(cc, *o, rng, mi_rows, mi_cols);

  av1pf_maps& m = o->f.maps;
  m.mi = o->mi.data();
  m.mi_stride = ms;
  m.cdef_stride = cdef_stride;
  m.cdef_idx = o->cdef.data();
  o->f.mi_count = int64_t(n);
  o->f.cdef_count = int64_t(o->cdef.size());
  for (int pl = 0; pl < 3; pl++) {
    m.lf_tx_size[pl] = pl < info.num_planes ? o->tx[pl].data() : nullptr;
    o->f.tx_count[pl] = pl < info.num_planes ? int64_t(n) : 0;
    m.lr_units[pl] = o->lr[pl].empty() ? nullptr : o->lr[pl].data();
    o->f.lr_count[pl] = int64_t(o->lr[pl].size());
  }
  {
    std::lock_guard<std::mutex> lk(g_owned_mu);
    g_owned[&o->f] = o;
  }
  *out = &o->f;
  return AV1PF_OK;
}

void synth_destroy(synth_frame* f) {
  if (!f) return;
  Owned* o = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_owned_mu);
    auto it = g_owned.find(f);
    if (it == g_owned.end()) return;
    o = it->second;
    g_owned.erase(it);
  }
  delete o;
}

}  // extern "C"
