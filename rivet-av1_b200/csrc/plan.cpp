// plan.cpp — validation, scratch layout, descriptors and work lists of the
// post-filter chain (see plan.h).
#include "plan.h"

#include <algorithm>
#include <cstring>

#include "kernels.h"

namespace av1pf {

namespace {

constexpr int kTile = 64;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int count_units_in_frame(int unit_size, int frame_size) {  // decoder/mod.rs:1229-1231
  return std::max((frame_size + (unit_size >> 1)) / unit_size, 1);
}

bool fail(std::string* why, const char* msg) {
  if (why) *why = msg;
  return false;
}

// Scratch bump allocator (offsets from a base that may be null while sizing).
struct Bump {
  uint8_t* base;
  size_t used = 0;
  uint8_t* take(size_t bytes) {
    used = align_up(used, 256);
    uint8_t* p = base ? base + used : nullptr;
    used += bytes;
    return p;
  }
  DPlane plane(int w, int h, int sb) {
    DPlane d{};
    d.stride = int64_t(align_up(size_t(w), 64));
    d.w = w;
    d.h = h;
    d.p = take(size_t(d.stride) * size_t(h) * size_t(sb));
    return d;
  }
};

DPlane from_abi(const av1pf_plane& p) {
  DPlane d{};
  d.p = static_cast<uint8_t*>(p.data);
  d.stride = p.stride;
  d.w = p.width;
  d.h = p.height;
  return d;
}

void add_tiles(std::vector<Item>& v, int frame, int plane, uint8_t kind, int w, int h, int tw, int th) {
  for (int y = 0; y < h; y += th)
    for (int x = 0; x < w; x += tw) {
      Item it{};
      it.frame = uint16_t(frame);
      it.plane = uint8_t(plane);
      it.kind = kind;
      it.x0 = uint16_t(x);
      it.y0 = uint16_t(y);
      it.x1 = uint16_t(std::min(x + tw, w));
      it.y1 = uint16_t(std::min(y + th, h));
      v.push_back(it);
    }
}

}  // namespace

size_t packed_frame_bytes(const av1pf_frame_info* i) {
  const size_t bps = i->bit_depth > 8 ? 2 : 1;
  size_t n = 0;
  for (int p = 0; p < i->num_planes; p++)
    n += size_t(plane_w(i, p, i->upscaled_width)) * size_t(plane_h(i, p));
  return n * bps;
}

int validate_frame(const av1pf_frame_info* i, const av1pf_params* params, const av1pf_plane* planes,
                   std::string* why) {
  if (!i) return fail(why, "null frame info"), AV1PF_ERR_INVALID_INPUT;
  if (i->bit_depth != 8 && i->bit_depth != 10 && i->bit_depth != 12)
    return fail(why, "bit_depth must be 8, 10 or 12"), AV1PF_ERR_INVALID_INPUT;
  if (i->sample_bytes != 2 && !(i->sample_bytes == 1 && i->bit_depth == 8))
    return fail(why, "sample_bytes must be 2, or 1 at 8-bit"), AV1PF_ERR_INVALID_INPUT;
  if (i->num_planes != 1 && i->num_planes != 3) return fail(why, "num_planes must be 1 or 3"), AV1PF_ERR_INVALID_INPUT;
  if (i->subsampling_x < 0 || i->subsampling_x > 1 || i->subsampling_y < 0 || i->subsampling_y > 1 ||
      (i->subsampling_y && !i->subsampling_x))
    return fail(why, "subsampling must be 4:2:0, 4:2:2 or 4:4:4"), AV1PF_ERR_UNSUPPORTED;
  if (i->frame_width <= 0 || i->frame_height <= 0 || i->upscaled_width < i->frame_width)
    return fail(why, "bad frame size"), AV1PF_ERR_INVALID_INPUT;
  if (i->upscaled_width > 16384 || i->frame_height > 16384)
    return fail(why, "frame larger than 16384"), AV1PF_ERR_UNSUPPORTED;
  if (i->mi_cols != 2 * ((i->frame_width + 7) >> 3) || i->mi_rows != 2 * ((i->frame_height + 7) >> 3))
    return fail(why, "mi_rows/mi_cols do not match the frame size"), AV1PF_ERR_INVALID_INPUT;
  if (params) {
    const int rc = validate_params(i, params, why);
    if (rc != AV1PF_OK) return rc;
  }
  if (planes) {
    for (int p = 0; p < i->num_planes; p++) {
      const av1pf_plane& pl = planes[p];
      const int sx = p ? i->subsampling_x : 0, sy = p ? i->subsampling_y : 0;
      if (!pl.data) return fail(why, "null plane"), AV1PF_ERR_INVALID_INPUT;
      if ((reinterpret_cast<uintptr_t>(pl.data) & 15) || ((pl.stride * i->sample_bytes) & 15))
        return fail(why, "planes and rows must be 16-byte aligned"), AV1PF_ERR_INVALID_INPUT;
      if (pl.stride < pl.width) return fail(why, "stride < width"), AV1PF_ERR_INVALID_INPUT;
      // the filters read up to 8 samples past the mode-info area (postfilter.rs:178-184,
      // 421-422, 540-541); the reference allocates 32 more (decoder/mod.rs:562-567)
      if (pl.width < ((i->mi_cols * 4) >> sx) + 8 || pl.height < ((i->mi_rows * 4) >> sy) + 8)
        return fail(why, "plane smaller than the mode-info area + 8"), AV1PF_ERR_INVALID_INPUT;
    }
  }
  return AV1PF_OK;
}

int validate_params(const av1pf_frame_info* i, const av1pf_params* p, std::string* why) {
  for (int k = 0; k < 4; k++)
    if (p->loop_filter_level[k] < 0 || p->loop_filter_level[k] > 63)
      return fail(why, "loop_filter_level out of range"), AV1PF_ERR_INVALID_INPUT;
  if (p->loop_filter_sharpness < 0 || p->loop_filter_sharpness > 7)
    return fail(why, "sharpness out of range"), AV1PF_ERR_INVALID_INPUT;
  if (p->cdef_enabled) {
    if (p->cdef_damping < 3 || p->cdef_damping > 6) return fail(why, "cdef_damping out of range"), AV1PF_ERR_INVALID_INPUT;
    for (int k = 0; k < 8; k++) {
      if (p->cdef_y_pri_strength[k] < 0 || p->cdef_y_pri_strength[k] > 15 || p->cdef_uv_pri_strength[k] < 0 ||
          p->cdef_uv_pri_strength[k] > 15 || p->cdef_y_sec_strength[k] < 0 || p->cdef_y_sec_strength[k] > 4 ||
          p->cdef_uv_sec_strength[k] < 0 || p->cdef_uv_sec_strength[k] > 4)
        return fail(why, "cdef strength out of range"), AV1PF_ERR_INVALID_INPUT;
    }
  }
  if (!p->use_superres && i->frame_width != i->upscaled_width)
    return fail(why, "frame_width != upscaled_width without superres"), AV1PF_ERR_INVALID_INPUT;
  if (p->use_superres && 2 * i->frame_width < i->upscaled_width)
    return fail(why, "superres ratio out of range"), AV1PF_ERR_INVALID_INPUT;
  if (p->uses_lr) {
    for (int k = 0; k < i->num_planes; k++) {
      if (p->frame_restoration_type[k] < 0 || p->frame_restoration_type[k] > 3)
        return fail(why, "frame_restoration_type out of range"), AV1PF_ERR_INVALID_INPUT;
      if (p->frame_restoration_type[k] == 0) continue;
      const int us = p->loop_restoration_size[k];
      if (us != 32 && us != 64 && us != 128 && us != 256)
        return fail(why, "loop_restoration_size must be 32..256"), AV1PF_ERR_INVALID_INPUT;
      const int sx = k ? i->subsampling_x : 0, sy = k ? i->subsampling_y : 0;
      if (p->lr_unit_rows[k] != count_units_in_frame(us, (i->frame_height + sy) >> sy) ||
          p->lr_unit_cols[k] != count_units_in_frame(us, (i->upscaled_width + sx) >> sx))
        return fail(why, "lr unit counts do not match count_units_in_frame"), AV1PF_ERR_INVALID_INPUT;
    }
  }
  const av1pf_film_grain& g = p->film_grain;
  if (g.apply) {
    if (g.num_y_points < 0 || g.num_y_points > 14 || g.num_cb_points < 0 || g.num_cb_points > 10 ||
        g.num_cr_points < 0 || g.num_cr_points > 10 || g.ar_coeff_lag < 0 || g.ar_coeff_lag > 3 ||
        g.grain_scaling_minus_8 < 0 || g.grain_scaling_minus_8 > 3 || g.ar_coeff_shift_minus_6 < 0 ||
        g.ar_coeff_shift_minus_6 > 3 || g.grain_scale_shift < 0 || g.grain_scale_shift > 3)
      return fail(why, "film grain parameter out of range"), AV1PF_ERR_INVALID_INPUT;
    auto increasing = [](const int32_t* v, int n) {
      for (int k = 0; k < n; k++)
        if (v[k] < 0 || v[k] > 255 || (k > 0 && v[k] <= v[k - 1])) return false;
      return true;
    };
    if (!increasing(g.point_y_value, g.num_y_points) || !increasing(g.point_cb_value, g.num_cb_points) ||
        !increasing(g.point_cr_value, g.num_cr_points))
      return fail(why, "film grain points must increase (header.rs:1254,1280-1281)"), AV1PF_ERR_INVALID_INPUT;
  }
  return AV1PF_OK;
}

int build_plan(const FrameJob* jobs, int n, uint8_t* scratch_base, Plan& plan, std::string* why, bool items) {
  plan.frames.clear();
  plan.scratch_bytes = 0;
  if (items) {
    // the lists keep their capacity from call to call (a chain call plans
    // one frame of the same shape again and again)
    for (auto* v : {&plan.lf_items, &plan.lft_items, &plan.lff_items, &plan.cdef_items, &plan.sr_items,
                    &plan.lr_items, &plan.grain_items, &plan.out_items, &plan.copy_items})
      v->clear();
    plan.edge_cap = 0;
    plan.any_hlist = false;
    plan.any_lfh = false;
    plan.cdef_half = false;
    plan.sr_row_max = 0;
    plan.any_lf = plan.any_cdef = plan.any_sr = plan.any_lr = plan.any_grain = plan.any_out = false;
    plan.off_frames = plan.off_lf = plan.off_lft = plan.off_lff = plan.off_cdef = plan.off_sr = plan.off_lr = plan.off_grain =
        plan.off_out = plan.off_copy = plan.off_edges_v = plan.off_edges_h = plan.off_counts = plan.meta_bytes =
            plan.upload_bytes = 0;
  }
  if (n <= 0 || n > 65535) return fail(why, "bad job count"), AV1PF_ERR_INVALID_INPUT;
  Bump bump{scratch_base};
  uint32_t cap = 0;
  // readiness flags (FrameDesc::lf_flag_base ...): their count, and whether every
  // frame's stages fit them
  size_t nflags = 0;
  bool flags_fit = true;
  for (int fi = 0; fi < n; fi++) {
    const FrameJob& j = jobs[fi];
    const av1pf_frame_info* i = j.info;
    const av1pf_params* p = j.params;
    FrameDesc d;
    std::memset(&d, 0, sizeof(d));
    d.bd = i->bit_depth;
    d.sb = i->sample_bytes;
    d.ssx = i->subsampling_x;
    d.ssy = i->subsampling_y;
    d.np = i->num_planes;
    d.fw = i->frame_width;
    d.fh = i->frame_height;
    d.uw = i->upscaled_width;
    d.mi_rows = i->mi_rows;
    d.mi_cols = i->mi_cols;
    d.mc = i->matrix_coefficients;
    if (j.maps) {
      d.mi = j.maps->mi;
      d.mi_stride = j.maps->mi_stride;
      d.cdef_idx = j.maps->cdef_idx;
      d.cdef_stride = j.maps->cdef_stride;
      for (int k = 0; k < 3; k++) {
        d.tx[k] = j.maps->lf_tx_size[k];
        d.lru[k] = j.maps->lr_units[k];
      }
    }
    // parameters
    for (int k = 0; k < 4; k++) d.lf_level[k] = p->loop_filter_level[k];
    d.sharpness = p->loop_filter_sharpness;
    d.delta_enabled = p->loop_filter_delta_enabled;
    d.delta_lf_multi = p->delta_lf_multi;
    for (int k = 0; k < 8; k++) d.ref_deltas[k] = p->loop_filter_ref_deltas[k];
    for (int k = 0; k < 2; k++) d.mode_deltas[k] = p->loop_filter_mode_deltas[k];
    d.seg_enabled = p->segmentation_enabled;
    for (int s = 0; s < 8; s++)
      for (int k = 0; k < 4; k++) {
        d.seg_lf_on[s][k] = p->feature_enabled[s][1 + k];  // SEG_LVL_ALT_LF_Y_V + i
        d.seg_lf_data[s][k] = p->feature_data[s][1 + k];
      }
    d.cdef_damping = p->cdef_damping;
    for (int k = 0; k < 8; k++) {
      d.cdef_y_pri[k] = p->cdef_y_pri_strength[k];
      d.cdef_y_sec[k] = p->cdef_y_sec_strength[k];
      d.cdef_uv_pri[k] = p->cdef_uv_pri_strength[k];
      d.cdef_uv_sec[k] = p->cdef_uv_sec_strength[k];
    }
    d.stripes = (i->frame_height + 8 + 63) / 64;
    d.lr_on = p->uses_lr;
    for (int k = 0; k < 3; k++) {
      d.lr_type[k] = p->frame_restoration_type[k];
      d.lr_unit_size[k] = p->loop_restoration_size[k];
      d.lr_unit_rows[k] = p->lr_unit_rows[k];
      d.lr_unit_cols[k] = p->lr_unit_cols[k];
    }
    d.g = p->film_grain;

    const int np = i->num_planes, sb = i->sample_bytes;
    const bool chain = (j.stages & ST_CHAIN) == ST_CHAIN;
    // --- loop filter: postfilter.rs:67-70, decoder/mod.rs:748 ---
    const bool lf_frame = (j.stages & ST_LF) && (p->loop_filter_level[0] || p->loop_filter_level[1]);
    // horizontal edges inside the CDEF kernel: needs the chain's copy of the
    // input (cur is not the caller's) and a CDEF pass to carry them
    const bool tiles = !j.in_place_lf && (j.lf_mode == 1 || j.lf_mode == 2);
    const bool fused = !j.in_place_lf && j.lf_mode == 3;
    const bool fuse_h = lf_frame && chain && tiles && j.lf_mode == 2 && (j.stages & ST_CDEF) && p->cdef_enabled;
    for (int k = 0; k < np; k++) {
      d.in[k] = from_abi(j.in[k]);
      const bool lf_plane = lf_frame && (k == 0 || p->loop_filter_level[1 + k] != 0);
      if (!lf_plane) {
        d.cur[k] = d.in[k];
        continue;
      }
      if (fused) {
        // one flag per 64x64 tile of the fused kernel
        const int tx = (d.in[k].w + kTile - 1) / kTile, ty = (d.in[k].h + kTile - 1) / kTile;
        d.lf_flag_base[k] = int32_t(nflags);
        d.lf_tiles_x[k] = tx;
        nflags += size_t(tx) * size_t(ty);
      } else {
        flags_fit = false;
      }
      plan.any_lf = true;
      const int sx = k ? d.ssx : 0, sy = k ? d.ssy : 0;
      const int gw = i->mi_cols >> sx, gh = i->mi_rows >> sy;
      if (j.in_place_lf) {
        d.cur[k] = d.in[k];
        if (items) add_tiles(plan.lf_items, fi, k, 2, gw * 4, gh * 4, kTile, kTile);
      } else if (fused) {
        // copy in -> cur with both passes filtered per tile
        d.cur[k] = bump.plane(d.in[k].w, d.in[k].h, sb);
        const int W = d.in[k].w, H = d.in[k].h;
        for (int y = 0; items && y < H; y += kTile)
          for (int x = 0; x < W; x += kTile) {
            Item it{};
            it.frame = uint16_t(fi);
            it.plane = uint8_t(k);
            it.kind = uint8_t(1 | ((x < gw * 4 && y < gh * 4) ? 2 : 0));
            it.x0 = uint16_t(x);
            it.y0 = uint16_t(y);
            it.x1 = uint16_t(std::min(x + kTile, W));
            it.y1 = uint16_t(std::min(y + kTile, H));
            plan.lff_items.push_back(it);
          }
      } else if (!tiles) {
        // copy in -> cur and decide every 4x4 edge into the two edge lists
        d.cur[k] = bump.plane(d.in[k].w, d.in[k].h, sb);
        const int W = d.in[k].w, H = d.in[k].h;
        for (int y = 0; items && y < H; y += kTile)
          for (int x = 0; x < W; x += kTile) {
            Item it{};
            it.frame = uint16_t(fi);
            it.plane = uint8_t(k);
            it.kind = uint8_t(1 | ((x < gw * 4 && y < gh * 4) ? 2 : 0));
            it.x0 = uint16_t(x);
            it.y0 = uint16_t(y);
            it.x1 = uint16_t(std::min(x + kTile, W));
            it.y1 = uint16_t(std::min(y + kTile, H));
            if (items) plan.lf_items.push_back(it);
          }
        plan.any_hlist = true;
      } else {
        // copy in -> cur with the vertical edges filtered per tile; the
        // horizontal edges go to the edge list
        d.cur[k] = bump.plane(d.in[k].w, d.in[k].h, sb);
        const int W = d.in[k].w, H = d.in[k].h;
        for (int y = 0; items && y < H; y += kTile)
          for (int x = 0; x < W; x += kTile) {
            Item it{};
            it.frame = uint16_t(fi);
            it.plane = uint8_t(k);
            it.kind = uint8_t(1 | ((x < gw * 4 && y < gh * 4) ? (fuse_h ? 2 : 2 | 4) : 0));
            it.x0 = uint16_t(x);
            it.y0 = uint16_t(y);
            it.x1 = uint16_t(std::min(x + kTile, W));
            it.y1 = uint16_t(std::min(y + kTile, H));
            if (items) plan.lft_items.push_back(it);
          }
        if (fuse_h) {
          d.lfh_mask |= 1 << k;
          if (d.stripes > 1) d.prelf[k] = bump.plane(d.in[k].w, (d.stripes - 1) * 4, sb);
        } else {
          plan.any_hlist = true;
        }
      }
      if (j.in_place_lf) plan.any_hlist = true;
      cap += uint32_t(gw) * uint32_t(gh);
    }
    // --- CDEF: postfilter.rs:273-301 ---
    const bool cdef_stage = j.stages & ST_CDEF;
    if (cdef_stage && !chain) {
      // av1pf_cdef: cur = the given planes, output = the caller's planes
      for (int k = 0; k < np; k++) d.cur[k] = from_abi(j.in[k]);
    }
    const bool cdef_on = cdef_stage && p->cdef_enabled;
    if (!cdef_on) flags_fit = false;  // loop restoration would read the loop filter's output unflagged
    for (int k = 0; k < np; k++) {
      if (cdef_on)
        d.cdef[k] = chain ? bump.plane(d.cur[k].w, d.cur[k].h, sb) : from_abi(j.out[k]);
      else
        d.cdef[k] = d.cur[k];
    }
    if (cdef_on) {
      plan.any_cdef = true;
      const int sbr = (i->mi_rows + 15) / 16, sbc = (i->mi_cols + 15) / 16;
      if (d.lfh_mask) plan.any_lfh = true;
      // one flag per half superblock
      d.cdef_flag_base = int32_t(nflags);
      d.cdef_sbc = sbc;
      nflags += size_t(2 * sbr) * size_t(sbc);
      if (d.lfh_mask || !chain) flags_fit = false;
      for (int r = 0; items && r < sbr; r++)
        for (int c = 0; c < sbc; c++) {
          Item it{};
          it.frame = uint16_t(fi);
          it.kind = uint8_t(d.lfh_mask ? 1 : 0);
          it.x0 = uint16_t(c);
          it.y0 = uint16_t(r);
          plan.cdef_items.push_back(it);
        }
    } else if (cdef_stage && !chain) {
      // the reference returns a clone of cur when CDEF is off: copy the MI area
      for (int k = 0; k < np; k++) {
        d.in[k] = d.cur[k];
        d.cur[k] = from_abi(j.out[k]);
        const int sx = k ? d.ssx : 0, sy = k ? d.ssy : 0;
        if (items) add_tiles(plan.copy_items, fi, k, 1, (i->mi_cols * 4) >> sx, (i->mi_rows * 4) >> sy, kTile, kTile);
      }
    }
    // --- superres: postfilter.rs:521-566, decoder/mod.rs:752-757 ---
    const bool sr_stage = (j.stages & ST_SR) && p->use_superres;
    if ((j.stages & ST_SR) && !chain) {
      for (int k = 0; k < np; k++) d.cdef[k] = from_abi(j.in[k]);
    }
    for (int k = 0; k < np; k++) {
      const int sx = k ? d.ssx : 0;
      const int64_t down = (i->frame_width + sx) >> sx, up = (i->upscaled_width + sx) >> sx;
      const int64_t step = ((down << 14) + up / 2) / up;
      const int64_t err = up * step - (down << 14);
      int64_t init = (-((up - down) << 13) + up / 2) / up + (1 << 7) - err / 2;
      init &= 0x3fff;
      d.sr_step[k] = int32_t(step);
      d.sr_init[k] = int32_t(init);
      d.sr_maxx[k] = (i->mi_cols >> sx) * 4 - 1;
      d.sr_w[k] = int32_t(up);
    }
    d.sr_on = sr_stage && chain ? 1 : 0;
    for (int k = 0; k < np; k++) {
      const int ph = plane_h(i, k);
      if (sr_stage) {
        plan.any_sr = true;
        d.up[k] = chain ? bump.plane(d.sr_w[k], ph, sb) : from_abi(j.out[k]);
        if (items) add_tiles(plan.sr_items, fi, k, 0, 1, ph, 1, 4);
        plan.sr_row_max = std::max(plan.sr_row_max, d.sr_maxx[k] + 1);
        if (chain && d.stripes > 1) {
          const int lines = (d.stripes - 1) * 4;
          d.lines[k] = bump.plane(d.sr_w[k], lines, sb);
          if (items) add_tiles(plan.sr_items, fi, k, 1, 1, lines, 1, 4);
        }
      } else {
        d.up[k] = d.cdef[k];
      }
    }
    // --- loop restoration: postfilter.rs:608-716 ---
    if (j.stages & ST_LR) {
      plan.any_lr = true;
      if (!chain) {
        for (int k = 0; k < np; k++) {
          d.up[k] = from_abi(j.in[k]);
          d.cur[k] = from_abi(j.cur[k]);
        }
      }
      for (int k = 0; k < np; k++) {
        d.ref[k] = from_abi(j.out[k]);
        const int pex = plane_w(i, k, i->upscaled_width) - 1;
        const bool has_lr = p->uses_lr && p->frame_restoration_type[k] != 0;
        const int us = has_lr ? p->loop_restoration_size[k] : 1 << 30;
        const int ucols = has_lr ? p->lr_unit_cols[k] : 1;
        const int rw = j.lr_cols == 32 ? 32 : kTile;  // rectangle width (the kernel takes <= 64)
        for (int s = 0; items && s < d.stripes; s++) {
          const int sy = k ? d.ssy : 0;
          const int ss = (-8 + s * 64) >> sy;
          const int y0 = std::max(ss, 0), y1 = std::min(ss + (64 >> sy) - 1, plane_h(i, k) - 1);
          if (y0 > y1) continue;
          for (int uc = 0; uc < ucols; uc++) {
            // lr_unit_cols (postfilter.rs:664-675)
            const int x0 = uc * std::min(us, 1 << 20);
            const int x1 = uc + 1 == ucols ? pex : std::min((uc + 1) * us - 1, pex);
            if (x0 > pex) continue;
            for (int cx = x0; cx <= x1; cx += rw) {
              Item it{};
              it.frame = uint16_t(fi);
              it.plane = uint8_t(k);
              it.x0 = uint16_t(cx);
              it.x1 = uint16_t(std::min(cx + rw, x1 + 1));
              it.a = uint16_t(s);
              it.b = uint16_t(uc);
              if (items) plan.lr_items.push_back(it);
            }
          }
        }
      }
    }
    // --- output: decoder/mod.rs:846-917 ---
    if ((j.stages & ST_OUT) && j.frame_out) {
      if (!chain)
        for (int k = 0; k < np; k++) d.ref[k] = from_abi(j.in[k]);
      d.frame_out = j.frame_out;
      // a whole chain without film grain packs inside the loop-restoration
      // kernel, which writes every visible sample of the reference frame
      d.lr_pack = chain && !p->film_grain.apply ? 1 : 0;
      const int64_t bps = i->bit_depth > 8 ? 2 : 1;
      int64_t off = 0;
      for (int k = 0; k < np; k++) {
        d.out_off[k] = off;
        const int pw = plane_w(i, k, i->upscaled_width), ph = plane_h(i, k);
        off += int64_t(pw) * ph * bps;
        // 256 columns by one noise stripe (32 rows, 16 in vertically subsampled chroma)
        if (!d.lr_pack) {
          plan.any_out = true;
          if (items) add_tiles(plan.out_items, fi, k, 0, pw, ph, 256, k ? 32 >> i->subsampling_y : 32);
        }
      }
      if (p->film_grain.apply) {
        plan.any_grain = true;
        d.grain_on = 1;
        d.grain = reinterpret_cast<GrainScratch*>(bump.take(sizeof(GrainScratch)));
        d.grain_ns = ((i->frame_height + 1) / 2 + 15) / 16;
        d.grain_nb = ((i->upscaled_width + 1) / 2 + 15) / 16;
        d.grain_off = bump.take(size_t(d.grain_ns) * size_t(d.grain_nb));
        Item it{};
        it.frame = uint16_t(fi);
        if (items) plan.grain_items.push_back(it);
      }
    }
    plan.frames.push_back(d);
  }
  plan.scratch_bytes = align_up(bump.used, 256);
  if (!items) return AV1PF_OK;  // the lists and their layout are the previous call's
  plan.flag_sync = flags_fit && plan.any_lf && plan.any_cdef && plan.any_lr && !plan.any_sr && !plan.any_hlist &&
                   plan.lf_items.empty() && plan.lft_items.empty() && plan.copy_items.empty();
  plan.n_flags = plan.flag_sync ? nflags : 0;
  // At most one wave of superblocks (4 CTAs on each SM): CDEF runs a CTA per
  // half superblock instead, so the SMs end up with equal shares.
  plan.cdef_half = !plan.cdef_items.empty() && plan.cdef_items.size() <= size_t(kNumSMs) * 4;
  if (plan.cdef_half) {
    std::vector<Item> halves;
    halves.reserve(plan.cdef_items.size() * 2);
    for (const Item& it : plan.cdef_items) {
      for (int half = 0; half < 2; half++) {
        // the bottom half of a superblock row past the mode-info area is empty
        if (it.y0 * 16 + half * 8 >= jobs[it.frame].info->mi_rows) continue;
        Item h = it;
        h.a = uint16_t(half);
        halves.push_back(h);
      }
    }
    plan.cdef_items.swap(halves);
  }
  plan.edge_cap = cap;
  // meta layout: [frames][items...] uploaded, then [edges v][edges h][counts] device-only
  size_t off = 0;
  auto place = [&](size_t bytes) {
    off = align_up(off, 256);
    const size_t at = off;
    off += bytes;
    return at;
  };
  plan.off_frames = place(plan.frames.size() * sizeof(FrameDesc));
  plan.off_lf = place(plan.lf_items.size() * sizeof(Item));
  plan.off_lft = place(plan.lft_items.size() * sizeof(Item));
  plan.off_lff = place(plan.lff_items.size() * sizeof(Item));
  plan.off_cdef = place(plan.cdef_items.size() * sizeof(Item));
  plan.off_sr = place(plan.sr_items.size() * sizeof(Item));
  plan.off_lr = place(plan.lr_items.size() * sizeof(Item));
  plan.off_grain = place(plan.grain_items.size() * sizeof(Item));
  plan.off_out = place(plan.out_items.size() * sizeof(Item));
  plan.off_copy = place(plan.copy_items.size() * sizeof(Item));
  plan.upload_bytes = align_up(off, 256);
  plan.off_edges_v = place(size_t(cap) * 8);
  plan.off_edges_h = place(size_t(cap) * 8);
  plan.off_counts = place(16);
  plan.off_flags = place(plan.n_flags * 4);
  {
    plan.grain_meta.assign(plan.frames.size(), {SIZE_MAX, SIZE_MAX});
    size_t g = 0;
    for (size_t fi = 0; fi < plan.frames.size(); fi++) {
      const FrameDesc& d = plan.frames[fi];
      if (!d.grain_on) continue;
      plan.grain_meta[fi].first = g;
      g = align_up(g + sizeof(GrainScratch), 256);
      plan.grain_meta[fi].second = g;
      g = align_up(g + size_t(d.grain_ns) * size_t(d.grain_nb), 256);
    }
    plan.off_grain_meta = place(g);
  }
  plan.meta_bytes = align_up(off, 256);
  return AV1PF_OK;
}

void structure_key(const FrameJob* jobs, int n, std::vector<int64_t>& key) {
  key.clear();
  key.push_back(n);
  for (int fi = 0; fi < n; fi++) {
    const FrameJob& j = jobs[fi];
    const av1pf_frame_info* i = j.info;
    const av1pf_params* p = j.params;
    key.insert(key.end(), {i->bit_depth, i->sample_bytes, i->subsampling_x, i->subsampling_y, i->num_planes,
                           i->frame_width, i->frame_height, i->upscaled_width, i->mi_rows, i->mi_cols,
                           int64_t(j.stages), int64_t(j.in_place_lf), j.lf_mode, j.lr_cols,
                           int64_t(j.frame_out != nullptr), int64_t(j.maps != nullptr),
                           int64_t(p->loop_filter_level[0] != 0 || p->loop_filter_level[1] != 0),
                           int64_t(p->loop_filter_level[2] != 0), int64_t(p->loop_filter_level[3] != 0),
                           p->cdef_enabled, p->use_superres, p->uses_lr, p->film_grain.apply});
    for (int k = 0; k < 3; k++) {
      key.insert(key.end(), {p->frame_restoration_type[k], p->loop_restoration_size[k], p->lr_unit_rows[k],
                             p->lr_unit_cols[k]});
      if (k < i->num_planes && j.in) key.insert(key.end(), {j.in[k].width, j.in[k].height});
    }
  }
}

void pack_meta(const Plan& plan, uint8_t* host) {
  std::memset(host, 0, plan.upload_bytes);
  auto put = [&](size_t at, const void* src, size_t bytes) {
    if (bytes) std::memcpy(host + at, src, bytes);
  };
  put(plan.off_frames, plan.frames.data(), plan.frames.size() * sizeof(FrameDesc));
  put(plan.off_lf, plan.lf_items.data(), plan.lf_items.size() * sizeof(Item));
  put(plan.off_lft, plan.lft_items.data(), plan.lft_items.size() * sizeof(Item));
  put(plan.off_lff, plan.lff_items.data(), plan.lff_items.size() * sizeof(Item));
  put(plan.off_cdef, plan.cdef_items.data(), plan.cdef_items.size() * sizeof(Item));
  put(plan.off_sr, plan.sr_items.data(), plan.sr_items.size() * sizeof(Item));
  put(plan.off_lr, plan.lr_items.data(), plan.lr_items.size() * sizeof(Item));
  put(plan.off_grain, plan.grain_items.data(), plan.grain_items.size() * sizeof(Item));
  put(plan.off_out, plan.out_items.data(), plan.out_items.size() * sizeof(Item));
  put(plan.off_copy, plan.copy_items.data(), plan.copy_items.size() * sizeof(Item));
}

void launch_plan(const Plan& plan, uint8_t* meta, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                 cudaEvent_t join, const cudaEvent_t* stage_ev, bool counts_zeroed, bool flags,
                 bool grain_private) {
  uint32_t* sync = flags && plan.flag_sync ? reinterpret_cast<uint32_t*>(meta + plan.off_flags) : nullptr;
  auto mark = [&](int k) {
    if (stage_ev) cudaEventRecord(stage_ev[k], s);
  };
  const FrameDesc* frames = reinterpret_cast<const FrameDesc*>(meta + plan.off_frames);
  auto items = [&](size_t off) { return reinterpret_cast<const Item*>(meta + off); };
  uint64_t* ev = reinterpret_cast<uint64_t*>(meta + plan.off_edges_v);
  uint64_t* eh = reinterpret_cast<uint64_t*>(meta + plan.off_edges_h);
  uint32_t* counts = reinterpret_cast<uint32_t*>(meta + plan.off_counts);
  if (plan.any_grain) {
    // the grain templates depend only on the parameters: run them beside the
    // chain; into a scratch that the previous call's output kernel may still
    // read, only once `s` has got this far
    if (!grain_private) {
      cudaEventRecord(fork, s);
      cudaStreamWaitEvent(side, fork, 0);
    }
    launch_grain_prep(frames, items(plan.off_grain), int(plan.grain_items.size()), side);
    cudaEventRecord(join, side);
  }
  mark(0);
  if (!plan.copy_items.empty()) {
    if (!counts_zeroed) cudaMemsetAsync(counts, 0, 16, s);
    counts_zeroed = false;
    launch_lf_prep(frames, items(plan.off_copy), int(plan.copy_items.size()), ev, eh, counts, 0, s);
  }
  if (plan.any_lf && !plan.lf_items.empty()) {
    // in place: decisions into both edge lists, then one pass per direction
    if (!counts_zeroed) cudaMemsetAsync(counts, 0, 16, s);
    counts_zeroed = false;
    launch_lf_prep(frames, items(plan.off_lf), int(plan.lf_items.size()), ev, eh, counts, plan.edge_cap, s);
    launch_lf_edges(0, frames, ev, counts + 0, plan.edge_cap, s);
    launch_lf_edges(1, frames, eh, counts + 1, plan.edge_cap, s);
  }
  if (plan.any_lf && !plan.lft_items.empty()) {
    // copy + vertical edges per tile, then the horizontal edge list
    if (!counts_zeroed) cudaMemsetAsync(counts, 0, 16, s);
    counts_zeroed = false;
    launch_lf_tiles(frames, items(plan.off_lft), int(plan.lft_items.size()), eh, counts, plan.edge_cap, s);
    if (plan.any_hlist) launch_lf_edges(1, frames, eh, counts + 1, plan.edge_cap, s);
  }
  if (plan.any_lf && !plan.lff_items.empty())
    launch_lf_fused(frames, items(plan.off_lff), int(plan.lff_items.size()), sync, s);
  mark(1);
  if (plan.any_cdef)
    launch_cdef(frames, items(plan.off_cdef), int(plan.cdef_items.size()), plan.any_lfh, plan.cdef_half, sync, s);
  mark(2);
  if (plan.any_sr) launch_superres(frames, items(plan.off_sr), int(plan.sr_items.size()), plan.sr_row_max, s);
  mark(3);
  if (plan.any_lr) launch_lr(frames, items(plan.off_lr), int(plan.lr_items.size()), sync, s);
  mark(4);
  if (plan.any_out) {
    if (plan.any_grain) cudaStreamWaitEvent(s, join, 0);
    launch_output(frames, items(plan.off_out), int(plan.out_items.size()), s);
  }
  mark(5);
}

}  // namespace av1pf
