// common.cuh — shared device definitions of the post-filter kernels:
// the per-frame descriptor the kernels read, the work-item format, the
// specification tables in constant memory, and integer helpers.
//
// Every stage kernel takes (frames[], items[], n_items) and loops over items
// with a grid stride, so one launch serves one frame or a whole batch of
// frames of different shape, bit depth and subsampling.
#pragma once

#include <cstdint>

#include "av1pf.h"
#include "av1_tables.h"

namespace av1pf {

// Sample planes on the device: `p` points at sample (0,0), rows `stride`
// samples apart; samples are u8 when the frame's sample_bytes is 1, else u16.
struct DPlane {
  uint8_t* p;
  int64_t stride;
  int32_t w, h;
};

// Film-grain scratch of one frame (filled by the template kernel).
struct GrainScratch {
  int16_t tmpl[3][73][82];  // luma, cb, cr grain templates (7.18.3.3)
  uint8_t lut[3][256];      // scaling lookup (7.18.3.4)
  uint8_t offsets[4096];    // per (stripe, 32-col block) random offsets
};

// Everything a stage kernel needs about one frame. Built on the host,
// copied to device memory once per call (or once per captured batch).
struct FrameDesc {
  // geometry (av1pf_frame_info)
  int32_t bd, sb, ssx, ssy, np;
  int32_t fw, fh, uw, mi_rows, mi_cols, mc;
  // stage buffers, per plane
  DPlane in[3];     // pre-filter planes (LF-V source)
  DPlane lfv[3];    // after the vertical-edge pass
  DPlane cur[3];    // after the loop filter (CDEF source, pre-CDEF rows for LR)
  DPlane cdef[3];   // after CDEF
  DPlane up[3];     // after superres (LR source)
  DPlane lines[3];  // upscaled pre-CDEF stripe-boundary rows (superres only)
  DPlane ref[3];    // LR output = reference frame
  uint8_t* frame_out;
  int64_t out_off[3];
  // maps (av1pf_maps)
  const av1pf_mi* mi;
  const uint8_t* tx[3];
  const int8_t* cdef_idx;
  const av1pf_lr_unit* lru[3];
  int32_t mi_stride, cdef_stride;
  // loop filter (7.14.4-5)
  int32_t lf_level[4];
  int32_t sharpness, delta_enabled, delta_lf_multi;
  int32_t ref_deltas[8], mode_deltas[2];
  int32_t seg_enabled;
  int32_t seg_lf_on[8][4];
  int32_t seg_lf_data[8][4];
  // CDEF
  int32_t cdef_damping;
  int32_t cdef_y_pri[8], cdef_y_sec[8], cdef_uv_pri[8], cdef_uv_sec[8];
  // superres
  int32_t sr_on;
  // LR
  int32_t lr_on;
  int32_t lr_type[3], lr_unit_size[3], lr_unit_rows[3], lr_unit_cols[3];
  int32_t stripes;
  // film grain
  int32_t grain_on;
  GrainScratch* grain;
  av1pf_film_grain g;
};

// One unit of work of a stage: a tile of one plane of one frame.
struct Item {
  uint16_t frame;
  uint8_t plane;
  uint8_t kind;
  uint16_t x0, y0;  // tile origin (plane samples, or stage-specific units)
  uint16_t x1, y1;  // tile end (exclusive)
  uint16_t a, b;    // stage-specific (LR: stripe, unit column)
};
static_assert(sizeof(Item) == 16, "Item is 16 bytes");

// ---------------------------------------------------------------------------
// Tables (av1_tables.h is extracted from the specification data of the
// reference's src/tables.rs).
// ---------------------------------------------------------------------------
extern __constant__ int8_t c_cdef_dirs[8][2][2];
extern __constant__ uint8_t c_cdef_uv_dir[2][2][8];
extern __constant__ int32_t c_div_table[9];
extern __constant__ uint8_t c_subsampled_size[23][2][2];
extern __constant__ uint8_t c_tx_w[19];
extern __constant__ uint8_t c_tx_h[19];
extern __constant__ uint8_t c_n4w[23];
extern __constant__ uint8_t c_n4h[23];
extern __constant__ int32_t c_sgr_params[16][4];
extern __device__ int16_t g_upscale_filter[64][8];
extern __device__ int16_t g_gaussian[2048];

// ---------------------------------------------------------------------------
// Integer helpers (consts.rs:328-368, bits.rs:112)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t round2(int32_t x, int n) {
  return n == 0 ? x : (x + (1 << (n - 1))) >> n;
}
__device__ __forceinline__ int64_t round2_64(int64_t x, int n) {
  return n == 0 ? x : (x + (int64_t(1) << (n - 1))) >> n;
}
__device__ __forceinline__ int32_t clip3(int32_t lo, int32_t hi, int32_t x) {
  return max(lo, min(hi, x));
}
__device__ __forceinline__ int32_t floor_log2(uint32_t x) { return 31 - __clz(x); }

// Sample access with the frame's storage width.
__device__ __forceinline__ int32_t ld_sample(const DPlane& p, int sb, int x, int y) {
  const uint8_t* row = p.p + (int64_t(y) * p.stride) * sb;
  return sb == 1 ? int32_t(row[x]) : int32_t(reinterpret_cast<const uint16_t*>(row)[x]);
}
__device__ __forceinline__ void st_sample(const DPlane& p, int sb, int x, int y, int32_t v) {
  uint8_t* row = p.p + (int64_t(y) * p.stride) * sb;
  if (sb == 1)
    row[x] = uint8_t(v);
  else
    reinterpret_cast<uint16_t*>(row)[x] = uint16_t(v);
}

// Plane dimensions helpers.
__device__ __forceinline__ int plane_ssx(const FrameDesc& f, int plane) { return plane ? f.ssx : 0; }
__device__ __forceinline__ int plane_ssy(const FrameDesc& f, int plane) { return plane ? f.ssy : 0; }

// Grid-stride loop over the items of a launch.
#define FOR_EACH_ITEM(it, n)                                   \
  for (int it = blockIdx.x; it < (n); it += gridDim.x)

}  // namespace av1pf
