// desc.h — the per-frame descriptor and work-item format shared by the host
// planner and the stage kernels (plain structs, host-safe).
#pragma once

#include <cstdint>

#include "av1pf.h"

namespace av1pf {

// Sample planes on the device: `p` points at sample (0,0), rows `stride`
// samples apart; samples are u8 when the frame's sample_bytes is 1, else u16.
struct DPlane {
  uint8_t* p;
  int64_t stride;
  int32_t w, h;
};

// Film-grain scratch of one frame (filled by the template kernel).
constexpr int kTmplStride = 5992;  // 73 * 82 = 5986 samples, padded
struct GrainScratch {
  // luma, cb, cr grain templates (7.18.3.3): 73 rows of 82, each plane
  // padded to a multiple of 16 bytes so that it moves as one bulk copy
  alignas(16) int16_t tmpl[3][kTmplStride];
  // the scaling function (7.18.3.4) at every sample value 0 .. 2^bitdepth - 1:
  // the 256-entry lookup, interpolated between entries above 8 bits
  alignas(16) uint8_t scale[3][4096];
};

// Everything a stage kernel needs about one frame. Built on the host,
// copied to device memory once per call (or once per captured batch).
struct FrameDesc {
  // geometry (av1pf_frame_info)
  int32_t bd, sb, ssx, ssy, np;
  int32_t fw, fh, uw, mi_rows, mi_cols, mc;
  // stage buffers, per plane
  DPlane in[3];     // pre-filter planes
  DPlane cur[3];    // loop-filtered in place (CDEF source, pre-CDEF rows for LR)
  DPlane cdef[3];   // after CDEF
  DPlane up[3];     // after superres (LR source)
  DPlane lines[3];  // upscaled pre-CDEF stripe-boundary rows (superres only)
  DPlane ref[3];    // LR output = reference frame
  // Post-loop-filter rows at the stripe boundaries (rows B-2 .. B+1 of each
  // boundary B, 4 rows per boundary, boundary b at rows (b-1)*4) for planes
  // whose horizontal loop-filter edges the CDEF kernel filters (lfh_mask);
  // loop restoration and superres read the pre-CDEF rows from here then.
  DPlane prelf[3];
  int32_t lfh_mask;
  uint8_t* frame_out;
  int64_t out_off[3];
  // Without film grain the packed frame holds the reference frame's samples
  // unchanged: the loop-restoration kernel then writes both and the frame
  // has no output items.
  int32_t lr_pack;
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
  // superres (7.16): per plane step, initial position, last source column
  int32_t sr_on;
  int32_t sr_step[3], sr_init[3], sr_maxx[3], sr_w[3];
  // LR
  int32_t lr_on;
  int32_t lr_type[3], lr_unit_size[3], lr_unit_rows[3], lr_unit_cols[3];
  int32_t stripes;
  // film grain
  int32_t grain_on;
  GrainScratch* grain;
  uint8_t* grain_off;      // [stripe][block] random offsets (7.18.3.5)
  int32_t grain_nb;        // blocks per stripe
  int32_t grain_ns;        // stripes
  av1pf_film_grain g;
  // Readiness flags between the stages, when a launch is given a flag array
  // (else each stage waits for the whole previous stage): the loop-filter
  // kernel sets one flag per 64x64 tile (plane p's tiles from
  // lf_flag_base[p], lf_tiles_x[p] a row; lf_tiles_x[p] = 0 where the plane
  // is not loop filtered), and the CDEF kernel one per half superblock (from
  // cdef_flag_base, cdef_sbc a row of halves, two rows per superblock row).
  // A CDEF CTA waits for the tiles under its window and a loop-restoration
  // CTA for the half superblocks under its rectangle, instead of for the
  // whole previous stage.
  int32_t lf_flag_base[3], lf_tiles_x[3];
  int32_t cdef_flag_base, cdef_sbc;
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

// The encoder's CDEF search (encoder/cdef.rs:52-251): candidate strength
// pairs and the per-block error table.
constexpr int kSearchMaxY = 48, kSearchMaxUV = 32;
struct CdefSearchDesc {
  DPlane src[3];           // source planes (frame area)
  int32_t ny, nuv;         // candidate pairs
  int32_t damping;         // cdef_damping (damping_minus_3 + 3)
  int32_t fb_rows, fb_cols;
  int8_t y_pri[kSearchMaxY], y_sec[kSearchMaxY];     // secondary decoded (coded 3 -> 4)
  int8_t uv_pri[kSearchMaxUV], uv_sec[kSearchMaxUV];
  uint64_t* sse;           // [ny + nuv][fb_rows * fb_cols], candidate-major
  uint64_t* best;          // [fb_rows * fb_cols]: the greedy's per-block minimum
  // one frame of a batched search: its descriptor, greedy state, candidate
  // totals, input table and outputs, and its first CTA in each grid
  const FrameDesc* frame;
  struct CdefGreedy* g;
  uint64_t* tot;           // [ny * nuv]
  const int8_t* cdef_idx;
  int32_t cdef_stride;
  int8_t* table;           // [fb_rows * cdef_stride]
  int32_t* res;            // [18]: nb, bits, the chosen pairs' indices
  double lambda;
  int32_t block0, table0;  // first CTA in the table kernel, first entry in the finish kernel
};

// The encoder's loop-restoration search (encoder/lr.rs:64-430): one job
// per restoration unit, its stripe rectangles, and the chosen filter.
struct LrSearchJob {
  int32_t frame, plane, x0, w;  // unit columns x0 .. x0 + w - 1
  int32_t r0, nr;               // rectangles r0 .. r0 + nr - 1 (one per stripe)
};
// One frame of a (batched) loop-restoration search.
struct LrSearchFrame {
  DPlane cur[3], cdef[3], src[3];  // deblocked frame, CDEF output, source
  int32_t bd, sb;
  int32_t pex[3], pey[3];  // last column / row of each plane
  double lambda;
};
struct LrSearchRect {
  int32_t ss, se;  // StripeStartY, StripeEndY
  int32_t y0, h;   // rows restored
};
// Per unit: the unfiltered error, the first Wiener pass's vertical
// solution, the quantised Wiener coefficients and their error.
struct LrJobState {
  uint64_t none, wiener;
  double vc[3];  // first-pass solution of a unit of several rectangles
  int32_t coef[2][3];
};
// Per (unit, self-guided set): the projection weights and their error.
struct LrSgrResult {
  int32_t xqd[2];
  uint64_t sse;
};
struct LrSearchDesc {
  const LrSearchFrame* frames;
  int32_t wmax, hmax;      // the widest unit and tallest rectangle
  int32_t step;            // fit on every step-th row and column
  int32_t band, cache_px;  // self-guided rows per band; filter outputs kept per unit
  int32_t both;            // 1: radius-2 and radius-1 box sums from one sweep (their buffers fit)
  int32_t multi_rect;      // 1: some job has several stripe rectangles (the first-pass kernel runs)
  int32_t nsets, sets[16];
  const LrSearchJob* jobs;
  const LrSearchRect* rects;
  LrJobState* state;   // one per job
  LrSgrResult* sgr;    // one per (job, set), set-minor
  av1pf_lr_unit* out;  // one per job
};

// State of the greedy choice of (luma, chroma) pairs (encoder/cdef.rs:195-240).
struct CdefGreedy {
  uint32_t arrived;        // CTAs of the current step done (the last one picks)
  int32_t n;               // pairs chosen so far
  int32_t set_y[8], set_uv[8];
  uint32_t nb;             // blocks that code an index
  int32_t best_bits;
  double best_cost;
};

}  // namespace av1pf
