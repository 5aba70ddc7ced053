/*
 * synth.h — seeded synthetic post-filter inputs (pre-filter planes, per-4x4
 * maps, filter parameters) for the measured configurations and the parity
 * tests. The reference's conformance streams need a full AV1 decoder to
 * produce pre-filter planes, so these generators stand in for decoded data:
 * every frame they make is conformant in the ways the filters rely on
 * (blocks tile 64x64 superblocks, transform blocks tile each block, chroma
 * block sizes are valid for the subsampling, chroma data sits on the block
 * that "has chroma", cdef_idx is -1 exactly where a 64x64 is all skip).
 *
 * Host memory only; the library owns the buffers until synth_destroy.
 */
#ifndef AV1PF_SYNTH_H
#define AV1PF_SYNTH_H

#include "av1pf.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SYNTH_CONTENT_FIELD = 0,   /* low-frequency field + steps on the tx grid + noise */
  SYNTH_CONTENT_MOVING = 1   /* gradient + 4 rectangles moving 2 px/frame + noise */
};

typedef struct synth_config {
  int32_t width;          /* output (upscaled) width */
  int32_t height;
  int32_t bit_depth;      /* 8, 10, 12 */
  int32_t sample_bytes;   /* 1 (8-bit only) or 2 */
  int32_t subsampling_x;
  int32_t subsampling_y;
  int32_t mono;
  int32_t superres_denom; /* 8 = off, 9..16 = coded width (w*8 + d/2)/d */
  int32_t content;        /* SYNTH_CONTENT_* */
  int32_t noise_sigma;    /* in 8-bit units scaled to the bit depth; <0 = default */
  int32_t frame_index;
  uint64_t seed;
  int32_t enable_lf;
  int32_t enable_cdef;
  int32_t enable_lr;
  int32_t enable_grain;
  int32_t lr_unit_shift;   /* luma unit = 64 << shift, 0..2 */
  int32_t lr_uv_shift;     /* 0/1 (only with 4:2:0) */
  int32_t segmentation;    /* random segment ids + LF segment features */
  int32_t delta_lf;        /* random per-block delta_lf (multi when 2) */
  int32_t min_block_log2;  /* smallest block side 2 (4x4) .. 6 (64x64) */
  int32_t skip_pct;        /* percent of blocks with skip set */
} synth_config;

typedef struct synth_frame {
  av1pf_frame_info info;
  av1pf_params params;
  av1pf_maps maps;                     /* host pointers */
  av1pf_plane planes[AV1PF_MAX_PLANES]; /* host pre-filter planes */
  /* element counts of each map array (for copies to the device) */
  int64_t mi_count;
  int64_t tx_count[AV1PF_MAX_PLANES];
  int64_t cdef_count;
  int64_t lr_count[AV1PF_MAX_PLANES];
  int64_t plane_bytes[AV1PF_MAX_PLANES];
} synth_frame;

/* Fills `cfg` with the defaults (everything on, 4:2:0, 10-bit 1920x1080). */
void synth_default_config(synth_config* cfg);
int synth_create(const synth_config* cfg, synth_frame** out);
void synth_destroy(synth_frame* f);

#ifdef __cplusplus
}
#endif
#endif
