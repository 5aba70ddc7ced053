// plan.h — host-side planning of the post-filter chain: validation, the
// per-frame scratch layout, the device descriptors and the per-stage work
// lists. Shared by the per-frame entry points, the batched path and the
// serving loop.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "av1pf.h"
#include "desc.h"

namespace av1pf {

// Which stages a plan runs and where their buffers come from.
enum StageMask : uint32_t {
  ST_LF = 1u,
  ST_CDEF = 2u,
  ST_SR = 4u,
  ST_LR = 8u,
  ST_OUT = 16u,
  ST_CHAIN = ST_LF | ST_CDEF | ST_SR | ST_LR | ST_OUT,
};

// One frame to plan. Planes are device pointers.
struct FrameJob {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_maps* maps;   // device
  const av1pf_plane* in;    // chain input / per-stage input
  const av1pf_plane* cur;   // per-stage: LR's pre-CDEF source (may be null)
  av1pf_plane* out;         // chain: reference frame; per-stage: the stage's output
  uint8_t* frame_out;       // packed output or null
  uint32_t stages;          // StageMask
  bool in_place_lf;         // av1pf_loop_filter: filter `in` in place
  // chain only (av1pf_tuning.lf_mode): 0 decisions + edge lists, 1 vertical
  // edges per tile, 2 as 1 with the horizontal edges inside the CDEF kernel,
  // 3 both directions per tile in one kernel
  int lf_mode = 0;
  int lr_cols = 64;  // loop-restoration rectangle width (<= 64)
};

// Work lists of every stage for a set of frames.
struct Plan {
  std::vector<FrameDesc> frames;
  std::vector<Item> lf_items, lft_items, lff_items, cdef_items, sr_items, lr_items, grain_items, out_items,
      copy_items;
  uint32_t edge_cap = 0;
  size_t scratch_bytes = 0;   // bytes of per-frame scratch (planes, grain)
  bool any_hlist = false;  // some plane's horizontal loop-filter edges run as their own pass
  bool any_lfh = false;    // some frame's horizontal loop-filter edges run inside the CDEF kernel
  bool cdef_half = false;  // CDEF items are half superblocks (Item::a: 0 top, 1 bottom)
  // the stages can wait on readiness flags (FrameDesc::lf_flag_base ...)
  // instead of on the whole previous stage: every frame runs the fused loop filter,
  // CDEF and loop restoration, without superres or the horizontal
  // loop-filter pass inside CDEF; n_flags flags at off_flags in the meta
  // buffer, cleared before every call
  bool flag_sync = false;
  size_t n_flags = 0, off_flags = 0;
  // A call's own film-grain scratch (templates, scaling tables, block
  // offsets) in the descriptor buffer, one per frame with grain:
  // grain_meta[frame] = {scratch offset, block-offsets offset} from
  // off_grain_meta (SIZE_MAX: no grain). Single calls point their
  // descriptors here, so a call's template kernel never writes what the
  // previous call's output kernel reads.
  size_t off_grain_meta = 0;
  std::vector<std::pair<size_t, size_t>> grain_meta;
  int sr_row_max = 0;      // superres: the most source samples in a row (sr_maxx + 1)
  bool any_lf = false, any_cdef = false, any_sr = false, any_lr = false, any_grain = false, any_out = false;
  // byte offsets of each list in the device meta buffer
  size_t off_frames = 0, off_lf = 0, off_lft = 0, off_lff = 0, off_cdef = 0, off_sr = 0, off_lr = 0, off_grain = 0, off_out = 0,
         off_copy = 0, off_edges_v = 0, off_edges_h = 0, off_counts = 0, meta_bytes = 0, upload_bytes = 0;
};

// Validation shared by av1pf_validate and every entry point.
int validate_frame(const av1pf_frame_info* info, const av1pf_params* params, const av1pf_plane* planes,
                   std::string* why);
int validate_params(const av1pf_frame_info* info, const av1pf_params* p, std::string* why);

// Builds the plan of `jobs`. Scratch pointers are laid out from
// `scratch_base` (pass nullptr first to learn plan.scratch_bytes, then again
// with the allocation). With items == false only the descriptors are built:
// the work lists, flags and layout stay those of the previous call, for jobs
// with the same structure (structure_key). Returns AV1PF_OK or an error code.
int build_plan(const FrameJob* jobs, int n, uint8_t* scratch_base, Plan& plan, std::string* why, bool items = true);

// Everything build_plan's work lists, flags, layout and scratch layout
// depend on: jobs with equal keys get equal lists (their descriptors differ).
void structure_key(const FrameJob* jobs, int n, std::vector<int64_t>& key);

// Serialises the plan's descriptors and items into `host` (plan.upload_bytes
// long) in the layout of the device meta buffer.
void pack_meta(const Plan& plan, uint8_t* host);

// Enqueues the plan's kernels on `s`; `meta` is the device meta buffer.
// `side`/`fork`/`join` run the grain templates concurrently when present.
// `stage_ev`, when not null, holds 6 events recorded before the loop
// filter and after each of the 5 stages (for av1pf_stage_times).
// `counts_zeroed`: the edge-list counters in `meta` are already zero (the
// caller cleared them in stream order), so the first loop-filter pass needs
// no memset on `s`. `flags`: the stages wait on the readiness flags at
// plan.off_flags in `meta` (plan.flag_sync; the caller cleared them in
// stream order) instead of on the whole previous stage. `grain_private`:
// the frames' film-grain scratch is this call's own (plan.grain_meta, no
// earlier kernel still reads it), so the template kernel starts on the side
// stream without waiting for `s`.
void launch_plan(const Plan& plan, uint8_t* meta, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                 cudaEvent_t join, const cudaEvent_t* stage_ev = nullptr, bool counts_zeroed = false,
                 bool flags = false, bool grain_private = false);

// Plane helpers.
inline int plane_w(const av1pf_frame_info* i, int p, int width) {
  const int sx = p ? i->subsampling_x : 0;
  return (width + sx) >> sx;
}
inline int plane_h(const av1pf_frame_info* i, int p) {
  const int sy = p ? i->subsampling_y : 0;
  return (i->frame_height + sy) >> sy;
}
size_t packed_frame_bytes(const av1pf_frame_info* info);

}  // namespace av1pf
