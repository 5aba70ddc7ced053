// tune.cpp — kernel-variant choices and the autotuner.
//
// Two knobs change how the chain's work is cut, never what it computes:
//   - lf_mode: the loop filter as a decision kernel plus one edge-list pass
//     per direction (0); vertical edges per 64x64 tile in shared memory plus
//     the horizontal edge list (1); as 1 with the horizontal edges inside
//     the CDEF kernel on the superblock window it stages anyway, 11 rows of
//     halo instead of 2 (2); or both directions per 64x64 tile in shared
//     memory, one kernel (3);
//   - lr_rect_cols: loop-restoration rectangles of 64 or 32 columns (more,
//     smaller CTAs balance better on small frames; wider ones re-read less
//     halo).
// The autotuner times each variant per frame shape as a one-frame batch
// replayed from a CUDA graph (device time only), keeps the fastest in the
// context, and the chain and serving paths read it from there. A batch
// created with AV1PF_BATCH_AUTOTUNE is tuned as a whole instead: each variant
// applied to every frame, and the per-shape choices, timed on the batch
// itself (a batch's throughput and a single frame's latency can favour
// different cuts).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "av1pf.h"
#include "batch.h"
#include "ctx.h"
#include "plan.h"

namespace av1pf {

ShapeKey shape_of(const av1pf_frame_info* i) {
  return ShapeKey{i->frame_width,   i->upscaled_width, i->frame_height, i->bit_depth,
                  i->subsampling_x, i->subsampling_y,  i->num_planes};
}

void Ctx::apply_tuning(FrameJob& j) const {
  std::lock_guard<std::mutex> lk(tune_mu);
  int mode = 3;  // unmeasured shapes: both loop-filter passes in one kernel
  int cols = 64;
  const auto it = tuned.find(shape_of(j.info));
  if (it != tuned.end()) {
    mode = it->second.lf_mode;
    cols = it->second.lr_cols;
  }
  if (tuning.lf_mode >= 0) mode = tuning.lf_mode;
  if (tuning.lr_rect_cols) cols = tuning.lr_rect_cols;
  j.lf_mode = mode;
  j.lr_cols = cols;
}

namespace {

// Median device time (ms) of `reps` replays of the batch of `fj` in
// `groups` frame groups.
int time_variant(Ctx* ctx, const FrameJob* fj, int n, int reps, float* ms, int groups = 1) {
  av1pf_batch* b = nullptr;
  int rc = create_batch(ctx, fj, n, uint32_t(groups) << AV1PF_BATCH_GROUPS_SHIFT, &b);
  if (rc != AV1PF_OK) return rc;
  cudaStream_t s = ctx->own;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  std::vector<float> t;
  for (int k = 0; k < 2 && e == cudaSuccess; k++) {  // warm-up
    rc = av1pf_batch_run(b, s);
    if (rc != AV1PF_OK) break;
  }
  for (int k = 0; k < reps && e == cudaSuccess && rc == AV1PF_OK; k++) {
    e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) rc = av1pf_batch_run(b, s);
    if (e == cudaSuccess && rc == AV1PF_OK) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess && rc == AV1PF_OK) e = cudaEventSynchronize(e1);
    float v = 0;
    if (e == cudaSuccess && rc == AV1PF_OK) e = cudaEventElapsedTime(&v, e0, e1);
    t.push_back(v);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  av1pf_batch_destroy(b);
  if (rc != AV1PF_OK) return rc;
  if (e != cudaSuccess) return cuda_status(e, "autotune timing");
  std::sort(t.begin(), t.end());
  *ms = t.empty() ? 0.f : t[t.size() / 2];
  return AV1PF_OK;
}

}  // namespace

int tune_shapes(Ctx* ctx, const av1pf_job* jobs, int n_jobs, int reps, bool only_new, int* n_shapes) {
  if (n_shapes) *n_shapes = 0;
  reps = std::max(1, std::min(reps, 1000));
  std::map<ShapeKey, int> first;  // shape -> first job of that shape
  for (int i = 0; i < n_jobs; i++) first.emplace(shape_of(jobs[i].info), i);
  for (const auto& kv : first) {
    if (only_new) {
      std::lock_guard<std::mutex> lk(ctx->tune_mu);
      if (ctx->tuned.count(kv.first)) continue;
    }
    const av1pf_job& j = jobs[kv.second];
    const av1pf_params* p = j.params;
    const bool lf_on = p->loop_filter_level[0] || p->loop_filter_level[1];
    // modes that differ for this frame: none without the loop filter, no
    // horizontal pass inside CDEF without CDEF
    std::vector<int> modes{0};
    if (lf_on) {
      modes.push_back(1);
      if (p->cdef_enabled) modes.push_back(2);
      modes.push_back(3);
    }
    const bool lr_on = p->uses_lr && (p->frame_restoration_type[0] || p->frame_restoration_type[1] ||
                                      p->frame_restoration_type[2]);
    ShapeChoice best{0, 64, 0.f};
    bool have = false;
    for (int mode : modes)
      for (int cols : {64, 32}) {
        if (cols == 32 && !lr_on) continue;
        FrameJob fj{j.info, j.params, j.maps, j.in, nullptr, j.ref_out, j.frame_out, ST_CHAIN, false};
        fj.lf_mode = mode;
        fj.lr_cols = cols;
        float ms = 0;
        const int rc = time_variant(ctx, &fj, 1, reps, &ms);
        if (rc != AV1PF_OK) return rc;
        if (!have || ms < best.ms) {
          best = ShapeChoice{mode, cols, ms};
          have = true;
        }
      }
    {
      std::lock_guard<std::mutex> lk(ctx->tune_mu);
      ctx->tuned[kv.first] = best;
    }
    if (n_shapes) ++*n_shapes;
  }
  return AV1PF_OK;
}

int tune_batch(Ctx* ctx, const av1pf_job* jobs, int n_jobs, int reps, std::vector<FrameJob>& best,
               int* best_groups) {
  reps = std::max(1, std::min(reps, 1000));
  auto base = [&](int i) {
    const av1pf_job& j = jobs[i];
    return FrameJob{j.info, j.params, j.maps, j.in, nullptr, j.ref_out, j.frame_out, ST_CHAIN, false};
  };
  bool any_cdef = false;
  for (int i = 0; i < n_jobs; i++) any_cdef = any_cdef || jobs[i].params->cdef_enabled;
  // candidates: each variant for every frame, and the per-shape record
  std::vector<std::vector<FrameJob>> cands;
  for (int mode : {0, 1, 2, 3})
    for (int cols : {64, 32}) {
      if (mode == 2 && !any_cdef) continue;
      std::vector<FrameJob> v;
      for (int i = 0; i < n_jobs; i++) {
        FrameJob fj = base(i);
        fj.lf_mode = mode;
        fj.lr_cols = cols;
        v.push_back(fj);
      }
      cands.push_back(std::move(v));
    }
  {
    std::vector<FrameJob> v;
    for (int i = 0; i < n_jobs; i++) {
      FrameJob fj = base(i);
      ctx->apply_tuning(fj);
      v.push_back(fj);
    }
    cands.push_back(std::move(v));
  }
  float best_ms = 0;
  bool have = false;
  *best_groups = 1;
  for (int groups = 1; groups <= std::min(3, n_jobs); groups++)
    for (auto& v : cands) {
      float ms = 0;
      const int rc = time_variant(ctx, v.data(), n_jobs, reps, &ms, groups);
      if (rc != AV1PF_OK) return rc;
      if (!have || ms < best_ms) {
        best_ms = ms;
        best = v;
        *best_groups = groups;
        have = true;
      }
    }
  return AV1PF_OK;
}

}  // namespace av1pf

using namespace av1pf;

extern "C" {

int av1pf_set_tuning(av1pf_ctx* ctx, const av1pf_tuning* t) {
  if (!ctx || !t) return AV1PF_ERR_INVALID_INPUT;
  if (t->lf_mode < -1 || t->lf_mode > 3 ||
      (t->lr_rect_cols != 0 && t->lr_rect_cols != 32 && t->lr_rect_cols != 64)) {
    set_error("av1pf_set_tuning: lf_mode must be -1, 0, 1, 2 or 3 and lr_rect_cols 0, 32 or 64");
    return AV1PF_ERR_INVALID_INPUT;
  }
  std::lock_guard<std::mutex> lk(ctx->tune_mu);
  ctx->tuning = *t;
  return AV1PF_OK;
}

int av1pf_get_tuning(av1pf_ctx* ctx, av1pf_tuning* t) {
  if (!ctx || !t) return AV1PF_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(ctx->tune_mu);
  *t = ctx->tuning;
  return AV1PF_OK;
}

int av1pf_autotune(av1pf_ctx* ctx, const av1pf_job* jobs, int n_jobs, int32_t reps, int32_t* n_shapes) {
  if (n_shapes) *n_shapes = 0;
  if (!ctx || !jobs || n_jobs <= 0) return AV1PF_ERR_INVALID_INPUT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  for (int i = 0; i < n_jobs; i++) {
    const int rc = validate_job(jobs[i], i);
    if (rc != AV1PF_OK) return rc;
  }
  int n = 0;
  const int rc = tune_shapes(ctx, jobs, n_jobs, reps, false, &n);
  if (n_shapes) *n_shapes = n;
  return rc;
}

int av1pf_tuned_choice(av1pf_ctx* ctx, const av1pf_frame_info* info, av1pf_tuning* choice, float* ms) {
  if (!ctx || !info) return AV1PF_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(ctx->tune_mu);
  const auto it = ctx->tuned.find(shape_of(info));
  if (it == ctx->tuned.end()) {
    set_error("shape not measured");
    return AV1PF_ERR_NOT_FOUND;
  }
  if (choice) {
    choice->lf_mode = it->second.lf_mode;
    choice->lr_rect_cols = it->second.lr_cols;
  }
  if (ms) *ms = it->second.ms;
  return AV1PF_OK;
}

}  // extern "C"
