// batch.h — internal interface of the batched path, shared with the
// autotuner (tune.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "av1pf.h"
#include "ctx.h"
#include "plan.h"

namespace av1pf {

// Checks one av1pf_job (index i names it in the error text).
int validate_job(const av1pf_job& j, int i);

// The number of frame groups `flags` asks for (see AV1PF_BATCH_GROUPS_SHIFT).
int batch_groups_of(uint32_t flags, int n_jobs);

// Plans `fj` (variants already chosen) in the frame groups `flags` asks for,
// uploads the work lists and, unless AV1PF_BATCH_NO_GRAPH, captures the
// launches into a graph.
int create_batch(Ctx* ctx, const FrameJob* fj, int n_jobs, uint32_t flags, av1pf_batch** out);

// av1pf_autotune over `jobs` (validated by the caller); only_new skips the
// shapes the context has recorded.
int tune_shapes(Ctx* ctx, const av1pf_job* jobs, int n_jobs, int reps, bool only_new, int* n_shapes);

// Times every variant applied to the whole batch, and the per-shape choices,
// each with 1 to 3 frame groups, and returns the fastest set of frame jobs
// in `best` and its group count in `best_groups`.
int tune_batch(Ctx* ctx, const av1pf_job* jobs, int n_jobs, int reps, std::vector<FrameJob>& best,
               int* best_groups);

}  // namespace av1pf
