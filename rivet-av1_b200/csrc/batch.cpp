// batch.cpp — the batched path: many frames of mixed shape, bit depth and
// subsampling through one launch per stage (the stage kernels stride over a
// work list spanning every frame), captured once into a CUDA graph and
// replayed by av1pf_batch_run.
//
// The frames may be split into groups, each a chain of stage launches of
// its own; the groups' chains are parallel branches of the graph, so the
// stages of different groups overlap on the device (a latency-bound stage of
// one group and an ALU-bound stage of another share the SMs).
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "av1pf.h"
#include "batch.h"
#include "ctx.h"
#include "kernels.h"
#include "plan.h"

namespace av1pf {

// One group of a batch: its plan, buffers, and the streams and events its
// chain runs on (group 0's main stream is the batch's own).
struct BatchGroup {
  Plan plan;
  DevBuf scratch, meta;
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, done = nullptr;
};

struct Batch {
  Ctx* ctx = nullptr;
  std::vector<BatchGroup> groups;
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t start = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels_per_run = 0;
};

}  // namespace av1pf

struct av1pf_batch : av1pf::Batch {};

namespace av1pf {

int validate_job(const av1pf_job& j, int i) {
  std::string why;
  int rc = validate_frame(j.info, j.params, j.in, &why);
  if (rc != AV1PF_OK) {
    set_error("job " + std::to_string(i) + ": " + why);
    return rc;
  }
  if (!j.maps || !j.ref_out) {
    set_error("job " + std::to_string(i) + ": null maps or ref_out");
    return AV1PF_ERR_INVALID_INPUT;
  }
  return AV1PF_OK;
}

namespace {

// Enqueues every group's chain on `s`: groups 1.. fork from `s` and join
// back, group 0 runs on `s` itself.
void launch_groups(Batch& b, cudaStream_t s) {
  const size_t n = b.groups.size();
  if (n > 1) cudaEventRecord(b.start, s);
  for (size_t g = 1; g < n; g++) cudaStreamWaitEvent(b.groups[g].stream, b.start, 0);
  for (size_t g = 0; g < n; g++) {
    BatchGroup& G = b.groups[g];
    uint8_t* meta = static_cast<uint8_t*>(G.meta.ptr);
    cudaStream_t gs = g ? G.stream : s;
    // the stages' readiness flags start cleared on every run
    if (G.plan.n_flags) cudaMemsetAsync(meta + G.plan.off_flags, 0, G.plan.n_flags * 4, gs);
    launch_plan(G.plan, meta, gs, G.side, G.fork, G.join, nullptr, false, true);
  }
  for (size_t g = 1; g < n; g++) {
    cudaEventRecord(b.groups[g].done, b.groups[g].stream);
    cudaStreamWaitEvent(s, b.groups[g].done, 0);
  }
}

// Splits frames into `n` groups of about equal samples (largest first, each
// to the lightest group), keeping each group's frames in submission order.
std::vector<std::vector<int>> split_groups(const FrameJob* fj, int n_jobs, int n) {
  std::vector<int> order(static_cast<size_t>(n_jobs));
  std::iota(order.begin(), order.end(), 0);
  auto samples = [&](int i) {
    const av1pf_frame_info* f = fj[i].info;
    const int64_t luma = int64_t(f->upscaled_width) * f->frame_height;
    const int64_t chroma = f->num_planes > 1 ? 2 * (luma >> (f->subsampling_x + f->subsampling_y)) : 0;
    return luma + chroma;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return samples(a) > samples(c); });
  std::vector<std::vector<int>> out(static_cast<size_t>(n));
  std::vector<int64_t> load(static_cast<size_t>(n), 0);
  for (int i : order) {
    const size_t g = size_t(std::min_element(load.begin(), load.end()) - load.begin());
    out[g].push_back(i);
    load[g] += samples(i);
  }
  for (auto& v : out) std::sort(v.begin(), v.end());
  out.erase(std::remove_if(out.begin(), out.end(), [](const std::vector<int>& v) { return v.empty(); }), out.end());
  return out;
}

void free_batch(Batch* b) {
  cudaSetDevice(b->ctx->device);
  cudaDeviceSynchronize();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (BatchGroup& G : b->groups) {
    if (G.stream) cudaStreamDestroy(G.stream);
    if (G.side) cudaStreamDestroy(G.side);
    if (G.fork) cudaEventDestroy(G.fork);
    if (G.join) cudaEventDestroy(G.join);
    if (G.done) cudaEventDestroy(G.done);
    b->ctx->release(G.scratch);
    b->ctx->release(G.meta);
  }
  if (b->start) cudaEventDestroy(b->start);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
}

}  // namespace

int batch_groups_of(uint32_t flags, int n_jobs) {
  const int g = int((flags >> AV1PF_BATCH_GROUPS_SHIFT) & 15u);
  if (g) return std::max(1, std::min(g, n_jobs));
  return n_jobs >= 8 ? 2 : 1;
}

int create_batch(Ctx* ctx, const FrameJob* fj, int n_jobs, uint32_t flags, av1pf_batch** out) {
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  av1pf_batch* b = new av1pf_batch();
  b->ctx = ctx;
  const auto parts = split_groups(fj, n_jobs, batch_groups_of(flags, n_jobs));
  b->groups.resize(parts.size());
  int rc = AV1PF_OK;
  std::string why;
  for (size_t g = 0; g < parts.size() && rc == AV1PF_OK; g++) {
    BatchGroup& G = b->groups[g];
    std::vector<FrameJob> jobs;
    for (int i : parts[g]) jobs.push_back(fj[i]);
    const int n = int(jobs.size());
    rc = build_plan(jobs.data(), n, nullptr, G.plan, &why);
    if (rc == AV1PF_OK) rc = ctx->ensure(G.scratch, G.plan.scratch_bytes + 256);
    if (rc == AV1PF_OK) rc = build_plan(jobs.data(), n, static_cast<uint8_t*>(G.scratch.ptr), G.plan, &why, false);
    if (rc == AV1PF_OK) rc = ctx->ensure(G.meta, G.plan.meta_bytes + 256);
    if (rc == AV1PF_OK) {
      // the work lists and descriptors are uploaded once
      std::vector<uint8_t> host(G.plan.upload_bytes);
      pack_meta(G.plan, host.data());
      e = cudaMemcpy(G.meta.ptr, host.data(), G.plan.upload_bytes, cudaMemcpyHostToDevice);
      if (e == cudaSuccess && g > 0) e = cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&G.side, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&G.fork, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&G.join, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming);
      if (e != cudaSuccess) rc = cuda_status(e, "batch create");
    }
  }
  if (rc == AV1PF_OK) {
    e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming);
    if (e == cudaSuccess && !(flags & AV1PF_BATCH_NO_GRAPH)) {
      CaptureScope cs;
      e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        launch_groups(*b, b->cap_stream);
        e = cudaStreamEndCapture(b->cap_stream, &b->graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      b->kernels_per_run = cs.launches();
    }
    if (e != cudaSuccess) rc = cuda_status(e, "batch create");
  }
  if (rc != AV1PF_OK) {
    if (!why.empty()) set_error(why);
    free_batch(b);
    return rc;
  }
  *out = b;
  return AV1PF_OK;
}

}  // namespace av1pf

using namespace av1pf;

extern "C" {

int av1pf_batch_create(av1pf_ctx* ctx, const av1pf_job* jobs, int n_jobs, uint32_t flags, av1pf_batch** out) {
  if (!ctx || !jobs || n_jobs <= 0 || !out) return AV1PF_ERR_INVALID_INPUT;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  for (int i = 0; i < n_jobs; i++) {
    const int rc = validate_job(jobs[i], i);
    if (rc != AV1PF_OK) return rc;
  }
  std::vector<FrameJob> fj(static_cast<size_t>(n_jobs));
  if (flags & AV1PF_BATCH_AUTOTUNE) {
    int groups = 1;
    int rc = tune_shapes(ctx, jobs, n_jobs, 10, true, nullptr);
    if (rc == AV1PF_OK) rc = tune_batch(ctx, jobs, n_jobs, 5, fj, &groups);
    if (rc != AV1PF_OK) return rc;
    flags = (flags & ~(15u << AV1PF_BATCH_GROUPS_SHIFT)) | (uint32_t(groups) << AV1PF_BATCH_GROUPS_SHIFT);
  } else {
    for (int i = 0; i < n_jobs; i++) {
      const av1pf_job& j = jobs[i];
      fj[size_t(i)] = FrameJob{j.info, j.params, j.maps, j.in, nullptr, j.ref_out, j.frame_out, ST_CHAIN, false};
      ctx->apply_tuning(fj[size_t(i)]);
    }
  }
  return create_batch(ctx, fj.data(), n_jobs, flags, out);
}

int av1pf_batch_run(av1pf_batch* b, void* stream) {
  if (!b) return AV1PF_ERR_INVALID_INPUT;
  cudaError_t e = cudaSetDevice(b->ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (b->exec) {
    e = cudaGraphLaunch(b->exec, s);
    note_launch(b->kernels_per_run);
  } else {
    launch_groups(*b, s);
    e = cudaGetLastError();
  }
  return cuda_status(e, "batch run");
}

int av1pf_batch_destroy(av1pf_batch* b) {
  if (!b) return AV1PF_OK;
  free_batch(b);
  return AV1PF_OK;
}

}  // extern "C"
