// batch.cpp — the batched path: many frames of mixed shape, bit depth and
// subsampling through one launch per stage (the stage kernels stride over a
// work list spanning every frame), captured once into a CUDA graph and
// replayed by av1pf_batch_run.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "av1pf.h"
#include "batch.h"
#include "ctx.h"
#include "kernels.h"
#include "plan.h"

namespace av1pf {

struct Batch {
  Ctx* ctx = nullptr;
  Plan plan;
  DevBuf scratch, meta;
  cudaStream_t cap_stream = nullptr;
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

int create_batch(Ctx* ctx, const FrameJob* fj, int n_jobs, uint32_t flags, av1pf_batch** out) {
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  av1pf_batch* b = new av1pf_batch();
  b->ctx = ctx;
  std::string why;
  int rc = build_plan(fj, n_jobs, nullptr, b->plan, &why);
  if (rc == AV1PF_OK) rc = ctx->ensure(b->scratch, b->plan.scratch_bytes + 256);
  if (rc == AV1PF_OK) rc = build_plan(fj, n_jobs, static_cast<uint8_t*>(b->scratch.ptr), b->plan, &why);
  if (rc == AV1PF_OK) rc = ctx->ensure(b->meta, b->plan.meta_bytes + 256);
  if (rc != AV1PF_OK) {
    if (!why.empty()) set_error(why);
    ctx->release(b->scratch);
    ctx->release(b->meta);
    delete b;
    return rc;
  }
  // the work lists and descriptors are uploaded once
  std::vector<uint8_t> host(b->plan.upload_bytes);
  pack_meta(b->plan, host.data());
  e = cudaMemcpy(b->meta.ptr, host.data(), b->plan.upload_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && !(flags & AV1PF_BATCH_NO_GRAPH)) {
    CaptureScope cs;
    e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      launch_plan(b->plan, static_cast<uint8_t*>(b->meta.ptr), b->cap_stream, ctx->side, ctx->fork, ctx->join);
      e = cudaStreamEndCapture(b->cap_stream, &b->graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    b->kernels_per_run = cs.launches();
  }
  if (e != cudaSuccess) {
    rc = cuda_status(e, "batch create");
    av1pf_batch_destroy(b);
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
    int rc = tune_shapes(ctx, jobs, n_jobs, 10, true, nullptr);
    if (rc == AV1PF_OK) rc = tune_batch(ctx, jobs, n_jobs, 5, fj);
    if (rc != AV1PF_OK) return rc;
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
    launch_plan(b->plan, static_cast<uint8_t*>(b->meta.ptr), s, b->ctx->side, b->ctx->fork, b->ctx->join);
    e = cudaGetLastError();
  }
  return cuda_status(e, "batch run");
}

int av1pf_batch_destroy(av1pf_batch* b) {
  if (!b) return AV1PF_OK;
  cudaSetDevice(b->ctx->device);
  if (b->cap_stream) cudaStreamSynchronize(b->cap_stream);
  cudaDeviceSynchronize();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  b->ctx->release(b->scratch);
  b->ctx->release(b->meta);
  delete b;
  return AV1PF_OK;
}

}  // extern "C"
