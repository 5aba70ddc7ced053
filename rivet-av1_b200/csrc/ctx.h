// ctx.h — the context behind av1pf_ctx: device, streams, grow-only device
// buffers and the pinned staging buffer of the per-frame path.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "av1pf.h"
#include "plan.h"

namespace av1pf {

struct DevBuf {
  void* ptr = nullptr;
  size_t size = 0;
};
struct HostBuf {
  void* ptr = nullptr;
  size_t size = 0;
};

struct Ctx {
  int device = 0;
  uint64_t cap = 0;   // 0 = no cap
  uint64_t held = 0;  // device bytes held by this context
  int threads = 2;
  cudaStream_t side = nullptr;  // grain templates beside the chain
  cudaStream_t own = nullptr;   // the host-buffer entry points
  cudaEvent_t fork = nullptr, join = nullptr, staged = nullptr;
  bool staged_once = false;
  DevBuf scratch, meta;
  DevBuf h_in, h_ref, h_maps, h_frame;  // av1pf_chain_host
  HostBuf meta_host;
  Plan plan;
  // profiling: a ring of event sets, one per profiled call
  static constexpr int kProfSlots = 64;
  bool prof = false;
  cudaEvent_t prof_ev[kProfSlots][6] = {};
  bool prof_used[kProfSlots] = {};
  int prof_next = 0;
  double prof_ms[5] = {0, 0, 0, 0, 0};
  uint32_t prof_calls = 0;
  void prof_collect(int slot);

  int ensure(DevBuf& b, size_t bytes);
  int ensure_host(HostBuf& b, size_t bytes);
  void release(DevBuf& b);
  int run(const FrameJob* jobs, int n, cudaStream_t s);
};

void set_error(const std::string& s);
int cuda_status(cudaError_t e, const char* what);

}  // namespace av1pf

struct av1pf_ctx : av1pf::Ctx {};
