// ctx.h — the context behind av1pf_ctx: device, streams, grow-only device
// buffers and the pinned staging buffer of the per-frame path.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

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

// The frame shape the autotuner keys its choices by.
struct ShapeKey {
  int32_t fw, uw, fh, bd, ssx, ssy, np;
  bool operator<(const ShapeKey& o) const {
    return std::tie(fw, uw, fh, bd, ssx, ssy, np) < std::tie(o.fw, o.uw, o.fh, o.bd, o.ssx, o.ssy, o.np);
  }
};
ShapeKey shape_of(const av1pf_frame_info* info);

struct ShapeChoice {
  int lf_mode;
  int lr_cols;
  float ms;  // measured device time per frame
};

// While alive, kernel launches on this thread are not counted (they are
// being captured into a graph, and count when the graph runs).
struct CaptureScope {
  CaptureScope();
  ~CaptureScope();
  uint64_t launches() const;  // launches enqueued in this scope so far
  uint64_t start;
};

struct Ctx {
  int device = 0;
  uint64_t cap = 0;   // 0 = no cap
  uint64_t held = 0;  // device bytes held by this context
  int threads = 3;  // av1pf_set_threads: device frame slots of av1pf_chain_host_many
  cudaStream_t side = nullptr;  // grain templates beside the chain
  cudaStream_t own = nullptr;   // the host-buffer entry points
  cudaEvent_t fork = nullptr, join = nullptr;
  DevBuf scratch;
  DevBuf h_in, h_ref, h_maps, h_frame;  // av1pf_chain_host
  HostBuf h_maps_stage;                  // its small maps, packed for one upload
  // encoder searches: descriptors, error tables and greedy state; the
  // loop-filter search's filtered copies; pinned staging of both
  DevBuf search_dev, search_planes;
  HostBuf search_host;
  // av1pf_chain_host_many: device frame slots used in turn (`threads` of
  // them), with the events that order a slot's upload (pipe_up), chain
  // (own) and download (pipe_down) against its next use
  static constexpr int kPipeSlots = 8;
  struct PipeSlot {
    DevBuf in, ref, maps, frame;
    HostBuf maps_stage;  // the frame's small maps, packed for one upload
    cudaEvent_t uploaded = nullptr, computed = nullptr, downloaded = nullptr;
  };
  PipeSlot pipe[kPipeSlots];
  cudaStream_t pipe_up = nullptr, pipe_down = nullptr;
  cudaError_t pipe_streams();  // creates the streams and events on first use
  Plan plan;
  // the structure `plan`'s work lists were built for (structure_key)
  std::vector<int64_t> host_key, key_scratch;
  bool host_ready = false;
  // descriptor buffers used in turn: device copy, pinned staging, the
  // upload's and the reading launches' events, and the structure whose work
  // lists the device copy holds
  struct MetaSlot {
    DevBuf dev;
    HostBuf host;
    cudaEvent_t uploaded = nullptr, done = nullptr;
    bool used = false, ready = false;
    std::vector<int64_t> key;
  };
  MetaSlot metas[2];
  int meta_next = 0;
  cudaStream_t upload = nullptr;  // descriptor uploads
  // the chain's stream, not the host, waits for the descriptor upload: set
  // by callers whose chains begin with a stream wait anyway (the host-buffer
  // pipeline waits for each frame's planes), so that the host keeps queueing
  // uploads instead of waiting behind them
  bool stream_upload_wait = false;
  // the stream the descriptor uploads go on instead of `upload` (null: that
  // one): the host-buffer pipeline puts each frame's descriptors right after
  // its planes, in the same stream, since a small copy on a stream of its own
  // was measured landing 0.5 ms late behind the frames' large copies
  cudaStream_t upload_override = nullptr;
  // profiling: a ring of event sets, one per profiled call
  static constexpr int kProfSlots = 64;
  bool prof = false;
  cudaEvent_t prof_ev[kProfSlots][6] = {};
  bool prof_used[kProfSlots] = {};
  int prof_next = 0;
  double prof_ms[5] = {0, 0, 0, 0, 0};
  uint32_t prof_calls = 0;
  void prof_collect(int slot);

  // kernel variants (av1pf_tuning) and the autotuner's record per shape
  av1pf_tuning tuning{-1, 0};
  std::map<ShapeKey, ShapeChoice> tuned;
  mutable std::mutex tune_mu;
  // Sets j.lf_mode and j.lr_cols from the tuning and the record.
  void apply_tuning(FrameJob& j) const;

  int ensure(DevBuf& b, size_t bytes);
  int ensure_host(HostBuf& b, size_t bytes);
  void release(DevBuf& b);
  int run(const FrameJob* jobs, int n, cudaStream_t s);
  int launch_on(uint8_t* dmeta, cudaStream_t s);
};

void set_error(const std::string& s);
int cuda_status(cudaError_t e, const char* what);

}  // namespace av1pf

struct av1pf_ctx : av1pf::Ctx {};
