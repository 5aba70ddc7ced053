// api.cpp — the C ABI (include/av1pf.h): context, per-stage and whole-chain
// entry points, the host-buffer chain, and the DSP entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "av1pf.h"
#include "ctx.h"
#include "kernels.h"
#include "plan.h"

namespace av1pf {

namespace {
std::atomic<uint64_t> g_launches{0};
thread_local std::string t_last_error;
std::mutex g_tables_mu;
bool g_tables_ready[64] = {};
}  // namespace

namespace {
// launches enqueued while capturing a graph are counted when it runs
thread_local int t_capturing = 0;
thread_local uint64_t t_captured = 0;
}  // namespace

void note_launch(uint64_t n) {
  if (t_capturing)
    t_captured += n;
  else
    g_launches.fetch_add(n, std::memory_order_relaxed);
}

CaptureScope::CaptureScope() : start(t_captured) { ++t_capturing; }
CaptureScope::~CaptureScope() { --t_capturing; }
uint64_t CaptureScope::launches() const { return t_captured - start; }

void set_error(const std::string& s) { t_last_error = s; }

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return AV1PF_OK;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? AV1PF_ERR_OOM : AV1PF_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Context resources
// ---------------------------------------------------------------------------
int Ctx::ensure(DevBuf& b, size_t bytes) {
  if (b.size >= bytes) return AV1PF_OK;
  if (b.ptr) {
    cudaFree(b.ptr);
    held -= b.size;
    b.ptr = nullptr;
    b.size = 0;
  }
  if (cap && held + bytes > cap) {
    set_error("allocation would exceed the context's HBM cap");
    return AV1PF_ERR_ADMISSION;
  }
  cudaError_t e = cudaMalloc(&b.ptr, bytes);
  if (e != cudaSuccess) {
    b.ptr = nullptr;
    return cuda_status(e, "cudaMalloc");
  }
  b.size = bytes;
  held += bytes;
  return AV1PF_OK;
}

int Ctx::ensure_host(HostBuf& b, size_t bytes) {
  if (b.size >= bytes) return AV1PF_OK;
  if (b.ptr) cudaFreeHost(b.ptr);
  b.ptr = nullptr;
  b.size = 0;
  cudaError_t e = cudaMallocHost(&b.ptr, bytes);
  if (e != cudaSuccess) return cuda_status(e, "cudaMallocHost");
  b.size = bytes;
  return AV1PF_OK;
}

cudaError_t Ctx::pipe_streams() {
  cudaError_t e = cudaSuccess;
  if (!pipe_up) e = cudaStreamCreateWithFlags(&pipe_up, cudaStreamNonBlocking);
  if (e == cudaSuccess && !pipe_down) e = cudaStreamCreateWithFlags(&pipe_down, cudaStreamNonBlocking);
  for (PipeSlot& ps : pipe) {
    for (cudaEvent_t* ev : {&ps.uploaded, &ps.computed, &ps.downloaded})
      if (e == cudaSuccess && !*ev) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  }
  return e;
}

void Ctx::release(DevBuf& b) {
  if (b.ptr) {
    cudaFree(b.ptr);
    held -= b.size;
  }
  b.ptr = nullptr;
  b.size = 0;
}

// Pipeline trace of av1pf_chain_host_many, in the tracing build only
// (AV1PF_TRACE; av1pf_trace_pipeline reads it): per frame of the last call,
// CUDA events at the start and end of its upload, chain, download and
// descriptor upload on their streams, and host timestamps of its enqueue
// steps. Elsewhere the calls are empty.
namespace pipe_trace {
#ifdef AV1PF_TRACE
constexpr int kCap = 256;
cudaEvent_t g_ev[kCap][8] = {};
double g_host[kCap][4] = {};
int g_n = 0, g_cur = -1;
std::chrono::steady_clock::time_point g_t0;
void begin(int frames) {
  if (!g_ev[0][0])
    for (auto& row : g_ev)
      for (cudaEvent_t& e : row) cudaEventCreate(&e);
  g_n = frames < kCap ? frames : kCap;
  g_t0 = std::chrono::steady_clock::now();
}
void frame(int k) { g_cur = k < kCap ? k : -1; }
void mark(int j, cudaStream_t s) {
  if (g_cur >= 0) cudaEventRecord(g_ev[g_cur][j], s);
}
void stamp(int j) {
  if (g_cur >= 0)
    g_host[g_cur][j] = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - g_t0).count();
}
void end() { g_cur = -1; }
#else
inline void begin(int) {}
inline void frame(int) {}
inline void mark(int, cudaStream_t) {}
inline void stamp(int) {}
inline void end() {}
#endif
}  // namespace pipe_trace

// Plans `jobs`, sizes scratch and a descriptor buffer, uploads and launches
// on `s`.
int Ctx::run(const FrameJob* jobs, int n, cudaStream_t s) {
  std::string why;
  int rc = AV1PF_OK;
  // Jobs with the structure of the previous call (a decoder filtering frame
  // after frame of one stream) get the same work lists: only the frame
  // descriptors are rebuilt, and uploaded where the buffer already holds
  // the lists. Anything else is planned in full.
  structure_key(jobs, n, key_scratch);
  if (host_ready && key_scratch == host_key) {
    rc = build_plan(jobs, n, static_cast<uint8_t*>(scratch.ptr), plan, &why, false);
    if (rc != AV1PF_OK) return set_error(why), rc;
  } else {
    host_ready = false;
    rc = build_plan(jobs, n, nullptr, plan, &why);
    if (rc != AV1PF_OK) return set_error(why), rc;
    if ((rc = ensure(scratch, plan.scratch_bytes + 256)) != AV1PF_OK) return rc;
    // the lists are built; with the scratch in place only the descriptors change
    rc = build_plan(jobs, n, static_cast<uint8_t*>(scratch.ptr), plan, &why, false);
    if (rc != AV1PF_OK) return set_error(why), rc;
    host_key = key_scratch;
    host_ready = true;
  }
  // Two descriptor buffers in turn: call k's upload runs on its own stream
  // while call k-1's kernels read the other buffer, and a buffer is
  // rewritten only after the launches that read it are done.
  cudaError_t e = cudaSuccess;
  if (!upload) {
    e = cudaStreamCreateWithFlags(&upload, cudaStreamNonBlocking);
    for (MetaSlot& q : metas)
      for (cudaEvent_t* ev : {&q.uploaded, &q.done})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_status(e, "descriptor stream");
  }
  MetaSlot& m = metas[meta_next];
  meta_next ^= 1;
  if (m.dev.size < plan.meta_bytes + 256) {
    if (m.used && (e = cudaEventSynchronize(m.done)) != cudaSuccess) return cuda_status(e, "descriptor wait");
    m.ready = false;
    if ((rc = ensure(m.dev, plan.meta_bytes + 256)) != AV1PF_OK) return rc;
  }
  // the pinned staging buffer: its last upload must be done before it is
  // overwritten
  if (m.used && (e = cudaEventSynchronize(m.uploaded)) != cudaSuccess) return cuda_status(e, "staging wait");
  if ((rc = ensure_host(m.host, plan.upload_bytes + 256)) != AV1PF_OK) return rc;
  cudaStream_t ups = upload_override ? upload_override : upload;
  if (m.used) cudaStreamWaitEvent(ups, m.done, 0);
  pipe_trace::mark(6, ups);
  uint8_t* dmeta = static_cast<uint8_t*>(m.dev.ptr);
  uint8_t* hmeta = static_cast<uint8_t*>(m.host.ptr);
  // film grain: this buffer's own scratch (the previous call's output kernel
  // reads the other buffer's), so the template kernel can start at once
  for (size_t fi = 0; fi < plan.frames.size() && fi < plan.grain_meta.size(); fi++) {
    if (plan.grain_meta[fi].first == SIZE_MAX) continue;
    plan.frames[fi].grain = reinterpret_cast<GrainScratch*>(dmeta + plan.off_grain_meta + plan.grain_meta[fi].first);
    plan.frames[fi].grain_off = dmeta + plan.off_grain_meta + plan.grain_meta[fi].second;
  }
  if (m.ready && m.key == key_scratch) {
    const size_t fbytes = plan.frames.size() * sizeof(FrameDesc);
    std::memcpy(hmeta + plan.off_frames, plan.frames.data(), fbytes);
    e = cudaMemcpyAsync(dmeta + plan.off_frames, hmeta + plan.off_frames, fbytes, cudaMemcpyHostToDevice, ups);
  } else {
    m.ready = false;
    pack_meta(plan, hmeta);
    e = cudaMemcpyAsync(dmeta, hmeta, plan.upload_bytes, cudaMemcpyHostToDevice, ups);
    if (e == cudaSuccess) {
      m.key = key_scratch;
      m.ready = true;
    }
  }
  // the loop filter's edge-list counters start at zero: cleared here, in the
  // upload's stream order, so the chain's stream holds kernels only
  if (e == cudaSuccess) e = cudaMemsetAsync(dmeta + plan.off_counts, 0, 16, ups);
  // and the stages' readiness flags start cleared
  if (e == cudaSuccess && plan.n_flags) e = cudaMemsetAsync(dmeta + plan.off_flags, 0, plan.n_flags * 4, ups);
  if (e == cudaSuccess) e = cudaEventRecord(m.uploaded, ups);
  pipe_trace::mark(7, ups);
  // The kernels read the upload: the host waits for it rather than the
  // chain's stream. It waited only for the chain that used this buffer two
  // calls ago, so it has usually landed already; and with nothing between
  // the previous call's last kernel and this call's first on the stream,
  // programmatic dependent launch chains them (a stream-side wait here made
  // every call boundary a full one: 9 us per 1080p frame).
  if (e == cudaSuccess) e = stream_upload_wait ? cudaStreamWaitEvent(s, m.uploaded, 0) : cudaEventSynchronize(m.uploaded);
  if (e != cudaSuccess) return cuda_status(e, "descriptor upload");
  m.used = true;
  rc = launch_on(dmeta, s);
  cudaEventRecord(m.done, s);
  return rc;
}

// Launches the planned stages reading descriptor buffer `dmeta` as stream
// launches with programmatic dependent launch, so consecutive calls' kernels
// chain without a gap at the call boundary (the first loop-filter kernel of
// a call starts its launch while the previous call's last kernel drains);
// profiled calls record stage events between the stages.
int Ctx::launch_on(uint8_t* dmeta, cudaStream_t s) {
  const cudaEvent_t* ev = nullptr;
  if (prof) {
    const int slot = prof_next;
    prof_next = (prof_next + 1) % kProfSlots;
    if (prof_used[slot]) prof_collect(slot);
    if (!prof_ev[slot][0])
      for (int k = 0; k < 6; k++) cudaEventCreate(&prof_ev[slot][k]);
    prof_used[slot] = true;
    ev = prof_ev[slot];
  }
  launch_plan(plan, dmeta, s, side, fork, join, ev, true, true, true);
  return cuda_status(cudaGetLastError(), "kernel launch");
}

void Ctx::prof_collect(int slot) {
  cudaEventSynchronize(prof_ev[slot][5]);
  for (int k = 0; k < 5; k++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, prof_ev[slot][k], prof_ev[slot][k + 1]) == cudaSuccess) prof_ms[k] += ms;
  }
  prof_calls++;
  prof_used[slot] = false;
}

}  // namespace av1pf

using namespace av1pf;

namespace {

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int check_ctx(av1pf_ctx* ctx) {
  if (!ctx) {
    set_error("null context");
    return AV1PF_ERR_INVALID_INPUT;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  return cuda_status(e, "cudaSetDevice");
}

int validate_all(const av1pf_frame_info* info, const av1pf_params* params, const av1pf_plane* planes) {
  std::string why;
  const int rc = validate_frame(info, params, planes, &why);
  if (rc != AV1PF_OK) set_error(why);
  return rc;
}

int validate_maps(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* m, bool need_lf,
                  bool need_cdef, bool need_lr) {
  if (!m) {
    set_error("null maps");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if ((need_lf || need_cdef) && (!m->mi || m->mi_stride < info->mi_cols)) {
    set_error("mi map missing or mi_stride < mi_cols");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if (need_lf)
    for (int k = 0; k < info->num_planes; k++)
      if (!m->lf_tx_size[k]) {
        set_error("lf_tx_size map missing");
        return AV1PF_ERR_INVALID_INPUT;
      }
  if (need_cdef && (!m->cdef_idx || m->cdef_stride < (info->mi_cols + 15) / 16)) {
    set_error("cdef_idx missing or cdef_stride too small");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if (need_lr && p->uses_lr)
    for (int k = 0; k < info->num_planes; k++)
      if (p->frame_restoration_type[k] && !m->lr_units[k]) {
        set_error("lr_units missing");
        return AV1PF_ERR_INVALID_INPUT;
      }
  return AV1PF_OK;
}

bool lf_active(const av1pf_params* p) { return p->loop_filter_level[0] || p->loop_filter_level[1]; }

}  // namespace

extern "C" {

int av1pf_ctx_create(int device, uint64_t hbm_cap_bytes, av1pf_ctx** out) {
  if (!out) return AV1PF_ERR_INVALID_INPUT;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) {
    set_error("no such CUDA device");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  {
    std::lock_guard<std::mutex> lk(g_tables_mu);
    if (device < 64 && !g_tables_ready[device]) {
      if ((e = upload_grain_tables()) != cudaSuccess) return cuda_status(e, "grain tables");
      if ((e = lr_init()) != cudaSuccess) return cuda_status(e, "loop restoration kernel attributes");
      if ((e = superres_init()) != cudaSuccess) return cuda_status(e, "superres kernel attributes");
      if ((e = cdef_init()) != cudaSuccess) return cuda_status(e, "CDEF kernel attributes");
      if ((e = output_init()) != cudaSuccess) return cuda_status(e, "output kernel attributes");
      g_tables_ready[device] = true;
    }
  }
  av1pf_ctx* c = new av1pf_ctx();
  c->device = device;
  c->cap = hbm_cap_bytes;
  if ((e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming)) != cudaSuccess) {
    delete c;
    return cuda_status(e, "stream/event create");
  }
  *out = c;
  return AV1PF_OK;
}

int av1pf_ctx_destroy(av1pf_ctx* ctx) {
  if (!ctx) return AV1PF_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  ctx->release(ctx->scratch);
  for (Ctx::MetaSlot& m : ctx->metas) {
    ctx->release(m.dev);
    if (m.host.ptr) cudaFreeHost(m.host.ptr);
    for (cudaEvent_t ev : {m.uploaded, m.done})
      if (ev) cudaEventDestroy(ev);
  }
  if (ctx->upload) cudaStreamDestroy(ctx->upload);
  for (auto* b : {&ctx->h_in, &ctx->h_ref, &ctx->h_maps, &ctx->h_frame, &ctx->search_dev, &ctx->search_planes})
    ctx->release(*b);
  if (ctx->search_host.ptr) cudaFreeHost(ctx->search_host.ptr);
  if (ctx->h_maps_stage.ptr) cudaFreeHost(ctx->h_maps_stage.ptr);
  for (Ctx::PipeSlot& ps : ctx->pipe) {
    for (auto* b : {&ps.in, &ps.ref, &ps.maps, &ps.frame}) ctx->release(*b);
    if (ps.maps_stage.ptr) cudaFreeHost(ps.maps_stage.ptr);
    for (cudaEvent_t ev : {ps.uploaded, ps.computed, ps.downloaded})
      if (ev) cudaEventDestroy(ev);
  }
  if (ctx->pipe_up) cudaStreamDestroy(ctx->pipe_up);
  if (ctx->pipe_down) cudaStreamDestroy(ctx->pipe_down);
  cudaStreamDestroy(ctx->side);
  cudaStreamDestroy(ctx->own);
  cudaEventDestroy(ctx->fork);
  cudaEventDestroy(ctx->join);
  for (auto& slot : ctx->prof_ev)
    for (auto& e : slot)
      if (e) cudaEventDestroy(e);
  delete ctx;
  return AV1PF_OK;
}

int av1pf_set_threads(av1pf_ctx* ctx, int n) {
  if (!ctx || n < 0) return AV1PF_ERR_INVALID_INPUT;
  ctx->threads = n == 0 ? 3 : std::min(n, Ctx::kPipeSlots);
  return AV1PF_OK;
}

int av1pf_ctx_memory(const av1pf_ctx* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return AV1PF_ERR_INVALID_INPUT;
  *bytes = ctx->held;
  return AV1PF_OK;
}

int av1pf_validate(const av1pf_frame_info* info, const av1pf_params* params, const av1pf_plane* planes) {
  return validate_all(info, params, planes);
}

size_t av1pf_frame_bytes(const av1pf_frame_info* info) { return info ? packed_frame_bytes(info) : 0; }

int av1pf_loop_filter(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                      const av1pf_maps* maps, av1pf_plane* planes, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, planes))) return rc;
  if (!lf_active(params)) return AV1PF_OK;
  if ((rc = validate_maps(info, params, maps, true, false, false))) return rc;
  FrameJob j{info, params, maps, planes, nullptr, planes, nullptr, ST_LF, true};
  return ctx->run(&j, 1, as_stream(stream));
}

int av1pf_cdef(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params, const av1pf_maps* maps,
               const av1pf_plane* cur, av1pf_plane* out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, cur)) || (rc = validate_all(info, params, out))) return rc;
  if ((rc = validate_maps(info, params, maps, false, params->cdef_enabled != 0, false))) return rc;
  FrameJob j{info, params, maps, cur, nullptr, out, nullptr, ST_CDEF, false};
  return ctx->run(&j, 1, as_stream(stream));
}

int av1pf_superres(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                   const av1pf_plane* in, av1pf_plane* out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, in))) return rc;
  if (!params->use_superres || !out) {
    set_error("superres is off for this frame");
    return AV1PF_ERR_INVALID_INPUT;
  }
  for (int k = 0; k < info->num_planes; k++) {
    if (!out[k].data || out[k].width < plane_w(info, k, info->upscaled_width) || out[k].height < plane_h(info, k)) {
      set_error("superres output plane too small");
      return AV1PF_ERR_INVALID_INPUT;
    }
  }
  FrameJob j{info, params, nullptr, in, nullptr, out, nullptr, ST_SR, false};
  return ctx->run(&j, 1, as_stream(stream));
}

int av1pf_loop_restoration(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                           const av1pf_maps* maps, const av1pf_plane* cur, const av1pf_plane* cdef,
                           av1pf_plane* out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, nullptr))) return rc;
  if (!cur || !cdef || !out) {
    set_error("null planes");
    return AV1PF_ERR_INVALID_INPUT;
  }
  for (int k = 0; k < info->num_planes; k++) {
    const int pw = plane_w(info, k, info->upscaled_width), ph = plane_h(info, k);
    if (!cur[k].data || !cdef[k].data || !out[k].data || cur[k].width < pw || cdef[k].width < pw ||
        out[k].width < pw || cur[k].height < ph || cdef[k].height < ph || out[k].height < ph) {
      set_error("loop restoration planes smaller than the visible area");
      return AV1PF_ERR_INVALID_INPUT;
    }
  }
  if ((rc = validate_maps(info, params, maps, false, false, true))) return rc;
  FrameJob j{info, params, maps, cdef, cur, out, nullptr, ST_LR, false};
  return ctx->run(&j, 1, as_stream(stream));
}

int av1pf_output(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params, const av1pf_plane* ref,
                 uint8_t* frame_out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, nullptr))) return rc;
  if (!ref || !frame_out) {
    set_error("null planes / output");
    return AV1PF_ERR_INVALID_INPUT;
  }
  FrameJob j{info, params, nullptr, ref, nullptr, nullptr, frame_out, ST_OUT, false};
  return ctx->run(&j, 1, as_stream(stream));
}

int av1pf_chain(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params, const av1pf_maps* maps,
                const av1pf_plane* in, av1pf_plane* ref_out, uint8_t* frame_out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, in))) return rc;
  if (!ref_out) {
    set_error("null ref_out");
    return AV1PF_ERR_INVALID_INPUT;
  }
  for (int k = 0; k < info->num_planes; k++) {
    if (!ref_out[k].data || ref_out[k].width < plane_w(info, k, info->upscaled_width) ||
        ref_out[k].height < plane_h(info, k)) {
      set_error("ref_out plane smaller than the visible area");
      return AV1PF_ERR_INVALID_INPUT;
    }
  }
  if ((rc = validate_maps(info, params, maps, lf_active(params), params->cdef_enabled != 0, true))) return rc;
  FrameJob j{info, params, maps, in, nullptr, ref_out, frame_out, ST_CHAIN, false};
  ctx->apply_tuning(j);
  return ctx->run(&j, 1, as_stream(stream));
}

namespace {

// Device layout of one host-buffer job: input planes with 64-sample-aligned
// strides, visible-size reference planes, the maps, the packed frame.
struct HostLayout {
  size_t in_off[3] = {0, 0, 0}, ref_off[3] = {0, 0, 0}, map_off[8] = {};
  size_t total_in = 0, total_ref = 0, total_maps = 0, fbytes = 0;
  size_t mi_n = 0, tx_rows[3] = {0, 0, 0}, cdef_n = 0, lr_n[3] = {0, 0, 0};
  av1pf_plane din[3] = {}, dref[3] = {};
};

void host_layout(const av1pf_frame_info* info, const av1pf_params* params, const av1pf_maps* maps,
                 const av1pf_plane* in, HostLayout& L) {
  const int np = info->num_planes, sb = info->sample_bytes;
  for (int k = 0; k < np; k++) {
    // host rows 16-byte aligned: the device plane keeps their stride and the
    // upload is one contiguous copy; else 64-sample rows and a 2D copy
    const bool flat = ((in[k].stride * sb) & 15) == 0 && in[k].stride >= in[k].width;
    const int64_t stride = flat ? in[k].stride : (int64_t(in[k].width) + 63) / 64 * 64;
    L.in_off[k] = L.total_in;
    L.total_in += (size_t(stride) * size_t(in[k].height) * size_t(sb) + 255) / 256 * 256;
    L.din[k] = av1pf_plane{nullptr, stride, in[k].width, in[k].height};
    const int pw = plane_w(info, k, info->upscaled_width), ph = plane_h(info, k);
    const int64_t rstride = (int64_t(pw) + 63) / 64 * 64;
    L.ref_off[k] = L.total_ref;
    L.total_ref += (size_t(rstride) * size_t(ph) * size_t(sb) + 255) / 256 * 256;
    L.dref[k] = av1pf_plane{nullptr, rstride, pw, ph};
  }
  const int sy_c = np > 1 ? info->subsampling_y : 0;
  L.mi_n = size_t(info->mi_rows) * size_t(maps->mi_stride);
  L.tx_rows[0] = size_t(info->mi_rows);
  L.tx_rows[1] = L.tx_rows[2] = size_t((info->mi_rows + (1 << sy_c) - 1) >> sy_c);
  L.cdef_n = size_t((info->mi_rows + 15) / 16) * size_t(maps->cdef_stride);
  for (int k = 0; k < np; k++)
    if (params->uses_lr && params->frame_restoration_type[k] && maps->lr_units[k])
      L.lr_n[k] = size_t(params->lr_unit_rows[k]) * size_t(params->lr_unit_cols[k]);
  auto put = [&](int slot, size_t bytes) {
    L.map_off[slot] = L.total_maps;
    L.total_maps += (bytes + 255) / 256 * 256;
  };
  put(0, L.mi_n * sizeof(av1pf_mi));
  for (int k = 0; k < 3; k++) put(1 + k, k < np ? L.tx_rows[k] * size_t(maps->mi_stride) : 0);
  put(4, L.cdef_n);
  for (int k = 0; k < 3; k++) put(5 + k, L.lr_n[k] * sizeof(av1pf_lr_unit));
  L.fbytes = packed_frame_bytes(info);
}

// Enqueues the uploads of a job's planes and maps into device buffers laid
// out by `L`; fills din / dref / dm with the device-side descriptions.
cudaError_t upload_job(const HostLayout& L, const av1pf_frame_info* info, const av1pf_maps* maps,
                       const av1pf_plane* in, uint8_t* bin, uint8_t* bref, uint8_t* bmap, av1pf_plane* din,
                       av1pf_plane* dref, av1pf_maps& dm, uint8_t* stage, cudaStream_t s) {
  const int np = info->num_planes, sb = info->sample_bytes;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < np && e == cudaSuccess; k++) {
    din[k] = L.din[k];
    dref[k] = L.dref[k];
    din[k].data = bin + L.in_off[k];
    dref[k].data = bref + L.ref_off[k];
    if (din[k].stride == in[k].stride) {
      const size_t bytes = (size_t(in[k].stride) * size_t(in[k].height - 1) + size_t(in[k].width)) * size_t(sb);
      e = cudaMemcpyAsync(din[k].data, in[k].data, bytes, cudaMemcpyHostToDevice, s);
    } else {
      e = cudaMemcpy2DAsync(din[k].data, size_t(din[k].stride) * sb, in[k].data, size_t(in[k].stride) * sb,
                            size_t(in[k].width) * sb, size_t(in[k].height), cudaMemcpyHostToDevice, s);
    }
  }
  dm = *maps;
  dm.mi = reinterpret_cast<const av1pf_mi*>(bmap + L.map_off[0]);
  if (e == cudaSuccess && L.mi_n && maps->mi)
    e = cudaMemcpyAsync(bmap + L.map_off[0], maps->mi, L.mi_n * sizeof(av1pf_mi), cudaMemcpyHostToDevice, s);
  // the maps after the mode info (transform sizes, CDEF indices, LR units):
  // with `stage`, packed on the host in their device layout and uploaded as
  // one copy (each copy costs the copy engine a few microseconds, and small
  // ones also slow the concurrent download), else one copy each
  const size_t s0 = L.map_off[1];
  auto put = [&](size_t off, const void* src, size_t bytes) {
    if (!bytes || e != cudaSuccess) return;
    if (stage) std::memcpy(stage + (off - s0), src, bytes);
    else e = cudaMemcpyAsync(bmap + off, src, bytes, cudaMemcpyHostToDevice, s);
  };
  for (int k = 0; k < 3; k++) {
    dm.lf_tx_size[k] = nullptr;
    if (k < np && maps->lf_tx_size[k]) {
      dm.lf_tx_size[k] = bmap + L.map_off[1 + k];
      put(L.map_off[1 + k], maps->lf_tx_size[k], L.tx_rows[k] * size_t(maps->mi_stride));
    }
  }
  dm.cdef_idx = nullptr;
  if (maps->cdef_idx) {
    dm.cdef_idx = reinterpret_cast<const int8_t*>(bmap + L.map_off[4]);
    put(L.map_off[4], maps->cdef_idx, L.cdef_n);
  }
  for (int k = 0; k < 3; k++) {
    dm.lr_units[k] = nullptr;
    if (L.lr_n[k]) {
      dm.lr_units[k] = reinterpret_cast<const av1pf_lr_unit*>(bmap + L.map_off[5 + k]);
      put(L.map_off[5 + k], maps->lr_units[k], L.lr_n[k] * sizeof(av1pf_lr_unit));
    }
  }
  if (stage && e == cudaSuccess && L.total_maps > s0)
    e = cudaMemcpyAsync(bmap + s0, stage, L.total_maps - s0, cudaMemcpyHostToDevice, s);
  return e;
}

// Enqueues the downloads of the reference planes (when ref_out is set) and
// the packed frame (when frame_out is set).
cudaError_t download_job(const HostLayout& L, const av1pf_frame_info* info, const av1pf_plane* dref,
                         av1pf_plane* ref_out, const uint8_t* dframe, uint8_t* frame_out, cudaStream_t s) {
  const int np = info->num_planes, sb = info->sample_bytes;
  cudaError_t e = cudaSuccess;
  for (int k = 0; ref_out && k < np && e == cudaSuccess; k++) {
    const int pw = plane_w(info, k, info->upscaled_width), ph = plane_h(info, k);
    e = cudaMemcpy2DAsync(ref_out[k].data, size_t(ref_out[k].stride) * sb, dref[k].data, size_t(dref[k].stride) * sb,
                          size_t(pw) * sb, size_t(ph), cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess && frame_out) e = cudaMemcpyAsync(frame_out, dframe, L.fbytes, cudaMemcpyDeviceToHost, s);
  return e;
}

// The host planes' own geometry (their size against the frame is checked
// on the device copies by av1pf_chain).
int check_host_planes(const av1pf_frame_info* info, const av1pf_plane* in) {
  for (int k = 0; k < info->num_planes; k++)
    if (!in[k].data || in[k].width <= 0 || in[k].height <= 0 || in[k].stride < in[k].width) {
      set_error("host plane: null data, empty, or stride < width");
      return AV1PF_ERR_INVALID_INPUT;
    }
  return AV1PF_OK;
}

// While alive, the context's descriptor uploads go on `up` (the stream that
// uploads the frames' planes, so each lands right after its frame's planes)
// and its chains wait for them on their own stream, not on the host.
struct UploadsAfterPlanes {
  Ctx* c;
  UploadsAfterPlanes(Ctx* c_, cudaStream_t up) : c(c_) {
    c->stream_upload_wait = true;
    c->upload_override = up;
  }
  ~UploadsAfterPlanes() {
    c->stream_upload_wait = false;
    c->upload_override = nullptr;
  }
};

int check_error_flags(cudaStream_t s) {
  uint32_t flags = 0;
  cudaError_t e = read_error_flags(&flags, s);
  if (e != cudaSuccess) return cuda_status(e, "error flags");
  if (flags & kErrfStall) {
    set_error("a kernel's bounded wait gave up; the output is not valid");
    return AV1PF_ERR_TIMEOUT;
  }
  if (flags) {
    set_error("the maps broke a conformance requirement (bad block / transform size or edge position)");
    return AV1PF_ERR_INVALID_INPUT;
  }
  return AV1PF_OK;
}

}  // namespace

int av1pf_chain_host(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                     const av1pf_maps* maps, const av1pf_plane* in, av1pf_plane* ref_out, uint8_t* frame_out) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = validate_all(info, params, nullptr))) return rc;
  if (!in || !maps) {
    set_error("null input");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if ((rc = check_host_planes(info, in))) return rc;
  cudaStream_t s = ctx->own;
  HostLayout L;
  host_layout(info, params, maps, in, L);
  if ((rc = ctx->ensure(ctx->h_in, L.total_in)) || (rc = ctx->ensure(ctx->h_ref, L.total_ref)) ||
      (rc = ctx->ensure(ctx->h_maps, L.total_maps)) || (rc = ctx->ensure(ctx->h_frame, L.fbytes + 16)) ||
      (rc = ctx->ensure_host(ctx->h_maps_stage, L.total_maps - L.map_off[1] + 16)))
    return rc;
  av1pf_plane din[3], dref[3];
  av1pf_maps dm;
  cudaError_t e = upload_job(L, info, maps, in, static_cast<uint8_t*>(ctx->h_in.ptr),
                             static_cast<uint8_t*>(ctx->h_ref.ptr), static_cast<uint8_t*>(ctx->h_maps.ptr), din, dref,
                             dm, static_cast<uint8_t*>(ctx->h_maps_stage.ptr), s);
  if (e != cudaSuccess) return cuda_status(e, "host-to-device copy");
  uint8_t* dframe = frame_out ? static_cast<uint8_t*>(ctx->h_frame.ptr) : nullptr;
  {
    // the descriptors follow the planes on `s`: the chain is queued at once
    UploadsAfterPlanes uploads_after_planes(ctx, s);
    rc = av1pf_chain(ctx, info, params, &dm, din, dref, dframe, s);
  }
  if (rc != AV1PF_OK) return rc;
  e = download_job(L, info, dref, ref_out, dframe, frame_out, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "chain_host");
  return check_error_flags(s);
}

int av1pf_chain_host_many(av1pf_ctx* ctx, int n, const av1pf_host_job* jobs) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (n < 0 || (n > 0 && !jobs)) {
    set_error("bad job list");
    return AV1PF_ERR_INVALID_INPUT;
  }
  if (n == 0) return AV1PF_OK;
  // every job is checked, and the slots sized for the largest, before
  // anything is queued
  std::vector<HostLayout> lay(static_cast<size_t>(n));
  size_t need_in = 0, need_ref = 0, need_maps = 0, need_frame = 0, need_stage = 0;
  for (int k = 0; k < n; k++) {
    const av1pf_host_job& j = jobs[k];
    if ((rc = validate_all(j.info, j.params, nullptr))) return rc;
    if (!j.in || !j.maps) {
      set_error("null input");
      return AV1PF_ERR_INVALID_INPUT;
    }
    if ((rc = check_host_planes(j.info, j.in))) return rc;
    host_layout(j.info, j.params, j.maps, j.in, lay[size_t(k)]);
    need_in = std::max(need_in, lay[size_t(k)].total_in);
    need_ref = std::max(need_ref, lay[size_t(k)].total_ref);
    need_maps = std::max(need_maps, lay[size_t(k)].total_maps);
    need_frame = std::max(need_frame, lay[size_t(k)].fbytes + 16);
    need_stage = std::max(need_stage, lay[size_t(k)].total_maps - lay[size_t(k)].map_off[1] + 16);
  }
  const int slots = std::min(n, ctx->threads);
  for (int q = 0; q < slots; q++) {
    Ctx::PipeSlot& ps = ctx->pipe[q];
    if ((rc = ctx->ensure(ps.in, need_in)) || (rc = ctx->ensure(ps.ref, need_ref)) ||
        (rc = ctx->ensure(ps.maps, need_maps)) || (rc = ctx->ensure(ps.frame, need_frame)))
      return rc;
    // (the staging is rewritten only after the upload that read it: at the
    // start of a call every earlier call's uploads are done)
    if ((rc = ctx->ensure_host(ps.maps_stage, need_stage))) return rc;
  }
  cudaError_t e = ctx->pipe_streams();
  if (e != cudaSuccess) return cuda_status(e, "pipeline streams");
  cudaStream_t up = ctx->pipe_up, comp = ctx->own, down = ctx->pipe_down;
  // each chain already waits for its planes on `comp`: its descriptor upload
  // goes on `up` right after them and is waited for on `comp` too, and the
  // host goes on queueing uploads
  UploadsAfterPlanes uploads_after_planes(ctx, up);
  pipe_trace::begin(n);
  // frame k uses slot k % slots: its upload waits for the chain that last
  // read the slot's inputs, its chain for its upload and for the download
  // that last read the slot's outputs
  for (int k = 0; k < n && e == cudaSuccess; k++) {
    const av1pf_host_job& j = jobs[k];
    Ctx::PipeSlot& ps = ctx->pipe[k % slots];
    const bool reused = k >= slots;
    pipe_trace::frame(k);
    pipe_trace::stamp(0);
    if (reused) e = cudaStreamWaitEvent(up, ps.computed, 0);
    // the slot's map staging is read by its previous upload
    if (e == cudaSuccess && reused) e = cudaEventSynchronize(ps.uploaded);
    av1pf_plane din[3], dref[3];
    av1pf_maps dm;
    pipe_trace::mark(0, up);
    if (e == cudaSuccess)
      e = upload_job(lay[size_t(k)], j.info, j.maps, j.in, static_cast<uint8_t*>(ps.in.ptr),
                     static_cast<uint8_t*>(ps.ref.ptr), static_cast<uint8_t*>(ps.maps.ptr), din, dref, dm,
                     static_cast<uint8_t*>(ps.maps_stage.ptr), up);
    pipe_trace::mark(1, up);
    pipe_trace::stamp(1);
    if (e == cudaSuccess) e = cudaEventRecord(ps.uploaded, up);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(comp, ps.uploaded, 0);
    if (e == cudaSuccess && reused) e = cudaStreamWaitEvent(comp, ps.downloaded, 0);
    if (e != cudaSuccess) break;
    uint8_t* dframe = j.frame_out ? static_cast<uint8_t*>(ps.frame.ptr) : nullptr;
    pipe_trace::mark(2, comp);
    rc = av1pf_chain(ctx, j.info, j.params, &dm, din, dref, dframe, comp);
    pipe_trace::mark(3, comp);
    pipe_trace::stamp(2);
    if (rc != AV1PF_OK) {
      pipe_trace::end();
      cudaStreamSynchronize(up);
      cudaStreamSynchronize(comp);
      cudaStreamSynchronize(down);
      return rc;
    }
    e = cudaEventRecord(ps.computed, comp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(down, ps.computed, 0);
    pipe_trace::mark(4, down);
    if (e == cudaSuccess) e = download_job(lay[size_t(k)], j.info, dref, j.ref_out, dframe, j.frame_out, down);
    pipe_trace::mark(5, down);
    pipe_trace::stamp(3);
    if (e == cudaSuccess) e = cudaEventRecord(ps.downloaded, down);
  }
  pipe_trace::end();
  // every download waits for its chain, which waits for its upload
  const cudaError_t e_up = cudaStreamSynchronize(up);
  const cudaError_t e_comp = cudaStreamSynchronize(comp);
  const cudaError_t e_down = cudaStreamSynchronize(down);
  if (e == cudaSuccess) e = e_up != cudaSuccess ? e_up : (e_comp != cudaSuccess ? e_comp : e_down);
  if (e != cudaSuccess) return cuda_status(e, "chain_host_many");
  return check_error_flags(comp);
}

int av1pf_dsp_lf_filter(av1pf_ctx* ctx, int32_t* edges, const av1pf_lf_edge_params* params, int n, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!edges || !params || n < 0) return AV1PF_ERR_INVALID_INPUT;
  launch_dsp_lf(edges, params, n, as_stream(stream));
  return cuda_status(cudaGetLastError(), "dsp_lf launch");
}

int av1pf_dsp_cdef_filter(av1pf_ctx* ctx, const int32_t* win, const av1pf_cdef_taps* taps, uint16_t* res, int n,
                          void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!win || !taps || !res || n < 0) return AV1PF_ERR_INVALID_INPUT;
  launch_dsp_cdef(win, taps, res, n, as_stream(stream));
  return cuda_status(cudaGetLastError(), "dsp_cdef launch");
}

int av1pf_set_profiling(av1pf_ctx* ctx, int on) {
  if (!ctx) return AV1PF_ERR_INVALID_INPUT;
  ctx->prof = on != 0;
  return AV1PF_OK;
}

int av1pf_stage_times(av1pf_ctx* ctx, float ms[5], uint32_t* calls) {
  if (!ctx || !ms) return AV1PF_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  for (int k = 0; k < Ctx::kProfSlots; k++)
    if (ctx->prof_used[k]) ctx->prof_collect(k);
  for (int k = 0; k < 5; k++) {
    ms[k] = float(ctx->prof_ms[k]);
    ctx->prof_ms[k] = 0;
  }
  if (calls) *calls = ctx->prof_calls;
  ctx->prof_calls = 0;
  return AV1PF_OK;
}

const char* av1pf_last_error(void) { return t_last_error.c_str(); }

uint64_t av1pf_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"

#ifdef AV1PF_TRACE
// The tracing build's read-out of the last av1pf_chain_host_many call: per
// frame (at most `max`), 8 device times in us from frame 0's upload start
// (upload start, end; chain start, end; download start, end; descriptor
// upload start, end; -1 where not recorded) and 4 host times in us from the
// call's start (frame begun, upload queued, chain queued, download queued).
// Returns the frame count.
extern "C" int av1pf_trace_pipeline(float* dev_us, double* host_us, int max) {
  using namespace av1pf::pipe_trace;
  const int n = g_n < max ? g_n : max;
  for (int k = 0; k < n; k++) {
    for (int j = 0; j < 8; j++) {
      float ms = -1.f;
      if (cudaEventElapsedTime(&ms, g_ev[0][0], g_ev[k][j]) != cudaSuccess) ms = -1e-3f;
      dev_us[k * 8 + j] = ms * 1e3f;
    }
    for (int j = 0; j < 4; j++) host_us[k * 4 + j] = g_host[k][j];
  }
  return n;
}
#endif
