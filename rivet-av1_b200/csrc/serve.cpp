// serve.cpp — the serving loop: continuous batching of post-filter jobs from
// many concurrent streams (no reference counterpart; north_star's serving
// mode).
//
// A stream registers its frame geometry once; the server then keeps, per
// stream, a few device-resident frame slots (input planes, maps, reference
// frame, packed output) and a pool of pinned host buffers. Admission is by
// device memory: a stream is refused if its slots would push the server past
// its HBM cap. Submissions never block on the GPU: a host request is packed
// straight into a pinned buffer of its stream's pool (the only host copy of
// its input) and queued; a device request (planes and maps a GPU decoder
// already wrote to device memory) is queued as pointers. A worker thread runs ticks: it retires batches whose
// completion callback fired (recording submit -> completion latency), then,
// while a batch stream is free, admits queued requests into free slots of
// their streams (FIFO, up to max_batch_frames), uploads each with one copy,
// plans the whole admitted set as one batch (one launch per stage over every
// frame), launches it and queues the output copies. Several batches are in
// flight at once on separate streams, so requests that arrive while others
// run are admitted as slots free up and overlap with them on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "av1pf.h"
#include "ctx.h"
#include "kernels.h"
#include "plan.h"

namespace av1pf {

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Device layout of one frame of a stream (offsets into one blob).
struct Layout {
  int64_t stride[3] = {0, 0, 0};
  int32_t pw[3] = {0, 0, 0}, ph[3] = {0, 0, 0};
  size_t plane_off[3] = {0, 0, 0};
  int32_t mi_stride = 0, cdef_stride = 0;
  size_t mi_rows = 0, tx_rows[3] = {0, 0, 0}, cdef_rows = 0, lr_cap[3] = {0, 0, 0};
  size_t mi_off = 0, tx_off[3] = {0, 0, 0}, cdef_off = 0, lr_off[3] = {0, 0, 0};
  size_t bytes = 0;
  // visible reference planes and packed output
  int64_t rstride[3] = {0, 0, 0};
  size_t ref_off[3] = {0, 0, 0}, ref_bytes = 0, frame_bytes = 0;

  void build(const av1pf_frame_info& i) {
    const int np = i.num_planes, sb = i.sample_bytes;
    const int aw = (i.mi_cols * 4 + 127) & ~127, ah = (i.mi_rows * 4 + 127) & ~127;
    size_t off = 0;
    for (int p = 0; p < np; p++) {
      const int sx = p ? i.subsampling_x : 0, sy = p ? i.subsampling_y : 0;
      pw[p] = (aw >> sx) + 32;  // the reference's allocation (decoder/mod.rs:562-567)
      ph[p] = (ah >> sy) + 32;
      stride[p] = (pw[p] + 63) / 64 * 64;
      plane_off[p] = off;
      off += align256(size_t(stride[p]) * size_t(ph[p]) * size_t(sb));
    }
    mi_stride = i.mi_cols;
    mi_rows = size_t(i.mi_rows);
    mi_off = off;
    off += align256(mi_rows * size_t(mi_stride) * sizeof(av1pf_mi));
    for (int p = 0; p < np; p++) {
      const int sy = p ? i.subsampling_y : 0;
      tx_rows[p] = size_t((i.mi_rows + (1 << sy) - 1) >> sy);
      tx_off[p] = off;
      off += align256(tx_rows[p] * size_t(mi_stride));
    }
    cdef_stride = (i.mi_cols + 15) / 16;
    cdef_rows = size_t((i.mi_rows + 15) / 16);
    cdef_off = off;
    off += align256(cdef_rows * size_t(cdef_stride));
    for (int p = 0; p < np; p++) {
      const int sx = p ? i.subsampling_x : 0, sy = p ? i.subsampling_y : 0;
      // room for the smallest unit size (32): count_units_in_frame <= size / 32 + 1
      const size_t uw = size_t(((i.upscaled_width + sx) >> sx) / 32 + 1);
      const size_t uh = size_t(((i.frame_height + sy) >> sy) / 32 + 1);
      lr_cap[p] = uw * uh;
      lr_off[p] = off;
      off += align256(lr_cap[p] * sizeof(av1pf_lr_unit));
    }
    bytes = off;
    size_t roff = 0;
    for (int p = 0; p < np; p++) {
      const int w = plane_w(&i, p, i.upscaled_width), h = plane_h(&i, p);
      rstride[p] = (w + 63) / 64 * 64;
      ref_off[p] = roff;
      roff += align256(size_t(rstride[p]) * size_t(h) * size_t(sb));
    }
    ref_bytes = roff;
    frame_bytes = packed_frame_bytes(&i);
  }
};

struct Stream;

struct Slot {
  void* dblob = nullptr;   // input planes + maps (host requests)
  void* dref = nullptr;    // reference frame
  void* dframe = nullptr;  // packed output
  bool busy = false;
};

struct Request {
  uint64_t ticket = 0;
  int32_t stream = 0;
  Stream* st = nullptr;               // its stream (kept until the request retires)
  bool device = false;                // planes and maps are device pointers
  av1pf_params params{};
  av1pf_maps dmaps{};                 // device maps (given, or in the slot once admitted)
  av1pf_plane din[3]{}, dref[3]{};
  uint8_t* dframe_out = nullptr;      // device packed output (device requests)
  void* hin = nullptr;                // pinned: packed input (host requests)
  void* hres = nullptr;               // pinned: packed output (host requests)
  double t_submit = 0, t_done = 0;
  int state = 0;                      // 0 queued, 1 running, 2 done, 3 failed
  int status = AV1PF_OK;
  int slot = -1;
};

struct Stream {
  int32_t id = 0;
  av1pf_frame_info info{};
  Layout lay;
  std::vector<Slot> slots;
  std::vector<void*> pool_in, pool_out;  // free pinned buffers
  std::vector<void*> all_pinned;         // every pinned buffer (freed at close)
  int running = 0;
  int copying = 0;  // polls copying a result out of this stream's pinned buffers
  bool closing = false;
};

struct InFlight {
  std::condition_variable* wake = nullptr;  // the worker's condition variable
  cudaStream_t s = nullptr;
  void* scratch = nullptr;
  size_t scratch_size = 0;
  void* meta = nullptr;
  size_t meta_size = 0;
  void* meta_host = nullptr;
  size_t meta_host_size = 0;
  std::vector<Request*> reqs;
  std::atomic<bool> done{false};
  std::atomic<double> t_done{0};
  bool active = false;
  Plan plan;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaStream_t side = nullptr;
};

}  // namespace

struct Server {
  Ctx* ctx = nullptr;
  av1pf_serve_config cfg{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::deque<Request*> queue;
  std::map<uint64_t, Request*> tickets;
  std::map<int32_t, Stream*> streams;
  std::vector<InFlight*> inflight;
  bool stop = false;
  uint64_t next_ticket = 1;
  int32_t next_stream = 1;
  std::atomic<uint64_t> held{0};  // device bytes held by streams and batches
  // stats
  uint64_t submitted = 0, completed = 0, refused = 0, batches = 0, batch_frames = 0;
  std::vector<double> latencies;

  int dev_alloc(void** p, size_t bytes) {
    if (cfg.hbm_cap_bytes && held + bytes > cfg.hbm_cap_bytes) {
      set_error("serving: the HBM cap would be exceeded");
      return AV1PF_ERR_ADMISSION;
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_status(e, "serving: cudaMalloc");
    held += bytes;
    return AV1PF_OK;
  }
  void dev_free(void* p, size_t bytes) {
    if (p) {
      cudaFree(p);
      held -= bytes;
    }
  }

  // A pinned buffer of `bytes` from `pool` (the lock must be held; a new
  // one is allocated while the pool is empty).
  void* take_pinned(Stream* st, std::vector<void*>& pool, size_t bytes) {
    if (!pool.empty()) {
      void* p = pool.back();
      pool.pop_back();
      return p;
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    st->all_pinned.push_back(p);
    return p;
  }

  void run();
  int start_batch(InFlight& b, std::vector<Request*>& reqs);
};

namespace {

// Runs on a CUDA callback thread when a batch's stream reaches its end:
// records the completion time and wakes the worker (no CUDA calls here).
void CUDART_CB batch_done(void* arg) {
  InFlight* b = static_cast<InFlight*>(arg);
  b->t_done.store(now_ms());
  b->done.store(true);
  b->wake->notify_one();
}

int ensure_dev(Server& sv, void** p, size_t* size, size_t bytes) {
  if (*size >= bytes) return AV1PF_OK;
  sv.dev_free(*p, *size);
  *p = nullptr;
  *size = 0;
  const int rc = sv.dev_alloc(p, bytes);
  if (rc == AV1PF_OK) *size = bytes;
  return rc;
}

}  // namespace

int Server::start_batch(InFlight& b, std::vector<Request*>& reqs) {
  // host requests: one copy of the pinned input into the slot's device blob
  std::vector<FrameJob> jobs;
  jobs.reserve(reqs.size());
  for (Request* r : reqs) {
    Stream* st = r->st;
    Slot& sl = st->slots[size_t(r->slot)];
    const Layout& L = st->lay;
    uint8_t* rbase = static_cast<uint8_t*>(sl.dref);
    if (!r->device) {
      cudaMemcpyAsync(sl.dblob, r->hin, L.bytes, cudaMemcpyHostToDevice, b.s);
      uint8_t* base = static_cast<uint8_t*>(sl.dblob);
      for (int p = 0; p < st->info.num_planes; p++)
        r->din[p] = av1pf_plane{base + L.plane_off[p], L.stride[p], L.pw[p], L.ph[p]};
      av1pf_maps& m = r->dmaps;
      m.mi = reinterpret_cast<const av1pf_mi*>(base + L.mi_off);
      m.mi_stride = L.mi_stride;
      m.cdef_stride = L.cdef_stride;
      m.cdef_idx = reinterpret_cast<const int8_t*>(base + L.cdef_off);
      for (int p = 0; p < 3; p++) {
        m.lf_tx_size[p] = p < st->info.num_planes ? base + L.tx_off[p] : nullptr;
        m.lr_units[p] = p < st->info.num_planes ? reinterpret_cast<const av1pf_lr_unit*>(base + L.lr_off[p]) : nullptr;
      }
      r->dframe_out = static_cast<uint8_t*>(sl.dframe);
    }
    if (!r->dref[0].data)
      for (int p = 0; p < st->info.num_planes; p++)
        r->dref[p] = av1pf_plane{rbase + L.ref_off[p], L.rstride[p], plane_w(&st->info, p, st->info.upscaled_width),
                                 plane_h(&st->info, p)};
    jobs.push_back(FrameJob{&st->info, &r->params, &r->dmaps, r->din, nullptr, r->dref, r->dframe_out, ST_CHAIN,
                            false});
    ctx->apply_tuning(jobs.back());
  }
  std::string why;
  int rc = build_plan(jobs.data(), int(jobs.size()), nullptr, b.plan, &why);
  if (rc == AV1PF_OK) rc = ensure_dev(*this, &b.scratch, &b.scratch_size, b.plan.scratch_bytes + 256);
  if (rc == AV1PF_OK)
    // the lists are built; with the scratch in place only the descriptors change
    rc = build_plan(jobs.data(), int(jobs.size()), static_cast<uint8_t*>(b.scratch), b.plan, &why, false);
  if (rc == AV1PF_OK) rc = ensure_dev(*this, &b.meta, &b.meta_size, b.plan.meta_bytes + 256);
  if (rc != AV1PF_OK) return rc;
  if (b.meta_host_size < b.plan.upload_bytes) {
    if (b.meta_host) cudaFreeHost(b.meta_host);
    b.meta_host = nullptr;
    b.meta_host_size = 0;
    if (cudaMallocHost(&b.meta_host, b.plan.upload_bytes) != cudaSuccess) return AV1PF_ERR_OOM;
    b.meta_host_size = b.plan.upload_bytes;
  }
  pack_meta(b.plan, static_cast<uint8_t*>(b.meta_host));
  cudaMemcpyAsync(b.meta, b.meta_host, b.plan.upload_bytes, cudaMemcpyHostToDevice, b.s);
  // the stages' readiness flags start cleared
  if (b.plan.n_flags)
    cudaMemsetAsync(static_cast<uint8_t*>(b.meta) + b.plan.off_flags, 0, b.plan.n_flags * 4, b.s);
  launch_plan(b.plan, static_cast<uint8_t*>(b.meta), b.s, b.side, b.fork, b.join, nullptr, false, true);
  for (Request* r : reqs)
    if (!r->device)
      cudaMemcpyAsync(r->hres, r->dframe_out, r->st->lay.frame_bytes, cudaMemcpyDeviceToHost, b.s);
  b.done.store(false);
  cudaError_t e = cudaLaunchHostFunc(b.s, batch_done, &b);
  if (e == cudaSuccess) e = cudaGetLastError();
  return cuda_status(e, "serving: batch launch");
}

void Server::run() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    bool progressed = false;
    // 1. retire finished batches
    for (InFlight* b : inflight) {
      if (!b->active || !b->done.load()) continue;
      const double t = b->t_done.load();
      for (Request* r : b->reqs) {
        Stream* st = r->st;
        st->slots[size_t(r->slot)].busy = false;
        if (r->hin) {
          st->pool_in.push_back(r->hin);
          r->hin = nullptr;
        }
        st->running--;
        r->t_done = t;
        r->state = 2;
        latencies.push_back(t - r->t_submit);
        completed++;
      }
      b->reqs.clear();
      b->active = false;
      progressed = true;
    }
    if (progressed) cv_done.notify_all();
    // 2. admit queued requests into a free batch stream
    InFlight* free_b = nullptr;
    for (InFlight* b : inflight)
      if (!b->active) {
        free_b = b;
        break;
      }
    if (free_b && !queue.empty()) {
      std::vector<Request*> take;
      const int maxn = cfg.max_batch_frames > 0 ? cfg.max_batch_frames : 64;
      for (auto it = queue.begin(); it != queue.end() && int(take.size()) < maxn;) {
        Request* r = *it;
        Stream* st = r->st;
        int slot = -1;
        for (size_t k = 0; k < st->slots.size(); k++)
          if (!st->slots[k].busy) {
            slot = int(k);
            break;
          }
        if (slot < 0) {
          ++it;
          continue;
        }
        if (!r->device && !r->hres) {
          r->hres = take_pinned(st, st->pool_out, st->lay.frame_bytes);
          if (!r->hres) {
            ++it;
            continue;
          }
        }
        st->slots[size_t(slot)].busy = true;
        st->running++;
        r->slot = slot;
        r->state = 1;
        take.push_back(r);
        it = queue.erase(it);
      }
      if (!take.empty()) {
        free_b->active = true;
        free_b->reqs = take;
        // plan and launch without the lock, so submissions are not held up
        lk.unlock();
        const int rc = start_batch(*free_b, free_b->reqs);
        lk.lock();
        if (rc != AV1PF_OK) {
          // the batch could not be planned: fail its requests and free the slots
          for (Request* r : free_b->reqs) {
            Stream* st = r->st;
            st->slots[size_t(r->slot)].busy = false;
            st->running--;
            if (r->hin) st->pool_in.push_back(r->hin);
            if (r->hres) st->pool_out.push_back(r->hres);
            r->hin = r->hres = nullptr;
            r->state = 3;
            r->status = rc;
          }
          free_b->reqs.clear();
          free_b->active = false;
          cv_done.notify_all();
        } else {
          batches++;
          batch_frames += take.size();
        }
        continue;
      }
    }
    cv.wait_for(lk, std::chrono::microseconds(cfg.tick_us > 0 ? cfg.tick_us : 100));
  }
}

}  // namespace av1pf

struct av1pf_server : av1pf::Server {};

using namespace av1pf;

namespace {

bool same_geometry(const av1pf_frame_info& a, const av1pf_frame_info& b) {
  return a.bit_depth == b.bit_depth && a.sample_bytes == b.sample_bytes && a.subsampling_x == b.subsampling_x &&
         a.subsampling_y == b.subsampling_y && a.num_planes == b.num_planes && a.frame_width == b.frame_width &&
         a.frame_height == b.frame_height && a.upscaled_width == b.upscaled_width && a.mi_rows == b.mi_rows &&
         a.mi_cols == b.mi_cols;
}

}  // namespace

namespace {

// Checks one request and, for a host request, packs its input into a pinned
// buffer of its stream's pool; the request is not queued yet.
int prepare_request(av1pf_server* s, int32_t stream_id, const av1pf_request* req, Request** out) {
  *out = nullptr;
  if (!s || !req || !req->info || !req->params || !req->maps || !req->in) return AV1PF_ERR_INVALID_INPUT;
  Stream* st = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end() || it->second->closing) return AV1PF_ERR_NOT_FOUND;
    st = it->second;
  }
  const av1pf_frame_info& i = st->info;
  if (!same_geometry(i, *req->info)) {
    set_error("serving: the frame's geometry differs from its stream's");
    return AV1PF_ERR_INVALID_INPUT;
  }
  std::string why;
  int rc = validate_frame(req->info, req->params, req->in, &why);
  if (rc != AV1PF_OK) {
    set_error(why);
    return rc;
  }
  const av1pf_maps& m = *req->maps;
  if (!m.mi || m.mi_stride < i.mi_cols || !m.cdef_idx || m.cdef_stride < (i.mi_cols + 15) / 16) {
    set_error("serving: maps missing or too narrow");
    return AV1PF_ERR_INVALID_INPUT;
  }
  const Layout& L = st->lay;
  Request* r = new Request();
  r->stream = stream_id;
  r->st = st;
  r->params = *req->params;
  r->device = req->device != 0;
  if (r->device) {
    // planes and maps already on the device: queued as pointers
    for (int p = 0; p < i.num_planes; p++) r->din[p] = req->in[p];
    r->dmaps = m;
    if (req->ref_out)
      for (int p = 0; p < i.num_planes; p++) r->dref[p] = req->ref_out[p];
    r->dframe_out = req->frame_out;
  } else {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->hin = s->take_pinned(st, st->pool_in, L.bytes);
    }
    if (!r->hin) {
      delete r;
      set_error("serving: pinned staging allocation failed");
      return AV1PF_ERR_OOM;
    }
    uint8_t* b = static_cast<uint8_t*>(r->hin);
    const int sb = i.sample_bytes;
    for (int p = 0; p < i.num_planes; p++) {
      const av1pf_plane& pl = req->in[p];
      const int rows = std::min(pl.height, L.ph[p]);
      const size_t cols = size_t(std::min(pl.width, L.pw[p])) * size_t(sb);
      for (int y = 0; y < rows; y++)
        std::memcpy(b + L.plane_off[p] + size_t(y) * size_t(L.stride[p]) * sb,
                    static_cast<const uint8_t*>(pl.data) + int64_t(y) * pl.stride * sb, cols);
    }
    for (size_t y = 0; y < L.mi_rows; y++)
      std::memcpy(b + L.mi_off + y * size_t(L.mi_stride) * sizeof(av1pf_mi), m.mi + int64_t(y) * m.mi_stride,
                  size_t(L.mi_stride) * sizeof(av1pf_mi));
    for (int p = 0; p < i.num_planes; p++) {
      if (!m.lf_tx_size[p]) continue;
      for (size_t y = 0; y < L.tx_rows[p]; y++)
        std::memcpy(b + L.tx_off[p] + y * size_t(L.mi_stride), m.lf_tx_size[p] + int64_t(y) * m.mi_stride,
                    size_t(L.mi_stride));
    }
    for (size_t y = 0; y < L.cdef_rows; y++)
      std::memcpy(b + L.cdef_off + y * size_t(L.cdef_stride), m.cdef_idx + int64_t(y) * m.cdef_stride,
                  size_t(L.cdef_stride));
    for (int p = 0; p < i.num_planes; p++) {
      if (!r->params.uses_lr || !r->params.frame_restoration_type[p] || !m.lr_units[p]) continue;
      const size_t n = size_t(r->params.lr_unit_rows[p]) * size_t(r->params.lr_unit_cols[p]);
      if (n > L.lr_cap[p]) {
        std::lock_guard<std::mutex> lk(s->mu);
        st->pool_in.push_back(r->hin);
        delete r;
        set_error("serving: too many restoration units");
        return AV1PF_ERR_INVALID_INPUT;
      }
      std::memcpy(b + L.lr_off[p], m.lr_units[p], n * sizeof(av1pf_lr_unit));
    }
  }
  *out = r;
  return AV1PF_OK;
}

// Gives back what prepare_request took for a request that will not run.
void discard_request(av1pf_server* s, Request* r) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->hin) r->st->pool_in.push_back(r->hin);
  delete r;
}

// Queues prepared requests in order under one lock, so the worker sees them
// together.
void enqueue(av1pf_server* s, Request* const* rs, int n, uint64_t* tickets) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const double t = now_ms();
    for (int k = 0; k < n; k++) {
      Request* r = rs[k];
      r->ticket = s->next_ticket++;
      r->t_submit = t;
      s->tickets[r->ticket] = r;
      s->queue.push_back(r);
      s->submitted++;
      tickets[k] = r->ticket;
    }
  }
  s->cv.notify_one();
}

}  // namespace

extern "C" {

int av1pf_serve_open(av1pf_ctx* ctx, const av1pf_serve_config* cfg, av1pf_server** out) {
  if (!ctx || !out) return AV1PF_ERR_INVALID_INPUT;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  av1pf_server* s = new av1pf_server();
  s->ctx = ctx;
  if (cfg) s->cfg = *cfg;
  const int nb = s->cfg.inflight_batches > 0 ? s->cfg.inflight_batches : 2;
  for (int i = 0; i < nb; i++) {
    InFlight* b = new InFlight();
    b->wake = &s->cv;
    if ((e = cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming)) != cudaSuccess) {
      delete b;
      av1pf_serve_close(s);
      return cuda_status(e, "serving: stream create");
    }
    s->inflight.push_back(b);
  }
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return AV1PF_OK;
}

int av1pf_serve_open_stream(av1pf_server* s, const av1pf_frame_info* info, int32_t* stream_id) {
  if (!s || !info || !stream_id) return AV1PF_ERR_INVALID_INPUT;
  std::string why;
  int rc = validate_frame(info, nullptr, nullptr, &why);
  if (rc != AV1PF_OK) {
    set_error(why);
    return rc;
  }
  cudaSetDevice(s->ctx->device);
  Stream* st = new Stream();
  st->info = *info;
  st->lay.build(*info);
  const int nslots = s->cfg.slots_per_stream > 0 ? std::min(s->cfg.slots_per_stream, 64) : 2;
  std::lock_guard<std::mutex> lk(s->mu);
  const size_t need = nslots * (st->lay.bytes + st->lay.ref_bytes + align256(st->lay.frame_bytes)) + 3 * 256;
  if (s->cfg.hbm_cap_bytes && s->held + need > s->cfg.hbm_cap_bytes) {
    delete st;
    s->refused++;
    set_error("serving: stream refused, its frame slots would exceed the HBM cap");
    return AV1PF_ERR_ADMISSION;
  }
  st->slots.resize(nslots);
  for (Slot& sl : st->slots) {
    if ((rc = s->dev_alloc(&sl.dblob, st->lay.bytes)) || (rc = s->dev_alloc(&sl.dref, st->lay.ref_bytes)) ||
        (rc = s->dev_alloc(&sl.dframe, align256(st->lay.frame_bytes)))) {
      for (Slot& x : st->slots) {
        s->dev_free(x.dblob, st->lay.bytes);
        s->dev_free(x.dref, st->lay.ref_bytes);
        s->dev_free(x.dframe, align256(st->lay.frame_bytes));
      }
      delete st;
      return rc;
    }
  }
  st->id = s->next_stream++;
  s->streams[st->id] = st;
  *stream_id = st->id;
  return AV1PF_OK;
}

int av1pf_serve_close_stream(av1pf_server* s, int32_t stream_id) {
  if (!s) return AV1PF_ERR_INVALID_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->streams.find(stream_id);
  if (it == s->streams.end()) return AV1PF_ERR_NOT_FOUND;
  Stream* st = it->second;
  st->closing = true;
  // wait for the stream's queued and running frames
  auto busy = [&] {
    if (st->running || st->copying) return true;
    for (Request* r : s->queue)
      if (r->stream == stream_id) return true;
    return false;
  };
  while (busy()) s->cv_done.wait_for(lk, std::chrono::milliseconds(5));
  // results not polled yet lose their buffers with the stream: a later poll
  // of such a ticket reports the loss instead of reading freed memory
  for (auto& tr : s->tickets) {
    Request* r = tr.second;
    if (r->stream != stream_id || !r->hres) continue;
    r->hres = nullptr;
    if (r->state == 2) {
      r->state = 3;
      r->status = AV1PF_ERR_NOT_FOUND;
    }
  }
  cudaSetDevice(s->ctx->device);
  for (Slot& x : st->slots) {
    s->dev_free(x.dblob, st->lay.bytes);
    s->dev_free(x.dref, st->lay.ref_bytes);
    s->dev_free(x.dframe, align256(st->lay.frame_bytes));
  }
  for (void* p : st->all_pinned) cudaFreeHost(p);
  s->streams.erase(it);
  delete st;
  return AV1PF_OK;
}

int av1pf_serve_submit(av1pf_server* s, int32_t stream_id, const av1pf_request* req, uint64_t* ticket) {
  if (!ticket) return AV1PF_ERR_INVALID_INPUT;
  Request* r = nullptr;
  const int rc = prepare_request(s, stream_id, req, &r);
  if (rc != AV1PF_OK) return rc;
  enqueue(s, &r, 1, ticket);
  return AV1PF_OK;
}

int av1pf_serve_submit_many(av1pf_server* s, int32_t n, const int32_t* stream_ids, const av1pf_request* reqs,
                            uint64_t* tickets) {
  if (!s || n < 0 || (n > 0 && (!stream_ids || !reqs || !tickets))) return AV1PF_ERR_INVALID_INPUT;
  std::vector<Request*> rs(size_t(n), nullptr);
  std::vector<int> rcs(size_t(n), AV1PF_OK);
  std::vector<std::string> why(static_cast<size_t>(n));
  // Host requests are copied into pinned staging at submit time; a large
  // group spreads those copies over a few threads (host memory bandwidth,
  // not one core, then bounds them). Each thread takes every nt-th request.
  int host_reqs = 0;
  for (int k = 0; k < n; k++) host_reqs += reqs[k].device ? 0 : 1;
  const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
  const int nt = std::max(1, std::min({8, hw / 2, host_reqs / 4}));
  auto prep = [&](int t) {
    for (int k = t; k < n; k += nt) {
      rcs[size_t(k)] = prepare_request(s, stream_ids[k], &reqs[k], &rs[size_t(k)]);
      if (rcs[size_t(k)] != AV1PF_OK) why[size_t(k)] = av1pf_last_error();
    }
  };
  if (nt == 1) {
    prep(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(prep, t);
    prep(0);
    for (std::thread& x : th) x.join();
  }
  for (int k = 0; k < n; k++) {
    if (rcs[size_t(k)] == AV1PF_OK) continue;
    for (Request* q : rs)
      if (q) discard_request(s, q);
    set_error("serving: request " + std::to_string(k) + " of the group refused (none queued): " + why[size_t(k)]);
    return rcs[size_t(k)];
  }
  if (n > 0) enqueue(s, rs.data(), n, tickets);
  return AV1PF_OK;
}

int av1pf_serve_poll(av1pf_server* s, uint64_t ticket, int32_t wait_ms, uint8_t* frame_out, double* latency_ms) {
  if (!s) return AV1PF_ERR_INVALID_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return AV1PF_ERR_NOT_FOUND;
  Request* r = it->second;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(std::max(0, wait_ms));
  while (r->state < 2) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && r->state < 2) return AV1PF_ERR_TIMEOUT;
  }
  const int status = r->state == 2 ? AV1PF_OK : r->status;
  s->tickets.erase(it);
  // the result copy runs without the lock, so the worker and other callers
  // are not held up by it; the request is this caller's alone now, and the
  // stream's pinned buffers stay allocated while `copying` counts it
  if (r->hres) r->st->copying++;
  lk.unlock();
  if (status == AV1PF_OK) {
    if (frame_out && r->hres) std::memcpy(frame_out, r->hres, r->st->lay.frame_bytes);
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
  }
  if (r->hres) {
    lk.lock();
    r->st->pool_out.push_back(r->hres);
    r->st->copying--;
    lk.unlock();
    s->cv_done.notify_all();
  }
  delete r;
  return status;
}

int av1pf_serve_stats_get(av1pf_server* s, av1pf_serve_stats* out) {
  if (!s || !out) return AV1PF_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->refused = s->refused;
  out->batches = s->batches;
  out->mean_batch_frames = s->batches ? double(s->batch_frames) / double(s->batches) : 0.0;
  out->resident_bytes = s->held;
  if (!s->latencies.empty()) {
    std::vector<double> v = s->latencies;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v[std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
  }
  return AV1PF_OK;
}

int av1pf_serve_close(av1pf_server* s) {
  if (!s) return AV1PF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->device);
  for (InFlight* b : s->inflight) {
    if (b->s) cudaStreamSynchronize(b->s);
    if (b->side) cudaStreamSynchronize(b->side);
  }
  for (auto& kv : s->streams) {
    Stream* st = kv.second;
    for (Slot& x : st->slots) {
      s->dev_free(x.dblob, st->lay.bytes);
      s->dev_free(x.dref, st->lay.ref_bytes);
      s->dev_free(x.dframe, align256(st->lay.frame_bytes));
    }
    for (void* p : st->all_pinned) cudaFreeHost(p);
    delete st;
  }
  for (InFlight* b : s->inflight) {
    s->dev_free(b->scratch, b->scratch_size);
    s->dev_free(b->meta, b->meta_size);
    if (b->meta_host) cudaFreeHost(b->meta_host);
    if (b->s) cudaStreamDestroy(b->s);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    delete b;
  }
  for (auto& kv : s->tickets) delete kv.second;
  delete s;
  return AV1PF_OK;
}

}  // extern "C"
