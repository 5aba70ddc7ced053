// refs.cpp — device-resident reference frames: the reference frame update
// process (7.20) over frames the filter chain leaves on the device.
//
// Reference: rivet-av1 src/decoder/mod.rs:797-806 (the update:
// `self.refs[i] = Some(data.clone())` for every bit i of
// refresh_frame_flags) and :819-842 (show_existing_frame: the output process
// on a slot's frame, and for a key frame the update with that frame), with
// RefData (src/decoder/state.rs:79-101) shared between slots by Arc.
//
// Here a slot holds a device frame (the loop-restoration output over the
// visible area) by reference count: av1pf_refs_chain runs the chain with its
// reference frame written straight into a frame of the table, and the slots
// named by refresh_frame_flags take it. A frame no slot holds returns to the
// table's pool; later calls reuse it in stream order, so a table is used on
// one stream (or the caller orders its streams). A GPU decoder upstream reads
// the slots' planes for inter prediction without a copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "av1pf.h"
#include "ctx.h"
#include "plan.h"

namespace av1pf {

struct RefFrame {
  DevBuf buf;
  av1pf_frame_info info{};
  av1pf_plane planes[AV1PF_MAX_PLANES]{};
  uint32_t order_hint = 0;
  uint64_t id = 0;
  int holders = 0;  // slots that hold this frame
};

}  // namespace av1pf

struct av1pf_refs {
  av1pf_ctx* ctx = nullptr;
  std::vector<std::unique_ptr<av1pf::RefFrame>> frames;  // the pool
  av1pf::RefFrame* slot[8] = {};
  uint64_t next_id = 1;
};

namespace av1pf {
namespace {

// Bytes of a frame's visible planes, rows 64 samples apart, each plane 256-byte aligned.
size_t frame_bytes_of(const av1pf_frame_info* i, int64_t stride[3]) {
  size_t total = 0;
  for (int k = 0; k < i->num_planes; k++) {
    const int w = plane_w(i, k, i->upscaled_width), h = plane_h(i, k);
    stride[k] = (w + 63) / 64 * 64;
    total += (size_t(stride[k]) * size_t(h) * size_t(i->sample_bytes) + 255) / 256 * 256;
  }
  return total;
}

// A pool frame no slot holds, with room for a frame of `info` (grown when
// needed); a new one when every frame is held.
int take_frame(av1pf_refs* r, const av1pf_frame_info* info, RefFrame** out) {
  int64_t stride[3] = {0, 0, 0};
  const size_t need = frame_bytes_of(info, stride);
  RefFrame* f = nullptr;
  for (auto& p : r->frames)
    if (p->holders == 0 && (!f || (p->buf.size >= need && f->buf.size < need))) f = p.get();
  if (!f) {
    r->frames.push_back(std::make_unique<RefFrame>());
    f = r->frames.back().get();
  }
  const int rc = r->ctx->ensure(f->buf, need);
  if (rc != AV1PF_OK) return rc;
  f->info = *info;
  uint8_t* base = static_cast<uint8_t*>(f->buf.ptr);
  std::memset(f->planes, 0, sizeof(f->planes));
  for (int k = 0; k < info->num_planes; k++) {
    const int h = plane_h(info, k);
    f->planes[k].data = base;
    f->planes[k].stride = stride[k];
    f->planes[k].width = int32_t(stride[k]);
    f->planes[k].height = h;
    base += (size_t(stride[k]) * size_t(h) * size_t(info->sample_bytes) + 255) / 256 * 256;
  }
  *out = f;
  return AV1PF_OK;
}

// The reference frame update process: every slot with its bit set takes `f`.
void update_slots(av1pf_refs* r, RefFrame* f, uint32_t refresh_frame_flags) {
  for (int i = 0; i < 8; i++) {
    if (!((refresh_frame_flags >> i) & 1u)) continue;
    if (r->slot[i]) r->slot[i]->holders--;
    r->slot[i] = f;
    f->holders++;
  }
}

}  // namespace
}  // namespace av1pf

using namespace av1pf;

extern "C" {

int av1pf_refs_create(av1pf_ctx* ctx, av1pf_refs** out) {
  if (!ctx || !out) return AV1PF_ERR_INVALID_INPUT;
  *out = new av1pf_refs();
  (*out)->ctx = ctx;
  return AV1PF_OK;
}

int av1pf_refs_destroy(av1pf_refs* r) {
  if (!r) return AV1PF_ERR_INVALID_INPUT;
  cudaSetDevice(r->ctx->device);
  // frames may still be read by work in flight on the device
  cudaDeviceSynchronize();
  for (auto& f : r->frames) r->ctx->release(f->buf);
  delete r;
  return AV1PF_OK;
}

int av1pf_refs_chain(av1pf_refs* r, const av1pf_frame_info* info, const av1pf_params* params,
                     const av1pf_maps* maps, const av1pf_plane* in, uint32_t refresh_frame_flags,
                     uint32_t order_hint, uint8_t* frame_out, void* stream) {
  if (!r || !info || !params) return AV1PF_ERR_INVALID_INPUT;
  if (refresh_frame_flags > 0xffu) {
    set_error("refresh_frame_flags has 8 bits");
    return AV1PF_ERR_INVALID_INPUT;
  }
  cudaError_t e = cudaSetDevice(r->ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  int rc = av1pf_validate(info, params, in);
  if (rc != AV1PF_OK) return rc;
  RefFrame* f = nullptr;
  if ((rc = take_frame(r, info, &f)) != AV1PF_OK) return rc;
  if ((rc = av1pf_chain(r->ctx, info, params, maps, in, f->planes, frame_out, stream)) != AV1PF_OK) return rc;
  f->order_hint = order_hint;
  f->id = r->next_id++;
  update_slots(r, f, refresh_frame_flags);
  return AV1PF_OK;
}

int av1pf_refs_get(const av1pf_refs* r, int slot, av1pf_ref_frame* out) {
  if (!r || !out || slot < 0 || slot >= 8) return AV1PF_ERR_INVALID_INPUT;
  std::memset(out, 0, sizeof(*out));
  const RefFrame* f = r->slot[slot];
  if (!f) return AV1PF_OK;
  out->valid = 1;
  out->info = f->info;
  out->order_hint = f->order_hint;
  out->frame_id = f->id;
  for (int k = 0; k < AV1PF_MAX_PLANES; k++) out->planes[k] = f->planes[k];
  return AV1PF_OK;
}

int av1pf_refs_show(av1pf_refs* r, int slot, const av1pf_params* params, uint32_t refresh_frame_flags,
                    uint8_t* frame_out, void* stream) {
  if (!r || !params || !frame_out || slot < 0 || slot >= 8 || refresh_frame_flags > 0xffu)
    return AV1PF_ERR_INVALID_INPUT;
  RefFrame* f = r->slot[slot];
  if (!f) {
    set_error("show_existing_frame of an empty slot");
    return AV1PF_ERR_INVALID_INPUT;
  }
  cudaError_t e = cudaSetDevice(r->ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  const int rc = av1pf_output(r->ctx, &f->info, params, f->planes, frame_out, stream);
  if (rc != AV1PF_OK) return rc;
  update_slots(r, f, refresh_frame_flags);
  return AV1PF_OK;
}

int av1pf_refs_memory(const av1pf_refs* r, uint64_t* bytes, int32_t* frames) {
  if (!r || !bytes) return AV1PF_ERR_INVALID_INPUT;
  uint64_t b = 0;
  for (const auto& f : r->frames) b += f->buf.size;
  *bytes = b;
  if (frames) *frames = int32_t(r->frames.size());
  return AV1PF_OK;
}

}  // extern "C"
