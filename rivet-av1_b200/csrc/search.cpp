// search.cpp — C ABI of the encoder's filter searches: av1pf_cdef_search
// (encoder/cdef.rs:52-251) and av1pf_lf_search (encoder/mod.rs:1457-1506).
// Both run every candidate on the device in a few launches and return once
// the choice is on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "av1pf.h"
#include "ctx.h"
#include "desc.h"
#include "kernels.h"
#include "plan.h"

using namespace av1pf;

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int fail_input(const char* why) {
  set_error(why);
  return AV1PF_ERR_INVALID_INPUT;
}

int enter(av1pf_ctx* ctx) {
  if (!ctx) return fail_input("null context");
  return cuda_status(cudaSetDevice(ctx->device), "cudaSetDevice");
}

DPlane dplane(const av1pf_plane& p) {
  DPlane d{};
  d.p = static_cast<uint8_t*>(p.data);
  d.stride = p.stride;
  d.w = p.width;
  d.h = p.height;
  return d;
}

// Source planes: 16-byte aligned rows covering each plane's frame area.
int check_src(const av1pf_frame_info* i, const av1pf_plane* src) {
  if (!src) return fail_input("null source planes");
  for (int p = 0; p < i->num_planes; p++) {
    const int sx = p ? i->subsampling_x : 0, sy = p ? i->subsampling_y : 0;
    const av1pf_plane& pl = src[p];
    if (!pl.data) return fail_input("null source plane");
    if ((reinterpret_cast<uintptr_t>(pl.data) & 15) || ((pl.stride * i->sample_bytes) & 15))
      return fail_input("source planes and rows must be 16-byte aligned");
    if (pl.stride < pl.width || pl.width < ((i->frame_width + sx) >> sx) || pl.height < ((i->frame_height + sy) >> sy))
      return fail_input("source plane smaller than the frame");
  }
  return AV1PF_OK;
}

// encoder/cdef.rs:60-80
void cdef_candidates(bool thorough, std::vector<std::pair<int, int>>& y, std::vector<std::pair<int, int>>& uv) {
  static const int kYFast[] = {0, 1, 2, 4, 6, 9, 12}, kYThorough[] = {0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15};
  static const int kUvFast[] = {0, 1, 2, 4, 7}, kUvThorough[] = {0, 1, 2, 3, 4, 6, 8, 11};
  y.clear();
  uv.clear();
  if (thorough) {
    for (int p : kYThorough)
      for (int s = 0; s < 4; s++) y.emplace_back(p, s);
    for (int p : kUvThorough)
      for (int s = 0; s < 3; s++) uv.emplace_back(p, s);
  } else {
    for (int p : kYFast)
      for (int s = 0; s < 4; s++) y.emplace_back(p, s);
    for (int p : kUvFast)
      for (int s = 0; s < 3; s++) uv.emplace_back(p, s);
  }
}

int coded_sec(int coded) { return coded == 3 ? 4 : coded; }  // encoder/cdef.rs:43-46
int damping_for(int qidx) { return std::min(qidx >> 6, 3); }  // encoder/cdef.rs:255-258

}  // namespace

extern "C" {

int av1pf_cdef_search(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_maps* maps, const av1pf_plane* cur,
                      const av1pf_plane* src, int32_t base_q_idx, double lambda, int32_t thorough,
                      av1pf_cdef_search_result* result, int8_t* cdef_idx_out, uint64_t* block_sse, void* stream) {
  int rc = enter(ctx);
  if (rc) return rc;
  std::string why;
  if ((rc = validate_frame(info, nullptr, cur, &why)) != AV1PF_OK) return set_error(why), rc;
  if ((rc = check_src(info, src)) != AV1PF_OK) return rc;
  const int fb_rows = (info->mi_rows + 15) / 16, fb_cols = (info->mi_cols + 15) / 16;
  if (!maps || !maps->mi || maps->mi_stride < info->mi_cols) return fail_input("mi map missing or mi_stride < mi_cols");
  if (!maps->cdef_idx || maps->cdef_stride < fb_cols) return fail_input("cdef_idx missing or cdef_stride too small");
  if (base_q_idx < 0 || base_q_idx > 255) return fail_input("base_q_idx out of range");
  if (!std::isfinite(lambda) || lambda < 0) return fail_input("lambda must be finite and >= 0");
  if (!result) return fail_input("null result");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  std::vector<std::pair<int, int>> yc, uvc;
  cdef_candidates(thorough != 0, yc, uvc);
  FrameDesc f{};
  f.bd = info->bit_depth;
  f.sb = info->sample_bytes;
  f.ssx = info->subsampling_x;
  f.ssy = info->subsampling_y;
  f.np = info->num_planes;
  f.fw = info->frame_width;
  f.fh = info->frame_height;
  f.uw = info->upscaled_width;
  f.mi_rows = info->mi_rows;
  f.mi_cols = info->mi_cols;
  f.mc = info->matrix_coefficients;
  for (int p = 0; p < f.np; p++) f.cur[p] = dplane(cur[p]);
  f.mi = maps->mi;
  f.mi_stride = maps->mi_stride;
  f.cdef_idx = maps->cdef_idx;
  f.cdef_stride = maps->cdef_stride;

  CdefSearchDesc d{};
  for (int p = 0; p < f.np; p++) d.src[p] = dplane(src[p]);
  d.ny = int32_t(yc.size());
  d.nuv = int32_t(uvc.size());
  d.damping = damping_for(base_q_idx) + 3;
  d.fb_rows = fb_rows;
  d.fb_cols = fb_cols;
  for (size_t k = 0; k < yc.size(); k++) {
    d.y_pri[k] = int8_t(yc[k].first);
    d.y_sec[k] = int8_t(coded_sec(yc[k].second));
  }
  for (size_t k = 0; k < uvc.size(); k++) {
    d.uv_pri[k] = int8_t(uvc[k].first);
    d.uv_sec[k] = int8_t(coded_sec(uvc[k].second));
  }
  const size_t nfb = size_t(fb_rows) * size_t(fb_cols), nc = size_t(d.ny + d.nuv), ncand = size_t(d.ny * d.nuv);
  const size_t table_bytes = size_t(fb_rows) * size_t(maps->cdef_stride);
  // device: descriptor | greedy state | candidate totals | error table | minima | table | result
  const size_t o_desc = 0, o_g = align256(sizeof(FrameDesc)), o_tot = o_g + align256(sizeof(CdefGreedy));
  const size_t o_sse = o_tot + align256(ncand * 8), o_best = o_sse + align256(nc * nfb * 8);
  const size_t o_table = o_best + align256(nfb * 8), o_res = o_table + align256(table_bytes);
  const size_t dev_bytes = o_res + 256;
  // host staging: descriptor | result | table | error table
  const size_t h_res = align256(sizeof(FrameDesc)), h_table = h_res + 256, h_sse = h_table + align256(table_bytes);
  const size_t host_bytes = h_sse + (block_sse ? nc * nfb * 8 : 0);
  if ((rc = ctx->ensure(ctx->search_dev, dev_bytes)) != AV1PF_OK) return rc;
  if ((rc = ctx->ensure_host(ctx->search_host, host_bytes)) != AV1PF_OK) return rc;
  uint8_t* dv = static_cast<uint8_t*>(ctx->search_dev.ptr);
  uint8_t* hs = static_cast<uint8_t*>(ctx->search_host.ptr);
  d.sse = reinterpret_cast<uint64_t*>(dv + o_sse);
  d.best = reinterpret_cast<uint64_t*>(dv + o_best);
  auto* g = reinterpret_cast<CdefGreedy*>(dv + o_g);
  std::memcpy(hs, &f, sizeof(FrameDesc));
  cudaError_t e = cudaMemcpyAsync(dv + o_desc, hs, sizeof(FrameDesc), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g, 0, sizeof(CdefGreedy), s);
  if (e != cudaSuccess) return cuda_status(e, "search upload");
  launch_cdef_search(reinterpret_cast<const FrameDesc*>(dv + o_desc), d, g, s);
  for (int step = 0; step < 8; step++)
    launch_cdef_greedy_step(d, g, reinterpret_cast<uint64_t*>(dv + o_tot), lambda, s);
  launch_cdef_greedy_finish(d, g, maps->cdef_idx, maps->cdef_stride, reinterpret_cast<int8_t*>(dv + o_table),
                            reinterpret_cast<int32_t*>(dv + o_res), s);
  e = cudaMemcpyAsync(hs + h_res, dv + o_res, 18 * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hs + h_table, dv + o_table, table_bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && block_sse)
    e = cudaMemcpyAsync(hs + h_sse, dv + o_sse, nc * nfb * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "CDEF search");

  const int32_t* res = reinterpret_cast<const int32_t*>(hs + h_res);
  std::memset(result, 0, sizeof(*result));
  if (res[0] > 0) {  // else CdefParams::off(): one all-zero entry, damping_minus_3 0
    result->damping_minus_3 = damping_for(base_q_idx);
    result->bits = res[1];
    for (int i = 0; i < (1 << res[1]); i++) {
      result->y_pri[i] = yc[size_t(res[2 + i])].first;
      result->y_sec[i] = yc[size_t(res[2 + i])].second;
      result->uv_pri[i] = uvc[size_t(res[10 + i])].first;
      result->uv_sec[i] = uvc[size_t(res[10 + i])].second;
    }
  }
  if (cdef_idx_out) std::memcpy(cdef_idx_out, hs + h_table, table_bytes);
  if (block_sse) {  // candidate-major on the device, block-major for the caller
    const uint64_t* t = reinterpret_cast<const uint64_t*>(hs + h_sse);
    for (size_t k = 0; k < nc; k++)
      for (size_t b = 0; b < nfb; b++) block_sse[b * nc + k] = t[k * nfb + b];
  }
  return AV1PF_OK;
}

int av1pf_lf_search(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                    const av1pf_maps* maps, const av1pf_plane* cur, const av1pf_plane* src, int32_t levels_out[4],
                    uint64_t* sse_out, void* stream) {
  int rc = enter(ctx);
  if (rc) return rc;
  std::string why;
  if (!params) return fail_input("null params");
  if ((rc = validate_frame(info, params, cur, &why)) != AV1PF_OK) return set_error(why), rc;
  if ((rc = check_src(info, src)) != AV1PF_OK) return rc;
  if (!maps || !maps->mi || maps->mi_stride < info->mi_cols) return fail_input("mi map missing or mi_stride < mi_cols");
  for (int p = 0; p < info->num_planes; p++)
    if (!maps->lf_tx_size[p]) return fail_input("lf_tx_size map missing");
  if (!levels_out) return fail_input("null levels_out");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int np = info->num_planes, sb = info->sample_bytes;

  // the six scales of the starting levels (encoder/mod.rs:1470-1472)
  static const double kScales[6] = {0.0, 0.5, 0.75, 1.0, 1.25, 1.5};
  int32_t levels[6][4];
  for (int si = 0; si < 6; si++)
    for (int k = 0; k < 4; k++)
      levels[si][k] = std::min(int32_t(std::round(double(params->loop_filter_level[k]) * kScales[si])), 63);
  // a filtered copy of `cur` for each scale that filters
  size_t frame_bytes = 0;
  size_t plane_off[3] = {0, 0, 0};
  for (int p = 0; p < np; p++) {
    plane_off[p] = frame_bytes;
    frame_bytes += align256(size_t(cur[p].height) * size_t(cur[p].stride) * size_t(sb));
  }
  std::vector<int> filtered;
  for (int si = 0; si < 6; si++)
    if (levels[si][0] || levels[si][1]) filtered.push_back(si);
  if ((rc = ctx->ensure(ctx->search_planes, std::max<size_t>(1, filtered.size()) * frame_bytes)) != AV1PF_OK) return rc;
  if ((rc = ctx->ensure(ctx->search_dev, 256)) != AV1PF_OK) return rc;
  if ((rc = ctx->ensure_host(ctx->search_host, 256)) != AV1PF_OK) return rc;
  uint8_t* base = static_cast<uint8_t*>(ctx->search_planes.ptr);
  std::vector<av1pf_params> prm(filtered.size(), *params);
  std::vector<std::array<av1pf_plane, 3>> planes(filtered.size());
  std::vector<FrameJob> jobs;
  cudaError_t e = cudaSuccess;
  for (size_t i = 0; i < filtered.size(); i++) {
    for (int k = 0; k < 4; k++) prm[i].loop_filter_level[k] = levels[filtered[i]][k];
    for (int p = 0; p < np; p++) {
      uint8_t* dst = base + i * frame_bytes + plane_off[p];
      const size_t bytes = size_t(cur[p].height) * size_t(cur[p].stride) * size_t(sb);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dst, cur[p].data, bytes, cudaMemcpyDeviceToDevice, s);
      planes[i][size_t(p)] = cur[p];
      planes[i][size_t(p)].data = dst;
    }
    jobs.push_back(FrameJob{info, &prm[i], maps, planes[i].data(), nullptr, planes[i].data(), nullptr, ST_LF, true});
  }
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search copies");
  if (!jobs.empty() && (rc = ctx->run(jobs.data(), int(jobs.size()), s)) != AV1PF_OK) return rc;
  // the errors of every (scale, plane) in one launch
  std::vector<SsePlane> sj;
  int rows_max = 0;
  for (int si = 0; si < 6; si++) {
    const auto it = std::find(filtered.begin(), filtered.end(), si);
    for (int p = 0; p < np; p++) {
      const int sx = p ? info->subsampling_x : 0, sy = p ? info->subsampling_y : 0;
      SsePlane j{};
      j.a = it == filtered.end() ? static_cast<const uint8_t*>(cur[p].data)
                                 : base + size_t(it - filtered.begin()) * frame_bytes + plane_off[p];
      j.b = static_cast<const uint8_t*>(src[p].data);
      j.sa = cur[p].stride;
      j.sb_ = src[p].stride;
      j.w = (info->frame_width + sx) >> sx;
      j.h = (info->frame_height + sy) >> sy;
      rows_max = std::max(rows_max, j.h);
      sj.push_back(j);
    }
  }
  uint64_t* dsse = static_cast<uint64_t*>(ctx->search_dev.ptr);
  uint64_t* hsse = static_cast<uint64_t*>(ctx->search_host.ptr);
  e = cudaMemsetAsync(dsse, 0, 18 * sizeof(uint64_t), s);
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search");
  launch_plane_sse(sj.data(), int(sj.size()), sb, rows_max, dsse, s);
  e = cudaMemcpyAsync(hsse, dsse, 18 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search");

  // each plane's level with the least error, the first scale on ties
  // (encoder/mod.rs:1477-1492)
  uint64_t best_e[3] = {UINT64_MAX, UINT64_MAX, UINT64_MAX};
  int32_t best_l[3] = {0, 0, 0};
  for (int si = 0; si < 6; si++)
    for (int p = 0; p < np; p++) {
      const uint64_t err = hsse[si * np + p];
      if (sse_out) sse_out[si * 3 + p] = err;
      if (err < best_e[p]) {
        best_e[p] = err;
        best_l[p] = p == 0 ? levels[si][0] : levels[si][1 + p];
      }
    }
  if (sse_out)
    for (int si = 0; si < 6; si++)
      for (int p = np; p < 3; p++) sse_out[si * 3 + p] = 0;
  if (best_l[0] == 0) {
    for (int k = 0; k < 4; k++) levels_out[k] = 0;
  } else {
    levels_out[0] = levels_out[1] = best_l[0];
    levels_out[2] = best_l[1];
    levels_out[3] = best_l[2];
  }
  return AV1PF_OK;
}

}  // extern "C"
