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

// Planes covering each plane's visible (upscaled) area, 16-byte aligned rows.
int check_visible(const av1pf_frame_info* i, const av1pf_plane* pl, const char* what) {
  if (!pl) return fail_input(what);
  for (int p = 0; p < i->num_planes; p++) {
    const int sx = p ? i->subsampling_x : 0, sy = p ? i->subsampling_y : 0;
    if (!pl[p].data) return fail_input(what);
    if ((reinterpret_cast<uintptr_t>(pl[p].data) & 15) || ((pl[p].stride * i->sample_bytes) & 15))
      return fail_input("planes and rows must be 16-byte aligned");
    if (pl[p].stride < pl[p].width || pl[p].width < ((i->upscaled_width + sx) >> sx) ||
        pl[p].height < ((i->frame_height + sy) >> sy))
      return fail_input("plane smaller than the visible frame");
  }
  return AV1PF_OK;
}

int coded_sec(int coded) { return coded == 3 ? 4 : coded; }  // encoder/cdef.rs:43-46
int damping_for(int qidx) { return std::min(qidx >> 6, 3); }  // encoder/cdef.rs:255-258

}  // namespace

extern "C" {

int av1pf_cdef_search_many(av1pf_ctx* ctx, int n, const av1pf_cdef_search_job* jobs, int32_t thorough,
                           void* stream) {
  int rc = enter(ctx);
  if (rc) return rc;
  if (n <= 0 || n > 4096 || !jobs) return fail_input("bad job count");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<std::pair<int, int>> yc, uvc;
  cdef_candidates(thorough != 0, yc, uvc);
  const int ny = int(yc.size()), nuv = int(uvc.size()), nc = ny + nuv, ncand = ny * nuv;
  // layout: descriptors and greedy states, then per frame its totals, error
  // table and minima; the results (pairs and index table) of every frame
  // sit together so that one copy brings them back
  struct Geo {
    int fb_rows, fb_cols, nfb;
    size_t table_bytes, o_tot, o_sse, o_best, o_res;
  };
  std::vector<Geo> geo(static_cast<size_t>(n));
  std::string why;
  const size_t o_descs = align256(size_t(n) * sizeof(FrameDesc));
  const size_t o_g = o_descs + align256(size_t(n) * sizeof(CdefSearchDesc));
  size_t off = o_g + align256(size_t(n) * sizeof(CdefGreedy));
  size_t res_bytes = 0;
  int blocks = 0, entries = 0;
  for (int i = 0; i < n; i++) {
    const av1pf_cdef_search_job& jb = jobs[i];
    const av1pf_frame_info* info = jb.info;
    if ((rc = validate_frame(info, nullptr, jb.cur, &why)) != AV1PF_OK) return set_error(why), rc;
    if ((rc = check_src(info, jb.src)) != AV1PF_OK) return rc;
    Geo& G = geo[size_t(i)];
    G.fb_rows = (info->mi_rows + 15) / 16;
    G.fb_cols = (info->mi_cols + 15) / 16;
    G.nfb = G.fb_rows * G.fb_cols;
    const av1pf_maps* maps = jb.maps;
    if (!maps || !maps->mi || maps->mi_stride < info->mi_cols) return fail_input("mi map missing or mi_stride < mi_cols");
    if (!maps->cdef_idx || maps->cdef_stride < G.fb_cols) return fail_input("cdef_idx missing or cdef_stride too small");
    if (jb.base_q_idx < 0 || jb.base_q_idx > 255) return fail_input("base_q_idx out of range");
    if (!std::isfinite(jb.lambda) || jb.lambda < 0) return fail_input("lambda must be finite and >= 0");
    if (!jb.result) return fail_input("null result");
    G.table_bytes = size_t(G.fb_rows) * size_t(maps->cdef_stride);
    G.o_tot = off;
    G.o_sse = G.o_tot + align256(size_t(ncand) * 8);
    G.o_best = G.o_sse + align256(size_t(nc) * size_t(G.nfb) * 8);
    off = G.o_best + align256(size_t(G.nfb) * 8);
    G.o_res = res_bytes;  // within the results region: 18 ints, then the index table
    res_bytes += align256(18 * sizeof(int32_t) + G.table_bytes);
    blocks += G.nfb;
    entries += int(G.table_bytes);
  }
  const size_t o_results = off, dev_bytes = o_results + res_bytes;
  size_t sse_bytes = 0;
  for (int i = 0; i < n; i++)
    if (jobs[i].block_sse) sse_bytes += size_t(nc) * size_t(geo[size_t(i)].nfb) * 8;
  const size_t host_bytes = o_g + res_bytes + sse_bytes;
  if ((rc = ctx->ensure(ctx->search_dev, dev_bytes)) != AV1PF_OK) return rc;
  if ((rc = ctx->ensure_host(ctx->search_host, host_bytes)) != AV1PF_OK) return rc;
  uint8_t* dv = static_cast<uint8_t*>(ctx->search_dev.ptr);
  uint8_t* hs = static_cast<uint8_t*>(ctx->search_host.ptr);
  auto* hframes = reinterpret_cast<FrameDesc*>(hs);
  auto* hdescs = reinterpret_cast<CdefSearchDesc*>(hs + o_descs);
  const auto* dframes = reinterpret_cast<const FrameDesc*>(dv);
  auto* dg = reinterpret_cast<CdefGreedy*>(dv + o_g);
  int block0 = 0, table0 = 0;
  for (int i = 0; i < n; i++) {
    const av1pf_cdef_search_job& jb = jobs[i];
    const av1pf_frame_info* info = jb.info;
    const Geo& G = geo[size_t(i)];
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
    for (int p = 0; p < f.np; p++) f.cur[p] = dplane(jb.cur[p]);
    f.mi = jb.maps->mi;
    f.mi_stride = jb.maps->mi_stride;
    f.cdef_idx = jb.maps->cdef_idx;
    f.cdef_stride = jb.maps->cdef_stride;
    hframes[i] = f;
    CdefSearchDesc d{};
    for (int p = 0; p < f.np; p++) d.src[p] = dplane(jb.src[p]);
    d.ny = ny;
    d.nuv = nuv;
    d.damping = damping_for(jb.base_q_idx) + 3;
    d.fb_rows = G.fb_rows;
    d.fb_cols = G.fb_cols;
    for (int k = 0; k < ny; k++) {
      d.y_pri[k] = int8_t(yc[size_t(k)].first);
      d.y_sec[k] = int8_t(coded_sec(yc[size_t(k)].second));
    }
    for (int k = 0; k < nuv; k++) {
      d.uv_pri[k] = int8_t(uvc[size_t(k)].first);
      d.uv_sec[k] = int8_t(coded_sec(uvc[size_t(k)].second));
    }
    d.sse = reinterpret_cast<uint64_t*>(dv + G.o_sse);
    d.best = reinterpret_cast<uint64_t*>(dv + G.o_best);
    d.frame = dframes + i;
    d.g = dg + i;
    d.tot = reinterpret_cast<uint64_t*>(dv + G.o_tot);
    d.cdef_idx = jb.maps->cdef_idx;
    d.cdef_stride = jb.maps->cdef_stride;
    d.res = reinterpret_cast<int32_t*>(dv + o_results + G.o_res);
    d.table = reinterpret_cast<int8_t*>(dv + o_results + G.o_res + 18 * sizeof(int32_t));
    d.lambda = jb.lambda;
    d.block0 = block0;
    d.table0 = table0;
    block0 += G.nfb;
    table0 += int(G.table_bytes);
    hdescs[i] = d;
  }
  const auto* ddescs = reinterpret_cast<const CdefSearchDesc*>(dv + o_descs);
  cudaError_t e = cudaMemcpyAsync(dv, hs, o_g, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dg, 0, size_t(n) * sizeof(CdefGreedy), s);
  if (e != cudaSuccess) return cuda_status(e, "search upload");
  launch_cdef_search(ddescs, n, blocks, thorough != 0, s);
  for (int step = 0; step < 8; step++) launch_cdef_greedy_step(ddescs, n, ncand, s);
  launch_cdef_greedy_finish(ddescs, n, entries, s);
  e = cudaMemcpyAsync(hs + o_g, dv + o_results, res_bytes, cudaMemcpyDeviceToHost, s);
  size_t so = o_g + res_bytes;
  for (int i = 0; i < n && e == cudaSuccess; i++) {
    if (!jobs[i].block_sse) continue;
    const size_t bytes = size_t(nc) * size_t(geo[size_t(i)].nfb) * 8;
    e = cudaMemcpyAsync(hs + so, dv + geo[size_t(i)].o_sse, bytes, cudaMemcpyDeviceToHost, s);
    so += bytes;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "CDEF search");
  so = o_g + res_bytes;
  for (int i = 0; i < n; i++) {
    const av1pf_cdef_search_job& jb = jobs[i];
    const Geo& G = geo[size_t(i)];
    const int32_t* res = reinterpret_cast<const int32_t*>(hs + o_g + G.o_res);
    av1pf_cdef_search_result* result = jb.result;
    std::memset(result, 0, sizeof(*result));
    if (res[0] > 0) {  // else CdefParams::off(): one all-zero entry, damping_minus_3 0
      result->damping_minus_3 = damping_for(jb.base_q_idx);
      result->bits = res[1];
      for (int k = 0; k < (1 << res[1]); k++) {
        result->y_pri[k] = yc[size_t(res[2 + k])].first;
        result->y_sec[k] = yc[size_t(res[2 + k])].second;
        result->uv_pri[k] = uvc[size_t(res[10 + k])].first;
        result->uv_sec[k] = uvc[size_t(res[10 + k])].second;
      }
    }
    if (jb.cdef_idx_out) std::memcpy(jb.cdef_idx_out, hs + o_g + G.o_res + 18 * sizeof(int32_t), G.table_bytes);
    if (jb.block_sse) {  // candidate-major on the device, block-major for the caller
      const uint64_t* t = reinterpret_cast<const uint64_t*>(hs + so);
      for (int k = 0; k < nc; k++)
        for (int b = 0; b < G.nfb; b++) jb.block_sse[size_t(b) * size_t(nc) + size_t(k)] = t[size_t(k) * size_t(G.nfb) + size_t(b)];
      so += size_t(nc) * size_t(G.nfb) * 8;
    }
  }
  return AV1PF_OK;
}

int av1pf_cdef_search(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_maps* maps, const av1pf_plane* cur,
                      const av1pf_plane* src, int32_t base_q_idx, double lambda, int32_t thorough,
                      av1pf_cdef_search_result* result, int8_t* cdef_idx_out, uint64_t* block_sse, void* stream) {
  const av1pf_cdef_search_job job{info, maps, cur, src, base_q_idx, lambda, result, cdef_idx_out, block_sse};
  return av1pf_cdef_search_many(ctx, 1, &job, thorough, stream);
}

int av1pf_lf_search_many(av1pf_ctx* ctx, int n, av1pf_lf_search_job* jobs, void* stream) {
  int rc = enter(ctx);
  if (rc) return rc;
  if (n <= 0 || n > 1024 || !jobs) return fail_input("bad job count");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::string why;
  // the six scales of the starting levels (encoder/mod.rs:1470-1472)
  static const double kScales[6] = {0.0, 0.5, 0.75, 1.0, 1.25, 1.5};
  struct Frame {
    int32_t levels[6][4];
    size_t bytes, plane_off[3];
    int filtered[6];  // index of the filtered copy of each scale, or -1
  };
  std::vector<Frame> fr(static_cast<size_t>(n));
  size_t copy_bytes = 0;
  int copies = 0;
  for (int fi = 0; fi < n; fi++) {
    const av1pf_lf_search_job& jb = jobs[fi];
    const av1pf_frame_info* info = jb.info;
    if (!jb.params) return fail_input("null params");
    if ((rc = validate_frame(info, jb.params, jb.cur, &why)) != AV1PF_OK) return set_error(why), rc;
    if ((rc = check_src(info, jb.src)) != AV1PF_OK) return rc;
    const av1pf_maps* maps = jb.maps;
    if (!maps || !maps->mi || maps->mi_stride < info->mi_cols) return fail_input("mi map missing or mi_stride < mi_cols");
    for (int p = 0; p < info->num_planes; p++)
      if (!maps->lf_tx_size[p]) return fail_input("lf_tx_size map missing");
    Frame& F = fr[size_t(fi)];
    F.bytes = 0;
    for (int p = 0; p < info->num_planes; p++) {
      F.plane_off[p] = F.bytes;
      F.bytes += align256(size_t(jb.cur[p].height) * size_t(jb.cur[p].stride) * size_t(info->sample_bytes));
    }
    for (int si = 0; si < 6; si++) {
      for (int k = 0; k < 4; k++)
        F.levels[si][k] = std::min(int32_t(std::round(double(jb.params->loop_filter_level[k]) * kScales[si])), 63);
      F.filtered[si] = (F.levels[si][0] || F.levels[si][1]) ? copies++ : -1;
      if (F.filtered[si] >= 0) copy_bytes += F.bytes;
    }
  }
  // filtered copies, one per (frame, scale that filters), filtered in place as one batch
  if ((rc = ctx->ensure(ctx->search_planes, std::max<size_t>(1, copy_bytes))) != AV1PF_OK) return rc;
  uint8_t* base = static_cast<uint8_t*>(ctx->search_planes.ptr);
  std::vector<uint8_t*> copy_at(static_cast<size_t>(copies));
  std::vector<av1pf_params> prm(static_cast<size_t>(copies));
  std::vector<std::array<av1pf_plane, 3>> planes(static_cast<size_t>(copies));
  std::vector<FrameJob> fjobs;
  cudaError_t e = cudaSuccess;
  size_t at = 0;
  for (int fi = 0; fi < n; fi++) {
    const av1pf_lf_search_job& jb = jobs[fi];
    const Frame& F = fr[size_t(fi)];
    for (int si = 0; si < 6; si++) {
      const int ci = F.filtered[si];
      if (ci < 0) continue;
      copy_at[size_t(ci)] = base + at;
      prm[size_t(ci)] = *jb.params;
      for (int k = 0; k < 4; k++) prm[size_t(ci)].loop_filter_level[k] = F.levels[si][k];
      for (int p = 0; p < jb.info->num_planes; p++) {
        uint8_t* dst = base + at + F.plane_off[p];
        const size_t bytes = size_t(jb.cur[p].height) * size_t(jb.cur[p].stride) * size_t(jb.info->sample_bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, jb.cur[p].data, bytes, cudaMemcpyDeviceToDevice, s);
        planes[size_t(ci)][size_t(p)] = jb.cur[p];
        planes[size_t(ci)][size_t(p)].data = dst;
      }
      fjobs.push_back(FrameJob{jb.info, &prm[size_t(ci)], jb.maps, planes[size_t(ci)].data(), nullptr,
                               planes[size_t(ci)].data(), nullptr, ST_LF, true});
      at += F.bytes;
    }
  }
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search copies");
  if (!fjobs.empty() && (rc = ctx->run(fjobs.data(), int(fjobs.size()), s)) != AV1PF_OK) return rc;
  // the errors of every (frame, scale, plane) in one launch
  std::vector<SsePlane> sj;
  int rows_max = 0;
  for (int fi = 0; fi < n; fi++) {
    const av1pf_lf_search_job& jb = jobs[fi];
    const av1pf_frame_info* info = jb.info;
    const Frame& F = fr[size_t(fi)];
    for (int si = 0; si < 6; si++)
      for (int p = 0; p < info->num_planes; p++) {
        const int sx = p ? info->subsampling_x : 0, sy = p ? info->subsampling_y : 0;
        SsePlane j{};
        j.a = F.filtered[si] < 0 ? static_cast<const uint8_t*>(jb.cur[p].data)
                                 : copy_at[size_t(F.filtered[si])] + F.plane_off[p];
        j.b = static_cast<const uint8_t*>(jb.src[p].data);
        j.sa = jb.cur[p].stride;
        j.sb_ = jb.src[p].stride;
        j.w = (info->frame_width + sx) >> sx;
        j.h = (info->frame_height + sy) >> sy;
        j.sb = info->sample_bytes;
        rows_max = std::max(rows_max, j.h);
        sj.push_back(j);
      }
  }
  const size_t jb_bytes = sj.size() * sizeof(SsePlane), o_sse = align256(jb_bytes);
  const size_t total = o_sse + align256(sj.size() * sizeof(uint64_t));
  if ((rc = ctx->ensure(ctx->search_dev, total)) != AV1PF_OK) return rc;
  if ((rc = ctx->ensure_host(ctx->search_host, total)) != AV1PF_OK) return rc;
  uint8_t* dv = static_cast<uint8_t*>(ctx->search_dev.ptr);
  uint8_t* hs = static_cast<uint8_t*>(ctx->search_host.ptr);
  std::memcpy(hs, sj.data(), jb_bytes);
  e = cudaMemcpyAsync(dv, hs, jb_bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dv + o_sse, 0, sj.size() * sizeof(uint64_t), s);
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search");
  launch_plane_sse(reinterpret_cast<const SsePlane*>(dv), int(sj.size()), rows_max,
                   reinterpret_cast<uint64_t*>(dv + o_sse), s);
  e = cudaMemcpyAsync(hs + o_sse, dv + o_sse, sj.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "loop-filter search");
  // each plane's level with the least error, the first scale on ties
  // (encoder/mod.rs:1477-1492)
  const uint64_t* hsse = reinterpret_cast<const uint64_t*>(hs + o_sse);
  size_t k = 0;
  for (int fi = 0; fi < n; fi++) {
    av1pf_lf_search_job& jb = jobs[fi];
    const int np = jb.info->num_planes;
    const Frame& F = fr[size_t(fi)];
    uint64_t best_e[3] = {UINT64_MAX, UINT64_MAX, UINT64_MAX};
    int32_t best_l[3] = {0, 0, 0};
    if (jb.sse_out)
      for (int q = 0; q < 18; q++) jb.sse_out[q] = 0;
    for (int si = 0; si < 6; si++)
      for (int p = 0; p < np; p++) {
        const uint64_t err = hsse[k++];
        if (jb.sse_out) jb.sse_out[si * 3 + p] = err;
        if (err < best_e[p]) {
          best_e[p] = err;
          best_l[p] = p == 0 ? F.levels[si][0] : F.levels[si][1 + p];
        }
      }
    if (best_l[0] == 0) {
      for (int q = 0; q < 4; q++) jb.levels_out[q] = 0;
    } else {
      jb.levels_out[0] = jb.levels_out[1] = best_l[0];
      jb.levels_out[2] = best_l[1];
      jb.levels_out[3] = best_l[2];
    }
  }
  return AV1PF_OK;
}

int av1pf_lf_search(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                    const av1pf_maps* maps, const av1pf_plane* cur, const av1pf_plane* src, int32_t levels_out[4],
                    uint64_t* sse_out, void* stream) {
  if (!levels_out) return fail_input("null levels_out");
  av1pf_lf_search_job job{};
  job.info = info;
  job.params = params;
  job.maps = maps;
  job.cur = cur;
  job.src = src;
  job.sse_out = sse_out;
  if (!info) return fail_input("null frame info");
  const int rc = av1pf_lf_search_many(ctx, 1, &job, stream);
  if (rc == AV1PF_OK)
    for (int q = 0; q < 4; q++) levels_out[q] = job.levels_out[q];
  return rc;
}

int av1pf_lr_search_many(av1pf_ctx* ctx, int n, av1pf_lr_search_job* jobs_in, int32_t effort, void* stream) {
  int rc = enter(ctx);
  if (rc) return rc;
  if (n <= 0 || n > 4096 || !jobs_in) return fail_input("bad job count");
  if (effort < 0 || effort > 2) return fail_input("effort must be 0 (fast), 1 (normal) or 2 (thorough)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  LrSearchDesc d{};
  // encoder/lr.rs:74-81: parameter sets and the fit's sampling step
  static const int kNormal[6] = {0, 3, 6, 10, 13, 14}, kFast[2] = {3, 10};
  if (effort == 2) {
    d.nsets = 16;
    for (int k = 0; k < 16; k++) d.sets[k] = k;
  } else if (effort == 1) {
    d.nsets = 6;
    for (int k = 0; k < 6; k++) d.sets[k] = kNormal[k];
  } else {
    d.nsets = 2;
    for (int k = 0; k < 2; k++) d.sets[k] = kFast[k];
  }
  d.step = effort == 0 ? 2 : 1;
  std::vector<LrSearchFrame> frames(static_cast<size_t>(n));
  std::vector<av1pf_params> grids(static_cast<size_t>(n));
  std::vector<LrSearchJob> jobs;
  std::vector<LrSearchRect> rects;
  std::vector<std::array<int, 4>> where;  // (frame, plane, unit row, unit column) of each job
  std::string why;
  for (int fi = 0; fi < n; fi++) {
    const av1pf_lr_search_job& jb = jobs_in[fi];
    const av1pf_frame_info* info = jb.info;
    if (!jb.params) return fail_input("null params");
    // the unit grid as a frame whose planes all use switchable restoration
    av1pf_params& q = grids[size_t(fi)];
    q = *jb.params;
    q.uses_lr = 1;
    for (int k = 0; k < 3; k++) q.frame_restoration_type[k] = 3;
    q.cdef_enabled = 0;
    if ((rc = validate_frame(info, &q, nullptr, &why)) != AV1PF_OK) return set_error(why), rc;
    if ((rc = check_visible(info, jb.cur, "null deblocked planes")) != AV1PF_OK ||
        (rc = check_visible(info, jb.cdef, "null CDEF planes")) != AV1PF_OK ||
        (rc = check_visible(info, jb.src, "null source planes")) != AV1PF_OK)
      return rc;
    if (!std::isfinite(jb.lambda)) return fail_input("lambda must be finite");
    LrSearchFrame& F = frames[size_t(fi)];
    F = LrSearchFrame{};
    F.bd = info->bit_depth;
    F.sb = info->sample_bytes;
    F.lambda = jb.lambda;
    const int np = info->num_planes;
    const int stripes = (info->frame_height + 8 + 63) / 64;
    for (int p = 0; p < np; p++) {
      const int sx = p ? info->subsampling_x : 0, sy = p ? info->subsampling_y : 0;
      F.cur[p] = dplane(jb.cur[p]);
      F.cdef[p] = dplane(jb.cdef[p]);
      F.src[p] = dplane(jb.src[p]);
      F.pex[p] = ((info->upscaled_width + sx) >> sx) - 1;
      F.pey[p] = ((info->frame_height + sy) >> sy) - 1;
      const int us = q.loop_restoration_size[p], urows = q.lr_unit_rows[p], ucols = q.lr_unit_cols[p];
      // lr_stripe (postfilter.rs:640-661): each stripe's unit row
      std::vector<std::vector<LrSearchRect>> by_row(static_cast<size_t>(urows));
      for (int st = 0; st < stripes; st++) {
        const int ss = (-8 + st * 64) >> sy, se = ss + (64 >> sy) - 1;
        const int y0 = std::max(ss, 0), y1 = std::min(se, F.pey[p]);
        if (y0 > y1) continue;
        const int luma_row = st * 64 >= 8 ? st * 64 - 8 : 0;
        const int ur = std::min(urows - 1, ((luma_row + 8) >> sy) / us);
        by_row[size_t(ur)].push_back(LrSearchRect{ss, se, y0, y1 - y0 + 1});
      }
      // jobs: every unit with a stripe and columns inside the plane (encoder/lr.rs:84-122)
      for (int ur = 0; ur < urows; ur++)
        for (int uc = 0; uc < ucols; uc++) {
          // lr_unit_cols (postfilter.rs:664-675)
          const int x0 = uc * us;
          const int x1 = uc + 1 == ucols ? F.pex[p] : std::min((uc + 1) * us - 1, F.pex[p]);
          if (x0 > F.pex[p] || by_row[size_t(ur)].empty()) continue;
          LrSearchJob job{fi, p, x0, x1 - x0 + 1, int32_t(rects.size()), int32_t(by_row[size_t(ur)].size())};
          for (const LrSearchRect& r : by_row[size_t(ur)]) {
            rects.push_back(r);
            d.hmax = std::max(d.hmax, r.h);
          }
          d.wmax = std::max(d.wmax, job.w);
          jobs.push_back(job);
          where.push_back({fi, p, ur, uc});
        }
    }
  }
  std::vector<av1pf_lr_unit> chosen(jobs.size());
  if (!jobs.empty()) {
    int upx_max = 0;
    for (const LrSearchJob& jb : jobs) {
      int px = 0;
      for (int r = 0; r < jb.nr; r++) px += rects[size_t(jb.r0 + r)].h * jb.w;
      upx_max = std::max(upx_max, px);
      if (jb.nr > 1) d.multi_rect = 1;
    }
    lr_search_shape(d.wmax, d.hmax, upx_max, d.band, d.cache_px, d.both);
    cudaError_t e = lr_search_init();
    if (e != cudaSuccess) return cuda_status(e, "loop-restoration search attributes");
    const size_t fb = frames.size() * sizeof(LrSearchFrame);
    const size_t jbb = jobs.size() * sizeof(LrSearchJob), rb = rects.size() * sizeof(LrSearchRect);
    const size_t ob = jobs.size() * sizeof(av1pf_lr_unit);
    const size_t stb = jobs.size() * sizeof(LrJobState), sgb = jobs.size() * size_t(d.nsets) * sizeof(LrSgrResult);
    const size_t o_jobs = align256(fb), o_rects = o_jobs + align256(jbb), o_out = o_rects + align256(rb);
    const size_t o_state = o_out + align256(ob), o_sgr = o_state + align256(stb), total = o_sgr + align256(sgb);
    if ((rc = ctx->ensure(ctx->search_dev, total)) != AV1PF_OK) return rc;
    if ((rc = ctx->ensure_host(ctx->search_host, o_state)) != AV1PF_OK) return rc;
    uint8_t* dv = static_cast<uint8_t*>(ctx->search_dev.ptr);
    uint8_t* hs = static_cast<uint8_t*>(ctx->search_host.ptr);
    std::memcpy(hs, frames.data(), fb);
    std::memcpy(hs + o_jobs, jobs.data(), jbb);
    std::memcpy(hs + o_rects, rects.data(), rb);
    d.frames = reinterpret_cast<const LrSearchFrame*>(dv);
    d.jobs = reinterpret_cast<const LrSearchJob*>(dv + o_jobs);
    d.rects = reinterpret_cast<const LrSearchRect*>(dv + o_rects);
    d.out = reinterpret_cast<av1pf_lr_unit*>(dv + o_out);
    d.state = reinterpret_cast<LrJobState*>(dv + o_state);
    d.sgr = reinterpret_cast<LrSgrResult*>(dv + o_sgr);
    e = cudaMemcpyAsync(dv, hs, o_out, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "loop-restoration search upload");
    launch_lr_search(d, int(jobs.size()), s, ctx->side, ctx->fork, ctx->join);
    e = cudaMemcpyAsync(hs + o_out, dv + o_out, ob, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "loop-restoration search");
    std::memcpy(chosen.data(), hs + o_out, ob);
  }
  // the plans: units without a job keep no filter (encoder/lr.rs:188-208)
  for (int fi = 0; fi < n; fi++) {
    av1pf_lr_search_job& jb = jobs_in[fi];
    const av1pf_params& q = grids[size_t(fi)];
    for (int p = 0; p < 3; p++) {
      jb.frame_type_out[p] = 0;
      if (p >= jb.info->num_planes || !jb.units_out[p]) continue;
      const size_t cnt = size_t(q.lr_unit_rows[p]) * size_t(q.lr_unit_cols[p]);
      for (size_t k = 0; k < cnt; k++) jb.units_out[p][k] = av1pf_lr_unit{};
    }
  }
  std::vector<std::array<std::array<bool, 3>, 3>> used(static_cast<size_t>(n));
  for (auto& u : used)
    for (auto& pl : u) pl = {false, false, false};
  for (size_t k = 0; k < jobs.size(); k++) {
    const int fi = where[k][0], p = where[k][1];
    av1pf_lr_search_job& jb = jobs_in[fi];
    used[size_t(fi)][size_t(p)][chosen[k].type] = true;
    if (jb.units_out[p])
      jb.units_out[p][size_t(where[k][2]) * size_t(grids[size_t(fi)].lr_unit_cols[p]) + size_t(where[k][3])] =
          chosen[k];
  }
  for (int fi = 0; fi < n; fi++) {
    av1pf_lr_search_job& jb = jobs_in[fi];
    for (int p = 0; p < jb.info->num_planes; p++) {
      const bool wu = used[size_t(fi)][size_t(p)][AV1PF_RESTORE_WIENER];
      const bool su = used[size_t(fi)][size_t(p)][AV1PF_RESTORE_SGRPROJ];
      jb.frame_type_out[p] = wu ? (su ? 3 : AV1PF_RESTORE_WIENER) : (su ? AV1PF_RESTORE_SGRPROJ : AV1PF_RESTORE_NONE);
    }
  }
  return AV1PF_OK;
}

int av1pf_lr_search(av1pf_ctx* ctx, const av1pf_frame_info* info, const av1pf_params* params,
                    const av1pf_plane* cur, const av1pf_plane* cdef, const av1pf_plane* src, double lambda,
                    int32_t effort, av1pf_lr_unit* const units_out[3], int32_t frame_type_out[3], void* stream) {
  if (!units_out || !frame_type_out) return fail_input("null outputs");
  av1pf_lr_search_job job{};
  job.info = info;
  job.params = params;
  job.cur = cur;
  job.cdef = cdef;
  job.src = src;
  job.lambda = lambda;
  for (int p = 0; p < 3; p++) job.units_out[p] = units_out[p];
  if (!info) return fail_input("null frame info");
  const int rc = av1pf_lr_search_many(ctx, 1, &job, effort, stream);
  if (rc == AV1PF_OK)
    for (int p = 0; p < 3; p++) frame_type_out[p] = job.frame_type_out[p];
  return rc;
}

}  // extern "C"
