// lf.cu — the deblocking loop filter (7.14) on the device.
//
// Reference: rivet-av1 src/decoder/postfilter.rs:63-264 (edge walk, filter
// size and strength) and src/dsp/lf.rs:58-211 (the sample filters).
//
// Design. The reference walks every 4x4 of a plane and filters edges in
// place, vertical edges first (bands of rows), then horizontal edges (bands
// of columns). Here:
//   1. lf_prep_kernel copies the pre-filter tile into the working plane and
//      decides, for every 4x4 and both passes, whether its edge is filtered
//      and with which size and level (edge_loop_filter's tests and
//      filter_strength, postfilter.rs:107-172, 207-264). Active edges are
//      appended (warp-aggregated) to one compact list per pass.
//   2. lf_edge_kernel<pass> runs one thread per (edge, lane) over the list,
//      in place, writing only the samples the chosen filter changes.
// Writing only changed samples makes the in-place passes order-independent:
// for conformant maps (transform blocks tile the plane) an edge's samples
// are read or changed by no other edge of the same pass, which is also what
// lets the reference run its bands on threads. The reference writes back
// its whole read span per edge; the extra samples it writes hold the values
// it read, so the results are the same.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

// 7.14.4-5 filter_strength (postfilter.rs:207-246): the level of one 4x4
// from its mode-info words.
__device__ __forceinline__ int lf_level_raw(const FrameDesc& f, uint2 raw, int plane, int pass) {
  const int mi_segment = int((raw.x >> 24) & 7u);
  const int rf = int(int8_t((raw.x >> 16) & 0xffu));
  const int mode = int((raw.x >> 8) & 0xffu);
  const int mode_type = (mode >= 14 && mode != 16 && mode != 24) ? 1 : 0;  // NEARESTMV.., !GLOBALMV, !GLOBAL_GLOBALMV
  const int i = plane == 0 ? pass : plane + 1;
  const int didx = f.delta_lf_multi ? i : 0;
  const int delta_lf = int(int8_t((raw.y >> (8 * didx)) & 0xffu));
  int lvl = clip3(0, 63, delta_lf + f.lf_level[i]);
  if (f.seg_enabled && f.seg_lf_on[mi_segment][i]) lvl = clip3(0, 63, f.seg_lf_data[mi_segment][i] + lvl);
  if (f.delta_enabled) {
    const int n_shift = lvl >> 5;
    if (rf == 0) {
      lvl += f.ref_deltas[0] * (1 << n_shift);
    } else if (rf > 0) {
      lvl += f.ref_deltas[rf & 7] * (1 << n_shift) + f.mode_deltas[mode_type] * (1 << n_shift);
    }
    lvl = clip3(0, 63, lvl);
  }
  return lvl;
}

__device__ __forceinline__ int lf_level(const FrameDesc& f, int row, int col, int plane, int pass) {
  return lf_level_raw(f, *reinterpret_cast<const uint2*>(f.mi + int64_t(row) * f.mi_stride + col), plane, pass);
}

// Small tables the decisions index with per-lane values, copied to shared
// memory (constant memory serialises divergent indices).
struct LfTables {
  uint8_t subsampled[22][2][2];
  uint8_t bw_log2[23], bh_log2[23];  // log2 of block width/height in samples (22 = invalid)
  uint8_t txw_log2[19], txh_log2[19];
  uint8_t txw[19], txh[19];
};

__device__ __forceinline__ void load_lf_tables(LfTables& t) {
  for (int k = threadIdx.x; k < 22 * 4; k += blockDim.x) (&t.subsampled[0][0][0])[k] = (&c_subsampled_size[0][0][0])[k];
  for (int k = threadIdx.x; k < 23; k += blockDim.x) {
    t.bw_log2[k] = k < 22 ? uint8_t(2 + (31 - __clz(c_n4w[k]))) : 0;
    t.bh_log2[k] = k < 22 ? uint8_t(2 + (31 - __clz(c_n4h[k]))) : 0;
  }
  for (int k = threadIdx.x; k < 19; k += blockDim.x) {
    t.txw[k] = c_tx_w[k];
    t.txh[k] = c_tx_h[k];
    t.txw_log2[k] = uint8_t(31 - __clz(c_tx_w[k]));
    t.txh_log2[k] = uint8_t(31 - __clz(c_tx_h[k]));
  }
}

// edge_loop_filter's decisions (postfilter.rs:107-172) for the 4x4 at plane
// position (cx, cy), both passes: 0 = not filtered, else (size code << 6) |
// lvl with size code 1 = 4, 2 = 8, 3 = 16. Block and transform sizes are
// powers of two, so the edge tests are masks. The mode-info word and the
// three transform sizes (this 4x4, its left and upper neighbours) are all
// loaded before any is used.
__device__ __forceinline__ void lf_decide2(const FrameDesc& f, const LfTables& tb, int plane, int cx, int cy,
                                           int& dv, int& dh) {
  dv = dh = 0;
  const int sx = plane_ssx(f, plane), sy = plane_ssy(f, plane);
  int row = cy << sy, col = cx << sx;
  const int x = col * 4, y = row * 4;
  if (x >= f.fw || y >= f.fh) return;
  const int xp = x >> sx, yp = y >> sy;
  row |= sy;
  col |= sx;
  const int ms = f.mi_stride;
  const uint8_t* txm = f.tx[plane];
  const bool has_v = x != 0, has_h = y != 0;
  const uint2 raw = *reinterpret_cast<const uint2*>(f.mi + int64_t(row) * ms + col);
  const int tx_sz = txm[int64_t(row >> sy) * ms + (col >> sx)];
  const int tx_v = has_v ? txm[int64_t(row >> sy) * ms + ((col - (1 << sx)) >> sx)] : 0;
  const int tx_h = has_h ? txm[int64_t((row - (1 << sy)) >> sy) * ms + (col >> sx)] : 0;
  const int mi_size = int(raw.x & 0xffu);
  const bool skip = (raw.x >> 24) & AV1PF_MI_SKIP;
  const bool is_intra = int(int8_t((raw.x >> 16) & 0xffu)) <= 0;
  if (mi_size >= 22 || tx_sz >= 19 || tx_v >= 19 || tx_h >= 19) {
    atomicOr(&g_error_flags, ERRF_BAD_MAP);
    return;
  }
  const int plane_size = tb.subsampled[mi_size][sx][sy];
  if (plane_size >= 22) {
    atomicOr(&g_error_flags, ERRF_BAD_MAP);
    return;
  }
  const int cap = plane == 0 ? 16 : 8;
  if (has_v) {
    const bool is_block_edge = (xp & ((1 << tb.bw_log2[plane_size]) - 1)) == 0;
    const bool is_tx_edge = (xp & ((1 << tb.txw_log2[tx_sz]) - 1)) == 0;
    if (is_tx_edge && (is_block_edge || !skip || is_intra)) {
      const int size = min(cap, min(int(tb.txw[tx_v]), int(tb.txw[tx_sz])));
      int lvl = lf_level_raw(f, raw, plane, 0);
      if (lvl == 0) lvl = lf_level(f, row, col - (1 << sx), plane, 0);
      if (lvl) dv = ((size >= 16 ? 3 : (size >= 8 ? 2 : 1)) << 6) | lvl;
    }
  }
  if (has_h) {
    const bool is_block_edge = (yp & ((1 << tb.bh_log2[plane_size]) - 1)) == 0;
    const bool is_tx_edge = (yp & ((1 << tb.txh_log2[tx_sz]) - 1)) == 0;
    if (is_tx_edge && (is_block_edge || !skip || is_intra)) {
      const int size = min(cap, min(int(tb.txh[tx_h]), int(tb.txh[tx_sz])));
      int lvl = lf_level_raw(f, raw, plane, 1);
      if (lvl == 0) lvl = lf_level(f, row - (1 << sy), col, plane, 1);
      if (lvl) dh = ((size >= 16 ? 3 : (size >= 8 ? 2 : 1)) << 6) | lvl;
    }
  }
}

// Edge list entry: frame:16 | plane:2 | code:2 | lvl:6 | cx:14 | cy:14.
__device__ __forceinline__ uint64_t pack_edge(int frame, int plane, int dec, int cx, int cy) {
  return uint64_t(frame) | (uint64_t(plane) << 16) | (uint64_t(dec) << 18) | (uint64_t(cx) << 26) |
         (uint64_t(cy) << 40);
}

__device__ __forceinline__ void append_edge(uint64_t* list, uint32_t* count, uint32_t cap, bool active,
                                            uint64_t e) {
  const unsigned mask = __ballot_sync(0xffffffffu, active);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, uint32_t(__popc(mask)));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (active) {
    const uint32_t pos = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
    if (pos < cap)
      list[pos] = e;
    else
      atomicOr(&g_error_flags, ERRF_BAD_ITEM);
  }
}

// Item: tile [x0,x1) x [y0,y1) of plane `plane` (samples). kind bit 0: copy
// in -> cur over the tile; bit 1: decide the tile's 4x4 edges. 256 threads.
__global__ void __launch_bounds__(256, 4) lf_prep_kernel(const FrameDesc* __restrict__ frames,
                                                      const Item* __restrict__ items, int n_items,
                                                      uint64_t* __restrict__ list_v, uint64_t* __restrict__ list_h,
                                                      uint32_t* __restrict__ counts, uint32_t cap) {
  __shared__ LfTables tb;
  load_lf_tables(tb);
  __syncthreads();
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int plane = item.plane;
    if (item.kind & 1) {
      // Copy the tile, 16 bytes at a time (rows are 16-byte aligned).
      const DPlane src = f.in[plane], dst = f.cur[plane];
      const int sb = f.sb;
      const int x0 = item.x0, x1 = min(int(item.x1), src.w);
      const int y0 = item.y0, y1 = min(int(item.y1), src.h);
      const int bx0 = x0 * sb, bx1 = x1 * sb;  // byte columns (a tile row is at most 128 bytes)
      const int nvec = (bx1 - bx0) >> 4;
      const int rows = y1 - y0;
      // 64 rows x 8 chunk slots = 2 per thread: both loads issue before the stores
      for (int k0 = threadIdx.x; k0 < rows * 8; k0 += 2 * blockDim.x) {
        uint4 q[2];
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const int k = k0 + m * blockDim.x;
          const int r = y0 + (k >> 3), c = bx0 + (k & 7) * 16;
          if (k < rows * 8 && (k & 7) < nvec)
            q[m] = *reinterpret_cast<const uint4*>(src.p + int64_t(r) * src.stride * sb + c);
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const int k = k0 + m * blockDim.x;
          const int r = y0 + (k >> 3), c = bx0 + (k & 7) * 16;
          if (k < rows * 8 && (k & 7) < nvec)
            *reinterpret_cast<uint4*>(dst.p + int64_t(r) * dst.stride * sb + c) = q[m];
        }
      }
      const int tail = (bx1 - bx0) & 15;
      if (tail) {
        for (int k = threadIdx.x; k < rows * 16; k += blockDim.x) {
          const int e = k & 15;
          if (e >= tail) continue;
          const int r = y0 + (k >> 4), c = bx0 + nvec * 16 + e;
          dst.p[int64_t(r) * dst.stride * sb + c] = src.p[int64_t(r) * src.stride * sb + c];
        }
      }
    }
    if (item.kind & 2) {
      const int sx = plane_ssx(f, plane), sy = plane_ssy(f, plane);
      const int gw = f.mi_cols >> sx, gh = f.mi_rows >> sy;  // 4x4 grid of the plane
      const int cx0 = item.x0 >> 2, cy0 = item.y0 >> 2;
      const int tw = (int(item.x1) - int(item.x0) + 3) >> 2;  // <= 16 (64-sample tiles)
      const int th = (int(item.y1) - int(item.y0) + 3) >> 2;
      for (int k = threadIdx.x; k < th * 16; k += blockDim.x) {
        const int cx = cx0 + (k & 15), cy = cy0 + (k >> 4);
        const bool in = (k & 15) < tw && cx < gw && cy < gh;
        int dv = 0, dh = 0;
        if (in) lf_decide2(f, tb, plane, cx, cy, dv, dh);
        append_edge(list_v, &counts[0], cap, dv != 0, pack_edge(item.frame, plane, dv, cx, cy));
        append_edge(list_h, &counts[1], cap, dh != 0, pack_edge(item.frame, plane, dh, cx, cy));
      }
    }
  }
}

// The wide filter of 7.14.6.4 with N taps each side (inner weight-2 taps
// |j| <= N2), output positions 7-N .. 7+N-1, all indices compile-time.
template <int N, int N2, int LOG2>
__device__ __forceinline__ void lf_wide(int32_t v[14]) {
  int32_t o[14];
#pragma unroll
  for (int k = 0; k < 14; k++) o[k] = v[k];
#pragma unroll
  for (int i = -N; i < N; i++) {
    int32_t acc = 0;
#pragma unroll
    for (int j = -N; j <= N; j++) {
      const int pp = (i + j) < -(N + 1) ? -(N + 1) : ((i + j) > N ? N : (i + j));
      acc += o[7 + pp] * ((j <= N2 && j >= -N2) ? 2 : 1);
    }
    v[7 + i] = (acc + (1 << (LOG2 - 1))) >> LOG2;
  }
}

// One lane of one edge (the one-sample process of 7.14.6, as lf.rs:218-306
// states it; lf.rs:58-211 computes the same per lane). v[7] is q0. Returns the
// first and one-past-last index of the samples the chosen filter changes
// (lo == hi: none).
__device__ __forceinline__ void lf_filter_one(int32_t v[14], int filter_size, bool chroma, int bd, int limit,
                                              int blimit, int thresh, int& lo, int& hi) {
  lo = hi = 0;
  const int sh = bd - 8;
  const int32_t q0 = v[7], q1 = v[8], q2 = v[9], q3 = v[10];
  const int32_t p0 = v[6], p1 = v[5], p2 = v[4], p3 = v[3];
  const int32_t thresh_bd = thresh << sh, limit_bd = limit << sh, blimit_bd = blimit << sh;
  const bool hev = abs(p1 - p0) > thresh_bd || abs(q1 - q0) > thresh_bd;
  const int filter_len = filter_size == 4 ? 4 : (chroma ? 6 : (filter_size == 8 ? 8 : 16));
  bool mask = abs(p1 - p0) > limit_bd || abs(q1 - q0) > limit_bd || abs(p0 - q0) * 2 + abs(p1 - q1) / 2 > blimit_bd;
  if (filter_len >= 6) mask = mask || abs(p2 - p1) > limit_bd || abs(q2 - q1) > limit_bd;
  if (filter_len >= 8) mask = mask || abs(p3 - p2) > limit_bd || abs(q3 - q2) > limit_bd;
  if (mask) return;
  const int32_t t = 1 << sh;
  bool flat = false;
  if (filter_size >= 8) {
    bool m = abs(p1 - p0) > t || abs(q1 - q0) > t || abs(p2 - p0) > t || abs(q2 - q0) > t;
    if (filter_len >= 8) m = m || abs(p3 - p0) > t || abs(q3 - q0) > t;
    flat = !m;
  }
  bool flat2 = false;
  if (filter_size >= 16) {
    const bool m = abs(v[0] - p0) > t || abs(v[13] - q0) > t || abs(v[1] - p0) > t || abs(v[12] - q0) > t ||
                   abs(v[2] - p0) > t || abs(v[11] - q0) > t;
    flat2 = !m;
  }
  if (filter_size == 4 || !flat) {
    // narrow filter (7.14.6.3)
    const int32_t clo = -(1 << (bd - 1)), chi = (1 << (bd - 1)) - 1;
    const int32_t off = 0x80 << sh;
    const int32_t ps1 = p1 - off, ps0 = p0 - off, qs0 = q0 - off, qs1 = q1 - off;
    int32_t fl = hev ? clip3(clo, chi, ps1 - qs1) : 0;
    fl = clip3(clo, chi, fl + 3 * (qs0 - ps0));
    const int32_t filter1 = clip3(clo, chi, fl + 4) >> 3;
    const int32_t filter2 = clip3(clo, chi, fl + 3) >> 3;
    v[7] = clip3(clo, chi, qs0 - filter1) + off;
    v[6] = clip3(clo, chi, ps0 + filter2) + off;
    if (!hev) {
      const int32_t fr = (filter1 + 1) >> 1;
      v[8] = clip3(clo, chi, qs1 - fr) + off;
      v[5] = clip3(clo, chi, ps1 + fr) + off;
    }
    lo = 5;
    hi = 9;
    return;
  }
  // wide filters (7.14.6.4)
  if (filter_size == 8 || !flat2) {
    if (chroma) {
      lf_wide<2, 1, 3>(v);
      lo = 5;
      hi = 9;
    } else {
      lf_wide<3, 0, 3>(v);
      lo = 4;
      hi = 10;
    }
  } else {
    lf_wide<6, 1, 4>(v);
    lo = 1;
    hi = 13;
  }
}

__device__ __forceinline__ void lf_limits(int lvl, int sharp, int& limit, int& blimit, int& thresh) {
  // postfilter.rs:248-262
  const int shift = sharp > 4 ? 2 : (sharp > 0 ? 1 : 0);
  limit = sharp > 0 ? clip3(1, 9 - sharp, lvl >> shift) : max(lvl >> shift, 1);
  blimit = 2 * (lvl + 2) + limit;
  thresh = lvl >> 4;
}

// Loads samples s[e+k], k in [k0, k0+n), along the filter direction.
template <int PASS>
__device__ __forceinline__ void lf_load(const DPlane& p, int sb, int e, int lanepos, int k0, int n, int32_t* out) {
  if (PASS == 0) {
    // row `lanepos`, columns e+k0 .. (k0 is -4 or -8: 4-sample aligned)
    const uint8_t* row = p.p + int64_t(lanepos) * p.stride * sb;
    if (sb == 2) {
      const uint2* q = reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(row) + e + k0);
      for (int g = 0; g < n / 4; g++) {
        const uint2 w = q[g];
        out[4 * g + 0] = int32_t(w.x & 0xffffu);
        out[4 * g + 1] = int32_t(w.x >> 16);
        out[4 * g + 2] = int32_t(w.y & 0xffffu);
        out[4 * g + 3] = int32_t(w.y >> 16);
      }
    } else {
      const uint32_t* q = reinterpret_cast<const uint32_t*>(row + e + k0);
      for (int g = 0; g < n / 4; g++) {
        const uint32_t w = q[g];
        out[4 * g + 0] = int32_t(w & 0xffu);
        out[4 * g + 1] = int32_t((w >> 8) & 0xffu);
        out[4 * g + 2] = int32_t((w >> 16) & 0xffu);
        out[4 * g + 3] = int32_t(w >> 24);
      }
    }
  } else {
    for (int k = 0; k < n; k++) out[k] = ld_sample(p, sb, lanepos, e + k0 + k);
  }
}

template <int PASS>
__global__ void __launch_bounds__(256, 4) lf_edge_kernel(const FrameDesc* __restrict__ frames,
                                                      const uint64_t* __restrict__ list,
                                                      const uint32_t* __restrict__ count_ptr, uint32_t cap) {
  const uint32_t n = min(*count_ptr, cap) * 4u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t e = list[i >> 2];
    const int lane = int(i & 3u);
    const int frame = int(e & 0xffffu);
    const int plane = int((e >> 16) & 3u);
    const int code = int((e >> 24) & 3u);
    const int lvl = int((e >> 18) & 63u);
    const int cx = int((e >> 26) & 0x3fffu), cy = int((e >> 40) & 0x3fffu);
    const FrameDesc& f = frames[frame];
    const int sb = f.sb, bd = f.bd;
    const DPlane p = f.cur[plane];
    const int filter_size = code == 3 ? 16 : (code == 2 ? 8 : 4);
    int limit, blimit, thresh;
    lf_limits(lvl, f.sharpness, limit, blimit, thresh);
    const int epos = PASS == 0 ? cx * 4 : cy * 4;              // q0 along the filter direction
    const int lanepos = PASS == 0 ? cy * 4 + lane : cx * 4 + lane;  // row (pass 0) / column (pass 1)
    // A conformant map never puts a wide edge this close to the plane start
    // (the transform before it is at least as wide as the filter).
    if (epos < (filter_size >= 16 ? 8 : 4)) {
      atomicOr(&g_error_flags, ERRF_BAD_MAP);
      continue;
    }
    int32_t v[14];
#pragma unroll
    for (int k = 0; k < 14; k++) v[k] = 0;
    if (filter_size >= 16) {
      int32_t tmp[16];
      lf_load<PASS>(p, sb, epos, lanepos, -8, 16, tmp);
#pragma unroll
      for (int k = 0; k < 14; k++) v[k] = tmp[k + 1];
    } else {
      int32_t tmp[8];
      lf_load<PASS>(p, sb, epos, lanepos, -4, 8, tmp);
#pragma unroll
      for (int k = 0; k < 8; k++) v[k + 3] = tmp[k];
    }
    int lo, hi;
    lf_filter_one(v, filter_size, plane != 0, bd, limit, blimit, thresh, lo, hi);
#pragma unroll
    for (int k = 1; k < 13; k++) {
      if (k < lo || k >= hi) continue;
      const int pos = epos + k - 7;
      if (PASS == 0)
        st_sample(p, sb, pos, lanepos, v[k]);
      else
        st_sample(p, sb, lanepos, pos, v[k]);
    }
  }
}

// dsp::lf::filter (lf.rs:25) on independent edges: one thread per lane.
__global__ void dsp_lf_kernel(int32_t* __restrict__ edges, const av1pf_lf_edge_params* __restrict__ prm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * 4) return;
  const int e = i >> 2, lane = i & 3;
  const av1pf_lf_edge_params p = prm[e];
  int32_t v[14];
#pragma unroll
  for (int k = 0; k < 14; k++) v[k] = edges[int64_t(e) * 56 + k * 4 + lane];
  int lo, hi;
  lf_filter_one(v, p.filter_size, p.chroma != 0, p.bit_depth, p.limit, p.blimit, p.thresh, lo, hi);
#pragma unroll
  for (int k = 0; k < 14; k++)
    if (k >= lo && k < hi) edges[int64_t(e) * 56 + k * 4 + lane] = v[k];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_lf_prep(const FrameDesc* frames, const Item* items, int n_items, uint64_t* list_v, uint64_t* list_h,
                    uint32_t* counts, uint32_t cap, cudaStream_t s) {
  if (n_items <= 0) return;
  const int grid = min(n_items, kItemGrid);
  lf_prep_kernel<<<grid, 256, 0, s>>>(frames, items, n_items, list_v, list_h, counts, cap);
  note_launch();
}

void launch_lf_edges(int pass, const FrameDesc* frames, const uint64_t* list, const uint32_t* count, uint32_t cap,
                     cudaStream_t s) {
  // The edge count is only known on the device: a fixed grid strides over it.
  const int grid = kMaxGrid;
  if (pass == 0)
    lf_edge_kernel<0><<<grid, 256, 0, s>>>(frames, list, count, cap);
  else
    lf_edge_kernel<1><<<grid, 256, 0, s>>>(frames, list, count, cap);
  note_launch();
}

void launch_dsp_lf(int32_t* edges, const av1pf_lf_edge_params* prm, int n, cudaStream_t s) {
  if (n <= 0) return;
  dsp_lf_kernel<<<(n * 4 + 255) / 256, 256, 0, s>>>(edges, prm, n);
  note_launch();
}

}  // namespace av1pf
