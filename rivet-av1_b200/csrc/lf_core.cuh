// lf_core.cuh — loop-filter device functions shared by the loop-filter
// kernels (lf.cu) and the CDEF kernel, which can run the horizontal-edge
// pass on its staged window (cdef.cu).
//
// Reference: rivet-av1 src/decoder/postfilter.rs:107-264 (edge_loop_filter,
// filter_strength) and src/dsp/lf.rs:58-306 (the sample filters).
#pragma once

#include "av1_tables.h"
#include "common.cuh"

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

// Small tables the decisions index with per-lane values (constant memory
// serialises divergent indices), built at compile time into global memory
// and read through the L1, so no CTA sets them up.
struct LfTables {
  uint8_t subsampled[22][2][2];
  uint8_t bw_log2[23], bh_log2[23];  // log2 of block width/height in samples (22 = invalid)
  uint8_t txw_log2[19], txh_log2[19];
  uint8_t txw[19], txh[19];
};

constexpr int lf_ilog2(int v) {
  int r = 0;
  while (v > 1) {
    v >>= 1;
    r++;
  }
  return r;
}

constexpr LfTables make_lf_tables() {
  LfTables t{};
  constexpr uint8_t sub[22][2][2] = AV1T_SUBSAMPLED_SIZE;
  constexpr uint8_t n4w[22] = AV1T_NUM_4X4_BLOCKS_WIDE;
  constexpr uint8_t n4h[22] = AV1T_NUM_4X4_BLOCKS_HIGH;
  constexpr uint8_t txw[19] = AV1T_TX_WIDTH;
  constexpr uint8_t txh[19] = AV1T_TX_HEIGHT;
  for (int i = 0; i < 22; i++)
    for (int j = 0; j < 2; j++)
      for (int k = 0; k < 2; k++) t.subsampled[i][j][k] = sub[i][j][k];
  for (int k = 0; k < 23; k++) {
    t.bw_log2[k] = uint8_t(k < 22 ? 2 + lf_ilog2(n4w[k]) : 0);
    t.bh_log2[k] = uint8_t(k < 22 ? 2 + lf_ilog2(n4h[k]) : 0);
  }
  for (int k = 0; k < 19; k++) {
    t.txw[k] = txw[k];
    t.txh[k] = txh[k];
    t.txw_log2[k] = uint8_t(lf_ilog2(txw[k]));
    t.txh_log2[k] = uint8_t(lf_ilog2(txh[k]));
  }
  return t;
}

extern __device__ const LfTables g_lf_tables;  // lf.cu

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

// The wide filter of 7.14.6.4 with N taps each side (inner weight-2 taps
// |j| <= N2), output positions 7-N .. 7+N-1, all indices compile-time. Each
// output's tap sum is the previous one's with the tap that leaves the
// window taken out and the one that enters added (taps past the ends repeat
// the end samples), so an output costs four adds instead of 2N + 1.
template <int N, int N2, int LOG2>
__device__ __forceinline__ void lf_wide(int32_t v[14]) {
  int32_t o[14];
#pragma unroll
  for (int k = 0; k < 14; k++) o[k] = v[k];
  // the sample at offset k from q0, with the clamp to the filter's ends
  auto at = [&](int k) { return o[7 + (k < -(N + 1) ? -(N + 1) : (k > N ? N : k))]; };
  int32_t all = 0, inner = 0;  // the window sums of the first output (i = -N)
#pragma unroll
  for (int j = -N; j <= N; j++) all += at(-N + j);
#pragma unroll
  for (int j = -N2; j <= N2; j++) inner += at(-N + j);
#pragma unroll
  for (int i = -N; i < N; i++) {
    v[7 + i] = (all + inner + (1 << (LOG2 - 1))) >> LOG2;
    all += at(i + N + 1) - at(i - N);
    inner += at(i + N2 + 1) - at(i - N2);
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
  bool mask = abs(p1 - p0) > limit_bd || abs(q1 - q0) > limit_bd || abs(p0 - q0) * 2 + (abs(p1 - q1) >> 1) > blimit_bd;
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

// One edge lane filtered in shared memory: q0p points at q0, `step` is the
// distance between successive samples across the edge (1 for a vertical
// edge, the row stride for a horizontal one). Only the samples the chosen
// filter changes are written.
template <typename T>
__device__ __forceinline__ void lf_filter_smem(T* q0p, int step, int code, bool chroma, int bd, int lvl, int sharp) {
  const int filter_size = code == 3 ? 16 : (code == 2 ? 8 : 4);
  int limit, blimit, thresh;
  lf_limits(lvl, sharp, limit, blimit, thresh);
  int32_t v[14];
#pragma unroll
  for (int k = 0; k < 14; k++) v[k] = 0;
  if (filter_size >= 16) {
#pragma unroll
    for (int k = 0; k < 14; k++) v[k] = q0p[(k - 7) * step];
  } else {
#pragma unroll
    for (int k = 3; k < 11; k++) v[k] = q0p[(k - 7) * step];
  }
  int lo, hi;
  lf_filter_one(v, filter_size, chroma, bd, limit, blimit, thresh, lo, hi);
#pragma unroll
  for (int k = 1; k < 13; k++)
    if (k >= lo && k < hi) q0p[(k - 7) * step] = T(v[k]);
}

}  // namespace av1pf
