/*
 * oracle.cpp — CPU restatement of rivet-av1's frame post-filter chain.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline. Every function names the reference function and file:line it
 * restates; the arithmetic, loop order and threading (parallel_map bands)
 * follow the reference. Samples are kept as u16, as the reference does
 * (src/decoder/state.rs:9-11).
 *
 * Parity: pinned by the reference's known-answer tests for this path
 * (lf.rs:213-353, cdef.rs:244-312, restated below); at the frame boundary the
 * reference's own output is unpinned (no Rust toolchain, no plane dumps).
 */
#include "oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "av1_tables.h"

namespace {

// ---------------------------------------------------------------------------
// Specification tables (av1_tables.h is extracted from the reference's
// src/tables.rs) and constants (src/consts.rs).
// ---------------------------------------------------------------------------
const int8_t CDEF_DIRECTIONS AV1T_CDEF_DIRECTIONS_DIMS = AV1T_CDEF_DIRECTIONS;
const int8_t CDEF_PRI_TAPS AV1T_CDEF_PRI_TAPS_DIMS = AV1T_CDEF_PRI_TAPS;
const int8_t CDEF_SEC_TAPS AV1T_CDEF_SEC_TAPS_DIMS = AV1T_CDEF_SEC_TAPS;
const uint8_t CDEF_UV_DIR AV1T_CDEF_UV_DIR_DIMS = AV1T_CDEF_UV_DIR;
const int32_t DIV_TABLE AV1T_DIV_TABLE_DIMS = AV1T_DIV_TABLE;
const int16_t GAUSSIAN_SEQUENCE AV1T_GAUSSIAN_SEQUENCE_DIMS = AV1T_GAUSSIAN_SEQUENCE;
const int32_t SGR_PARAMS AV1T_SGR_PARAMS_DIMS = AV1T_SGR_PARAMS;
const uint8_t SUBSAMPLED_SIZE AV1T_SUBSAMPLED_SIZE_DIMS = AV1T_SUBSAMPLED_SIZE;
const uint8_t TX_WIDTH AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH;
const uint8_t TX_HEIGHT AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT;
const int16_t UPSCALE_FILTER AV1T_UPSCALE_FILTER_DIMS = AV1T_UPSCALE_FILTER;
const uint8_t NUM_4X4_BLOCKS_WIDE AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE;
const uint8_t NUM_4X4_BLOCKS_HIGH AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH;

constexpr int SEG_LVL_ALT_LF_Y_V = 1;     // consts.rs:11
constexpr int MAX_LOOP_FILTER = 63;       // consts.rs:16
constexpr size_t MI_SIZE = 4;             // consts.rs:18
constexpr size_t MI_SIZE_LOG2 = 2;        // consts.rs:19
constexpr int INTRA_FRAME = 0;            // consts.rs:107
constexpr size_t NEARESTMV = 14;          // consts.rs:226
constexpr size_t GLOBALMV = 16;           // consts.rs:228
constexpr size_t GLOBAL_GLOBALMV = 24;    // consts.rs:236
constexpr int SUPERRES_FILTER_TAPS = 8;   // consts.rs:28
constexpr int SUPERRES_FILTER_OFFSET = 3; // consts.rs:29
constexpr unsigned SUPERRES_SCALE_BITS = 14;
constexpr int64_t SUPERRES_SCALE_MASK = (1 << 14) - 1;
constexpr unsigned SUPERRES_EXTRA_BITS = 8;
constexpr int FILTER_BITS = 7;            // consts.rs:59
constexpr int SGRPROJ_PRJ_BITS = 7;       // consts.rs:87
constexpr int SGRPROJ_RST_BITS = 4;
constexpr int SGRPROJ_MTABLE_BITS = 20;
constexpr int SGRPROJ_RECIP_BITS = 12;
constexpr int SGRPROJ_SGR_BITS = 8;
constexpr uint8_t RESTORE_NONE = 0, RESTORE_WIENER = 1, RESTORE_SGRPROJ = 2;
constexpr uint32_t MC_IDENTITY = 0;

// consts.rs:328-368, bits.rs:112-114
inline int32_t round2(int32_t x, unsigned n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }
inline int64_t round2_64(int64_t x, unsigned n) {
  return n == 0 ? x : (x + (int64_t(1) << (n - 1))) >> n;
}
inline int32_t clip3(int32_t lo, int32_t hi, int32_t x) { return x < lo ? lo : (x > hi ? hi : x); }
inline uint32_t floor_log2(uint32_t x) { return 31u - uint32_t(__builtin_clz(x)); }
inline size_t block_width(size_t b) { return 4 * NUM_4X4_BLOCKS_WIDE[b]; }
inline size_t block_height(size_t b) { return 4 * NUM_4X4_BLOCKS_HIGH[b]; }
inline int32_t iclamp(int32_t v, int32_t lo, int32_t hi) { return std::max(lo, std::min(hi, v)); }

// ---------------------------------------------------------------------------
// State (decoder/state.rs:9-75, decoder/mod.rs:31-80, header.rs:14-177)
// ---------------------------------------------------------------------------
struct PlaneBuf {  // state.rs:11-42
  std::vector<uint16_t> data;
  size_t stride = 0, w = 0, h = 0;
  PlaneBuf() = default;
  PlaneBuf(size_t w_, size_t h_, uint16_t fill) : data(w_ * h_, fill), stride(w_), w(w_), h(h_) {}
  uint16_t get(size_t x, size_t y) const { return data[y * stride + x]; }
  void set(size_t x, size_t y, uint16_t v) { data[y * stride + x] = v; }
  const uint16_t* row(size_t y) const { return &data[y * stride]; }
};
struct FrameBuf {
  std::vector<PlaneBuf> planes;
};

struct Mi {  // state.rs:55-75 (the fields the filters read)
  uint8_t mi_size = 0, y_mode = 0;
  int8_t ref_frame0 = 0;
  bool skip = false;
  uint8_t segment_id = 0;
  int8_t delta_lf[4] = {0, 0, 0, 0};
};

struct LrPlane {  // decoder/mod.rs:31-41
  size_t unit_rows = 0, unit_cols = 0;
  std::vector<uint8_t> lr_type;
  std::vector<std::array<std::array<int32_t, 3>, 2>> wiener;
  std::vector<uint8_t> sgr_set;
  std::vector<std::array<int32_t, 2>> sgr_xqd;
};

struct Hdr {  // FrameHeader filter fields, header.rs:89-177
  int32_t frame_width = 0, frame_height = 0, upscaled_width = 0;
  int32_t loop_filter_level[4] = {};
  int32_t loop_filter_sharpness = 0;
  bool loop_filter_delta_enabled = false;
  int32_t loop_filter_ref_deltas[8] = {};
  int32_t loop_filter_mode_deltas[2] = {};
  bool delta_lf_multi = false;
  bool segmentation_enabled = false;
  bool feature_enabled[8][8] = {};
  int32_t feature_data[8][8] = {};
  bool cdef_on = false;  // !coded_lossless && !allow_intrabc && enable_cdef
  int32_t cdef_damping = 3;
  int32_t cdef_y_pri_strength[8] = {}, cdef_y_sec_strength[8] = {};
  int32_t cdef_uv_pri_strength[8] = {}, cdef_uv_sec_strength[8] = {};
  bool use_superres = false;
  bool uses_lr = false;
  uint8_t frame_restoration_type[3] = {};
  size_t loop_restoration_size[3] = {};
};

struct FrameCtx {  // decoder/mod.rs:44-80
  Hdr hdr;
  uint32_t bit_depth = 8;
  size_t ssx = 0, ssy = 0, num_planes = 1;
  size_t mi_rows = 0, mi_cols = 0, ms = 0;
  std::vector<Mi> mi;
  std::vector<uint8_t> lf_tx_sizes[3];
  std::vector<int8_t> cdef_idx;
  size_t cdef_stride = 0;
  LrPlane lr[3];
  FrameBuf cur;

  std::pair<size_t, size_t> plane_ss(size_t plane) const {  // predict.rs:1169-1175
    return plane == 0 ? std::make_pair(size_t(0), size_t(0)) : std::make_pair(ssx, ssy);
  }
  size_t plane_residual_size(size_t subsize, size_t plane) const {  // decoder/mod.rs:249-252
    auto ss = plane_ss(plane);
    return SUBSAMPLED_SIZE[subsize][ss.first][ss.second];
  }
  struct Rounding {
    unsigned round0, round1;
  };
  Rounding rounding_variables(bool is_compound) const {  // predict.rs:1152-1167
    unsigned round0 = 3, round1 = is_compound ? 7 : 11;
    if (bit_depth == 12) round0 += 2;
    if (bit_depth == 12 && !is_compound) round1 -= 2;
    return {round0, round1};
  }
};

// ---------------------------------------------------------------------------
// Threads: parallel_map (decoder/mod.rs:1140-1167)
// ---------------------------------------------------------------------------
size_t resolve_threads(int threads) {
  if (threads > 0) return size_t(threads);
  unsigned n = std::thread::hardware_concurrency();
  return n ? n : 1;
}

template <class F>
void parallel_map(size_t n, size_t threads, const F& job) {
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (;;) {
      size_t i = next.fetch_add(1, std::memory_order_relaxed);
      if (i >= n) break;
      job(i);
    }
  };
  std::vector<std::thread> ts;
  for (size_t t = 1; t < std::min(threads, n); t++) ts.emplace_back(work);
  work();
  for (auto& t : ts) t.join();
}

template <class F>
void run_bands(size_t n, size_t threads, const F& job) {
  if (threads > 1) {
    parallel_map(n, threads, job);
  } else {
    for (size_t i = 0; i < n; i++) job(i);
  }
}

// SharedPlane (postfilter.rs:15-61): raw access under a disjoint-write contract.
struct SharedPlane {
  uint16_t* ptr;
  size_t len, stride;
  explicit SharedPlane(PlaneBuf& p) : ptr(p.data.data()), len(p.data.size()), stride(p.stride) {}
  uint16_t get(size_t i) const { return ptr[i]; }
  void set(size_t i, uint16_t v) const { ptr[i] = v; }
  void write_row(size_t x0, size_t y, const uint16_t* src, size_t n) const {
    std::memcpy(ptr + y * stride + x0, src, n * sizeof(uint16_t));
  }
};

// ---------------------------------------------------------------------------
// dsp::lf (lf.rs)
// ---------------------------------------------------------------------------
struct LfParams {  // lf.rs:14-21
  int32_t limit, blimit, thresh;
  size_t filter_size;
  bool chroma;
  uint32_t bit_depth;
};
using Edge = int32_t[14][4];  // lf.rs:10

// lf.rs:58-211 `filter_lanes`
void filter_lanes(Edge& v, const LfParams& p) {
  const uint32_t sh = p.bit_depth - 8;
  int32_t q0[4], q1[4], q2[4], q3[4], p0[4], p1[4], p2[4], p3[4];
  for (int l = 0; l < 4; l++) {
    q0[l] = v[7][l]; q1[l] = v[8][l]; q2[l] = v[9][l]; q3[l] = v[10][l];
    p0[l] = v[6][l]; p1[l] = v[5][l]; p2[l] = v[4][l]; p3[l] = v[3][l];
  }
  const int32_t thresh_bd = p.thresh << sh, limit_bd = p.limit << sh, blimit_bd = p.blimit << sh;
  const int filter_len = p.filter_size == 4 ? 4 : (p.chroma ? 6 : (p.filter_size == 8 ? 8 : 16));
  bool hev[4], skip[4];
  for (int l = 0; l < 4; l++) {
    hev[l] = std::abs(p1[l] - p0[l]) > thresh_bd || std::abs(q1[l] - q0[l]) > thresh_bd;
    int32_t a = std::abs(p0[l] - q0[l]), b = std::abs(p1[l] - q1[l]);
    skip[l] = a * 2 + b / 2 > blimit_bd;
    skip[l] = skip[l] || std::abs(p1[l] - p0[l]) > limit_bd || std::abs(q1[l] - q0[l]) > limit_bd;
    if (filter_len >= 6)
      skip[l] = skip[l] || std::abs(p2[l] - p1[l]) > limit_bd || std::abs(q2[l] - q1[l]) > limit_bd;
    if (filter_len >= 8)
      skip[l] = skip[l] || std::abs(p3[l] - p2[l]) > limit_bd || std::abs(q3[l] - q2[l]) > limit_bd;
  }
  if (skip[0] && skip[1] && skip[2] && skip[3]) return;
  const int32_t t = 1 << sh;
  bool flat[4] = {false, false, false, false};
  if (p.filter_size >= 8) {
    for (int l = 0; l < 4; l++) {
      bool m = std::abs(p1[l] - p0[l]) > t || std::abs(q1[l] - q0[l]) > t ||
               std::abs(p2[l] - p0[l]) > t || std::abs(q2[l] - q0[l]) > t;
      if (filter_len >= 8) m = m || std::abs(p3[l] - p0[l]) > t || std::abs(q3[l] - q0[l]) > t;
      flat[l] = !m;
    }
  }
  bool flat2[4] = {false, false, false, false};
  if (p.filter_size >= 16) {
    for (int l = 0; l < 4; l++) {
      bool m = std::abs(v[0][l] - p0[l]) > t || std::abs(v[13][l] - q0[l]) > t ||
               std::abs(v[1][l] - p0[l]) > t || std::abs(v[12][l] - q0[l]) > t ||
               std::abs(v[2][l] - p0[l]) > t || std::abs(v[11][l] - q0[l]) > t;
      flat2[l] = !m;
    }
  }
  // narrow filter (7.14.6.3), lf.rs:123-149
  const uint32_t bd = p.bit_depth;
  const int32_t lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
  auto c = [&](int32_t x) { return iclamp(x, lo, hi); };
  const int32_t off = 0x80 << sh;
  int32_t n_out[4][4];
  for (int l = 0; l < 4; l++) {
    int32_t ps1 = p1[l] - off, ps0 = p0[l] - off, qs0 = q0[l] - off, qs1 = q1[l] - off;
    int32_t fl = hev[l] ? c(ps1 - qs1) : 0;
    fl = c(fl + 3 * (qs0 - ps0));
    int32_t filter1 = c(fl + 4) >> 3;
    int32_t filter2 = c(fl + 3) >> 3;
    n_out[2][l] = c(qs0 - filter1) + off;
    n_out[1][l] = c(ps0 + filter2) + off;
    if (hev[l]) {
      n_out[0][l] = p1[l];
      n_out[3][l] = q1[l];
    } else {
      int32_t f = (filter1 + 1) >> 1;
      n_out[3][l] = c(qs1 - f) + off;
      n_out[0][l] = c(ps1 + f) + off;
    }
  }
  // wide filters (7.14.6.4), lf.rs:152-178
  auto wide = [&](unsigned log2_size, int32_t out[12][4]) {
    int n = log2_size == 4 ? 6 : (!p.chroma ? 3 : 2);
    int n2 = (log2_size == 3 && !p.chroma) ? 0 : 1;
    for (int i = -n; i < n; i++) {
      int32_t acc[4] = {0, 0, 0, 0};
      for (int j = -n; j <= n; j++) {
        int pp = iclamp(i + j, -(n + 1), n);
        int tap = std::abs(j) <= n2 ? 2 : 1;
        for (int l = 0; l < 4; l++) acc[l] += v[7 + pp][l] * tap;
      }
      int32_t add = 1 << (log2_size - 1);
      for (int l = 0; l < 4; l++) out[i + 6][l] = (acc[l] + add) >> log2_size;
    }
  };
  int32_t w8[12][4] = {}, w16[12][4] = {};
  if (p.filter_size >= 8) wide(3, w8);
  if (p.filter_size >= 16) wide(4, w16);
  const int n8 = p.chroma ? 2 : 3;
  for (int l = 0; l < 4; l++) {
    if (skip[l]) continue;
    if (p.filter_size == 4 || !flat[l]) {
      v[5][l] = n_out[0][l];
      v[6][l] = n_out[1][l];
      v[7][l] = n_out[2][l];
      v[8][l] = n_out[3][l];
    } else if (p.filter_size == 8 || !flat2[l]) {
      for (int i = -n8; i < n8; i++) v[7 + i][l] = w8[i + 6][l];
    } else {
      for (int i = -6; i < 6; i++) v[7 + i][l] = w16[i + 6][l];
    }
  }
}

// lf.rs:218-306: the one-sample process of 7.14.6, as written.
void lf_reference_one(int32_t v[14], const LfParams& p) {
  const uint32_t sh = p.bit_depth - 8;
  const int32_t q0 = v[7], q1 = v[8], q2 = v[9], q3 = v[10];
  const int32_t p0 = v[6], p1 = v[5], p2 = v[4], p3 = v[3];
  const int32_t thresh_bd = p.thresh << sh;
  const bool hev_mask = std::abs(p1 - p0) > thresh_bd || std::abs(q1 - q0) > thresh_bd;
  const int filter_len = p.filter_size == 4 ? 4 : (p.chroma ? 6 : (p.filter_size == 8 ? 8 : 16));
  const int32_t limit_bd = p.limit << sh, blimit_bd = p.blimit << sh;
  bool mask = std::abs(p1 - p0) > limit_bd || std::abs(q1 - q0) > limit_bd ||
              std::abs(p0 - q0) * 2 + std::abs(p1 - q1) / 2 > blimit_bd;
  if (filter_len >= 6) mask = mask || std::abs(p2 - p1) > limit_bd || std::abs(q2 - q1) > limit_bd;
  if (filter_len >= 8) mask = mask || std::abs(p3 - p2) > limit_bd || std::abs(q3 - q2) > limit_bd;
  if (mask) return;
  const int32_t t = 1 << sh;
  bool flat = false;
  if (p.filter_size >= 8) {
    bool m = std::abs(p1 - p0) > t || std::abs(q1 - q0) > t || std::abs(p2 - p0) > t ||
             std::abs(q2 - q0) > t;
    if (filter_len >= 8) m = m || std::abs(p3 - p0) > t || std::abs(q3 - q0) > t;
    flat = !m;
  }
  bool flat2 = false;
  if (p.filter_size >= 16) {
    bool m = std::abs(v[0] - p0) > t || std::abs(v[13] - q0) > t || std::abs(v[1] - p0) > t ||
             std::abs(v[12] - q0) > t || std::abs(v[2] - p0) > t || std::abs(v[11] - q0) > t;
    flat2 = !m;
  }
  if (p.filter_size == 4 || !flat) {
    const uint32_t bd = p.bit_depth;
    auto c = [&](int32_t x) { return iclamp(x, -(1 << (bd - 1)), (1 << (bd - 1)) - 1); };
    const int32_t off = 0x80 << sh;
    int32_t ps1 = p1 - off, ps0 = p0 - off, qs0 = q0 - off, qs1 = q1 - off;
    int32_t fl = hev_mask ? c(ps1 - qs1) : 0;
    fl = c(fl + 3 * (qs0 - ps0));
    int32_t filter1 = c(fl + 4) >> 3;
    int32_t filter2 = c(fl + 3) >> 3;
    v[7] = c(qs0 - filter1) + off;
    v[6] = c(ps0 + filter2) + off;
    if (!hev_mask) {
      int32_t f = (filter1 + 1) >> 1;
      v[8] = c(qs1 - f) + off;
      v[5] = c(ps1 + f) + off;
    }
  } else {
    unsigned log2_size = (p.filter_size == 8 || !flat2) ? 3 : 4;
    int n = log2_size == 4 ? 6 : (!p.chroma ? 3 : 2);
    int n2 = (log2_size == 3 && !p.chroma) ? 0 : 1;
    int32_t orig[14];
    std::memcpy(orig, v, sizeof(orig));
    for (int i = -n; i < n; i++) {
      int32_t tt = 0;
      for (int j = -n; j <= n; j++) {
        int pp = iclamp(i + j, -(n + 1), n);
        int tap = std::abs(j) <= n2 ? 2 : 1;
        tt += orig[7 + pp] * tap;
      }
      v[7 + i] = (tt + (1 << (log2_size - 1))) >> log2_size;
    }
  }
}

// ---------------------------------------------------------------------------
// Loop filter (postfilter.rs:63-264)
// ---------------------------------------------------------------------------
struct Strength {
  int32_t lvl, limit, blimit, thresh;
};

// postfilter.rs:207-264 `filter_strength`
Strength filter_strength(const FrameCtx& f, size_t row, size_t col, size_t plane, size_t pass) {
  const Hdr& h = f.hdr;
  const Mi& m = f.mi[row * f.ms + col];
  size_t segment = m.segment_id;
  int32_t rf = m.ref_frame0;
  size_t mode = m.y_mode;
  size_t mode_type = (mode >= NEARESTMV && mode != GLOBALMV && mode != GLOBAL_GLOBALMV) ? 1 : 0;
  int32_t delta_lf = h.delta_lf_multi ? int32_t(m.delta_lf[plane == 0 ? pass : plane + 1])
                                      : int32_t(m.delta_lf[0]);
  size_t i = plane == 0 ? pass : plane + 1;
  int32_t base_filter_level = clip3(0, MAX_LOOP_FILTER, delta_lf + h.loop_filter_level[i]);
  int32_t lvl_seg = base_filter_level;
  size_t feature = SEG_LVL_ALT_LF_Y_V + i;
  if (h.segmentation_enabled && h.feature_enabled[segment][feature]) {
    lvl_seg = clip3(0, MAX_LOOP_FILTER, h.feature_data[segment][feature] + lvl_seg);
  }
  if (h.loop_filter_delta_enabled) {
    int32_t n_shift = lvl_seg >> 5;
    if (rf == INTRA_FRAME) {
      lvl_seg += h.loop_filter_ref_deltas[INTRA_FRAME] << n_shift;
    } else if (rf > INTRA_FRAME) {
      lvl_seg += (h.loop_filter_ref_deltas[rf] << n_shift) +
                 (h.loop_filter_mode_deltas[mode_type] << n_shift);
    }
    lvl_seg = clip3(0, MAX_LOOP_FILTER, lvl_seg);
  }
  int32_t lvl = lvl_seg;
  int32_t sharp = h.loop_filter_sharpness;
  int32_t shift = sharp > 4 ? 2 : (sharp > 0 ? 1 : 0);
  int32_t limit = sharp > 0 ? clip3(1, 9 - sharp, lvl >> shift) : std::max(lvl >> shift, 1);
  int32_t blimit = 2 * (lvl + 2) + limit;
  int32_t thresh = lvl >> 4;
  return {lvl, limit, blimit, thresh};
}

// postfilter.rs:107-203 `edge_loop_filter`
void edge_loop_filter(const FrameCtx& f, SharedPlane p, size_t plane, size_t pass, size_t row,
                      size_t col) {
  auto ss = f.plane_ss(plane);
  size_t sub_x = ss.first, sub_y = ss.second;
  int dx = pass == 0 ? 1 : 0, dy = pass == 0 ? 0 : 1;
  size_t x = col * MI_SIZE, y = row * MI_SIZE;
  row = row | sub_y;
  col = col | sub_x;
  bool on_screen = !(x >= size_t(f.hdr.frame_width) || y >= size_t(f.hdr.frame_height) ||
                     (pass == 0 && x == 0) || (pass == 1 && y == 0));
  if (!on_screen) return;
  size_t xp = x >> sub_x, yp = y >> sub_y;
  size_t prev_row = row - (size_t(dy) << sub_y);
  size_t prev_col = col - (size_t(dx) << sub_x);
  size_t cols = f.ms;
  const Mi& m = f.mi[row * cols + col];
  size_t mi_size = m.mi_size;
  size_t tx_sz = f.lf_tx_sizes[plane][(row >> sub_y) * cols + (col >> sub_x)];
  size_t plane_size = f.plane_residual_size(mi_size, plane);
  bool skip = m.skip;
  bool is_intra = int32_t(m.ref_frame0) <= INTRA_FRAME;
  size_t prev_tx_sz = f.lf_tx_sizes[plane][(prev_row >> sub_y) * cols + (prev_col >> sub_x)];
  bool is_block_edge = pass == 0 ? (xp % block_width(plane_size) == 0)
                                 : (yp % block_height(plane_size) == 0);
  bool is_tx_edge = pass == 0 ? (xp % TX_WIDTH[tx_sz] == 0) : (yp % TX_HEIGHT[tx_sz] == 0);
  bool apply_filter = is_tx_edge && (is_block_edge || !skip || is_intra);
  if (!apply_filter) return;
  size_t base_size = pass == 0 ? std::min<size_t>(TX_WIDTH[prev_tx_sz], TX_WIDTH[tx_sz])
                               : std::min<size_t>(TX_HEIGHT[prev_tx_sz], TX_HEIGHT[tx_sz]);
  size_t filter_size = plane == 0 ? std::min<size_t>(16, base_size) : std::min<size_t>(8, base_size);
  Strength s = filter_strength(f, row, col, plane, pass);
  if (s.lvl == 0) s = filter_strength(f, prev_row, prev_col, plane, pass);
  if (s.lvl == 0) return;
  ptrdiff_t stride = ptrdiff_t(p.stride);
  ptrdiff_t step = ptrdiff_t(dy) * stride + dx;
  ptrdiff_t along = ptrdiff_t(dx) * stride + dy;
  ptrdiff_t base = ptrdiff_t(yp) * stride + ptrdiff_t(xp);
  ptrdiff_t reach = filter_size >= 16 ? 7 : 4;
  Edge v = {};
  for (ptrdiff_t l = 0; l < 4; l++)
    for (ptrdiff_t k = -reach; k < reach; k++)
      v[7 + k][l] = p.get(size_t(base + l * along + k * step));
  LfParams params{s.limit, s.blimit, s.thresh, filter_size, plane != 0, f.bit_depth};
  filter_lanes(v, params);
  ptrdiff_t span = filter_size >= 16 ? 6 : 3;
  for (ptrdiff_t l = 0; l < 4; l++)
    for (ptrdiff_t k = -span; k < span; k++)
      p.set(size_t(base + l * along + k * step), uint16_t(v[7 + k][l]));
}

// postfilter.rs:67-104 `loop_filter_threads`
void loop_filter_threads(FrameCtx& f, size_t threads) {
  for (size_t plane = 0; plane < f.num_planes; plane++) {
    if (plane == 0 || f.hdr.loop_filter_level[1 + plane] != 0) {
      SharedPlane sp(f.cur.planes[plane]);
      const FrameCtx& fr = f;
      size_t row_step = plane == 0 ? 1 : (size_t(1) << fr.ssy);
      size_t col_step = plane == 0 ? 1 : (size_t(1) << fr.ssx);
      for (size_t pass = 0; pass < 2; pass++) {
        size_t extent = pass == 0 ? fr.mi_rows : fr.mi_cols;
        size_t bands = (extent + 15) / 16;
        auto band = [&](size_t b) {
          size_t r0, r1, c0, c1;
          if (pass == 0) {
            r0 = b * 16; r1 = std::min((b + 1) * 16, fr.mi_rows); c0 = 0; c1 = fr.mi_cols;
          } else {
            r0 = 0; r1 = fr.mi_rows; c0 = b * 16; c1 = std::min((b + 1) * 16, fr.mi_cols);
          }
          for (size_t row = r0; row < r1; row += row_step)
            for (size_t col = c0; col < c1; col += col_step)
              edge_loop_filter(fr, sp, plane, pass, row, col);
        };
        run_bands(bands, threads, band);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// CDEF (postfilter.rs:266-513, dsp/cdef.rs)
// ---------------------------------------------------------------------------
constexpr int32_t NA = INT32_MIN;  // cdef.rs:6
constexpr size_t WS = 12;          // cdef.rs:9

struct Taps {  // cdef.rs:13-25
  int32_t pri_str, sec_str, pri_adj, sec_adj;
  int32_t pri_taps[2], sec_taps[2];
  ptrdiff_t pri_off[2];
  ptrdiff_t sec_off[2][2];
};

// cdef.rs:48-51
inline int32_t constrain(int32_t diff, int32_t threshold, int32_t adj) {
  int32_t mag = std::min(std::abs(diff), std::max(threshold - (std::abs(diff) >> adj), 0));
  return diff < 0 ? -mag : mag;
}

// cdef.rs:54-90 `filter_scalar`
void cdef_filter_scalar(const int32_t* win, size_t w, size_t h, const Taps& t, uint16_t* res) {
  for (size_t i = 0; i < h; i++) {
    for (size_t j = 0; j < w; j++) {
      ptrdiff_t ci = ptrdiff_t((i + 2) * WS + j + 2);
      int32_t x = win[ci];
      int32_t sum = 0, mx = x, mn = x;
      for (int k = 0; k < 2; k++) {
        for (int sign : {-1, 1}) {
          int32_t pv = win[ci + sign * t.pri_off[k]];
          if (pv != NA) {
            sum += t.pri_taps[k] * constrain(pv - x, t.pri_str, t.pri_adj);
            mx = std::max(mx, pv);
            mn = std::min(mn, pv);
          }
          for (int so = 0; so < 2; so++) {
            int32_t s = win[ci + sign * t.sec_off[k][so]];
            if (s != NA) {
              sum += t.sec_taps[k] * constrain(s - x, t.sec_str, t.sec_adj);
              mx = std::max(mx, s);
              mn = std::min(mn, s);
            }
          }
        }
      }
      int32_t v = x + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
      res[i * w + j] = uint16_t(iclamp(v, mn, mx));
    }
  }
}

// postfilter.rs:345-401 `cdef_direction`
std::pair<size_t, int32_t> cdef_direction(const FrameCtx& f, size_t r, size_t c) {
  int32_t cost[8] = {};
  int32_t partial[8][15] = {};
  size_t x0 = c << MI_SIZE_LOG2, y0 = r << MI_SIZE_LOG2;
  const PlaneBuf& p = f.cur.planes[0];
  uint32_t sh = f.bit_depth - 8;
  for (size_t i = 0; i < 8; i++) {
    for (size_t j = 0; j < 8; j++) {
      int32_t x = (int32_t(p.get(x0 + j, y0 + i)) >> sh) - 128;
      partial[0][i + j] += x;
      partial[1][i + j / 2] += x;
      partial[2][i] += x;
      partial[3][3 + i - j / 2] += x;
      partial[4][7 + i - j] += x;
      partial[5][3 - i / 2 + j] += x;
      partial[6][j] += x;
      partial[7][i / 2 + j] += x;
    }
  }
  for (size_t i = 0; i < 8; i++) {
    cost[2] += partial[2][i] * partial[2][i];
    cost[6] += partial[6][i] * partial[6][i];
  }
  cost[2] *= DIV_TABLE[8];
  cost[6] *= DIV_TABLE[8];
  for (size_t i = 0; i < 7; i++) {
    cost[0] += (partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) *
               DIV_TABLE[i + 1];
    cost[4] += (partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) *
               DIV_TABLE[i + 1];
  }
  cost[0] += partial[0][7] * partial[0][7] * DIV_TABLE[8];
  cost[4] += partial[4][7] * partial[4][7] * DIV_TABLE[8];
  for (size_t i = 1; i < 8; i += 2) {
    for (size_t j = 0; j < 5; j++) cost[i] += partial[i][3 + j] * partial[i][3 + j];
    cost[i] *= DIV_TABLE[8];
    for (size_t j = 0; j < 3; j++)
      cost[i] += (partial[i][j] * partial[i][j] + partial[i][10 - j] * partial[i][10 - j]) *
                 DIV_TABLE[2 * j + 2];
  }
  int32_t best_cost = 0;
  size_t y_dir = 0;
  for (size_t i = 0; i < 8; i++) {
    if (cost[i] > best_cost) {
      best_cost = cost[i];
      y_dir = i;
    }
  }
  int32_t var = (best_cost - cost[(y_dir + 4) & 7]) >> 10;
  return {y_dir, var};
}

// postfilter.rs:449-513 `cdef_filter_block`
void cdef_filter_block(const PlaneBuf& src, size_t x0, size_t y0, size_t w, size_t h, size_t xlim,
                       size_t ylim, int32_t pri_str, int32_t sec_str, int32_t damping, size_t dir,
                       uint32_t coeff_shift, uint16_t* res) {
  const size_t B = 2;
  int32_t win[WS * WS];
  for (auto& v : win) v = NA;
  bool inside_x = x0 >= B && x0 + w + B <= xlim;
  for (size_t i = 0; i < h + 2 * B; i++) {
    ptrdiff_t y = ptrdiff_t(y0) + ptrdiff_t(i) - ptrdiff_t(B);
    if (y < 0 || size_t(y) >= ylim) continue;
    const uint16_t* row = &src.data[size_t(y) * src.stride];
    int32_t* out = &win[i * WS];
    if (inside_x) {
      for (size_t j = 0; j < w + 2 * B; j++) out[j] = row[x0 - B + j];
    } else {
      for (size_t j = 0; j < w + 2 * B; j++) {
        ptrdiff_t x = ptrdiff_t(x0) + ptrdiff_t(j) - ptrdiff_t(B);
        if (x >= 0 && size_t(x) < xlim) out[j] = row[x];
      }
    }
  }
  auto adj = [&](int32_t s) {
    return s != 0 ? std::max(damping - int32_t(floor_log2(uint32_t(s))), 0) : 0;
  };
  auto off = [&](size_t d, size_t k) -> ptrdiff_t {
    return ptrdiff_t(CDEF_DIRECTIONS[d][k][0]) * ptrdiff_t(WS) + ptrdiff_t(CDEF_DIRECTIONS[d][k][1]);
  };
  size_t d_lo = (dir + 6) & 7, d_hi = (dir + 2) & 7;
  size_t tsel = size_t((pri_str >> coeff_shift) & 1);
  Taps t;
  t.pri_str = pri_str;
  t.sec_str = sec_str;
  t.pri_adj = adj(pri_str);
  t.sec_adj = adj(sec_str);
  t.pri_taps[0] = CDEF_PRI_TAPS[tsel][0];
  t.pri_taps[1] = CDEF_PRI_TAPS[tsel][1];
  t.sec_taps[0] = CDEF_SEC_TAPS[tsel][0];
  t.sec_taps[1] = CDEF_SEC_TAPS[tsel][1];
  t.pri_off[0] = off(dir, 0);
  t.pri_off[1] = off(dir, 1);
  t.sec_off[0][0] = off(d_lo, 0);
  t.sec_off[0][1] = off(d_hi, 0);
  t.sec_off[1][0] = off(d_lo, 1);
  t.sec_off[1][1] = off(d_hi, 1);
  cdef_filter_scalar(win, w, h, t, res);
}

// postfilter.rs:405-442 `cdef_filter`
void cdef_filter(const FrameCtx& f, const std::vector<SharedPlane>& out, size_t plane, size_t r,
                 size_t c, int32_t pri_str, int32_t sec_str, int32_t damping, size_t dir) {
  auto ss = f.plane_ss(plane);
  size_t x0 = (c * MI_SIZE) >> ss.first, y0 = (r * MI_SIZE) >> ss.second;
  size_t w = 8 >> ss.first, h = 8 >> ss.second;
  size_t xlim = (f.mi_cols * MI_SIZE) >> ss.first, ylim = (f.mi_rows * MI_SIZE) >> ss.second;
  uint16_t res[64] = {};
  cdef_filter_block(f.cur.planes[plane], x0, y0, w, h, xlim, ylim, pri_str, sec_str, damping, dir,
                    f.bit_depth - 8, res);
  for (size_t i = 0; i < h; i++) out[plane].write_row(x0, y0 + i, &res[i * w], w);
}

// postfilter.rs:304-342 `cdef_block`
void cdef_block(const FrameCtx& f, const std::vector<SharedPlane>& out, size_t r, size_t c,
                size_t idx) {
  size_t cols = f.ms;
  auto sk = [&](size_t rr, size_t cc) { return f.mi[rr * cols + cc].skip; };
  bool skip = sk(r, c) && sk(r + 1, c) && sk(r, c + 1) && sk(r + 1, c + 1);
  if (skip) return;
  uint32_t coeff_shift = f.bit_depth - 8;
  auto dv = cdef_direction(f, r, c);
  size_t y_dir = dv.first;
  int32_t var = dv.second;
  const Hdr& h = f.hdr;
  int32_t pri_str = h.cdef_y_pri_strength[idx] << coeff_shift;
  int32_t sec_str = h.cdef_y_sec_strength[idx] << coeff_shift;
  size_t dir = pri_str == 0 ? 0 : y_dir;
  int32_t var_str = (var >> 6) != 0 ? std::min(int32_t(floor_log2(uint32_t(var >> 6))), 12) : 0;
  pri_str = var != 0 ? (pri_str * (4 + var_str) + 8) >> 4 : 0;
  int32_t damping = h.cdef_damping + int32_t(coeff_shift);
  cdef_filter(f, out, 0, r, c, pri_str, sec_str, damping, dir);
  if (f.num_planes == 1) return;
  pri_str = h.cdef_uv_pri_strength[idx] << coeff_shift;
  sec_str = h.cdef_uv_sec_strength[idx] << coeff_shift;
  dir = pri_str == 0 ? 0 : CDEF_UV_DIR[f.ssx][f.ssy][y_dir];
  damping = h.cdef_damping + int32_t(coeff_shift) - 1;
  cdef_filter(f, out, 1, r, c, pri_str, sec_str, damping, dir);
  cdef_filter(f, out, 2, r, c, pri_str, sec_str, damping, dir);
}

// postfilter.rs:273-301 `cdef`
FrameBuf cdef(const FrameCtx& f, size_t threads) {
  FrameBuf out = f.cur;
  if (!f.hdr.cdef_on) return out;
  std::vector<SharedPlane> planes;
  for (auto& p : out.planes) planes.emplace_back(p);
  auto band = [&](size_t b) {
    for (size_t r = b * 16; r < std::min((b + 1) * 16, f.mi_rows); r += 2) {
      for (size_t c = 0; c < f.mi_cols; c += 2) {
        int8_t idx = f.cdef_idx[(r >> 4) * f.cdef_stride + (c >> 4)];
        if (idx >= 0) cdef_block(f, planes, r, c, size_t(idx));
      }
    }
  };
  run_bands((f.mi_rows + 15) / 16, threads, band);
  return out;
}

// ---------------------------------------------------------------------------
// Super-resolution (postfilter.rs:515-566)
// ---------------------------------------------------------------------------
bool upscale(const FrameCtx& f, const FrameBuf& input, FrameBuf& out) {
  if (!f.hdr.use_superres) return false;
  int32_t maxv = (1 << f.bit_depth) - 1;
  out.planes.clear();
  for (size_t plane = 0; plane < f.num_planes; plane++) {
    auto ss = f.plane_ss(plane);
    int64_t downscaled_w = round2(f.hdr.frame_width, unsigned(ss.first));
    int64_t upscaled_w = round2(f.hdr.upscaled_width, unsigned(ss.first));
    size_t plane_h = size_t(round2(f.hdr.frame_height, unsigned(ss.second)));
    int64_t step_x = ((downscaled_w << SUPERRES_SCALE_BITS) + upscaled_w / 2) / upscaled_w;
    int64_t err = upscaled_w * step_x - (downscaled_w << SUPERRES_SCALE_BITS);
    int64_t initial_subpel_x =
        (-((upscaled_w - downscaled_w) << (SUPERRES_SCALE_BITS - 1)) + upscaled_w / 2) / upscaled_w +
        (1 << (SUPERRES_EXTRA_BITS - 1)) - err / 2;
    initial_subpel_x &= SUPERRES_SCALE_MASK;
    int64_t mi_w = int64_t(f.mi_cols >> ss.first);
    int64_t max_x = mi_w * int64_t(MI_SIZE) - 1;
    const PlaneBuf& src = input.planes[plane];
    PlaneBuf dst(size_t(upscaled_w) + 32, src.h, 0);
    for (size_t y = 0; y < plane_h; y++) {
      const uint16_t* row = src.row(y);
      for (int64_t x = 0; x < upscaled_w; x++) {
        int64_t src_x = -(int64_t(1) << SUPERRES_SCALE_BITS) + initial_subpel_x + x * step_x;
        int64_t src_x_px = src_x >> SUPERRES_SCALE_BITS;
        size_t src_x_subpel = size_t((src_x & SUPERRES_SCALE_MASK) >> SUPERRES_EXTRA_BITS);
        int32_t sum = 0;
        for (int k = 0; k < SUPERRES_FILTER_TAPS; k++) {
          int64_t sx = std::max<int64_t>(0, std::min<int64_t>(max_x, src_x_px + (k - SUPERRES_FILTER_OFFSET)));
          sum += int32_t(row[sx]) * UPSCALE_FILTER[src_x_subpel][k];
        }
        dst.set(size_t(x), y, uint16_t(iclamp(round2(sum, FILTER_BITS), 0, maxv)));
      }
    }
    out.planes.push_back(std::move(dst));
  }
  return true;
}

// ---------------------------------------------------------------------------
// Loop restoration (postfilter.rs:568-1004)
// ---------------------------------------------------------------------------
struct LrCtx {  // postfilter.rs:572-597
  const PlaneBuf* cur;
  const PlaneBuf* cdef;
  int32_t stripe_start_y, stripe_end_y, plane_end_x, plane_end_y;
  int32_t sample(int32_t x, int32_t y) const {
    size_t xx = size_t(std::max(std::min(x, plane_end_x), 0));
    y = std::max(std::min(y, plane_end_y), 0);
    if (y < stripe_start_y) {
      size_t yy = size_t(std::max(stripe_start_y - 2, y));
      return cur->get(xx, yy);
    } else if (y > stripe_end_y) {
      size_t yy = size_t(std::min(stripe_end_y + 2, y));
      return cur->get(xx, yy);
    }
    return cdef->get(xx, size_t(y));
  }
};

struct LrParams {  // postfilter.rs:720-725
  bool wiener;
  std::array<std::array<int32_t, 3>, 2> coef;
  size_t set;
  std::array<int32_t, 2> xqd;
};

struct LrBuffers {  // postfilter.rs:729-740
  std::vector<int32_t> win, inter, flt[2], a, b;
  std::vector<int64_t> sq, sum;
  bool integral = false;
  std::vector<uint16_t> out;
};
constexpr size_t LRB = 3;  // postfilter.rs:744

// postfilter.rs:884-898
struct SgrA2Table {
  int32_t t[256];
  SgrA2Table() {
    for (int z = 0; z < 256; z++)
      t[z] = z >= 255 ? 256 : (z == 0 ? 1 : int32_t(((z << SGRPROJ_SGR_BITS) + z / 2) / (z + 1)));
  }
};
const SgrA2Table SGR_A2;

// postfilter.rs:640-661 `lr_stripe`
bool lr_stripe(const FrameCtx& f, size_t plane, size_t s, int32_t& ss0, int32_t& se, int32_t& y0,
               int32_t& y1, size_t& unit_row) {
  auto ss = f.plane_ss(plane);
  int32_t plane_end_y = round2(f.hdr.frame_height, unsigned(ss.second)) - 1;
  int32_t stripe_start_y = (-8 + int32_t(s) * 64) >> ss.second;
  int32_t stripe_end_y = stripe_start_y + (64 >> ss.second) - 1;
  y0 = std::max(stripe_start_y, 0);
  y1 = std::min(stripe_end_y, plane_end_y);
  if (y0 > y1) return false;
  size_t unit_size = f.hdr.loop_restoration_size[plane];
  size_t unit_rows = f.lr[plane].unit_rows;
  size_t luma_row = s * 64 >= 8 ? s * 64 - 8 : 0;
  unit_row = std::min(unit_rows - 1, ((luma_row + 8) >> ss.second) / unit_size);
  ss0 = stripe_start_y;
  se = stripe_end_y;
  return true;
}

// postfilter.rs:664-675 `lr_unit_cols`
std::pair<int32_t, int32_t> lr_unit_cols(const FrameCtx& f, size_t plane, size_t uc) {
  auto ss = f.plane_ss(plane);
  int32_t plane_end_x = round2(f.hdr.upscaled_width, unsigned(ss.first)) - 1;
  int32_t unit_size = int32_t(f.hdr.loop_restoration_size[plane]);
  int32_t x0 = int32_t(uc) * unit_size;
  int32_t x1 = uc + 1 == f.lr[plane].unit_cols ? plane_end_x
                                                : std::min((int32_t(uc) + 1) * unit_size - 1, plane_end_x);
  return {x0, x1};
}

// postfilter.rs:765-777 `lr_window`
void lr_window(const LrCtx& ctx, int32_t x0, int32_t y0, size_t w, size_t h, LrBuffers& buf) {
  size_t ww = w + 2 * LRB, wh = h + 2 * LRB;
  buf.win.resize(ww * wh, 0);
  buf.integral = false;
  for (size_t r = 0; r < wh; r++) {
    int32_t y = y0 + int32_t(r) - int32_t(LRB);
    int32_t* row = &buf.win[r * ww];
    for (size_t c = 0; c < ww; c++) row[c] = ctx.sample(x0 + int32_t(c) - int32_t(LRB), y);
  }
}

// postfilter.rs:860-880 `integral_images`
void integral_images(LrBuffers& buf, size_t ww, size_t wh) {
  size_t iw = ww + 1;
  buf.sq.resize(iw * (wh + 1), 0);
  buf.sum.resize(iw * (wh + 1), 0);
  std::fill(buf.sq.begin(), buf.sq.begin() + iw, 0);
  std::fill(buf.sum.begin(), buf.sum.begin() + iw, 0);
  for (size_t y = 0; y < wh; y++) {
    int64_t rs = 0, rq = 0;
    buf.sq[(y + 1) * iw] = 0;
    buf.sum[(y + 1) * iw] = 0;
    for (size_t x = 0; x < ww; x++) {
      int64_t c = buf.win[y * ww + x];
      rs += c;
      rq += c * c;
      buf.sum[(y + 1) * iw + x + 1] = buf.sum[y * iw + x + 1] + rs;
      buf.sq[(y + 1) * iw + x + 1] = buf.sq[y * iw + x + 1] + rq;
    }
  }
  buf.integral = true;
}

// postfilter.rs:901-991 `box_filter_rect`
void box_filter_rect(const FrameCtx& f, const LrCtx& ctx, int32_t x0, int32_t y0, size_t w, size_t h,
                     size_t set, size_t pass, LrBuffers& buf) {
  int32_t r = SGR_PARAMS[set][pass * 2];
  buf.flt[pass].resize(w * h, 0);
  if (r == 0) return;
  size_t ww = w + 2 * LRB, wh = h + 2 * LRB;
  size_t iw = ww + 1;
  if (!buf.integral) integral_images(buf, ww, wh);
  int32_t eps = SGR_PARAMS[set][pass * 2 + 1];
  uint32_t bd = f.bit_depth;
  int32_t n = (2 * r + 1) * (2 * r + 1);
  int32_t n2e = n * n * eps;
  int32_t s = ((1 << SGRPROJ_MTABLE_BITS) + n2e / 2) / n2e;
  int32_t one_over_n = ((1 << SGRPROJ_RECIP_BITS) + n / 2) / n;
  size_t aw = w + 2;
  buf.a.resize(aw * (h + 2), 0);
  buf.b.resize(aw * (h + 2), 0);
  size_t ru = size_t(r);
  for (size_t i = 0; i < h + 2; i++) {
    if (pass == 0 && ((y0 + int32_t(i) - 1) & 1) == 0) continue;
    size_t wy = i + LRB - 1;
    size_t ya = wy - ru, yb = wy + ru + 1;
    for (size_t j = 0; j < w + 2; j++) {
      size_t wx = j + LRB - 1;
      size_t xa = wx - ru, xb = wx + ru + 1;
      auto boxed = [&](const std::vector<int64_t>& t) {
        return t[yb * iw + xb] - t[ya * iw + xb] - t[yb * iw + xa] + t[ya * iw + xa];
      };
      int64_t a = boxed(buf.sq);
      int32_t b = int32_t(boxed(buf.sum));
      a = round2_64(a, 2 * (bd - 8));
      int64_t d = round2(b, bd - 8);
      int64_t p = std::max<int64_t>(a * n - d * d, 0);
      int64_t z = round2_64(p * s, SGRPROJ_MTABLE_BITS);
      int32_t a2 = SGR_A2.t[std::min<int64_t>(z, 255)];
      int64_t b2 = int64_t((1 << SGRPROJ_SGR_BITS) - a2) * int64_t(b) * int64_t(one_over_n);
      buf.a[i * aw + j] = a2;
      buf.b[i * aw + j] = int32_t(round2_64(b2, SGRPROJ_RECIP_BITS));
    }
  }
  for (size_t i = 0; i < h; i++) {
    int32_t yabs = y0 + int32_t(i);
    int32_t shift = (pass == 0 && (yabs & 1) != 0) ? 4 : 5;
    for (size_t j = 0; j < w; j++) {
      int32_t a = 0, b = 0;
      for (int32_t dy = -1; dy <= 1; dy++) {
        for (int32_t dx = -1; dx <= 1; dx++) {
          int32_t weight;
          if (pass == 0) {
            weight = ((yabs + dy) & 1) != 0 ? (dx == 0 ? 6 : 5) : 0;
          } else {
            weight = (dx == 0 || dy == 0) ? 4 : 3;
          }
          size_t k = size_t(int32_t(i) + 1 + dy) * aw + size_t(int32_t(j) + 1 + dx);
          a += weight * buf.a[k];
          b += weight * buf.b[k];
        }
      }
      int32_t v = a * int32_t(ctx.cdef->get(size_t(x0) + j, size_t(y0) + i)) + b;
      buf.flt[pass][i * w + j] = round2(v, unsigned(SGRPROJ_SGR_BITS + shift - SGRPROJ_RST_BITS));
    }
  }
}

// postfilter.rs:994-1004 `wiener_coefficient`
std::array<int32_t, 7> wiener_coefficient(const std::array<int32_t, 3>& coeff) {
  std::array<int32_t, 7> filter{};
  filter[3] = 128;
  for (int i = 0; i < 3; i++) {
    int32_t c = coeff[i];
    filter[i] = c;
    filter[6 - i] = c;
    filter[3] -= 2 * c;
  }
  return filter;
}

// postfilter.rs:781-853 `restore_rect_from_window`
void restore_rect_from_window(const FrameCtx& f, const LrCtx& ctx, int32_t x0, int32_t y0, size_t w,
                              size_t h, const LrParams& params, LrBuffers& buf) {
  size_t ww = w + 2 * LRB;
  int32_t maxv = (1 << f.bit_depth) - 1;
  buf.out.resize(w * h, 0);
  if (params.wiener) {
    auto rv = f.rounding_variables(false);
    auto vfilter = wiener_coefficient(params.coef[0]);
    auto hfilter = wiener_coefficient(params.coef[1]);
    int32_t bd = int32_t(f.bit_depth);
    int32_t offset = 1 << (bd + FILTER_BITS - int32_t(rv.round0) - 1);
    int32_t limit = (1 << (bd + 1 + FILTER_BITS - int32_t(rv.round0))) - 1;
    buf.inter.resize((h + 6) * w, 0);
    for (size_t r = 0; r < h + 6; r++) {
      const int32_t* src = &buf.win[r * ww];
      for (size_t c = 0; c < w; c++) {
        int32_t s = 0;
        for (int t = 0; t < 7; t++) s += hfilter[t] * src[c + t];
        buf.inter[r * w + c] = clip3(-offset, limit - offset, round2(s, rv.round0));
      }
    }
    for (size_t r = 0; r < h; r++) {
      for (size_t c = 0; c < w; c++) {
        int32_t s = 0;
        for (int t = 0; t < 7; t++) s += vfilter[t] * buf.inter[(r + t) * w + c];
        buf.out[r * w + c] = uint16_t(iclamp(round2(s, rv.round1), 0, maxv));
      }
    }
  } else {
    for (size_t pass = 0; pass < 2; pass++) box_filter_rect(f, ctx, x0, y0, w, h, params.set, pass, buf);
    int32_t w0 = params.xqd[0], w1 = params.xqd[1];
    int32_t w2 = (1 << SGRPROJ_PRJ_BITS) - w0 - w1;
    int32_t r0 = SGR_PARAMS[params.set][0], r1 = SGR_PARAMS[params.set][2];
    for (size_t i = 0; i < h; i++) {
      for (size_t j = 0; j < w; j++) {
        int32_t u = int32_t(ctx.cdef->get(size_t(x0) + j, size_t(y0) + i)) << SGRPROJ_RST_BITS;
        int32_t v = w1 * u;
        v += r0 != 0 ? w0 * buf.flt[0][i * w + j] : w0 * u;
        v += r1 != 0 ? w2 * buf.flt[1][i * w + j] : w2 * u;
        int32_t s = round2(v, unsigned(SGRPROJ_RST_BITS + SGRPROJ_PRJ_BITS));
        buf.out[i * w + j] = uint16_t(iclamp(s, 0, maxv));
      }
    }
  }
}

// postfilter.rs:677-716 `restore_stripe`
void restore_stripe(const FrameCtx& f, const FrameBuf& cur, const FrameBuf& cdefb, SharedPlane out,
                    size_t plane, size_t s) {
  int32_t stripe_start_y, stripe_end_y, y0, y1;
  size_t unit_row;
  if (!lr_stripe(f, plane, s, stripe_start_y, stripe_end_y, y0, y1, unit_row)) return;
  auto ss = f.plane_ss(plane);
  LrCtx ctx{&cur.planes[plane], &cdefb.planes[plane], stripe_start_y, stripe_end_y,
            round2(f.hdr.upscaled_width, unsigned(ss.first)) - 1,
            round2(f.hdr.frame_height, unsigned(ss.second)) - 1};
  const LrPlane& lp = f.lr[plane];
  LrBuffers buf;
  for (size_t uc = 0; uc < lp.unit_cols; uc++) {
    auto xr = lr_unit_cols(f, plane, uc);
    int32_t x0 = xr.first, x1 = xr.second;
    if (x0 > ctx.plane_end_x) continue;
    size_t uidx = unit_row * lp.unit_cols + uc;
    LrParams params{};
    if (lp.lr_type[uidx] == RESTORE_WIENER) {
      params.wiener = true;
      params.coef = lp.wiener[uidx];
    } else if (lp.lr_type[uidx] == RESTORE_SGRPROJ) {
      params.wiener = false;
      params.set = lp.sgr_set[uidx];
      params.xqd = lp.sgr_xqd[uidx];
    } else {
      continue;
    }
    size_t w = size_t(x1 - x0 + 1), h = size_t(y1 - y0 + 1);
    lr_window(ctx, x0, y0, w, h, buf);
    restore_rect_from_window(f, ctx, x0, y0, w, h, params, buf);
    for (size_t i = 0; i < h; i++) out.write_row(size_t(x0), size_t(y0) + i, &buf.out[i * w], w);
  }
}

// postfilter.rs:608-636 `loop_restoration`
FrameBuf loop_restoration(const FrameCtx& f, const FrameBuf& cur, const FrameBuf& cdefb,
                          size_t threads) {
  if (!f.hdr.uses_lr) return cdefb;
  FrameBuf lr = cdefb;
  std::vector<SharedPlane> planes;
  for (auto& p : lr.planes) planes.emplace_back(p);
  size_t stripes = (size_t(f.hdr.frame_height) + 8 + 63) / 64;
  std::vector<std::pair<size_t, size_t>> jobs;
  for (size_t plane = 0; plane < f.num_planes; plane++)
    if (f.hdr.frame_restoration_type[plane] != RESTORE_NONE)
      for (size_t s = 0; s < stripes; s++) jobs.emplace_back(plane, s);
  auto job = [&](size_t i) { restore_stripe(f, cur, cdefb, planes[jobs[i].first], jobs[i].first, jobs[i].second); };
  run_bands(jobs.size(), threads, job);
  return lr;
}

// ---------------------------------------------------------------------------
// Film grain (grain.rs)
// ---------------------------------------------------------------------------
struct Rng {  // grain.rs:8-19
  uint32_t s;
  int32_t get(uint32_t bits) {
    uint32_t r = s;
    uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
    r = (r >> 1) | (bit << 15);
    s = r;
    return int32_t((r >> (16 - bits)) & ((1u << bits) - 1));
  }
};

// grain.rs:24-354 `apply`
void grain_apply(bool mono, uint32_t matrix_coefficients, uint32_t bit_depth, size_t sub_x,
                 size_t sub_y, size_t w, size_t h, const av1pf_film_grain& g,
                 std::vector<std::vector<uint16_t>>& planes) {
  int32_t bd = int32_t(bit_depth);
  size_t num_planes = mono ? 1 : 3;
  int32_t grain_center = 128 << (bd - 8);
  int32_t grain_min = -grain_center;
  int32_t grain_max = (256 << (bd - 8)) - 1 - grain_center;
  Rng rng{uint32_t(g.grain_seed)};

  // 7.18.3.3
  std::vector<std::array<int32_t, 82>> luma_grain(73), cb_grain(73), cr_grain(73);
  for (auto& r : luma_grain) r.fill(0);
  for (auto& r : cb_grain) r.fill(0);
  for (auto& r : cr_grain) r.fill(0);
  unsigned shift = unsigned(12 - bd + g.grain_scale_shift);
  for (auto& row : luma_grain)
    for (auto& v : row) {
      int32_t gv = g.num_y_points > 0 ? GAUSSIAN_SEQUENCE[rng.get(11)] : 0;
      v = round2(gv, shift);
    }
  unsigned ar_shift = unsigned(g.ar_coeff_shift_minus_6 + 6);
  int32_t lag = g.ar_coeff_lag;
  for (int y = 3; y < 73; y++) {
    for (int x = 3; x < 82 - 3; x++) {
      int32_t s = 0;
      int pos = 0;
      bool done = false;
      for (int dr = -lag; dr <= 0 && !done; dr++) {
        for (int dc = -lag; dc <= lag; dc++) {
          if (dr == 0 && dc == 0) {
            done = true;
            break;
          }
          int32_t c = g.ar_coeffs_y_plus_128[pos] - 128;
          s += luma_grain[y + dr][x + dc] * c;
          pos++;
        }
      }
      luma_grain[y][x] = clip3(grain_min, grain_max, luma_grain[y][x] + round2(s, ar_shift));
    }
  }
  size_t chroma_w = sub_x != 0 ? 44 : 82;
  size_t chroma_h = sub_y != 0 ? 38 : 73;
  if (!mono) {
    rng = Rng{uint32_t(g.grain_seed) ^ 0xb524u};
    for (size_t r = 0; r < chroma_h; r++)
      for (size_t c = 0; c < chroma_w; c++) {
        int32_t gv = (g.num_cb_points > 0 || g.chroma_scaling_from_luma) ? GAUSSIAN_SEQUENCE[rng.get(11)] : 0;
        cb_grain[r][c] = round2(gv, shift);
      }
    rng = Rng{uint32_t(g.grain_seed) ^ 0x49d8u};
    for (size_t r = 0; r < chroma_h; r++)
      for (size_t c = 0; c < chroma_w; c++) {
        int32_t gv = (g.num_cr_points > 0 || g.chroma_scaling_from_luma) ? GAUSSIAN_SEQUENCE[rng.get(11)] : 0;
        cr_grain[r][c] = round2(gv, shift);
      }
    for (size_t y = 3; y < chroma_h; y++) {
      for (size_t x = 3; x < chroma_w - 3; x++) {
        int32_t s0 = 0, s1 = 0;
        int pos = 0;
        bool done = false;
        for (int dr = -lag; dr <= 0 && !done; dr++) {
          for (int dc = -lag; dc <= lag; dc++) {
            int32_t c0 = g.ar_coeffs_cb_plus_128[pos] - 128;
            int32_t c1 = g.ar_coeffs_cr_plus_128[pos] - 128;
            if (dr == 0 && dc == 0) {
              if (g.num_y_points > 0) {
                int32_t luma = 0;
                size_t luma_x = ((x - 3) << sub_x) + 3;
                size_t luma_y = ((y - 3) << sub_y) + 3;
                for (size_t i = 0; i <= sub_y; i++)
                  for (size_t j = 0; j <= sub_x; j++) luma += luma_grain[luma_y + i][luma_x + j];
                luma = round2(luma, unsigned(sub_x + sub_y));
                s0 += luma * c0;
                s1 += luma * c1;
              }
              done = true;
              break;
            }
            s0 += cb_grain[size_t(int(y) + dr)][size_t(int(x) + dc)] * c0;
            s1 += cr_grain[size_t(int(y) + dr)][size_t(int(x) + dc)] * c1;
            pos++;
          }
        }
        cb_grain[y][x] = clip3(grain_min, grain_max, cb_grain[y][x] + round2(s0, ar_shift));
        cr_grain[y][x] = clip3(grain_min, grain_max, cr_grain[y][x] + round2(s1, ar_shift));
      }
    }
  }

  // 7.18.3.4 scaling lookup
  int32_t scaling_lut[3][256] = {};
  for (size_t plane = 0; plane < num_planes; plane++) {
    int32_t num_points;
    const int32_t *xs, *ys;
    if (plane == 0 || g.chroma_scaling_from_luma) {
      num_points = g.num_y_points; xs = g.point_y_value; ys = g.point_y_scaling;
    } else if (plane == 1) {
      num_points = g.num_cb_points; xs = g.point_cb_value; ys = g.point_cb_scaling;
    } else {
      num_points = g.num_cr_points; xs = g.point_cr_value; ys = g.point_cr_scaling;
    }
    if (num_points == 0) continue;
    int32_t* lut = scaling_lut[plane];
    for (int32_t x = 0; x < xs[0]; x++) lut[x] = ys[0];
    for (int32_t i = 0; i < num_points - 1; i++) {
      int32_t delta_y = ys[i + 1] - ys[i];
      int32_t delta_x = xs[i + 1] - xs[i];
      int32_t delta = delta_y * ((65536 + (delta_x >> 1)) / delta_x);
      for (int32_t x = 0; x < delta_x; x++) {
        int32_t v = ys[i] + ((x * delta + 32768) >> 16);
        lut[xs[i] + x] = v;
      }
    }
    for (int32_t x = xs[num_points - 1]; x < 256; x++) lut[x] = ys[num_points - 1];
  }
  auto scale_lut = [&](size_t plane, int32_t index) -> int32_t {
    int32_t sh = bd - 8;
    int32_t x = index >> sh;
    int32_t rem = index - (x << sh);
    if (bd == 8 || x == 255) return scaling_lut[plane][x];
    int32_t start = scaling_lut[plane][x];
    int32_t end = scaling_lut[plane][x + 1];
    return start + round2((end - start) * rem, unsigned(sh));
  };

  // 7.18.3.5 add noise
  size_t hh = (h + 1) / 2;
  size_t chroma_cols = (w + sub_x) >> sub_x;
  size_t noise_w[3] = {w + 34, chroma_cols + 34, chroma_cols + 34};
  std::vector<std::array<std::vector<int32_t>, 3>> noise_stripe;
  size_t luma_num = 0;
  for (size_t y = 0; y < hh; y += 16) {
    std::array<std::vector<int32_t>, 3> ns;
    for (int pl = 0; pl < 3; pl++) ns[pl].assign(34 * noise_w[pl], 0);
    rng = Rng{uint32_t(g.grain_seed)};
    rng.s ^= uint32_t(((luma_num * 37 + 178) & 255) << 8);
    rng.s ^= uint32_t((luma_num * 173 + 105) & 255);
    for (size_t x = 0; x < (w + 1) / 2; x += 16) {
      int32_t rand = rng.get(8);
      size_t offset_x = size_t(rand >> 4), offset_y = size_t(rand & 15);
      for (size_t plane = 0; plane < num_planes; plane++) {
        size_t psx = plane > 0 ? sub_x : 0, psy = plane > 0 ? sub_y : 0;
        size_t pox = psx != 0 ? 6 + offset_x : 9 + offset_x * 2;
        size_t poy = psy != 0 ? 6 + offset_y : 9 + offset_y * 2;
        size_t nw = noise_w[plane];
        for (size_t i = 0; i < (size_t(34) >> psy); i++) {
          for (size_t j = 0; j < (size_t(34) >> psx); j++) {
            int32_t gv = plane == 0 ? luma_grain[poy + i][pox + j]
                                    : (plane == 1 ? cb_grain[poy + i][pox + j] : cr_grain[poy + i][pox + j]);
            if (psx == 0) {
              size_t idx = i * nw + x * 2 + j;
              if (j < 2 && g.overlap_flag && x > 0) {
                int32_t old = ns[plane][idx];
                gv = j == 0 ? old * 27 + gv * 17 : old * 17 + gv * 27;
                gv = clip3(grain_min, grain_max, round2(gv, 5));
              }
              ns[plane][idx] = gv;
            } else {
              size_t idx = i * nw + x + j;
              if (j == 0 && g.overlap_flag && x > 0) {
                int32_t old = ns[plane][idx];
                gv = old * 23 + gv * 22;
                gv = clip3(grain_min, grain_max, round2(gv, 5));
              }
              ns[plane][idx] = gv;
            }
          }
        }
      }
    }
    noise_stripe.push_back(std::move(ns));
    luma_num++;
  }
  std::vector<int32_t> noise_image[3];
  for (size_t plane = 0; plane < num_planes; plane++) {
    size_t psx = plane > 0 ? sub_x : 0, psy = plane > 0 ? sub_y : 0;
    size_t pw = (w + psx) >> psx, ph = (h + psy) >> psy;
    size_t nw = noise_w[plane];
    std::vector<int32_t> img(pw * ph, 0);
    for (size_t yy = 0; yy < ph; yy++) {
      size_t ln = yy >> (5 - psy);
      size_t i = yy - (ln << (5 - psy));
      for (size_t xx = 0; xx < pw; xx++) {
        int32_t gv = noise_stripe[ln][plane][i * nw + xx];
        if (psy == 0) {
          if (i < 2 && ln > 0 && g.overlap_flag) {
            int32_t old = noise_stripe[ln - 1][plane][(i + 32) * nw + xx];
            gv = i == 0 ? old * 27 + gv * 17 : old * 17 + gv * 27;
            gv = clip3(grain_min, grain_max, round2(gv, 5));
          }
        } else if (i < 1 && ln > 0 && g.overlap_flag) {
          int32_t old = noise_stripe[ln - 1][plane][(i + 16) * nw + xx];
          gv = old * 23 + gv * 22;
          gv = clip3(grain_min, grain_max, round2(gv, 5));
        }
        img[yy * pw + xx] = gv;
      }
    }
    noise_image[plane] = std::move(img);
  }
  int32_t min_value, max_luma, max_chroma;
  if (g.clip_to_restricted_range) {
    min_value = 16 << (bd - 8);
    max_luma = 235 << (bd - 8);
    max_chroma = matrix_coefficients == MC_IDENTITY ? max_luma : (240 << (bd - 8));
  } else {
    min_value = 0;
    max_luma = (256 << (bd - 8)) - 1;
    max_chroma = (256 << (bd - 8)) - 1;
  }
  unsigned scaling_shift = unsigned(g.grain_scaling_minus_8 + 8);
  int32_t maxv = (1 << bd) - 1;
  if (num_planes > 1) {
    size_t cw = (w + sub_x) >> sub_x, ch = (h + sub_y) >> sub_y;
    for (size_t yy = 0; yy < ch; yy++) {
      for (size_t xx = 0; xx < cw; xx++) {
        size_t luma_x = xx << sub_x, luma_y = yy << sub_y;
        size_t luma_next_x = std::min(luma_x + 1, w - 1);
        int32_t average_luma = sub_x != 0 ? round2(int32_t(planes[0][luma_y * w + luma_x]) +
                                                       int32_t(planes[0][luma_y * w + luma_next_x]), 1)
                                          : int32_t(planes[0][luma_y * w + luma_x]);
        if (g.num_cb_points > 0 || g.chroma_scaling_from_luma) {
          int32_t orig = planes[1][yy * cw + xx];
          int32_t merged;
          if (g.chroma_scaling_from_luma) {
            merged = average_luma;
          } else {
            int32_t combined = average_luma * (g.cb_luma_mult - 128) + orig * (g.cb_mult - 128);
            merged = iclamp((combined >> 6) + ((g.cb_offset - 256) << (bd - 8)), 0, maxv);
          }
          int32_t noise = noise_image[1][yy * cw + xx];
          noise = round2(scale_lut(1, merged) * noise, scaling_shift);
          planes[1][yy * cw + xx] = uint16_t(clip3(min_value, max_chroma, orig + noise));
        }
        if (g.num_cr_points > 0 || g.chroma_scaling_from_luma) {
          int32_t orig = planes[2][yy * cw + xx];
          int32_t merged;
          if (g.chroma_scaling_from_luma) {
            merged = average_luma;
          } else {
            int32_t combined = average_luma * (g.cr_luma_mult - 128) + orig * (g.cr_mult - 128);
            merged = iclamp((combined >> 6) + ((g.cr_offset - 256) << (bd - 8)), 0, maxv);
          }
          int32_t noise = noise_image[2][yy * cw + xx];
          noise = round2(scale_lut(2, merged) * noise, scaling_shift);
          planes[2][yy * cw + xx] = uint16_t(clip3(min_value, max_chroma, orig + noise));
        }
      }
    }
  }
  if (g.num_y_points > 0) {
    for (size_t yy = 0; yy < h; yy++) {
      for (size_t xx = 0; xx < w; xx++) {
        int32_t orig = planes[0][yy * w + xx];
        int32_t noise = noise_image[0][yy * w + xx];
        noise = round2(scale_lut(0, orig) * noise, scaling_shift);
        planes[0][yy * w + xx] = uint16_t(clip3(min_value, max_luma, orig + noise));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Adapters between the C ABI descriptors and the restated state.
// ---------------------------------------------------------------------------
bool info_ok(const av1pf_frame_info* info) {
  if (!info) return false;
  if (info->bit_depth != 8 && info->bit_depth != 10 && info->bit_depth != 12) return false;
  if (info->sample_bytes != 2 && !(info->sample_bytes == 1 && info->bit_depth == 8)) return false;
  if (info->num_planes != 1 && info->num_planes != 3) return false;
  if (info->frame_width <= 0 || info->frame_height <= 0 || info->upscaled_width < info->frame_width)
    return false;
  if (info->mi_cols != 2 * ((info->frame_width + 7) >> 3) || info->mi_rows != 2 * ((info->frame_height + 7) >> 3))
    return false;
  return true;
}

PlaneBuf plane_from(const av1pf_plane& p, int sample_bytes) {
  PlaneBuf b(size_t(p.width), size_t(p.height), 0);
  for (int y = 0; y < p.height; y++) {
    if (sample_bytes == 1) {
      const uint8_t* s = static_cast<const uint8_t*>(p.data) + int64_t(y) * p.stride;
      for (int x = 0; x < p.width; x++) b.data[size_t(y) * b.stride + size_t(x)] = s[x];
    } else {
      const uint16_t* s = static_cast<const uint16_t*>(p.data) + int64_t(y) * p.stride;
      std::memcpy(&b.data[size_t(y) * b.stride], s, size_t(p.width) * 2);
    }
  }
  return b;
}

// Writes rows [0,h) x cols [0,w) of `b` into `p` (clipped to p's size).
void plane_to(const PlaneBuf& b, av1pf_plane& p, int sample_bytes, size_t w, size_t h) {
  w = std::min({w, size_t(p.width), b.w});
  h = std::min({h, size_t(p.height), b.h});
  for (size_t y = 0; y < h; y++) {
    if (sample_bytes == 1) {
      uint8_t* d = static_cast<uint8_t*>(p.data) + int64_t(y) * p.stride;
      for (size_t x = 0; x < w; x++) d[x] = uint8_t(b.get(x, y));
    } else {
      uint16_t* d = static_cast<uint16_t*>(p.data) + int64_t(y) * p.stride;
      std::memcpy(d, &b.data[y * b.stride], w * 2);
    }
  }
}

void hdr_from(Hdr& h, const av1pf_frame_info* info, const av1pf_params* p) {
  h.frame_width = info->frame_width;
  h.frame_height = info->frame_height;
  h.upscaled_width = info->upscaled_width;
  if (!p) return;
  for (int i = 0; i < 4; i++) h.loop_filter_level[i] = p->loop_filter_level[i];
  h.loop_filter_sharpness = p->loop_filter_sharpness;
  h.loop_filter_delta_enabled = p->loop_filter_delta_enabled != 0;
  for (int i = 0; i < 8; i++) h.loop_filter_ref_deltas[i] = p->loop_filter_ref_deltas[i];
  for (int i = 0; i < 2; i++) h.loop_filter_mode_deltas[i] = p->loop_filter_mode_deltas[i];
  h.delta_lf_multi = p->delta_lf_multi != 0;
  h.segmentation_enabled = p->segmentation_enabled != 0;
  for (int s = 0; s < 8; s++)
    for (int k = 0; k < 8; k++) {
      h.feature_enabled[s][k] = p->feature_enabled[s][k] != 0;
      h.feature_data[s][k] = p->feature_data[s][k];
    }
  h.cdef_on = p->cdef_enabled != 0;
  h.cdef_damping = p->cdef_damping;
  for (int i = 0; i < 8; i++) {
    h.cdef_y_pri_strength[i] = p->cdef_y_pri_strength[i];
    h.cdef_y_sec_strength[i] = p->cdef_y_sec_strength[i];
    h.cdef_uv_pri_strength[i] = p->cdef_uv_pri_strength[i];
    h.cdef_uv_sec_strength[i] = p->cdef_uv_sec_strength[i];
  }
  h.use_superres = p->use_superres != 0;
  h.uses_lr = p->uses_lr != 0;
  for (int i = 0; i < 3; i++) {
    h.frame_restoration_type[i] = uint8_t(p->frame_restoration_type[i]);
    h.loop_restoration_size[i] = size_t(p->loop_restoration_size[i]);
  }
}

// Builds the FrameCtx the reference's filters read from the descriptors.
void ctx_from(FrameCtx& f, const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
              const av1pf_plane* planes) {
  hdr_from(f.hdr, info, p);
  f.bit_depth = uint32_t(info->bit_depth);
  f.ssx = size_t(info->subsampling_x);
  f.ssy = size_t(info->subsampling_y);
  f.num_planes = size_t(info->num_planes);
  f.mi_rows = size_t(info->mi_rows);
  f.mi_cols = size_t(info->mi_cols);
  if (maps) {
    f.ms = size_t(maps->mi_stride);
    size_t n = (f.mi_rows + 32) * f.ms;
    f.mi.assign(n, Mi{});
    if (maps->mi) {
      for (size_t i = 0; i < f.mi_rows * f.ms; i++) {
        const av1pf_mi& s = maps->mi[i];
        Mi& d = f.mi[i];
        d.mi_size = s.mi_size;
        d.y_mode = s.y_mode;
        d.ref_frame0 = s.ref_frame0;
        d.skip = (s.skip_segment & AV1PF_MI_SKIP) != 0;
        d.segment_id = s.skip_segment & 7;
        for (int k = 0; k < 4; k++) d.delta_lf[k] = s.delta_lf[k];
      }
    }
    for (size_t pl = 0; pl < 3; pl++) {
      f.lf_tx_sizes[pl].assign(n, 0);
      if (pl < f.num_planes && maps->lf_tx_size[pl]) {
        size_t sy = pl == 0 ? 0 : f.ssy;
        size_t rows = (f.mi_rows + (size_t(1) << sy) - 1) >> sy;
        std::memcpy(f.lf_tx_sizes[pl].data(), maps->lf_tx_size[pl], rows * f.ms);
      }
    }
    f.cdef_stride = size_t(maps->cdef_stride);
    f.cdef_idx.assign(f.cdef_stride * ((f.mi_rows >> 4) + 2), -1);
    if (maps->cdef_idx) {
      size_t rows = (f.mi_rows + 15) >> 4;
      std::memcpy(f.cdef_idx.data(), maps->cdef_idx, rows * f.cdef_stride);
    }
    for (size_t pl = 0; pl < f.num_planes && p; pl++) {
      LrPlane& l = f.lr[pl];
      if (f.hdr.frame_restoration_type[pl] == RESTORE_NONE) continue;
      l.unit_rows = size_t(p->lr_unit_rows[pl]);
      l.unit_cols = size_t(p->lr_unit_cols[pl]);
      size_t units = l.unit_rows * l.unit_cols;
      l.lr_type.assign(units, RESTORE_NONE);
      l.wiener.assign(units, {});
      l.sgr_set.assign(units, 0);
      l.sgr_xqd.assign(units, {});
      const av1pf_lr_unit* u = maps->lr_units[pl];
      if (!u) continue;
      for (size_t i = 0; i < units; i++) {
        l.lr_type[i] = u[i].type;
        l.sgr_set[i] = u[i].sgr_set;
        l.sgr_xqd[i] = {u[i].sgr_xqd[0], u[i].sgr_xqd[1]};
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 3; b++) l.wiener[i][size_t(a)][size_t(b)] = u[i].wiener[a][b];
      }
    }
  }
  if (planes)
    for (size_t pl = 0; pl < f.num_planes; pl++) f.cur.planes.push_back(plane_from(planes[pl], info->sample_bytes));
}

FrameBuf frame_from(const av1pf_frame_info* info, const av1pf_plane* planes) {
  FrameBuf fb;
  for (int pl = 0; pl < info->num_planes; pl++) fb.planes.push_back(plane_from(planes[pl], info->sample_bytes));
  return fb;
}

void frame_to(const FrameBuf& fb, const av1pf_frame_info* info, av1pf_plane* planes, bool visible_only) {
  for (int pl = 0; pl < info->num_planes; pl++) {
    size_t sx = pl ? size_t(info->subsampling_x) : 0, sy = pl ? size_t(info->subsampling_y) : 0;
    size_t w = visible_only ? size_t(round2(info->upscaled_width, unsigned(sx))) : fb.planes[size_t(pl)].w;
    size_t h = visible_only ? size_t(round2(info->frame_height, unsigned(sy))) : fb.planes[size_t(pl)].h;
    plane_to(fb.planes[size_t(pl)], planes[pl], info->sample_bytes, w, h);
  }
}

// decoder/mod.rs:846-917 `output` (the sample path: crop, grain, pack)
void output(const av1pf_frame_info* info, const av1pf_params* p, const FrameBuf& frame, uint8_t* out) {
  size_t w = size_t(info->upscaled_width), h = size_t(info->frame_height);
  size_t sxs = size_t(info->subsampling_x), sys = size_t(info->subsampling_y);
  bool grain_on = p && p->film_grain.apply;
  std::vector<std::vector<uint16_t>> planes;
  size_t np = size_t(info->num_planes);
  if (grain_on) {
    for (size_t pl = 0; pl < np; pl++) {
      size_t sx = pl ? sxs : 0, sy = pl ? sys : 0;
      size_t pw = (w + sx) >> sx, ph = (h + sy) >> sy;
      std::vector<uint16_t> v;
      v.reserve(pw * ph);
      for (size_t y = 0; y < ph; y++) {
        const uint16_t* r = frame.planes[pl].row(y);
        v.insert(v.end(), r, r + pw);
      }
      planes.push_back(std::move(v));
    }
    grain_apply(np == 1, uint32_t(info->matrix_coefficients), uint32_t(info->bit_depth), sxs, sys, w, h,
                p->film_grain, planes);
  }
  bool wide = info->bit_depth > 8;
  size_t off = 0;
  for (size_t pl = 0; pl < np; pl++) {
    size_t sx = pl ? sxs : 0, sy = pl ? sys : 0;
    size_t pw = (w + sx) >> sx, ph = (h + sy) >> sy;
    for (size_t y = 0; y < ph; y++) {
      const uint16_t* src = grain_on ? &planes[pl][y * pw] : frame.planes[pl].row(y);
      if (wide) {
        for (size_t x = 0; x < pw; x++) {
          out[off + (y * pw + x) * 2] = uint8_t(src[x] & 0xff);
          out[off + (y * pw + x) * 2 + 1] = uint8_t(src[x] >> 8);
        }
      } else {
        for (size_t x = 0; x < pw; x++) out[off + y * pw + x] = uint8_t(src[x]);
      }
    }
    off += pw * ph * (wide ? 2 : 1);
  }
}

// xorshift of the reference's KATs (lf.rs:311-317, cdef.rs:252-258)
struct XorShift {
  uint64_t seed;
  uint64_t operator()(uint64_t n) {
    seed ^= seed << 13;
    seed ^= seed >> 7;
    seed ^= seed << 17;
    return seed % n;
  }
};

LfParams lf_params_from(const av1pf_lf_edge_params& p) {
  return LfParams{p.limit, p.blimit, p.thresh, size_t(p.filter_size), p.chroma != 0, uint32_t(p.bit_depth)};
}

// ---------------------------------------------------------------------------
// Encoder filter searches (encoder/cdef.rs, encoder/mod.rs:1457-1506)
// ---------------------------------------------------------------------------
using Pair = std::pair<uint32_t, uint32_t>;

// encoder/cdef.rs:43-46 `sec`
int32_t coded_sec(uint32_t coded) { return coded == 3 ? 4 : int32_t(coded); }

// encoder/cdef.rs:255-258 `damping_for`
uint32_t damping_for(uint32_t qidx) { return std::min(qidx >> 6, 3u); }

// encoder/cdef.rs:60-80: the candidate (primary, coded secondary) pairs
void cdef_candidates(bool thorough, std::vector<Pair>& y, std::vector<Pair>& uv) {
  const std::vector<uint32_t> y_pri = thorough ? std::vector<uint32_t>{0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15}
                                               : std::vector<uint32_t>{0, 1, 2, 4, 6, 9, 12};
  const std::vector<uint32_t> uv_pri = thorough ? std::vector<uint32_t>{0, 1, 2, 3, 4, 6, 8, 11}
                                                : std::vector<uint32_t>{0, 1, 2, 4, 7};
  y.clear();
  uv.clear();
  for (uint32_t p : y_pri)
    for (uint32_t s : {0u, 1u, 2u, 3u}) y.emplace_back(p, s);
  for (uint32_t p : uv_pri)
    for (uint32_t s : {0u, 1u, 2u}) uv.emplace_back(p, s);
}

// encoder/cdef.rs:261-285 `block_sse`
uint64_t block_sse(const uint16_t* res, size_t w, size_t h, const PlaneBuf& src, size_t x0, size_t y0,
                   const FrameCtx& f, size_t plane) {
  auto ss = f.plane_ss(plane);
  size_t fw = (size_t(f.hdr.frame_width) + ss.first) >> ss.first;
  size_t fh = (size_t(f.hdr.frame_height) + ss.second) >> ss.second;
  size_t hh = std::min(h, fh > y0 ? fh - y0 : 0), ww = std::min(w, fw > x0 ? fw - x0 : 0);
  uint64_t s = 0;
  for (size_t i = 0; i < hh; i++)
    for (size_t j = 0; j < ww; j++) {
      int64_t d = int64_t(res[i * w + j]) - int64_t(src.get(x0 + j, y0 + i));
      s += uint64_t(d * d);
    }
  return s;
}

struct CdefSearch {
  uint32_t damping_minus_3 = 0, bits = 0;
  std::vector<Pair> y, uv;           // the chosen pairs, one per index
  std::vector<int8_t> table;         // cdef_idx with each coding block's index
  std::vector<std::pair<size_t, size_t>> blocks;  // (fb row, fb col) of the coding blocks
  std::vector<uint64_t> ysse, uvsse;  // [block][candidate]
  size_t ny = 0, nuv = 0;
};

// encoder/cdef.rs:52-251 `search`. `f.cur` holds the deblocked frame.
CdefSearch cdef_search(const FrameCtx& f, const FrameBuf& src, uint32_t qidx, double lambda, bool thorough,
                       size_t threads) {
  CdefSearch out;
  std::vector<Pair> ycands, uvcands;
  cdef_candidates(thorough, ycands, uvcands);
  const uint32_t damping_minus_3 = damping_for(qidx);
  const uint32_t coeff_shift = f.bit_depth - 8;
  const int32_t damping = int32_t(damping_minus_3) + 3;
  const size_t fb_rows = (f.mi_rows + 15) / 16, fb_cols = (f.mi_cols + 15) / 16;
  for (size_t fr = 0; fr < fb_rows; fr++)
    for (size_t fc = 0; fc < fb_cols; fc++)
      if (f.cdef_idx[fr * f.cdef_stride + fc] >= 0) out.blocks.emplace_back(fr, fc);
  out.table = f.cdef_idx;
  out.ny = ycands.size();
  out.nuv = uvcands.size();
  if (out.blocks.empty()) {  // CdefParams::off()
    out.y = {Pair(0, 0)};
    out.uv = {Pair(0, 0)};
    return out;
  }
  const size_t ny = out.ny, nuv = out.nuv, nb = out.blocks.size();
  out.ysse.assign(nb * ny, 0);
  out.uvsse.assign(nb * nuv, 0);
  const size_t cols = f.ms;
  auto per_block = [&](size_t bi) {
    size_t fr = out.blocks[bi].first, fc = out.blocks[bi].second;
    uint64_t* ysse = &out.ysse[bi * ny];
    uint64_t* uvsse = &out.uvsse[bi * nuv];
    uint16_t res[64];
    for (size_t r = fr * 16; r < std::min(fr * 16 + 16, f.mi_rows); r += 2) {
      for (size_t c = fc * 16; c < std::min(fc * 16 + 16, f.mi_cols); c += 2) {
        auto sk = [&](size_t rr, size_t cc) { return f.mi[rr * cols + cc].skip; };
        if (sk(r, c) && sk(r + 1, c) && sk(r, c + 1) && sk(r + 1, c + 1)) continue;
        auto dv = cdef_direction(f, r, c);
        size_t y_dir = dv.first;
        int32_t var = dv.second;
        size_t x0 = c * MI_SIZE, y0 = r * MI_SIZE;
        size_t xlim = f.mi_cols * MI_SIZE, ylim = f.mi_rows * MI_SIZE;
        for (size_t k = 0; k < ny; k++) {
          int32_t pri_str = int32_t(ycands[k].first) << coeff_shift;
          int32_t sec_str = coded_sec(ycands[k].second) << coeff_shift;
          size_t dir = pri_str == 0 ? 0 : y_dir;
          int32_t var_str = (var >> 6) != 0 ? std::min(int32_t(floor_log2(uint32_t(var >> 6))), 12) : 0;
          pri_str = var != 0 ? (pri_str * (4 + var_str) + 8) >> 4 : 0;
          int32_t d = damping + int32_t(coeff_shift);
          cdef_filter_block(f.cur.planes[0], x0, y0, 8, 8, xlim, ylim, pri_str, sec_str, d, dir, coeff_shift, res);
          ysse[k] += block_sse(res, 8, 8, src.planes[0], x0, y0, f, 0);
        }
        if (f.num_planes > 1) {
          size_t w = 8 >> f.ssx, h = 8 >> f.ssy;
          size_t cx0 = x0 >> f.ssx, cy0 = y0 >> f.ssy;
          size_t cxlim = xlim >> f.ssx, cylim = ylim >> f.ssy;
          for (size_t k = 0; k < nuv; k++) {
            int32_t pri_str = int32_t(uvcands[k].first) << coeff_shift;
            int32_t sec_str = coded_sec(uvcands[k].second) << coeff_shift;
            size_t dir = pri_str == 0 ? 0 : CDEF_UV_DIR[f.ssx][f.ssy][y_dir];
            int32_t d = damping + int32_t(coeff_shift) - 1;
            uint64_t total = 0;
            for (size_t p = 1; p < 3; p++) {
              cdef_filter_block(f.cur.planes[p], cx0, cy0, w, h, cxlim, cylim, pri_str, sec_str, d, dir,
                                coeff_shift, res);
              total += block_sse(res, w, h, src.planes[p], cx0, cy0, f, p);
            }
            uvsse[k] += total;
          }
        }
      }
    }
  };
  run_bands(nb, threads, per_block);
  // Greedy choice of up to 2^bits (luma, chroma) pairs, for each bits
  // (encoder/cdef.rs:195-240).
  auto best_for = [&](const std::vector<std::pair<size_t, size_t>>& set, std::vector<size_t>* pick) {
    double total = 0;
    for (size_t b = 0; b < nb; b++) {
      uint64_t best = UINT64_MAX;
      for (size_t i = 0; i < set.size(); i++) {
        uint64_t v = out.ysse[b * ny + set[i].first] + out.uvsse[b * nuv + set[i].second];
        if (v < best) {
          best = v;
          if (pick) (*pick)[b] = i;
        }
      }
      total += double(best);
    }
    return total;
  };
  double best_cost = DBL_MAX;
  std::vector<std::pair<size_t, size_t>> set, best_set;
  std::vector<size_t> best_pick;
  for (uint32_t bits = 0; bits <= 3; bits++) {
    while (set.size() < (size_t(1) << bits)) {
      double add_t = DBL_MAX;
      std::pair<size_t, size_t> add(0, 0);
      for (size_t yk = 0; yk < ny; yk++) {
        for (size_t uk = 0; uk < nuv; uk++) {
          if (std::find(set.begin(), set.end(), std::make_pair(yk, uk)) != set.end()) continue;
          set.emplace_back(yk, uk);
          double t = best_for(set, nullptr);
          set.pop_back();
          if (t < add_t) {
            add_t = t;
            add = {yk, uk};
          }
        }
      }
      set.push_back(add);
    }
    std::vector<size_t> pick(nb, 0);
    double t = best_for(set, &pick);
    // lambda * (bits as f64) * nb as f64, evaluated left to right
    double cost = t + lambda * double(bits) * double(nb);
    if (cost < best_cost) {
      best_cost = cost;
      best_set = set;
      best_pick = pick;
    }
  }
  out.damping_minus_3 = damping_minus_3;
  out.bits = uint32_t(__builtin_ctz(unsigned(best_set.size())));
  for (size_t b = 0; b < nb; b++)
    out.table[out.blocks[b].first * f.cdef_stride + out.blocks[b].second] = int8_t(best_pick[b]);
  for (auto& s : best_set) {
    out.y.push_back(ycands[s.first]);
    out.uv.push_back(uvcands[s.second]);
  }
  return out;
}

// encoder/mod.rs:1494-1506 `plane_sse`
uint64_t plane_sse(const FrameCtx& f, const FrameBuf& src, size_t p) {
  auto ss = f.plane_ss(p);
  size_t w = (size_t(f.hdr.frame_width) + ss.first) >> ss.first;
  size_t h = (size_t(f.hdr.frame_height) + ss.second) >> ss.second;
  uint64_t s = 0;
  for (size_t y = 0; y < h; y++) {
    const uint16_t* a = src.planes[p].row(y);
    const uint16_t* b = f.cur.planes[p].row(y);
    for (size_t x = 0; x < w; x++) {
      int64_t d = int64_t(a[x]) - int64_t(b[x]);
      s += uint64_t(d * d);
    }
  }
  return s;
}

// encoder/mod.rs:1457-1493 `search_lf`: f.cur is left unfiltered.
std::array<uint32_t, 4> search_lf(FrameCtx& f, const FrameBuf& src, const std::array<uint32_t, 4>& start,
                                  size_t threads, uint64_t* sse_out) {
  const FrameBuf saved = f.cur;
  std::pair<uint64_t, uint32_t> best[3] = {{UINT64_MAX, 0}, {UINT64_MAX, 0}, {UINT64_MAX, 0}};
  const size_t planes = f.num_planes;
  const double scales[6] = {0.0, 0.5, 0.75, 1.0, 1.25, 1.5};
  for (size_t si = 0; si < 6; si++) {
    auto lv = [&](uint32_t l) { return std::min(uint32_t(std::round(double(l) * scales[si])), 63u); };
    uint32_t levels[4] = {lv(start[0]), lv(start[1]), lv(start[2]), lv(start[3])};
    for (int i = 0; i < 4; i++) f.hdr.loop_filter_level[i] = int32_t(levels[i]);
    if (levels[0] != 0 || levels[1] != 0) loop_filter_threads(f, threads);
    for (size_t p = 0; p < planes; p++) {
      uint64_t e = plane_sse(f, src, p);
      if (sse_out) sse_out[si * 3 + p] = e;
      if (e < best[p].first) best[p] = {e, p == 0 ? levels[0] : levels[1 + p]};
    }
    f.cur.planes = saved.planes;
  }
  // Chroma is filtered only when luma is.
  if (best[0].second == 0) return {0, 0, 0, 0};
  return {best[0].second, best[0].second, best[1].second, best[2].second};
}

// encoder/lr.rs:212-233 `solve`: m x = v by Gaussian elimination with
// partial pivoting (the last row of equal magnitude wins, as Iterator::max_by
// keeps the last maximum); zeros when singular.
template <size_t N>
std::array<double, N> lr_solve(std::array<std::array<double, N>, N> m, std::array<double, N> v) {
  for (size_t i = 0; i < N; i++) {
    size_t piv = i;
    for (size_t a = i + 1; a < N; a++)
      if (!(std::fabs(m[a][i]) < std::fabs(m[piv][i]))) piv = a;  // >=: the last maximum
    std::swap(m[i], m[piv]);
    std::swap(v[i], v[piv]);
    if (std::fabs(m[i][i]) < 1e-9) return {};
    for (size_t r = 0; r < N; r++) {
      if (r != i) {
        double fct = m[r][i] / m[i][i];
        for (size_t c = i; c < N; c++) m[r][c] -= fct * m[i][c];
        v[r] -= fct * v[i];
      }
    }
  }
  std::array<double, N> x{};
  for (size_t i = 0; i < N; i++) x[i] = v[i] / m[i][i];
  return x;
}

// f64 -> i32 as Rust's `as` converts (saturating, NaN to 0).
int32_t f64_to_i32(double x) {
  if (std::isnan(x)) return 0;
  if (x <= -2147483648.0) return INT32_MIN;
  if (x >= 2147483647.0) return INT32_MAX;
  return int32_t(x);
}

const int32_t WIENER_TAPS_MIN_T[3] = AV1T_WIENER_TAPS_MIN, WIENER_TAPS_MAX_T[3] = AV1T_WIENER_TAPS_MAX;
const int32_t SGRPROJ_XQD_MIN_T[2] = AV1T_SGRPROJ_XQD_MIN, SGRPROJ_XQD_MAX_T[2] = AV1T_SGRPROJ_XQD_MAX;

struct LrRect {
  LrCtx ctx;
  int32_t y0;
  size_t h;
};

// encoder/lr.rs:235-328 `fit_wiener`: [vertical, horizontal] coefficients.
std::array<std::array<int32_t, 3>, 2> fit_wiener(size_t plane, const std::vector<LrRect>& rects, int32_t x0, size_t w,
                                                 const PlaneBuf& src, size_t step, LrBuffers& buf) {
  const size_t first = plane == 0 ? 0 : 1;
  const size_t ww = w + 2 * LRB;
  std::array<double, 3> hc{}, vc{};
  for (int iter = 0; iter < 3; iter++) {
    const bool vertical = iter % 2 == 0;
    std::array<std::array<double, 3>, 3> m{};
    std::array<double, 3> v{};
    for (const LrRect& rc : rects) {
      lr_window(rc.ctx, x0, rc.y0, w, rc.h, buf);
      auto at = [&](size_t r, size_t c) { return double(buf.win[r * ww + c]); };
      for (size_t i = 0; i < rc.h; i += step) {
        const uint16_t* srow = src.row(size_t(rc.y0) + i) + x0;
        for (size_t j = 0; j < w; j += step) {
          double line[7];
          for (size_t t = 0; t < 7; t++) {
            size_t r = vertical ? i + t : i + LRB, c = vertical ? j + LRB : j + t;
            const std::array<double, 3>& other = vertical ? hc : vc;
            double center = at(r, c);
            double sum = center;
            for (size_t k = 0; k < 3; k++) {
              size_t d = 3 - k;
              double a = vertical ? at(r, c - d) : at(r - d, c);
              double b = vertical ? at(r, c + d) : at(r + d, c);
              sum += other[k] * (a + b - 2.0 * center);
            }
            line[t] = sum;
          }
          double target = double(srow[j]) - line[3];
          double d[3];
          for (size_t k = 0; k < 3; k++) d[k] = line[k] + line[6 - k] - 2.0 * line[3];
          for (size_t a = first; a < 3; a++) {
            for (size_t b = first; b < 3; b++) m[a][b] += d[a] * d[b];
            v[a] += d[a] * target;
          }
        }
      }
    }
    std::array<double, 3> sol{};
    if (first == 0) {
      sol = lr_solve<3>(m, v);
    } else {
      std::array<double, 2> s2 = lr_solve<2>({{{m[1][1], m[1][2]}, {m[2][1], m[2][2]}}}, {v[1], v[2]});
      sol = {0.0, s2[0], s2[1]};
    }
    if (vertical)
      vc = sol;
    else
      hc = sol;
  }
  auto q = [&](const std::array<double, 3>& c) {
    std::array<int32_t, 3> o{};
    for (size_t k = 0; k < 3; k++)
      o[k] = k < first ? 0 : iclamp(f64_to_i32(std::round(c[k] * 128.0)), WIENER_TAPS_MIN_T[k], WIENER_TAPS_MAX_T[k]);
    return o;
  };
  return {q(vc), q(hc)};
}

// encoder/lr.rs:330-430 `fit_sgr`: the projection weights of set `set` and
// their error.
std::pair<std::array<int32_t, 2>, uint64_t> fit_sgr(const FrameCtx& f, size_t set, const std::vector<LrRect>& rects,
                                                    int32_t x0, size_t w, const PlaneBuf& src, size_t step,
                                                    LrBuffers& buf) {
  const int32_t r0 = SGR_PARAMS[set][0], r1 = SGR_PARAMS[set][2];
  double m[2][2] = {{0, 0}, {0, 0}}, v[2] = {0, 0};
  std::vector<std::array<std::vector<int32_t>, 2>> flts;
  for (const LrRect& rc : rects) {
    lr_window(rc.ctx, x0, rc.y0, w, rc.h, buf);
    for (size_t pass = 0; pass < 2; pass++) box_filter_rect(f, rc.ctx, x0, rc.y0, w, rc.h, set, pass, buf);
    flts.push_back({buf.flt[0], buf.flt[1]});
    for (size_t i = 0; i < rc.h; i += step) {
      const uint16_t* srow = src.row(size_t(rc.y0) + i) + x0;
      for (size_t j = 0; j < w; j += step) {
        double u = double(int32_t(rc.ctx.cdef->get(size_t(x0) + j, size_t(rc.y0) + i)) << SGRPROJ_RST_BITS);
        double a = r0 != 0 ? double(buf.flt[0][i * w + j]) - u : 0.0;
        double b = r1 != 0 ? double(buf.flt[1][i * w + j]) - u : 0.0;
        double t = 128.0 * (double(int32_t(srow[j]) << SGRPROJ_RST_BITS) - u);
        m[0][0] += a * a;
        m[0][1] += a * b;
        m[1][1] += b * b;
        v[0] += a * t;
        v[1] += b * t;
      }
    }
  }
  m[1][0] = m[0][1];
  double w0, w2;
  if (r0 != 0 && r1 != 0) {
    std::array<double, 2> s2 = lr_solve<2>({{{m[0][0], m[0][1]}, {m[1][0], m[1][1]}}}, {v[0], v[1]});
    w0 = s2[0];
    w2 = s2[1];
  } else if (r0 != 0) {
    w0 = m[0][0] > 0.0 ? v[0] / m[0][0] : 0.0;
    w2 = 0.0;
  } else {
    w0 = 0.0;
    w2 = m[1][1] > 0.0 ? v[1] / m[1][1] : 0.0;
  }
  int32_t x0q = r0 != 0 ? iclamp(f64_to_i32(std::round(w0)), SGRPROJ_XQD_MIN_T[0], SGRPROJ_XQD_MAX_T[0]) : 0;
  int32_t x1q;
  if (r1 != 0) {
    // i32 arithmetic wraps as the reference's release build does
    int32_t diff = int32_t(uint32_t(1 << SGRPROJ_PRJ_BITS) - uint32_t(x0q) - uint32_t(f64_to_i32(std::round(w2))));
    x1q = iclamp(diff, SGRPROJ_XQD_MIN_T[1], SGRPROJ_XQD_MAX_T[1]);
  } else {
    x1q = iclamp((1 << SGRPROJ_PRJ_BITS) - x0q, SGRPROJ_XQD_MIN_T[1], SGRPROJ_XQD_MAX_T[1]);
  }
  const int32_t pw0 = x0q, pw1 = x1q, pw2 = (1 << SGRPROJ_PRJ_BITS) - pw0 - pw1;
  const int32_t maxv = (1 << f.bit_depth) - 1;
  uint64_t sse = 0;
  for (size_t ri = 0; ri < rects.size(); ri++) {
    const LrRect& rc = rects[ri];
    for (size_t i = 0; i < rc.h; i++) {
      const uint16_t* srow = src.row(size_t(rc.y0) + i) + x0;
      for (size_t j = 0; j < w; j++) {
        int32_t u = int32_t(rc.ctx.cdef->get(size_t(x0) + j, size_t(rc.y0) + i)) << SGRPROJ_RST_BITS;
        int32_t val = pw1 * u;
        val += r0 != 0 ? pw0 * flts[ri][0][i * w + j] : pw0 * u;
        val += r1 != 0 ? pw2 * flts[ri][1][i * w + j] : pw2 * u;
        int32_t out = iclamp(round2(val, unsigned(SGRPROJ_RST_BITS + SGRPROJ_PRJ_BITS)), 0, maxv);
        int64_t d = int64_t(out) - int64_t(srow[j]);
        sse += uint64_t(d * d);
      }
    }
  }
  return {{x0q, x1q}, sse};
}

struct LrChoice {  // encoder/lr.rs:22-29
  uint8_t t = RESTORE_NONE;
  std::array<std::array<int32_t, 3>, 2> wiener{};
  uint8_t set = 0;
  std::array<int32_t, 2> xqd{};
};

// encoder/lr.rs:64-210 `search`: each unit's restoration and each plane's
// frame restoration type. `f.lr` holds the unit grid, `cur` the deblocked
// frame, `cdefb` the CDEF output.
void lr_search(const FrameCtx& f, const FrameBuf& cur, const FrameBuf& cdefb, const FrameBuf& src, double lambda,
               int effort, size_t threads, std::vector<LrChoice> units[3], uint8_t frame_type[3]) {
  static const size_t kNormal[6] = {0, 3, 6, 10, 13, 14}, kFast[2] = {3, 10};
  std::vector<size_t> sets;
  if (effort == 2)
    for (size_t k = 0; k < 16; k++) sets.push_back(k);
  else if (effort == 1)
    sets.assign(kNormal, kNormal + 6);
  else
    sets.assign(kFast, kFast + 2);
  const size_t step = effort == 0 ? 2 : 1;
  const size_t stripes = (size_t(f.hdr.frame_height) + 8 + 63) / 64;
  struct Stripe {
    int32_t ss, se, y0, y1;
  };
  std::vector<std::vector<Stripe>> rows[3];
  struct Job {
    size_t plane, ur, uc;
  };
  std::vector<Job> jobs;
  for (size_t plane = 0; plane < f.num_planes; plane++) {
    const LrPlane& lp = f.lr[plane];
    rows[plane].assign(lp.unit_rows, {});
    for (size_t s = 0; s < stripes; s++) {
      int32_t ss, se, y0, y1;
      size_t ur;
      if (lr_stripe(f, plane, s, ss, se, y0, y1, ur)) rows[plane][ur].push_back({ss, se, y0, y1});
    }
    for (size_t ur = 0; ur < lp.unit_rows; ur++)
      for (size_t uc = 0; uc < lp.unit_cols; uc++) jobs.push_back({plane, ur, uc});
  }
  std::vector<LrChoice> results(jobs.size());
  std::vector<uint8_t> present(jobs.size(), 0);
  auto unit = [&](size_t ji) {
    const Job& jb = jobs[ji];
    const size_t plane = jb.plane;
    auto ssv = f.plane_ss(plane);
    const int32_t plane_end_x = round2(f.hdr.upscaled_width, unsigned(ssv.first)) - 1;
    const int32_t plane_end_y = round2(f.hdr.frame_height, unsigned(ssv.second)) - 1;
    auto xr = lr_unit_cols(f, plane, jb.uc);
    const int32_t x0 = xr.first, x1 = xr.second;
    if (x0 > plane_end_x || rows[plane][jb.ur].empty()) return;
    LrBuffers buf;
    const size_t w = size_t(x1 - x0 + 1);
    std::vector<LrRect> rects;
    for (const Stripe& st : rows[plane][jb.ur])
      rects.push_back({LrCtx{&cur.planes[plane], &cdefb.planes[plane], st.ss, st.se, plane_end_x, plane_end_y}, st.y0,
                       size_t(st.y1 - st.y0 + 1)});
    const PlaneBuf& sp = src.planes[plane];
    auto sse_of = [&](const LrParams* prm) {
      uint64_t total = 0;
      for (const LrRect& rc : rects) {
        if (prm) {
          lr_window(rc.ctx, x0, rc.y0, w, rc.h, buf);
          restore_rect_from_window(f, rc.ctx, x0, rc.y0, w, rc.h, *prm, buf);
        }
        for (size_t i = 0; i < rc.h; i++) {
          const size_t y = size_t(rc.y0) + i;
          const uint16_t* srow = sp.row(y) + x0;
          for (size_t j = 0; j < w; j++) {
            int64_t val = prm ? int64_t(buf.out[i * w + j]) : int64_t(rc.ctx.cdef->get(size_t(x0) + j, y));
            int64_t d = val - int64_t(srow[j]);
            total += uint64_t(d * d);
          }
        }
      }
      return total;
    };
    const uint64_t none = sse_of(nullptr);
    double best_cost = double(none) + lambda;
    LrChoice best{};
    auto coef = fit_wiener(plane, rects, x0, w, sp, step, buf);
    LrParams pw{};
    pw.wiener = true;
    pw.coef = coef;
    double cost = double(sse_of(&pw)) + lambda * (plane == 0 ? 40.0 : 28.0);
    if (cost < best_cost) {
      best_cost = cost;
      best = LrChoice{};
      best.t = RESTORE_WIENER;
      best.wiener = coef;
    }
    for (size_t set : sets) {
      auto fit = fit_sgr(f, set, rects, x0, w, sp, step, buf);
      cost = double(fit.second) + lambda * 20.0;
      if (cost < best_cost) {
        best_cost = cost;
        best = LrChoice{};
        best.t = RESTORE_SGRPROJ;
        best.set = uint8_t(set);
        best.xqd = fit.first;
      }
    }
    results[ji] = best;
    present[ji] = 1;
  };
  run_bands(jobs.size(), threads, unit);
  for (size_t plane = 0; plane < f.num_planes; plane++)
    units[plane].assign(f.lr[plane].unit_rows * f.lr[plane].unit_cols, LrChoice{});
  for (size_t ji = 0; ji < jobs.size(); ji++)
    if (present[ji]) units[jobs[ji].plane][jobs[ji].ur * f.lr[jobs[ji].plane].unit_cols + jobs[ji].uc] = results[ji];
  for (size_t plane = 0; plane < f.num_planes; plane++) {
    bool wu = false, su = false;
    for (const LrChoice& c : units[plane]) {
      wu |= c.t == RESTORE_WIENER;
      su |= c.t == RESTORE_SGRPROJ;
    }
    frame_type[plane] = wu ? (su ? 3 : RESTORE_WIENER) : (su ? RESTORE_SGRPROJ : RESTORE_NONE);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int oracle_loop_filter(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
                       av1pf_plane* planes, int threads) {
  if (!info_ok(info) || !p || !maps || !planes) return AV1PF_ERR_INVALID_INPUT;
  FrameCtx f;
  ctx_from(f, info, p, maps, planes);
  loop_filter_threads(f, resolve_threads(threads));
  frame_to(f.cur, info, planes, false);
  return AV1PF_OK;
}

int oracle_cdef(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
                const av1pf_plane* cur, av1pf_plane* out, int threads) {
  if (!info_ok(info) || !p || !maps || !cur || !out) return AV1PF_ERR_INVALID_INPUT;
  FrameCtx f;
  ctx_from(f, info, p, maps, cur);
  FrameBuf o = cdef(f, resolve_threads(threads));
  frame_to(o, info, out, false);
  return AV1PF_OK;
}

int oracle_superres(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_plane* in,
                    av1pf_plane* out) {
  if (!info_ok(info) || !p || !in || !out) return AV1PF_ERR_INVALID_INPUT;
  FrameCtx f;
  ctx_from(f, info, p, nullptr, nullptr);
  FrameBuf src = frame_from(info, in), dst;
  if (!upscale(f, src, dst)) return AV1PF_ERR_INVALID_INPUT;
  for (int pl = 0; pl < info->num_planes; pl++) {
    size_t sx = pl ? size_t(info->subsampling_x) : 0, sy = pl ? size_t(info->subsampling_y) : 0;
    plane_to(dst.planes[size_t(pl)], out[pl], info->sample_bytes, size_t(round2(info->upscaled_width, unsigned(sx))),
             size_t(round2(info->frame_height, unsigned(sy))));
  }
  return AV1PF_OK;
}

int oracle_loop_restoration(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
                            const av1pf_plane* cur, const av1pf_plane* cdefp, av1pf_plane* out, int threads) {
  if (!info_ok(info) || !p || !maps || !cur || !cdefp || !out) return AV1PF_ERR_INVALID_INPUT;
  FrameCtx f;
  ctx_from(f, info, p, maps, nullptr);
  FrameBuf c = frame_from(info, cur), d = frame_from(info, cdefp);
  FrameBuf lr = loop_restoration(f, c, d, resolve_threads(threads));
  frame_to(lr, info, out, true);
  return AV1PF_OK;
}

int oracle_output(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_plane* ref,
                  uint8_t* frame_out) {
  if (!info_ok(info) || !p || !ref || !frame_out) return AV1PF_ERR_INVALID_INPUT;
  FrameBuf fb = frame_from(info, ref);
  output(info, p, fb, frame_out);
  return AV1PF_OK;
}

int oracle_chain(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
                 const av1pf_plane* in, av1pf_plane* ref_out, uint8_t* frame_out, int threads) {
  if (!info_ok(info) || !p || !maps || !in) return AV1PF_ERR_INVALID_INPUT;
  size_t th = resolve_threads(threads);
  FrameCtx f;
  ctx_from(f, info, p, maps, in);
  // decoder/mod.rs:748-759
  if (f.hdr.loop_filter_level[0] != 0 || f.hdr.loop_filter_level[1] != 0) loop_filter_threads(f, th);
  FrameBuf cd = cdef(f, th);
  FrameBuf up_cdef, up_cur;
  const FrameBuf* ucd = upscale(f, cd, up_cdef) ? &up_cdef : &cd;
  const FrameBuf* ucur = upscale(f, f.cur, up_cur) ? &up_cur : &f.cur;
  FrameBuf lr = loop_restoration(f, *ucur, *ucd, th);
  if (ref_out) frame_to(lr, info, ref_out, true);
  if (frame_out) output(info, p, lr, frame_out);
  return AV1PF_OK;
}

void oracle_lf_filter_lanes(int32_t* edges, const av1pf_lf_edge_params* p, int n) {
  for (int e = 0; e < n; e++) {
    Edge v;
    std::memcpy(v, edges + size_t(e) * 56, sizeof(v));
    filter_lanes(v, lf_params_from(p[e]));
    std::memcpy(edges + size_t(e) * 56, v, sizeof(v));
  }
}

void oracle_lf_reference(int32_t* edges, const av1pf_lf_edge_params* p, int n) {
  for (int e = 0; e < n; e++) {
    int32_t* v = edges + size_t(e) * 56;
    for (int l = 0; l < 4; l++) {
      int32_t one[14];
      for (int k = 0; k < 14; k++) one[k] = v[k * 4 + l];
      lf_reference_one(one, lf_params_from(p[e]));
      for (int k = 0; k < 14; k++) v[k * 4 + l] = one[k];
    }
  }
}

// lf.rs:309-353 `lanes_match_the_process`: the cases.
void oracle_lf_kat_cases(uint64_t seed, int cases, int32_t* edges, av1pf_lf_edge_params* params) {
  XorShift rnd{seed};
  for (int c = 0; c < cases; c++) {
    size_t cs = size_t(c);
    int32_t bd = int32_t(std::array<uint32_t, 3>{8, 10, 12}[cs % 3]);
    av1pf_lf_edge_params pr{};
    pr.limit = 1 + int32_t(rnd(9));
    pr.blimit = int32_t(rnd(130));
    pr.thresh = int32_t(rnd(4));
    int32_t sizes[4] = {4, 8, 16, 6};
    pr.filter_size = std::min(sizes[rnd(4)], cs % 5 == 0 ? 8 : 16);
    pr.chroma = cs % 5 == 0;
    pr.bit_depth = bd;
    if (pr.chroma) pr.filter_size = std::min(pr.filter_size, 8);
    int32_t base = int32_t(rnd(uint64_t(1) << bd));
    uint64_t spreads[4] = {1, 4, 16, 64};
    uint64_t spread = spreads[rnd(4)] << (bd - 8);
    int32_t* v = edges + cs * 56;
    for (int k = 0; k < 14; k++)
      for (int l = 0; l < 4; l++)
        v[k * 4 + l] = iclamp(base + int32_t(rnd(spread)) - int32_t(spread / 2), 0, (1 << bd) - 1);
    params[c] = pr;
  }
}

void oracle_cdef_filter(const int32_t* win, const av1pf_cdef_taps* taps, uint16_t* res, int n) {
  for (int e = 0; e < n; e++) {
    const av1pf_cdef_taps& a = taps[e];
    Taps t;
    t.pri_str = a.pri_str;
    t.sec_str = a.sec_str;
    t.pri_adj = a.pri_adj;
    t.sec_adj = a.sec_adj;
    for (int k = 0; k < 2; k++) {
      t.pri_taps[k] = a.pri_taps[k];
      t.sec_taps[k] = a.sec_taps[k];
      t.pri_off[k] = a.pri_off[k];
      for (int s = 0; s < 2; s++) t.sec_off[k][s] = a.sec_off[k][s];
    }
    uint16_t out[64] = {};
    cdef_filter_scalar(win + size_t(e) * 144, size_t(a.w), size_t(a.h), t, out);
    std::memcpy(res + size_t(e) * 64, out, sizeof(out));
  }
}

// cdef.rs:250-311 `simd_matches_scalar`: the cases (each window x 3 shapes).
void oracle_cdef_kat_cases(uint64_t seed, int cases, int32_t* win, av1pf_cdef_taps* taps) {
  XorShift rnd{seed};
  const int shapes[3][2] = {{8, 8}, {4, 4}, {4, 8}};
  for (int c = 0; c < cases; c++) {
    int32_t bd = c % 2 == 0 ? 8 : 10;
    int32_t w[144];
    int32_t base = int32_t(rnd(uint64_t(1) << bd));
    for (auto& v : w) {
      v = iclamp(base + int32_t(rnd(64)) - 32, 0, (1 << bd) - 1);
      if (rnd(9) == 0) v = int32_t(rnd(uint64_t(1) << bd));
    }
    switch (rnd(5)) {
      case 0:
        for (size_t i = 0; i < 2 * WS; i++) w[i] = NA;
        break;
      case 1:
        for (size_t r = 0; r < WS; r++) w[r * WS + WS - 1] = NA;
        break;
      default:
        break;
    }
    int32_t shift = bd - 8;
    int32_t pri_str = int32_t(rnd(16)) << shift;
    int32_t secs[4] = {0, 1, 2, 4};
    int32_t sec_str = secs[rnd(4)] << shift;
    int32_t damping = 3 + int32_t(rnd(4)) + shift;
    size_t dir = size_t(rnd(8));
    auto off = [&](size_t d, size_t k) {
      return int32_t(CDEF_DIRECTIONS[d][k][0]) * int32_t(WS) + int32_t(CDEF_DIRECTIONS[d][k][1]);
    };
    auto adj = [&](int32_t s) { return s != 0 ? std::max(damping - int32_t(floor_log2(uint32_t(s))), 0) : 0; };
    av1pf_cdef_taps t{};
    t.pri_str = pri_str;
    t.sec_str = sec_str;
    t.pri_adj = adj(pri_str);
    t.sec_adj = adj(sec_str);
    size_t tsel = size_t((pri_str >> shift) & 1);
    for (int k = 0; k < 2; k++) {
      t.pri_taps[k] = CDEF_PRI_TAPS[tsel][k];
      t.sec_taps[k] = CDEF_SEC_TAPS[tsel][k];
    }
    t.pri_off[0] = off(dir, 0);
    t.pri_off[1] = off(dir, 1);
    t.sec_off[0][0] = off((dir + 6) & 7, 0);
    t.sec_off[0][1] = off((dir + 2) & 7, 0);
    t.sec_off[1][0] = off((dir + 6) & 7, 1);
    t.sec_off[1][1] = off((dir + 2) & 7, 1);
    for (int s = 0; s < 3; s++) {
      size_t e = size_t(c) * 3 + size_t(s);
      std::memcpy(win + e * 144, w, sizeof(w));
      t.w = shapes[s][0];
      t.h = shapes[s][1];
      taps[e] = t;
    }
  }
}

int oracle_cdef_search(const av1pf_frame_info* info, const av1pf_maps* maps, const av1pf_plane* cur,
                       const av1pf_plane* src, int32_t base_q_idx, double lambda, int32_t thorough,
                       av1pf_cdef_search_result* result, int8_t* cdef_idx_out, uint64_t* block_sse, int threads) {
  if (!info_ok(info) || !maps || !maps->mi || !maps->cdef_idx || !cur || !src || !result || base_q_idx < 0)
    return AV1PF_ERR_INVALID_INPUT;
  FrameCtx f;
  ctx_from(f, info, nullptr, maps, cur);
  FrameBuf s = frame_from(info, src);
  CdefSearch o = cdef_search(f, s, uint32_t(base_q_idx), lambda, thorough != 0, resolve_threads(threads));
  std::memset(result, 0, sizeof(*result));
  result->damping_minus_3 = int32_t(o.damping_minus_3);
  result->bits = int32_t(o.bits);
  for (size_t i = 0; i < o.y.size(); i++) {
    result->y_pri[i] = int32_t(o.y[i].first);
    result->y_sec[i] = int32_t(o.y[i].second);
    result->uv_pri[i] = int32_t(o.uv[i].first);
    result->uv_sec[i] = int32_t(o.uv[i].second);
  }
  const size_t fb_rows = (f.mi_rows + 15) / 16, fb_cols = (f.mi_cols + 15) / 16;
  if (cdef_idx_out) std::memcpy(cdef_idx_out, o.table.data(), fb_rows * f.cdef_stride);
  if (block_sse) {
    const size_t nc = o.ny + o.nuv;
    std::memset(block_sse, 0, fb_rows * fb_cols * nc * sizeof(uint64_t));
    for (size_t b = 0; b < o.blocks.size(); b++) {
      uint64_t* row = block_sse + (o.blocks[b].first * fb_cols + o.blocks[b].second) * nc;
      std::memcpy(row, &o.ysse[b * o.ny], o.ny * sizeof(uint64_t));
      std::memcpy(row + o.ny, &o.uvsse[b * o.nuv], o.nuv * sizeof(uint64_t));
    }
  }
  return AV1PF_OK;
}

int oracle_lf_search(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_maps* maps,
                     const av1pf_plane* cur, const av1pf_plane* src, int32_t levels_out[4], uint64_t* sse_out,
                     int threads) {
  if (!info_ok(info) || !p || !maps || !cur || !src || !levels_out) return AV1PF_ERR_INVALID_INPUT;
  std::array<uint32_t, 4> start;
  for (int i = 0; i < 4; i++) {
    if (p->loop_filter_level[i] < 0 || p->loop_filter_level[i] > 63) return AV1PF_ERR_INVALID_INPUT;
    start[size_t(i)] = uint32_t(p->loop_filter_level[i]);
  }
  FrameCtx f;
  ctx_from(f, info, p, maps, cur);
  FrameBuf s = frame_from(info, src);
  if (sse_out) std::memset(sse_out, 0, 6 * 3 * sizeof(uint64_t));
  std::array<uint32_t, 4> lv = search_lf(f, s, start, resolve_threads(threads), sse_out);
  for (int i = 0; i < 4; i++) levels_out[i] = int32_t(lv[size_t(i)]);
  return AV1PF_OK;
}

int oracle_lr_search(const av1pf_frame_info* info, const av1pf_params* p, const av1pf_plane* cur,
                     const av1pf_plane* cdefp, const av1pf_plane* src, double lambda, int32_t effort,
                     av1pf_lr_unit* const units_out[3], int32_t frame_type_out[3], int threads) {
  if (!info_ok(info) || !p || !cur || !cdefp || !src || !units_out || !frame_type_out || effort < 0 || effort > 2)
    return AV1PF_ERR_INVALID_INPUT;
  av1pf_params q = *p;
  q.uses_lr = 1;
  for (int k = 0; k < 3; k++) q.frame_restoration_type[k] = 3;
  av1pf_maps none{};
  FrameCtx f;
  ctx_from(f, info, &q, &none, nullptr);
  FrameBuf c = frame_from(info, cur), d = frame_from(info, cdefp), s = frame_from(info, src);
  std::vector<LrChoice> units[3];
  uint8_t ft[3] = {0, 0, 0};
  lr_search(f, c, d, s, lambda, effort, resolve_threads(threads), units, ft);
  for (size_t pl = 0; pl < 3; pl++) {
    frame_type_out[pl] = pl < f.num_planes ? ft[pl] : 0;
    if (pl >= f.num_planes || !units_out[pl]) continue;
    for (size_t i = 0; i < units[pl].size(); i++) {
      const LrChoice& ch = units[pl][i];
      av1pf_lr_unit& u = units_out[pl][i];
      std::memset(&u, 0, sizeof(u));
      u.type = ch.t;
      u.sgr_set = ch.set;
      u.sgr_xqd[0] = int8_t(ch.xqd[0]);
      u.sgr_xqd[1] = int8_t(ch.xqd[1]);
      for (int a = 0; a < 2; a++)
        for (int b = 0; b < 3; b++) u.wiener[a][b] = int8_t(ch.wiener[size_t(a)][size_t(b)]);
    }
  }
  return AV1PF_OK;
}

}  // extern "C"
