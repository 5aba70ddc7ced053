// lr.cu — loop restoration (7.17): Wiener and self-guided filters.
//
// Reference: rivet-av1 src/decoder/postfilter.rs:568-1004 (LrCtx::sample,
// loop_restoration, lr_stripe, lr_unit_cols, restore_stripe, lr_window,
// restore_rect_from_window, box_filter_rect, wiener_coefficient).
//
// One CTA restores one rectangle: the rows of one stripe (64 luma rows,
// offset by 8) and up to 64 columns of one restoration unit. 288 threads are
// 4 row groups x 72 columns (8 x 36 for rectangles of up to 32 columns, as
// 4:2:0 chroma units are), so every thread owns a column and no loop
// divides by a runtime width. The window the rectangle reads (3-sample
// border, the stripe-boundary rule of LrCtx::sample) is staged in shared
// memory with one row-uniform source choice per row. Wiener runs its
// horizontal pass into an int16 intermediate, then the vertical pass. The
// self-guided filter slides each column's box sums down its rows (one new
// and one old row of horizontal sums per step), then walks each column's
// output rows with three rows of A and B in registers. The sums are exact in
// 32 bits for <= 12-bit samples (25 * 4095^2 < 2^31); the products the
// reference forms in 64 bits (p * s and the B term) are 32x32->64 multiplies
// here. Rectangles of
// units without restoration (and planes or frames without it) pass their
// samples through, so the kernel writes the whole visible area of the
// reference frame. Every rectangle's output gathers in a shared-memory tile
// and leaves in 16-byte row chunks: to the reference frame and, for a frame
// without film grain, to the packed output frame too, so such a frame needs
// no output pass.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {
constexpr int kThreads = 288;
constexpr int kMaxW = 64;                // columns per rectangle
constexpr int kMaxH = 64;                // rows per stripe
constexpr int kWS = 72;                  // window row stride (u16): w + 6 <= 70
constexpr int kAS = 72;                  // A/B row stride (int32): w + 2 <= 66
constexpr int kWinBytes = (kMaxH + 6) * kWS * 2;
constexpr int kABytes = (kMaxH + 2) * kAS * 4;
constexpr int kF0Bytes = kMaxH * kMaxW * 4;  // the first self-guided filter's output
constexpr int kSmemBytes = kWinBytes + 2 * kABytes + kF0Bytes;
static_assert((kMaxH + 6) * kWS * 2 <= kABytes, "Wiener intermediate must fit the A area");

// SGR_A2 (postfilter.rs:884-898), built at compile time into global memory:
// the self-guided passes read it through the L1, so no CTA sets it up.
struct A2Table {
  int32_t v[256];
};
constexpr A2Table make_a2() {
  A2Table t{};
  for (int z = 0; z < 256; z++) t.v[z] = z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
  return t;
}
}  // namespace

__device__ const A2Table g_sgr_a2 = make_a2();

struct LrGeom {
  int ss, se, y0, y1, pex, pey;
};

// The three sources LrCtx::sample (postfilter.rs:584-596) draws rows from,
// read once per rectangle: the upscaled CDEF plane, the loop-filtered plane
// and (with superres) the line buffer of upscaled pre-CDEF rows.
struct LrSrc {
  const uint8_t* up;
  const uint8_t* cur;
  const uint8_t* lines;
  int32_t up_pitch, cur_pitch, lines_pitch;  // bytes
  bool sr;  // the pre-CDEF rows come from `lines` (4 per stripe boundary), not `cur`
};

// The row LrCtx::sample reads for window row y of stripe `s`. With superres
// (or with the loop filter's horizontal pass run inside the CDEF kernel) the
// pre-CDEF rows come from a line buffer, 4 rows per stripe boundary:
// boundary b (the first row B of stripe b) holds rows B-2 .. B+1 at line
// rows (b-1)*4 ...
__device__ __forceinline__ const uint8_t* lr_row(const LrSrc& src, const LrGeom& g, int s, int y) {
  y = max(min(y, g.pey), 0);
  if (y < g.ss) {
    const int yy = max(g.ss - 2, y);
    return src.sr ? src.lines + int64_t((s - 1) * 4 + (yy - (g.ss - 2))) * src.lines_pitch
                  : src.cur + int64_t(yy) * src.cur_pitch;
  }
  if (y > g.se) {
    const int yy = min(g.se + 2, y);
    return src.sr ? src.lines + int64_t(s * 4 + (yy - (g.se - 1))) * src.lines_pitch
                  : src.cur + int64_t(yy) * src.cur_pitch;
  }
  return src.up + int64_t(y) * src.up_pitch;
}

__device__ __forceinline__ int ld_row(const uint8_t* row, int sb, int x) {
  return sb == 1 ? int(row[x]) : int(reinterpret_cast<const uint16_t*>(row)[x]);
}

// Reads the w x h samples at (x0, y0) of `src` (sample width sb) into `tile`
// (int32, row stride kMaxW): 16-byte chunks where the rows allow them, else
// single samples. Rows hold MW >> cs chunk slots (w <= MW).
template <int MW>
__device__ __forceinline__ void load_tile(const DPlane& src, int sb, int x0, int y0, int w, int h, int32_t* tile,
                                          int tid) {
  const uint8_t* s0 = src.p + (int64_t(y0) * src.stride + x0) * sb;
  const int64_t sp = src.stride * sb;
  const bool vec = ((reinterpret_cast<uintptr_t>(s0) | uintptr_t(sp)) & 15) == 0;
  const int cs = sb == 2 ? 3 : 4;                  // log2 samples per chunk
  const int ls = (MW == 64 ? 6 : 5) - cs;          // log2 chunk slots per row
  for (int k = tid; k < (h << ls); k += kThreads) {
    const int r = k >> ls, e0 = (k & ((1 << ls) - 1)) << cs;
    if (e0 >= w) continue;
    const uint8_t* row = s0 + int64_t(r) * sp;
    int32_t* t = tile + r * kMaxW + e0;
    if (vec && e0 + (1 << cs) <= w) {
      const uint4 q = *reinterpret_cast<const uint4*>(row + e0 * sb);
      if (sb == 2) {
        reinterpret_cast<int4*>(t)[0] = make_int4(q.x & 0xffff, q.x >> 16, q.y & 0xffff, q.y >> 16);
        reinterpret_cast<int4*>(t)[1] = make_int4(q.z & 0xffff, q.z >> 16, q.w & 0xffff, q.w >> 16);
      } else {
        const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; j++)
          reinterpret_cast<int4*>(t)[j] =
              make_int4(wd[j] & 0xff, (wd[j] >> 8) & 0xff, (wd[j] >> 16) & 0xff, wd[j] >> 24);
      }
    } else {
      for (int e = e0; e < min(w, e0 + (1 << cs)); e++) t[e - e0] = ld_row(row, sb, e);
    }
  }
}

// Writes the w x h output samples of `tile` (int32, row stride kMaxW) to
// rows of `width`-byte samples from `base`, `pitch` bytes apart: 16-byte
// chunks (8 or 16 samples) where `vec` says the rows allow them, else single
// samples. Rows hold MW >> cs chunk slots (w <= MW).
template <int MW>
__device__ __forceinline__ void store_tile(const int32_t* tile, uint8_t* base, int64_t pitch, int width, bool vec,
                                           int w, int h, int tid) {
  const int cs = width == 2 ? 3 : 4;      // log2 samples per chunk
  const int ls = (MW == 64 ? 6 : 5) - cs;  // log2 chunk slots per row
  for (int k = tid; k < (h << ls); k += kThreads) {
    const int r = k >> ls, e0 = (k & ((1 << ls) - 1)) << cs;
    if (e0 >= w) continue;
    const int32_t* t = tile + r * kMaxW + e0;
    uint8_t* row = base + int64_t(r) * pitch;
    if (vec && e0 + (1 << cs) <= w) {
      const int4 a = *reinterpret_cast<const int4*>(t);
      const int4 b = *reinterpret_cast<const int4*>(t + 4);
      uint4 q;
      if (width == 2) {
        q.x = uint32_t(a.x) | (uint32_t(a.y) << 16);
        q.y = uint32_t(a.z) | (uint32_t(a.w) << 16);
        q.z = uint32_t(b.x) | (uint32_t(b.y) << 16);
        q.w = uint32_t(b.z) | (uint32_t(b.w) << 16);
      } else {
        const int4 c = *reinterpret_cast<const int4*>(t + 8);
        const int4 d = *reinterpret_cast<const int4*>(t + 12);
        q.x = uint32_t(a.x) | (uint32_t(a.y) << 8) | (uint32_t(a.z) << 16) | (uint32_t(a.w) << 24);
        q.y = uint32_t(b.x) | (uint32_t(b.y) << 8) | (uint32_t(b.z) << 16) | (uint32_t(b.w) << 24);
        q.z = uint32_t(c.x) | (uint32_t(c.y) << 8) | (uint32_t(c.z) << 16) | (uint32_t(c.w) << 24);
        q.w = uint32_t(d.x) | (uint32_t(d.y) << 8) | (uint32_t(d.z) << 16) | (uint32_t(d.w) << 24);
      }
      *reinterpret_cast<uint4*>(row + e0 * width) = q;
    } else {
      for (int e = e0; e < min(w, e0 + (1 << cs)); e++) {
        if (width == 2)
          reinterpret_cast<uint16_t*>(row)[e] = uint16_t(t[e - e0]);
        else
          row[e] = uint8_t(t[e - e0]);
      }
    }
  }
}

// Box sums of radius R over the window and the A / B of box_filter_rect
// (postfilter.rs:935-959) for positions (i, j), i in [0, h+2), j = c - 1,
// stored at [i][c]. Each of the G row groups owns a contiguous run of rows
// and slides down it.
template <int PASS, int G>
__device__ __forceinline__ void sgr_ab(const uint16_t* win, int32_t* A, int32_t* B, const int32_t* a2tab, int eps,
                                       int bd, int y0, int h, int w, int c, int g) {
  constexpr int R = PASS == 0 ? 2 : 1;  // SGR_PARAMS radii: first 0 or 2, second 0 or 1
  constexpr int n = (2 * R + 1) * (2 * R + 1);
  const int n2e = n * n * eps;
  const uint32_t sc = uint32_t(((1 << 20) + n2e / 2) / n2e);
  constexpr int one_over_n = ((1 << 12) + n / 2) / n;
  if (c >= w + 2) return;
  const int rows = h + 2;
  const int rpg = (rows + G - 1) / G;
  const int i0 = g * rpg, i1 = min(i0 + rpg, rows);
  if (i0 >= i1) return;
  // horizontal sums of window row wr around column c + 2
  auto hs = [&](int wr, int& s1, int& s2) {
    s1 = 0;
    s2 = 0;
    const uint16_t* rp = win + wr * kWS + c + 2;
#pragma unroll
    for (int dx = -R; dx <= R; dx++) {
      const int v = rp[dx];
      s1 += v;
      s2 += v * v;
    }
  };
  // ring of the horizontal sums of the 2R+1 rows in the box: the row that
  // enters at step i goes to slot (i - i0 + 2R) mod N, the row that leaves
  // is in slot (i - i0) mod N; unrolling by N makes the slots constants
  constexpr int N = 2 * R + 1;
  int r1[N], r2[N];
  int bsum = 0, bsq = 0;
#pragma unroll
  for (int m = 0; m < 2 * R; m++) {
    hs(i0 + 2 - R + m, r1[m], r2[m]);
    bsum += r1[m];
    bsq += r2[m];
  }
  for (int ib = i0; ib < i1; ib += N) {
#pragma unroll
    for (int u = 0; u < N; u++) {
      const int i = ib + u;
      if (i < i1) {
        const int sn = (u + 2 * R) % N;
        hs(i + 2 + R, r1[sn], r2[sn]);
        bsum += r1[sn];
        bsq += r2[sn];
        // the first filter weighs only the odd rows' A and B (postfilter.rs:937)
        if (PASS == 1 || ((y0 + i - 1) & 1) != 0) {
          const int a = round2(bsq, 2 * (bd - 8));
          const int d = round2(bsum, bd - 8);
          const int pp = max(a * n - d * d, 0);
          const uint64_t z = (uint64_t(uint32_t(pp)) * sc + (1u << 19)) >> 20;
          const int a2 = __ldg(a2tab + (z > 255 ? 255 : int(z)));
          const uint32_t k = uint32_t(256 - a2) * uint32_t(one_over_n);
          const uint64_t b2 = uint64_t(k) * uint32_t(bsum);
          A[i * kAS + c] = a2;
          B[i * kAS + c] = int32_t((b2 + (1u << 11)) >> 12);
        }
        bsum -= r1[u];
        bsq -= r2[u];
      }
    }
  }
}

// The self-guided filter's value at rows [i0, i1) of column c
// (postfilter.rs:960-989), handed to emit(i, window sample, value). The walk
// down the column keeps the three A and B rows around row i in registers,
// each as its centre value and the sum of its left and right neighbours, so
// a row costs three loads of A and three of B.
template <int PASS, typename Emit>
__device__ __forceinline__ void sgr_flt_col(const int32_t* A, const int32_t* B, const uint16_t* win, int c, int i0,
                                            int i1, int y0, Emit emit) {
  const int32_t* pa = A + c + 1;
  const int32_t* pb = B + c + 1;
  auto row = [&](const int32_t* q, int& m, int& sum) {
    m = q[0];
    sum = q[-1] + q[1];
  };
  int am0, as0, am1, as1, bm0, bs0, bm1, bs1;
  row(pa + i0 * kAS, am0, as0);
  row(pb + i0 * kAS, bm0, bs0);
  row(pa + (i0 + 1) * kAS, am1, as1);
  row(pb + (i0 + 1) * kAS, bm1, bs1);
  for (int i = i0; i < i1; i++) {
    int am2, as2, bm2, bs2;
    row(pa + (i + 2) * kAS, am2, as2);
    row(pb + (i + 2) * kAS, bm2, bs2);
    const int cd = win[(i + 3) * kWS + c + 3];
    int a, b, shift;
    if (PASS == 0) {
      if ((y0 + i) & 1) {
        a = 6 * am1 + 5 * as1;
        b = 6 * bm1 + 5 * bs1;
        shift = 4;
      } else {
        a = 6 * (am0 + am2) + 5 * (as0 + as2);
        b = 6 * (bm0 + bm2) + 5 * (bs0 + bs2);
        shift = 5;
      }
    } else {
      a = 4 * (am1 + as1 + am0 + am2) + 3 * (as0 + as2);
      b = 4 * (bm1 + bs1 + bm0 + bm2) + 3 * (bs0 + bs2);
      shift = 5;
    }
    emit(i, cd, round2(a * cd + b, 8 + shift - 4));
    am0 = am1;
    as0 = as1;
    bm0 = bm1;
    bs0 = bs1;
    am1 = am2;
    as1 = as2;
    bm1 = bm2;
    bs1 = bs2;
  }
}

// A rectangle without restoration: its samples of the upscaled CDEF frame
// go straight to the reference frame and (frames without film grain) the
// packed frame, 8 samples per thread and step, with no shared-memory round
// trip and no barrier.
__device__ __noinline__ void pass_through(const FrameDesc& f, int p, int x0, int y0, int w, int h, int tid) {
  const int sb = f.sb, bps = f.bd > 8 ? 2 : 1;
  const DPlane src = f.up[p], dst = f.ref[p];
  const int pw = ((f.uw + plane_ssx(f, p)) >> plane_ssx(f, p));
  uint8_t* out = f.lr_pack ? f.frame_out + f.out_off[p] : nullptr;
  const int ng = (w + 7) >> 3;
  for (int k = tid; k < h * ng; k += kThreads) {
    const int r = k / ng, c = (k - r * ng) * 8;
    const int n = min(8, w - c);
    const int y = y0 + r, x = x0 + c;
    const uint8_t* sp = src.p + (int64_t(y) * src.stride + x) * sb;
    uint8_t* dp = dst.p + (int64_t(y) * dst.stride + x) * sb;
    uint8_t* op = out ? out + (int64_t(y) * pw + x) * bps : nullptr;
    uint32_t v[8];
    const bool sv = n == 8 && (reinterpret_cast<uintptr_t>(sp) & (8 * sb - 1)) == 0;
    if (sv && sb == 2) {
      const uint4 q = *reinterpret_cast<const uint4*>(sp);
      v[0] = q.x & 0xffffu; v[1] = q.x >> 16; v[2] = q.y & 0xffffu; v[3] = q.y >> 16;
      v[4] = q.z & 0xffffu; v[5] = q.z >> 16; v[6] = q.w & 0xffffu; v[7] = q.w >> 16;
    } else if (sv) {
      const uint2 q = *reinterpret_cast<const uint2*>(sp);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        v[e] = (q.x >> (8 * e)) & 0xffu;
        v[4 + e] = (q.y >> (8 * e)) & 0xffu;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 8; e++) v[e] = e < n ? uint32_t(ld_row(sp, sb, e)) : 0u;
    }
    auto put = [&](uint8_t* base, int width) {
      if (n == 8 && (reinterpret_cast<uintptr_t>(base) & (8 * width - 1)) == 0) {
        if (width == 2)
          *reinterpret_cast<uint4*>(base) =
              make_uint4(v[0] | (v[1] << 16), v[2] | (v[3] << 16), v[4] | (v[5] << 16), v[6] | (v[7] << 16));
        else
          *reinterpret_cast<uint2*>(base) = make_uint2(v[0] | (v[1] << 8) | (v[2] << 16) | (v[3] << 24),
                                                       v[4] | (v[5] << 8) | (v[6] << 16) | (v[7] << 24));
      } else {
        for (int e = 0; e < n; e++) {
          if (width == 2)
            reinterpret_cast<uint16_t*>(base)[e] = uint16_t(v[e]);
          else
            base[e] = uint8_t(v[e]);
        }
      }
    };
    put(dp, sb);
    if (op) put(op, bps);
  }
}

// The shared-memory areas of one CTA.
struct LrSmem {
  uint16_t* win;    // the window, rows kWS apart
  int32_t* A;       // self-guided A (Wiener: the int16 intermediate)
  int32_t* B;       // self-guided B
  const int32_t* a2tab;  // SGR_A2 (global memory)
  int32_t* F0;      // first self-guided output, then every rectangle's output
  av1pf_lr_unit* unit;
};

// Restores one rectangle of w <= MW columns into the output tile. CW is the
// width of a row group (threads per group: 72 for rectangles up to 64
// columns, 36 for those up to 32, so narrow rectangles keep most threads
// busy); the window is staged by groups SW threads wide.
template <int CW>
__device__ __forceinline__ void restore_rect(const FrameDesc& f, const LrSmem& sm, const LrGeom& geo, int p, int s,
                                             int x0, int w, int h, int type, const av1pf_lr_unit* unit_p, int tid) {
  constexpr int G = kThreads / CW;          // row groups
  constexpr int MW = CW == 72 ? 64 : 32;    // widest rectangle
  constexpr int SW = CW == 72 ? 72 : 48;    // staging group width (>= MW + 6)
  constexpr int SG = kThreads / SW;         // staging groups
  static_assert(G * CW == kThreads && SG * SW == kThreads, "layouts cover the CTA");
  const int g = tid / CW, c = tid - g * CW;
  const int sb = f.sb, bd = f.bd;
  const int maxv = (1 << bd) - 1;
  int32_t* F0 = sm.F0;
  if (type != AV1PF_RESTORE_WIENER && type != AV1PF_RESTORE_SGRPROJ) {
    // a unit without restoration passes its samples through
    load_tile<MW>(f.up[p], sb, x0, geo.y0, w, h, F0, tid);
    return;
  }
  uint16_t* win = sm.win;
  // the unit's coefficients wait in shared memory while the window loads
  if (tid == 0) *sm.unit = *unit_p;
  // lr_window (postfilter.rs:765-777): a thread's loads all issue before its stores
  const int ww = w + 6, wh = h + 6;
  {
    LrSrc src;
    src.up = f.up[p].p;
    src.cur = f.cur[p].p;
    // superres: upscaled boundary rows; fused horizontal LF pass: the
    // loop filter's boundary rows; else the loop-filtered plane itself
    const DPlane lines = f.sr_on ? f.lines[p] : f.prelf[p];
    src.lines = lines.p;
    src.up_pitch = int32_t(f.up[p].stride * sb);
    src.cur_pitch = int32_t(f.cur[p].stride * sb);
    src.lines_pitch = int32_t(lines.stride * sb);
    src.sr = f.sr_on != 0 || f.prelf[p].p != nullptr;
    // Window row r, columns 8q .. 8q+7 (samples x0-3+8q ..) per task. Where
    // the two aligned 8-sample chunks that hold them lie inside the plane
    // row (and the row is 16-byte aligned) they come as two vector loads
    // and are shifted into place; other chunks (the plane's left and right
    // edges) take one clamped scalar load per sample. The loads of two tasks
    // issue before their stores.
    const int nq = (ww + 7) >> 3;  // chunks per window row (<= 9)
    constexpr int kTasks = ((kMaxH + 6) * 9 + kThreads - 1) / kThreads;
    const int ntask = wh * nq;
    constexpr int kBatch = 2;  // tasks whose loads are in flight together
#pragma unroll
    for (int m0 = 0; m0 < kTasks; m0 += kBatch) {
      uint32_t wv[kBatch][5];  // the loaded words a window chunk is cut from
      bool vec[kBatch];
#pragma unroll
      for (int m = 0; m < kBatch; m++) {
        const int k = tid + (m0 + m) * kThreads;
        vec[m] = false;
        if (m0 + m >= kTasks || k >= ntask) continue;
        const int r = k / nq, q = k - r * nq;
        const uint8_t* row = lr_row(src, geo, s, geo.y0 + r - 3);
        const int gx = x0 - 8 + 8 * q;  // first sample of the left chunk
        if (gx < 0 || gx + 16 > geo.pex + 1 || (reinterpret_cast<uintptr_t>(row) & 15) != 0) continue;
        vec[m] = true;
        if (sb == 2) {
          // samples 4..7 of the left chunk and 0..5 of the right one
          const uint2 a = *reinterpret_cast<const uint2*>(row + int64_t(gx) * 2 + 8);
          const uint4 b = *reinterpret_cast<const uint4*>(row + int64_t(gx) * 2 + 16);
          wv[m][0] = a.x; wv[m][1] = a.y; wv[m][2] = b.x; wv[m][3] = b.y; wv[m][4] = b.z;
        } else {
          // bytes 4..15 of the 16 samples
          const uint4 a = *reinterpret_cast<const uint4*>(row + gx);
          wv[m][0] = a.y; wv[m][1] = a.z; wv[m][2] = a.w;
        }
      }
#pragma unroll
      for (int m = 0; m < kBatch; m++) {
        const int k = tid + (m0 + m) * kThreads;
        if (m0 + m >= kTasks || k >= ntask) continue;
        const int r = k / nq, q = k - r * nq;
        uint16_t* wp = &win[r * kWS + 8 * q];
        if (vec[m]) {
          uint4 o;
          if (sb == 2) {
            // window sample 2j of the chunk is sample 5 + 2j of the 16 from gx
            o.x = __funnelshift_r(wv[m][0], wv[m][1], 16);
            o.y = __funnelshift_r(wv[m][1], wv[m][2], 16);
            o.z = __funnelshift_r(wv[m][2], wv[m][3], 16);
            o.w = __funnelshift_r(wv[m][3], wv[m][4], 16);
          } else {
            const uint32_t lo = __funnelshift_r(wv[m][0], wv[m][1], 8);  // bytes 5..8
            const uint32_t hi = __funnelshift_r(wv[m][1], wv[m][2], 8);  // bytes 9..12
            o.x = __byte_perm(lo, 0, 0x4140);
            o.y = __byte_perm(lo, 0, 0x4342);
            o.z = __byte_perm(hi, 0, 0x4140);
            o.w = __byte_perm(hi, 0, 0x4342);
          }
          *reinterpret_cast<uint4*>(wp) = o;
        } else {
          const uint8_t* row = lr_row(src, geo, s, geo.y0 + r - 3);
#pragma unroll
          for (int e = 0; e < 8; e++) {
            const int c = 8 * q + e;
            if (c < ww) wp[e] = uint16_t(ld_row(row, sb, max(min(x0 - 3 + c, geo.pex), 0)));
          }
        }
      }
    }
  }
  __syncthreads();
  const av1pf_lr_unit& unit = *sm.unit;
  // each row group's contiguous run of output rows
  const int per = (h + G - 1) / G;
  const int i0 = g * per, i1 = min(h, i0 + per);
  const bool col = c < w && i0 < i1;
  if (type == AV1PF_RESTORE_WIENER) {
    // postfilter.rs:795-822
    int16_t* inter = reinterpret_cast<int16_t*>(sm.A);
    const int round0 = bd == 12 ? 5 : 3, round1 = bd == 12 ? 9 : 11;
    const int offset = 1 << (bd + 7 - round0 - 1);
    const int limit = (1 << (bd + 1 + 7 - round0)) - 1;
    const int h0 = unit.wiener[1][0], h1 = unit.wiener[1][1], h2 = unit.wiener[1][2];
    const int v0 = unit.wiener[0][0], v1 = unit.wiener[0][1], v2 = unit.wiener[0][2];
    const int h3 = 128 - 2 * (h0 + h1 + h2), v3 = 128 - 2 * (v0 + v1 + v2);
    // horizontal pass: two adjacent outputs per task from 8 window samples
    // (four aligned 32-bit loads), packed into one 32-bit store
    constexpr int LP = MW == 64 ? 5 : 4;  // log2 column pairs per row
    for (int k = tid; k < (wh << LP); k += kThreads) {
      const int r = k >> LP, c2 = (k & ((1 << LP) - 1)) * 2;
      if (c2 >= w) continue;
      const uint32_t* sp = reinterpret_cast<const uint32_t*>(&win[r * kWS + c2]);
      const uint32_t q0 = sp[0], q1 = sp[1], q2 = sp[2], q3 = sp[3];
      const int s0 = int(q0 & 0xffffu), s1 = int(q0 >> 16), s2 = int(q1 & 0xffffu), s3 = int(q1 >> 16);
      const int s4 = int(q2 & 0xffffu), s5 = int(q2 >> 16), s6 = int(q3 & 0xffffu), s7 = int(q3 >> 16);
      const int a0 = h0 * (s0 + s6) + h1 * (s1 + s5) + h2 * (s2 + s4) + h3 * s3;
      const int a1 = h0 * (s1 + s7) + h1 * (s2 + s6) + h2 * (s3 + s5) + h3 * s4;
      const int o0 = clip3(-offset, limit - offset, round2(a0, round0));
      const int o1 = clip3(-offset, limit - offset, round2(a1, round0));
      *reinterpret_cast<uint32_t*>(&inter[r * kWS + c2]) = uint32_t(uint16_t(o0)) | (uint32_t(uint16_t(o1)) << 16);
    }
    __syncthreads();
    // vertical pass: each row group slides a 7-row window down its column
    if (col) {
      const int16_t* ip = &inter[i0 * kWS + c];
      int t0 = ip[0], t1 = ip[kWS], t2 = ip[2 * kWS], t3 = ip[3 * kWS], t4 = ip[4 * kWS], t5 = ip[5 * kWS];
      for (int i = i0; i < i1; i++) {
        const int t6 = inter[(i + 6) * kWS + c];
        const int acc = v0 * (t0 + t6) + v1 * (t1 + t5) + v2 * (t2 + t4) + v3 * t3;
        F0[i * kMaxW + c] = clip3(0, maxv, round2(acc, round1));
        t0 = t1;
        t1 = t2;
        t2 = t3;
        t3 = t4;
        t4 = t5;
        t5 = t6;
      }
    }
    return;
  }
  // postfilter.rs:823-851 with box_filter_rect (postfilter.rs:901-991)
  int32_t* A = sm.A;
  int32_t* B = sm.B;
  const int set = unit.sgr_set & 15;
  const int r0 = c_sgr_params[set][0], r1 = c_sgr_params[set][2];
  if (r0) {
    sgr_ab<0, G>(win, A, B, sm.a2tab, c_sgr_params[set][1], bd, geo.y0, h, w, c, g);
    __syncthreads();
    if (col) sgr_flt_col<0>(A, B, win, c, i0, i1, geo.y0, [&](int i, int, int v) { F0[i * kMaxW + c] = v; });
    __syncthreads();
  }
  if (r1) {
    sgr_ab<1, G>(win, A, B, sm.a2tab, c_sgr_params[set][3], bd, geo.y0, h, w, c, g);
    __syncthreads();
  }
  const int w0 = unit.sgr_xqd[0], w1 = unit.sgr_xqd[1];
  const int w2 = (1 << 7) - w0 - w1;
  if (col) {
    // the weighted sum of the two filters and the sample itself; this
    // thread's own slot of the output tile
    auto combine = [&](int i, int cd, int flt1) {
      const int u = cd << 4;
      int v = w1 * u;
      v += r0 != 0 ? w0 * F0[i * kMaxW + c] : w0 * u;
      v += w2 * flt1;
      F0[i * kMaxW + c] = clip3(0, maxv, round2(v, 11));
    };
    if (r1) {
      sgr_flt_col<1>(A, B, win, c, i0, i1, geo.y0, combine);
    } else {
      for (int i = i0; i < i1; i++) {
        const int cd = win[(i + 3) * kWS + c + 3];
        combine(i, cd, cd << 4);
      }
    }
  }
}

// With readiness flags: waits (threads 0..15, one flag each) for the CDEF
// half superblocks under a rectangle: the stripe's rows y0 .. y1, which it
// reads from the CDEF planes, over its columns and 3 on either side. (The
// rows past the stripe come from the loop filter's output: the half
// superblocks at the stripe's first and last rows waited for the tiles
// under their windows, which reach 2 rows further.)
__device__ __forceinline__ void lr_wait_cdef(const FrameDesc& f, const uint32_t* flags, int p, const LrGeom& geo, int x0,
                                             int w, int tid) {
  if (tid >= 16) return;
  const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
  const int xa = max(x0 - 3, 0), xb = min(x0 + w + 2, geo.pex);
  const int h0 = (geo.y0 << sy) >> 5, h1 = ((geo.y1 << sy) + sy) >> 5;
  const int c0 = (xa << sx) >> 6, c1 = min(((xb << sx) + sx) >> 6, f.cdef_sbc - 1);
  const int hr = h0 + (tid >> 2), c = c0 + (tid & 3);
  if (hr > h1 || c > c1) return;
  flag_wait(flags + f.cdef_flag_base + hr * f.cdef_sbc + c);
}

__global__ void __launch_bounds__(kThreads, 3) lr_kernel(const FrameDesc* __restrict__ frames,
                                                         const Item* __restrict__ items, int n_items,
                                                         const uint32_t* __restrict__ flags) {
  AV1PF_TRACE_BEGIN();
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ av1pf_lr_unit s_unit;
  LrSmem sm;
  sm.win = reinterpret_cast<uint16_t*>(smem);
  sm.A = reinterpret_cast<int32_t*>(smem + kWinBytes);
  sm.B = reinterpret_cast<int32_t*>(smem + kWinBytes + kABytes);
  sm.a2tab = g_sgr_a2.v;
  sm.F0 = reinterpret_cast<int32_t*>(smem + kWinBytes + 2 * kABytes);
  sm.unit = &s_unit;
  const int tid = threadIdx.x;

  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int p = item.plane;
    const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
    // lr_stripe (postfilter.rs:640-661)
    LrGeom geo;
    const int s = item.a;
    geo.pey = ((f.fh + sy) >> sy) - 1;
    geo.pex = ((f.uw + sx) >> sx) - 1;
    geo.ss = (-8 + s * 64) >> sy;
    geo.se = geo.ss + (64 >> sy) - 1;
    geo.y0 = max(geo.ss, 0);
    geo.y1 = min(geo.se, geo.pey);
    const int x0 = item.x0, w = int(item.x1) - int(item.x0);
    const int h = geo.y1 - geo.y0 + 1;
    if (h <= 0 || w <= 0) {
      // without flags every CTA waits, so the kernel never completes before
      // its predecessor
      if (flags)
        pdl_trigger();
      else
        pdl_wait();
      continue;
    }
    int type = AV1PF_RESTORE_NONE;
    const av1pf_lr_unit* unit_p = nullptr;
    if (f.lr_on && f.lr_type[p] != AV1PF_RESTORE_NONE) {
      const int unit_size = f.lr_unit_size[p];
      const int luma_row = max(s * 64 - 8, 0);
      const int unit_row = min(f.lr_unit_rows[p] - 1, ((luma_row + 8) >> sy) / unit_size);
      unit_p = &f.lru[p][unit_row * f.lr_unit_cols[p] + item.b];
      type = unit_p->type;
    }
    // the descriptor and the unit are inputs of the chain; the planes below
    // are the previous stage's output: all of it, or with readiness flags
    // the half superblocks under the rectangle
    if (flags) {
      pdl_trigger();
      lr_wait_cdef(f, flags, p, geo, x0, w, tid);
      __syncthreads();
    } else {
      pdl_wait();
    }
    if (type != AV1PF_RESTORE_WIENER && type != AV1PF_RESTORE_SGRPROJ) {
      pass_through(f, p, x0, geo.y0, w, h, tid);  // uniform across the CTA: no barrier needed
      continue;
    }
    if (w > 32)
      restore_rect<72>(f, sm, geo, p, s, x0, w, h, type, unit_p, tid);
    else
      restore_rect<36>(f, sm, geo, p, s, x0, w, h, type, unit_p, tid);
    __syncthreads();
    // the rectangle's output samples, from shared memory to the reference
    // frame and (frames without film grain) the packed frame: u8 samples at
    // 8 bits, little-endian u16 above (frame.rs:153-158), rows of the plane's
    // width (decoder/mod.rs:846-917)
    {
      const int sb = f.sb, bd = f.bd;
      const DPlane dst = f.ref[p];
      uint8_t* d0 = dst.p + (int64_t(geo.y0) * dst.stride + x0) * sb;
      const int64_t dp = dst.stride * sb;
      const bool d_vec = ((reinterpret_cast<uintptr_t>(d0) | uintptr_t(dp)) & 15) == 0;
      const int bps = bd > 8 ? 2 : 1;
      const int64_t op = int64_t(geo.pex + 1) * bps;
      uint8_t* o0 = f.lr_pack ? f.frame_out + f.out_off[p] + int64_t(geo.y0) * op + int64_t(x0) * bps : nullptr;
      const bool o_vec = ((reinterpret_cast<uintptr_t>(o0) | uintptr_t(op)) & 15) == 0;
      if (w > 32) {
        store_tile<64>(sm.F0, d0, dp, sb, d_vec, w, h, tid);
        if (o0) store_tile<64>(sm.F0, o0, op, bps, o_vec, w, h, tid);
      } else {
        store_tile<32>(sm.F0, d0, dp, sb, d_vec, w, h, tid);
        if (o0) store_tile<32>(sm.F0, o0, op, bps, o_vec, w, h, tid);
      }
    }
    __syncthreads();
  }
  AV1PF_TRACE_END(3);
}

cudaError_t lr_init() {
  return cudaFuncSetAttribute(lr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
}

void launch_lr(const FrameDesc* frames, const Item* items, int n_items, uint32_t* flags, cudaStream_t s) {
  if (n_items <= 0) return;
  // one CTA per rectangle: the block scheduler hands rectangles of uneven
  // cost (copy, Wiener, self-guided) to SMs as they free up
  launch_pdl(lr_kernel, min(n_items, kItemGrid), kThreads, size_t(kSmemBytes), s, frames, items, n_items,
             static_cast<const uint32_t*>(flags));
}

}  // namespace av1pf
