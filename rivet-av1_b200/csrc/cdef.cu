// cdef.cu — the constrained directional enhancement filter (7.15).
//
// Reference: rivet-av1 src/decoder/postfilter.rs:266-513 (cdef, cdef_block,
// cdef_direction, cdef_filter, cdef_filter_block) and src/dsp/cdef.rs:13-90
// (Taps, constrain, filter_scalar).
//
// One CTA per superblock (64x64 luma and its chroma; R = 64 rows, 256
// threads), or per half superblock (R = 32 rows, 128 threads) when a launch
// has at most one wave of superblocks: 510 superblocks of a 1080p frame
// would leave 66 SMs with 4 and 82 with 3, 1020 halves spread within 2%.
// The rows plus a 2-sample border of every plane are staged in shared
// memory as int16 with
// unavailable samples (outside the frame's mode-info area, postfilter.rs:
// 421-422, 464-488) stored as -32768. That value needs no special case:
// constrain() of a difference that large is 0 for every strength/damping
// pair the format allows (|d| >= 2^(damping+1) >= str << adj), a signed max
// never picks it, and an unsigned min never picks it. In the direction
// search each thread takes one 8x8 block and two of the 8 directions (one
// pair per warp), so the partial-sum bins are compile-time register indices.
#include "av1_tables.h"
#include "common.cuh"
#include "kernels.h"
#include "lf_core.cuh"

namespace av1pf {

namespace {

// Shared-memory window of one plane: up to 54 rows (32 + 2*2, or 32 + 2*11
// with the horizontal loop-filter pass fused in) x 80 columns
// (64 + 8 on each side, so global loads stay 8-sample aligned), row stride
// 82 int16 = 41 words: a warp's 4 rows x 8 blocks of centre loads then hit
// 32 different banks.
constexpr int kS = 82;
constexpr int kTopLfh = 11;     // rows above (and below) with the horizontal LF pass fused
constexpr int kColOff = 8;       // window column of plane x = px0
constexpr int16_t kNA = -32768;  // unavailable sample
// The direction search reads the R luma rows of the superblock's 64 columns
// from a copy with 16-byte aligned rows (kDS int16 each): one 16-byte load
// per block row, and the 8 lanes of a load phase (8 blocks side by side)
// read 32 consecutive words. (From the filter window, whose odd row stride
// keeps the filter's loads apart, blocks 8 rows apart would share banks: a
// 4-way conflict on every load.)
constexpr int kDS = 72;
// dynamic shared memory: the direction-search copy, then the three windows
// of R + 2*2 rows, or R + 2*11 with the horizontal loop-filter pass fused in
constexpr int cdef_dir_bytes(int R) { return R * kDS * 2; }
constexpr int cdef_smem(int R, bool lfh) { return cdef_dir_bytes(R) + 3 * (R + 2 * (lfh ? kTopLfh : 2)) * kS * 2; }

// Per 8x8 block and plane: strengths, tap weights and window offsets.
struct BlkTaps {
  int16_t pri, sec;
  int16_t po0, po1, so00, so01, so10, so11;
  int8_t pri_adj, sec_adj, pt0, pt1;
  int8_t copy, one, pad1, pad2;  // one: always 1 (see cdef_tap)
};

}  // namespace

// One filtered sample (cdef.rs:54-90 for one position) from a window with
// row stride `st`; offsets are in samples of that window.
struct TapsDev {
  int pri, sec, pri_adj, sec_adj, pt0, pt1;
  int po0, po1, so00, so01, so10, so11;
  int one, mone;  // 1 and -1, read from shared memory (see cdef_tap)
};

// `one` is 1 and `mone` -1 at run time but opaque to the compiler, so the
// differences below are integer multiply-adds: the kernel is bound by the
// integer ALU pipe, and these move three of a tap's operations to the
// multiply-add pipe, which is otherwise mostly idle. nx = -x.
__device__ __forceinline__ void cdef_tap(int p, int nx, int one, int mone, int str, int adj, int w, int& sum, int& mx,
                                         unsigned& mn) {
  const int d = p * one + nx;                              // p - x
  const int lim = max(0, (abs(d) >> adj) * mone + str);    // max(0, str - (|d| >> adj))
  sum += w * min(max(d, lim * mone), lim);                 // constrain(d)
  mx = max(mx, p);
  mn = min(mn, unsigned(p));
}

// MODE 0: primary and secondary taps, result clamped to the available taps'
// [min, max]. MODE 1 (secondary strength 0) and MODE 2 (primary strength
// 0) leave out the zero-strength taps, whose constrain() is 0, and the
// clamp: with one kind of tap the weights sum to 12 < 16, so
// x + round(sum / 16) already lies within [x - D, x + D'] where D, D' are the
// largest negative and positive differences of the taps in use.
template <int MODE>
__device__ __forceinline__ int cdef_px(const int16_t* c, const TapsDev& t) {
  const int x = c[0];
  const int nx = x * t.mone;
  int sum = 0, mx = x;
  unsigned mn = unsigned(x);
  if (MODE != 2) {
    cdef_tap(c[t.po0], nx, t.one, t.mone, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
    cdef_tap(c[-t.po0], nx, t.one, t.mone, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
    cdef_tap(c[t.po1], nx, t.one, t.mone, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
    cdef_tap(c[-t.po1], nx, t.one, t.mone, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  }
  if (MODE != 1) {
    cdef_tap(c[t.so00], nx, t.one, t.mone, t.sec, t.sec_adj, 2, sum, mx, mn);
    cdef_tap(c[-t.so00], nx, t.one, t.mone, t.sec, t.sec_adj, 2, sum, mx, mn);
    cdef_tap(c[t.so01], nx, t.one, t.mone, t.sec, t.sec_adj, 2, sum, mx, mn);
    cdef_tap(c[-t.so01], nx, t.one, t.mone, t.sec, t.sec_adj, 2, sum, mx, mn);
    cdef_tap(c[t.so10], nx, t.one, t.mone, t.sec, t.sec_adj, 1, sum, mx, mn);
    cdef_tap(c[-t.so10], nx, t.one, t.mone, t.sec, t.sec_adj, 1, sum, mx, mn);
    cdef_tap(c[t.so11], nx, t.one, t.mone, t.sec, t.sec_adj, 1, sum, mx, mn);
    cdef_tap(c[-t.so11], nx, t.one, t.mone, t.sec, t.sec_adj, 1, sum, mx, mn);
  }
  const int v = x + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
  return MODE == 0 ? min(max(v, int(mn)), mx) : v;
}

// The Taps of cdef_filter_block (postfilter.rs:489-511); doff[d][k] is the
// window offset of CDEF_DIRECTIONS[d][k] (shared memory: the threads index
// it by their blocks' directions). CDEF_SEC_TAPS is [2, 1] for both
// primary-tap parities.
__device__ __forceinline__ BlkTaps make_blk_taps(int pri, int sec, int damping, int dir, int coeff_shift,
                                                 const int16_t (*doff)[2]) {
  BlkTaps t;
  t.pri = int16_t(pri);
  t.sec = int16_t(sec);
  t.pri_adj = int8_t(pri ? max(damping - floor_log2(uint32_t(pri)), 0) : 0);
  t.sec_adj = int8_t(sec ? max(damping - floor_log2(uint32_t(sec)), 0) : 0);
  const bool odd = (pri >> coeff_shift) & 1;  // CDEF_PRI_TAPS[(pri >> cs) & 1]: [4,2] / [3,3]
  t.pt0 = int8_t(odd ? 3 : 4);
  t.pt1 = int8_t(odd ? 3 : 2);
  const int dlo = (dir + 6) & 7, dhi = (dir + 2) & 7;
  t.po0 = doff[dir][0];
  t.po1 = doff[dir][1];
  t.so00 = doff[dlo][0];
  t.so01 = doff[dhi][0];
  t.so10 = doff[dlo][1];
  t.so11 = doff[dhi][1];
  t.copy = (pri == 0 && sec == 0) ? 1 : 0;  // a zero-strength filter is the identity
  t.one = 1;
  t.pad1 = t.pad2 = 0;
  return t;
}

__device__ __forceinline__ TapsDev taps_of(const BlkTaps& b) {
  TapsDev t;
  t.pri = b.pri;
  t.sec = b.sec;
  t.pri_adj = b.pri_adj;
  t.sec_adj = b.sec_adj;
  t.pt0 = b.pt0;
  t.pt1 = b.pt1;
  t.po0 = b.po0;
  t.po1 = b.po1;
  t.so00 = b.so00;
  t.so01 = b.so01;
  t.so10 = b.so10;
  t.so11 = b.so11;
  t.one = b.one;
  t.mone = -t.one;
  return t;
}

// Partial-sum bin of direction D for pixel (i, j) (postfilter.rs:352-363).
template <int D>
__device__ __forceinline__ constexpr int cdef_bin(int i, int j) {
  return D == 0 ? i + j
       : D == 1 ? i + j / 2
       : D == 2 ? i
       : D == 3 ? 3 + i - j / 2
       : D == 4 ? 7 + i - j
       : D == 5 ? 3 - i / 2 + j
       : D == 6 ? j
                : i / 2 + j;
}

// The cost of direction D from its partial sums (postfilter.rs:365-390).
template <int D>
__device__ __forceinline__ int32_t cdef_cost_of(const int32_t* p) {
  int32_t cost = 0;
  if (D == 2 || D == 6) {
#pragma unroll
    for (int i = 0; i < 8; i++) cost += p[i] * p[i];
    cost *= c_div_table[8];
  } else if (D == 0 || D == 4) {
#pragma unroll
    for (int i = 0; i < 7; i++) cost += (p[i] * p[i] + p[14 - i] * p[14 - i]) * c_div_table[i + 1];
    cost += p[7] * p[7] * c_div_table[8];
  } else {
#pragma unroll
    for (int j = 0; j < 5; j++) cost += p[3 + j] * p[3 + j];
    cost *= c_div_table[8];
#pragma unroll
    for (int j = 0; j < 3; j++) cost += (p[j] * p[j] + p[10 - j] * p[10 - j]) * c_div_table[2 * j + 2];
  }
  return cost;
}

// Costs of directions P and P + 4 of the 8x8 block whose top-left sample is
// `s`, rows ST samples apart; samples are >> sh then - 128. With ST = kDS the
// rows are 16-byte aligned and each is one 16-byte load, else 4-byte words.
template <int P, int ST = kS>
__device__ __forceinline__ void cdef_cost_pair(const int16_t* s, int sh, int one, int32_t& c1, int32_t& c2) {
  int32_t a[15], b[15];
#pragma unroll
  for (int k = 0; k < 15; k++) a[k] = b[k] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    uint32_t row[4];
    if (ST == kDS) {
      const uint4 v = *reinterpret_cast<const uint4*>(s + i * ST);
      row[0] = v.x;
      row[1] = v.y;
      row[2] = v.z;
      row[3] = v.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++) row[q] = reinterpret_cast<const uint32_t*>(s + i * ST)[q];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t w = row[q];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = 2 * q + h;
        const int x = ((int(int16_t(h ? (w >> 16) : (w & 0xffffu)))) >> sh) - 128;
        // multiply-adds by an opaque 1: the bins accumulate on the multiply-add pipe
        a[cdef_bin<P>(i, j)] = x * one + a[cdef_bin<P>(i, j)];
        b[cdef_bin<P + 4>(i, j)] = x * one + b[cdef_bin<P + 4>(i, j)];
      }
    }
  }
  c1 = cdef_cost_of<P>(a);
  c2 = cdef_cost_of<P + 4>(b);
}

// Stages plane p of the half superblock at superblock column sc and luma
// row y0 with `top` rows above and below (the 2-sample CDEF border, or 11
// with the horizontal loop-filter pass) into the window `wp` as int16,
// samples outside the mode-info area as kNA. Window rows are NCH chunks of 8
// samples (the first chunk starts 8 samples left of the superblock, so loads
// stay 8-sample aligned); loads issue two at a time before their stores.
// With `dw` (luma only) the superblock's R rows x 64 columns also go to the
// direction-search copy (rows kDS apart).
template <int R, int SX>
__device__ __forceinline__ void stage_plane(const FrameDesc& f, int p, int sc, int y0, int top, int16_t* wp, int tid,
                                            int16_t* dw = nullptr) {
  constexpr int NT = 4 * R;
  constexpr int NCH = ((64 >> SX) + 16) / 8;
  constexpr int kSlots = ((R + 2 * kTopLfh) * NCH + NT - 1) / NT;
  const int sy = plane_ssy(f, p), sb = f.sb;
  const int bh = (R >> sy) + 2 * top;
  const int px0 = (sc * 64) >> SX, py0 = (y0 >> sy) - top;
  const int xlim = (f.mi_cols * 4) >> SX, ylim = (f.mi_rows * 4) >> sy;
  const DPlane src = f.cur[p];
  // chunk class: 0 none, 1 unavailable, 2 inside (vector load), 3 straddles the edge
  auto kind_of = [&](int r, int gy, int gx0) {
    if (r >= bh) return 0;
    if (gy < 0 || gy >= ylim || gx0 + 8 <= 0 || gx0 >= xlim) return 1;
    return (gx0 >= 0 && gx0 + 8 <= xlim) ? 2 : 3;
  };
#pragma unroll
  for (int m0 = 0; m0 < kSlots; m0 += 2) {
    uint4 q[2];
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const int k = tid + NT * (m0 + m), r = k / NCH, ch = k - r * NCH;
      const int gy = py0 + r, gx0 = px0 - kColOff + ch * 8;
      if (m0 + m < kSlots && kind_of(r, gy, gx0) == 2) {
        const uint8_t* rowp = src.p + int64_t(gy) * src.stride * sb;
        if (sb == 2) {
          q[m] = *reinterpret_cast<const uint4*>(rowp + int64_t(gx0) * 2);
        } else {
          const uint2 h2 = *reinterpret_cast<const uint2*>(rowp + gx0);
          q[m] = make_uint4(h2.x, h2.y, 0, 0);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 2; m++) {
      if (m0 + m >= kSlots) continue;
      const int k = tid + NT * (m0 + m), r = k / NCH, ch = k - r * NCH;
      const int gy = py0 + r, gx0 = px0 - kColOff + ch * 8;
      const int kind = kind_of(r, gy, gx0);
      if (kind == 0) continue;
      uint32_t o[4];
      if (kind == 2 && sb == 2) {
        o[0] = q[m].x;
        o[1] = q[m].y;
        o[2] = q[m].z;
        o[3] = q[m].w;
      } else if (kind == 2) {
        // bytes b0..b3 -> int16 pairs
        o[0] = __byte_perm(q[m].x, 0, 0x4140);
        o[1] = __byte_perm(q[m].x, 0, 0x4342);
        o[2] = __byte_perm(q[m].y, 0, 0x4140);
        o[3] = __byte_perm(q[m].y, 0, 0x4342);
      } else {
        int16_t v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const int gx = gx0 + e;
          v[e] = (kind == 3 && gx >= 0 && gx < xlim) ? int16_t(ld_sample(src, sb, gx, gy)) : kNA;
        }
#pragma unroll
        for (int e = 0; e < 4; e++) o[e] = uint32_t(uint16_t(v[2 * e])) | (uint32_t(uint16_t(v[2 * e + 1])) << 16);
      }
      uint32_t* dst = reinterpret_cast<uint32_t*>(wp + r * kS + ch * 8);
#pragma unroll
      for (int e = 0; e < 4; e++) dst[e] = o[e];
      if (dw && r >= top && r < top + R && ch >= 1 && ch <= 8)
        *reinterpret_cast<uint4*>(dw + (r - top) * kDS + (ch - 1) * 8) = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
}

// One horizontal-edge lane on the window (kept out of line: the CDEF
// kernel's register budget is sized for the CDEF phases).
__device__ __noinline__ void lfh_lane(int16_t* q0p, int code, bool chroma, int bd, int lvl, int sharp) {
  lf_filter_smem(q0p, kS, code, chroma, bd, lvl, sharp);
}

// The horizontal loop-filter edges (postfilter.rs:67-104 pass 1) of plane p
// that change rows of the staged window: edges at plane rows py0-4 ..
// py0+bh+4 (py0 the half's first row) across the superblock's columns and
// one 4x4 column on each side.
// Every edge reads at most 7 rows on either side, which the 11-row halo
// holds, so the window ends up holding the loop filter's output on the
// rows CDEF reads. Edges of a pass never touch each other's samples in a
// conformant frame, so they run in parallel in place.
template <int R>
__device__ __forceinline__ void lfh_window(const FrameDesc& f, const LfTables& tb, int p, int sc, int y0,
                                           int16_t* wp, uint16_t* hdec, int tid) {
  constexpr int NT = 4 * R;
  const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
  const int bhs = R >> sy;
  const int px0 = (sc * 64) >> sx, py0 = y0 >> sy;
  const int cx0 = (px0 >> 2) - 1, cy0 = (py0 >> 2) - 1;
  const int ncx = ((64 >> sx) >> 2) + 2;  // 18 or 10
  const int ncy = (bhs >> 2) + 3;         // 19, 11 or 7
  const int gw = f.mi_cols >> sx, gh = f.mi_rows >> sy;
  for (int k = tid; k < ncy * 18; k += NT) {
    const int cyi = k / 18, cxi = k - cyi * 18;
    const int cx = cx0 + cxi, cy = cy0 + cyi;
    int dv = 0, dh = 0;
    if (cxi < ncx && cx >= 0 && cy >= 0 && cx < gw && cy < gh) lf_decide2(f, tb, p, cx, cy, dv, dh);
    hdec[k] = uint16_t(dh);
  }
  __syncthreads();
  const int bd = f.bd, sharp = f.sharpness;
  for (int k = tid; k < ncy * 18 * 4; k += NT) {
    const int lane = k & 3, cell = k >> 2;
    const int d = hdec[cell];
    if (!d) continue;
    const int cyi = cell / 18, cxi = cell - cyi * 18;
    const int code = d >> 6, lvl = d & 63;
    const int e = (cy0 + cyi) * 4;  // plane row of q0
    if (e < (code == 3 ? 8 : 4)) {  // a conformant map keeps wide edges off the plane start
      atomicOr(&g_error_flags, ERRF_BAD_MAP);
      continue;
    }
    const int col = (cx0 + cxi) * 4 + lane;
    lfh_lane(&wp[(e - py0 + kTopLfh) * kS + (col - px0 + kColOff)], code, p != 0, bd, lvl, sharp);
  }
  __syncthreads();
}

// Rows B-2 .. B+1 of the stripe boundary B inside superblock row sr (the
// loop filter's output, which loop restoration reads across the boundary)
// from the window to f.prelf[p], over the superblock's columns. B is 8 luma
// rows above the superblock row's end: a half superblock CTA writes them
// from the bottom half (the window starting R rows above the row's end).
template <int R>
__device__ __forceinline__ void write_prelf(const FrameDesc& f, int p, int sc, int sr, const int16_t* wp, int tid) {
  constexpr int NT = 4 * R;
  const DPlane dst = f.prelf[p];
  const int b = sr + 1;  // the boundary inside superblock row sr
  if (!dst.p || b >= f.stripes) return;
  const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
  const int px0 = (sc * 64) >> sx, py0 = (sr * 64 + 64 - R) >> sy;  // the window's first plane row
  const int B = (64 * b - 8) >> sy;
  const int xlim = (f.mi_cols * 4) >> sx, ylim = (f.mi_rows * 4) >> sy;
  const int ws = 6 - sx;  // log2 of the superblock's width in the plane
  for (int k = tid; k < (4 << ws); k += NT) {
    const int j = k >> ws, c = k & ((1 << ws) - 1);  // 4 rows x 64 >> sx columns
    const int y = B - 2 + j, x = px0 + c;
    if (y < ylim && x < xlim)
      st_sample(dst, f.sb, x, (b - 1) * 4 + j, wp[(y - py0 + kTopLfh) * kS + c + kColOff]);
  }
}

// Item: R luma rows of a superblock (x0 = SB column, y0 = SB row, a = which
// R rows). 4R threads, one warp per 8x8 block row. Item kind 1: the frame's
// horizontal loop-filter edges (planes in f.lfh_mask) are filtered here, on
// the staged window, before CDEF. `wrows` is the rows of one plane's window
// (R + 22 when the launch has kind-1 items, else R + 4).
// LFH: the launch has kind-1 items (the fused horizontal loop-filter pass);
// without it the kernel carries none of that pass's code, which keeps the
// default kernel's instruction footprint small.
// With readiness flags: waits (threads 0..47, one flag each) for the
// loop-filter tiles under the CTA's windows, the rows and columns
// stage_plane reads: plane rows (y0 >> sy) - 2 .. ((y0 + R) >> sy) + 1 and
// 8 columns past the superblock on either side, within the plane.
template <int R>
__device__ __forceinline__ void cdef_wait_lf(const FrameDesc& f, const uint32_t* flags, int sc, int y0, int tid) {
  if (tid >= 48) return;
  const int p = tid >> 4, dy = (tid >> 2) & 3, dx = tid & 3;
  if (p >= f.np || f.lf_tiles_x[p] == 0) return;
  const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
  const int W = f.cur[p].w, H = f.cur[p].h;
  const int r0 = max((y0 >> sy) - 2, 0), r1 = min(((y0 + R) >> sy) + 1, H - 1);
  const int c0 = max(((sc * 64) >> sx) - 8, 0), c1 = min(((sc * 64 + 64) >> sx) + 7, W - 1);
  const int ty = (r0 >> 6) + dy, tx = (c0 >> 6) + dx;
  if (r0 > r1 || c0 > c1 || ty > (r1 >> 6) || tx > (c1 >> 6)) return;
  flag_wait(flags + f.lf_flag_base[p] + ty * f.lf_tiles_x[p] + tx);
}

template <int R, bool LFH>
__global__ void __launch_bounds__(4 * R, 256 / R) cdef_kernel(const FrameDesc* __restrict__ frames,
                                                           const Item* __restrict__ items, int n_items, int wrows,
                                                           uint32_t* __restrict__ flags) {
  AV1PF_TRACE_BEGIN();
  extern __shared__ __align__(16) int16_t cdef_smem_base[];  // [R][kDS] direction copy, then [3][wrows * kS]
  int16_t* const dwin = cdef_smem_base;
  int16_t* const cdef_win = cdef_smem_base + cdef_dir_bytes(R) / 2;
  auto win = [&](int p) { return cdef_win + p * wrows * kS; };  // plane p's window
  __shared__ int32_t cost[R][8];
  __shared__ BlkTaps taps[3][R];
  __shared__ uint8_t bstate[R];  // 0 = outside the MI area, 1 = copy, 2 = filter
  const LfTables& tb = g_lf_tables;
  __shared__ uint16_t hdec[(R / 4 + 3) * 18];  // horizontal-edge decisions of one plane
  __shared__ int16_t doff[8][2];      // window offsets of CDEF_DIRECTIONS
  __shared__ uint8_t uvdir[2][2][8];  // CDEF_UV_DIR
  __shared__ int s_one;               // 1, opaque to the compiler (see cdef_tap)
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (tid < 16) doff[tid >> 1][tid & 1] = int16_t(c_cdef_dirs[tid >> 1][tid & 1][0] * kS + c_cdef_dirs[tid >> 1][tid & 1][1]);
  if (tid < 32) (&uvdir[0][0][0])[tid] = (&c_cdef_uv_dir[0][0][0])[tid];
  if (tid == 0) s_one = 1;
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int sc = item.x0, sr = item.y0;
    const int y0 = sr * 64 + item.a * R;  // luma row of the CTA's first row
    const int np = f.np, sb = f.sb;
    const int cs = f.bd - 8;
    const int idx = f.cdef_idx[int64_t(sr) * f.cdef_stride + sc];  // postfilter.rs:285
    const bool lfh = LFH && item.kind != 0;
    const int top = lfh ? kTopLfh : 2;  // window row of the superblock's first row
    // --- per 8x8: inside the MI area? skipped? (postfilter.rs:281-287, 306-310) ---
    // (the maps are inputs of the chain: read before waiting for the loop filter)
    uint8_t st = 0;
    if (tid < R) {
      const int by = tid >> 3, bx = tid & 7;
      const int r = (y0 >> 2) + 2 * by, c = sc * 16 + 2 * bx;
      if (r < f.mi_rows && c < f.mi_cols) {
        st = 1;
        if (idx >= 0) {
          const av1pf_mi* m = f.mi + int64_t(r) * f.mi_stride + c;
          const int ms = f.mi_stride;
          const bool skip = (m[0].skip_segment & AV1PF_MI_SKIP) && (m[ms].skip_segment & AV1PF_MI_SKIP) &&
                            (m[1].skip_segment & AV1PF_MI_SKIP) && (m[ms + 1].skip_segment & AV1PF_MI_SKIP);
          if (!skip) st = 2;
        }
      }
    }
    if (flags) {
      // only the loop-filter tiles this CTA reads
      pdl_trigger();
      cdef_wait_lf<R>(f, flags, sc, y0, tid);
    } else {
      pdl_wait();  // the loop filter's output is complete past this point
    }
    __syncthreads();  // the previous item is done with the windows and block states
    if (tid < R) bstate[tid] = st;
    // --- stage the windows (postfilter.rs:464-488): 8-sample chunks ---
    for (int p = 0; p < np; p++) {
      if (plane_ssx(f, p))
        stage_plane<R, 1>(f, p, sc, y0, top, win(p), tid);
      else
        stage_plane<R, 0>(f, p, sc, y0, top, win(p), tid, p == 0 && !lfh ? dwin : nullptr);
    }
    if (lfh) {
      __syncthreads();
      for (int p = 0; p < np; p++)
        if ((f.lfh_mask >> p) & 1) lfh_window<R>(f, tb, p, sc, y0, win(p), hdec, tid);
      if (y0 + R == sr * 64 + 64)  // the rows that end the superblock row
        for (int p = 0; p < np; p++)
          if ((f.lfh_mask >> p) & 1) write_prelf<R>(f, p, sc, sr, win(p), tid);
      // the direction search reads the loop-filtered luma
      for (int k = tid; k < R * 8; k += 4 * R) {
        const int r = k >> 3, ch = k & 7;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(win(0) + (top + r) * kS + kColOff + ch * 8);
        *reinterpret_cast<uint4*>(dwin + r * kDS + ch * 8) = make_uint4(src[0], src[1], src[2], src[3]);
      }
    }
    __syncthreads();
    // --- direction search (postfilter.rs:345-401): each thread two directions of one block ---
    {
      const int pair = warp & 3;
      const int b = (warp >> 2) * 32 + lane;
      if (bstate[b] == 2) {
        const int by = b >> 3, bx = b & 7;
        const int16_t* s = &dwin[by * 8 * kDS + bx * 8];
        int32_t c1, c2;
        switch (pair) {
          case 0: cdef_cost_pair<0, kDS>(s, cs, s_one, c1, c2); break;
          case 1: cdef_cost_pair<1, kDS>(s, cs, s_one, c1, c2); break;
          case 2: cdef_cost_pair<2, kDS>(s, cs, s_one, c1, c2); break;
          default: cdef_cost_pair<3, kDS>(s, cs, s_one, c1, c2); break;
        }
        cost[b][pair] = c1;
        cost[b][pair + 4] = c2;
      }
    }
    __syncthreads();
    // --- per-block strengths and taps (postfilter.rs:311-341) ---
    if (tid < R) {
      const int b = tid;
      int lp = 0, ls = 0, ld = 0, up = 0, us = 0, ud = 0;
      bool filt = bstate[b] == 2;
      if (filt) {
        int32_t best = 0;
        int y_dir = 0;
#pragma unroll
        for (int d = 0; d < 8; d++) {
          if (cost[b][d] > best) {
            best = cost[b][d];
            y_dir = d;
          }
        }
        const int32_t var = (best - cost[b][(y_dir + 4) & 7]) >> 10;
        int pri = f.cdef_y_pri[idx] << cs;
        ls = f.cdef_y_sec[idx] << cs;
        ld = pri == 0 ? 0 : y_dir;
        const int var_str = (var >> 6) != 0 ? min(floor_log2(uint32_t(var >> 6)), 12) : 0;
        lp = var != 0 ? (pri * (4 + var_str) + 8) >> 4 : 0;
        up = f.cdef_uv_pri[idx] << cs;
        us = f.cdef_uv_sec[idx] << cs;
        ud = up == 0 ? 0 : uvdir[f.ssx][f.ssy][y_dir];
      }
      BlkTaps L = make_blk_taps(lp, ls, f.cdef_damping + cs, ld, cs, doff);
      BlkTaps U = make_blk_taps(up, us, f.cdef_damping + cs - 1, ud, cs, doff);
      if (!filt) L.copy = U.copy = 1;
      taps[0][b] = L;
      taps[1][b] = U;
      taps[2][b] = U;
    }
    __syncthreads();
    // --- filter + write (postfilter.rs:405-442): warp = block row, lane = (row, block) ---
    for (int p = 0; p < np; p++) {
      const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
      const int w = 8 >> sx, bhp = 8 >> sy;
      const DPlane dst = f.cdef[p];
      for (int q = 0; q < bhp / 4; q++) {
        const int by = warp, bx = lane & 7, rr = q * 4 + (lane >> 3);
        const int b = by * 8 + bx;
        if (bstate[b] == 0) continue;
        const int lx = bx * w, ly = by * bhp + rr;
        const int16_t* c = &win(p)[(top + ly) * kS + kColOff + lx];
        // results packed two int16 per word as they are produced
        uint32_t o[4] = {0, 0, 0, 0};
        const BlkTaps bt = taps[p][b];
#define CDEF_ROW(EXPR)                                                   \
  _Pragma("unroll") for (int j = 0; j < 8; j++) if (j < w) {             \
    const uint32_t v_ = uint32_t(EXPR);                                   \
    o[j >> 1] = (j & 1) ? (o[j >> 1] | (v_ << 16)) : v_;                  \
  }
        if (bt.copy) {
          CDEF_ROW(uint16_t(c[j]))
        } else {
          const TapsDev t = taps_of(bt);
          if (t.pri != 0 && t.sec != 0) {
            CDEF_ROW(cdef_px<0>(c + j, t))
          } else if (t.pri != 0) {
            CDEF_ROW(cdef_px<1>(c + j, t))
          } else {
            CDEF_ROW(cdef_px<2>(c + j, t))
          }
        }
#undef CDEF_ROW
        const int gx = ((sc * 64) >> sx) + lx, gy = (y0 >> sy) + ly;
        uint8_t* row = dst.p + int64_t(gy) * dst.stride * sb;
        if (sb == 2) {
          uint16_t* r16 = reinterpret_cast<uint16_t*>(row) + gx;
          if (w == 8)
            *reinterpret_cast<uint4*>(r16) = make_uint4(o[0], o[1], o[2], o[3]);
          else
            *reinterpret_cast<uint2*>(r16) = make_uint2(o[0], o[1]);
        } else {
          uint8_t* r8 = row + gx;
          if (w == 8)
            *reinterpret_cast<uint2*>(r8) = make_uint2(__byte_perm(o[0], o[1], 0x6420), __byte_perm(o[2], o[3], 0x6420));
          else
            *reinterpret_cast<uint32_t*>(r8) = __byte_perm(o[0], o[1], 0x6420);
        }
      }
    }
    __syncthreads();
    if (flags && tid == 0) {
      // the rows are in the CDEF planes: the half superblocks' flags
      uint32_t* fl = flags + f.cdef_flag_base + 2 * sr * f.cdef_sbc + sc;
      if (R == 64) {
        flag_set(fl);
        flag_set(fl + f.cdef_sbc);
      } else {
        flag_set(fl + item.a * f.cdef_sbc);
      }
    }
  }
  AV1PF_TRACE_END(2);
}

// Sum of a u32 over the warp, exactly (two 16-bit halves, so no lane sum
// overflows).
__device__ __forceinline__ uint64_t warp_sum_u32(uint32_t v) {
  const uint32_t lo = __reduce_add_sync(0xffffffffu, v & 0xffffu);
  const uint32_t hi = __reduce_add_sync(0xffffffffu, v >> 16);
  return (uint64_t(hi) << 16) + lo;
}

// The search's candidate strengths (encoder/cdef.rs:60-80): primaries of
// the fast and thorough lists, secondaries decoded (coded 3 is 4).
__host__ __device__ constexpr int search_y_pri(bool th, int i) {
  constexpr int f[7] = {0, 1, 2, 4, 6, 9, 12}, t[11] = {0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15};
  return th ? t[i] : f[i];
}
__host__ __device__ constexpr int search_uv_pri(bool th, int i) {
  constexpr int f[5] = {0, 1, 2, 4, 7}, t[8] = {0, 1, 2, 3, 4, 6, 8, 11};
  return th ? t[i] : f[i];
}
__host__ __device__ constexpr int search_sec(int j) { return j == 3 ? 4 : j; }

// |constrain(d)| (cdef.rs:48-51) from |d|: min(|d|, max(0, str - (|d| >> adj))).
// `mone` is -1 at run time but opaque to the compiler, so the subtraction
// is a multiply-add (the integer ALU pipe is this kernel's bound).
__device__ __forceinline__ int cmag(int ad, int str, int adj, int mone) {
  return min(ad, max((ad >> adj) * mone + str, 0));
}

// Window offsets of the secondary taps of direction 0 (the taps of the
// candidates with primary strength 0, whose direction is 0): directions 6
// and 2 (postfilter.rs:489-511).
constexpr int8_t kSearchDirs[8][2][2] = AV1T_CDEF_DIRECTIONS;
constexpr int kA0 = kSearchDirs[6][0][0] * kS + kSearchDirs[6][0][1];  // weight 2
constexpr int kA1 = kSearchDirs[2][0][0] * kS + kSearchDirs[2][0][1];  // weight 2
constexpr int kA2 = kSearchDirs[6][1][0] * kS + kSearchDirs[6][1][1];  // weight 1
constexpr int kA3 = kSearchDirs[2][1][0] * kS + kSearchDirs[2][1][1];  // weight 1

// The squared error of one sample under every (primary, secondary) pair of
// a plane's list, added to acc[i * NS + j] (encoder/cdef.rs:113-188).
// A pair's filter sum is P(primary) + S(secondary): the primary taps'
// constrained sum depends on the primary strength alone and the secondary
// taps' on the secondary strength alone, so each distinct P and S is
// computed once per sample and every pair costs a few adds. A tap's
// constrained difference is sign(d) * cmag(|d|): |d| and the signed weight
// are set once per sample. Pairs with primary strength 0 filter in
// direction 0 (secondary taps at directions 6 and 2); the others in the
// block's direction (offsets `o`: primary k0, k1, secondary lo k0, hi k0,
// lo k1, hi k1). The result is clamped to the block direction's available
// taps (cdef.rs:54-90); with one kind of tap (a zero primary or secondary
// strength) the weights sum to 12 < 16 and the result already lies within
// the taps' range, so those pairs skip the clamp.
template <int NP, int NS>
__device__ __forceinline__ void sample_pairs(const int16_t* c, int s, const int (&o)[6], const int (&pstr)[NP],
                                             const int (&padj)[NP], const int (&pw0)[NP], const int (&pw1)[NP],
                                             const int (&sstr)[NS], const int (&sadj)[NS], int one, int mone,
                                             uint32_t (&acc)[NP * NS]) {
  const int x = c[0];
  const int nx = x * mone, ns = s * mone;
  int aB[12], gB[12];  // |d|, and sign(d) (primary) or the signed weight (secondary)
  int mx = x;
  unsigned mn = unsigned(x);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int p0 = c[o[k]], p1 = c[-o[k]];
    mx = max(mx, max(p0, p1));
    mn = min(mn, min(unsigned(p0), unsigned(p1)));
    const int d0 = p0 * one + nx, d1 = p1 * one + nx;
    const int w = k < 2 ? 1 : (k < 4 ? 2 : 1);
    aB[2 * k] = abs(d0);
    aB[2 * k + 1] = abs(d1);
    gB[2 * k] = (d0 >> 31) * (2 * w) + w;
    gB[2 * k + 1] = (d1 >> 31) * (2 * w) + w;
  }
  int aA[8], gA[8];
  {
    const int offs[4] = {kA0, kA1, kA2, kA3};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int d0 = c[offs[k]] * one + nx, d1 = c[-offs[k]] * one + nx;
      const int w = k < 2 ? 2 : 1;
      aA[2 * k] = abs(d0);
      aA[2 * k + 1] = abs(d1);
      gA[2 * k] = (d0 >> 31) * (2 * w) + w;
      gA[2 * k + 1] = (d1 >> 31) * (2 * w) + w;
    }
  }
  // secondary sums per nonzero secondary strength, both directions
  int SA[NS], SB[NS];
  SA[0] = SB[0] = 0;
#pragma unroll
  for (int j = 1; j < NS; j++) {
    int sa = 0, sb = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      sa = gA[k] * cmag(aA[k], sstr[j], sadj[j], mone) + sa;
      sb = gB[4 + k] * cmag(aB[4 + k], sstr[j], sadj[j], mone) + sb;
    }
    SA[j] = sa;
    SB[j] = sb;
  }
  const int x16 = x * 16 + 8;  // x + round(sum / 16) = (x16 + sum - (sum < 0)) >> 4
#pragma unroll
  for (int j = 0; j < NS; j++) {  // primary strength 0: secondary taps alone
    const int v = (x16 + SA[j] + (SA[j] >> 31)) >> 4;
    const int e = v * one + ns;
    acc[j] = uint32_t(e * e) + acc[j];
  }
#pragma unroll
  for (int i = 1; i < NP; i++) {
    const int q0 = gB[0] * cmag(aB[0], pstr[i], padj[i], mone) + gB[1] * cmag(aB[1], pstr[i], padj[i], mone);
    const int q1 = gB[2] * cmag(aB[2], pstr[i], padj[i], mone) + gB[3] * cmag(aB[3], pstr[i], padj[i], mone);
    const int P = pw0[i] * q0 + pw1[i] * q1;
    {  // secondary strength 0: primary taps alone
      const int v = (x16 + P + (P >> 31)) >> 4;
      const int e = v * one + ns;
      acc[i * NS] = uint32_t(e * e) + acc[i * NS];
    }
#pragma unroll
    for (int j = 1; j < NS; j++) {
      const int sum = P * one + SB[j];
      const int v = min(max((x16 + sum + (sum >> 31)) >> 4, int(mn)), mx);
      const int e = v * one + ns;
      acc[i * NS + j] = uint32_t(e * e) + acc[i * NS + j];
    }
  }
}

// Strengths, damping adjustments and primary tap weights of one plane's
// list (postfilter.rs:489-511): pstr[i] is the primary strength after the
// block's variance adjustment (luma, postfilter.rs:318-323; `var` < 0 for
// chroma, which has none).
template <int NP, int NS, bool TH, bool LUMA>
__device__ __forceinline__ void pair_taps(int cs, int damping, int32_t var, int (&pstr)[NP], int (&padj)[NP],
                                          int (&pw0)[NP], int (&pw1)[NP], int (&sstr)[NS], int (&sadj)[NS]) {
  const int var_str = (var >> 6) != 0 ? min(floor_log2(uint32_t(var >> 6)), 12) : 0;
#pragma unroll
  for (int i = 0; i < NP; i++) {
    const int p0 = (LUMA ? search_y_pri(TH, i) : search_uv_pri(TH, i)) << cs;
    const int p = LUMA ? (var != 0 ? (p0 * (4 + var_str) + 8) >> 4 : 0) : p0;
    pstr[i] = p;
    padj[i] = p ? max(damping - floor_log2(uint32_t(p)), 0) : 0;
    const bool odd = (p >> cs) & 1;
    pw0[i] = odd ? 3 : 4;
    pw1[i] = odd ? 3 : 2;
  }
#pragma unroll
  for (int j = 0; j < NS; j++) {
    const int q = search_sec(j) << cs;
    sstr[j] = q;
    sadj[j] = q ? max(damping - floor_log2(uint32_t(q)), 0) : 0;
  }
}

// Block-direction offsets of the taps (primary k0, k1, secondary lo k0,
// hi k0, lo k1, hi k1) in window samples.
__device__ __forceinline__ void dir_offsets(const int16_t (*doff)[2], int dir, int (&o)[6]) {
  const int dlo = (dir + 6) & 7, dhi = (dir + 2) & 7;
  o[0] = doff[dir][0];
  o[1] = doff[dir][1];
  o[2] = doff[dlo][0];
  o[3] = doff[dhi][0];
  o[4] = doff[dlo][1];
  o[5] = doff[dhi][1];
}

// Adds warp sums of acc[] to red[warp][base + k].
template <int N>
__device__ __forceinline__ void warp_reduce_pairs(const uint32_t (&acc)[N], uint64_t (*red)[kSearchMaxY + kSearchMaxUV],
                                                  int warp, int lane, int base) {
#pragma unroll
  for (int k = 0; k < N; k++) {
    const uint64_t ws = warp_sum_u32(acc[k]);
    if (lane == 0) red[warp][base + k] = ws;
  }
}

// The encoder's CDEF search, error tables (encoder/cdef.rs:103-190): one CTA
// per 64x64 block, 256 threads. The block's planes are staged as in the
// decoder's kernel (2-sample border, kNA outside the mode-info area) with
// the source beside them (kNA outside the frame, so block_sse's crop,
// encoder/cdef.rs:261-285, is a test per sample); the direction search is
// the decoder's. Then each thread takes 16 luma samples of one 8x8 block
// (rows r and r + 4; a warp per row of blocks) and scores every pair on
// each (sample_pairs), the errors of each pair accumulating in a register;
// the chroma samples of the same block follow. TH: the thorough lists. The
// grid covers every block of n frames: frame i's blocks start at CTA
// ds[i].block0.
template <bool TH>
__global__ void __launch_bounds__(256, 2) cdef_search_kernel(const CdefSearchDesc* __restrict__ ds, int n) {
  constexpr int NYP = TH ? 11 : 7, NUVP = TH ? 8 : 5, NYS = 4, NUVS = 3;
  constexpr int NY = NYP * NYS, NUV = NUVP * NUVS;
  constexpr int R = 64, top = 2, wrows = R + 2 * top;
  extern __shared__ __align__(16) int16_t cs_smem[];
  auto win = [&](int p) { return cs_smem + p * wrows * kS; };                // reconstruction windows
  auto srcw = [&](int p) { return cs_smem + 3 * wrows * kS + p * R * kS; };  // source
  __shared__ int32_t cost[R][8];
  __shared__ uint8_t bstate[R];
  __shared__ uint8_t bdir[R];
  __shared__ int32_t bvar[R];
  __shared__ int16_t doff[8][2];
  __shared__ uint8_t uvdir[2][2][8];
  __shared__ int s_one;
  __shared__ uint64_t red[8][kSearchMaxY + kSearchMaxUV];
  int fi = 0;
  for (int hi = n - 1; fi < hi;) {  // the last frame whose first block is at or before this CTA
    const int mid = (fi + hi + 1) >> 1;
    if (ds[mid].block0 <= int(blockIdx.x))
      fi = mid;
    else
      hi = mid - 1;
  }
  const CdefSearchDesc& d = ds[fi];
  const FrameDesc& f = *d.frame;
  CdefGreedy* g = d.g;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int fb = int(blockIdx.x) - d.block0, nfb = d.fb_rows * d.fb_cols;
  const int fr = fb / d.fb_cols, fc = fb - fr * d.fb_cols;
  const int idx = f.cdef_idx[int64_t(fr) * f.cdef_stride + fc];
  if (idx < 0) {  // codes no index: zero errors, and no part in the greedy's sums
    for (int k = tid; k < NY + NUV; k += blockDim.x) d.sse[int64_t(k) * nfb + fb] = 0;
    if (tid == 0) d.best[fb] = 0;
    return;
  }
  if (tid == 0) {
    d.best[fb] = ~uint64_t(0);
    atomicAdd(&g->nb, 1u);
  }
  if (tid < 16) doff[tid >> 1][tid & 1] = int16_t(c_cdef_dirs[tid >> 1][tid & 1][0] * kS + c_cdef_dirs[tid >> 1][tid & 1][1]);
  if (tid < 32) (&uvdir[0][0][0])[tid] = (&c_cdef_uv_dir[0][0][0])[tid];
  if (tid == 0) s_one = 1;
  const int np = f.np, sb = f.sb, cs = f.bd - 8;
  // --- the 8x8 blocks CDEF filters (encoder/cdef.rs:106-112) ---
  if (tid < R) {
    const int by = tid >> 3, bx = tid & 7;
    const int r = fr * 16 + 2 * by, c = fc * 16 + 2 * bx;
    uint8_t st = 0;
    if (r < f.mi_rows && c < f.mi_cols) {
      const av1pf_mi* m = f.mi + int64_t(r) * f.mi_stride + c;
      const int ms = f.mi_stride;
      const bool skip = (m[0].skip_segment & AV1PF_MI_SKIP) && (m[ms].skip_segment & AV1PF_MI_SKIP) &&
                        (m[1].skip_segment & AV1PF_MI_SKIP) && (m[ms + 1].skip_segment & AV1PF_MI_SKIP);
      st = skip ? 0 : 2;
    }
    bstate[tid] = st;
  }
  // --- stage the reconstruction and the source ---
  for (int p = 0; p < np; p++) {
    if (plane_ssx(f, p))
      stage_plane<R, 1>(f, p, fc, fr * 64, top, win(p), tid);
    else
      stage_plane<R, 0>(f, p, fc, fr * 64, top, win(p), tid);
    const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
    const int pw = R >> sx, ph = R >> sy;
    const int fw = (f.fw + sx) >> sx, fh = (f.fh + sy) >> sy;
    const int x0 = (fc * 64) >> sx, y0 = (fr * 64) >> sy;
    int16_t* sp = srcw(p);
    for (int k = tid; k < pw * ph; k += blockDim.x) {
      const int r = k / pw, c = k - r * pw;
      const int gx = x0 + c, gy = y0 + r;
      sp[r * kS + c] = (gx < fw && gy < fh) ? int16_t(ld_sample(d.src[p], sb, gx, gy)) : kNA;
    }
  }
  __syncthreads();
  // --- direction search (postfilter.rs:345-401), as in the decoder's kernel ---
  {
    const int pair = warp & 3;
    const int b = (warp >> 2) * 32 + lane;
    if (bstate[b] == 2) {
      const int by = b >> 3, bx = b & 7;
      const int16_t* s = &win(0)[(top + by * 8) * kS + kColOff + bx * 8];
      int32_t c1, c2;
      switch (pair) {
        case 0: cdef_cost_pair<0>(s, cs, s_one, c1, c2); break;
        case 1: cdef_cost_pair<1>(s, cs, s_one, c1, c2); break;
        case 2: cdef_cost_pair<2>(s, cs, s_one, c1, c2); break;
        default: cdef_cost_pair<3>(s, cs, s_one, c1, c2); break;
      }
      cost[b][pair] = c1;
      cost[b][pair + 4] = c2;
    }
  }
  __syncthreads();
  if (tid < R && bstate[tid] == 2) {
    int32_t best = 0;
    int y_dir = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      if (cost[tid][k] > best) {
        best = cost[tid][k];
        y_dir = k;
      }
    }
    bdir[tid] = uint8_t(y_dir);
    bvar[tid] = (best - cost[tid][(y_dir + 4) & 7]) >> 10;
  }
  __syncthreads();
  // --- every pair on every filtered sample (encoder/cdef.rs:113-188) ---
  const int by = warp, bx = lane & 7, rr = lane >> 3;
  const int b = by * 8 + bx;
  const bool act = bstate[b] == 2;
  const int y_dir = act ? bdir[b] : 0;
  const int one = s_one;
  {
    int pstr[NYP], padj[NYP], pw0[NYP], pw1[NYP], sstr[NYS], sadj[NYS], o[6];
    pair_taps<NYP, NYS, TH, true>(cs, d.damping + cs, act ? bvar[b] : 0, pstr, padj, pw0, pw1, sstr, sadj);
    dir_offsets(doff, y_dir, o);
    uint32_t acc[NY];
#pragma unroll
    for (int k = 0; k < NY; k++) acc[k] = 0;
    if (act) {
      const int16_t* c = &win(0)[(top + by * 8 + rr) * kS + kColOff + bx * 8];
      const int16_t* sv = &srcw(0)[(by * 8 + rr) * kS + bx * 8];
      for (int q = 0; q < 2; q++)
        for (int j = 0; j < 8; j++) {
          const int sval = sv[q * 4 * kS + j];
          if (sval != kNA)
            sample_pairs<NYP, NYS>(c + q * 4 * kS + j, sval, o, pstr, padj, pw0, pw1, sstr, sadj, one, -one, acc);
        }
    }
    warp_reduce_pairs<NY>(acc, red, warp, lane, 0);
  }
  if (np > 1) {
    const int sx = f.ssx, sy = f.ssy;
    const int w = 8 >> sx, h = 8 >> sy;  // h is 4 or 8: rows rr (and rr + 4)
    int pstr[NUVP], padj[NUVP], pw0[NUVP], pw1[NUVP], sstr[NUVS], sadj[NUVS], o[6];
    pair_taps<NUVP, NUVS, TH, false>(cs, d.damping + cs - 1, 0, pstr, padj, pw0, pw1, sstr, sadj);
    dir_offsets(doff, uvdir[sx][sy][y_dir], o);
    uint32_t acc[NUV];
#pragma unroll
    for (int k = 0; k < NUV; k++) acc[k] = 0;
    if (act) {
      for (int p = 1; p < 3; p++) {
        const int16_t* c = &win(p)[(top + by * h + rr) * kS + kColOff + bx * w];
        const int16_t* sv = &srcw(p)[(by * h + rr) * kS + bx * w];
        for (int q = 0; q < h / 4; q++)
          for (int j = 0; j < w; j++) {
            const int sval = sv[q * 4 * kS + j];
            if (sval != kNA)
              sample_pairs<NUVP, NUVS>(c + q * 4 * kS + j, sval, o, pstr, padj, pw0, pw1, sstr, sadj, one, -one,
                                       acc);
          }
      }
    }
    warp_reduce_pairs<NUV>(acc, red, warp, lane, NY);
  }
  __syncthreads();
  for (int k = tid; k < NY + NUV; k += blockDim.x) {
    uint64_t s = 0;
    if (k < NY || np > 1)
      for (int w8 = 0; w8 < 8; w8++) s += red[w8][k];
    d.sse[int64_t(k) * nfb + fb] = s;
  }
}

constexpr int kSearchSmem = 3 * (64 + 4) * kS * 2 + 3 * 64 * kS * 2;

// dsp::cdef::filter (cdef.rs:29) on independent 12x12 windows: one CTA per
// window, one thread per output sample.
__global__ void dsp_cdef_kernel(const int32_t* __restrict__ win, const av1pf_cdef_taps* __restrict__ taps,
                                uint16_t* __restrict__ res, int n) {
  __shared__ int16_t w[144];
  const int e = blockIdx.x;
  if (e >= n) return;
  for (int k = threadIdx.x; k < 144; k += blockDim.x) {
    const int32_t v = win[int64_t(e) * 144 + k];
    w[k] = v == INT32_MIN ? kNA : int16_t(v);
  }
  __syncthreads();
  const av1pf_cdef_taps a = taps[e];
  const int i = threadIdx.x / 8, j = threadIdx.x % 8;
  if (i >= a.h || j >= a.w) return;
  TapsDev t;
  t.pri = a.pri_str;
  t.sec = a.sec_str;
  t.pri_adj = a.pri_adj;
  t.sec_adj = a.sec_adj;
  t.pt0 = a.pri_taps[0];
  t.pt1 = a.pri_taps[1];
  t.po0 = a.pri_off[0];
  t.po1 = a.pri_off[1];
  t.so00 = a.sec_off[0][0];
  t.so01 = a.sec_off[0][1];
  t.so10 = a.sec_off[1][0];
  t.so11 = a.sec_off[1][1];
  // The secondary weights are the taps' own (cdef.rs:79), not fixed.
  const int16_t* c = &w[(i + 2) * 12 + j + 2];
  const int x = c[0];
  int sum = 0, mx = x;
  unsigned mn = unsigned(x);
  cdef_tap(c[t.po0], -x, 1, -1, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[-t.po0], -x, 1, -1, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[t.so00], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[-t.so00], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[t.so01], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[-t.so01], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[t.po1], -x, 1, -1, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[-t.po1], -x, 1, -1, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[t.so10], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[-t.so10], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[t.so11], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[-t.so11], -x, 1, -1, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  const int v = x + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
  res[int64_t(e) * 64 + i * a.w + j] = uint16_t(min(max(v, int(mn)), mx));
}

cudaError_t cdef_init() {
  cudaError_t e = cudaFuncSetAttribute(cdef_kernel<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       cdef_smem(64, true));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cdef_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             cdef_smem(32, true));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cdef_kernel<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             cdef_smem(64, false));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cdef_kernel<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             cdef_smem(32, false));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cdef_search_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSearchSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cdef_search_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSearchSmem);
  return e;
}

void launch_cdef(const FrameDesc* frames, const Item* items, int n_items, bool lfh, bool half, uint32_t* flags,
                 cudaStream_t s) {
  if (n_items <= 0) return;
  // without the fused horizontal pass the windows hold 2 border rows each
  // side: smaller windows, more CTAs per SM
  const int R = half ? 32 : 64;
  const int wrows = R + 2 * (lfh ? kTopLfh : 2);
  const int grid = min(n_items, kItemGrid);
  if (half && lfh)
    launch_pdl(cdef_kernel<32, true>, grid, 128, size_t(cdef_smem(32, true)), s, frames, items, n_items, wrows, flags);
  else if (half)
    launch_pdl(cdef_kernel<32, false>, grid, 128, size_t(cdef_smem(32, false)), s, frames, items, n_items, wrows, flags);
  else if (lfh)
    launch_pdl(cdef_kernel<64, true>, grid, 256, size_t(cdef_smem(64, true)), s, frames, items, n_items, wrows, flags);
  else
    launch_pdl(cdef_kernel<64, false>, grid, 256, size_t(cdef_smem(64, false)), s, frames, items, n_items, wrows, flags);
}

void launch_cdef_search(const CdefSearchDesc* ds, int n, int blocks, bool thorough, cudaStream_t s) {
  if (blocks <= 0) return;
  if (thorough)
    cdef_search_kernel<true><<<blocks, 256, kSearchSmem, s>>>(ds, n);
  else
    cdef_search_kernel<false><<<blocks, 256, kSearchSmem, s>>>(ds, n);
  note_launch();
}

void launch_dsp_cdef(const int32_t* win, const av1pf_cdef_taps* taps, uint16_t* res, int n, cudaStream_t s) {
  if (n <= 0) return;
  dsp_cdef_kernel<<<n, 64, 0, s>>>(win, taps, res, n);
  note_launch();
}

}  // namespace av1pf
