// lr_search.cu — the encoder's loop-restoration search on the device
// (encoder/lr.rs:64-430): per restoration unit, the error of no filter, of
// a Wiener filter fitted to the source and of a self-guided filter fitted
// for each parameter set, priced with lambda; the cheapest is the unit's
// choice.
//
// One CTA per unit, 256 threads. Each of the unit's stripe rectangles is
// staged as the decoder's restoration window (postfilter.rs:765-777:
// clamped to the plane, rows beyond the stripe from the deblocked frame)
// in shared memory, once per phase.
//
// Exactness. The reference fits in f64, summing over the unit's samples in
// row-major order. Sums whose terms are integers (the first Wiener pass,
// whose lines are plain samples, and the self-guided fit, whose terms are
// products of filter outputs and samples) are exact in any order while the
// sum of the terms' magnitudes stays below 2^53: they are summed in int64
// in parallel (the self-guided sums check that bound and otherwise redo the
// sum in order on one thread). The second and third Wiener passes have
// real-valued terms, so their sums run in the reference's order: warps 1-3
// produce four rows of terms at a time into shared memory while lanes of
// warp 0 each add one accumulator's terms in sample order. Every f64 operation is a
// round-to-nearest multiply, add or divide in the reference's order (this
// file is compiled without floating-point contraction, and the sums use
// the explicit _rn intrinsics).
#include <cfloat>

#include "av1_tables.h"
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {

constexpr int kB = 3;            // window border (postfilter.rs:744 LRB)
constexpr int kSgrCachePx = 6144;  // filter outputs kept between the fit and its error (units up to 96 x 64)
constexpr int kThreads = 256;
constexpr int kWienerChunk = 4;  // rows of Wiener terms handed from the producing warps to the adding lanes at a time
constexpr int kWienerErrBand = 32;  // output rows per band of the Wiener error pass (its int16 rows fit the term region)
__constant__ int32_t kSgrParams[16][4] = AV1T_SGR_PARAMS;
__constant__ int32_t kWienerMin[3] = AV1T_WIENER_TAPS_MIN, kWienerMax[3] = AV1T_WIENER_TAPS_MAX;
__constant__ int32_t kXqdMin[2] = AV1T_SGRPROJ_XQD_MIN, kXqdMax[2] = AV1T_SGRPROJ_XQD_MAX;
constexpr uint64_t kExact = uint64_t(1) << 53;

__device__ __forceinline__ int ld(const DPlane& p, int sb, int x, int y) { return ld_sample(p, sb, x, y); }

// f64 -> i32 as Rust's `as` converts: saturating, NaN to 0.
__device__ __forceinline__ int32_t f64_to_i32(double x) {
  if (isnan(x)) return 0;
  if (x <= -2147483648.0) return INT32_MIN;
  if (x >= 2147483647.0) return INT32_MAX;
  return int32_t(x);
}

struct Win {
  const int16_t* w;
  int ws;  // row stride
  __device__ __forceinline__ int at(int r, int c) const { return w[r * ws + c]; }
};

// lr_window (postfilter.rs:765-777) of rectangle `rc` into shared memory.
__device__ void stage_window(const LrSearchFrame& d, int p, const LrSearchRect& rc, int x0, int w, int16_t* win,
                             int ws, int16_t* srcw = nullptr) {
  // a warp per window row, lanes along it (no index division), eight rows'
  // loads in flight before their stores; with `srcw`, the rectangle's source
  // samples too (row stride w)
  constexpr int kR = 8;
  const int ww = w + 2 * kB, wh = rc.h + 2 * kB, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  const int pex = d.pex[p], pey = d.pey[p];
  const int rows_all = wh + (srcw ? rc.h : 0);
  for (int r0 = threadIdx.x >> 5; r0 < rows_all; r0 += kR * nw) {
    for (int c = lane; c < ww; c += 32) {
      int v[kR];
#pragma unroll
      for (int m = 0; m < kR; m++) {
        const int r = r0 + m * nw;
        v[m] = 0;
        if (r < wh) {
          const int y = max(min(rc.y0 + r - kB, pey), 0);
          const DPlane& pl = y < rc.ss || y > rc.se ? d.cur[p] : d.cdef[p];
          const int yy = y < rc.ss ? max(rc.ss - 2, y) : (y > rc.se ? min(rc.se + 2, y) : y);
          v[m] = ld(pl, d.sb, max(min(x0 + c - kB, pex), 0), yy);
        } else if (r < rows_all && c < w) {
          v[m] = ld(d.src[p], d.sb, x0 + c, rc.y0 + r - wh);
        }
      }
#pragma unroll
      for (int m = 0; m < kR; m++) {
        const int r = r0 + m * nw;
        if (r < wh)
          win[r * ws + c] = int16_t(v[m]);
        else if (r < rows_all && c < w)
          srcw[(r - wh) * w + c] = int16_t(v[m]);
      }
    }
  }
}

// Block sum of 64-bit values (every thread gets the result).
__device__ int64_t block_sum_i64(int64_t v, int64_t* red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int64_t t = 0;
  for (int w = 0; w < kThreads / 32; w++) t += red[w];
  __syncthreads();
  return t;
}

// Block sums of N 64-bit values in one round (every thread gets the totals).
template <int N>
__device__ void block_sums_i64(int64_t (&v)[N], int64_t (*red)[kThreads / 32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < N; q++) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0) red[q][warp] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; q++) {
    int64_t t = 0;
    for (int k = 0; k < nw; k++) t += red[q][k];
    v[q] = t;
  }
}

// Gaussian elimination with partial pivoting (encoder/lr.rs:212-233): the
// last row of largest magnitude is the pivot (Iterator::max_by); zeros when
// singular.
template <int N>
__device__ __noinline__ void solve(double (&m)[N][N], double (&v)[N], double (&x)[N]) {
  for (int i = 0; i < N; i++) {
    int piv = i;
    for (int a = i + 1; a < N; a++)
      if (!(fabs(m[a][i]) < fabs(m[piv][i]))) piv = a;
    for (int c = 0; c < N; c++) {
      const double t = m[i][c];
      m[i][c] = m[piv][c];
      m[piv][c] = t;
    }
    const double tv = v[i];
    v[i] = v[piv];
    v[piv] = tv;
    if (fabs(m[i][i]) < 1e-9) {
      for (int k = 0; k < N; k++) x[k] = 0.0;
      return;
    }
    for (int r = 0; r < N; r++) {
      if (r != i) {
        const double f = __ddiv_rn(m[r][i], m[i][i]);
        for (int c = i; c < N; c++) m[r][c] = __dsub_rn(m[r][c], __dmul_rn(f, m[i][c]));
        v[r] = __dsub_rn(v[r], __dmul_rn(f, v[i]));
      }
    }
  }
  for (int i = 0; i < N; i++) x[i] = __ddiv_rn(v[i], m[i][i]);
}

// The 7 samples of a Wiener line at (i, j) with the other direction's
// filter applied first (encoder/lr.rs:265-285); the line's taps run along
// columns (vertical) or rows.
__device__ __forceinline__ void wiener_line(const Win& W, bool vertical, int i, int j, const double* other,
                                            double (&line)[7]) {
#pragma unroll
  for (int t = 0; t < 7; t++) {
    const int r = vertical ? i + t : i + kB, c = vertical ? j + kB : j + t;
    const int center = W.at(r, c);
    double s = double(center);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int dd = 3 - k;
      const int a = vertical ? W.at(r, c - dd) : W.at(r - dd, c);
      const int b = vertical ? W.at(r, c + dd) : W.at(r + dd, c);
      // a + b - 2 * center is an integer below 2^17: the f64 expression of
      // encoder/lr.rs is exact, so integer arithmetic gives the same value
      s = __dadd_rn(s, __dmul_rn(other[k], double(a + b - 2 * center)));
    }
    line[t] = s;
  }
}

// One self-guided A/B pair (postfilter.rs:918-948) at A/B position (ai, aj)
// of the rectangle (window position ai + 2, aj + 2).
__device__ __forceinline__ void sgr_ab(const Win& W, int ai, int aj, int r, int n, int s, int one_over_n, int bd,
                                       int32_t& A, int32_t& B) {
  const int wy = ai + kB - 1, wx = aj + kB - 1;
  int32_t bs = 0;
  int64_t as = 0;
  for (int dy = -r; dy <= r; dy++)
    for (int dx = -r; dx <= r; dx++) {
      const int v = W.at(wy + dy, wx + dx);
      bs += v;
      as += int64_t(v) * v;
    }
  const int64_t a = round2_64(as, 2 * (bd - 8));
  const int64_t dd = round2(bs, bd - 8);
  const int64_t p = max(a * n - dd * dd, int64_t(0));
  const int64_t z = round2_64(p * s, 20);  // SGRPROJ_MTABLE_BITS
  const int zc = int(min(z, int64_t(255)));
  const int32_t a2 = zc >= 255 ? 256 : (zc == 0 ? 1 : ((zc << 8) + zc / 2) / (zc + 1));
  const int64_t b2 = int64_t(256 - a2) * int64_t(bs) * int64_t(one_over_n);
  A = a2;
  B = int32_t(round2_64(b2, 12));  // SGRPROJ_RECIP_BITS
}

struct SgrPass {
  int r, n, s, one_over_n;
};

__device__ __forceinline__ SgrPass sgr_pass(int set, int pass) {
  SgrPass q;
  q.r = kSgrParams[set][pass * 2];
  const int eps = kSgrParams[set][pass * 2 + 1];
  q.n = (2 * q.r + 1) * (2 * q.r + 1);
  const int n2e = q.n * q.n * eps;
  q.s = q.r ? ((1 << 20) + n2e / 2) / n2e : 0;
  q.one_over_n = ((1 << 12) + q.n / 2) / q.n;
  return q;
}

// A self-guided filter output (postfilter.rs:950-988) at (i, j) from A/B
// rows held in shared memory (`ab`: rows ai0.., stride aw; A then B).
__device__ __forceinline__ int32_t sgr_flt(int pass, int yabs, int i_rel, int j, const int32_t* Ab, const int32_t* Bb,
                                           int aw, int cval) {
  int32_t a = 0, b = 0;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++) {
#pragma unroll
    for (int dx = -1; dx <= 1; dx++) {
      int wgt;
      if (pass == 0)
        wgt = ((yabs + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
      else
        wgt = (dx == 0 || dy == 0) ? 4 : 3;
      if (wgt) {
        const int k = (i_rel + 1 + dy) * aw + (j + 1 + dx);
        a += wgt * Ab[k];
        b += wgt * Bb[k];
      }
    }
  }
  const int shift = (pass == 0 && (yabs & 1)) ? 4 : 5;
  return round2(a * cval + b, 8 + shift - 4);
}

// The same output with A/B computed on the spot (the in-order fallback).
__device__ int32_t sgr_flt_direct(const Win& W, int pass, const SgrPass& q, int bd, int yabs, int i, int j, int cval) {
  int32_t a = 0, b = 0;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      int wgt;
      if (pass == 0)
        wgt = ((yabs + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
      else
        wgt = (dx == 0 || dy == 0) ? 4 : 3;
      if (wgt) {
        int32_t A, B;
        sgr_ab(W, i + 1 + dy, j + 1 + dx, q.r, q.n, q.s, q.one_over_n, bd, A, B);
        a += wgt * A;
        b += wgt * B;
      }
    }
  const int shift = (pass == 0 && (yabs & 1)) ? 4 : 5;
  return round2(a * cval + b, 8 + shift - 4);
}

// SGR_A2 (postfilter.rs:884-898), built at compile time.
struct LrsA2 {
  int32_t v[256];
};
constexpr LrsA2 make_lrs_a2() {
  LrsA2 t{};
  for (int z = 0; z < 256; z++) t.v[z] = z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
  return t;
}
__device__ const LrsA2 g_lrs_a2 = make_lrs_a2();

// Fills A/B rows for output rows [i0, i0 + rows) of a rectangle (A/B rows
// i0 .. i0 + rows + 1) for one pass (postfilter.rs:918-948), with separable
// box sums: first each window row's horizontal sums of the samples and of
// their squares (int32: 25 squares of 12-bit samples fit), then the
// vertical sums. Pass 0 computes odd absolute rows only (the others have
// weight 0). `hs`/`hq` hold (rows + 2 + 2r) x (w + 2) sums.
// The vertical half: A/B rows 0 .. rows + 1 of the band from the window
// rows' horizontal sums `hs`/`hq` (rows + 2 + 2r rows of stride w + 2).
template <int r>
__device__ __forceinline__ void sgr_vert_ab(const SgrPass& q, int pass, int bd, int y0, int i0, int rows, int w,
                                            int32_t* Ab, int32_t* Bb, int aw, const int32_t* hs, const int32_t* hq) {
  // n and 1/n follow from the radius (sgr_pass computes the same values)
  constexpr int n = (2 * r + 1) * (2 * r + 1), one_over_n = ((1 << 12) + n / 2) / n;
  const int cw = w + 2;
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sh = 2 * (bd - 8);
  for (int ir = warp; ir < rows + 2; ir += nw) {
    if (pass == 0 && ((y0 + i0 + ir - 1) & 1) == 0) continue;
    for (int aj = lane; aj < cw; aj += 32) {
      int32_t bs = 0, as = 0;
#pragma unroll
      for (int dy = 0; dy <= 2 * r; dy++) {
        bs += hs[(ir + dy) * cw + aj];
        as += hq[(ir + dy) * cw + aj];
      }
      // a * n and dd^2 stay below 2^31 (25 * 25 * 255^2); p * s needs 64 bits
      const int32_t a = round2(as, sh);
      const int32_t dd = round2(bs, bd - 8);
      const int32_t p = max(a * n - dd * dd, 0);
      const int64_t z = (int64_t(p) * q.s + (int64_t(1) << 19)) >> 20;  // SGRPROJ_MTABLE_BITS
      const int32_t a2 = g_lrs_a2.v[z < 255 ? int(z) : 255];
      const int64_t b2 = int64_t((256 - a2) * bs) * one_over_n;
      Ab[ir * aw + aj] = a2;
      Bb[ir * aw + aj] = int32_t((b2 + (1 << 11)) >> 12);  // SGRPROJ_RECIP_BITS
    }
  }
}

// Fills A/B rows for output rows [i0, i0 + rows) of a rectangle (A/B rows
// i0 .. i0 + rows + 1) for one pass (postfilter.rs:918-948), with separable
// box sums: first each window row's horizontal sums of the samples and of
// their squares (int32: 25 squares of 12-bit samples fit), then the
// vertical sums. Pass 0 computes odd absolute rows only (the others have
// weight 0). `hs`/`hq` hold (rows + 2 + 2r) x (w + 2) sums.
template <int r>
__device__ void sgr_band_ab_r(const Win& W, const SgrPass& q, int pass, int bd, int y0, int i0, int rows, int w,
                              int32_t* Ab, int32_t* Bb, int aw, int32_t* hs, int32_t* hq) {
  const int cw = w + 2;
  const int nrow = rows + 2 + 2 * r, wy0 = i0 + kB - 1 - r;
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // the previous users of hs / hq are done
  for (int rr = warp; rr < nrow; rr += nw) {
    const int wy = wy0 + rr;
    for (int aj = lane; aj < cw; aj += 32) {
      const int wx = aj + kB - 1;
      int32_t sum = 0, sq = 0;
#pragma unroll
      for (int dx = -r; dx <= r; dx++) {
        const int v = W.at(wy, wx + dx);
        sum += v;
        sq += v * v;
      }
      hs[rr * cw + aj] = sum;
      hq[rr * cw + aj] = sq;
    }
  }
  __syncthreads();
  sgr_vert_ab<r>(q, pass, bd, y0, i0, rows, w, Ab, Bb, aw, hs, hq);
}

// Both passes of a band (pass 0 of radius 2, pass 1 of radius 1) from one
// horizontal sweep: a row's 3-wide sums are the middle of its 5-wide ones.
// `hs5`/`hq5` hold rows + 6 rows, `hs3`/`hq3` rows + 4 (window rows one
// lower).
__device__ void sgr_band_ab_both(const Win& W, const SgrPass& q0, const SgrPass& q1, int bd, int y0, int i0, int rows,
                                 int w, int32_t* Ab0, int32_t* Bb0, int32_t* Ab1, int32_t* Bb1, int aw, int32_t* hs5,
                                 int32_t* hq5, int32_t* hs3, int32_t* hq3) {
  const int cw = w + 2;
  const int nrow = rows + 6, wy0 = i0 + kB - 3;
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // the previous users of the sums are done
  for (int rr = warp; rr < nrow; rr += nw) {
    const int wy = wy0 + rr;
    const bool mid = rr >= 1 && rr < nrow - 1;  // also a row of the radius-1 sums (row rr - 1)
    for (int aj = lane; aj < cw; aj += 32) {
      const int wx = aj + kB - 1;
      const int v0 = W.at(wy, wx - 2), v1 = W.at(wy, wx - 1), v2 = W.at(wy, wx), v3 = W.at(wy, wx + 1),
                v4 = W.at(wy, wx + 2);
      const int32_t s3 = v1 + v2 + v3, q3 = v1 * v1 + v2 * v2 + v3 * v3;
      hs5[rr * cw + aj] = s3 + v0 + v4;
      hq5[rr * cw + aj] = q3 + v0 * v0 + v4 * v4;
      if (mid) {
        hs3[(rr - 1) * cw + aj] = s3;
        hq3[(rr - 1) * cw + aj] = q3;
      }
    }
  }
  __syncthreads();
  sgr_vert_ab<2>(q0, 0, bd, y0, i0, rows, w, Ab0, Bb0, aw, hs5, hq5);
  sgr_vert_ab<1>(q1, 1, bd, y0, i0, rows, w, Ab1, Bb1, aw, hs3, hq3);
}

// The band's A/B for the pass's radius (1 or 2): the box sums' loops unrolled.
__device__ __forceinline__ void sgr_band_ab(const Win& W, const SgrPass& q, int pass, int bd, int y0, int i0, int rows,
                                            int w, int32_t* Ab, int32_t* Bb, int aw, int32_t* hs, int32_t* hq) {
  if (q.r == 2)
    sgr_band_ab_r<2>(W, q, pass, bd, y0, i0, rows, w, Ab, Bb, aw, hs, hq);
  else
    sgr_band_ab_r<1>(W, q, pass, bd, y0, i0, rows, w, Ab, Bb, aw, hs, hq);
}

}  // namespace

// Shared memory of a search kernel: the window, then a region used as the
// Wiener pass's term rows or the self-guided A/B bands.
size_t lr_window_bytes(int wmax, int hmax) {
  const size_t ws = size_t(wmax + 2 * kB + 1) & ~size_t(1);
  return ((size_t(hmax + 2 * kB) * ws * 2) + 15) & ~size_t(15);
}
size_t lr_search_smem(int wmax, int hmax, int kind, int band, int cache_px, int both) {
  const size_t win = lr_window_bytes(wmax, hmax);
  if (kind == 0) return win;  // the first-pass kernel
  if (kind == 1) return win + size_t(2) * 4 * kWienerChunk * size_t(wmax + 1) * sizeof(double);  // Wiener passes
  // self-guided: A/B of both passes, the band's box sums, the filter-output cache
  return win + size_t(4) * (band + 2) * size_t(wmax + 2) * sizeof(int32_t) +
         size_t(2) * (band + 6) * size_t(wmax + 2) * sizeof(int32_t) +
         size_t(both ? 2 : 0) * (band + 4) * size_t(wmax + 2) * sizeof(int32_t) +
         size_t(cache_px) * 2 * sizeof(int32_t) +
         ((size_t(hmax) * size_t(wmax) * sizeof(int16_t) + 15) & ~size_t(15));
}

void lr_search_shape(int wmax, int hmax, int upx_max, int& band, int& cache_px, int& both) {
  // Filter outputs are kept when every unit's fit fits the cache; then the
  // tallest band that leaves room for two CTAs per SM, else the tallest that
  // fits at all; the one-sweep box sums where their buffers fit beside that
  // band.
  constexpr size_t kTwo = 113 * 1024, kLimit = 220 * 1024;
  cache_px = upx_max <= kSgrCachePx ? upx_max : 0;
  for (size_t lim : {kTwo, kLimit})
    for (band = 32; band >= 4; band /= 2)
      for (both = 1; both >= 0; both--)
        if (lr_search_smem(wmax, hmax, 2, band, cache_px, both) <= lim) return;
  band = 4;
  cache_px = 0;
  both = 0;
}

namespace {

// Window stride and the region after the window.
struct Smem {
  int16_t* win;
  int ws;
  uint8_t* region;
};
__device__ __forceinline__ Smem smem_of(uint8_t* base, const LrSearchDesc& d) {
  Smem m;
  m.ws = (d.wmax + 2 * kB + 1) & ~1;
  m.win = reinterpret_cast<int16_t*>(base);
  m.region = base + ((((size_t(d.hmax + 2 * kB) * m.ws * 2) + 15) & ~size_t(15)));
  return m;
}

}  // namespace

// For units of several stripe rectangles, one CTA per unit (256 threads):
// the error without a filter (encoder/lr.rs:134-146), and the first Wiener
// pass (vertical, the other direction's filter still zero: its lines are
// plain samples, so its sums are exact integer sums in any order) and its
// solve. A one-rectangle unit's Wiener CTA does this itself, on the window
// it keeps for its other passes.
__global__ void __launch_bounds__(kThreads, 2) lr_search_prep_kernel(const LrSearchDesc d) {
  extern __shared__ __align__(16) uint8_t lrs_smem[];
  __shared__ int64_t red10[10][kThreads / 32];
  const LrSearchJob job = d.jobs[blockIdx.x];
  if (job.nr == 1) return;
  const LrSearchFrame& F = d.frames[job.frame];
  const int p = job.plane, x0 = job.x0, w = job.w, sb = F.sb, tid = threadIdx.x, step = d.step;
  const Smem sm = smem_of(lrs_smem, d);
  const Win W{sm.win, sm.ws};
  const LrSearchRect* rects = d.rects + job.r0;
  LrJobState& st = d.state[blockIdx.x];
  int64_t acc = 0, m00 = 0, m01 = 0, m02 = 0, m11 = 0, m12 = 0, m22 = 0, v0 = 0, v1 = 0, v2 = 0;
  const int nci = (w + step - 1) / step;
  for (int ri = 0; ri < job.nr; ri++) {
    const LrSearchRect rc = rects[ri];
    __syncthreads();
    stage_window(F, p, rc, x0, w, sm.win, sm.ws);
    __syncthreads();
    // no filter: the window's interior is the rectangle's CDEF output (its
    // rows lie in its stripe, its columns in the plane)
    for (int i = tid >> 5; i < rc.h; i += blockDim.x >> 5)
      for (int j = tid & 31; j < w; j += 32) {
        const int e = W.at(i + kB, j + kB) - ld(F.src[p], sb, x0 + j, rc.y0 + i);
        acc += int64_t(e) * e;
      }
    const int nri = (rc.h + step - 1) / step;
    for (int ii = tid >> 5; ii < nri; ii += blockDim.x >> 5)
      for (int jj = tid & 31; jj < nci; jj += 32) {
      const int i = ii * step, j = jj * step;
      int ln[7];
#pragma unroll
      for (int t = 0; t < 7; t++) ln[t] = W.at(i + t, j + kB);
      const int64_t tg = ld(F.src[p], sb, x0 + j, rc.y0 + i) - ln[3];
      const int64_t d0 = ln[0] + ln[6] - 2 * ln[3], d1 = ln[1] + ln[5] - 2 * ln[3], d2 = ln[2] + ln[4] - 2 * ln[3];
      m00 += d0 * d0;
      m01 += d0 * d1;
      m02 += d0 * d2;
      m11 += d1 * d1;
      m12 += d1 * d2;
      m22 += d2 * d2;
      v0 += d0 * tg;
      v1 += d1 * tg;
      v2 += d2 * tg;
      }
  }
  int64_t sums[10] = {m00, m01, m02, m11, m12, m22, v0, v1, v2, acc};
  block_sums_i64(sums, red10);
  double tot[9];
#pragma unroll
  for (int q = 0; q < 9; q++) tot[q] = double(sums[q]);
  if (tid == 0) {
    st.none = uint64_t(sums[9]);
    double sol[3] = {0.0, 0.0, 0.0};
    if (p == 0) {
      double m[3][3] = {{tot[0], tot[1], tot[2]}, {tot[1], tot[3], tot[4]}, {tot[2], tot[4], tot[5]}};
      double v[3] = {tot[6], tot[7], tot[8]};
      solve<3>(m, v, sol);
    } else {
      double m[2][2] = {{tot[3], tot[4]}, {tot[4], tot[5]}}, v[2] = {tot[7], tot[8]}, x2[2];
      solve<2>(m, v, x2);
      sol[1] = x2[0];
      sol[2] = x2[1];
    }
    for (int k = 0; k < 3; k++) st.vc[k] = sol[k];
  }
}

// One CTA per unit (128 threads). For a one-rectangle unit, first the error
// without a filter and the first Wiener pass and its solve, as the kernel
// above does for the others. Then the second
// (horizontal) and third (vertical) Wiener passes, whose terms are
// real-valued, so each of their sums runs in the reference's sample order:
// warps 1-3 produce four rows of terms into shared memory (two buffers)
// while lane q of warp 0 adds accumulator q's terms (m00 m01 m02 m11 m12 m22
// v0 v1 v2). Then the solves, the quantised coefficients
// (encoder/lr.rs:316-327) and the filter's error.
__global__ void __launch_bounds__(128, 4) lr_search_wiener_kernel(const LrSearchDesc d) {
  extern __shared__ __align__(16) uint8_t lrs_smem[];
  __shared__ int64_t red[4];
  __shared__ int64_t red10[10][kThreads / 32];
  __shared__ double s_m[3][3], s_v[3], s_other[3], s_vc[3];
  __shared__ int s_coef[2][3];
  const LrSearchJob job = d.jobs[blockIdx.x];
  const LrSearchFrame& F = d.frames[job.frame];
  const int p = job.plane, x0 = job.x0, w = job.w, sb = F.sb, tid = threadIdx.x, step = d.step;
  const int lane = tid & 31, warp = tid >> 5;
  const Smem sm = smem_of(lrs_smem, d);
  const Win W{sm.win, sm.ws};
  const LrSearchRect* rects = d.rects + job.r0;
  LrJobState& st = d.state[blockIdx.x];
  const int first = p == 0 ? 0 : 1;
  const int bd = F.bd, maxv = (1 << bd) - 1;
  const int nci = (w + step - 1) / step;
  if (job.nr == 1) {  // the no-filter error and the first pass (CTA-uniform)
    int64_t acc = 0, m00 = 0, m01 = 0, m02 = 0, m11 = 0, m12 = 0, m22 = 0, v0 = 0, v1 = 0, v2 = 0;
    for (int ri = 0; ri < job.nr; ri++) {
      const LrSearchRect rc = rects[ri];
      __syncthreads();
      stage_window(F, p, rc, x0, w, sm.win, sm.ws);
      __syncthreads();
      // no filter: the window's interior is the rectangle's CDEF output (its
      // rows lie in its stripe, its columns in the plane)
      for (int i = tid >> 5; i < rc.h; i += blockDim.x >> 5)
        for (int j = tid & 31; j < w; j += 32) {
          const int e = W.at(i + kB, j + kB) - ld(F.src[p], sb, x0 + j, rc.y0 + i);
          acc += int64_t(e) * e;
        }
      const int nri = (rc.h + step - 1) / step;
      for (int ii = tid >> 5; ii < nri; ii += blockDim.x >> 5)
        for (int jj = tid & 31; jj < nci; jj += 32) {
        const int i = ii * step, j = jj * step;
        int ln[7];
#pragma unroll
        for (int t = 0; t < 7; t++) ln[t] = W.at(i + t, j + kB);
        const int64_t tg = ld(F.src[p], sb, x0 + j, rc.y0 + i) - ln[3];
        const int64_t d0 = ln[0] + ln[6] - 2 * ln[3], d1 = ln[1] + ln[5] - 2 * ln[3], d2 = ln[2] + ln[4] - 2 * ln[3];
        m00 += d0 * d0;
        m01 += d0 * d1;
        m02 += d0 * d2;
        m11 += d1 * d1;
        m12 += d1 * d2;
        m22 += d2 * d2;
        v0 += d0 * tg;
        v1 += d1 * tg;
        v2 += d2 * tg;
        }
    }
    int64_t sums[10] = {m00, m01, m02, m11, m12, m22, v0, v1, v2, acc};
    block_sums_i64(sums, red10);
    if (tid == 0) {
      st.none = uint64_t(sums[9]);
      double sol[3] = {0.0, 0.0, 0.0};
      const double tot[9] = {double(sums[0]), double(sums[1]), double(sums[2]), double(sums[3]), double(sums[4]),
                             double(sums[5]), double(sums[6]), double(sums[7]), double(sums[8])};
      if (p == 0) {
        double m[3][3] = {{tot[0], tot[1], tot[2]}, {tot[1], tot[3], tot[4]}, {tot[2], tot[4], tot[5]}};
        double v[3] = {tot[6], tot[7], tot[8]};
        solve<3>(m, v, sol);
      } else {
        double m[2][2] = {{tot[3], tot[4]}, {tot[4], tot[5]}}, v[2] = {tot[7], tot[8]}, x2[2];
        solve<2>(m, v, x2);
        sol[1] = x2[0];
        sol[2] = x2[1];
      }
      for (int k = 0; k < 3; k++) s_vc[k] = sol[k];
    }
  } else if (tid < 3) {
    s_vc[tid] = st.vc[tid];  // from the kernel above
  }
  __syncthreads();
  double vc[3] = {s_vc[0], s_vc[1], s_vc[2]}, hc[3] = {0.0, 0.0, 0.0};
  const int qa = lane < 6 ? (lane < 3 ? 0 : (lane < 5 ? 1 : 2)) : lane - 6;
  const int qb = lane < 6 ? (lane < 3 ? lane : (lane < 5 ? lane - 2 : 2)) : 3;  // 3: the target
  const bool owner = warp == 0 && lane < 9 && qa >= first && (qb == 3 || qb >= first);
  // [2 buffers][4 terms: d0 d1 d2 t][kWienerChunk rows][wmax + 1]: the odd
  // row stride puts the four terms of a sample on different banks for the
  // accumulating lanes
  double* terms = reinterpret_cast<double*>(sm.region);
  const int ts = d.wmax + 1, tq_stride = kWienerChunk * ts;
  for (int iter = 1; iter < 3; iter++) {
    const bool vertical = iter == 2;
    if (tid < 3) s_other[tid] = vertical ? hc[tid] : vc[tid];
    double macc = 0.0;
    for (int ri = 0; ri < job.nr; ri++) {
      const LrSearchRect rc = rects[ri];
      __syncthreads();
      // one rectangle: its window, staged for the first pass, stays in place
      // (the term rows and band rows lie outside it)
      if (job.nr > 1) stage_window(F, p, rc, x0, w, sm.win, sm.ws);
      __syncthreads();
      const int nri = (rc.h + step - 1) / step, nch = (nri + kWienerChunk - 1) / kWienerChunk;
      // chunks of rows in turn, two buffers: warps 1.. fill chunk c + 1 while
      // warp 0 adds chunk c, row by row in sample order
      for (int ch = 0; ch <= nch; ch++) {
        if (ch < nch && warp > 0) {
          double* tb = terms + (ch & 1) * 4 * tq_stride;
          const int rows = min(kWienerChunk, nri - ch * kWienerChunk);
          const double oth[3] = {s_other[0], s_other[1], s_other[2]};
          for (int k = tid - 32; k < rows * nci; k += blockDim.x - 32) {
            const int r = k / nci, jj = k - r * nci;
            const int i = (ch * kWienerChunk + r) * step, j = jj * step;
            double line[7];
            wiener_line(W, vertical, i, j, oth, line);
            const double two3 = __dmul_rn(2.0, line[3]);
            double* tr = tb + r * ts + jj;
            tr[0 * tq_stride] = __dsub_rn(__dadd_rn(line[0], line[6]), two3);
            tr[1 * tq_stride] = __dsub_rn(__dadd_rn(line[1], line[5]), two3);
            tr[2 * tq_stride] = __dsub_rn(__dadd_rn(line[2], line[4]), two3);
            tr[3 * tq_stride] = __dsub_rn(double(ld(F.src[p], sb, x0 + j, rc.y0 + i)), line[3]);
          }
        }
        if (ch > 0 && owner) {
          const double* tb = terms + ((ch - 1) & 1) * 4 * tq_stride;
          const int rows = min(kWienerChunk, nri - (ch - 1) * kWienerChunk);
          for (int r = 0; r < rows; r++) {
            const double* ta = tb + qa * tq_stride + r * ts;
            const double* tq = tb + qb * tq_stride + r * ts;
            // the products of 8 terms are independent of the sum: form them
            // first, then add them one after another in sample order
            int jj = 0;
            for (; jj + 8 <= nci; jj += 8) {
              double pr[8];
#pragma unroll
              for (int u = 0; u < 8; u++) pr[u] = __dmul_rn(ta[jj + u], tq[jj + u]);
#pragma unroll
              for (int u = 0; u < 8; u++) macc = __dadd_rn(macc, pr[u]);
            }
            for (; jj < nci; jj++) macc = __dadd_rn(macc, __dmul_rn(ta[jj], tq[jj]));
          }
        }
        __syncthreads();
      }
    }
    if (owner) {
      if (qb == 3)
        s_v[qa] = macc;
      else
        s_m[qa][qb] = s_m[qb][qa] = macc;
    }
    __syncthreads();
    if (tid == 0) {
      double sol[3] = {0.0, 0.0, 0.0};
      if (first == 0) {
        double m[3][3], v[3];
        for (int a = 0; a < 3; a++) {
          v[a] = s_v[a];
          for (int b = 0; b < 3; b++) m[a][b] = s_m[a][b];
        }
        solve<3>(m, v, sol);
      } else {
        double m[2][2] = {{s_m[1][1], s_m[1][2]}, {s_m[2][1], s_m[2][2]}}, v[2] = {s_v[1], s_v[2]}, x2[2];
        solve<2>(m, v, x2);
        sol[1] = x2[0];
        sol[2] = x2[1];
      }
      for (int k = 0; k < 3; k++) s_other[k] = sol[k];  // the pass's solution
    }
    __syncthreads();
    for (int k = 0; k < 3; k++) (vertical ? vc : hc)[k] = s_other[k];
    __syncthreads();
  }
  if (tid == 0) {
    for (int k = 0; k < 3; k++) {
      s_coef[0][k] = k < first ? 0 : min(max(f64_to_i32(round(vc[k] * 128.0)), kWienerMin[k]), kWienerMax[k]);
      s_coef[1][k] = k < first ? 0 : min(max(f64_to_i32(round(hc[k] * 128.0)), kWienerMin[k]), kWienerMax[k]);
    }
  }
  __syncthreads();
  // the Wiener filter's error (postfilter.rs:781-822 restoration)
  int vf[7], hf[7];
  vf[3] = hf[3] = 128;
  for (int k = 0; k < 3; k++) {
    vf[k] = vf[6 - k] = s_coef[0][k];
    hf[k] = hf[6 - k] = s_coef[1][k];
    vf[3] -= 2 * s_coef[0][k];
    hf[3] -= 2 * s_coef[1][k];
  }
  const int round0 = bd == 12 ? 5 : 3, round1 = bd == 12 ? 9 : 11;
  const int off = 1 << (bd + 7 - round0 - 1), lim = (1 << (bd + 1 + 7 - round0)) - 1;
  // separable: each band's horizontally filtered window rows go to the term
  // region as int16 (clipped to [-off, lim - off], within [-2^13, 2^15)),
  // then the vertical taps run over them
  int16_t* hrow = reinterpret_cast<int16_t*>(sm.region);
  const int nw = blockDim.x >> 5;
  int64_t acc = 0;
  for (int ri = 0; ri < job.nr; ri++) {
    const LrSearchRect rc = rects[ri];
    __syncthreads();
    if (job.nr > 1) stage_window(F, p, rc, x0, w, sm.win, sm.ws);  // else still staged
    for (int i0 = 0; i0 < rc.h; i0 += kWienerErrBand) {
      const int rows = min(kWienerErrBand, rc.h - i0);
      __syncthreads();  // the window is staged; the previous band's rows are read
      for (int r = warp; r < rows + 2 * kB; r += nw)
        for (int j = lane; j < w; j += 32) {
          int h = 0;
#pragma unroll
          for (int u = 0; u < 7; u++) h += hf[u] * W.at(i0 + r, j + u);
          hrow[r * w + j] = int16_t(clip3(-off, lim - off, round2(h, round0)));
        }
      __syncthreads();
      for (int ir = warp; ir < rows; ir += nw)
        for (int j = lane; j < w; j += 32) {
          int sv = 0;
#pragma unroll
          for (int t = 0; t < 7; t++) sv += vf[t] * hrow[(ir + t) * w + j];
          const int e = min(max(round2(sv, round1), 0), maxv) - ld(F.src[p], sb, x0 + j, rc.y0 + i0 + ir);
          acc += int64_t(e) * e;
        }
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (tid == 0) {
    st.wiener = uint64_t(red[0] + red[1] + red[2] + red[3]);
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 3; b++) st.coef[a][b] = s_coef[a][b];
  }
}

// The self-guided fit's f64 sums in the reference's sample order, on one
// thread (rare: very large units with large errors at 12 bits, where the
// exact integer sums could round differently); the thread rebuilds each
// rectangle's window itself.
__device__ __noinline__ void sgr_fit_in_order(const LrSearchDesc& d, const LrSearchFrame& F, const LrSearchJob& job,
                                              const LrSearchRect* rects,
                                              const Win& W, const Smem& sm, const SgrPass& q0, const SgrPass& q1,
                                              double& m00, double& m01, double& m11, double& v0, double& v1) {
  const int p = job.plane, x0 = job.x0, w = job.w, sb = F.sb, step = d.step, bd = F.bd;
  const int r0 = q0.r, r1 = q1.r;
  m00 = m01 = m11 = v0 = v1 = 0.0;
  for (int ri = 0; ri < job.nr; ri++) {
    const LrSearchRect rc = rects[ri];
    const int ww = w + 2 * kB, wh = rc.h + 2 * kB;
    for (int k = 0; k < ww * wh; k++) {
      const int rr = k / ww, c = k - rr * ww;
      const int x = max(min(x0 + c - kB, F.pex[p]), 0), y = max(min(rc.y0 + rr - kB, F.pey[p]), 0);
      sm.win[rr * sm.ws + c] = int16_t(y < rc.ss   ? ld(F.cur[p], sb, x, max(rc.ss - 2, y))
                                       : y > rc.se ? ld(F.cur[p], sb, x, min(rc.se + 2, y))
                                                   : ld(F.cdef[p], sb, x, y));
    }
    for (int i = 0; i < rc.h; i += step)
      for (int j = 0; j < w; j += step) {
        const int yabs = rc.y0 + i;
        const int cval = ld(F.cdef[p], sb, x0 + j, yabs);
        const double u = double(cval << 4);
        const double a = r0 ? __dsub_rn(double(sgr_flt_direct(W, 0, q0, bd, yabs, i, j, cval)), u) : 0.0;
        const double b = r1 ? __dsub_rn(double(sgr_flt_direct(W, 1, q1, bd, yabs, i, j, cval)), u) : 0.0;
        const double t = __dmul_rn(128.0, __dsub_rn(double(ld(F.src[p], sb, x0 + j, yabs) << 4), u));
        m00 = __dadd_rn(m00, __dmul_rn(a, a));
        m01 = __dadd_rn(m01, __dmul_rn(a, b));
        m11 = __dadd_rn(m11, __dmul_rn(b, b));
        v0 = __dadd_rn(v0, __dmul_rn(a, t));
        v1 = __dadd_rn(v1, __dmul_rn(b, t));
      }
  }
}

// Phase 3, one CTA per (unit, parameter set) (256 threads): the self-guided
// fit (encoder/lr.rs:330-430) — the two box filters in bands of rows, the
// fit's sums exact in int64 under the 2^53 magnitude bound (else in order
// on one thread), the projection weights — and the restoration's error.
__global__ void __launch_bounds__(kThreads, 2) lr_search_sgr_kernel(const LrSearchDesc d) {
  extern __shared__ __align__(16) uint8_t lrs_smem[];
  __shared__ int64_t red[kThreads / 32];
  __shared__ int s_xqd[2];
  const int ji = blockIdx.x / d.nsets, si = blockIdx.x - ji * d.nsets;
  const LrSearchJob job = d.jobs[ji];
  const LrSearchFrame& F = d.frames[job.frame];
  const int p = job.plane, x0 = job.x0, w = job.w, sb = F.sb, tid = threadIdx.x, step = d.step;
  const Smem sm = smem_of(lrs_smem, d);
  const Win W{sm.win, sm.ws};
  const LrSearchRect* rects = d.rects + job.r0;
  const int bd = F.bd, maxv = (1 << bd) - 1;
  const int set = d.sets[si];
  const SgrPass q0 = sgr_pass(set, 0), q1 = sgr_pass(set, 1);
  const int r0 = q0.r, r1 = q1.r;
  const int aw = d.wmax + 2, band = d.band;
  int32_t* Ab[2];
  int32_t* Bb[2];
  int32_t* reg = reinterpret_cast<int32_t*>(sm.region);
  for (int q = 0; q < 2; q++) {
    Ab[q] = reg + (2 * q) * (band + 2) * aw;
    Bb[q] = reg + (2 * q + 1) * (band + 2) * aw;
  }
  int32_t* hs = reg + 4 * (band + 2) * aw;
  int32_t* hq = hs + (band + 6) * aw;
  int32_t* hs3 = hq + (band + 6) * aw;  // the radius-1 sums of the one-sweep box sums
  int32_t* hq3 = hs3 + (band + 4) * aw;
  int32_t* cache = d.both ? hq3 + (band + 4) * aw : hs3;  // [px][2] filter outputs of the unit
  int16_t* srcw = reinterpret_cast<int16_t*>(cache + 2 * d.cache_px);  // the rectangle's source samples
  int upx = 0;
  for (int ri = 0; ri < job.nr; ri++) upx += rects[ri].h * w;
  const bool cached = upx <= d.cache_px;
  int64_t f00 = 0, f01 = 0, f11 = 0, g0 = 0, g1 = 0, acc = 0;
  uint64_t b01 = 0, bg0 = 0, bg1 = 0;
  for (int pass_sse = 0; pass_sse < 2; pass_sse++) {
    // pass_sse 0: the fit; 1: the error with the quantised weights
    int pw0 = 0, pw1 = 0, pw2 = 0;
    if (pass_sse == 1) {
      pw0 = s_xqd[0];
      pw1 = s_xqd[1];
      pw2 = (1 << 7) - pw0 - pw1;
    }
    if (pass_sse == 1 && cached) {
      // the fit pass kept every filter output
      int off = 0;
      for (int ri = 0; ri < job.nr; ri++) {
        const LrSearchRect rc = rects[ri];
        for (int i = tid >> 5; i < rc.h; i += blockDim.x >> 5)
          for (int j = tid & 31; j < w; j += 32) {
          const int k = i * w + j;
          // one rectangle: its window and source are still staged
          const int u = (job.nr == 1 ? W.at(i + kB, j + kB) : ld(F.cdef[p], sb, x0 + j, rc.y0 + i)) << 4;
          const int fl0 = cache[2 * (off + k)], fl1 = cache[2 * (off + k) + 1];
          int32_t val = pw1 * u;
          val += r0 ? pw0 * fl0 : pw0 * u;
          val += r1 ? pw2 * fl1 : pw2 * u;
          const int out = min(max(round2(val, 4 + 7), 0), maxv);
          const int e = out - (job.nr == 1 ? srcw[k] : ld(F.src[p], sb, x0 + j, rc.y0 + i));
          acc += int64_t(e) * e;
          }
        off += rc.h * w;
      }
      break;
    }
    int off = 0;
    for (int ri = 0; ri < job.nr; ri++) {
      const LrSearchRect rc = rects[ri];
      __syncthreads();
      stage_window(F, p, rc, x0, w, sm.win, sm.ws, srcw);
      for (int i0 = 0; i0 < rc.h; i0 += band) {
        const int rows = min(band, rc.h - i0);
        __syncthreads();
        if (d.both && r0 == 2 && r1 == 1) {
          sgr_band_ab_both(W, q0, q1, bd, rc.y0, i0, rows, w, Ab[0], Bb[0], Ab[1], Bb[1], aw, hs, hq, hs3, hq3);
        } else {
          if (r0) sgr_band_ab(W, q0, 0, bd, rc.y0, i0, rows, w, Ab[0], Bb[0], aw, hs, hq);
          if (r1) sgr_band_ab(W, q1, 1, bd, rc.y0, i0, rows, w, Ab[1], Bb[1], aw, hs, hq);
        }
        __syncthreads();
        for (int ir = tid >> 5; ir < rows; ir += blockDim.x >> 5)
          for (int j = tid & 31; j < w; j += 32) {
          const int i = i0 + ir, yabs = rc.y0 + i;
          const bool fit_px = ((i | j) & (step - 1)) == 0;  // step is 1 or 2
          if (pass_sse == 0 && !fit_px && !cached) continue;
          const int cval = W.at(i + kB, j + kB);  // the rectangle's rows lie in its stripe: CDEF output
          const int u = cval << 4;  // SGRPROJ_RST_BITS
          const int fl0 = r0 ? sgr_flt(0, yabs, ir, j, Ab[0], Bb[0], aw, cval) : 0;
          const int fl1 = r1 ? sgr_flt(1, yabs, ir, j, Ab[1], Bb[1], aw, cval) : 0;
          if (pass_sse == 0 && cached) {
            cache[2 * (off + i * w + j)] = fl0;
            cache[2 * (off + i * w + j) + 1] = fl1;
          }
          if (pass_sse == 0 && !fit_px) continue;
          const int sv = srcw[i * w + j];
          if (pass_sse == 0) {
            // |a|, |b| < 2^17 and |t| < 2^23: 32-bit operands, 64-bit products
            const int32_t a = r0 ? fl0 - u : 0, b = r1 ? fl1 - u : 0;
            const int32_t t = 128 * ((sv << 4) - u);
            f00 += int64_t(a) * a;
            f01 += int64_t(a) * b;
            f11 += int64_t(b) * b;
            g0 += int64_t(a) * t;
            g1 += int64_t(b) * t;
            const uint32_t ua = uint32_t(abs(a)), ub = uint32_t(abs(b)), ut = uint32_t(abs(t));
            b01 += uint64_t(ua) * ub;
            bg0 += uint64_t(ua) * ut;
            bg1 += uint64_t(ub) * ut;
          } else {
            int32_t val = pw1 * u;
            val += r0 ? pw0 * fl0 : pw0 * u;
            val += r1 ? pw2 * fl1 : pw2 * u;
            const int out = min(max(round2(val, 4 + 7), 0), maxv);
            const int e = out - sv;
            acc += int64_t(e) * e;
          }
        }
      }
      off += rc.h * w;
    }
    if (pass_sse == 1) break;
    const int64_t t00 = block_sum_i64(f00, red), t01 = block_sum_i64(f01, red), t11 = block_sum_i64(f11, red);
    const int64_t tg0 = block_sum_i64(g0, red), tg1 = block_sum_i64(g1, red);
    // each f64 partial sum is exact (so any order gives the reference's sums)
    // while the terms' magnitudes sum below 2^53
    const uint64_t sb01 = uint64_t(block_sum_i64(int64_t(b01), red));
    const uint64_t sbg0 = uint64_t(block_sum_i64(int64_t(bg0), red));
    const uint64_t sbg1 = uint64_t(block_sum_i64(int64_t(bg1), red));
    const bool exact = uint64_t(t00) < kExact && uint64_t(t11) < kExact && sb01 < kExact && sbg0 < kExact &&
                       sbg1 < kExact;
    if (tid == 0) {
      double m00, m01, m11, v0, v1;
      if (exact) {
        m00 = double(t00);
        m01 = double(t01);
        m11 = double(t11);
        v0 = double(tg0);
        v1 = double(tg1);
      } else {
        sgr_fit_in_order(d, F, job, rects, W, sm, q0, q1, m00, m01, m11, v0, v1);
      }
      double w0, w2;
      if (r0 && r1) {
        double m[2][2] = {{m00, m01}, {m01, m11}}, v[2] = {v0, v1}, x2[2];
        solve<2>(m, v, x2);
        w0 = x2[0];
        w2 = x2[1];
      } else if (r0) {
        w0 = m00 > 0.0 ? __ddiv_rn(v0, m00) : 0.0;
        w2 = 0.0;
      } else {
        w0 = 0.0;
        w2 = m11 > 0.0 ? __ddiv_rn(v1, m11) : 0.0;
      }
      const int x0q = r0 ? min(max(f64_to_i32(round(w0)), kXqdMin[0]), kXqdMax[0]) : 0;
      int x1q;
      if (r1) {
        // i32 arithmetic wraps as the reference's release build does
        const int diff = int(uint32_t(1 << 7) - uint32_t(x0q) - uint32_t(f64_to_i32(round(w2))));
        x1q = min(max(diff, kXqdMin[1]), kXqdMax[1]);
      } else {
        x1q = min(max((1 << 7) - x0q, kXqdMin[1]), kXqdMax[1]);
      }
      s_xqd[0] = x0q;
      s_xqd[1] = x1q;
    }
    __syncthreads();
  }
  const int64_t e = block_sum_i64(acc, red);
  if (tid == 0) {
    LrSgrResult& r = d.sgr[blockIdx.x];
    r.xqd[0] = s_xqd[0];
    r.xqd[1] = s_xqd[1];
    r.sse = uint64_t(e);
  }
}

// Phase 4, one thread per unit: the cheapest of no filter (error + lambda),
// the Wiener filter (+ 40 or 28 lambda) and each self-guided set in order
// (+ 20 lambda), the first on ties (encoder/lr.rs:147-186).
__global__ void lr_search_choose_kernel(const LrSearchDesc d, int njobs) {
  const int ji = blockIdx.x * blockDim.x + threadIdx.x;
  if (ji >= njobs) return;
  const LrJobState& st = d.state[ji];
  const int p = d.jobs[ji].plane;
  const LrSearchFrame& F = d.frames[d.jobs[ji].frame];
  av1pf_lr_unit best{};
  double best_cost = __dadd_rn(__ull2double_rn(st.none), F.lambda);
  double cost = __dadd_rn(__ull2double_rn(st.wiener), __dmul_rn(F.lambda, p == 0 ? 40.0 : 28.0));
  if (cost < best_cost) {
    best_cost = cost;
    best.type = AV1PF_RESTORE_WIENER;
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 3; b++) best.wiener[a][b] = int8_t(st.coef[a][b]);
  }
  for (int si = 0; si < d.nsets; si++) {
    const LrSgrResult& r = d.sgr[ji * d.nsets + si];
    cost = __dadd_rn(__ull2double_rn(r.sse), __dmul_rn(F.lambda, 20.0));
    if (cost < best_cost) {
      best_cost = cost;
      best = av1pf_lr_unit{};
      best.type = AV1PF_RESTORE_SGRPROJ;
      best.sgr_set = uint8_t(d.sets[si]);
      best.sgr_xqd[0] = int8_t(r.xqd[0]);
      best.sgr_xqd[1] = int8_t(r.xqd[1]);
    }
  }
  d.out[ji] = best;
}

namespace {
// Raises a kernel's dynamic shared-memory limit to all the device allows
// beside its static shared memory. The attribute is process-wide, so every
// call sets the same value: searches on several contexts and host threads
// cannot lower it under one another's launches.
template <typename K>
cudaError_t allow_max_smem(K kernel, int optin) {
  cudaFuncAttributes a{};
  cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(a.sharedSizeBytes));
}
}  // namespace

cudaError_t lr_search_init() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = allow_max_smem(lr_search_prep_kernel, optin);
  if (e == cudaSuccess) e = allow_max_smem(lr_search_wiener_kernel, optin);
  if (e == cudaSuccess) e = allow_max_smem(lr_search_sgr_kernel, optin);
  return e;
}

void launch_lr_search(const LrSearchDesc& d, int njobs, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                      cudaEvent_t join) {
  if (njobs <= 0) return;
  const size_t s0 = lr_search_smem(d.wmax, d.hmax, 0, d.band, d.cache_px, d.both);
  const size_t s1 = lr_search_smem(d.wmax, d.hmax, 1, d.band, d.cache_px, d.both);
  const size_t s2 = lr_search_smem(d.wmax, d.hmax, 2, d.band, d.cache_px, d.both);
  // the self-guided fits depend on nothing else: they run beside the Wiener passes
  cudaEventRecord(fork, s);
  cudaStreamWaitEvent(side, fork, 0);
  lr_search_sgr_kernel<<<njobs * d.nsets, kThreads, s2, side>>>(d);
  if (d.multi_rect) lr_search_prep_kernel<<<njobs, kThreads, s0, s>>>(d);
  lr_search_wiener_kernel<<<njobs, 128, s1, s>>>(d);
  cudaEventRecord(join, side);
  cudaStreamWaitEvent(s, join, 0);
  lr_search_choose_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(d, njobs);
  note_launch(d.multi_rect ? 4 : 3);
}

}  // namespace av1pf
