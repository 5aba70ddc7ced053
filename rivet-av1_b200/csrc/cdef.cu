// cdef.cu — the constrained directional enhancement filter (7.15).
//
// Reference: rivet-av1 src/decoder/postfilter.rs:266-513 (cdef, cdef_block,
// cdef_direction, cdef_filter, cdef_filter_block) and src/dsp/cdef.rs:13-90
// (Taps, constrain, filter_scalar).
//
// One CTA per 64x64 luma superblock (and its chroma): the superblock plus a
// 2-sample border of every plane is staged in shared memory as int16 with
// unavailable samples (outside the frame's mode-info area, postfilter.rs:
// 421-422, 464-488) stored as -32768. That value needs no special case:
// constrain() of a difference that large is 0 for every strength/damping
// pair the format allows (|d| >= 2^(damping+1) >= str << adj), a signed max
// never picks it, and an unsigned min never picks it. The direction search
// gives each warp one of the 8 directions and each lane one 8x8 block, so
// the partial-sum bins are compile-time register indices.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {

constexpr int kWin = 72;         // smem row stride (int16) of a plane window
constexpr int kWinRows = 68;     // 64 + 2*2 rows
constexpr int16_t kNA = -32768;  // unavailable sample

struct CdefBlk {
  int16_t pri, sec;  // strengths (after the luma variance adjustment)
  int8_t dir;        // filter direction
  int8_t damping;    // damping (+coeff_shift, -1 for chroma)
  int8_t copy;       // 1: skipped / CDEF off: output = input
  int8_t pad;
};

}  // namespace

// One filtered sample (cdef.rs:54-90 for one position) from a window with
// row stride `st`; offsets are in samples of that window.
struct TapsDev {
  int pri, sec, pri_adj, sec_adj, pt0, pt1;
  int po0, po1, so00, so01, so10, so11;
};

__device__ __forceinline__ void cdef_tap(int p, int x, int str, int adj, int w, int& sum, int& mx, unsigned& mn) {
  const int d = p - x;
  const int lim = max(0, str - (abs(d) >> adj));
  sum += w * min(max(d, -lim), lim);
  mx = max(mx, p);
  mn = min(mn, unsigned(p));
}

__device__ __forceinline__ int cdef_px(const int16_t* c, const TapsDev& t) {
  const int x = c[0];
  int sum = 0, mx = x;
  unsigned mn = unsigned(x);
  cdef_tap(c[t.po0], x, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[-t.po0], x, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[t.so00], x, t.sec, t.sec_adj, 2, sum, mx, mn);
  cdef_tap(c[-t.so00], x, t.sec, t.sec_adj, 2, sum, mx, mn);
  cdef_tap(c[t.so01], x, t.sec, t.sec_adj, 2, sum, mx, mn);
  cdef_tap(c[-t.so01], x, t.sec, t.sec_adj, 2, sum, mx, mn);
  cdef_tap(c[t.po1], x, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[-t.po1], x, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[t.so10], x, t.sec, t.sec_adj, 1, sum, mx, mn);
  cdef_tap(c[-t.so10], x, t.sec, t.sec_adj, 1, sum, mx, mn);
  cdef_tap(c[t.so11], x, t.sec, t.sec_adj, 1, sum, mx, mn);
  cdef_tap(c[-t.so11], x, t.sec, t.sec_adj, 1, sum, mx, mn);
  const int v = x + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
  return min(max(v, int(mn)), mx);
}

// The Taps of cdef_filter_block (postfilter.rs:489-511) for a window of row
// stride `st`. CDEF_SEC_TAPS is [2, 1] for both primary-tap parities.
__device__ __forceinline__ TapsDev make_taps(int pri, int sec, int damping, int dir, int coeff_shift, int st) {
  TapsDev t;
  t.pri = pri;
  t.sec = sec;
  t.pri_adj = pri ? max(damping - floor_log2(uint32_t(pri)), 0) : 0;
  t.sec_adj = sec ? max(damping - floor_log2(uint32_t(sec)), 0) : 0;
  const bool odd = (pri >> coeff_shift) & 1;  // CDEF_PRI_TAPS[(pri >> cs) & 1]: [4,2] / [3,3]
  t.pt0 = odd ? 3 : 4;
  t.pt1 = odd ? 3 : 2;
  const int dlo = (dir + 6) & 7, dhi = (dir + 2) & 7;
  t.po0 = c_cdef_dirs[dir][0][0] * st + c_cdef_dirs[dir][0][1];
  t.po1 = c_cdef_dirs[dir][1][0] * st + c_cdef_dirs[dir][1][1];
  t.so00 = c_cdef_dirs[dlo][0][0] * st + c_cdef_dirs[dlo][0][1];
  t.so01 = c_cdef_dirs[dhi][0][0] * st + c_cdef_dirs[dhi][0][1];
  t.so10 = c_cdef_dirs[dlo][1][0] * st + c_cdef_dirs[dlo][1][1];
  t.so11 = c_cdef_dirs[dhi][1][0] * st + c_cdef_dirs[dhi][1][1];
  return t;
}

// cdef_direction's cost of direction D (postfilter.rs:345-390) for the 8x8
// block at `s` (row stride st); samples are >> sh then - 128.
template <int D>
__device__ __forceinline__ int32_t cdef_cost(const int16_t* s, int st, int sh) {
  int32_t p[15];
#pragma unroll
  for (int k = 0; k < 15; k++) p[k] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int x = (int(s[i * st + j]) >> sh) - 128;
      const int k = D == 0 ? i + j
                  : D == 1 ? i + j / 2
                  : D == 2 ? i
                  : D == 3 ? 3 + i - j / 2
                  : D == 4 ? 7 + i - j
                  : D == 5 ? 3 - i / 2 + j
                  : D == 6 ? j
                           : i / 2 + j;
      p[k] += x;
    }
  }
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

__device__ __forceinline__ int32_t cdef_cost_dir(int d, const int16_t* s, int st, int sh) {
  switch (d) {
    case 0: return cdef_cost<0>(s, st, sh);
    case 1: return cdef_cost<1>(s, st, sh);
    case 2: return cdef_cost<2>(s, st, sh);
    case 3: return cdef_cost<3>(s, st, sh);
    case 4: return cdef_cost<4>(s, st, sh);
    case 5: return cdef_cost<5>(s, st, sh);
    case 6: return cdef_cost<6>(s, st, sh);
    default: return cdef_cost<7>(s, st, sh);
  }
}

// Item: superblock (x0 = SB column, y0 = SB row). 256 threads.
__global__ void __launch_bounds__(256) cdef_kernel(const FrameDesc* __restrict__ frames,
                                                   const Item* __restrict__ items, int n_items) {
  __shared__ int16_t win[3][kWinRows * kWin];
  __shared__ int32_t cost[64][8];
  __shared__ CdefBlk blk[3][64];
  __shared__ uint8_t bstate[64];  // 0 = outside the MI area, 1 = copy, 2 = filter
  const int tid = threadIdx.x;
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int sc = item.x0, sr = item.y0;
    const int np = f.np, sb = f.sb;
    const int cs = f.bd - 8;
    const int idx = f.cdef_idx[int64_t(sr) * f.cdef_stride + sc];  // postfilter.rs:285
    // --- stage the windows (postfilter.rs:464-488) ---
    for (int p = 0; p < np; p++) {
      const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
      const int bw = (64 >> sx) + 4, bh = (64 >> sy) + 4;
      const int px0 = ((sc * 64) >> sx) - 2, py0 = ((sr * 64) >> sy) - 2;
      const int xlim = (f.mi_cols * 4) >> sx, ylim = (f.mi_rows * 4) >> sy;
      const DPlane src = f.cur[p];
      for (int k = tid; k < bw * bh; k += 256) {
        const int r = k / bw, c = k - r * bw;
        const int gx = px0 + c, gy = py0 + r;
        int16_t v = kNA;
        if (gx >= 0 && gx < xlim && gy >= 0 && gy < ylim) v = int16_t(ld_sample(src, sb, gx, gy));
        win[p][r * kWin + c] = v;
      }
    }
    // --- per 8x8: inside the MI area? skipped? (postfilter.rs:281-287, 306-310) ---
    if (tid < 64) {
      const int by = tid >> 3, bx = tid & 7;
      const int r = sr * 16 + 2 * by, c = sc * 16 + 2 * bx;
      uint8_t st = 0;
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
      bstate[tid] = st;
    }
    __syncthreads();
    // --- direction search (postfilter.rs:345-401): warp = direction, lane = block ---
    {
      const int d = tid >> 5, lane = tid & 31;
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const int b = lane + 32 * half;
        if (bstate[b] == 2) {
          const int by = b >> 3, bx = b & 7;
          const int16_t* s = &win[0][(2 + by * 8) * kWin + 2 + bx * 8];
          cost[b][d] = cdef_cost_dir(d, s, kWin, cs);
        }
      }
    }
    __syncthreads();
    // --- per-block strengths (postfilter.rs:311-341) ---
    if (tid < 64) {
      const int b = tid;
      CdefBlk L{0, 0, 0, 0, 1, 0}, U{0, 0, 0, 0, 1, 0};
      if (bstate[b] == 2) {
        int32_t best = 0;
        int y_dir = 0;
        for (int d = 0; d < 8; d++) {
          if (cost[b][d] > best) {
            best = cost[b][d];
            y_dir = d;
          }
        }
        const int32_t var = (best - cost[b][(y_dir + 4) & 7]) >> 10;
        int pri = f.cdef_y_pri[idx] << cs;
        const int sec = f.cdef_y_sec[idx] << cs;
        const int dir = pri == 0 ? 0 : y_dir;
        const int var_str = (var >> 6) != 0 ? min(floor_log2(uint32_t(var >> 6)), 12) : 0;
        pri = var != 0 ? (pri * (4 + var_str) + 8) >> 4 : 0;
        L.pri = int16_t(pri);
        L.sec = int16_t(sec);
        L.dir = int8_t(dir);
        L.damping = int8_t(f.cdef_damping + cs);
        L.copy = (pri == 0 && sec == 0) ? 1 : 0;  // a zero-strength filter is the identity
        const int upri = f.cdef_uv_pri[idx] << cs;
        const int usec = f.cdef_uv_sec[idx] << cs;
        U.pri = int16_t(upri);
        U.sec = int16_t(usec);
        U.dir = int8_t(upri == 0 ? 0 : c_cdef_uv_dir[f.ssx][f.ssy][y_dir]);
        U.damping = int8_t(f.cdef_damping + cs - 1);
        U.copy = (upri == 0 && usec == 0) ? 1 : 0;
      }
      blk[0][b] = L;
      blk[1][b] = U;
      blk[2][b] = U;
    }
    __syncthreads();
    // --- filter + write: one block row per step (postfilter.rs:405-442) ---
    {
      const int csx = f.ssx, csy = f.ssy;
      const int rows_l = 64 * 8;
      const int ch_h = 8 >> csy;
      const int rows_c = np > 1 ? 64 * ch_h : 0;
      const int total = rows_l + 2 * rows_c;
      for (int k = tid; k < total; k += 256) {
        int p, b, rr;
        if (k < rows_l) {
          p = 0;
          b = k >> 3;
          rr = k & 7;
        } else {
          const int kk = k - rows_l;
          p = 1 + kk / rows_c;
          const int q = kk % rows_c;
          b = q / ch_h;
          rr = q - b * ch_h;
        }
        if (bstate[b] == 0) continue;
        const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
        const int w = 8 >> sx;
        const int by = b >> 3, bx = b & 7;
        const int lx = bx * w, ly = by * (8 >> sy) + rr;  // position within the plane's SB
        const int16_t* c = &win[p][(2 + ly) * kWin + 2 + lx];
        int out[8];
        const CdefBlk pb = blk[p][b];
        if (pb.copy) {
#pragma unroll
          for (int j = 0; j < 8; j++) out[j] = j < w ? c[j] : 0;
        } else {
          const TapsDev t = make_taps(pb.pri, pb.sec, pb.damping, pb.dir, cs, kWin);
#pragma unroll
          for (int j = 0; j < 8; j++) out[j] = j < w ? cdef_px(c + j, t) : 0;
        }
        const DPlane dst = f.cdef[p];
        const int gx = ((sc * 64) >> sx) + lx, gy = ((sr * 64) >> sy) + ly;
        uint8_t* row = dst.p + int64_t(gy) * dst.stride * sb;
        if (sb == 2) {
          uint16_t* r16 = reinterpret_cast<uint16_t*>(row) + gx;
          if (w == 8) {
            uint4 v;
            v.x = uint32_t(out[0]) | (uint32_t(out[1]) << 16);
            v.y = uint32_t(out[2]) | (uint32_t(out[3]) << 16);
            v.z = uint32_t(out[4]) | (uint32_t(out[5]) << 16);
            v.w = uint32_t(out[6]) | (uint32_t(out[7]) << 16);
            *reinterpret_cast<uint4*>(r16) = v;
          } else {
            uint2 v;
            v.x = uint32_t(out[0]) | (uint32_t(out[1]) << 16);
            v.y = uint32_t(out[2]) | (uint32_t(out[3]) << 16);
            *reinterpret_cast<uint2*>(r16) = v;
          }
        } else {
          uint8_t* r8 = row + gx;
          if (w == 8) {
            uint2 v;
            v.x = uint32_t(out[0]) | (uint32_t(out[1]) << 8) | (uint32_t(out[2]) << 16) | (uint32_t(out[3]) << 24);
            v.y = uint32_t(out[4]) | (uint32_t(out[5]) << 8) | (uint32_t(out[6]) << 16) | (uint32_t(out[7]) << 24);
            *reinterpret_cast<uint2*>(r8) = v;
          } else {
            *reinterpret_cast<uint32_t*>(r8) =
                uint32_t(out[0]) | (uint32_t(out[1]) << 8) | (uint32_t(out[2]) << 16) | (uint32_t(out[3]) << 24);
          }
        }
      }
    }
    __syncthreads();
  }
}

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
  cdef_tap(c[t.po0], x, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[-t.po0], x, t.pri, t.pri_adj, t.pt0, sum, mx, mn);
  cdef_tap(c[t.so00], x, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[-t.so00], x, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[t.so01], x, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[-t.so01], x, t.sec, t.sec_adj, a.sec_taps[0], sum, mx, mn);
  cdef_tap(c[t.po1], x, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[-t.po1], x, t.pri, t.pri_adj, t.pt1, sum, mx, mn);
  cdef_tap(c[t.so10], x, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[-t.so10], x, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[t.so11], x, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  cdef_tap(c[-t.so11], x, t.sec, t.sec_adj, a.sec_taps[1], sum, mx, mn);
  const int v = x + ((8 + sum - (sum < 0 ? 1 : 0)) >> 4);
  res[int64_t(e) * 64 + i * a.w + j] = uint16_t(min(max(v, int(mn)), mx));
}

void launch_cdef(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  cdef_kernel<<<min(n_items, kNumSMs * 4), 256, 0, s>>>(frames, items, n_items);
  note_launch();
}

void launch_dsp_cdef(const int32_t* win, const av1pf_cdef_taps* taps, uint16_t* res, int n, cudaStream_t s) {
  if (n <= 0) return;
  dsp_cdef_kernel<<<n, 64, 0, s>>>(win, taps, res, n);
  note_launch();
}

}  // namespace av1pf
