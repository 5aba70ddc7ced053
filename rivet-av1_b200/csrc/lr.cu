// lr.cu — loop restoration (7.17): Wiener and self-guided filters.
//
// Reference: rivet-av1 src/decoder/postfilter.rs:568-1004 (LrCtx::sample,
// loop_restoration, lr_stripe, lr_unit_cols, restore_stripe, lr_window,
// restore_rect_from_window, box_filter_rect, wiener_coefficient).
//
// One CTA restores one rectangle: the rows of one stripe (64 luma rows,
// offset by 8) and up to 64 columns of one restoration unit. The window of
// samples the rectangle reads (3-sample border, the stripe-boundary rule of
// LrCtx::sample) is staged in shared memory; Wiener runs its horizontal then
// vertical 7-tap passes there, the self-guided filter forms its 3x3 / 5x5
// box sums from separable column sums (exact in 32 bits for <= 12-bit
// samples: 25 * 4095^2 < 2^31) with the 64-bit products of the reference
// kept where they are needed (p * s and the B term). Rectangles of units
// without restoration (and planes or frames without it) are copied, so the
// kernel writes the whole visible area of the reference frame.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {
constexpr int kMaxW = 64;            // columns per rectangle
constexpr int kWS = kMaxW + 8;       // window row stride (u16)
constexpr int kMaxH = 64;            // rows per stripe
constexpr int kWinBytes = (kMaxH + 6) * kWS * 2;
constexpr int kCsStride = kMaxW + 6;
constexpr int kCsBytes = (kMaxH + 2) * kCsStride * 4;
constexpr int kAbStride = kMaxW + 2;
constexpr int kAbBytes = (kMaxH + 2) * kAbStride * 4;
constexpr int kSmemBytes = kWinBytes + 2 * kCsBytes + 2 * kAbBytes + 256 * 4;
constexpr int kPxPerThread = (kMaxW * kMaxH + 255) / 256;
}  // namespace

struct LrGeom {
  int ss, se, y0, y1, pex, pey;
};


// LrCtx::sample (postfilter.rs:584-596) for stripe `s`. With superres the
// pre-CDEF rows come from the line buffer: 4 rows per boundary, boundary b
// (the start row of stripe b) holding rows B-2 .. B+1 at (b-1)*4 ...
__device__ __forceinline__ int lr_sample(const FrameDesc& f, int p, const LrGeom& g, int s, int x, int y) {
  x = max(min(x, g.pex), 0);
  y = max(min(y, g.pey), 0);
  const int sb = f.sb;
  if (y < g.ss) {
    const int yy = max(g.ss - 2, y);
    if (f.sr_on) return ld_sample(f.lines[p], sb, x, (s - 1) * 4 + (yy - (g.ss - 2)));
    return ld_sample(f.cur[p], sb, x, yy);
  }
  if (y > g.se) {
    const int yy = min(g.se + 2, y);
    if (f.sr_on) return ld_sample(f.lines[p], sb, x, s * 4 + (yy - (g.se - 1)));
    return ld_sample(f.cur[p], sb, x, yy);
  }
  return ld_sample(f.up[p], sb, x, y);
}

// One self-guided pass (box_filter_rect, postfilter.rs:901-991) of radius r
// over the h x w rectangle whose window is in `win`; flt receives the
// filtered values of the pixels tid + 256*m.
template <int PASS>
__device__ __forceinline__ void sgr_pass(const uint16_t* win, int32_t* cs_sum, int32_t* cs_sq, int32_t* A, int32_t* B,
                                         const int32_t* a2tab, int r, int eps, int bd, int y0, int h, int w,
                                         int32_t (&flt)[kPxPerThread]) {
  const int tid = threadIdx.x;
  const int ww = w + 6;
  const int n = (2 * r + 1) * (2 * r + 1);
  const int n2e = n * n * eps;
  const int sc = ((1 << 20) + n2e / 2) / n2e;
  const int one_over_n = ((1 << 12) + n / 2) / n;
  // column sums over 2r+1 window rows, for positions i in [0, h+2)
  for (int k = tid; k < (h + 2) * ww; k += 256) {
    const int i = k / ww, c = k - i * ww;
    if (PASS == 0 && ((y0 + i - 1) & 1) == 0) continue;  // only odd rows' A, B are weighed
    int s1 = 0, s2 = 0;
    for (int dy = -r; dy <= r; dy++) {
      const int v = win[(i + 2 + dy) * kWS + c];
      s1 += v;
      s2 += v * v;
    }
    cs_sum[i * kCsStride + c] = s1;
    cs_sq[i * kCsStride + c] = s2;
  }
  __syncthreads();
  for (int k = tid; k < (h + 2) * (w + 2); k += 256) {
    const int i = k / (w + 2), j = k - i * (w + 2);
    if (PASS == 0 && ((y0 + i - 1) & 1) == 0) continue;
    int bsum = 0, bsq = 0;
    for (int dx = -r; dx <= r; dx++) {
      bsum += cs_sum[i * kCsStride + j + 2 + dx];
      bsq += cs_sq[i * kCsStride + j + 2 + dx];
    }
    const int a = round2(bsq, 2 * (bd - 8));
    const int d = round2(bsum, bd - 8);
    const int64_t pp = max(int64_t(a) * n - int64_t(d) * d, int64_t(0));
    const int64_t z = round2_64(pp * sc, 20);
    const int a2 = a2tab[z > 255 ? 255 : int(z)];
    const int64_t b2 = int64_t(256 - a2) * int64_t(bsum) * int64_t(one_over_n);
    A[i * kAbStride + j] = a2;
    B[i * kAbStride + j] = int32_t(round2_64(b2, 12));
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < kPxPerThread; m++) {
    const int k = tid + 256 * m;
    if (k < h * w) {
      const int i = k / w, j = k - i * w;
      const int yabs = y0 + i;
      const int32_t* Ar = &A[(i + 1) * kAbStride + j + 1];
      const int32_t* Br = &B[(i + 1) * kAbStride + j + 1];
      const int32_t* Au = Ar - kAbStride;
      const int32_t* Ad = Ar + kAbStride;
      const int32_t* Bu = Br - kAbStride;
      const int32_t* Bd = Br + kAbStride;
      int a, b, shift;
      if (PASS == 0) {
        if (yabs & 1) {
          a = 6 * Ar[0] + 5 * (Ar[-1] + Ar[1]);
          b = 6 * Br[0] + 5 * (Br[-1] + Br[1]);
          shift = 4;
        } else {
          a = 6 * (Au[0] + Ad[0]) + 5 * (Au[-1] + Au[1] + Ad[-1] + Ad[1]);
          b = 6 * (Bu[0] + Bd[0]) + 5 * (Bu[-1] + Bu[1] + Bd[-1] + Bd[1]);
          shift = 5;
        }
      } else {
        a = 4 * (Ar[0] + Ar[-1] + Ar[1] + Au[0] + Ad[0]) + 3 * (Au[-1] + Au[1] + Ad[-1] + Ad[1]);
        b = 4 * (Br[0] + Br[-1] + Br[1] + Bu[0] + Bd[0]) + 3 * (Bu[-1] + Bu[1] + Bd[-1] + Bd[1]);
        shift = 5;
      }
      const int v = a * int(win[(i + 3) * kWS + j + 3]) + b;
      flt[m] = round2(v, 8 + shift - 4);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) lr_kernel(const FrameDesc* __restrict__ frames,
                                                 const Item* __restrict__ items, int n_items) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint16_t* win = reinterpret_cast<uint16_t*>(smem);
  int32_t* cs_sum = reinterpret_cast<int32_t*>(smem + kWinBytes);
  int32_t* cs_sq = reinterpret_cast<int32_t*>(smem + kWinBytes + kCsBytes);
  int32_t* A = reinterpret_cast<int32_t*>(smem + kWinBytes + 2 * kCsBytes);
  int32_t* B = reinterpret_cast<int32_t*>(smem + kWinBytes + 2 * kCsBytes + kAbBytes);
  int32_t* a2tab = reinterpret_cast<int32_t*>(smem + kWinBytes + 2 * kCsBytes + 2 * kAbBytes);
  int16_t* inter = reinterpret_cast<int16_t*>(cs_sum);  // Wiener reuses the column-sum space
  const int tid = threadIdx.x;
  // SGR_A2 (postfilter.rs:884-898)
  for (int z = tid; z < 256; z += 256) a2tab[z] = z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
  __syncthreads();

  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int p = item.plane;
    const int sx = plane_ssx(f, p), sy = plane_ssy(f, p);
    const int sb = f.sb, bd = f.bd;
    const int maxv = (1 << bd) - 1;
    // lr_stripe (postfilter.rs:640-661)
    LrGeom g;
    const int s = item.a;
    g.pey = ((f.fh + sy) >> sy) - 1;
    g.pex = ((f.uw + sx) >> sx) - 1;
    g.ss = (-8 + s * 64) >> sy;
    g.se = g.ss + (64 >> sy) - 1;
    g.y0 = max(g.ss, 0);
    g.y1 = min(g.se, g.pey);
    const int x0 = item.x0, w = int(item.x1) - int(item.x0);
    const int h = g.y1 - g.y0 + 1;
    if (h <= 0 || w <= 0) continue;
    int type = AV1PF_RESTORE_NONE;
    av1pf_lr_unit unit{};
    if (f.lr_on && f.lr_type[p] != AV1PF_RESTORE_NONE) {
      const int unit_size = f.lr_unit_size[p];
      const int luma_row = max(s * 64 - 8, 0);
      const int unit_row = min(f.lr_unit_rows[p] - 1, ((luma_row + 8) >> sy) / unit_size);
      unit = f.lru[p][unit_row * f.lr_unit_cols[p] + item.b];
      type = unit.type;
    }
    const DPlane dst = f.ref[p];
    if (type != AV1PF_RESTORE_WIENER && type != AV1PF_RESTORE_SGRPROJ) {
      const DPlane src = f.up[p];
      for (int k = tid; k < w * h; k += 256) {
        const int r = k / w, c = k - r * w;
        st_sample(dst, sb, x0 + c, g.y0 + r, ld_sample(src, sb, x0 + c, g.y0 + r));
      }
      continue;
    }
    // lr_window (postfilter.rs:765-777)
    const int ww = w + 6, wh = h + 6;
    for (int k = tid; k < ww * wh; k += 256) {
      const int r = k / ww, c = k - r * ww;
      win[r * kWS + c] = uint16_t(lr_sample(f, p, g, s, x0 + c - 3, g.y0 + r - 3));
    }
    __syncthreads();
    if (type == AV1PF_RESTORE_WIENER) {
      // postfilter.rs:795-822
      const int round0 = bd == 12 ? 5 : 3, round1 = bd == 12 ? 9 : 11;
      const int offset = 1 << (bd + 7 - round0 - 1);
      const int limit = (1 << (bd + 1 + 7 - round0)) - 1;
      int hf[7], vf[7];
      {
        const int h0 = unit.wiener[1][0], h1 = unit.wiener[1][1], h2 = unit.wiener[1][2];
        const int v0 = unit.wiener[0][0], v1 = unit.wiener[0][1], v2 = unit.wiener[0][2];
        hf[0] = hf[6] = h0; hf[1] = hf[5] = h1; hf[2] = hf[4] = h2; hf[3] = 128 - 2 * (h0 + h1 + h2);
        vf[0] = vf[6] = v0; vf[1] = vf[5] = v1; vf[2] = vf[4] = v2; vf[3] = 128 - 2 * (v0 + v1 + v2);
      }
      for (int k = tid; k < wh * w; k += 256) {
        const int r = k / w, c = k - r * w;
        const uint16_t* sp = &win[r * kWS + c];
        int acc = 0;
#pragma unroll
        for (int t = 0; t < 7; t++) acc += hf[t] * int(sp[t]);
        inter[r * kMaxW + c] = int16_t(clip3(-offset, limit - offset, round2(acc, round0)));
      }
      __syncthreads();
      for (int k = tid; k < h * w; k += 256) {
        const int r = k / w, c = k - r * w;
        int acc = 0;
#pragma unroll
        for (int t = 0; t < 7; t++) acc += vf[t] * int(inter[(r + t) * kMaxW + c]);
        st_sample(dst, sb, x0 + c, g.y0 + r, clip3(0, maxv, round2(acc, round1)));
      }
    } else {
      // postfilter.rs:823-851 with box_filter_rect (postfilter.rs:901-991)
      const int set = unit.sgr_set & 15;
      const int r0 = c_sgr_params[set][0], r1 = c_sgr_params[set][2];
      int32_t flt0[kPxPerThread], flt1[kPxPerThread];
      if (r0) sgr_pass<0>(win, cs_sum, cs_sq, A, B, a2tab, r0, c_sgr_params[set][1], bd, g.y0, h, w, flt0);
      if (r1) sgr_pass<1>(win, cs_sum, cs_sq, A, B, a2tab, r1, c_sgr_params[set][3], bd, g.y0, h, w, flt1);
      const int w0 = unit.sgr_xqd[0], w1 = unit.sgr_xqd[1];
      const int w2 = (1 << 7) - w0 - w1;
#pragma unroll
      for (int m = 0; m < kPxPerThread; m++) {
        const int k = tid + 256 * m;
        if (k >= h * w) break;
        const int i = k / w, j = k - i * w;
        const int u = int(win[(i + 3) * kWS + j + 3]) << 4;
        int v = w1 * u;
        v += r0 != 0 ? w0 * flt0[m] : w0 * u;
        v += r1 != 0 ? w2 * flt1[m] : w2 * u;
        st_sample(dst, sb, x0 + j, g.y0 + i, clip3(0, maxv, round2(v, 11)));
      }
    }
    __syncthreads();
  }
}

void launch_lr(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(lr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    attr = true;
  }
  lr_kernel<<<min(n_items, kNumSMs * 2), 256, kSmemBytes, s>>>(frames, items, n_items);
  note_launch();
}

}  // namespace av1pf
