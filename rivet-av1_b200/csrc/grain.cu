// grain.cu — film grain synthesis (7.18.3) and the output packing of
// Decoder::output.
//
// Reference: rivet-av1 src/decoder/grain.rs:8-354 (`Rng`, `apply`) and
// src/decoder/mod.rs:846-917 (`output`: crop, grain, pack into the Frame
// layout of src/frame.rs:135-192).
//
// grain_prep_kernel: one CTA per frame builds the three grain templates, the
// scaling lookup tables and the per-stripe block offsets.
//   - The Gaussian fill is a serial LFSR walk in the reference. The LFSR is
//     linear over GF(2), so the state at step n is M^n applied to the seed;
//     the host precomputes M^(82r) and M^(44r) (one 16x16 bit matrix per
//     template row) and each thread starts its row from there.
//   - The auto-regressive filter is a raster recurrence whose reach is at
//     most 3 columns left and 3 rows up (3 columns right on earlier rows),
//     so cells with equal (x - 3) + 4 (y - 3) are independent: one thread
//     per template row walks the anti-diagonal wavefront.
// output_kernel: per 256-column tile of a plane's visible area, reads the reference
// frame, adds grain (noise assembled from the templates, the 32x32 block
// offsets and the overlap blends of grain.rs:179-283, evaluated per sample
// instead of through the reference's noise-stripe and noise-image buffers),
// and writes the packed output frame. Chroma reads un-grained luma.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {
__device__ __forceinline__ uint32_t rng_step(uint32_t r) {  // grain.rs:12-18 (state update)
  const uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1u;
  return (r >> 1) | (bit << 15);
}

__device__ __forceinline__ uint32_t rng_jump(uint32_t seed, const uint16_t* cols) {
  uint32_t s = 0;
#pragma unroll
  for (int b = 0; b < 16; b++)
    if ((seed >> b) & 1u) s ^= cols[b];
  return s;
}

constexpr int kTH = 73, kTW = 82;
// Staged block offsets per output item: 256 columns span at most 16 grain
// blocks (16 columns wide in subsampled chroma), plus the block to the left.
constexpr int kOutOffs = 18;
}  // namespace

// Luma auto-regression (grain.rs:55-73) with lag LAG: thread `rr` owns
// template row 3 + rr and walks the wavefront (x - 3) + 4 * rr = t, so every
// cell's earlier neighbours (left in its row, up to LAG right in the rows
// above) are done one step earlier. Coefficients live in registers.
template <int LAG>
__device__ __forceinline__ void ar_luma(int16_t (*T)[kTW], const int32_t* coef_s, int ar_shift, int gmin, int gmax) {
  constexpr int NC = 2 * LAG * (LAG + 1);
  int c[NC > 0 ? NC : 1];
#pragma unroll
  for (int k = 0; k < NC; k++) c[k] = coef_s[k];
  const int rr = threadIdx.x;
  const int y = 3 + rr;
  const int steps = (kTW - 3 - 3 - 1) + 4 * (kTH - 3 - 1) + 1;
  for (int t = 0; t < steps; t++) {
    const int x = 3 + t - 4 * rr;
    if (y < kTH && x >= 3 && x < kTW - 3) {
      int s = 0, pos = 0;
#pragma unroll
      for (int dr = -LAG; dr <= 0; dr++)
#pragma unroll
        for (int dc = -LAG; dc <= LAG; dc++) {
          if (dr == 0 && dc >= 0) continue;
          s += T[y + dr][x + dc] * c[pos];
          pos++;
        }
      T[y][x] = int16_t(clip3(gmin, gmax, T[y][x] + round2(s, ar_shift)));
    }
    __syncthreads();
  }
}

// Chroma auto-regression with the luma term (grain.rs:101-134): threads
// 0..127 take Cb rows, 128..255 Cr rows, same wavefront as the luma one.
template <int LAG>
__device__ __forceinline__ void ar_chroma(int16_t (*T)[kTH][kTW], const int32_t (*coef_s)[25], int ar_shift, int gmin,
                                          int gmax, int chroma_w, int chroma_h, int sub_x, int sub_y, bool luma_on) {
  constexpr int NC = 2 * LAG * (LAG + 1);
  const int plane = threadIdx.x < 128 ? 1 : 2;
  int c[NC + 1];
#pragma unroll
  for (int k = 0; k <= NC; k++) c[k] = coef_s[plane][k];
  const int rr = threadIdx.x & 127;
  const int y = 3 + rr;
  const int steps = (chroma_w - 3 - 3 - 1) + 4 * (chroma_h - 3 - 1) + 1;
  for (int t = 0; t < steps; t++) {
    const int x = 3 + t - 4 * rr;
    if (y < chroma_h && x >= 3 && x < chroma_w - 3) {
      int s = 0, pos = 0;
#pragma unroll
      for (int dr = -LAG; dr <= 0; dr++)
#pragma unroll
        for (int dc = -LAG; dc <= LAG; dc++) {
          if (dr == 0 && dc >= 0) continue;
          s += T[plane][y + dr][x + dc] * c[pos];
          pos++;
        }
      if (luma_on) {
        int luma = 0;
        const int lx = ((x - 3) << sub_x) + 3, ly = ((y - 3) << sub_y) + 3;
        for (int i = 0; i <= sub_y; i++)
          for (int j = 0; j <= sub_x; j++) luma += T[0][ly + i][lx + j];
        luma = round2(luma, sub_x + sub_y);
        s += luma * c[NC];
      }
      T[plane][y][x] = int16_t(clip3(gmin, gmax, T[plane][y][x] + round2(s, ar_shift)));
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) grain_prep_kernel(const FrameDesc* __restrict__ frames,
                                                         const Item* __restrict__ items, int n_items) {
  __shared__ int16_t T[3][kTH][kTW];
  __shared__ int32_t coef[3][25];
  __shared__ int32_t lut[3][256];
  __shared__ int16_t gauss[2048];
  const int tid = threadIdx.x;
  for (int k = tid; k < 2048; k += 256) gauss[k] = g_gaussian[k];
  pdl_wait();  // the previous stage's output is complete past this point
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const av1pf_film_grain& g = f.g;
    const int bd = f.bd;
    const bool mono = f.np == 1;
    const int sub_x = f.ssx, sub_y = f.ssy;
    const int grain_center = 128 << (bd - 8);
    const int grain_min = -grain_center, grain_max = (256 << (bd - 8)) - 1 - grain_center;
    const int shift = 12 - bd + g.grain_scale_shift;
    const int chroma_w = sub_x ? 44 : 82, chroma_h = sub_y ? 38 : 73;
    const uint32_t seed = uint32_t(g.grain_seed) & 0xffffu;
    // --- Gaussian fill (grain.rs:43-54, 78-100) ---
    for (int k = tid; k < 3 * kTH * kTW; k += 256) (&T[0][0][0])[k] = 0;
    if (tid < 25) {
      coef[0][tid] = tid < 24 ? g.ar_coeffs_y_plus_128[tid] - 128 : 0;
      coef[1][tid] = g.ar_coeffs_cb_plus_128[tid] - 128;
      coef[2][tid] = g.ar_coeffs_cr_plus_128[tid] - 128;
    }
    __syncthreads();
    {
      int plane = -1, row = 0;
      if (tid < kTH) {
        plane = 0;
        row = tid;
      } else if (tid >= 80 && tid < 80 + chroma_h && !mono) {
        plane = 1;
        row = tid - 80;
      } else if (tid >= 160 && tid < 160 + chroma_h && !mono) {
        plane = 2;
        row = tid - 160;
      }
      if (plane >= 0) {
        const bool on = plane == 0 ? g.num_y_points > 0
                                   : ((plane == 1 ? g.num_cb_points : g.num_cr_points) > 0 || g.chroma_scaling_from_luma);
        const int width = plane == 0 ? kTW : chroma_w;
        if (on) {
          const uint32_t s0 = plane == 0 ? seed : (plane == 1 ? seed ^ 0xb524u : seed ^ 0x49d8u);
          uint32_t r = rng_jump(s0, width == 82 ? g_rng_jump82[row] : g_rng_jump44[row]);
          for (int c = 0; c < width; c++) {
            r = rng_step(r);
            T[plane][row][c] = int16_t(round2(gauss[(r >> 5) & 2047u], shift));
          }
        }
      }
    }
    __syncthreads();
    // --- auto-regression (grain.rs:55-134) ---
    const int lag = g.ar_coeff_lag;
    const int ar_shift = g.ar_coeff_shift_minus_6 + 6;
    switch (lag) {
      case 0: ar_luma<0>(T[0], coef[0], ar_shift, grain_min, grain_max); break;
      case 1: ar_luma<1>(T[0], coef[0], ar_shift, grain_min, grain_max); break;
      case 2: ar_luma<2>(T[0], coef[0], ar_shift, grain_min, grain_max); break;
      default: ar_luma<3>(T[0], coef[0], ar_shift, grain_min, grain_max); break;
    }
    if (!mono) {
      const bool luma_on = g.num_y_points > 0;
      switch (lag) {
        case 0: ar_chroma<0>(T, coef, ar_shift, grain_min, grain_max, chroma_w, chroma_h, sub_x, sub_y, luma_on); break;
        case 1: ar_chroma<1>(T, coef, ar_shift, grain_min, grain_max, chroma_w, chroma_h, sub_x, sub_y, luma_on); break;
        case 2: ar_chroma<2>(T, coef, ar_shift, grain_min, grain_max, chroma_w, chroma_h, sub_x, sub_y, luma_on); break;
        default: ar_chroma<3>(T, coef, ar_shift, grain_min, grain_max, chroma_w, chroma_h, sub_x, sub_y, luma_on); break;
      }
    }
    // --- scaling lookup (grain.rs:137-165): one thread per plane, as written ---
    if (tid < 3) {
      const int plane = tid;
      int np = 0;
      const int32_t *xs = nullptr, *ys = nullptr;
      if (plane == 0 || g.chroma_scaling_from_luma) {
        np = g.num_y_points; xs = g.point_y_value; ys = g.point_y_scaling;
      } else if (plane == 1) {
        np = g.num_cb_points; xs = g.point_cb_value; ys = g.point_cb_scaling;
      } else {
        np = g.num_cr_points; xs = g.point_cr_value; ys = g.point_cr_scaling;
      }
      for (int x = 0; x < 256; x++) lut[plane][x] = 0;
      if (np > 0 && !(mono && plane > 0)) {
        for (int x = 0; x < min(xs[0], 256); x++) lut[plane][x] = ys[0];
        for (int i = 0; i < np - 1; i++) {
          const int dy = ys[i + 1] - ys[i], dx = xs[i + 1] - xs[i];
          if (dx <= 0) continue;  // the format requires increasing points
          const int delta = dy * ((65536 + (dx >> 1)) / dx);
          for (int x = 0; x < dx; x++) {
            const int idx = xs[i] + x;
            if (idx >= 0 && idx < 256) lut[plane][idx] = ys[i] + ((x * delta + 32768) >> 16);
          }
        }
        for (int x = max(xs[np - 1], 0); x < 256; x++) lut[plane][x] = ys[np - 1];
      }
    }
    // --- per-stripe block offsets (grain.rs:192-199) ---
    for (int s = tid; s < f.grain_ns; s += 256) {
      uint32_t r = seed;
      r ^= uint32_t(((s * 37 + 178) & 255) << 8);
      r ^= uint32_t((s * 173 + 105) & 255);
      for (int b = 0; b < f.grain_nb; b++) {
        r = rng_step(r);
        f.grain_off[int64_t(s) * f.grain_nb + b] = uint8_t((r >> 8) & 255u);
      }
    }
    __syncthreads();
    GrainScratch* gs = f.grain;
    for (int k = tid; k < 3 * kTH * kTW; k += 256) (&gs->tmpl[0][0][0])[k] = (&T[0][0][0])[k];
    for (int k = tid; k < 3 * 256; k += 256) (&gs->lut[0][0])[k] = uint8_t(lut[k >> 8][k & 255]);
    __syncthreads();
  }
}

// scale_lut of grain.rs:166-177 (`lut` in shared memory).
__device__ __forceinline__ int grain_scale(const int16_t* lut, int index, int sh) {
  const int x = index >> sh;
  const int rem = index - (x << sh);
  if (sh == 0 || x == 255) return lut[x];
  const int start = lut[x], end = lut[x + 1];
  return start + round2((end - start) * rem, sh);
}

// Per-item constants of the output stage, held in registers: the stores to
// the packed frame are byte stores, which the compiler must otherwise assume
// alias the frame descriptor.
struct OutParams {
  const uint8_t* src;
  int64_t src_pitch;  // bytes
  const uint8_t* luma;
  int64_t luma_pitch;
  uint8_t* out;
  int pw, w, sb, bd, psx, psy, ssx, ssy;
  bool wide, grain, overlap, csfl;
  const uint8_t* off;
  int nb, gmin, gmax, min_value, max_v, maxpix, scaling_shift;
  int mult, lmult, offs;
};

// One noise sample from the template in shared memory (grain.rs:200-243 for
// the horizontal overlap): stripe offsets `rnd` (this block) and `rnd_prev`
// (the block to its left).
__device__ __forceinline__ int noise_at(const int16_t* T, int psx, int psy, int row, int j, int rnd, int rnd_prev,
                                        bool blend, int gmin, int gmax) {
  const int ox = rnd >> 4, oy = rnd & 15;
  const int pox = psx ? 6 + ox : 9 + 2 * ox;
  const int poy = psy ? 6 + oy : 9 + 2 * oy;
  int gv = T[(poy + row) * kTW + pox + j];
  if (blend) {
    const int oxp = rnd_prev >> 4, oyp = rnd_prev & 15;
    const int poxp = psx ? 6 + oxp : 9 + 2 * oxp;
    const int poyp = psy ? 6 + oyp : 9 + 2 * oyp;
    const int old = T[(poyp + row) * kTW + poxp + j + (32 >> psx)];
    gv = psx ? old * 23 + gv * 22 : (j == 0 ? old * 27 + gv * 17 : old * 17 + gv * 27);
    gv = clip3(gmin, gmax, round2(gv, 5));
  }
  return gv;
}

// Item: rows y0..y1 of a plane by up to 256 columns from x0, a multiple of
// 256 (so of the grain block width). The rows are taken one noise stripe
// (32 rows, 16 for vertically subsampled chroma) at a time, with the
// stripe's block offsets staged in shared memory; 256 threads, 8 consecutive
// samples (one grain block) per thread per step.
__global__ void __launch_bounds__(256, 3) output_kernel(const FrameDesc* __restrict__ frames,
                                                     const Item* __restrict__ items, int n_items) {
  __shared__ __align__(16) int16_t T[kTH * kTW];
  __shared__ int16_t lut[256];
  // block offsets of stripes s and s-1, blocks b0-1 .. b0+16
  __shared__ uint8_t offs_cur[kOutOffs], offs_prev[kOutOffs];
  int loaded = -1;  // frame * 4 + plane whose template is in T
  pdl_wait();  // the previous stage's output is complete past this point
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    OutParams P;
    {
      const FrameDesc& f = frames[item.frame];
      const int p = item.plane;
      P.bd = f.bd;
      P.sb = f.sb;
      P.psx = plane_ssx(f, p);
      P.psy = plane_ssy(f, p);
      P.ssx = f.ssx;
      P.ssy = f.ssy;
      P.w = f.uw;
      P.pw = (f.uw + P.psx) >> P.psx;
      P.wide = P.bd > 8;
      P.out = f.frame_out + f.out_off[p];
      P.src = f.ref[p].p;
      P.src_pitch = f.ref[p].stride * P.sb;
      P.luma = f.ref[0].p;
      P.luma_pitch = f.ref[0].stride * P.sb;
      const av1pf_film_grain& g = f.g;
      P.grain = f.grain_on != 0 &&
                (p == 0 ? g.num_y_points > 0
                        : ((p == 1 ? g.num_cb_points : g.num_cr_points) > 0 || g.chroma_scaling_from_luma));
      if (P.grain) {
        const int bd = P.bd;
        const int grain_center = 128 << (bd - 8);
        P.gmin = -grain_center;
        P.gmax = (256 << (bd - 8)) - 1 - grain_center;
        P.off = f.grain_off;
        P.nb = f.grain_nb;
        P.overlap = g.overlap_flag != 0;
        P.csfl = g.chroma_scaling_from_luma != 0;
        if (g.clip_to_restricted_range) {
          P.min_value = 16 << (bd - 8);
          const int max_luma = 235 << (bd - 8);
          P.max_v = p == 0 ? max_luma : (f.mc == 0 ? max_luma : (240 << (bd - 8)));  // MC_IDENTITY
        } else {
          P.min_value = 0;
          P.max_v = (256 << (bd - 8)) - 1;
        }
        P.maxpix = (1 << bd) - 1;
        P.scaling_shift = g.grain_scaling_minus_8 + 8;
        P.mult = p == 1 ? g.cb_mult : g.cr_mult;
        P.lmult = p == 1 ? g.cb_luma_mult : g.cr_luma_mult;
        P.offs = p == 1 ? g.cb_offset : g.cr_offset;
        const int key = int(item.frame) * 4 + p;
        if (key != loaded) {  // the plane's template and scaling table
          __syncthreads();
          // the template goes to shared memory as asynchronous copies, all
          // in flight at once (a thread's 12 words would otherwise wait
          // for each other's loads); the barrier before the stripe's
          // samples follows the wait
          const uint32_t* tg = reinterpret_cast<const uint32_t*>(&f.grain->tmpl[p][0][0]);
          const uint32_t tbase = static_cast<uint32_t>(__cvta_generic_to_shared(T));
          for (int k = threadIdx.x; k < kTH * kTW / 2; k += 256)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(tbase + 4u * uint32_t(k)), "l"(tg + k)
                         : "memory");
          for (int k = threadIdx.x; k < 256; k += 256) lut[k] = f.grain->lut[p][k];
          asm volatile("cp.async.wait_all;" ::: "memory");
          loaded = key;
        }
      }
    }
    const int x0 = item.x0, x1 = item.x1;
    const int ngroups = (x1 - x0 + 7) >> 3;  // 8-sample groups per row (<= 32)
    const int sh = P.bd - 8;
    const int bshift = 5 - P.psx;  // grain block width 32 >> psx
    const int sshift = 5 - P.psy;  // noise stripe height 32 >> psy
    const int b0 = x0 >> bshift;
    for (int ys = item.y0; ys < int(item.y1);) {
      const int stripe = ys >> sshift;
      const int ye = min(int(item.y1), (stripe + 1) << sshift);
      if (P.grain && threadIdx.x < kOutOffs) {
        const int b = b0 - 1 + int(threadIdx.x);
        const bool ok = b >= 0 && b < P.nb;
        offs_cur[threadIdx.x] = ok ? P.off[int64_t(stripe) * P.nb + b] : 0;
        offs_prev[threadIdx.x] = ok && stripe > 0 ? P.off[int64_t(stripe - 1) * P.nb + b] : 0;
      }
      __syncthreads();
      for (int k = threadIdx.x; k < (ye - ys) * 32; k += 256) {
        const int gx = k & 31, r = k >> 5;
        if (gx >= ngroups) continue;
        const int yy = ys + r;
        const int xs = x0 + gx * 8;
        const int n = min(8, x1 - xs);
        int v[8];
        const uint8_t* sp = P.src + int64_t(yy) * P.src_pitch + int64_t(xs) * P.sb;
        const bool vec = n == 8 && (reinterpret_cast<uintptr_t>(sp) & (8 * P.sb - 1)) == 0;
        if (vec && P.sb == 2) {
          const uint4 q = *reinterpret_cast<const uint4*>(sp);
          v[0] = q.x & 0xffff; v[1] = q.x >> 16; v[2] = q.y & 0xffff; v[3] = q.y >> 16;
          v[4] = q.z & 0xffff; v[5] = q.z >> 16; v[6] = q.w & 0xffff; v[7] = q.w >> 16;
        } else if (vec) {
          const uint2 q = *reinterpret_cast<const uint2*>(sp);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            v[e] = (q.x >> (8 * e)) & 0xff;
            v[4 + e] = (q.y >> (8 * e)) & 0xff;
          }
        } else {
#pragma unroll
          for (int e = 0; e < 8; e++)
            v[e] = e < n ? (P.sb == 1 ? int(sp[e]) : int(reinterpret_cast<const uint16_t*>(sp)[e])) : 0;
        }
        if (P.grain) {
          // noise image (grain.rs:251-283); the 8 samples share one grain block
          const int i = yy - (stripe << sshift);
          const int b = xs >> bshift;
          const int jb = xs - (b << bshift);
          const int li = b - b0 + 1;  // index into the staged offsets
          const bool vblend = P.overlap && stripe > 0 && i < (P.psy ? 1 : 2);
          int lum[8];
          if (item.plane != 0) {
            // un-grained luma under each chroma sample (grain.rs:303-314)
            const int ly = yy << P.ssy;
            const uint8_t* lrow = P.luma + int64_t(ly) * P.luma_pitch;
#pragma unroll
            for (int e = 0; e < 8; e++) {
              if (e < n) {
                const int lx = (xs + e) << P.ssx;
                const int lnx = min(lx + 1, P.w - 1);
                const int l0 = P.sb == 1 ? int(lrow[lx]) : int(reinterpret_cast<const uint16_t*>(lrow)[lx]);
                const int l1 = P.sb == 1 ? int(lrow[lnx]) : int(reinterpret_cast<const uint16_t*>(lrow)[lnx]);
                lum[e] = P.ssx ? round2(l0 + l1, 1) : l0;
              }
            }
          }
#pragma unroll
          for (int e = 0; e < 8; e++) {
            if (e >= n) continue;
            const int j = jb + e;
            const bool hblend = P.overlap && b > 0 && j < (P.psx ? 1 : 2);
            int noise = noise_at(T, P.psx, P.psy, i, j, offs_cur[li], offs_cur[li - 1], hblend, P.gmin, P.gmax);
            if (vblend) {
              const int old = noise_at(T, P.psx, P.psy, i + (32 >> P.psy), j, offs_prev[li], offs_prev[li - 1],
                                       hblend, P.gmin, P.gmax);
              noise = P.psy ? old * 23 + noise * 22 : (i == 0 ? old * 27 + noise * 17 : old * 17 + noise * 27);
              noise = clip3(P.gmin, P.gmax, round2(noise, 5));
            }
            const int orig = v[e];
            int idx = orig;
            if (item.plane != 0) {
              if (P.csfl) {
                idx = lum[e];
              } else {
                const int combined = lum[e] * (P.lmult - 128) + orig * (P.mult - 128);
                idx = clip3(0, P.maxpix, (combined >> 6) + ((P.offs - 256) * (1 << sh)));
              }
            }
            noise = round2(grain_scale(lut, idx, sh) * noise, P.scaling_shift);
            v[e] = clip3(P.min_value, P.max_v, orig + noise);
          }
        }
        // pack (frame.rs:153-158): u8 at 8-bit, little-endian u16 above
        const int64_t o = int64_t(yy) * P.pw + xs;
        if (P.wide) {
          uint16_t* op = reinterpret_cast<uint16_t*>(P.out) + o;
          if (n == 8 && (reinterpret_cast<uintptr_t>(op) & 15) == 0) {
            uint4 q;
            q.x = uint32_t(v[0]) | (uint32_t(v[1]) << 16);
            q.y = uint32_t(v[2]) | (uint32_t(v[3]) << 16);
            q.z = uint32_t(v[4]) | (uint32_t(v[5]) << 16);
            q.w = uint32_t(v[6]) | (uint32_t(v[7]) << 16);
            *reinterpret_cast<uint4*>(op) = q;
          } else {
#pragma unroll
            for (int e = 0; e < 8; e++)
              if (e < n) op[e] = uint16_t(v[e]);
          }
        } else {
          uint8_t* op = P.out + o;
          if (n == 8 && (reinterpret_cast<uintptr_t>(op) & 7) == 0) {
            uint2 q;
            q.x = uint32_t(v[0]) | (uint32_t(v[1]) << 8) | (uint32_t(v[2]) << 16) | (uint32_t(v[3]) << 24);
            q.y = uint32_t(v[4]) | (uint32_t(v[5]) << 8) | (uint32_t(v[6]) << 16) | (uint32_t(v[7]) << 24);
            *reinterpret_cast<uint2*>(op) = q;
          } else {
#pragma unroll
            for (int e = 0; e < 8; e++)
              if (e < n) op[e] = uint8_t(v[e]);
          }
        }
      }
      __syncthreads();
      ys = ye;
    }
  }
}

void launch_grain_prep(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  launch_pdl(grain_prep_kernel, n_items, 256, 0, s, frames, items, n_items);
}

void launch_output(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  launch_pdl(output_kernel, min(n_items, kItemGrid), 256, 0, s, frames, items, n_items);
}

}  // namespace av1pf
