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
// output_kernel: per tile of a plane's visible area, reads the reference
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
}  // namespace

__global__ void __launch_bounds__(256) grain_prep_kernel(const FrameDesc* __restrict__ frames,
                                                         const Item* __restrict__ items, int n_items) {
  __shared__ int16_t T[3][kTH][kTW];
  __shared__ int32_t coef[3][25];
  __shared__ int32_t lut[3][256];
  const int tid = threadIdx.x;
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
            T[plane][row][c] = int16_t(round2(g_gaussian[(r >> 5) & 2047u], shift));
          }
        }
      }
    }
    __syncthreads();
    // --- luma auto-regression (grain.rs:55-73): wavefront over (x-3) + 4(y-3) ---
    const int lag = g.ar_coeff_lag;
    const int ar_shift = g.ar_coeff_shift_minus_6 + 6;
    {
      const int y = 3 + tid;
      const int steps = (kTW - 3 - 3 - 1) + 4 * (kTH - 3 - 1) + 1;
      for (int t = 0; t < steps; t++) {
        const int x = 3 + t - 4 * tid;
        if (y < kTH && x >= 3 && x < kTW - 3) {
          int s = 0, pos = 0;
          for (int dr = -lag; dr <= 0; dr++) {
            for (int dc = -lag; dc <= lag; dc++) {
              if (dr == 0 && dc == 0) break;
              s += T[0][y + dr][x + dc] * coef[0][pos];
              pos++;
            }
          }
          T[0][y][x] = int16_t(clip3(grain_min, grain_max, T[0][y][x] + round2(s, ar_shift)));
        }
        __syncthreads();
      }
    }
    // --- chroma auto-regression with the luma term (grain.rs:101-134) ---
    if (!mono) {
      const int plane = tid < 128 ? 1 : 2;
      const int rr = tid & 127;
      const int y = 3 + rr;
      const int steps = (chroma_w - 3 - 3 - 1) + 4 * (chroma_h - 3 - 1) + 1;
      for (int t = 0; t < steps; t++) {
        const int x = 3 + t - 4 * rr;
        if (y < chroma_h && x >= 3 && x < chroma_w - 3) {
          int s = 0, pos = 0;
          for (int dr = -lag; dr <= 0; dr++) {
            bool done = false;
            for (int dc = -lag; dc <= lag; dc++) {
              const int c = coef[plane][pos];
              if (dr == 0 && dc == 0) {
                if (g.num_y_points > 0) {
                  int luma = 0;
                  const int lx = ((x - 3) << sub_x) + 3, ly = ((y - 3) << sub_y) + 3;
                  for (int i = 0; i <= sub_y; i++)
                    for (int j = 0; j <= sub_x; j++) luma += T[0][ly + i][lx + j];
                  luma = round2(luma, sub_x + sub_y);
                  s += luma * c;
                }
                done = true;
                break;
              }
              s += T[plane][y + dr][x + dc] * c;
              pos++;
            }
            if (done) break;
          }
          T[plane][y][x] = int16_t(clip3(grain_min, grain_max, T[plane][y][x] + round2(s, ar_shift)));
        }
        __syncthreads();
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

// The noise of stripe `s`, stripe row `row`, plane column x after the
// horizontal overlap of 32x32 (luma) blocks (grain.rs:200-243).
__device__ __forceinline__ int grain_hval(const int16_t* T, const uint8_t* off, int nb, int psx, int psy, int s,
                                          int row, int x, bool overlap, int gmin, int gmax) {
  const int bw = 32 >> psx;
  const int b = x >> (5 - psx);
  const int j = x - b * bw;
  const int rnd = off[s * nb + b];
  const int ox = rnd >> 4, oy = rnd & 15;
  const int pox = psx ? 6 + ox : 9 + 2 * ox;
  const int poy = psy ? 6 + oy : 9 + 2 * oy;
  int gv = T[(poy + row) * kTW + pox + j];
  if (overlap && b > 0 && j < (psx ? 1 : 2)) {
    const int rp = off[s * nb + b - 1];
    const int oxp = rp >> 4, oyp = rp & 15;
    const int poxp = psx ? 6 + oxp : 9 + 2 * oxp;
    const int poyp = psy ? 6 + oyp : 9 + 2 * oyp;
    const int old = T[(poyp + row) * kTW + poxp + j + bw];
    gv = psx ? old * 23 + gv * 22 : (j == 0 ? old * 27 + gv * 17 : old * 17 + gv * 27);
    gv = clip3(gmin, gmax, round2(gv, 5));
  }
  return gv;
}

// scale_lut of grain.rs:166-177.
__device__ __forceinline__ int grain_scale(const uint8_t* lut, int index, int bd) {
  const int sh = bd - 8;
  const int x = index >> sh;
  const int rem = index - (x << sh);
  if (bd == 8 || x == 255) return lut[x];
  const int start = lut[x], end = lut[x + 1];
  return start + round2((end - start) * rem, sh);
}

// Item: plane tile [x0,x1) x [y0,y1) of the visible area. 256 threads.
__global__ void __launch_bounds__(256) output_kernel(const FrameDesc* __restrict__ frames,
                                                     const Item* __restrict__ items, int n_items) {
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int p = item.plane;
    const int bd = f.bd, sb = f.sb;
    const int psx = plane_ssx(f, p), psy = plane_ssy(f, p);
    const int w = f.uw, h = f.fh;
    const int pw = (w + psx) >> psx;
    const bool wide = bd > 8;
    uint8_t* out = f.frame_out + f.out_off[p];
    const DPlane src = f.ref[p];
    const av1pf_film_grain& g = f.g;
    bool grain = f.grain_on != 0;
    if (grain) {
      grain = p == 0 ? g.num_y_points > 0
                     : ((p == 1 ? g.num_cb_points : g.num_cr_points) > 0 || g.chroma_scaling_from_luma);
    }
    // tiles are at most 64 columns wide: 64 fixed slots per row
    const int tw = int(item.x1) - int(item.x0);
    const int n = 64 * (int(item.y1) - int(item.y0));
    for (int k = threadIdx.x; k < n; k += 256) {
      if ((k & 63) >= tw) continue;
      const int yy = item.y0 + (k >> 6), xx = item.x0 + (k & 63);
      const int orig = ld_sample(src, sb, xx, yy);
      int v = orig;
      if (grain) {
        const int grain_center = 128 << (bd - 8);
        const int gmin = -grain_center, gmax = (256 << (bd - 8)) - 1 - grain_center;
        const int16_t* T = &f.grain->tmpl[p][0][0];
        const uint8_t* lut = f.grain->lut[p];
        const bool overlap = g.overlap_flag != 0;
        // noise image (grain.rs:251-283)
        const int stripe = yy >> (5 - psy);
        const int i = yy - (stripe << (5 - psy));
        int noise = grain_hval(T, f.grain_off, f.grain_nb, psx, psy, stripe, i, xx, overlap, gmin, gmax);
        if (overlap && stripe > 0 && i < (psy ? 1 : 2)) {
          const int old = grain_hval(T, f.grain_off, f.grain_nb, psx, psy, stripe - 1, i + (32 >> psy), xx, overlap,
                                     gmin, gmax);
          noise = psy ? old * 23 + noise * 22 : (i == 0 ? old * 27 + noise * 17 : old * 17 + noise * 27);
          noise = clip3(gmin, gmax, round2(noise, 5));
        }
        int min_value, max_luma, max_chroma;
        if (g.clip_to_restricted_range) {
          min_value = 16 << (bd - 8);
          max_luma = 235 << (bd - 8);
          max_chroma = f.mc == 0 ? max_luma : (240 << (bd - 8));  // MC_IDENTITY
        } else {
          min_value = 0;
          max_luma = max_chroma = (256 << (bd - 8)) - 1;
        }
        const int scaling_shift = g.grain_scaling_minus_8 + 8;
        if (p == 0) {
          noise = round2(grain_scale(lut, orig, bd) * noise, scaling_shift);
          v = clip3(min_value, max_luma, orig + noise);
        } else {
          // grain.rs:301-343
          const int lx = xx << f.ssx, ly = yy << f.ssy;
          const int lnx = min(lx + 1, w - 1);
          const DPlane L = f.ref[0];
          const int avg = f.ssx ? round2(ld_sample(L, sb, lx, ly) + ld_sample(L, sb, lnx, ly), 1)
                                : ld_sample(L, sb, lx, ly);
          int merged;
          if (g.chroma_scaling_from_luma) {
            merged = avg;
          } else {
            const int mult = p == 1 ? g.cb_mult : g.cr_mult;
            const int lmult = p == 1 ? g.cb_luma_mult : g.cr_luma_mult;
            const int offs = p == 1 ? g.cb_offset : g.cr_offset;
            const int combined = avg * (lmult - 128) + orig * (mult - 128);
            merged = clip3(0, (1 << bd) - 1, (combined >> 6) + ((offs - 256) * (1 << (bd - 8))));
          }
          noise = round2(grain_scale(lut, merged, bd) * noise, scaling_shift);
          v = clip3(min_value, max_chroma, orig + noise);
        }
      }
      const int64_t o = int64_t(yy) * pw + xx;
      if (wide)
        reinterpret_cast<uint16_t*>(out)[o] = uint16_t(v);  // little-endian u16 (frame.rs:153-158)
      else
        out[o] = uint8_t(v);
    }
  }
}

void launch_grain_prep(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  grain_prep_kernel<<<n_items, 256, 0, s>>>(frames, items, n_items);
  note_launch();
}

void launch_output(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  output_kernel<<<min(n_items, kMaxGrid), 256, 0, s>>>(frames, items, n_items);
  note_launch();
}

}  // namespace av1pf
