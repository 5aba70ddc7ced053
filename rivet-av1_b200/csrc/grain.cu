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
//     so cells with equal (x - 3) + 4 (y - 3) are independent: one warp per
//     template walks that wavefront, a lane per row on it. Every neighbour a
//     cell reads reaches its lane by warp shuffles from the lanes of the rows
//     above and is kept in register rings, so the recurrence runs without
//     shared-memory round trips or barriers; the chroma warps trail the luma
//     warp.
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

// Four steps of rng_step at once, the states after each into st[0..3]. The
// feedback bit of step j (1..4) is bit j - 1 of r ^ r>>1 ^ r>>3 ^ r>>12: its
// taps read bits j-1, j, j+2 and j+11 of the starting state, all below the
// bits the earlier steps shifted in (those reach bit 12 of the state only
// at step 5).
__device__ __forceinline__ void rng_step4(uint32_t r, uint32_t st[4]) {
  const uint32_t f = r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12);
  st[0] = (r >> 1) | ((f & 1u) << 15);
  st[1] = (r >> 2) | ((f & 3u) << 14);
  st[2] = (r >> 3) | ((f & 7u) << 13);
  st[3] = (r >> 4) | ((f & 15u) << 12);
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
// Staged row strides of the output kernel: 256 samples of up to 2 bytes, and
// the luma under 256 chroma columns (512 samples at 2:1).
constexpr int kStageSrc = 512, kStageLuma = 1024;
}  // namespace

// Auto-regression of one template (grain.rs:55-73 for luma, :101-134 for
// chroma with its luma term) by one warp, on a wavefront: the cell (y, x) is
// filtered at step t = (x - 3) + S (y - 3). Its neighbours reach LAG rows up
// and LAG columns to either side (left only in its own row), so with a slope
// S >= LAG + 1 each of them comes at an earlier step; S is at least 3 so
// that no more rows are on the wavefront at once than a warp has lanes.
// Template row 3 + rr belongs to lane rr % 32, which walks it left to right,
// one column per step, from column 0 (three steps before its first filtered
// cell) to the last column.
//
// At every step every lane emits the value of its cell: the filtered value,
// or the Gaussian value for the unfiltered border columns and the three top
// rows (rows -3 .. -1 of the wavefront, walked by lanes 29 .. 31). The lane
// k rows below receives the emission one step later by a warp shuffle: the
// emission of lane (l - k) at step t - 1 is the cell (y - k, x + kS - 1) of
// lane l at step t. Each lane keeps what it received from the lanes 1 .. LAG
// above in register rings (slot t % 16; the oldest value read is 3S + LAG - 1
// <= 14 steps old) and its own last LAG emissions: the filter reads no
// shared memory except the cell's own Gaussian value, and the warp needs no
// barrier between steps. The steps run in groups of 8 without branches
// (cells outside the filter compute and store their own value back), so the
// scheduler overlaps each step's sums over older values with the step
// before; the step-to-step chain is the shuffle, one multiply-add, the
// rounding and the clip.
//
// The luma warp publishes its completed step count in `progress` after every
// group of 8 steps (past a warp barrier that orders its lanes' template
// stores before the release); a chroma warp waits, before a group, for the
// luma cells the group's luma terms read (a bounded wait, polling with a
// short sleep: after kSpinLimit polls it flags ERRF_STALL and goes on).
constexpr int kSpinLimit = 1 << 20;
constexpr int kProgressBias = 64;  // progress holds (last luma step done) + 1 + bias; 0 is "none"

template <int LAG>
__device__ __forceinline__ constexpr int ar_slope() {
  return LAG + 1 > 3 ? LAG + 1 : 3;
}

__device__ __forceinline__ uint32_t ld_acquire_cta(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.cta.shared.u32 %0, [%1];"
               : "=r"(v)
               : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p)))
               : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(uint32_t* p, uint32_t v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))), "r"(v)
               : "memory");
}

// The cell lane `lane` holds at step t: row y, column x, whether the filter
// runs there, and a template offset that is always inside the template —
// the cell itself, or for a cell outside the template, a border cell (row 0,
// or the first or last column) that no step filters.
struct ArCell {
  int y, x, off;
  bool ar;
};
template <int S>
__device__ __forceinline__ ArCell ar_cell(int t, int lane, int H, int W) {
  const int q = (t + 3 + 16 * S) / S - 16;  // floor((t + 3) / S): rows change lanes at column 0
  const int rr = q - ((q - lane) & 31);
  ArCell c;
  c.y = 3 + rr;
  c.x = 3 + t - S * rr;
  c.ar = rr >= 0 && c.y < H && c.x >= 3 && c.x < W - 3;
  const int yc = c.y >= 0 && c.y < H ? c.y : 0;
  const int xc = min(max(c.x, 0), W - 1);
  c.off = yc * kTW + xc;
  return c;
}

template <int LAG, bool CHROMA>
__device__ __forceinline__ void ar_warp(int16_t (*T)[kTW], const int16_t (*Y)[kTW], const int32_t* coef_s, int H,
                                        int W, int ar_shift, int gmin, int gmax, int sub_x, int sub_y, bool luma_on,
                                        uint32_t* progress) {
  constexpr int S = ar_slope<LAG>();
  constexpr int NC = 2 * LAG * (LAG + 1);
  constexpr int RW = 2 * LAG + 1;  // coefficients per row above
  int c[NC + 1];
#pragma unroll
  for (int k = 0; k <= NC; k++) c[k] = coef_s[k];
  const int lane = threadIdx.x & 31;
  const int rows = H - 3;
  const int t_last = (W - 7) + S * (rows - 1);  // the last row's last filtered cell
  const bool luma_term = CHROMA && luma_on;
  int16_t* Tf = &T[0][0];
  const int16_t* Yf = &Y[0][0];
  int own[16];                   // the lane's emission of step t in slot t % 16
  int w[LAG > 0 ? LAG : 1][16];  // w[k - 1]: emissions of the lane k rows above, one step late
#pragma unroll
  for (int u = 0; u < 16; u++) {
    own[u] = 0;
#pragma unroll
    for (int k = 0; k < (LAG > 0 ? LAG : 1); k++) w[k][u] = 0;
  }
  uint32_t seen = 0;  // the luma progress last read
  // steps from -16 (the top row -3 starts at -S * 3 - 3 >= -15), in blocks of
  // 16 so that every ring slot is a constant, and groups of 8 whose steps
  // have no branches
  for (int tb = -16; tb <= t_last; tb += 16) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int t0 = tb + 8 * half;
      if (luma_term) {
        // the last luma step whose cell the group's luma terms read
        int need = -(1 << 20);
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const ArCell e = ar_cell<S>(t0 + j, lane, H, W);
          if (e.ar) need = max(need, ((e.x - 3) << sub_x) + sub_x + S * (((e.y - 3) << sub_y) + sub_y));
        }
        const int wneed = __reduce_max_sync(0xffffffffu, need) + kProgressBias;
        if (wneed >= int(seen)) {
          int spins = 0;
          while ((seen = ld_acquire_cta(progress)) <= uint32_t(wneed)) {
            if (++spins > kSpinLimit) {
              if (lane == 0) atomicOr(&g_error_flags, ERRF_STALL);
              break;
            }
            __nanosleep(32);
          }
        }
      }
      // the group's cells, their Gaussian values and luma terms, loaded
      // ahead: a cell is written by its own lane only
      int off[8], g[8], lum[8];
      uint32_t arm = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const ArCell e = ar_cell<S>(t0 + j, lane, H, W);
        off[j] = e.off;
        arm |= uint32_t(e.ar) << j;
        g[j] = Tf[e.off];
        lum[j] = 0;
        if (luma_term) {
          const int lo = e.ar ? (((e.y - 3) << sub_y) + 3) * kTW + ((e.x - 3) << sub_x) + 3 : 3 * kTW + 3;
          int l = Yf[lo];
          if (sub_x) l += Yf[lo + 1];
          if (sub_y) l += Yf[lo + kTW];
          if (sub_x && sub_y) l += Yf[lo + kTW + 1];
          lum[j] = round2(l, sub_x + sub_y) * c[NC];
        }
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int u = 8 * half + j;
        const int vprev = own[(u + 15) & 15];
#pragma unroll
        for (int k = 1; k <= LAG; k++) w[k - 1][u] = __shfl_sync(0xffffffffu, vprev, (lane - k) & 31);
        // four partial sums over the values from earlier steps; (y - k, x +
        // dc) came at step t + dc - kS + 1, and (y, x + dc) is the lane's
        // own emission of step t + dc
        int acc[4] = {lum[j], 0, 0, 0};
        int n = 0;
#pragma unroll
        for (int k = LAG; k >= 1; k--)
#pragma unroll
          for (int dc = -LAG; dc <= LAG; dc++)
            if (!(k == 1 && dc == LAG)) acc[n++ & 3] += w[k - 1][(u + dc - k * S + 1 + 32) & 15] * c[(LAG - k) * RW + dc + LAG];
#pragma unroll
        for (int dc = -LAG; dc <= -2; dc++) acc[n++ & 3] += own[(u + dc + 16) & 15] * c[LAG * RW + LAG + dc];
        int sum = (acc[0] + acc[1]) + (acc[2] + acc[3]);
        // the two values of the step before: the cell up and LAG to the
        // right (just received) and the cell to the left
        if (LAG > 0) sum += w[0][u] * c[(LAG - 1) * RW + 2 * LAG] + vprev * c[LAG * RW + LAG - 1];
        const int v = (arm >> j) & 1u ? clip3(gmin, gmax, g[j] + round2(sum, ar_shift)) : g[j];
        Tf[off[j]] = int16_t(v);  // a cell outside the filter gets its own value back
        own[u] = v;
      }
      if (!CHROMA) {
        // the warp barrier orders every lane's stores before the releases
        __syncwarp();
        st_release_cta(progress, uint32_t(t0 + 8 + kProgressBias));
      }
    }
  }
}

template <bool CHROMA>
__device__ __forceinline__ void ar_plane(int lag, int16_t (*T)[kTW], const int16_t (*Y)[kTW], const int32_t* coef,
                                         int H, int W, int ar_shift, int gmin, int gmax, int sub_x, int sub_y,
                                         bool luma_on, uint32_t* progress) {
  switch (lag) {
    case 0: ar_warp<0, CHROMA>(T, Y, coef, H, W, ar_shift, gmin, gmax, sub_x, sub_y, luma_on, progress); break;
    case 1: ar_warp<1, CHROMA>(T, Y, coef, H, W, ar_shift, gmin, gmax, sub_x, sub_y, luma_on, progress); break;
    case 2: ar_warp<2, CHROMA>(T, Y, coef, H, W, ar_shift, gmin, gmax, sub_x, sub_y, luma_on, progress); break;
    default: ar_warp<3, CHROMA>(T, Y, coef, H, W, ar_shift, gmin, gmax, sub_x, sub_y, luma_on, progress); break;
  }
}

// One CTA of 256 threads per frame. All threads fill the templates with
// Gaussian values (one template row each). Then warps 0, 1 and 2 run the
// luma, Cb and Cr auto-regressions side by side, chroma trailing luma,
// while warps 3-7 build the scaling tables (one entry per thread) and the
// per-stripe block offsets (one stripe per thread).
__global__ void __launch_bounds__(256) grain_prep_kernel(const FrameDesc* __restrict__ frames,
                                                         const Item* __restrict__ items, int n_items) {
  AV1PF_TRACE_BEGIN();
  __shared__ __align__(16) int16_t T[3][kTH][kTW];
  __shared__ int32_t coef[3][25];
  __shared__ uint8_t lut[3][256];
  __shared__ int16_t gauss[2048];
  __shared__ uint32_t progress;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
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
    for (int k = tid; k < 3 * kTH * kTW / 2; k += 256) reinterpret_cast<uint32_t*>(&T[0][0][0])[k] = 0u;
    if (tid < 25) {
      coef[0][tid] = tid < 24 ? g.ar_coeffs_y_plus_128[tid] - 128 : 0;
      coef[1][tid] = g.ar_coeffs_cb_plus_128[tid] - 128;
      coef[2][tid] = g.ar_coeffs_cr_plus_128[tid] - 128;
    }
    if (tid == 0) progress = 0u;
    __syncthreads();
    {
      int plane = -1, row = tid;
      if (row < kTH) {
        plane = 0;
      } else if (!mono && (row -= kTH) < chroma_h) {
        plane = 1;
      } else if (!mono && (row -= chroma_h) < chroma_h) {
        plane = 2;
      }
      if (plane >= 0) {
        const bool on = plane == 0 ? g.num_y_points > 0
                                   : ((plane == 1 ? g.num_cb_points : g.num_cr_points) > 0 || g.chroma_scaling_from_luma);
        const int width = plane == 0 ? kTW : chroma_w;
        if (on) {
          const uint32_t s0 = plane == 0 ? seed : (plane == 1 ? seed ^ 0xb524u : seed ^ 0x49d8u);
          uint32_t r = rng_jump(s0, width == 82 ? g_rng_jump82[row] : g_rng_jump44[row]);
          // four states per pass (rng_step4); the widths are even, so pairs
          // of values go out as 32-bit stores (a row is 164 bytes)
          uint32_t* dst = reinterpret_cast<uint32_t*>(&T[plane][row][0]);
          for (int c = 0; c < width; c += 4) {
            uint32_t st[4];
            rng_step4(r, st);
            r = st[3];
            const int v0 = round2(gauss[(st[0] >> 5) & 2047u], shift), v1 = round2(gauss[(st[1] >> 5) & 2047u], shift);
            const int v2 = round2(gauss[(st[2] >> 5) & 2047u], shift), v3 = round2(gauss[(st[3] >> 5) & 2047u], shift);
            dst[c >> 1] = uint32_t(uint16_t(v0)) | (uint32_t(uint16_t(v1)) << 16);
            if (c + 2 < width) dst[(c >> 1) + 1] = uint32_t(uint16_t(v2)) | (uint32_t(uint16_t(v3)) << 16);
          }
        }
      }
    }
    __syncthreads();
    const int lag = g.ar_coeff_lag;
    const int ar_shift = g.ar_coeff_shift_minus_6 + 6;
    if (warp == 0) {
      // --- luma auto-regression (grain.rs:55-73) ---
      ar_plane<false>(lag, T[0], T[0], coef[0], kTH, kTW, ar_shift, grain_min, grain_max, 0, 0, false, &progress);
    } else if (warp <= 2) {
      // --- chroma auto-regression with the luma term (grain.rs:101-134) ---
      if (!mono)
        ar_plane<true>(lag, T[warp], T[0], coef[warp], chroma_h, chroma_w, ar_shift, grain_min, grain_max, sub_x,
                       sub_y, g.num_y_points > 0, &progress);
    } else {
      // --- scaling lookup (grain.rs:137-165), one entry per thread: the
      // later of the reference's writes to an entry is the one kept ---
      for (int k = tid - 96; k < 3 * 256; k += 160) {
        const int plane = k >> 8, x = k & 255;
        int np = 0;
        const int32_t *xs = nullptr, *ys = nullptr;
        if (plane == 0 || g.chroma_scaling_from_luma) {
          np = g.num_y_points; xs = g.point_y_value; ys = g.point_y_scaling;
        } else if (plane == 1) {
          np = g.num_cb_points; xs = g.point_cb_value; ys = g.point_cb_scaling;
        } else {
          np = g.num_cr_points; xs = g.point_cr_value; ys = g.point_cr_scaling;
        }
        int v = 0;
        if (np > 0 && !(mono && plane > 0)) {
          if (x < xs[0]) v = ys[0];
          for (int i = 0; i < np - 1; i++) {
            const int dy = ys[i + 1] - ys[i], dx = xs[i + 1] - xs[i];
            if (dx <= 0 || x < xs[i] || x >= xs[i] + dx) continue;  // the format requires increasing points
            const int delta = dy * ((65536 + (dx >> 1)) / dx);
            v = ys[i] + (((x - xs[i]) * delta + 32768) >> 16);
          }
          if (x >= xs[np - 1]) v = ys[np - 1];
        }
        lut[plane][x] = uint8_t(v);
      }
      // --- per-stripe block offsets (grain.rs:192-199) ---
      for (int s = tid - 96; s < f.grain_ns; s += 160) {
        uint32_t r = seed;
        r ^= uint32_t(((s * 37 + 178) & 255) << 8);
        r ^= uint32_t((s * 173 + 105) & 255);
        for (int b = 0; b < f.grain_nb; b++) {
          r = rng_step(r);
          f.grain_off[int64_t(s) * f.grain_nb + b] = uint8_t((r >> 8) & 255u);
        }
      }
    }
    __syncthreads();
    GrainScratch* gs = f.grain;
    {
      // each plane's template, its padding zeroed
      constexpr int kPlaneWords = kTmplStride / 2, kTmplWords = kTH * kTW / 2;
      for (int k = tid; k < 3 * kPlaneWords; k += 256) {
        const int p = k / kPlaneWords, w = k - p * kPlaneWords;
        reinterpret_cast<uint32_t*>(&gs->tmpl[p][0])[w] =
            w < kTmplWords ? reinterpret_cast<const uint32_t*>(&T[p][0][0])[w] : 0u;
      }
    }
    // the scaling function at every sample value (scale_lut of
    // grain.rs:166-177: above 8 bits, interpolated between the two entries
    // around index >> (bitdepth - 8)), four values per 32-bit store
    {
      const int sh = bd - 8;
      const int wshift = bd - 2;  // log2 of the words per plane
      for (int k = tid; k < (3 << wshift); k += 256) {
        const int plane = k >> wshift, i0 = (k - (plane << wshift)) * 4;
        uint32_t word = 0;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int index = i0 + e;
          const int x = index >> sh, rem = index - (x << sh);
          int v = lut[plane][x];
          if (sh > 0 && x < 255) v += round2((int(lut[plane][x + 1]) - v) * rem, sh);
          word |= uint32_t(v) << (8 * e);
        }
        reinterpret_cast<uint32_t*>(&gs->scale[plane][0])[k - (plane << wshift)] = word;
      }
    }
    __syncthreads();
  }
  AV1PF_TRACE_END(6);
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

// Template positions (grain.rs:200-243): the sample of block column j and
// noise-stripe row `row` of a block with offsets `rnd` is at
// tmpl_at(...)[j], and the column of the block to its left that overlaps it
// at left_at(...)[j].
__device__ __forceinline__ const int16_t* tmpl_at(const int16_t* T, int psx, int psy, int row, int rnd) {
  const int ox = rnd >> 4, oy = rnd & 15;
  return T + ((psy ? 6 + oy : 9 + 2 * oy) + row) * kTW + (psx ? 6 + ox : 9 + 2 * ox);
}
__device__ __forceinline__ const int16_t* left_at(const int16_t* T, int psx, int psy, int row, int rnd_prev) {
  return tmpl_at(T, psx, psy, row, rnd_prev) + (32 >> psx);
}
// The horizontal overlap blend of column j (0 or 1) of a block.
__device__ __forceinline__ int hblend(int old, int g, int j, int psx, int gmin, int gmax) {
  const int gv = psx ? old * 23 + g * 22 : (j == 0 ? old * 27 + g * 17 : old * 17 + g * 27);
  return clip3(gmin, gmax, round2(gv, 5));
}

// The 8-sample groups of noise-stripe rows [ys, ye) of an item (columns
// x0 .. x1): load, film grain (grain.rs:186-354), pack. Specialised on the
// plane kind — CHROMA with its subsampling PSX / PSY (a chroma plane's
// luma sits at x << PSX, y << PSY), and the sample width — so the per-sample
// work has no run-time plane selects.
template <bool CHROMA, int PSX, int PSY, int SB>
__device__ __forceinline__ void out_stripe(const OutParams& P, const int16_t* T, const uint8_t* scale,
                                           const uint8_t* offs_cur, const uint8_t* offs_prev, const uint8_t* ssrc,
                                           const uint8_t* sluma, int x0, int x1, int ys, int ye, int stripe, int b0,
                                           bool grain) {
  // a lane keeps one 8-sample column group (one grain block's) on every
  // row it takes: the block, its template columns and the luma span are
  // found once
  const int ngroups = (x1 - x0 + 7) >> 3;  // 8-sample groups per row (<= 32)
  const int gx = threadIdx.x & 31;
  if (gx >= ngroups) return;
  const int sh = P.bd - 8;
  constexpr int bshift = 5 - PSX;  // grain block width 32 >> psx
  constexpr int sshift = 5 - PSY;  // noise stripe height 32 >> psy
  const int xs = x0 + gx * 8;
  const int n = min(8, x1 - xs);
  const int b = xs >> bshift;
  const int jb = xs - (b << bshift);
  const int li = b - b0 + 1;  // index into the staged offsets
  const bool hb = P.overlap && b > 0 && jb == 0;  // the block's first columns blend with the one to its left
  const int16_t* tp0 = tmpl_at(T, PSX, PSY, 0, offs_cur[li]) + jb;
  const int16_t* tl0 = left_at(T, PSX, PSY, 0, offs_cur[li - 1]);
  const int lx0 = xs << PSX, lbase = x0 << PSX;
  const bool lvec = n == 8 && lx0 + (8 << PSX) <= P.w;  // the luma span needs no edge clamp
  const int lm = P.lmult - 128, m = P.mult - 128, ov = (P.offs - 256) * (1 << sh);
  for (int r = threadIdx.x >> 5; r < ye - ys; r += 8) {
    const int yy = ys + r;
    int v[8];
    // the stripe's rows are staged (kStageSrc bytes a row, from column x0):
    // the group's 8 samples start 8 * SB-aligned
    const uint8_t* sp = ssrc + r * kStageSrc + gx * 8 * SB;
    const bool vec = n == 8;
    if (vec && SB == 2) {
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
        v[e] = e < n ? (SB == 1 ? int(sp[e]) : int(reinterpret_cast<const uint16_t*>(sp)[e])) : 0;
    }
    if (grain) {
      // noise image (grain.rs:251-283); the 8 samples share one grain block
      const int i = yy - (stripe << sshift);
      const bool vblend = P.overlap && stripe > 0 && i < (PSY ? 1 : 2);
      int lum[8];
      if (CHROMA) {
        // un-grained luma under each chroma sample (grain.rs:303-314), from
        // the staged luma row (kStageLuma bytes, from luma column x0 << PSX)
        const uint8_t* lrow = sluma + r * kStageLuma;
        const uint8_t* lp = lrow + (lx0 - lbase) * SB;
        // the group's whole luma span (8 or 16 samples) in 8-byte loads
        if (lvec) {
          uint32_t wv[8];
          const int nw = (8 << PSX) * SB / 4;  // 32-bit words: 2, 4 or 8
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (2 * q < nw) {
              const uint2 v2 = reinterpret_cast<const uint2*>(lp)[q];
              wv[2 * q] = v2.x;
              wv[2 * q + 1] = v2.y;
            }
          auto lsamp = [&](int k) {  // luma sample k of the span
            return SB == 2 ? int((wv[k >> 1] >> (16 * (k & 1))) & 0xffffu)
                             : int((wv[k >> 2] >> (8 * (k & 3))) & 0xffu);
          };
#pragma unroll
          for (int e = 0; e < 8; e++)
            lum[e] = PSX ? round2(lsamp(2 * e) + lsamp(2 * e + 1), 1) : lsamp(e);
        } else {
#pragma unroll
          for (int e = 0; e < 8; e++) {
            lum[e] = 0;  // (samples past the row's end: a valid table index, not stored)
            if (e < n) {
              const int lx = ((xs + e) << PSX) - lbase;
              const int lnx = min(lx + 1, P.w - 1 - lbase);
              const int l0 = SB == 1 ? int(lrow[lx]) : int(reinterpret_cast<const uint16_t*>(lrow)[lx]);
              const int l1 = SB == 1 ? int(lrow[lnx]) : int(reinterpret_cast<const uint16_t*>(lrow)[lnx]);
              lum[e] = PSX ? round2(l0 + l1, 1) : l0;
            }
          }
        }
      }
      // the group's noise (grain.rs:200-283): only a block's first 1-2
      // columns blend with the block to the left, and only a stripe's first
      // 1-2 rows with the stripe above
      const int16_t* tp = tp0 + i * kTW;
      int noise[8];
#pragma unroll
      for (int e = 0; e < 8; e++) noise[e] = tp[e];  // (all 8 inside the template row)
      // (the blend is computed for every group and kept where it applies:
      // the block to the left's columns are inside the template)
      const int16_t* tl = tl0 + i * kTW;
      noise[0] = hb ? hblend(tl[0], noise[0], 0, PSX, P.gmin, P.gmax) : noise[0];
      if (!PSX) noise[1] = hb ? hblend(tl[1], noise[1], 1, PSX, P.gmin, P.gmax) : noise[1];
      if (vblend) {
        const int vrow = i + (32 >> PSY);
        const int16_t* vp = tmpl_at(T, PSX, PSY, vrow, offs_prev[li]) + jb;
        int old[8];
#pragma unroll
        for (int e = 0; e < 8; e++) old[e] = vp[e];
        const int16_t* vl = left_at(T, PSX, PSY, vrow, offs_prev[li - 1]);
        old[0] = hb ? hblend(vl[0], old[0], 0, PSX, P.gmin, P.gmax) : old[0];
        if (!PSX) old[1] = hb ? hblend(vl[1], old[1], 1, PSX, P.gmin, P.gmax) : old[1];
        const int wo = PSY ? 23 : (i == 0 ? 27 : 17), wn = PSY ? 22 : (i == 0 ? 17 : 27);
#pragma unroll
        for (int e = 0; e < 8; e++) noise[e] = clip3(P.gmin, P.gmax, round2(old[e] * wo + noise[e] * wn, 5));
      }
      // scaling (grain.rs:166-177 through the full-resolution table), then
      // the sample plus scaled noise, clipped (grain.rs:316-350)
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int orig = v[e];
        int idx = orig;
        if (CHROMA) {
          const int mixed = clip3(0, P.maxpix, ((lum[e] * lm + orig * m) >> 6) + ov);
          idx = P.csfl ? lum[e] : mixed;
        }
        v[e] = clip3(P.min_value, P.max_v, orig + round2(int(scale[idx]) * noise[e], P.scaling_shift));
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
}

// Copies bytes [from, len) of `rows` rows, `pitch` bytes apart in global
// memory, to shared memory at `dst` (rows `stride` bytes apart), a warp per
// row: the part of a stripe's rows that the bulk copies do not move (a
// row's last len % 16 bytes, or whole rows of an unaligned plane).
__device__ __forceinline__ void copy_rows(uint8_t* dst, int stride, const uint8_t* src, int64_t pitch, int rows,
                                          int from, int len) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < rows; r += 8) {
    const uint8_t* g = src + int64_t(r) * pitch;
    uint8_t* d = dst + r * stride;
    for (int b = from + lane; b < len; b += 32) d[b] = g[b];
  }
}

// Dynamic shared memory of the output kernel: the bulk copies' barrier, the
// frame's descriptor, the plane's template and scaling table, the stripe's
// block offsets, and the stripe's source rows (up to 32 rows of 256
// samples) with, for chroma, the luma row under each (up to 512 luma
// samples: 256 chroma columns at 2:1).
struct OutSmem {
  uint64_t bar;
  FrameDesc fd;
  alignas(16) int16_t T[kTmplStride];
  alignas(16) uint8_t scale[4096];
  uint8_t offs_cur[kOutOffs + 6], offs_prev[kOutOffs + 6];  // block offsets of stripes s and s-1, blocks b0-1 ..
  alignas(16) uint8_t src[32 * kStageSrc];
  alignas(16) uint8_t luma[32 * kStageLuma];
};
constexpr int kOutSmem = int(sizeof(OutSmem));
constexpr int kOutWaitLimit = 1 << 16;  // bulk-copy waits of about 1 us each before ERRF_STALL

// Item: rows y0..y1 of a plane by up to 256 columns from x0, a multiple of
// 256 (so of the grain block width). A CTA works through a contiguous run of
// items. The rows are taken one noise stripe (32 rows, 16 for vertically
// subsampled chroma) at a time: the stripe's source rows and the luma rows a
// chroma stripe reads come into shared memory as one bulk copy per row (and
// a new plane's template and scaling table as two more), all completing on
// one barrier, while 18 threads fetch the stripe's block offsets; then 256
// threads take 8 consecutive samples (one grain block) each per row.
__global__ void __launch_bounds__(256, 2) output_kernel(const FrameDesc* __restrict__ frames,
                                                     const Item* __restrict__ items, int n_items) {
  AV1PF_TRACE_BEGIN();
  extern __shared__ __align__(16) uint8_t out_smem[];
  OutSmem& sm = *reinterpret_cast<OutSmem*>(out_smem);
  int16_t* T = sm.T;
  uint8_t* scale = sm.scale;
  uint8_t* offs_cur = sm.offs_cur;
  uint8_t* offs_prev = sm.offs_prev;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) mbar_init(&sm.bar, 1);
  uint32_t phase = 0;     // parity of the barrier's current phase
  int loaded = -1;        // frame * 4 + plane whose template is in T
  int loaded_frame = -1;  // the frame whose descriptor is in sm.fd
  // a CTA takes a contiguous run of items, the runs split as evenly as the
  // count allows: the items of a plane are consecutive, so a CTA stages that
  // plane's template once for its whole run
  const int it_begin = int(int64_t(blockIdx.x) * n_items / gridDim.x);
  const int it_end = int(int64_t(blockIdx.x + 1) * n_items / gridDim.x);
  if (it_begin < it_end) {
    // the first item's descriptor: copied from the host before any kernel
    // of the call ran, so it is fetched before waiting for the previous
    // stage (whose output, and the film-grain tables, are read only after)
    const Item first = items[it_begin];
    const uint2* fs = reinterpret_cast<const uint2*>(&frames[first.frame]);
    uint2* fdst = reinterpret_cast<uint2*>(&sm.fd);
    for (int k = tid; k < int(sizeof(FrameDesc) / 8); k += 256) fdst[k] = fs[k];
    loaded_frame = first.frame;
  }
  __syncthreads();  // (also publishes the barrier's initialisation)
  pdl_wait();  // the previous stage's output is complete past this point
  for (int it = it_begin; it < it_end; it++) {
    const Item item = items[it];
    if (int(item.frame) != loaded_frame) {
      // the descriptor's fields are read by every thread: from shared memory
      // (the previous stripe ended with a barrier, so no thread reads it now)
      const uint2* fs = reinterpret_cast<const uint2*>(&frames[item.frame]);
      uint2* fdst = reinterpret_cast<uint2*>(&sm.fd);
      for (int k = tid; k < int(sizeof(FrameDesc) / 8); k += 256) fdst[k] = fs[k];
      __syncthreads();
      loaded_frame = item.frame;
    }
    OutParams P;
    bool new_tables = false;  // the plane's template and table to fetch with the first stripe
    const FrameDesc& f = sm.fd;
    const int p = item.plane;
    {
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
        new_tables = key != loaded;
        loaded = key;
      }
    }
    const int x0 = item.x0, x1 = item.x1;
    const int bshift = 5 - P.psx;  // grain block width 32 >> psx
    const int sshift = 5 - P.psy;  // noise stripe height 32 >> psy
    const int b0 = x0 >> bshift;
    const bool luma_rows = p != 0 && P.grain;
    // the stripe's rows in global memory, and how much of each a bulk copy
    // moves (whole 16-byte units, when the plane's rows are 16-byte aligned)
    const uint8_t* s_src = P.src + int64_t(x0) * P.sb;
    const int s_len = (x1 - x0) * P.sb;
    const int s_bulk = ((reinterpret_cast<uintptr_t>(s_src) | uintptr_t(P.src_pitch)) & 15) == 0 ? s_len & ~15 : 0;
    const int64_t l_pitch = P.luma_pitch << P.psy;
    const uint8_t* l_src = P.luma + (int64_t(x0) << P.psx) * P.sb;
    const int l_len = (min(x1 << P.psx, P.w) - (x0 << P.psx)) * P.sb;
    const int l_bulk =
        luma_rows && ((reinterpret_cast<uintptr_t>(l_src) | uintptr_t(l_pitch)) & 15) == 0 ? l_len & ~15 : 0;
    for (int ys = item.y0; ys < int(item.y1);) {
      const int stripe = ys >> sshift;
      const int ye = min(int(item.y1), (stripe + 1) << sshift);
      const int rows = ye - ys;
      const uint8_t* srow = s_src + int64_t(ys) * P.src_pitch;
      const uint8_t* lrow = l_src + int64_t(ys) * l_pitch;
      const uint32_t tx = uint32_t(rows * (s_bulk + l_bulk)) +
                          (new_tables ? uint32_t(kTmplStride * 2 + (1 << P.bd)) : 0u);
      if (tx) {
        if (tid == 0) mbar_arrive_expect_tx(&sm.bar, tx);
        if (warp == 0 && lane < rows && s_bulk)
          bulk_g2s(sm.src + lane * kStageSrc, srow + int64_t(lane) * P.src_pitch, uint32_t(s_bulk), &sm.bar);
        if (warp == 1 && lane < rows && l_bulk)
          bulk_g2s(sm.luma + lane * kStageLuma, lrow + int64_t(lane) * l_pitch, uint32_t(l_bulk), &sm.bar);
        if (warp == 2 && new_tables) {
          if (lane == 0) bulk_g2s(T, &f.grain->tmpl[p][0], uint32_t(kTmplStride * 2), &sm.bar);
          if (lane == 1) bulk_g2s(scale, &f.grain->scale[p][0], uint32_t(1 << P.bd), &sm.bar);
        }
      }
      new_tables = false;
      // the rest of each row, by plain copies
      if (s_bulk < s_len) copy_rows(sm.src, kStageSrc, srow, P.src_pitch, rows, s_bulk, s_len);
      if (luma_rows && l_bulk < l_len) copy_rows(sm.luma, kStageLuma, lrow, l_pitch, rows, l_bulk, l_len);
      if (P.grain && tid < kOutOffs) {
        const int b = b0 - 1 + tid;
        const bool ok = b >= 0 && b < P.nb;
        offs_cur[tid] = ok ? P.off[int64_t(stripe) * P.nb + b] : 0;
        offs_prev[tid] = ok && stripe > 0 ? P.off[int64_t(stripe - 1) * P.nb + b] : 0;
      }
      if (tx) {
        if (!mbar_wait(&sm.bar, phase, kOutWaitLimit) && tid == 0) atomicOr(&g_error_flags, ERRF_STALL);
        phase ^= 1u;
      }
      __syncthreads();
      const uint8_t* ss = sm.src;
      const uint8_t* sl = sm.luma;
      if (p == 0) {
        if (P.sb == 2)
          out_stripe<false, 0, 0, 2>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain);
        else
          out_stripe<false, 0, 0, 1>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain);
      } else {
        const int k3 = (P.psx ? 2 : 0) + (P.psy ? 1 : 0) + (P.sb == 2 ? 4 : 0);
        switch (k3) {
          case 0: out_stripe<true, 0, 0, 1>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
          case 2: out_stripe<true, 1, 0, 1>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
          case 3: out_stripe<true, 1, 1, 1>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
          case 4: out_stripe<true, 0, 0, 2>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
          case 6: out_stripe<true, 1, 0, 2>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
          default: out_stripe<true, 1, 1, 2>(P, T, scale, offs_cur, offs_prev, ss, sl, x0, x1, ys, ye, stripe, b0, P.grain); break;
        }
      }
      __syncthreads();
      ys = ye;
    }
  }
  AV1PF_TRACE_END(4);
}

cudaError_t output_init() {
  return cudaFuncSetAttribute(output_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOutSmem);
}

void launch_grain_prep(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  launch_pdl(grain_prep_kernel, n_items, 256, 0, s, frames, items, n_items);
}

void launch_output(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  // one resident wave (2 CTAs per SM), each CTA a contiguous run of items
  launch_pdl(output_kernel, min(n_items, kNumSMs * 2), 256, size_t(kOutSmem), s, frames, items, n_items);
}

}  // namespace av1pf
