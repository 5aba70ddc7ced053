// lf.cu — the deblocking loop filter (7.14) on the device.
//
// Reference: rivet-av1 src/decoder/postfilter.rs:63-264 (edge walk, filter
// size and strength) and src/dsp/lf.rs:58-211 (the sample filters).
//
// Design. The reference walks every 4x4 of a plane and filters edges in
// place, vertical edges first (bands of rows), then horizontal edges (bands
// of columns). Here:
//   1. lf_prep_kernel copies the pre-filter tile into the working plane and
//      decides, for every 4x4 and both passes, whether its edge is filtered
//      and with which size and level (edge_loop_filter's tests and
//      filter_strength, postfilter.rs:107-172, 207-264). Active edges are
//      appended (warp-aggregated) to one compact list per pass.
//   2. lf_edge_kernel<pass> runs one thread per (edge, lane) over the list,
//      in place, writing only the samples the chosen filter changes.
// Writing only changed samples makes the in-place passes order-independent:
// for conformant maps (transform blocks tile the plane) an edge's samples
// are read or changed by no other edge of the same pass, which is also what
// lets the reference run its bands on threads. The reference writes back
// its whole read span per edge; the extra samples it writes hold the values
// it read, so the results are the same.
#include "common.cuh"
#include "kernels.h"
#include "lf_core.cuh"

namespace av1pf {

__device__ const LfTables g_lf_tables = make_lf_tables();

// Edge list entry: frame:16 | plane:2 | code:2 | lvl:6 | cx:14 | cy:14.
__device__ __forceinline__ uint64_t pack_edge(int frame, int plane, int dec, int cx, int cy) {
  return uint64_t(frame) | (uint64_t(plane) << 16) | (uint64_t(dec) << 18) | (uint64_t(cx) << 26) |
         (uint64_t(cy) << 40);
}

__device__ __forceinline__ void append_edge(uint64_t* list, uint32_t* count, uint32_t cap, bool active,
                                            uint64_t e) {
  const unsigned mask = __ballot_sync(0xffffffffu, active);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, uint32_t(__popc(mask)));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (active) {
    const uint32_t pos = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
    if (pos < cap)
      list[pos] = e;
    else
      atomicOr(&g_error_flags, ERRF_BAD_ITEM);
  }
}

// Shared state of append_edges_cta.
struct EdgeAgg {
  uint32_t warp_off[2][8];  // per list: the warps' counts, then their offsets
  uint32_t base[2];         // per list: the CTA's first slot
};

// Appends the active edges of all 256 threads of the CTA (every thread
// calls) to two lists with one global atomic per list: each warp counts its
// edges with a ballot, one thread sums the counts in shared memory and
// reserves the CTA's range, and each edge goes to base + warp offset + rank.
// (Every warp of every tile adding to the same two counters serialises on
// them.)
__device__ __forceinline__ void append_edges_cta(EdgeAgg& agg, uint64_t* list_a, uint64_t* list_b, uint32_t* counts,
                                                 uint32_t cap, bool act_a, uint64_t ea, bool act_b, uint64_t eb) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned ma = __ballot_sync(0xffffffffu, act_a), mb = __ballot_sync(0xffffffffu, act_b);
  if (lane == 0) {
    agg.warp_off[0][warp] = uint32_t(__popc(ma));
    agg.warp_off[1][warp] = uint32_t(__popc(mb));
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    const int l = threadIdx.x;
    uint32_t run = 0;
    for (int w = 0; w < 8; w++) {
      const uint32_t n = agg.warp_off[l][w];
      agg.warp_off[l][w] = run;
      run += n;
    }
    agg.base[l] = run ? atomicAdd(&counts[l], run) : 0u;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  if (act_a) {
    const uint32_t pos = agg.base[0] + agg.warp_off[0][warp] + uint32_t(__popc(ma & lt));
    if (pos < cap)
      list_a[pos] = ea;
    else
      atomicOr(&g_error_flags, ERRF_BAD_ITEM);
  }
  if (act_b) {
    const uint32_t pos = agg.base[1] + agg.warp_off[1][warp] + uint32_t(__popc(mb & lt));
    if (pos < cap)
      list_b[pos] = eb;
    else
      atomicOr(&g_error_flags, ERRF_BAD_ITEM);
  }
  __syncthreads();  // agg is free for the next call
}

// Item: tile [x0,x1) x [y0,y1) of plane `plane` (samples). kind bit 0: copy
// in -> cur over the tile; bit 1: decide the tile's 4x4 edges. 256 threads.
__global__ void __launch_bounds__(256, 5) lf_prep_kernel(const FrameDesc* __restrict__ frames,
                                                      const Item* __restrict__ items, int n_items,
                                                      uint64_t* __restrict__ list_v, uint64_t* __restrict__ list_h,
                                                      uint32_t* __restrict__ counts, uint32_t cap) {
  const LfTables& tb = g_lf_tables;
  __shared__ EdgeAgg agg;
  pdl_wait();  // the previous stage's output is complete past this point
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int plane = item.plane;
    if (item.kind & 1) {
      // Copy the tile, 16 bytes at a time (rows are 16-byte aligned).
      const DPlane src = f.in[plane], dst = f.cur[plane];
      const int sb = f.sb;
      const int x0 = item.x0, x1 = min(int(item.x1), src.w);
      const int y0 = item.y0, y1 = min(int(item.y1), src.h);
      const int bx0 = x0 * sb, bx1 = x1 * sb;  // byte columns (a tile row is at most 128 bytes)
      const int nvec = (bx1 - bx0) >> 4;
      const int rows = y1 - y0;
      // 64 rows x 8 chunk slots = 2 per thread: both loads issue before the stores
      for (int k0 = threadIdx.x; k0 < rows * 8; k0 += 2 * blockDim.x) {
        uint4 q[2];
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const int k = k0 + m * blockDim.x;
          const int r = y0 + (k >> 3), c = bx0 + (k & 7) * 16;
          if (k < rows * 8 && (k & 7) < nvec)
            q[m] = *reinterpret_cast<const uint4*>(src.p + int64_t(r) * src.stride * sb + c);
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const int k = k0 + m * blockDim.x;
          const int r = y0 + (k >> 3), c = bx0 + (k & 7) * 16;
          if (k < rows * 8 && (k & 7) < nvec)
            *reinterpret_cast<uint4*>(dst.p + int64_t(r) * dst.stride * sb + c) = q[m];
        }
      }
      const int tail = (bx1 - bx0) & 15;
      if (tail) {
        for (int k = threadIdx.x; k < rows * 16; k += blockDim.x) {
          const int e = k & 15;
          if (e >= tail) continue;
          const int r = y0 + (k >> 4), c = bx0 + nvec * 16 + e;
          dst.p[int64_t(r) * dst.stride * sb + c] = src.p[int64_t(r) * src.stride * sb + c];
        }
      }
    }
    if (item.kind & 2) {
      const int sx = plane_ssx(f, plane), sy = plane_ssy(f, plane);
      const int gw = f.mi_cols >> sx, gh = f.mi_rows >> sy;  // 4x4 grid of the plane
      const int cx0 = item.x0 >> 2, cy0 = item.y0 >> 2;
      const int tw = (int(item.x1) - int(item.x0) + 3) >> 2;  // <= 16 (64-sample tiles)
      const int th = (int(item.y1) - int(item.y0) + 3) >> 2;
      // one 4x4 per thread (a 64x64 tile has 16 x 16 of them)
      const int k = threadIdx.x;
      const int cx = cx0 + (k & 15), cy = cy0 + (k >> 4);
      const bool in = k < th * 16 && (k & 15) < tw && cx < gw && cy < gh;
      int dv = 0, dh = 0;
      if (in) lf_decide2(f, tb, plane, cx, cy, dv, dh);
      append_edges_cta(agg, list_v, list_h, counts, cap, dv != 0, pack_edge(item.frame, plane, dv, cx, cy), dh != 0,
                       pack_edge(item.frame, plane, dh, cx, cy));
    }
  }
}

// Loads samples s[e+k], k in [k0, k0+n), along the filter direction.
template <int PASS>
__device__ __forceinline__ void lf_load(const DPlane& p, int sb, int e, int lanepos, int k0, int n, int32_t* out) {
  if (PASS == 0) {
    // row `lanepos`, columns e+k0 .. (k0 is -4 or -8: 4-sample aligned)
    const uint8_t* row = p.p + int64_t(lanepos) * p.stride * sb;
    if (sb == 2) {
      const uint2* q = reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(row) + e + k0);
      for (int g = 0; g < n / 4; g++) {
        const uint2 w = q[g];
        out[4 * g + 0] = int32_t(w.x & 0xffffu);
        out[4 * g + 1] = int32_t(w.x >> 16);
        out[4 * g + 2] = int32_t(w.y & 0xffffu);
        out[4 * g + 3] = int32_t(w.y >> 16);
      }
    } else {
      const uint32_t* q = reinterpret_cast<const uint32_t*>(row + e + k0);
      for (int g = 0; g < n / 4; g++) {
        const uint32_t w = q[g];
        out[4 * g + 0] = int32_t(w & 0xffu);
        out[4 * g + 1] = int32_t((w >> 8) & 0xffu);
        out[4 * g + 2] = int32_t((w >> 16) & 0xffu);
        out[4 * g + 3] = int32_t(w >> 24);
      }
    }
  } else {
    for (int k = 0; k < n; k++) out[k] = ld_sample(p, sb, lanepos, e + k0 + k);
  }
}

template <int PASS>
__global__ void __launch_bounds__(256, 4) lf_edge_kernel(const FrameDesc* __restrict__ frames,
                                                      const uint64_t* __restrict__ list,
                                                      const uint32_t* __restrict__ count_ptr, uint32_t cap) {
  pdl_wait();  // the edge list and count are complete past this point
  const uint32_t n = min(*count_ptr, cap) * 4u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t e = list[i >> 2];
    const int lane = int(i & 3u);
    const int frame = int(e & 0xffffu);
    const int plane = int((e >> 16) & 3u);
    const int code = int((e >> 24) & 3u);
    const int lvl = int((e >> 18) & 63u);
    const int cx = int((e >> 26) & 0x3fffu), cy = int((e >> 40) & 0x3fffu);
    const FrameDesc& f = frames[frame];
    const int sb = f.sb, bd = f.bd;
    const DPlane p = f.cur[plane];
    const int filter_size = code == 3 ? 16 : (code == 2 ? 8 : 4);
    int limit, blimit, thresh;
    lf_limits(lvl, f.sharpness, limit, blimit, thresh);
    const int epos = PASS == 0 ? cx * 4 : cy * 4;              // q0 along the filter direction
    const int lanepos = PASS == 0 ? cy * 4 + lane : cx * 4 + lane;  // row (pass 0) / column (pass 1)
    // A conformant map never puts a wide edge this close to the plane start
    // (the transform before it is at least as wide as the filter).
    if (epos < (filter_size >= 16 ? 8 : 4)) {
      atomicOr(&g_error_flags, ERRF_BAD_MAP);
      continue;
    }
    int32_t v[14];
#pragma unroll
    for (int k = 0; k < 14; k++) v[k] = 0;
    if (filter_size >= 16) {
      int32_t tmp[16];
      lf_load<PASS>(p, sb, epos, lanepos, -8, 16, tmp);
#pragma unroll
      for (int k = 0; k < 14; k++) v[k] = tmp[k + 1];
    } else {
      int32_t tmp[8];
      lf_load<PASS>(p, sb, epos, lanepos, -4, 8, tmp);
#pragma unroll
      for (int k = 0; k < 8; k++) v[k + 3] = tmp[k];
    }
    int lo, hi;
    lf_filter_one(v, filter_size, plane != 0, bd, limit, blimit, thresh, lo, hi);
#pragma unroll
    for (int k = 1; k < 13; k++) {
      if (k < lo || k >= hi) continue;
      const int pos = epos + k - 7;
      if (PASS == 0)
        st_sample(p, sb, pos, lanepos, v[k]);
      else
        st_sample(p, sb, lanepos, pos, v[k]);
    }
  }
}

namespace {
constexpr int kLfTile = 64;                  // tile side (samples)
constexpr int kLfHalo = 16;                  // columns staged on each side
constexpr int kLfTS = 104;                   // tile row stride (u16): >= 64 + 2 * 16, rows 16-byte aligned
constexpr int kLfCells = kLfTile / 4 + 2;    // 4x4 columns decided: the tile's 16 plus one each side
}  // namespace

// Loop filter, vertical edges, one 64x64 tile per CTA (kind bit 0: the tile
// is copied in -> cur; bit 1: it overlaps the mode-info area and its
// vertical edges are filtered; bit 2: its horizontal edges are appended to
// list_h for lf_edge_kernel<1>). The tile and 16 columns on each side are
// staged from the unfiltered input, so edges of neighbouring tiles that
// reach into this one (at most 6 samples) are filtered here too, from the
// same input, and no tile reads what another writes. Each tile writes only
// its own samples of cur. 256 threads.
__global__ void __launch_bounds__(256, 4) lf_tile_kernel(const FrameDesc* __restrict__ frames,
                                                      const Item* __restrict__ items, int n_items,
                                                      uint64_t* __restrict__ list_h, uint32_t* __restrict__ counts,
                                                      uint32_t cap) {
  const LfTables& tb = g_lf_tables;
  __shared__ __align__(16) uint16_t T[kLfTile * kLfTS];
  __shared__ uint16_t dec[kLfTile / 4][kLfCells];  // vertical-edge decisions
  const int tid = threadIdx.x;
  pdl_wait();  // the previous stage's output is complete past this point
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int plane = item.plane;
    const DPlane src = f.in[plane], dst = f.cur[plane];
    const int sb = f.sb;
    const int x0 = item.x0, y0 = item.y0;
    const int x1 = min(int(item.x1), src.w), y1 = min(int(item.y1), src.h);
    const int rows = y1 - y0;
    const bool filt = (item.kind & 2) != 0;
    __syncthreads();  // the previous item's tile is written out
    // --- stage columns [x0 - 16, x0 + 80) of rows [y0, y1): 16-byte chunks ---
    {
      const int cw = 16 / sb;                    // samples per chunk
      const int nch = (kLfTile + 2 * kLfHalo) / cw;  // 6 or 12 chunks per row
      const int c_lo = filt ? 0 : kLfHalo / cw;  // a copy-only tile needs no halo
      const int c_hi = filt ? nch : (kLfHalo + kLfTile) / cw;
      for (int k = tid; k < rows * 12; k += 256) {
        const int r = k / 12, ch = k - r * 12;
        if (ch < c_lo || ch >= c_hi) continue;
        const int gx = x0 - kLfHalo + ch * cw;  // first sample of the chunk
        const uint8_t* rp = src.p + int64_t(y0 + r) * src.stride * sb;
        uint16_t* tp = &T[r * kLfTS + ch * cw];
        if (gx >= 0 && gx + cw <= src.w) {
          const uint4 q = *reinterpret_cast<const uint4*>(rp + int64_t(gx) * sb);
          if (sb == 2) {
            *reinterpret_cast<uint4*>(tp) = q;
          } else {
            const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
              reinterpret_cast<uint32_t*>(tp)[2 * e] = __byte_perm(w4[e], 0, 0x4140);
              reinterpret_cast<uint32_t*>(tp)[2 * e + 1] = __byte_perm(w4[e], 0, 0x4342);
            }
          }
        } else {
          for (int e = 0; e < cw; e++) {
            const int x = gx + e;
            tp[e] = (x >= 0 && x < src.w) ? uint16_t(sb == 1 ? rp[x] : reinterpret_cast<const uint16_t*>(rp)[x]) : 0;
          }
        }
      }
    }
    if (filt) {
      // --- decisions: the tile's 4x4 rows x (its 16 columns + one each side) ---
      const int sx = plane_ssx(f, plane), sy = plane_ssy(f, plane);
      const int gw = f.mi_cols >> sx, gh = f.mi_rows >> sy;
      const int cx0 = (x0 >> 2) - 1, cy0 = y0 >> 2;
      const int th = (rows + 3) >> 2;
      const int tw_end = (x1 - x0 + 3) >> 2;  // tile columns (cells 1 .. tw_end)
      for (int k = tid; k < (kLfTile / 4) * 32; k += 256) {
        const int cyi = k >> 5, cxi = k & 31;
        const int cx = cx0 + cxi, cy = cy0 + cyi;
        const bool in = cxi < kLfCells && cyi < th && cx >= 0 && cx < gw && cy < gh;
        int dv = 0, dh = 0;
        if (in) lf_decide2(f, tb, plane, cx, cy, dv, dh);
        if (cxi < kLfCells && cyi < kLfTile / 4) dec[cyi][cxi] = uint16_t(dv);
        if (item.kind & 4) {
          const bool own = in && cxi >= 1 && cxi <= tw_end && dh != 0;
          append_edge(list_h, &counts[1], cap, own, pack_edge(item.frame, plane, dh, cx, cy));
        }
      }
      __syncthreads();
      // --- vertical edges in shared memory: (cell, row lane) per thread ---
      const int bd = f.bd, sharp = f.sharpness;
      for (int k = tid; k < th * kLfCells * 4; k += 256) {
        const int lane = k & 3, cell = k >> 2;
        const int cyi = cell / kLfCells, cxi = cell - cyi * kLfCells;
        const int d = dec[cyi][cxi];
        if (!d) continue;
        const int code = d >> 6, lvl = d & 63;
        const int r = cyi * 4 + lane;
        if (r >= rows) continue;
        const int e = (cx0 + cxi) * 4;  // plane column of q0
        if (e < (code == 3 ? 8 : 4)) {  // a conformant map keeps wide edges off the plane start
          atomicOr(&g_error_flags, ERRF_BAD_MAP);
          continue;
        }
        lf_filter_smem(&T[r * kLfTS + (e - x0 + kLfHalo)], 1, code, plane != 0, bd, lvl, sharp);
      }
    }
    __syncthreads();
    // --- write the tile's own samples [x0, x1) x [y0, y1) ---
    {
      const int w = x1 - x0;
      const int nv = w >> 3;  // 8-sample groups
      for (int k = tid; k < rows * 8; k += 256) {
        const int r = k >> 3, g = k & 7;
        uint8_t* rp = dst.p + int64_t(y0 + r) * dst.stride * sb;
        const uint16_t* tp = &T[r * kLfTS + kLfHalo + g * 8];
        if (g < nv) {
          const uint4 q = *reinterpret_cast<const uint4*>(tp);
          if (sb == 2) {
            *reinterpret_cast<uint4*>(rp + int64_t(x0 + g * 8) * 2) = q;
          } else {
            *reinterpret_cast<uint2*>(rp + x0 + g * 8) =
                make_uint2(__byte_perm(q.x, q.y, 0x6420), __byte_perm(q.z, q.w, 0x6420));
          }
        } else if (g == nv) {
          for (int e = 0; e < w - nv * 8; e++) {
            if (sb == 2)
              reinterpret_cast<uint16_t*>(rp)[x0 + g * 8 + e] = tp[e];
            else
              rp[x0 + g * 8 + e] = uint8_t(tp[e]);
          }
        }
      }
    }
  }
}

namespace {
constexpr int kFT = 64;             // fused tile side (samples)
constexpr int kFH = 8;              // halo on each side: the widest filter reads 7 samples past its edge
constexpr int kFW = kFT + 2 * kFH;  // window side (80)
constexpr int kFS = 88;             // window row stride (u16): rows 16-byte aligned
constexpr int kFCR = kFW / 4;       // 4x4 rows of the window (20): vertical edges of every staged row
constexpr int kFCC = kFT / 4 + 1;   // 4x4 columns with vertical edges (17): the tile's 16 + the right neighbour's first
constexpr int kFCells = kFCR * kFCC;
constexpr int kFChunks = kFW / 8 * kFW;  // 8-sample chunks of the window (800)
}  // namespace

// Loop filter, both passes, one 64x64 tile per CTA (kind bit 0: the tile is
// copied in -> cur; bit 1: it overlaps the mode-info area and is filtered).
// The tile and 8 samples on every side are staged once from the unfiltered
// input. Every vertical edge that changes a staged row at the tile's columns
// (edges at x0 .. x0 + 64) is filtered in shared memory, including the 8
// halo rows above and below, which the horizontal edges at y0 .. y0 + 64
// read; then those horizontal edges are filtered, and only the tile's own
// samples are written to cur. Neighbouring tiles recompute the halo rows'
// vertical edges and the shared horizontal edge at their boundary from the
// same input, so no tile reads what another writes. This is exact by the
// same property as the in-place passes: for conformant maps no edge of a
// pass reads a sample another edge of that pass changes. The active edges of
// each pass are listed in shared memory grouped by filter size, so a warp's
// lanes mostly take one filter path. 256 threads.
__global__ void __launch_bounds__(256, 4) lf_fused_kernel(const FrameDesc* __restrict__ frames,
                                                       const Item* __restrict__ items, int n_items,
                                                       uint32_t* __restrict__ flags) {
  AV1PF_TRACE_BEGIN();
  const LfTables& tb = g_lf_tables;
  __shared__ __align__(16) uint16_t W[kFW * kFS];
  __shared__ uint32_t list_v[kFCells], list_h[kFCells];
  __shared__ uint32_t cnt[2][4], base[2][4];
  const int tid = threadIdx.x;
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int plane = item.plane;
    const DPlane src = f.in[plane], dst = f.cur[plane];
    const int sb = f.sb;
    const int x0 = item.x0, y0 = item.y0;
    const int x1 = min(int(item.x1), src.w), y1 = min(int(item.y1), src.h);
    const int rows = y1 - y0;
    const bool filt = (item.kind & 2) != 0;
    const int wx0 = x0 - kFH, wy0 = y0 - kFH;
    if (tid < 8) (&cnt[0][0])[tid] = 0u;  // every thread read the previous item's counts
    __syncthreads();  // the previous item's window is written out
    // --- stage the window: a filtered tile takes all of it, a copied one its own samples ---
    const int r_lo = filt ? 0 : kFH, r_hi = filt ? kFW : kFH + rows;
    const int c_lo = filt ? 0 : 1, c_hi = filt ? kFW / 8 : 1 + kFT / 8;
    uint2 q8[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int k = tid + m * 256;
      const int r = k / 10, ch = k - r * 10;
      q8[m] = make_uint2(0u, 0u);
      if (k >= kFChunks || r < r_lo || r >= r_hi || ch < c_lo || ch >= c_hi) continue;
      const int gy = wy0 + r, gx = wx0 + ch * 8;
      uint16_t* wp = &W[r * kFS + ch * 8];
      if (gy < 0 || gy >= src.h) {
        *reinterpret_cast<uint4*>(wp) = make_uint4(0u, 0u, 0u, 0u);
        continue;
      }
      const uint8_t* rp = src.p + int64_t(gy) * src.stride * sb;
      if (gx >= 0 && gx + 8 <= src.w) {
        if (sb == 2)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(
                           __cvta_generic_to_shared(wp))),
                       "l"(rp + int64_t(gx) * 2)
                       : "memory");
        else
          q8[m] = *reinterpret_cast<const uint2*>(rp + gx);
      } else {
        for (int e = 0; e < 8; e++) {
          const int x = gx + e;
          wp[e] = (x >= 0 && x < src.w) ? uint16_t(sb == 1 ? rp[x] : reinterpret_cast<const uint16_t*>(rp)[x]) : 0;
        }
      }
    }
    // --- decisions: vertical edges of the window's 20 x 17 cells, horizontal
    // edges of the tile's 17 x 16 (postfilter.rs:107-264) ---
    int dv[2] = {0, 0}, dh[2] = {0, 0};
    const int cx0 = x0 >> 2, cy0 = (y0 >> 2) - 2;
    if (filt) {
      const int sx = plane_ssx(f, plane), sy = plane_ssy(f, plane);
      const int gw = f.mi_cols >> sx, gh = f.mi_rows >> sy;
#pragma unroll
      for (int m = 0; m < 2; m++) {
        const int k = tid + m * 256;
        if (k >= kFCells) break;
        const int i = k / kFCC, j = k - i * kFCC;
        const int cx = cx0 + j, cy = cy0 + i;
        if (cx < 0 || cy < 0 || cx >= gw || cy >= gh) continue;
        int v = 0, h = 0;
        lf_decide2(f, tb, plane, cx, cy, v, h);
        // a conformant map keeps wide edges off the plane start
        if (v && cx * 4 < ((v >> 6) == 3 ? 8 : 4)) {
          atomicOr(&g_error_flags, ERRF_BAD_MAP);
          v = 0;
        }
        if (h && cy * 4 < ((h >> 6) == 3 ? 8 : 4)) {
          atomicOr(&g_error_flags, ERRF_BAD_MAP);
          h = 0;
        }
        dv[m] = v;
        if (i >= 2 && i <= 2 + kFT / 4 && j < kFT / 4) dh[m] = h;
      }
    }
    // u8 samples widen to the u16 window
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int k = tid + m * 256;
      const int r = k / 10, ch = k - r * 10;
      if (sb != 1 || k >= kFChunks || r < r_lo || r >= r_hi || ch < c_lo || ch >= c_hi) continue;
      const int gy = wy0 + r, gx = wx0 + ch * 8;
      if (gy < 0 || gy >= src.h || gx < 0 || gx + 8 > src.w) continue;
      uint16_t* wp = &W[r * kFS + ch * 8];
      *reinterpret_cast<uint4*>(wp) =
          make_uint4(__byte_perm(q8[m].x, 0, 0x4140), __byte_perm(q8[m].x, 0, 0x4342),
                     __byte_perm(q8[m].y, 0, 0x4140), __byte_perm(q8[m].y, 0, 0x4342));
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (filt) {
      // --- the active edges of each pass, grouped by filter size ---
      uint32_t iv[2], ih[2];
#pragma unroll
      for (int m = 0; m < 2; m++) {
        iv[m] = dv[m] ? atomicAdd(&cnt[0][dv[m] >> 6], 1u) : 0u;
        ih[m] = dh[m] ? atomicAdd(&cnt[1][dh[m] >> 6], 1u) : 0u;
      }
      __syncthreads();
      if (tid < 2) {
        uint32_t run = 0;
        for (int c = 3; c >= 1; c--) {
          base[tid][c] = run;
          run += cnt[tid][c];
        }
        cnt[tid][0] = run;  // the pass's edge count
      }
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 2; m++) {
        const int k = tid + m * 256;
        const int i = k / kFCC, j = k - i * kFCC;
        if (dv[m]) list_v[base[0][dv[m] >> 6] + iv[m]] = uint32_t(j) | (uint32_t(i) << 5) | (uint32_t(dv[m]) << 10);
        if (dh[m]) list_h[base[1][dh[m] >> 6] + ih[m]] = uint32_t(j) | (uint32_t(i - 2) << 5) | (uint32_t(dh[m]) << 10);
      }
      __syncthreads();
      const int bd = f.bd, sharp = f.sharpness;
      const bool chroma = plane != 0;
      // --- vertical edges: (edge, row lane) per thread ---
      const int nv = int(cnt[0][0]) * 4;
      for (int t = tid; t < nv; t += 256) {
        const uint32_t e = list_v[t >> 2];
        const int j = int(e & 31u), i = int((e >> 5) & 31u), d = int(e >> 10);
        lf_filter_smem(&W[(i * 4 + (t & 3)) * kFS + kFH + j * 4], 1, d >> 6, chroma, bd, d & 63, sharp);
      }
      __syncthreads();
      // --- horizontal edges: (edge, column lane) per thread ---
      const int nh = int(cnt[1][0]) * 4;
      for (int t = tid; t < nh; t += 256) {
        const uint32_t e = list_h[t >> 2];
        const int j = int(e & 31u), i = int((e >> 5) & 31u), d = int(e >> 10);
        lf_filter_smem(&W[(kFH + i * 4) * kFS + kFH + j * 4 + (t & 3)], kFS, d >> 6, chroma, bd, d & 63, sharp);
      }
    }
    __syncthreads();
    // Up to here the tile read only this call's inputs (the unfiltered
    // planes, the maps, the descriptor) and worked in shared memory, so it
    // ran while the previous call's stages drained; cur, which they read,
    // is written only past this wait.
    pdl_wait();
    // --- write the tile's own samples [x0, x1) x [y0, y1) ---
    {
      const int w = x1 - x0;
      const int nvec = w >> 3;  // 8-sample groups
      for (int k = tid; k < rows * 8; k += 256) {
        const int r = k >> 3, g = k & 7;
        uint8_t* rp = dst.p + int64_t(y0 + r) * dst.stride * sb;
        const uint16_t* wp = &W[(kFH + r) * kFS + kFH + g * 8];
        if (g < nvec) {
          const uint4 q = *reinterpret_cast<const uint4*>(wp);
          if (sb == 2)
            *reinterpret_cast<uint4*>(rp + int64_t(x0 + g * 8) * 2) = q;
          else
            *reinterpret_cast<uint2*>(rp + x0 + g * 8) =
                make_uint2(__byte_perm(q.x, q.y, 0x6420), __byte_perm(q.z, q.w, 0x6420));
        } else if (g == nvec) {
          for (int e = 0; e < w - nvec * 8; e++) {
            if (sb == 2)
              reinterpret_cast<uint16_t*>(rp)[x0 + g * 8 + e] = wp[e];
            else
              rp[x0 + g * 8 + e] = uint8_t(wp[e]);
          }
        }
      }
    }
    if (flags) {
      // the tile is in cur: its readiness flag (the barrier orders every
      // thread's stores before the release)
      __syncthreads();
      if (tid == 0) flag_set(flags + f.lf_flag_base[plane] + (y0 / kFT) * f.lf_tiles_x[plane] + x0 / kFT);
    }
  }
  AV1PF_TRACE_END(1);
}

// dsp::lf::filter (lf.rs:25) on independent edges: one thread per lane.
__global__ void dsp_lf_kernel(int32_t* __restrict__ edges, const av1pf_lf_edge_params* __restrict__ prm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * 4) return;
  const int e = i >> 2, lane = i & 3;
  const av1pf_lf_edge_params p = prm[e];
  int32_t v[14];
#pragma unroll
  for (int k = 0; k < 14; k++) v[k] = edges[int64_t(e) * 56 + k * 4 + lane];
  int lo, hi;
  lf_filter_one(v, p.filter_size, p.chroma != 0, p.bit_depth, p.limit, p.blimit, p.thresh, lo, hi);
#pragma unroll
  for (int k = 0; k < 14; k++)
    if (k >= lo && k < hi) edges[int64_t(e) * 56 + k * 4 + lane] = v[k];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_lf_prep(const FrameDesc* frames, const Item* items, int n_items, uint64_t* list_v, uint64_t* list_h,
                    uint32_t* counts, uint32_t cap, cudaStream_t s) {
  if (n_items <= 0) return;
  const int grid = min(n_items, kItemGrid);
  launch_pdl(lf_prep_kernel, grid, 256, 0, s, frames, items, n_items, list_v, list_h, counts, cap);
}

void launch_lf_tiles(const FrameDesc* frames, const Item* items, int n_items, uint64_t* list_h, uint32_t* counts,
                     uint32_t cap, cudaStream_t s) {
  if (n_items <= 0) return;
  launch_pdl(lf_tile_kernel, min(n_items, kItemGrid), 256, 0, s, frames, items, n_items, list_h, counts, cap);
}

void launch_lf_fused(const FrameDesc* frames, const Item* items, int n_items, uint32_t* flags, cudaStream_t s) {
  if (n_items <= 0) return;
  launch_pdl(lf_fused_kernel, min(n_items, kItemGrid), 256, 0, s, frames, items, n_items, flags);
}

void launch_lf_edges(int pass, const FrameDesc* frames, const uint64_t* list, const uint32_t* count, uint32_t cap,
                     cudaStream_t s) {
  // The edge count is only known on the device: a fixed grid strides over it.
  const int grid = kMaxGrid;
  if (pass == 0)
    launch_pdl(lf_edge_kernel<0>, grid, 256, 0, s, frames, list, count, cap);
  else
    launch_pdl(lf_edge_kernel<1>, grid, 256, 0, s, frames, list, count, cap);
}

void launch_dsp_lf(int32_t* edges, const av1pf_lf_edge_params* prm, int n, cudaStream_t s) {
  if (n <= 0) return;
  dsp_lf_kernel<<<(n * 4 + 255) / 256, 256, 0, s>>>(edges, prm, n);
  note_launch();
}

}  // namespace av1pf
