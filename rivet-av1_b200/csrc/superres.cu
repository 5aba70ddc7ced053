// superres.cu — super-resolution upscaling (7.16).
//
// Reference: rivet-av1 src/decoder/postfilter.rs:515-566 (`upscale`).
//
// The reference upscales the whole CDEF frame and the whole pre-CDEF frame;
// loop restoration reads the latter only at the 4 rows around each stripe
// boundary (LrCtx::sample, postfilter.rs:581-597), so here the pre-CDEF
// frame is upscaled only at those rows, into a small line buffer.
// Item kind 0: rows [y0, y1) of cdef -> up. Kind 1: line rows [y0, y1) of the
// line buffer (4 per stripe boundary: rows B-2 .. B+1 of the boundary at B).
// An item's (at most 4) source rows are staged together in shared memory
// (16-byte loads), behind one barrier; then the lanes of a warp make
// consecutive output samples, each reading its 8 taps from shared memory and
// its filter phase's 8 coefficients with one 16-byte load from global memory
// (through the L1). (Eight consecutive outputs per thread, stored as one
// vector, measured slower: a warp's lanes then read taps about 5 samples
// apart, and the bank conflicts cost more than the wider stores saved.)
// The row buffers are sized per launch to the widest source row among the
// launch's frames.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {
constexpr int kMaxRow = 16384 + 16;  // source samples staged per row, at most
constexpr int kRows = 4;             // rows per item
// row stride of the staged rows (u16): 16-byte aligned
__host__ __device__ constexpr int sr_stride(int n) { return (n + 7) & ~7; }
}  // namespace

__global__ void __launch_bounds__(256) superres_kernel(const FrameDesc* __restrict__ frames,
                                                       const Item* __restrict__ items, int n_items, int rs) {
  AV1PF_TRACE_BEGIN();
  extern __shared__ __align__(16) uint8_t sr_smem[];
  uint16_t* rows = reinterpret_cast<uint16_t*>(sr_smem);  // kRows staged source rows, rs apart
  pdl_wait();  // the previous stage's output is complete past this point
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    int p, sy, sb, maxv, step, init, max_x, w, plane_h, kind;
    bool prelf;
    DPlane src, dst;
    {
      const FrameDesc& f = frames[item.frame];
      p = item.plane;
      kind = item.kind;
      sy = plane_ssy(f, p);
      sb = f.sb;
      maxv = (1 << f.bd) - 1;
      step = f.sr_step[p];
      init = f.sr_init[p];
      max_x = f.sr_maxx[p];
      w = f.sr_w[p];
      plane_h = (f.fh + sy) >> sy;
      // kind 1 reads the loop filter's boundary rows: from the plane, or
      // from f.prelf when the CDEF kernel ran the horizontal LF pass
      prelf = kind == 1 && f.prelf[p].p != nullptr;
      src = kind == 0 ? f.cdef[p] : (prelf ? f.prelf[p] : f.cur[p]);
      dst = kind == 0 ? f.up[p] : f.lines[p];
    }
    const int n_src = max_x + 1;
    const int nr = min(int(item.y1) - int(item.y0), kRows);
    // the source row of output row y0 + k, or -1 outside the plane (uniform across the CTA)
    auto src_row_of = [&](int k) {
      const int r = item.y0 + k;
      int sr = r;
      if (kind == 1) {
        const int s = r / 4 + 1, j = r % 4;
        sr = ((64 * s - 8) >> sy) - 2 + j;
      }
      return sr >= 0 && sr < plane_h ? (prelf ? r : sr) : -1;
    };
    // --- stage the rows ---
    for (int k = 0; k < nr; k++) {
      const int sr = src_row_of(k);
      if (sr < 0) continue;
      const uint8_t* sp = src.p + int64_t(sr) * src.stride * sb;
      uint16_t* rp = rows + k * rs;
      if (sb == 2) {
        const int nv = n_src >> 3;
        for (int q = threadIdx.x; q < nv; q += blockDim.x)
          reinterpret_cast<uint4*>(rp)[q] = reinterpret_cast<const uint4*>(sp)[q];
        for (int q = nv * 8 + threadIdx.x; q < n_src; q += blockDim.x) rp[q] = reinterpret_cast<const uint16_t*>(sp)[q];
      } else {
        const int nv = n_src >> 4;
        for (int q = threadIdx.x; q < nv; q += blockDim.x) {
          const uint4 v = reinterpret_cast<const uint4*>(sp)[q];
          uint4* d = reinterpret_cast<uint4*>(rp + q * 16);
          d[0] = make_uint4(__byte_perm(v.x, 0, 0x4140), __byte_perm(v.x, 0, 0x4342), __byte_perm(v.y, 0, 0x4140),
                            __byte_perm(v.y, 0, 0x4342));
          d[1] = make_uint4(__byte_perm(v.z, 0, 0x4140), __byte_perm(v.z, 0, 0x4342), __byte_perm(v.w, 0, 0x4140),
                            __byte_perm(v.w, 0, 0x4342));
        }
        for (int q = nv * 16 + threadIdx.x; q < n_src; q += blockDim.x) rp[q] = sp[q];
      }
    }
    __syncthreads();
    // --- one output per thread and step (postfilter.rs:547-561): the lanes
    // of a warp make consecutive outputs, so their taps read neighbouring
    // (often the same) shared-memory words and their stores coalesce ---
    for (int k = 0; k < nr; k++) {
      if (src_row_of(k) < 0) continue;
      const uint16_t* rp = rows + k * rs;
      uint8_t* dp = dst.p + int64_t(item.y0 + k) * dst.stride * sb;
      for (int x = threadIdx.x; x < w; x += blockDim.x) {
        const int64_t src_x = -(int64_t(1) << 14) + init + int64_t(x) * step;
        const int px = int(src_x >> 14);
        const int phase = int((src_x & 0x3fff) >> 8);
        const int4 fq = __ldg(reinterpret_cast<const int4*>(g_upscale_filter[phase]));
        const uint32_t fw[4] = {uint32_t(fq.x), uint32_t(fq.y), uint32_t(fq.z), uint32_t(fq.w)};
        int sum = 0;
        if (px - 3 >= 0 && px + 4 <= max_x) {
#pragma unroll
          for (int t = 0; t < 4; t++) {
            sum += int(rp[px - 3 + 2 * t]) * int(int16_t(uint16_t(fw[t] & 0xffffu)));
            sum += int(rp[px - 2 + 2 * t]) * int(int16_t(uint16_t(fw[t] >> 16)));
          }
        } else {
#pragma unroll
          for (int t = 0; t < 4; t++) {
            sum += int(rp[min(max(px - 3 + 2 * t, 0), max_x)]) * int(int16_t(uint16_t(fw[t] & 0xffffu)));
            sum += int(rp[min(max(px - 2 + 2 * t, 0), max_x)]) * int(int16_t(uint16_t(fw[t] >> 16)));
          }
        }
        const int v = min(max(round2(sum, 7), 0), maxv);
        if (sb == 2)
          reinterpret_cast<uint16_t*>(dp)[x] = uint16_t(v);
        else
          dp[x] = uint8_t(v);
      }
    }
    __syncthreads();  // the rows are free for the next item
  }
  AV1PF_TRACE_END(5);
}

cudaError_t superres_init() {
  return cudaFuncSetAttribute(superres_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kRows * sr_stride(kMaxRow) * 2);
}

void launch_superres(const FrameDesc* frames, const Item* items, int n_items, int row_max, cudaStream_t s) {
  if (n_items <= 0) return;
  const int rs = sr_stride(min(max(row_max, 8), kMaxRow));
  launch_pdl(superres_kernel, min(n_items, kItemGrid), 256, size_t(kRows * rs * 2), s, frames, items, n_items, rs);
}

}  // namespace av1pf
