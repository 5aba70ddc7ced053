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
// Each source row is staged once in shared memory (16-byte loads), then every
// output sample reads its 8 taps from there and its filter phase's 8
// coefficients with one 16-byte load from global memory (through the L1),
// so CTAs start without staging the filter table. The row buffer is sized
// per launch to the widest source row among the launch's frames.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {
constexpr int kMaxRow = 16384 + 16;  // source samples staged per row, at most
}

__global__ void __launch_bounds__(256) superres_kernel(const FrameDesc* __restrict__ frames,
                                                       const Item* __restrict__ items, int n_items) {
  extern __shared__ __align__(16) uint8_t sr_smem[];
  uint16_t* row = reinterpret_cast<uint16_t*>(sr_smem);  // staged source row
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
    for (int r = item.y0; r < item.y1; r++) {
      int src_row = r;
      if (kind == 1) {
        const int s = r / 4 + 1, j = r % 4;
        const int B = (64 * s - 8) >> sy;
        src_row = B - 2 + j;
      }
      const bool live = src_row >= 0 && src_row < plane_h;  // uniform across the CTA
      if (live) {
        const uint8_t* sp = src.p + int64_t(prelf ? r : src_row) * src.stride * sb;
        if (sb == 2) {
          const int nv = n_src >> 3;
          for (int k = threadIdx.x; k < nv; k += blockDim.x)
            reinterpret_cast<uint4*>(row)[k] = reinterpret_cast<const uint4*>(sp)[k];
          for (int k = nv * 8 + threadIdx.x; k < n_src; k += blockDim.x)
            row[k] = reinterpret_cast<const uint16_t*>(sp)[k];
        } else {
          for (int k = threadIdx.x; k < n_src; k += blockDim.x) row[k] = sp[k];
        }
      }
      __syncthreads();
      if (live) {
        uint8_t* dp = dst.p + int64_t(r) * dst.stride * sb;
        for (int x = threadIdx.x; x < w; x += blockDim.x) {
          // postfilter.rs:547-561
          const int64_t src_x = -(int64_t(1) << 14) + init + int64_t(x) * step;
          const int px = int(src_x >> 14);
          const int phase = int((src_x & 0x3fff) >> 8);
          const int4 fq = __ldg(reinterpret_cast<const int4*>(g_upscale_filter[phase]));
          const uint32_t fw[4] = {uint32_t(fq.x), uint32_t(fq.y), uint32_t(fq.z), uint32_t(fq.w)};
          int fk[8];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            fk[2 * k] = int(int16_t(uint16_t(fw[k] & 0xffffu)));
            fk[2 * k + 1] = int(int16_t(uint16_t(fw[k] >> 16)));
          }
          int sum = 0;
          if (px - 3 >= 0 && px + 4 <= max_x) {
#pragma unroll
            for (int k = 0; k < 8; k++) sum += int(row[px - 3 + k]) * fk[k];
          } else {
#pragma unroll
            for (int k = 0; k < 8; k++) sum += int(row[min(max(px + k - 3, 0), max_x)]) * fk[k];
          }
          const int v = min(max(round2(sum, 7), 0), maxv);
          if (sb == 2)
            reinterpret_cast<uint16_t*>(dp)[x] = uint16_t(v);
          else
            dp[x] = uint8_t(v);
        }
      }
      __syncthreads();
    }
  }
}

cudaError_t superres_init() {
  return cudaFuncSetAttribute(superres_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxRow * 2);
}

void launch_superres(const FrameDesc* frames, const Item* items, int n_items, int row_max, cudaStream_t s) {
  if (n_items <= 0) return;
  const int row = min(max(row_max, 8), kMaxRow);
  launch_pdl(superres_kernel, min(n_items, kItemGrid), 256, size_t((row * 2 + 15) / 16 * 16), s, frames, items,
             n_items);
}

}  // namespace av1pf
