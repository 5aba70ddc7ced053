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
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

__global__ void __launch_bounds__(256) superres_kernel(const FrameDesc* __restrict__ frames,
                                                       const Item* __restrict__ items, int n_items) {
  __shared__ int16_t filt[64][8];
  for (int k = threadIdx.x; k < 64 * 8; k += blockDim.x) filt[k >> 3][k & 7] = g_upscale_filter[k >> 3][k & 7];
  __syncthreads();
  FOR_EACH_ITEM(it, n_items) {
    const Item item = items[it];
    const FrameDesc& f = frames[item.frame];
    const int p = item.plane;
    const int sy = plane_ssy(f, p);
    const int sb = f.sb;
    const int maxv = (1 << f.bd) - 1;
    const int step = f.sr_step[p], init = f.sr_init[p], max_x = f.sr_maxx[p], w = f.sr_w[p];
    const int plane_h = (f.fh + sy) >> sy;
    const DPlane src = item.kind == 0 ? f.cdef[p] : f.cur[p];
    const DPlane dst = item.kind == 0 ? f.up[p] : f.lines[p];
    for (int r = item.y0; r < item.y1; r++) {
      int sy_row = r;
      if (item.kind == 1) {
        const int s = r / 4 + 1, j = r % 4;
        const int B = (64 * s - 8) >> sy;
        sy_row = B - 2 + j;
        if (sy_row < 0 || sy_row >= plane_h) continue;
      }
      for (int x = threadIdx.x; x < w; x += blockDim.x) {
        // postfilter.rs:547-561
        const int64_t src_x = -(int64_t(1) << 14) + init + int64_t(x) * step;
        const int px = int(src_x >> 14);
        const int phase = int((src_x & 0x3fff) >> 8);
        int sum = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int sx = min(max(px + k - 3, 0), max_x);
          sum += ld_sample(src, sb, sx, sy_row) * filt[phase][k];
        }
        st_sample(dst, sb, x, r, min(max(round2(sum, 7), 0), maxv));
      }
    }
  }
}

void launch_superres(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s) {
  if (n_items <= 0) return;
  superres_kernel<<<min(n_items, kMaxGrid), 256, 0, s>>>(frames, items, n_items);
  note_launch();
}

}  // namespace av1pf
