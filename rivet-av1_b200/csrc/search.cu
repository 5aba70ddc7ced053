// search.cu — the encoder's filter searches on the device: the greedy choice
// of CDEF strength pairs (encoder/cdef.rs:195-250) over the error table that
// cdef_search_kernel (cdef.cu) fills, and the plane errors of the
// loop-filter level search (encoder/mod.rs:1494-1506).
//
// The reference sums block errors into an f64 in block order
// (`total += best as f64`). Every block error is an integer far below 2^53,
// so while a total stays below 2^53 each of those additions is exact and the
// f64 total equals the exact integer sum: the kernels sum in u64 (in any
// order) and convert. A total at or above 2^53 (frames of more than ~45,000
// 64x64 blocks at 12 bits) is summed again in f64, in block order, as the
// reference does. The cost of a choice, t + lambda * bits * nb, is evaluated
// with round-to-nearest multiplies and adds in the reference's order (no
// fused multiply-add).
#include <cfloat>

#include "common.cuh"
#include "kernels.h"

namespace av1pf {

namespace {

constexpr uint64_t kExact = uint64_t(1) << 53;

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The reference's f64 total, in block order, of min(best[b], last pair,
// pair (Y, U)) over the blocks (blocks that code no index hold 0 everywhere
// and add nothing). L / Y may be null (no last pair / no candidate).
__device__ double ordered_total(const uint64_t* best, const uint64_t* YL, const uint64_t* UL, const uint64_t* Y,
                                const uint64_t* U, int nfb) {
  double t = 0.0;
  for (int b = 0; b < nfb; b++) {
    uint64_t v = __ldcg(&best[b]);
    if (YL) v = min(v, YL[b] + UL[b]);
    if (Y) v = min(v, Y[b] + U[b]);
    t = __dadd_rn(t, double(v));
  }
  return t;
}

// (total, candidate) of the smaller, the first candidate on equal totals;
// candidate -1 is none.
__device__ __forceinline__ void argmin_pair(double& t, int& c, double t2, int c2) {
  if (c2 >= 0 && (c < 0 || t2 < t || (t2 == t && c2 < c))) {
    t = t2;
    c = c2;
  }
}

// Step k of the greedy (encoder/cdef.rs:215-232). A warp per candidate pair
// scores sum_b min(best[b], last[b], Y[yk][b] + UV[uk][b]) — the reference's
// best_for(set + pair): best[b] holds the minimum over the set but for its
// newest pair `last`, which every scorer folds in (and CTA 0 writes back;
// the min is idempotent, so readers that see either value agree). Lanes
// stride over the blocks (candidate-major table: coalesced, four blocks in
// flight per lane). The last CTA to finish (a fenced arrival count; no CTA
// waits) takes the smallest total, first in (yk, uk) order on ties, and adds
// its pair to the set. Its total is the new set's total, so at set sizes 1,
// 2, 4 and 8 it prices the set from it (encoder/cdef.rs:233-239). The
// candidate lists hold at least 420 pairs, so a pair always remains.
// Launched with programmatic dependent launch: the state is read after
// pdl_wait(). A batch of frames runs side by side: `cpf` CTAs per frame,
// each frame with its own state and arrival count.
__global__ void __launch_bounds__(256) cdef_greedy_step_kernel(const CdefSearchDesc* __restrict__ ds, int cpf) {
  const int fi = blockIdx.x / cpf, lb = blockIdx.x - fi * cpf;
  const CdefSearchDesc& d = ds[fi];
  CdefGreedy* g = d.g;
  uint64_t* tot = d.tot;
  const double lambda = d.lambda;
  const int nfb = d.fb_rows * d.fb_cols, ncand = d.ny * d.nuv;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  pdl_wait();
  const int n = g->n;
  const uint64_t* YL = n ? d.sse + int64_t(g->set_y[n - 1]) * nfb : nullptr;
  const uint64_t* UL = n ? d.sse + int64_t(d.ny + g->set_uv[n - 1]) * nfb : nullptr;
  if (n && lb == 0)
    for (int b = tid; b < nfb; b += blockDim.x) d.best[b] = min(d.best[b], YL[b] + UL[b]);
  const int c = lb * 8 + warp;
  if (c < ncand) {
    const int yk = c / d.nuv, uk = c - yk * d.nuv;
    bool in_set = false;
    for (int i = 0; i < n; i++) in_set |= g->set_y[i] == yk && g->set_uv[i] == uk;
    uint64_t acc = 0;
    if (!in_set) {
      const uint64_t* Y = d.sse + int64_t(yk) * nfb;
      const uint64_t* U = d.sse + int64_t(d.ny + uk) * nfb;
      const uint64_t* B = d.best;
      uint64_t a1 = 0, a2 = 0, a3 = 0;
      int b = lane;
      if (n) {
        for (; b + 96 < nfb; b += 128) {
          acc += min(min(B[b], YL[b] + UL[b]), Y[b] + U[b]);
          a1 += min(min(B[b + 32], YL[b + 32] + UL[b + 32]), Y[b + 32] + U[b + 32]);
          a2 += min(min(B[b + 64], YL[b + 64] + UL[b + 64]), Y[b + 64] + U[b + 64]);
          a3 += min(min(B[b + 96], YL[b + 96] + UL[b + 96]), Y[b + 96] + U[b + 96]);
        }
        for (; b < nfb; b += 32) acc += min(min(B[b], YL[b] + UL[b]), Y[b] + U[b]);
      } else {
        for (; b + 96 < nfb; b += 128) {
          acc += min(B[b], Y[b] + U[b]);
          a1 += min(B[b + 32], Y[b + 32] + U[b + 32]);
          a2 += min(B[b + 64], Y[b + 64] + U[b + 64]);
          a3 += min(B[b + 96], Y[b + 96] + U[b + 96]);
        }
        for (; b < nfb; b += 32) acc += min(B[b], Y[b] + U[b]);
      }
      acc = warp_sum_u64(acc + a1 + a2 + a3);
    }
    if (lane == 0) tot[c] = in_set ? ~uint64_t(0) : acc;
  }
  __shared__ bool s_last;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(&g->arrived, 1u) == unsigned(cpf) - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // --- argmin over (total, candidate): per thread, per warp, then all ---
  __shared__ double s_t[8];
  __shared__ int s_c[8];
  double bt = DBL_MAX;
  int bc = -1;
  for (int k = tid; k < ncand; k += blockDim.x) {
    const uint64_t u = __ldcg(&tot[k]);
    if (u == ~uint64_t(0)) continue;  // in the set
    const double t = u < kExact ? double(u)
                                 : ordered_total(d.best, YL, UL, d.sse + int64_t(k / d.nuv) * nfb,
                                                 d.sse + int64_t(d.ny + k % d.nuv) * nfb, nfb);
    argmin_pair(bt, bc, t, k);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const double t2 = __shfl_xor_sync(0xffffffffu, bt, o);
    const int c2 = __shfl_xor_sync(0xffffffffu, bc, o);
    argmin_pair(bt, bc, t2, c2);
  }
  if (lane == 0) {
    s_t[warp] = bt;
    s_c[warp] = bc;
  }
  __syncthreads();
  if (tid != 0) return;
  bt = s_t[0];
  bc = s_c[0];
  for (int w = 1; w < 8; w++) argmin_pair(bt, bc, s_t[w], s_c[w]);
  g->set_y[n] = bc / d.nuv;
  g->set_uv[n] = bc % d.nuv;
  g->n = n + 1;
  g->arrived = 0;
  const int size = n + 1;
  if ((size & (size - 1)) != 0) return;  // not a power of two: the level is not complete
  const int bits = __ffs(size) - 1;
  const double pen = __dmul_rn(__dmul_rn(lambda, double(bits)), double(g->nb));
  const double cost = __dadd_rn(bt, pen);
  const double prev = bits == 0 ? DBL_MAX : g->best_cost;
  if (cost < prev) {
    g->best_cost = cost;
    g->best_bits = bits;
  } else if (bits == 0) {
    g->best_cost = DBL_MAX;
  }
}

// The outcome (encoder/cdef.rs:241-250): each coding block's index is the
// first of the chosen 1 << best_bits pairs with its least error; the other
// table entries are copied.
__global__ void cdef_greedy_finish_kernel(const CdefSearchDesc* __restrict__ ds, int n, int total) {
  const int eg = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_wait();
  if (eg >= total) return;
  int fi = 0;
  for (int hi = n - 1; fi < hi;) {  // the last frame whose table starts at or before eg
    const int mid = (fi + hi + 1) >> 1;
    if (ds[mid].table0 <= eg)
      fi = mid;
    else
      hi = mid - 1;
  }
  const CdefSearchDesc& d = ds[fi];
  const CdefGreedy* g = d.g;
  const int nfb = d.fb_rows * d.fb_cols, stride = d.cdef_stride;
  const int m = 1 << g->best_bits;
  const int e = eg - d.table0;
  if (e == 0) {
    d.res[0] = int32_t(g->nb);
    d.res[1] = g->best_bits;
    for (int i = 0; i < 8; i++) {
      d.res[2 + i] = i < m ? g->set_y[i] : 0;
      d.res[10 + i] = i < m ? g->set_uv[i] : 0;
    }
  }
  const int r = e / stride, c = e - r * stride;
  int8_t v = d.cdef_idx[e];
  if (c < d.fb_cols && v >= 0) {
    const int b = r * d.fb_cols + c;
    uint64_t best = ~uint64_t(0);
    int pick = 0;
    for (int i = 0; i < m; i++) {
      const uint64_t x = d.sse[int64_t(g->set_y[i]) * nfb + b] + d.sse[int64_t(d.ny + g->set_uv[i]) * nfb + b];
      if (x < best) {
        best = x;
        pick = i;
      }
    }
    v = int8_t(pick);
  }
  d.table[e] = v;
}

// Squared error of one plane pair over rows [4*blockIdx.x, +4) of job
// blockIdx.y: 16-byte loads (planes and rows are 16-byte aligned), the
// ragged end of a row sample by sample.
__global__ void __launch_bounds__(256) plane_sse_kernel(const SsePlane* __restrict__ jobs, uint64_t* __restrict__ sse) {
  const SsePlane j = jobs[blockIdx.y];
  const int sb = j.sb;
  const int y0 = blockIdx.x * 4;
  uint64_t acc = 0;
  if (y0 < j.h) {
    const int per = 16 / sb;  // samples per 16 bytes
    const int nv = j.w / per;
    const int rows = min(4, j.h - y0);
    for (int k = threadIdx.x; k < rows * nv; k += blockDim.x) {
      const int r = y0 + k / nv, v = k % nv;
      const uint4 qa = *reinterpret_cast<const uint4*>(j.a + (int64_t(r) * j.sa + int64_t(v) * per) * sb);
      const uint4 qb = *reinterpret_cast<const uint4*>(j.b + (int64_t(r) * j.sb_ + int64_t(v) * per) * sb);
      const uint32_t wa[4] = {qa.x, qa.y, qa.z, qa.w}, wb[4] = {qb.x, qb.y, qb.z, qb.w};
      uint32_t s = 0;  // 8 squares below 4096^2, or 16 below 256^2: fits
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (sb == 2) {
          const int d0 = int(wa[q] & 0xffffu) - int(wb[q] & 0xffffu), d1 = int(wa[q] >> 16) - int(wb[q] >> 16);
          s += uint32_t(d0 * d0) + uint32_t(d1 * d1);
        } else {
#pragma unroll
          for (int h = 0; h < 4; h++) {
            const int dd = int((wa[q] >> (8 * h)) & 0xffu) - int((wb[q] >> (8 * h)) & 0xffu);
            s += uint32_t(dd * dd);
          }
        }
      }
      acc += s;
    }
    const int tail = j.w - nv * per;
    for (int k = threadIdx.x; k < rows * tail; k += blockDim.x) {
      const int r = y0 + k / tail, x = nv * per + k % tail;
      int dd;
      if (sb == 2)
        dd = int(reinterpret_cast<const uint16_t*>(j.a)[int64_t(r) * j.sa + x]) -
             int(reinterpret_cast<const uint16_t*>(j.b)[int64_t(r) * j.sb_ + x]);
      else
        dd = int(j.a[int64_t(r) * j.sa + x]) - int(j.b[int64_t(r) * j.sb_ + x]);
      acc += uint64_t(dd * dd);
    }
  }
  __shared__ uint64_t s_sum[8];
  acc = warp_sum_u64(acc);
  if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < 8; w++) t += s_sum[w];
    if (t) atomicAdd(reinterpret_cast<unsigned long long*>(&sse[blockIdx.y]), static_cast<unsigned long long>(t));
  }
}

}  // namespace

void launch_cdef_greedy_step(const CdefSearchDesc* ds, int n, int ncand, cudaStream_t s) {
  const int cpf = (ncand + 7) / 8;
  launch_pdl(cdef_greedy_step_kernel, n * cpf, 256, 0, s, ds, cpf);
}

void launch_cdef_greedy_finish(const CdefSearchDesc* ds, int n, int total, cudaStream_t s) {
  launch_pdl(cdef_greedy_finish_kernel, (total + 255) / 256, 256, 0, s, ds, n, total);
}

void launch_plane_sse(const SsePlane* jobs, int n, int rows_max, uint64_t* sse, cudaStream_t s) {
  if (n <= 0 || rows_max <= 0) return;
  plane_sse_kernel<<<dim3(unsigned((rows_max + 3) / 4), unsigned(n)), 256, 0, s>>>(jobs, sse);
  note_launch();
}

}  // namespace av1pf
