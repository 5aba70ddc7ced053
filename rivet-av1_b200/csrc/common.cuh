// common.cuh — shared device definitions of the post-filter kernels:
// the per-frame descriptor the kernels read, the work-item format, the
// specification tables in constant memory, and integer helpers.
//
// Every stage kernel takes (frames[], items[], n_items) and loops over items
// with a grid stride, so one launch serves one frame or a whole batch of
// frames of different shape, bit depth and subsampling.
#pragma once

#include <cstdint>

#include "av1pf.h"
#include "av1_tables.h"
#include "desc.h"

namespace av1pf {

// ---------------------------------------------------------------------------
// Tables (av1_tables.h is extracted from the specification data of the
// reference's src/tables.rs).
// ---------------------------------------------------------------------------
extern __constant__ int8_t c_cdef_dirs[8][2][2];
extern __constant__ uint8_t c_cdef_uv_dir[2][2][8];
extern __constant__ int32_t c_div_table[9];
extern __constant__ uint8_t c_subsampled_size[22][2][2];
extern __constant__ uint8_t c_tx_w[19];
extern __constant__ uint8_t c_tx_h[19];
extern __constant__ uint8_t c_n4w[22];
extern __constant__ uint8_t c_n4h[22];
extern __constant__ int32_t c_sgr_params[16][4];
extern __device__ const int16_t g_upscale_filter[64][8];  // 16-byte aligned rows
extern __device__ int16_t g_gaussian[2048];
// LFSR jump-ahead (7.18.3.2): column b of M^(82r) / M^(44r) is the state
// reached from state 1<<b after 82r / 44r steps.
extern __device__ uint16_t g_rng_jump82[73][16];
extern __device__ uint16_t g_rng_jump44[73][16];
// Sticky device-side error bits (bad map values met by a kernel).
extern __device__ uint32_t g_error_flags;
// ERRF_STALL (kErrfStall on the host): a bounded wait inside a kernel gave
// up, so its result is not valid.
enum : uint32_t { ERRF_BAD_MAP = 1u, ERRF_BAD_ITEM = 2u, ERRF_STALL = 4u };

// ---------------------------------------------------------------------------
// One-dimensional bulk copies (TMA) into this CTA's shared memory, completing
// on an mbarrier. Source and destination 16-byte aligned, size a multiple of
// 16. No multicast.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  // the initialisation is visible to the bulk copies' completions
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival that also expects `bytes` of copies on the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Waits for the phase of parity `phase` to complete: each try suspends the
// thread for up to about a microsecond; after `limit` tries the wait gives up
// and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int limit) {
  for (int k = 0; k < limit; k++) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase), "r"(1000u)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Integer helpers (consts.rs:328-368, bits.rs:112)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t round2(int32_t x, int n) {  // 0 <= n <= 30
  return (x + ((1 << n) >> 1)) >> n;
}
__device__ __forceinline__ int64_t round2_64(int64_t x, int n) {
  return n == 0 ? x : (x + (int64_t(1) << (n - 1))) >> n;
}
__device__ __forceinline__ int32_t clip3(int32_t lo, int32_t hi, int32_t x) {
  return max(lo, min(hi, x));
}
__device__ __forceinline__ int32_t floor_log2(uint32_t x) { return 31 - __clz(x); }

// Sample access with the frame's storage width.
__device__ __forceinline__ int32_t ld_sample(const DPlane& p, int sb, int x, int y) {
  const uint8_t* row = p.p + (int64_t(y) * p.stride) * sb;
  return sb == 1 ? int32_t(row[x]) : int32_t(reinterpret_cast<const uint16_t*>(row)[x]);
}
__device__ __forceinline__ void st_sample(const DPlane& p, int sb, int x, int y, int32_t v) {
  uint8_t* row = p.p + (int64_t(y) * p.stride) * sb;
  if (sb == 1)
    row[x] = uint8_t(v);
  else
    reinterpret_cast<uint16_t*>(row)[x] = uint16_t(v);
}

// Plane dimensions helpers.
__device__ __forceinline__ int plane_ssx(const FrameDesc& f, int plane) { return plane ? f.ssx : 0; }
__device__ __forceinline__ int plane_ssy(const FrameDesc& f, int plane) { return plane ? f.ssy : 0; }

// Programmatic dependent launch (sm_90 and later). The stage kernels are
// launched with programmatic stream serialization (launch_pdl): a kernel may
// be scheduled while its predecessor on the stream drains, so every stage
// kernel starts with pdl_wait(), which returns once the predecessor has
// completed and its writes are visible, and then lets its own successor
// start launching.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// For the stages that wait on readiness flags (FrameDesc::lf_flag_base ...)
// instead of pdl_wait: such a kernel lets its successor launch at once (all
// of its own CTAs have then started, so none waits for a place on an SM
// that a CTA of the successor holds) and waits per item for the flags of
// the data it reads. The chain's last stage (loop restoration) waits for
// flags that every CDEF item sets after its last read of the loop filter's
// output, so when that stage's grid is complete no kernel of the chain
// reads or writes the chain's buffers any more.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Per-CTA timeline, in the AV1PF_TRACE build only (libav1pf_trace.so, read
// by timeline.py): each stage kernel's CTAs record their start and end
// (%globaltimer, ns), their SM and block, and the kernel's id into g_trace.
// In the product build the two macros are empty.
#ifdef AV1PF_TRACE
constexpr int kTraceCap = 65536;
extern __device__ unsigned long long g_trace[3 * kTraceCap];
extern __device__ unsigned int g_trace_n;
__device__ __forceinline__ unsigned long long trace_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void trace_end(int kid, unsigned long long t0) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned sm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
    const unsigned i = atomicAdd(&g_trace_n, 1u);
    if (i < unsigned(kTraceCap)) {
      g_trace[3 * i] = t0;
      g_trace[3 * i + 1] = trace_clock();
      g_trace[3 * i + 2] = (static_cast<unsigned long long>(kid) << 40) | (static_cast<unsigned long long>(sm) << 24) |
                           blockIdx.x;
    }
  }
}
#define AV1PF_TRACE_BEGIN() const unsigned long long av1pf_trace_t0 = ::av1pf::trace_clock()
#define AV1PF_TRACE_END(kid) ::av1pf::trace_end((kid), av1pf_trace_t0)
#else
#define AV1PF_TRACE_BEGIN() \
  do {                      \
  } while (0)
#define AV1PF_TRACE_END(kid) \
  do {                       \
  } while (0)
#endif

// A readiness flag: set with release semantics at GPU scope after the CTA's
// barrier (so every thread's writes before the barrier are visible to a
// thread that sees the flag), waited for with acquire semantics. The wait is
// bounded: after kFlagSpins polls it flags ERRF_STALL and returns.
constexpr int kFlagSpins = 1 << 21;
__device__ __forceinline__ void flag_set(uint32_t* p) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(1u) : "memory");
}
__device__ __forceinline__ void flag_wait(const uint32_t* p) {
  for (int k = 0; k < kFlagSpins; k++) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    if (v) return;
    __nanosleep(100);
  }
  atomicOr(&g_error_flags, ERRF_STALL);
}

// Grid-stride loop over the items of a launch.
#define FOR_EACH_ITEM(it, n)                                   \
  for (int it = blockIdx.x; it < (n); it += gridDim.x)

}  // namespace av1pf
