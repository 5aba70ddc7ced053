// kernels.h — host-side launchers of the stage kernels (internal interface
// between the C ABI implementation and the .cu files).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "av1pf.h"

namespace av1pf {

struct FrameDesc;
struct Item;
struct CdefSearchDesc;
struct CdefGreedy;
struct LrSearchDesc;

// Grid cap of the grid-stride stage kernels: 8 resident CTAs on each of the
// B200's 148 SMs.
constexpr int kNumSMs = 148;
constexpr int kMaxGrid = kNumSMs * 8;
// Grid cap of the item kernels, which launch one CTA per item: the block
// scheduler then hands items of uneven cost to SMs as slots free up.
constexpr int kItemGrid = 1 << 20;

// Counts every kernel launch this library issues (av1pf_launch_count).
void note_launch(uint64_t n = 1);

// Launches a stage kernel with programmatic stream serialization: it may be
// scheduled while the previous kernel on `s` drains (the kernel waits for
// it in pdl_wait() before reading its output). Counts the launch.
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid));
  cfg.blockDim = dim3(unsigned(block));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  note_launch();
}

// Loop filter (lf.cu)
void launch_lf_prep(const FrameDesc* frames, const Item* items, int n_items, uint64_t* list_v, uint64_t* list_h,
                    uint32_t* counts, uint32_t cap, cudaStream_t s);
// Vertical edges filtered per 64x64 tile in shared memory (copy in -> cur
// included); horizontal decisions appended to list_h when item kind bit 2.
void launch_lf_tiles(const FrameDesc* frames, const Item* items, int n_items, uint64_t* list_h, uint32_t* counts,
                     uint32_t cap, cudaStream_t s);
// Both directions per 64x64 tile in shared memory (copy in -> cur included).
// `flags`: the readiness flags the kernel sets (see FrameDesc), or null.
void launch_lf_fused(const FrameDesc* frames, const Item* items, int n_items, uint32_t* flags, cudaStream_t s);
void launch_lf_edges(int pass, const FrameDesc* frames, const uint64_t* list, const uint32_t* count, uint32_t cap,
                     cudaStream_t s);
void launch_dsp_lf(int32_t* edges, const av1pf_lf_edge_params* prm, int n, cudaStream_t s);

// CDEF (cdef.cu)
// `lfh`: some item has the horizontal loop-filter pass fused (item kind 1).
// `half`: the items are half superblocks (Item::a = 0 top, 1 bottom).
// `flags`: the readiness flags the kernel waits for and sets, or null.
void launch_cdef(const FrameDesc* frames, const Item* items, int n_items, bool lfh, bool half, uint32_t* flags,
                 cudaStream_t s);
// Sets cdef_kernel's dynamic shared-memory limit on the current device.
cudaError_t cdef_init();
void launch_dsp_cdef(const int32_t* win, const av1pf_cdef_taps* taps, uint16_t* res, int n, cudaStream_t s);
// The encoder's CDEF search: per-block squared errors of every candidate
// (one CTA per 64x64 block of n frames, `blocks` in all); counts each
// frame's coding blocks into its greedy state.
void launch_cdef_search(const CdefSearchDesc* ds, int n, int blocks, bool thorough, cudaStream_t s);

// Encoder searches (search.cu)
// One greedy step of the CDEF search for n frames side by side: every pair
// not yet chosen is scored and the best is added (the last CTA of a frame
// to finish picks).
void launch_cdef_greedy_step(const CdefSearchDesc* ds, int n, int ncand, cudaStream_t s);
// The CDEF search's outcome: each coding block's index into each frame's
// table (a copy of its cdef_idx) and the chosen pairs into its result
// (`total` table entries over all frames).
void launch_cdef_greedy_finish(const CdefSearchDesc* ds, int n, int total, cudaStream_t s);
// Squared error of planes against the source over each plane's frame area:
// sse[i] += sum over plane job i (a, b: plane pointers and strides; `jobs`
// in device memory, at most 65535).
struct SsePlane {
  const uint8_t* a;
  const uint8_t* b;
  int64_t sa, sb_;  // strides in samples
  int32_t w, h;
  int32_t sb;       // bytes per sample
};
// The loop-restoration search (lr_search.cu): per unit job, the no-filter
// error and the Wiener passes on `s` (the first pass in a kernel of its own
// for jobs of several rectangles), the self-guided fits (one CTA per job
// and set) on `side` beside them, then the choice. Shared memory per kind:
// 0 the first-pass kernel, 1 the Wiener kernel, 2 the self-guided kernel.
size_t lr_search_smem(int wmax, int hmax, int kind, int band, int cache_px, int both);
// The self-guided band height and filter-output cache that fit shared memory.
void lr_search_shape(int wmax, int hmax, int upx_max, int& band, int& cache_px, int& both);
// Raises the kernels' dynamic shared-memory limits to the device's maximum
// (the same value on every call) on the current device.
cudaError_t lr_search_init();
void launch_lr_search(const LrSearchDesc& d, int njobs, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                      cudaEvent_t join);
void launch_plane_sse(const SsePlane* jobs, int n, int rows_max, uint64_t* sse, cudaStream_t s);

// Super-resolution (superres.cu)
// `row_max`: the most source samples in a row among the launch's frames.
void launch_superres(const FrameDesc* frames, const Item* items, int n_items, int row_max, cudaStream_t s);
// Sets superres_kernel's dynamic shared-memory limit on the current device.
cudaError_t superres_init();

// Loop restoration (lr.cu)
// `flags`: the readiness flags the kernel waits for, or null.
void launch_lr(const FrameDesc* frames, const Item* items, int n_items, uint32_t* flags, cudaStream_t s);
// Sets lr_kernel's dynamic shared-memory limit on the current device.
cudaError_t lr_init();
// Opts the output kernel into its dynamic shared memory (once per device).
cudaError_t output_init();

// Film grain + output packing (grain.cu)
void launch_grain_prep(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s);
void launch_output(const FrameDesc* frames, const Item* items, int n_items, cudaStream_t s);
// Uploads the LFSR jump-ahead tables (once per device).
cudaError_t upload_grain_tables();

// Device error flags (g_error_flags): read and clear. This bit of them
// means a kernel's bounded wait gave up (ERRF_STALL in common.cuh).
constexpr uint32_t kErrfStall = 4u;
cudaError_t read_error_flags(uint32_t* flags, cudaStream_t s);

}  // namespace av1pf
