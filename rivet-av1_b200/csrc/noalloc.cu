// noalloc.cu — av1pf_output_noalloc: the output stage (film grain + crop +
// packing into the Frame layout) for callers that cannot allocate device
// memory.
//
// Who needs it: a decoder embedded in a host whose device memory is owned
// by another allocator (a framework's caching allocator, a fixed per-process
// budget carved out up front), or a real-time output path that cannot take
// an allocation's latency or an out-of-memory failure in the middle of a
// stream. Such callers cannot let the library call cudaMalloc, and they may
// not hold an av1pf_ctx (whose scratch is allocated on demand).
//
// What it does instead: the scratch the grain-template and output kernels
// need — the frame descriptor, the work list, the three grain templates and
// scaling tables, and the per-stripe block offsets — lives in one file-scope
// device array of kNoAllocBytes, reserved when the library is loaded and
// kept by every GPU that loads it until the process exits. The kernels are
// the ones av1pf_output launches; only where their scratch lives differs.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "ctx.h"
#include "kernels.h"
#include "plan.h"

namespace av1pf {

namespace {

// Layout of the static scratch: [descriptor][work list][grain templates][block offsets].
constexpr size_t kDescBytes = 4096;
constexpr size_t kMaxItems = 9728;
constexpr size_t kItemsBytes = kMaxItems * sizeof(Item);
constexpr size_t kGrainBytes = (sizeof(GrainScratch) + 255) / 256 * 256;
constexpr size_t kMaxOffsets = 65536;  // ceil(h/32) * ceil(w/32) blocks: up to 8192 x 8192
constexpr size_t kNoAllocBytes = kDescBytes + kItemsBytes + kGrainBytes + kMaxOffsets;
static_assert(sizeof(FrameDesc) <= kDescBytes, "descriptor slot too small");

// The scratch itself. In host code `g_noalloc_scratch` only names the
// symbol; its device address comes from cudaGetSymbolAddress (see setup).
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

std::mutex g_setup_mu;
uint8_t* g_scratch_ptr[64] = {};     // per device: address of g_noalloc_scratch
unsigned long long g_ctx_id[64] = {};  // per device: the context the address and tables belong to

// The unique ID of the calling thread's current CUDA context (cuCtxGetId,
// reached through the runtime's driver entry points, so the library needs
// no link against the driver library); false if unavailable.
bool current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  CUcontext c = nullptr;
  return get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, id) == CUDA_SUCCESS;
}

// With the device current: look up the scratch's device address, upload
// the film-grain RNG jump tables and give the output kernel its shared
// memory, once per device context. After a cudaDeviceReset the device's
// next context loads the module again (the array at a possibly new address,
// the tables zeroed, the kernel attribute unset): that context has a new ID,
// so the lookup, upload and attribute run again.
int setup(int device, uint8_t** out) {
  if (device < 0 || device >= 64) {
    set_error("av1pf_output_noalloc: device index out of range");
    return AV1PF_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_setup_mu);
  void* p = nullptr;
  // (also makes the device's context current in this thread)
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_status(e, "av1pf_output_noalloc: cudaGetSymbolAddress");
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  if (g_scratch_ptr[device] != p || (have_id && g_ctx_id[device] != id)) {
    e = upload_grain_tables();
    if (e != cudaSuccess) return cuda_status(e, "av1pf_output_noalloc: grain tables");
    e = output_init();
    if (e != cudaSuccess) return cuda_status(e, "av1pf_output_noalloc: output kernel attributes");
    g_scratch_ptr[device] = static_cast<uint8_t*>(p);
    g_ctx_id[device] = have_id ? id : 0;
  }
  *out = g_scratch_ptr[device];
  return AV1PF_OK;
}

// Host staging of the descriptor and work list (reused call after call: the
// pageable copy below has read it before cudaMemcpyAsync returns).
struct Staging {
  uint8_t bytes[kDescBytes + kItemsBytes];
};
Staging g_staging;
std::mutex g_staging_mu;

}  // namespace

}  // namespace av1pf

using namespace av1pf;

extern "C" int av1pf_output_noalloc(const av1pf_frame_info* info, const av1pf_params* params,
                                    const av1pf_plane* ref, uint8_t* frame_out, void* stream) {
  int rc = validate_frame(info, params, nullptr, nullptr);
  if (rc != AV1PF_OK) {
    set_error("av1pf_output_noalloc: invalid frame info or parameters");
    return rc;
  }
  if (!params || !ref || !frame_out) {
    set_error("av1pf_output_noalloc: null params, planes or output");
    return AV1PF_ERR_INVALID_INPUT;
  }
  const bool grain = params->film_grain.apply != 0;
  const int ns = ((info->frame_height + 1) / 2 + 15) / 16;
  const int nb = ((info->upscaled_width + 1) / 2 + 15) / 16;
  if (grain && size_t(ns) * size_t(nb) > kMaxOffsets) {
    set_error("av1pf_output_noalloc: frame too large for the fixed scratch (film grain needs "
              "ceil(h/32)*ceil(w/32) <= 65536, e.g. at most 8192x8192)");
    return AV1PF_ERR_UNSUPPORTED;
  }
  const int np = info->num_planes;
  for (int k = 0; k < np; k++) {
    if (!ref[k].data || ref[k].width < plane_w(info, k, info->upscaled_width) || ref[k].height < plane_h(info, k) ||
        ref[k].stride < ref[k].width) {
      set_error("av1pf_output_noalloc: reference plane smaller than the visible area");
      return AV1PF_ERR_INVALID_INPUT;
    }
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_status(e, "av1pf_output_noalloc: cudaGetDevice");
  uint8_t* scratch = nullptr;
  if ((rc = setup(device, &scratch)) != AV1PF_OK) return rc;
  uint8_t* d_desc = scratch;
  uint8_t* d_items = scratch + kDescBytes;
  GrainScratch* d_grain = reinterpret_cast<GrainScratch*>(scratch + kDescBytes + kItemsBytes);
  uint8_t* d_off = scratch + kDescBytes + kItemsBytes + kGrainBytes;

  std::lock_guard<std::mutex> lk(g_staging_mu);
  FrameDesc& d = *reinterpret_cast<FrameDesc*>(g_staging.bytes);
  std::memset(&d, 0, sizeof(d));
  d.bd = info->bit_depth;
  d.sb = info->sample_bytes;
  d.ssx = info->subsampling_x;
  d.ssy = info->subsampling_y;
  d.np = np;
  d.fw = info->frame_width;
  d.fh = info->frame_height;
  d.uw = info->upscaled_width;
  d.mi_rows = info->mi_rows;
  d.mi_cols = info->mi_cols;
  d.mc = info->matrix_coefficients;
  d.frame_out = frame_out;
  d.g = params->film_grain;
  if (grain) {
    d.grain_on = 1;
    d.grain = d_grain;
    d.grain_off = d_off;
    d.grain_ns = ns;
    d.grain_nb = nb;
  }
  const int64_t bps = info->bit_depth > 8 ? 2 : 1;
  int64_t off = 0;
  int pw[3], ph[3];
  for (int k = 0; k < np; k++) {
    d.ref[k] = DPlane{static_cast<uint8_t*>(ref[k].data), ref[k].stride, ref[k].width, ref[k].height};
    d.out_off[k] = off;
    pw[k] = plane_w(info, k, info->upscaled_width);
    ph[k] = plane_h(info, k);
    off += int64_t(pw[k]) * ph[k] * bps;
  }
  // Work list: 256-column tiles (the kernel wants x0 a multiple of 256), as
  // tall as needed to fit the fixed list.
  Item* items = reinterpret_cast<Item*>(g_staging.bytes + kDescBytes);
  int th = 32;
  auto count = [&](int t) {
    size_t n = 0;
    for (int k = 0; k < np; k++) n += size_t((pw[k] + 255) / 256) * size_t((ph[k] + t - 1) / t);
    return n;
  };
  while (count(th) + 1 > kMaxItems) th *= 2;
  int n = 0;
  if (grain) {
    Item g{};
    items[n++] = g;  // one grain-template item (frame 0)
  }
  const int first_out = n;
  for (int k = 0; k < np; k++)
    for (int y = 0; y < ph[k]; y += th)
      for (int x = 0; x < pw[k]; x += 256) {
        Item it{};
        it.plane = uint8_t(k);
        it.x0 = uint16_t(x);
        it.y0 = uint16_t(y);
        it.x1 = uint16_t(x + 256 < pw[k] ? x + 256 : pw[k]);
        it.y1 = uint16_t(y + th < ph[k] ? y + th : ph[k]);
        items[n++] = it;
      }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemcpyAsync(d_desc, g_staging.bytes, kDescBytes + size_t(n) * sizeof(Item), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_status(e, "av1pf_output_noalloc: descriptor upload");
  const FrameDesc* frames = reinterpret_cast<const FrameDesc*>(d_desc);
  const Item* d_list = reinterpret_cast<const Item*>(d_items);
  if (grain) launch_grain_prep(frames, d_list, 1, s);
  launch_output(frames, d_list + first_out, n - first_out, s);
  return cuda_status(cudaGetLastError(), "av1pf_output_noalloc: launch");
}
