// tables.cu — the specification tables in device memory. Small tables read
// with warp-uniform indices live in constant memory; tables indexed per
// thread (upscale phases, Gaussian sequence) live in global memory.
#include "common.cuh"
#include "kernels.h"

namespace av1pf {

__constant__ int8_t c_cdef_dirs[8][2][2] = AV1T_CDEF_DIRECTIONS;
__constant__ uint8_t c_cdef_uv_dir[2][2][8] = AV1T_CDEF_UV_DIR;
__constant__ int32_t c_div_table[9] = AV1T_DIV_TABLE;
__constant__ uint8_t c_subsampled_size[22][2][2] = AV1T_SUBSAMPLED_SIZE;
__constant__ uint8_t c_tx_w[19] = AV1T_TX_WIDTH;
__constant__ uint8_t c_tx_h[19] = AV1T_TX_HEIGHT;
__constant__ uint8_t c_n4w[22] = AV1T_NUM_4X4_BLOCKS_WIDE;
__constant__ uint8_t c_n4h[22] = AV1T_NUM_4X4_BLOCKS_HIGH;
__constant__ int32_t c_sgr_params[16][4] = AV1T_SGR_PARAMS;
__device__ __align__(16) const int16_t g_upscale_filter[64][8] = AV1T_UPSCALE_FILTER;
__device__ int16_t g_gaussian[2048] = AV1T_GAUSSIAN_SEQUENCE;
__device__ uint16_t g_rng_jump82[73][16];
__device__ uint16_t g_rng_jump44[73][16];
__device__ uint32_t g_error_flags;

// LFSR of 7.18.3.2 as a GF(2) matrix: column b of M^n is the state reached
// from 1 << b after n steps; uploaded once per device.
cudaError_t upload_grain_tables() {
  auto step = [](uint32_t r) {
    const uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1u;
    return (r >> 1) | (bit << 15);
  };
  uint16_t j82[73][16], j44[73][16];
  for (int b = 0; b < 16; b++) {
    uint32_t s = 1u << b;
    for (int r = 0; r < 73; r++) {
      j82[r][b] = uint16_t(s);
      for (int k = 0; k < 82; k++) s = step(s);
    }
    s = 1u << b;
    for (int r = 0; r < 73; r++) {
      j44[r][b] = uint16_t(s);
      for (int k = 0; k < 44; k++) s = step(s);
    }
  }
  cudaError_t e = cudaMemcpyToSymbol(g_rng_jump82, j82, sizeof(j82));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(g_rng_jump44, j44, sizeof(j44));
}

cudaError_t read_error_flags(uint32_t* flags, cudaStream_t s) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(flags, g_error_flags, sizeof(uint32_t), 0, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  const uint32_t zero = 0;
  return cudaMemcpyToSymbol(g_error_flags, &zero, sizeof(zero));
}

}  // namespace av1pf

#ifdef AV1PF_TRACE
namespace av1pf {
__device__ unsigned long long g_trace[3 * kTraceCap];
__device__ unsigned int g_trace_n;
}  // namespace av1pf

// The trace build's read-out: copies the records (3 words each: start,
// end, kernel << 40 | SM << 24 | block) and their count, then clears the
// count. Returns a cudaError_t.
extern "C" int av1pf_trace_read(unsigned long long* out, unsigned* n) {
  cudaError_t e = cudaMemcpyFromSymbol(n, av1pf::g_trace_n, sizeof(unsigned));
  const unsigned m = *n < unsigned(av1pf::kTraceCap) ? *n : unsigned(av1pf::kTraceCap);
  if (e == cudaSuccess && m) e = cudaMemcpyFromSymbol(out, av1pf::g_trace, m * 3 * sizeof(unsigned long long));
  const unsigned z = 0;
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(av1pf::g_trace_n, &z, sizeof(unsigned));
  return int(e);
}
#endif
