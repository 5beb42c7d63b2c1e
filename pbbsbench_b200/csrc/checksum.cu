// checksum.cu -- order-free 64-bit checksums of BFS level arrays, so that
// results can be compared without moving them (every served query's levels
// are checked against an independent search through these).
//
// A row of n level bytes r[0..n) is read as ceil(n/8) little-endian 64-bit
// words w_j (bytes past n count as 0xFF, the "unreached" level); the checksum
// is  H = sum_j mix64(w_j + (j + 1) * 0x9E3779B97F4A7C15)  mod 2^64,  with
// mix64 the SplitMix64 output function.  The sum is order-free, so blocks
// accumulate it with 64-bit atomic adds.  uint32 level arrays (single-source
// output) are first mapped to bytes: l >= 255 (and unreached) -> 255.
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.cuh"

namespace pbg {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t word_term(uint64_t w, uint64_t j) {
  return mix64(w + (j + 1) * 0x9E3779B97F4A7C15ull);
}

__device__ __forceinline__ void add_warp(uint64_t* out, uint64_t s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(out), (unsigned long long)s);
}

// grid.y = row; each thread folds words j = tid, tid + stride, ...
__global__ void k_rows_u8(const uint8_t* __restrict__ lv, uint32_t n, uint64_t* __restrict__ out) {
  const uint64_t row = blockIdx.y;
  const uint8_t* r = lv + row * (uint64_t)n;
  const uint64_t words = ((uint64_t)n + 7) / 8;
  // whole words of an 8-byte aligned row are one 8-byte load each
  const bool aligned = (reinterpret_cast<uintptr_t>(r) & 7u) == 0;
  uint64_t s = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < words; j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t w = 0;
    if (aligned && j * 8 + 8 <= n) {
      w = __ldg(reinterpret_cast<const unsigned long long*>(r) + j);
    } else {
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const uint64_t i = j * 8 + b;
        const uint64_t byte = (i < n) ? r[i] : 0xFFu;
        w |= byte << (8 * b);
      }
    }
    s += word_term(w, j);
  }
  add_warp(out + row, s);
}

__global__ void k_row_u32(const uint32_t* __restrict__ lv, uint32_t n, uint64_t* __restrict__ out) {
  const uint64_t words = ((uint64_t)n + 7) / 8;
  uint64_t s = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < words; j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t w = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const uint64_t i = j * 8 + b;
      uint64_t byte = 0xFFu;
      if (i < n) {
        const uint32_t l = lv[i];
        byte = (l >= 255u) ? 0xFFu : l;
      }
      w |= byte << (8 * b);
    }
    s += word_term(w, j);
  }
  add_warp(out, s);
}

unsigned blocks_for(uint32_t n) {
  const uint64_t words = ((uint64_t)n + 7) / 8;
  uint64_t b = (words + 255) / 256;
  if (b > 1024) b = 1024;
  return (unsigned)(b ? b : 1);
}

}  // namespace

int checksum_rows_u8(const uint8_t* d_levels, uint32_t rows, uint32_t n, uint64_t* d_out, cudaStream_t s) {
  PBG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint64_t) * rows, s));
  if (rows == 0) return PBG_OK;
  k_rows_u8<<<dim3(blocks_for(n), rows), 256, 0, s>>>(d_levels, n, d_out);
  PBG_CUDA(cudaGetLastError());
  return PBG_OK;
}

}  // namespace pbg

using namespace pbg;

extern "C" int pbg_levels_checksum(const uint8_t* d_levels, uint32_t rows, uint32_t n, uint64_t* d_out,
                                   void* stream) {
  if ((!d_levels && rows) || !d_out) return fail(PBG_ERR_ARG, "NULL argument");
  if (rows > 65535) return fail(PBG_ERR_ARG, "at most 65535 rows per call");
  return checksum_rows_u8(d_levels, rows, n, d_out, static_cast<cudaStream_t>(stream));
}

extern "C" int pbg_levels32_checksum(const uint32_t* d_levels, uint32_t n, uint64_t* d_out, void* stream) {
  if (!d_levels || !d_out) return fail(PBG_ERR_ARG, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PBG_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint64_t), s));
  k_row_u32<<<blocks_for(n), 256, 0, s>>>(d_levels, n, d_out);
  PBG_CUDA(cudaGetLastError());
  return PBG_OK;
}
