// device_util.cuh -- device helpers shared by the BFS kernels: timers,
// acquire/relaxed loads, a bounded grid-wide barrier for cooperative
// launches, and block reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pbg {
namespace dev {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;  // 2 s per wait

// Barrier state of one cooperative launch (zeroed before the launch).
struct GridSync {
  unsigned long long arrived;  // monotonic count of block arrivals
  unsigned int error;
  unsigned int pad;
  unsigned long long line_pad[14];
  unsigned long long work;  // monotonic work-batch counter (own 128-byte line)
  unsigned long long work_pad[15];
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier on a monotonic arrival counter.  Thread 0 of each block
// arrives with one acquire-release atomic increment and, unless it was the
// last to arrive, waits with acquire loads until the counter reaches
// epoch * gridDim.x: one round trip to arrive, one to see the last arrival,
// no reset.  The acquire also makes the block's later plain loads see every
// block's writes from before the barrier.  `epoch` is thread 0's count of
// barriers passed (every block passes the same sequence).  The wait is bounded
// by BARRIER_TIMEOUT_NS of %globaltimer: on expiry it sets `timeout_bit` in the
// error word and returns false; it also returns false once another block has
// reported an error.
__device__ __forceinline__ bool grid_barrier(GridSync* s, unsigned timeout_bit, unsigned long long& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long target = (++epoch) * gridDim.x;
    unsigned long long old;
    asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;" : "=l"(old) : "l"(&s->arrived) : "memory");
    if (old + 1 < target) {
      const unsigned long long t0 = globaltimer();
      unsigned spins = 0;
      while (ld_acquire_u64(&s->arrived) < target) {
        if (++spins > 64) __nanosleep(32);
        if ((spins & 255) == 0) {
          if (ld_acquire_u32(&s->error) != 0) {
            ok = 0;
            break;
          }
          if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
            atomicOr(&s->error, timeout_bit);
            ok = 0;
            break;
          }
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum over the block; the result is valid in thread 0.  All threads call it.
__device__ __forceinline__ unsigned long long block_sum(unsigned long long x) {
  __shared__ unsigned long long s_part[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
  __syncthreads();
  if (lane == 0) s_part[wid] = x;
  __syncthreads();
  unsigned long long r = 0;
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    r = (lane < nw) ? s_part[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(FULL, r, o);
  }
  return r;
}

}  // namespace dev
}  // namespace pbg
