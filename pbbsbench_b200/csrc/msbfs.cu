// msbfs.cu -- batched multi-source BFS: up to 64 sources per job, many jobs
// (graphs of any sizes) in ONE persistent cooperative launch.
//
// No reference counterpart: PBBS runs one source per BFS() call
// (benchmarks/breadthFirstSearch/bench/BFS.h:11).  The result of each source
// is the level array of that single-source search (uint8, 255 = unreached),
// bit-exact against independent runs of the sequential BFS
// (serialBFS/BFS.C:32-55).
//
// Per job, in HBM:
//   vis[n]  u64   bit i set = vertex reached by source i
//   fr0/fr1 u64   frontier masks of the current / next level (bits newly set)
//   q0/q1   u32   queue of vertices whose frontier mask is non-zero
//   qb0/qb1 uint4 same for vertices with degree >= big_min_degree, in
//                 CHUNK-edge pieces (v, begin, end, first chunk)
//   levels  u8    [k][n], source-major
//
// Each level every job independently runs
//   pull (bottom-up): every not-fully-reached v ORs its neighbours' frontier
//     masks, stopping once every missing source bit is found (the bit-parallel
//     form of edge_map_dense, common/ligraLight.h:87-112), or
//   push (top-down): every frontier vertex u ORs fr[u] & ~vis[v] into the next
//     mask of each neighbour v (atomicOr on u64); the first writer enqueues v
//     (edge_map_sparse, ligraLight.h:70-85); a second phase folds the new bits
//     into vis and writes the levels,
// chosen by the switch of ligraLight.h:114-136 on the job's own frontier
// size and out-degree.  Work of all jobs in a level is spread over all warps
// of the grid through a prefix sum of per-job tile counts, so graphs of uneven
// size share one launch.  Barriers are bounded (device_util.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "device_util.cuh"
#include "internal.cuh"
#include "msbfs.cuh"

namespace pbg {
namespace {

using dev::FULL;
constexpr uint32_t CHUNK = 1024;
constexpr unsigned long long BIG_SHIFT = 40;
constexpr unsigned long long BIG_MASK = (1ull << BIG_SHIFT) - 1;
enum : uint32_t { M_DONE = 0, M_PULL = 1, M_PUSH = 2 };

struct MsParams {
  uint32_t alpha, beta, policy, warp_deg, big_deg;
};

__device__ __forceinline__ void write_levels(uint8_t* levels, uint32_t n, uint32_t v, unsigned long long bits,
                                             uint8_t lv) {
  while (bits) {
    const int i = __ffsll((long long)bits) - 1;
    bits &= bits - 1;
    levels[(size_t)i * n + v] = lv;
  }
}

// Warp-collective append (as in bfs.cu); deg goes to a per-block shared
// accumulator of the job.
__device__ __forceinline__ void ms_emit(const MsJob& J, LevelSlot* out, uint32_t* qout, uint4* qbout, bool win,
                                        uint32_t v, uint32_t b, uint32_t e, unsigned long long cap,
                                        uint32_t big_deg, unsigned long long* s_deg) {
  const unsigned wm = __ballot_sync(FULL, win);
  if (wm == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t deg = e - b;
  const bool big = win && deg >= big_deg;
  unsigned long long d = win ? deg : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(FULL, d, o);
  if (lane == 0 && d) atomicAdd(s_deg, d);
  const unsigned mm = __ballot_sync(FULL, win && !big);
  if (mm) {
    const int leader = __ffs(mm) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&out->nmain, (unsigned long long)__popc(mm));
    base = __shfl_sync(FULL, base, leader);
    if (win && !big) {
      const unsigned long long pos = base + __popc(mm & ((1u << lane) - 1u));
      if (pos < cap) qout[pos] = v;
    }
  }
  if (big) {
    const uint32_t nch = (deg + CHUNK - 1) / CHUNK;
    const unsigned long long old = atomicAdd(&out->big, (1ull << BIG_SHIFT) | nch);
    const uint32_t slot = (uint32_t)(old >> BIG_SHIFT);
    if (slot < J.big_cap)
      qbout[slot] = make_uint4(v, b, e, (uint32_t)(old & BIG_MASK));
    else
      atomicOr(&J.ctrl->error, MS_ERR_QUEUE);
  }
}

// Push one edge per lane: u's mask into v's next mask.
__device__ __forceinline__ void push_edge(const MsJob& J, const unsigned long long* fcur, unsigned long long* fnext,
                                          LevelSlot* out, uint32_t* qout, uint4* qbout, bool act,
                                          unsigned long long f, uint32_t j, uint32_t big_deg,
                                          unsigned long long* s_deg) {
  bool touched = false;
  uint32_t v = 0, b = 0, e = 0;
  if (act) {
    v = __ldg(J.edges + j);
    const unsigned long long mb = f & ~J.vis[v];
    if (mb) {
      const unsigned long long old = atomicOr(fnext + v, mb);
      if (old == 0) {
        touched = true;
        b = __ldg(J.offsets + v);
        e = __ldg(J.offsets + v + 1);
      }
    }
  }
  ms_emit(J, out, qout, qbout, touched, v, b, e, ~0ull, big_deg, s_deg);
}

// Pull for 32 consecutive vertices, one per lane.  Each lane ORs its
// neighbours' frontier masks PULL_STEP at a time (independent loads), stopping
// once every source bit it still misses is found; lists still unresolved
// after the first step are then pulled by the whole warp, 32 neighbours a
// step, with a warp OR-reduction and the same early exit.
constexpr int PULL_STEP = 8;

__device__ __forceinline__ unsigned long long warp_or(unsigned long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(FULL, x, o);
  return x;
}

__device__ void pull_tile(const MsJob& J, uint32_t tile, const unsigned long long* fcur, unsigned long long* fnext,
                          LevelSlot* out, uint32_t* qout, uint4* qbout, uint8_t next_level, unsigned long long cap,
                          uint32_t big_deg, unsigned long long* s_deg) {
  const int lane = threadIdx.x & 31;
  const uint32_t v = tile * 32 + lane;
  const bool active = v < J.n;
  const unsigned long long all = J.all;
  unsigned long long vv = all;
  uint32_t b = 0, e = 0;
  if (active) {
    vv = J.vis[v];
    if (vv != all) {
      b = __ldg(J.offsets + v);
      e = __ldg(J.offsets + v + 1);
    }
  }
  unsigned long long acc = 0;
  {
    uint32_t u[PULL_STEP];
#pragma unroll
    for (int i = 0; i < PULL_STEP; i++) u[i] = (b + i < e) ? __ldg(J.edges + b + i) : 0xFFFFFFFFu;
    unsigned long long f[PULL_STEP];
#pragma unroll
    for (int i = 0; i < PULL_STEP; i++) f[i] = (u[i] != 0xFFFFFFFFu) ? fcur[u[i]] : 0ull;
#pragma unroll
    for (int i = 0; i < PULL_STEP; i++) acc |= f[i];
  }
  unsigned mm = __ballot_sync(FULL, e - b > PULL_STEP && (acc | vv) != all);
  while (mm) {
    const int l = __ffs(mm) - 1;
    mm &= mm - 1;
    const uint32_t bb = __shfl_sync(FULL, b, l), ee = __shfl_sync(FULL, e, l);
    const unsigned long long need = __shfl_sync(FULL, vv, l);
    unsigned long long got = __shfl_sync(FULL, acc, l);
    for (uint32_t j0 = bb + PULL_STEP; j0 < ee && (got | need) != all; j0 += 32) {
      const uint32_t j = j0 + lane;
      const unsigned long long f = (j < ee) ? fcur[__ldg(J.edges + j)] : 0ull;
      got |= warp_or(f);
    }
    if (lane == l) acc = got;
  }
  const unsigned long long nb = acc & ~vv;
  const bool found = active && nb != 0;
  if (found) {
    J.vis[v] = vv | nb;
    write_levels(J.levels, J.n, v, nb, next_level);
  }
  if (active) fnext[v] = found ? nb : 0ull;
  ms_emit(J, out, qout, qbout, found, v, b, e, cap, big_deg, s_deg);
}

__device__ void push_main_tile(const MsJob& J, uint32_t tile, unsigned long long nmain, const uint32_t* qin,
                               const unsigned long long* fcur, unsigned long long* fnext, LevelSlot* out,
                               uint32_t* qout, uint4* qbout, uint32_t warp_deg, uint32_t big_deg,
                               unsigned long long* s_deg) {
  const int lane = threadIdx.x & 31;
  const unsigned long long idx = (unsigned long long)tile * 32 + lane;
  const bool have = idx < nmain;
  uint32_t b = 0, e = 0;
  unsigned long long f = 0;
  if (have) {
    const uint32_t u = qin[idx];
    f = fcur[u];
    b = __ldg(J.offsets + u);
    e = __ldg(J.offsets + u + 1);
  }
  const uint32_t deg = e - b;
  const bool med = have && deg >= warp_deg;
  const uint32_t sdeg = (have && !med) ? deg : 0u;
  const uint32_t maxd = __reduce_max_sync(FULL, sdeg);
  for (uint32_t j = 0; j < maxd; j++)
    push_edge(J, fcur, fnext, out, qout, qbout, j < sdeg, f, b + j, big_deg, s_deg);
  unsigned mm = __ballot_sync(FULL, med);
  while (mm) {
    const int l = __ffs(mm) - 1;
    mm &= mm - 1;
    const unsigned long long ff = __shfl_sync(FULL, f, l);
    const uint32_t bb = __shfl_sync(FULL, b, l);
    const uint32_t ee = __shfl_sync(FULL, e, l);
    for (uint32_t j0 = bb; j0 < ee; j0 += 32)
      push_edge(J, fcur, fnext, out, qout, qbout, j0 + lane < ee, ff, j0 + lane, big_deg, s_deg);
  }
}

__device__ void push_chunk_tile(const MsJob& J, uint32_t c, const uint4* qbin, uint32_t nbig,
                                const unsigned long long* fcur, unsigned long long* fnext, LevelSlot* out,
                                uint32_t* qout, uint4* qbout, uint32_t big_deg, unsigned long long* s_deg) {
  const int lane = threadIdx.x & 31;
  uint32_t lo = 0, hi = nbig - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (qbin[mid].w <= c)
      lo = mid;
    else
      hi = mid - 1;
  }
  const uint4 ent = qbin[lo];
  const unsigned long long f = fcur[ent.x];
  const uint32_t cb = ent.y + (c - ent.w) * CHUNK;
  const uint32_t ce = min(ent.z, cb + CHUNK);
  for (uint32_t j0 = cb; j0 < ce; j0 += 32)
    push_edge(J, fcur, fnext, out, qout, qbout, j0 + lane < ce, f, j0 + lane, big_deg, s_deg);
}

// Direction for a job's next level from its frontier (same rule as bfs.cu).
__device__ __forceinline__ uint32_t decide(const MsJob& J, const MsParams& p, bool prev_pull,
                                           unsigned long long nf, unsigned long long fdeg) {
  if (nf == 0) return M_DONE;
  if (p.policy == PBG_DIR_TOPDOWN || !J.symmetric) return M_PUSH;
  if (p.policy == PBG_DIR_BOTTOMUP) return M_PULL;
  if (!prev_pull) return (nf + fdeg > J.m / p.alpha) ? M_PULL : M_PUSH;
  return (nf > (unsigned long long)(J.n / p.beta)) ? M_PULL : M_PUSH;
}

__global__ void __launch_bounds__(512) ms_persistent(const MsJob* __restrict__ jobs, uint32_t njobs, MsParams p,
                                                     dev::GridSync* sync) {
  __shared__ uint32_t s_mode[MS_MAX_JOBS];
  __shared__ uint8_t s_prev_pull[MS_MAX_JOBS];
  __shared__ uint8_t s_done[MS_MAX_JOBS];
  __shared__ unsigned long long s_tile_end[MS_MAX_JOBS];
  __shared__ unsigned long long s_nmain[MS_MAX_JOBS];
  __shared__ uint32_t s_nbig[MS_MAX_JOBS];
  __shared__ unsigned long long s_deg[MS_MAX_JOBS];
  __shared__ unsigned long long s_total;
  __shared__ int s_any_phase_b;

  unsigned long long bar_epoch = 0;  // barriers passed (thread 0's count matters)
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
  const uint32_t gwarp = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;  // round-robin over blocks first
  const uint32_t nwarps = (uint32_t)(nth >> 5);

  // ---- init: masks to zero, levels to 255.
  for (uint32_t j = 0; j < njobs; j++) {
    const MsJob& J = jobs[j];
    for (unsigned long long i = tid; i < J.n; i += nth) {
      J.vis[i] = 0;
      J.fr0[i] = 0;
      J.fr1[i] = 0;
    }
    const unsigned long long nb = (unsigned long long)J.k * J.n;
    uint4* lv4 = reinterpret_cast<uint4*>(J.levels);
    const uint4 ff = make_uint4(FULL, FULL, FULL, FULL);
    for (unsigned long long i = tid; i < nb / 16; i += nth) lv4[i] = ff;
    for (unsigned long long i = (nb / 16) * 16 + tid; i < nb; i += nth) J.levels[i] = 255;
  }
  if (!dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch)) return;
  // ---- sources: one thread per job.
  if (blockIdx.x == 0) {
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const MsJob& J = jobs[j];
      LevelSlot* s0 = &J.ctrl->slot[0];
      for (uint32_t i = 0; i < J.k; i++) {
        const uint32_t s = J.srcs[i];
        const unsigned long long bit = 1ull << i;
        const unsigned long long old = J.fr0[s];
        J.fr0[s] = old | bit;
        J.vis[s] |= bit;
        J.levels[(size_t)i * J.n + s] = 0;
        if (old == 0) {
          const uint32_t b = __ldg(J.offsets + s), e = __ldg(J.offsets + s + 1);
          if (e - b >= p.big_deg) {
            const unsigned long long nch = (e - b + CHUNK - 1) / CHUNK;
            const unsigned long long slot = s0->big >> BIG_SHIFT;
            J.qb0[slot] = make_uint4(s, b, e, (uint32_t)(s0->big & BIG_MASK));
            s0->big += (1ull << BIG_SHIFT) | nch;
          } else {
            J.q0[s0->nmain++] = s;
          }
          s0->deg += e - b;
        }
      }
    }
  }
  for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
    s_prev_pull[j] = 0;
    s_done[j] = 0;
  }
  bool ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);

  uint32_t L = 0;
  while (ok) {
    // ---- per-job decision (every block computes the same)
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const MsJob& J = jobs[j];
      const LevelSlot* in = &J.ctrl->slot[L % 3];
      const unsigned long long nmain = dev::ld_relaxed_u64(&in->nmain);
      const unsigned long long big = dev::ld_relaxed_u64(&in->big);
      const unsigned long long fdeg = dev::ld_relaxed_u64(&in->deg);
      const uint32_t nbig = (uint32_t)(big >> BIG_SHIFT);
      uint32_t mode = s_done[j] ? M_DONE : decide(J, p, s_prev_pull[j], nmain + nbig, fdeg);
      if (mode != M_DONE && (L + 1 >= 255 || nbig > J.big_cap || nmain > J.n)) {
        if (blockIdx.x == 0) atomicOr(&J.ctrl->error, L + 1 >= 255 ? MS_ERR_OVERFLOW : MS_ERR_QUEUE);
        mode = M_DONE;
      }
      if (mode == M_DONE && !s_done[j]) {
        s_done[j] = 1;
        if (blockIdx.x == 0) J.ctrl->levels = L;
      }
      s_mode[j] = mode;
      s_nmain[j] = nmain;
      s_nbig[j] = nbig;
      s_deg[j] = 0;
      if (mode == M_PULL)
        s_tile_end[j] = (J.n + 31) / 32;
      else if (mode == M_PUSH)
        s_tile_end[j] = (nmain + 31) / 32 + (big & BIG_MASK);
      else
        s_tile_end[j] = 0;
      if (blockIdx.x == 0 && mode != M_DONE) {
        J.ctrl->slot[(L + 2) % 3] = LevelSlot{0, 0, 0, 0};
        if (mode == M_PULL)
          J.ctrl->pull_levels++;
        else
          J.ctrl->push_levels++;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long acc = 0;
      for (uint32_t j = 0; j < njobs; j++) {
        acc += s_tile_end[j];
        s_tile_end[j] = acc;
      }
      s_total = acc;
    }
    __syncthreads();
    const unsigned long long total = s_total;
    if (total == 0) break;

    // ---- phase A: all jobs' tiles over all warps
    for (unsigned long long t = gwarp; t < total; t += nwarps) {
      uint32_t lo = 0, hi = njobs - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_tile_end[mid] > t)
          hi = mid;
        else
          lo = mid + 1;
      }
      const uint32_t j = lo;
      const unsigned long long t0 = j ? s_tile_end[j - 1] : 0;
      const uint32_t lt = (uint32_t)(t - t0);
      const MsJob& J = jobs[j];
      const unsigned long long* fcur = (L & 1) ? J.fr1 : J.fr0;
      unsigned long long* fnext = (L & 1) ? J.fr0 : J.fr1;
      const uint32_t* qin = (L & 1) ? J.q1 : J.q0;
      uint32_t* qout = (L & 1) ? J.q0 : J.q1;
      const uint4* qbin = (L & 1) ? J.qb1 : J.qb0;
      uint4* qbout = (L & 1) ? J.qb0 : J.qb1;
      LevelSlot* out = &J.ctrl->slot[(L + 1) % 3];
      if (s_mode[j] == M_PULL) {
        const unsigned long long cap = (p.policy == PBG_DIR_AUTO) ? (unsigned long long)(J.n / p.beta) : J.n;
        pull_tile(J, lt, fcur, fnext, out, qout, qbout, (uint8_t)(L + 1), cap, p.big_deg, &s_deg[j]);
      } else {
        const uint32_t main_tiles = (uint32_t)((s_nmain[j] + 31) / 32);
        if (lt < main_tiles)
          push_main_tile(J, lt, s_nmain[j], qin, fcur, fnext, out, qout, qbout, p.warp_deg, p.big_deg, &s_deg[j]);
        else
          push_chunk_tile(J, lt - main_tiles, qbin, s_nbig[j], fcur, fnext, out, qout, qbout, p.big_deg,
                          &s_deg[j]);
      }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x)
      if (s_deg[j]) atomicAdd(&jobs[j].ctrl->slot[(L + 1) % 3].deg, s_deg[j]);
    ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
    if (!ok) break;

    // ---- phase B: push jobs fold the new masks into vis and write levels,
    // and clear their old frontier; a job going from pull to push clears its
    // old frontier buffer densely (it becomes the next level's target).
    if (threadIdx.x == 0) s_any_phase_b = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const MsJob& J = jobs[j];
      const uint32_t mode = s_mode[j];
      uint32_t nb_mode = M_DONE;
      if (mode != M_DONE) {
        const LevelSlot* o = &J.ctrl->slot[(L + 1) % 3];
        const unsigned long long big = dev::ld_relaxed_u64(&o->big);
        nb_mode = decide(J, p, mode == M_PULL, dev::ld_relaxed_u64(&o->nmain) + (big >> BIG_SHIFT),
                         dev::ld_relaxed_u64(&o->deg));
      }
      uint32_t b = 0;
      if (mode == M_PUSH) b = 1;
      if (mode == M_PULL && nb_mode == M_PUSH) b = 2;
      s_mode[j] = b;  // reused: 0 nothing, 1 push fold, 2 dense clear
      s_prev_pull[j] = (mode == M_PULL) ? 1 : (mode == M_PUSH ? 0 : s_prev_pull[j]);
      if (b) s_any_phase_b = 1;
    }
    __syncthreads();
    if (s_any_phase_b) {
      for (uint32_t j = 0; j < njobs; j++) {
        const MsJob& J = jobs[j];
        unsigned long long* fcur = (L & 1) ? J.fr1 : J.fr0;
        const unsigned long long* fnext = (L & 1) ? J.fr0 : J.fr1;
        if (s_mode[j] == 1) {
          const uint32_t* qin = (L & 1) ? J.q1 : J.q0;
          const uint32_t* qout = (L & 1) ? J.q0 : J.q1;
          const uint4* qbin = (L & 1) ? J.qb1 : J.qb0;
          const uint4* qbout = (L & 1) ? J.qb0 : J.qb1;
          const LevelSlot* o = &J.ctrl->slot[(L + 1) % 3];
          const unsigned long long onm = dev::ld_relaxed_u64(&o->nmain);
          const unsigned long long onb =
              min(dev::ld_relaxed_u64(&o->big) >> BIG_SHIFT, (unsigned long long)J.big_cap);
          for (unsigned long long i = tid; i < onm + onb; i += nth) {
            const uint32_t v = (i < onm) ? qout[i] : qbout[i - onm].x;
            const unsigned long long nb = fnext[v];
            J.vis[v] |= nb;
            write_levels(J.levels, J.n, v, nb, (uint8_t)(L + 1));
          }
          for (unsigned long long i = tid; i < s_nmain[j] + s_nbig[j]; i += nth) {
            const uint32_t u = (i < s_nmain[j]) ? qin[i] : qbin[i - s_nmain[j]].x;
            fcur[u] = 0;
          }
        } else if (s_mode[j] == 2) {
          for (unsigned long long i = tid; i < J.n; i += nth) fcur[i] = 0;
        }
      }
      ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
    }
    L++;
  }
}

std::mutex g_grid_mu;
int g_grid_dev = -1, g_grid = 0;

}  // namespace

int ms_full_grid(int num_sms) {
  std::lock_guard<std::mutex> lk(g_grid_mu);
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_grid_dev != dev) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_persistent, 512, 0);
    if (e != cudaSuccess || per_sm < 1) return -1;
    g_grid = per_sm * num_sms;
    g_grid_dev = dev;
  }
  return g_grid;
}

int ms_launch(const MsJob* d_jobs, uint32_t njobs, const pbg_bfs_opts& o, dev::GridSync* d_sync, int num_sms,
              cudaStream_t s, int max_blocks) {
  int grid = ms_full_grid(num_sms);
  if (grid < 1) return fail(PBG_ERR_CUDA, "multi-source kernel cannot be resident");
  if (max_blocks > 0 && max_blocks < grid) grid = max_blocks;
  MsParams p{o.alpha, o.beta, o.direction, std::min<uint32_t>(32u, o.chunk_min_degree),
             std::max<uint32_t>(1024u, o.chunk_min_degree)};
  void* params[] = {(void*)&d_jobs, &njobs, &p, &d_sync};
  PBG_CUDA(cudaLaunchCooperativeKernel((const void*)ms_persistent, dim3(grid), dim3(512), params, 0, s));
  return PBG_OK;
}

}  // namespace pbg
