// bfs.cu -- single-source, direction-optimizing BFS as ONE persistent
// cooperative kernel per search (sm_100a).
//
// Replaces the hot loop of backForwardBFS
// (benchmarks/breadthFirstSearch/backForwardBFS/BFS.C:38-61) and the two
// edge_map bodies of common/ligraLight.h:
//   * top-down   = edge_map_sparse (ligraLight.h:70-85): the frontier is a
//     queue; every frontier edge (u, v) tries to claim v;
//   * bottom-up  = edge_map_dense (ligraLight.h:87-112): every unvisited v
//     scans N(v) for a frontier vertex and stops at the first one;
//   * the switch = edge_map::operator() (ligraLight.h:114-136): go bottom-up
//     when |F| + sum deg(F) > m / alpha, stay bottom-up while |F| > n / beta.
//
// Device layout (all in HBM, resident across calls on the handle):
//   offsets u32[n+1], edges u32[m]     CSR, read through the read-only path
//   parent  u32[n]                     output (0xFFFFFFFF = unvisited)
//   level   u32[n]                     optional output
//   bm[2]   u32[nwords]                visited bitmaps (2 MiB at n = 2^24, L2-resident)
//   q[2]    u32[n]                     frontier queues of short lists (deg < chunk_min_degree),
//                                      expanded 32 lists per warp, one per lane
//   qbig[2] uint4[big_cap]             (v, begin, end, first chunk) of longer lists, cut
//                                      in 256-edge pieces that any warp of the grid expands
//   ctrl                               counters, barrier, statistics
//
// Invariant: at the start of level L, bm[cur] holds every vertex of level <= L
// (plus degree-0 vertices of symmetric graphs and the padding bits past n, so
// whole words can be skipped).  Bottom-up therefore needs no separate frontier
// bitmap: an unvisited v whose neighbour u is in bm[cur] has level(u) == L.
//
// Parent rules:
//   ANY: claim by atomicOr on bm[cur] in place; the winner writes parent.
//   MIN/MAX: every frontier edge into a vertex not in bm[cur] (read-only this
//     level) does atomicMin/atomicMax on parent; the claim that decides who
//     enqueues v goes to bm[cur^1], which holds level <= L-1 and receives the
//     frontier's own bits from the threads expanding it; then cur flips.
//   Bottom-up scans N(v) ascending (MAX: descending) and stops at the first
//   frontier neighbour, which is the min (max) because lists are sorted.
//
// One grid barrier per level.  Every barrier wait is bounded by a
// %globaltimer budget; on expiry the kernel sets an error bit and all blocks
// return, the host reports PBG_ERR_TIMEOUT.
//
// Graphs whose largest degree is below the chunk degree run bfs_lean, the
// same search without the chunk queue (see its comment).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "device_util.cuh"
#include "internal.cuh"

namespace pbg {
namespace {

using dev::block_sum;
using dev::FULL;
using dev::globaltimer;
using dev::ld_relaxed_u64;
constexpr uint32_t CHUNK = 256;  // edges per chunk task: 8 per lane of a warp
constexpr int PER_LANE = 8;      // independent loads each lane keeps in flight
constexpr unsigned long long BIG_SHIFT = 40;
constexpr unsigned long long BIG_MASK = (1ull << BIG_SHIFT) - 1;

enum { MODE_ANY = 0, MODE_MIN = 1, MODE_MAX = 2 };

struct BfsArgs {
  const uint32_t* __restrict__ offsets;
  const uint32_t* __restrict__ edges;
  const uint32_t* __restrict__ iso;
  uint32_t* parent;
  uint32_t* level;
  uint32_t* bm0;
  uint32_t* bm1;
  uint32_t* q0;
  uint32_t* q1;
  uint2* qr0;  // adjacency range (begin, end) of each q entry
  uint2* qr1;
  uint4* qb0;
  uint4* qb1;
  BfsCtrl* ctrl;
  unsigned long long m;
  uint32_t n;
  uint32_t nwords;
  uint32_t big_cap;
  uint32_t src;
  uint32_t alpha;
  uint32_t beta;
  uint32_t policy;
  uint32_t chunk_deg;
  uint32_t symmetric;
};

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Fills x[0, n) with 0xFFFFFFFF, 16 bytes per store where aligned.
__device__ __forceinline__ void init_fill(uint32_t* x, uint32_t n, unsigned long long tid, unsigned long long nth) {
  const uint32_t mis = (uint32_t)(((16 - (reinterpret_cast<uintptr_t>(x) & 15)) & 15) / 4);
  const uint32_t head = mis < n ? mis : n;
  for (unsigned long long i = tid; i < head; i += nth) x[i] = PBG_NONE;
  uint4* x4 = reinterpret_cast<uint4*>(x + head);
  const unsigned long long n4 = (n - head) / 4;
  const uint4 f = make_uint4(PBG_NONE, PBG_NONE, PBG_NONE, PBG_NONE);
  for (unsigned long long i = tid; i < n4; i += nth) x4[i] = f;
  for (unsigned long long i = head + n4 * 4 + tid; i < n; i += nth) x[i] = PBG_NONE;
}

// The adjacency ranges of the candidates v[i] (set bits of `act`), loaded
// before their claims are issued, so the winners' ranges, which the append
// needs, arrive during the claims' round trip instead of after it.
__device__ __forceinline__ void load_ranges(const BfsArgs& a, const uint32_t (&v)[PER_LANE], unsigned act,
                                            uint32_t (&ob)[PER_LANE], uint32_t (&oe)[PER_LANE]) {
#pragma unroll
  for (int i = 0; i < PER_LANE; i++) {
    ob[i] = ((act >> i) & 1u) ? __ldg(a.offsets + v[i]) : 0u;
    oe[i] = ((act >> i) & 1u) ? __ldg(a.offsets + v[i] + 1) : 0u;
  }
}

// Warp-collective append of up to K vertices per lane (cand[i] for the set
// bits i of `win`) to the next frontier.  Vertices with degree >= chunk_deg
// go to the chunk queue as (v, begin, end, first chunk) with their number of
// CHUNK-edge pieces; the rest to the main queue.  (ob[i], oe[i]) is cand[i]'s
// adjacency range (load_ranges).  Positions come from warp
// prefix sums and one atomic per queue per warp: entries of one warp are
// contiguous, and chunk numbering follows slot order across warps because
// slot and chunk counters move in one 64-bit atomic.
template <int K>
__device__ __forceinline__ void emit_k(const BfsArgs& a, LevelSlot* out, uint32_t* qout, uint2* qrout,
                                       uint4* qbout, const uint32_t (&cand)[K], unsigned win,
                                       unsigned long long& degacc, const uint32_t (&ob)[K],
                                       const uint32_t (&oe)[K]) {
  if (!__any_sync(FULL, win != 0)) return;
  const int lane = threadIdx.x & 31;
  // pass 1: classify (only a bit per candidate stays live)
  uint32_t ns = 0, nc = 0, nch = 0;
  unsigned chunked = 0;
#pragma unroll
  for (int i = 0; i < K; i++) {
    if ((win >> i) & 1u) {
      const uint32_t d = oe[i] - ob[i];
      degacc += d;
      if (d >= a.chunk_deg) {
        chunked |= 1u << i;
        nc++;
        nch += (d + CHUNK - 1) / CHUNK;
      } else {
        ns++;
      }
    }
  }
  const uint32_t ps = warp_incl_scan(ns), pc = warp_incl_scan(nc), pch = warp_incl_scan(nch);
  const uint32_t ts = __shfl_sync(FULL, ps, 31), tc = __shfl_sync(FULL, pc, 31), tch = __shfl_sync(FULL, pch, 31);
  unsigned long long bs = 0, bc = 0;
  if (lane == 0) {
    if (ts) bs = atomicAdd(&out->nmain, (unsigned long long)ts);
    if (tc) bc = atomicAdd(&out->big, ((unsigned long long)tc << BIG_SHIFT) | tch);
  }
  bs = __shfl_sync(FULL, bs, 0);
  bc = __shfl_sync(FULL, bc, 0);
  unsigned long long ps_pos = bs + ps - ns;
  uint32_t pc_pos = (uint32_t)(bc >> BIG_SHIFT) + pc - nc;
  uint32_t chunk = (uint32_t)(bc & BIG_MASK) + pch - nch;
  // pass 2: write
#pragma unroll
  for (int i = 0; i < K; i++) {
    if ((win >> i) & 1u) {
      const uint32_t b = ob[i], e = oe[i];
      if ((chunked >> i) & 1u) {
        if (pc_pos < a.big_cap)
          qbout[pc_pos] = make_uint4(cand[i], b, e, chunk);
        else
          atomicOr(&a.ctrl->sync.error, ERR_QUEUE);
        pc_pos++;
        chunk += (e - b + CHUNK - 1) / CHUNK;
      } else {
        qout[ps_pos] = cand[i];
        qrout[ps_pos] = make_uint2(b, e);
        ps_pos++;
        // the next level reads this list: start it on its way from HBM to L2
        if (e > b) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.edges + b));
      }
    }
  }
}

// Top-down claims of up to K neighbours v[i] (set bits of `act`) by the
// lane's vertex u.  Every load and atomic of the K candidates is issued before
// any store that depends on one, so the K round trips overlap instead of
// running one after another.  Returns the bits of the candidates this lane
// enqueues.
template <int MODE, int K>
__device__ __forceinline__ unsigned td_claim_k(const BfsArgs& a, const uint32_t* vis, uint32_t* claim, uint32_t u,
                                               const uint32_t (&v)[K], unsigned act, uint32_t next_level) {
  unsigned live = act;
  if (MODE != MODE_ANY) {
    // MIN/MAX test the read-only snapshot of the level's visited set first
    uint32_t w[K];
#pragma unroll
    for (int i = 0; i < K; i++) w[i] = ((act >> i) & 1u) ? vis[v[i] >> 5] : 0u;
#pragma unroll
    for (int i = 0; i < K; i++)
      if ((w[i] >> (v[i] & 31)) & 1u) live &= ~(1u << i);
#pragma unroll
    for (int i = 0; i < K; i++) {
      if ((live >> i) & 1u) {
        if (MODE == MODE_MIN)
          atomicMin(a.parent + v[i], u);
        else
          atomicMax(reinterpret_cast<int*>(a.parent) + v[i], (int)u);
      }
    }
  }
  uint32_t old[K];
#pragma unroll
  for (int i = 0; i < K; i++) old[i] = ((live >> i) & 1u) ? atomicOr(claim + (v[i] >> 5), 1u << (v[i] & 31)) : FULL;
  unsigned win = 0;
#pragma unroll
  for (int i = 0; i < K; i++)
    if (!((old[i] >> (v[i] & 31)) & 1u)) win |= 1u << i;
  if (MODE == MODE_ANY) {
#pragma unroll
    for (int i = 0; i < K; i++)
      if ((win >> i) & 1u) a.parent[v[i]] = u;
  }
  if (a.level && win) {
#pragma unroll
    for (int i = 0; i < K; i++)
      if ((win >> i) & 1u) a.level[v[i]] = next_level;
  }
  return win;
}

// One CHUNK-edge piece of a long list, expanded by a whole warp.
template <int MODE>
__device__ __forceinline__ void td_chunk(const BfsArgs& a, const uint4& ent, uint32_t c_local, const uint32_t* vis,
                                         uint32_t* claim, LevelSlot* out, uint32_t* qout, uint2* qrout,
                                         uint4* qbout, uint32_t next_level, unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const uint32_t u = ent.x;
  const uint32_t cb = ent.y + c_local * CHUNK;
  const uint32_t ce = min(ent.z, cb + CHUNK);
  if (MODE != MODE_ANY && c_local == 0 && lane == 0) atomicOr(claim + (u >> 5), 1u << (u & 31));
  uint32_t v[PER_LANE];
  unsigned act = 0;
#pragma unroll
  for (int i = 0; i < PER_LANE; i++) {
    const uint32_t j = cb + i * 32 + lane;
    v[i] = 0;
    if (j < ce) {
      v[i] = __ldg(a.edges + j);
      act |= 1u << i;
    }
  }
  uint32_t ob[PER_LANE], oe[PER_LANE];
  load_ranges(a, v, act, ob, oe);
  const unsigned win = td_claim_k<MODE, PER_LANE>(a, vis, claim, u, v, act, next_level);
  emit_k<PER_LANE>(a, out, qout, qrout, qbout, v, win, degacc, ob, oe);
}

// 32 short lists (degree < chunk_deg), one per lane, PER_LANE edges a step.
template <int MODE>
__device__ __forceinline__ void td_small(const BfsArgs& a, uint32_t tile, const uint32_t* qin,
                                         const uint2* qrin, unsigned long long nmain, const uint32_t* vis,
                                         uint32_t* claim, LevelSlot* out, uint32_t* qout, uint2* qrout,
                                         uint4* qbout, uint32_t next_level, unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const unsigned long long idx = (unsigned long long)tile * 32 + lane;
  uint32_t u = 0, b = 0, e = 0;
  if (idx < nmain) {
    u = qin[idx];
    const uint2 r = qrin[idx];  // range stored by the claimer: no offsets load
    b = r.x;
    e = r.y;
    if (MODE != MODE_ANY) atomicOr(claim + (u >> 5), 1u << (u & 31));
  }
  const uint32_t maxd = __reduce_max_sync(FULL, e - b);
  for (uint32_t k0 = 0; k0 < maxd; k0 += PER_LANE) {
    uint32_t v[PER_LANE];
    unsigned act = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; i++) {
      const uint32_t j = b + k0 + i;
      v[i] = 0;
      if (j < e) {
        v[i] = __ldg(a.edges + j);
        act |= 1u << i;
      }
    }
    uint32_t ob[PER_LANE], oe[PER_LANE];
    load_ranges(a, v, act, ob, oe);
    const unsigned win = td_claim_k<MODE, PER_LANE>(a, vis, claim, u, v, act, next_level);
    emit_k<PER_LANE>(a, out, qout, qrout, qbout, v, win, degacc, ob, oe);
  }
}

// Top-down level: chunk tasks first (edge-balanced over every warp of the
// grid), then 32-entry tiles of short lists.
template <int MODE>
__device__ void td_level(const BfsArgs& a, const uint32_t* qin, const uint2* qrin, unsigned long long nmain,
                         const uint4* qbin, uint32_t nbig, uint32_t nchunks, const uint32_t* vis, uint32_t* claim,
                         LevelSlot* out, uint32_t* qout, uint2* qrout, uint4* qbout, uint32_t next_level,
                         unsigned long long& degacc) {
  // tasks go round-robin over blocks first, so a small level still uses
  // every SM's load/store pipeline
  const uint32_t gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  const unsigned long long tasks = nchunks + (nmain + 31) / 32;
  for (unsigned long long t = gw; t < tasks; t += tw) {
    if (t < nchunks) {
      const uint32_t c = (uint32_t)t;
      uint32_t lo = 0, hi = nbig - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (qbin[mid].w <= c)
          lo = mid;
        else
          hi = mid - 1;
      }
      const uint4 ent = qbin[lo];
      td_chunk<MODE>(a, ent, c - ent.w, vis, claim, out, qout, qrout, qbout, next_level, degacc);
    } else {
      td_small<MODE>(a, (uint32_t)(t - nchunks), qin, qrin, nmain, vis, claim, out, qout, qrout, qbout, next_level,
                     degacc);
    }
  }
}

// Bottom-up over bitmap words, one warp per word, one lane per vertex.  Each
// unvisited lane probes the first LSHARE neighbours of its own list, PROBES
// independent loads a step (ascending; MAX: descending), while any lane of
// the warp is still unresolved; lists that are longer and still unresolved
// are then scanned by the whole warp, 32 neighbours per step, one list after
// another, the first frontier neighbour in scan order winning (the early
// exit of ligraLight.h:99-105).  A lane share of 16 in steps of 4 was the
// fastest of shares 4-64 and steps 1-8 on rMat 2^20 and 2^24: one probe a
// step leaves most of a warp's misses to the serial warp scan, wide steps
// issue requests a lane rarely needs.  The word loop is software-pipelined three deep: the
// bitmap word two steps ahead and the offsets one step ahead are in flight
// while the current word's probes run.  Counts and degree sums stay in
// registers.
template <int MODE>
__device__ __forceinline__ void bu_word(const BfsArgs& a, const uint32_t* vin, uint32_t* vout, uint32_t next_level,
                                        uint32_t w, uint32_t word, uint32_t b, uint32_t e, unsigned long long& cnt,
                                        unsigned long long& degacc) {
  constexpr int PROBES = 4;
  constexpr uint32_t LSHARE = 16;
  const int lane = threadIdx.x & 31;
  if (word == FULL) {
    if (lane == 0) vout[w] = word;
    return;
  }
  const uint32_t v = w * 32 + lane;
  const uint32_t deg = e - b;  // 0 for visited lanes
  bool found = false;
  uint32_t p = 0;
  for (uint32_t k0 = 0; k0 < LSHARE; k0 += PROBES) {
    if (!__any_sync(FULL, !found && deg > k0)) break;
    uint32_t cu[PROBES], cw[PROBES];
#pragma unroll
    for (int i = 0; i < PROBES; i++) {
      cu[i] = 0;
      if (!found && k0 + i < deg) cu[i] = __ldg(a.edges + ((MODE == MODE_MAX) ? (e - 1 - k0 - i) : (b + k0 + i)));
    }
#pragma unroll
    for (int i = 0; i < PROBES; i++) cw[i] = (!found && k0 + i < deg) ? vin[cu[i] >> 5] : 0u;
#pragma unroll
    for (int i = 0; i < PROBES; i++) {
      if (!found && k0 + i < deg && ((cw[i] >> (cu[i] & 31)) & 1u)) {
        found = true;
        p = cu[i];
      }
    }
  }
  unsigned mm = __ballot_sync(FULL, !found && deg > LSHARE);
  while (mm) {
    const int l = __ffs(mm) - 1;
    mm &= mm - 1;
    const uint32_t bb = __shfl_sync(FULL, b, l);
    const uint32_t ee = __shfl_sync(FULL, e, l);
    uint32_t hit = 0;
    bool got = false;
    if (MODE == MODE_MAX) {
      for (long long top = (long long)ee - LSHARE; top > (long long)bb && !got; top -= 32) {
        const long long j = top - 1 - lane;
        uint32_t x = 0;
        bool h = false;
        if (j >= (long long)bb) {
          x = __ldg(a.edges + j);
          h = (vin[x >> 5] >> (x & 31)) & 1u;
        }
        const unsigned hb = __ballot_sync(FULL, h);
        if (hb) {
          got = true;
          hit = __shfl_sync(FULL, x, __ffs(hb) - 1);
        }
      }
    } else {
      for (uint32_t j0 = bb + LSHARE; j0 < ee && !got; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t x = 0;
        bool h = false;
        if (j < ee) {
          x = __ldg(a.edges + j);
          h = (vin[x >> 5] >> (x & 31)) & 1u;
        }
        const unsigned hb = __ballot_sync(FULL, h);
        if (hb) {
          got = true;
          hit = __shfl_sync(FULL, x, __ffs(hb) - 1);
        }
      }
    }
    if (lane == l && got) {
      found = true;
      p = hit;
    }
  }
  const unsigned nb = __ballot_sync(FULL, found);
  if (lane == 0) vout[w] = word | nb;
  if (found) {
    a.parent[v] = p;
    if (a.level) a.level[v] = next_level;
    cnt += 1;
    degacc += deg;
  }
}

template <int MODE>
__device__ void bu_level(const BfsArgs& a, const uint32_t* vin, uint32_t* vout, uint32_t next_level,
                         unsigned long long& cnt, unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nw = a.nwords;
  uint32_t w0 = gw, w1 = gw + tw;
  uint32_t word0 = (w0 < nw) ? vin[w0] : FULL;
  uint32_t word1 = (w1 < nw) ? vin[w1] : FULL;
  uint32_t b0 = 0, e0 = 0;
  if (!((word0 >> lane) & 1u)) {
    b0 = __ldg(a.offsets + w0 * 32 + lane);
    e0 = __ldg(a.offsets + w0 * 32 + lane + 1);
  }
  while (w0 < nw) {
    const uint32_t w2 = w1 + tw;
    const uint32_t word2 = (w2 < nw) ? vin[w2] : FULL;
    uint32_t b1 = 0, e1 = 0;
    if (!((word1 >> lane) & 1u)) {
      b1 = __ldg(a.offsets + w1 * 32 + lane);
      e1 = __ldg(a.offsets + w1 * 32 + lane + 1);
    }
    bu_word<MODE>(a, vin, vout, next_level, w0, word0, b0, e0, cnt, degacc);
    w0 = w1;
    word0 = word1;
    b0 = b1;
    e0 = e1;
    w1 = w2;
    word1 = word2;
  }
}

// Rebuilds the frontier queues from the bitmap difference after a bottom-up
// level (the sparse form of the dense frontier, as pack_index does in
// ligraLight.h:132).  Lane l of a warp handles word w0 + l.
__device__ void dense_to_queue(const BfsArgs& a, const uint32_t* before, const uint32_t* after, LevelSlot* out,
                               uint32_t* qout, uint2* qrout, uint4* qbout) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long dummy = 0;
  for (uint32_t w0 = gw * 32; w0 < a.nwords; w0 += tw * 32) {
    const uint32_t w = w0 + lane;
    uint32_t diff = (w < a.nwords) ? (after[w] & ~before[w]) : 0u;
    while (__any_sync(FULL, diff != 0)) {
      uint32_t v[PER_LANE];
      unsigned act = 0;
#pragma unroll
      for (int i = 0; i < PER_LANE; i++) {
        v[i] = 0;
        if (diff) {
          v[i] = w * 32 + (__ffs(diff) - 1);
          diff &= diff - 1;
          act |= 1u << i;
        }
      }
      uint32_t ob[PER_LANE], oe[PER_LANE];
      load_ranges(a, v, act, ob, oe);
      emit_k<PER_LANE>(a, out, qout, qrout, qbout, v, act, dummy, ob, oe);
    }
  }
}

// BLOCK = 256 runs 4 blocks per SM at <= 64 registers, 512 one block at
// <= 128 registers (no spills), 1024 one block at <= 64 registers.
template <int MODE, int BLOCK>
__global__ void __launch_bounds__(BLOCK, BLOCK == 256 ? 4 : 1) bfs_persistent(BfsArgs a) {
  BfsCtrl* c = a.ctrl;
  __shared__ unsigned long long s_in[3];
  unsigned long long bar_epoch = 0;  // barriers passed (thread 0's count matters)

  // ---- init: parent/level = NONE, bitmaps = degree-0 + padding bits, source.
  {
    const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
    if (tid == 0) c->t_start = globaltimer();
    init_fill(a.parent, a.n, tid, nth);
    if (a.level) init_fill(a.level, a.n, tid, nth);
    const uint32_t sw = a.src >> 5, sbit = 1u << (a.src & 31);
    for (unsigned long long w = tid; w < a.nwords; w += nth) {
      const uint32_t x = a.iso[w];
      a.bm0[w] = (w == sw) ? (x | sbit) : x;
      a.bm1[w] = (MODE == MODE_ANY && w == sw) ? (x | sbit) : x;
    }
    if (tid == 0) {
      const uint32_t b = __ldg(a.offsets + a.src), e = __ldg(a.offsets + a.src + 1);
      const uint32_t deg = e - b;
      for (int s = 0; s < 3; s++) c->slot[s] = LevelSlot{0, 0, 0, 0};
      c->conv = LevelSlot{0, 0, 0, 0};
      if (deg >= a.chunk_deg) {
        a.qb0[0] = make_uint4(a.src, b, e, 0u);
        c->slot[0].big = (1ull << BIG_SHIFT) | ((deg + CHUNK - 1) / CHUNK);
      } else {
        a.q0[0] = a.src;
        a.qr0[0] = make_uint2(b, e);
        c->slot[0].nmain = 1;
      }
      c->slot[0].deg = deg;
    }
  }
  // the source's own entries, after every block has filled
  if (!dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.parent[a.src] = a.src;
    if (a.level) a.level[a.src] = 0;
  }
  bool ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);

  uint32_t cur = 0;
  bool prev_bu = false;
  unsigned long long visited = 0, reached = 0, bumask = 0;
  uint32_t tdl = 0, bul = 0;
  uint32_t L = 0;
  while (ok) {
    LevelSlot* in = &c->slot[L % 3];
    LevelSlot* out = &c->slot[(L + 1) % 3];
    if (threadIdx.x == 0) {
      s_in[0] = ld_relaxed_u64(&in->nmain);
      s_in[1] = ld_relaxed_u64(&in->big);
      s_in[2] = ld_relaxed_u64(&in->deg);
    }
    __syncthreads();
    unsigned long long nmain = s_in[0], big = s_in[1];
    const unsigned long long fdeg = s_in[2];
    __syncthreads();
    const unsigned long long nf = nmain + (big >> BIG_SHIFT);
    if (nf == 0) break;
    if (L >= a.n) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->sync.error, ERR_LEVEL_LIMIT);
      break;
    }

    bool bu;
    if (a.policy == PBG_DIR_TOPDOWN || !a.symmetric)
      bu = false;
    else if (a.policy == PBG_DIR_BOTTOMUP)
      bu = true;
    else if (!prev_bu)
      bu = (nf + fdeg) > a.m / a.alpha;
    else
      bu = nf > (unsigned long long)(a.n / a.beta);

    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->slot[(L + 2) % 3] = LevelSlot{0, 0, 0, 0};
      if (bu) c->conv = LevelSlot{0, 0, 0, 0};
      if (L < PBG_TRACE_LEVELS) {
        c->t_ns[L] = globaltimer();
        c->t_nf[L] = nf;
        c->t_deg[L] = fdeg;
        c->t_bu[L] = bu ? 1u : 0u;
      }
      visited += nf;
      reached += fdeg;
      if (bu) {
        bul++;
        if (L < 64) bumask |= 1ull << L;
      } else {
        tdl++;
      }
    }

    uint32_t* qin = (L & 1) ? a.q1 : a.q0;
    uint2* qrin = (L & 1) ? a.qr1 : a.qr0;
    uint2* qrout = (L & 1) ? a.qr0 : a.qr1;
    uint32_t* qout = (L & 1) ? a.q0 : a.q1;
    uint4* qbin = (L & 1) ? a.qb1 : a.qb0;
    uint4* qbout = (L & 1) ? a.qb0 : a.qb1;
    uint32_t* bcur = cur ? a.bm1 : a.bm0;
    uint32_t* both = cur ? a.bm0 : a.bm1;
    if (bu) {
      unsigned long long cnt = 0, degacc = 0;
      bu_level<MODE>(a, bcur, both, L + 1, cnt, degacc);
      const unsigned long long bc = block_sum(cnt);
      const unsigned long long bd = block_sum(degacc);
      if (threadIdx.x == 0) {
        if (bc) atomicAdd(&out->nmain, bc);
        if (bd) atomicAdd(&out->deg, bd);
      }
      cur ^= 1u;
    } else {
      if (prev_bu) {
        // the frontier came from a bottom-up level: build its queues first
        dense_to_queue(a, both, bcur, &c->conv, qin, qrin, qbin);
        ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
        if (!ok) break;
        if (threadIdx.x == 0) {
          s_in[0] = ld_relaxed_u64(&c->conv.nmain);
          s_in[1] = ld_relaxed_u64(&c->conv.big);
        }
        __syncthreads();
        nmain = s_in[0];
        big = s_in[1];
        __syncthreads();
      }
      const uint32_t nbig = (uint32_t)(big >> BIG_SHIFT);
      if (nbig > a.big_cap || nmain > a.n) {  // cannot happen: each vertex enters one frontier once
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->sync.error, ERR_QUEUE);
        break;
      }
      uint32_t* claim = (MODE == MODE_ANY) ? bcur : both;
      unsigned long long degacc = 0;
      td_level<MODE>(a, qin, qrin, nmain, qbin, nbig, (uint32_t)(big & BIG_MASK), bcur, claim, out, qout, qrout,
                     qbout, L + 1, degacc);
      const unsigned long long bd = block_sum(degacc);
      if (threadIdx.x == 0 && bd) atomicAdd(&out->deg, bd);
      if (MODE != MODE_ANY) cur ^= 1u;
    }
    prev_bu = bu;
    L++;
    ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (L <= PBG_TRACE_LEVELS) c->t_ns[L] = globaltimer();
    c->t_end = globaltimer();
    c->levels = L;
    c->td_levels = tdl;
    c->bu_levels = bul;
    c->final_bm = cur;
    c->visited = visited;
    c->edges_reached = reached;
    c->bu_mask = bumask;
  }
}

// ---------------------------------------------------------------- lean kernel
// For graphs whose every list is shorter than the chunk degree (a lattice, a
// road-like or random-local graph): the same direction-optimizing search as
// bfs_persistent without the chunk queue and its tasks, and with each warp
// adding its frontier degree (bottom-up: and count) to the level's counters
// itself instead of a block reduction; on the 3-D torus 160^3 about 20%
// faster a level.
// Bottom-up levels and the rebuild of queues after them are
// bfs_persistent's (bu_level, dense_to_queue).

// Appends the winners (bits of `win`) of a step to the next queue, one atomic
// per warp.
__device__ __forceinline__ void lean_emit(const BfsArgs& a, LevelSlot* out, uint32_t* qout, uint2* qrout,
                                          const uint32_t (&cand)[PER_LANE], unsigned win,
                                          unsigned long long& degacc, const uint32_t (&ob)[PER_LANE],
                                          const uint32_t (&oe)[PER_LANE]) {
  if (!__any_sync(FULL, win != 0)) return;
  const int lane = threadIdx.x & 31;
  const uint32_t ns = __popc(win);
  const uint32_t ps = warp_incl_scan(ns);
  const uint32_t ts = __shfl_sync(FULL, ps, 31);
  unsigned long long b0 = 0;
  if (lane == 0) b0 = atomicAdd(&out->nmain, (unsigned long long)ts);
  unsigned long long pos = __shfl_sync(FULL, b0, 0) + ps - ns;
#pragma unroll
  for (int i = 0; i < PER_LANE; i++) {
    if ((win >> i) & 1u) {
      const uint32_t b = ob[i], e = oe[i];
      degacc += e - b;
      qout[pos] = cand[i];
      qrout[pos] = make_uint2(b, e);
      pos++;
      // the next level reads this list: start it on its way from HBM to L2
      if (e > b) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.edges + b));
    }
  }
}

// 32 queue entries, one per lane, PER_LANE edges a step.
template <int MODE>
__device__ __forceinline__ void lean_tile(const BfsArgs& a, uint32_t tile, const uint32_t* qin, const uint2* qrin,
                                          unsigned long long nq, const uint32_t* vis, uint32_t* claim,
                                          LevelSlot* out, uint32_t* qout, uint2* qrout, uint32_t next_level,
                                          unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const unsigned long long idx = (unsigned long long)tile * 32 + lane;
  uint32_t u = 0, b = 0, e = 0;
  if (idx < nq) {
    u = qin[idx];
    const uint2 r = qrin[idx];  // range stored by the claimer: no offsets load
    b = r.x;
    e = r.y;
    if (MODE != MODE_ANY) atomicOr(claim + (u >> 5), 1u << (u & 31));
  }
  const uint32_t maxd = __reduce_max_sync(FULL, e - b);
  for (uint32_t k0 = 0; k0 < maxd; k0 += PER_LANE) {
    uint32_t v[PER_LANE];
    unsigned act = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; i++) {
      const uint32_t j = b + k0 + i;
      v[i] = 0;
      if (j < e) {
        v[i] = __ldg(a.edges + j);
        act |= 1u << i;
      }
    }
    uint32_t ob[PER_LANE], oe[PER_LANE];
    load_ranges(a, v, act, ob, oe);
    const unsigned win = td_claim_k<MODE, PER_LANE>(a, vis, claim, u, v, act, next_level);
    lean_emit(a, out, qout, qrout, v, win, degacc, ob, oe);
  }
}

template <int MODE>
__global__ void __launch_bounds__(1024, 1) bfs_lean(BfsArgs a) {
  BfsCtrl* c = a.ctrl;
  __shared__ unsigned long long s_in[3];
  unsigned long long bar_epoch = 0;
  {
    const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
    if (tid == 0) c->t_start = globaltimer();
    init_fill(a.parent, a.n, tid, nth);
    if (a.level) init_fill(a.level, a.n, tid, nth);
    const uint32_t sw = a.src >> 5, sbit = 1u << (a.src & 31);
    for (unsigned long long w = tid; w < a.nwords; w += nth) {
      const uint32_t x = a.iso[w];
      a.bm0[w] = (w == sw) ? (x | sbit) : x;
      a.bm1[w] = (MODE == MODE_ANY && w == sw) ? (x | sbit) : x;
    }
    if (tid == 0) {
      const uint32_t b = __ldg(a.offsets + a.src), e = __ldg(a.offsets + a.src + 1);
      for (int s = 0; s < 3; s++) c->slot[s] = LevelSlot{0, 0, 0, 0};
      c->conv = LevelSlot{0, 0, 0, 0};
      a.q0[0] = a.src;
      a.qr0[0] = make_uint2(b, e);
      c->slot[0].nmain = 1;
      c->slot[0].deg = e - b;
    }
  }
  if (!dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.parent[a.src] = a.src;
    if (a.level) a.level[a.src] = 0;
  }
  bool ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
  uint32_t cur = 0;
  bool prev_bu = false;
  unsigned long long visited = 0, reached = 0, bumask = 0;
  uint32_t tdl = 0, bul = 0;
  uint32_t L = 0;
  while (ok) {
    LevelSlot* in = &c->slot[L % 3];
    LevelSlot* out = &c->slot[(L + 1) % 3];
    if (threadIdx.x == 0) {
      s_in[0] = ld_relaxed_u64(&in->nmain);
      s_in[1] = ld_relaxed_u64(&in->deg);
    }
    __syncthreads();
    unsigned long long nq = s_in[0];
    const unsigned long long nf = nq, fdeg = s_in[1];
    __syncthreads();
    if (nf == 0) break;
    if (L >= a.n) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->sync.error, ERR_LEVEL_LIMIT);
      break;
    }
    bool bu;
    if (a.policy == PBG_DIR_TOPDOWN || !a.symmetric)
      bu = false;
    else if (a.policy == PBG_DIR_BOTTOMUP)
      bu = true;
    else if (!prev_bu)
      bu = (nf + fdeg) > a.m / a.alpha;
    else
      bu = nf > (unsigned long long)(a.n / a.beta);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->slot[(L + 2) % 3] = LevelSlot{0, 0, 0, 0};
      if (bu) c->conv = LevelSlot{0, 0, 0, 0};
      if (L < PBG_TRACE_LEVELS) {
        c->t_ns[L] = globaltimer();
        c->t_nf[L] = nf;
        c->t_deg[L] = fdeg;
        c->t_bu[L] = bu ? 1u : 0u;
      }
      visited += nf;
      reached += fdeg;
      if (bu) {
        bul++;
        if (L < 64) bumask |= 1ull << L;
      } else {
        tdl++;
      }
    }
    uint32_t* qin = (L & 1) ? a.q1 : a.q0;
    uint2* qrin = (L & 1) ? a.qr1 : a.qr0;
    uint2* qrout = (L & 1) ? a.qr0 : a.qr1;
    uint32_t* qout = (L & 1) ? a.q0 : a.q1;
    uint4* qbin = (L & 1) ? a.qb1 : a.qb0;
    uint32_t* bcur = cur ? a.bm1 : a.bm0;
    uint32_t* both = cur ? a.bm0 : a.bm1;
    unsigned long long cnt = 0, degacc = 0;
    if (bu) {
      bu_level<MODE>(a, bcur, both, L + 1, cnt, degacc);
      cur ^= 1u;
    } else {
      if (prev_bu) {
        // the frontier came from a bottom-up level: build its queue first
        // (every list is short, so nothing goes to the chunk queue)
        dense_to_queue(a, both, bcur, &c->conv, qin, qrin, qbin);
        ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
        if (!ok) break;
        if (threadIdx.x == 0) s_in[0] = ld_relaxed_u64(&c->conv.nmain);
        __syncthreads();
        nq = s_in[0];
        __syncthreads();
      }
      if (nq > a.n) {  // cannot happen: each vertex enters one frontier once
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->sync.error, ERR_QUEUE);
        break;
      }
      uint32_t* claim = (MODE == MODE_ANY) ? bcur : both;
      // tiles go round-robin over blocks first, so a small level still uses
      // every SM's load/store pipeline
      const uint32_t gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
      const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
      const unsigned long long tiles = (nq + 31) / 32;
      for (unsigned long long t = gw; t < tiles; t += tw)
        lean_tile<MODE>(a, (uint32_t)t, qin, qrin, nq, bcur, claim, out, qout, qrout, L + 1, degacc);
      if (MODE != MODE_ANY) cur ^= 1u;
    }
    // per warp: one reduction atomic per counter (no block barrier)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cnt += __shfl_down_sync(FULL, cnt, o);
      degacc += __shfl_down_sync(FULL, degacc, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (bu && cnt) atomicAdd(&out->nmain, cnt);  // a count: the frontier is the bitmap difference
      if (degacc) atomicAdd(&out->deg, degacc);
    }
    prev_bu = bu;
    L++;
    ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (L <= PBG_TRACE_LEVELS) c->t_ns[L] = globaltimer();
    c->t_end = globaltimer();
    c->levels = L;
    c->td_levels = tdl;
    c->bu_levels = bul;
    c->final_bm = cur;
    c->visited = visited;
    c->edges_reached = reached;
    c->bu_mask = bumask;
  }
}

template <int MODE>
int launch_lean(const BfsArgs& a, int num_sms, cudaStream_t s) {
  static std::mutex mu;
  static int grid = 0, dev_of = -1;
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  int g;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev_of != dev) {
      int per_sm = 0;
      PBG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_lean<MODE>, 1024, 0));
      if (per_sm < 1) return fail(PBG_ERR_CUDA, "BFS kernel cannot be resident with this block size");
      grid = per_sm * num_sms;
      dev_of = dev;
    }
    g = grid;
  }
  BfsArgs args = a;
  void* params[] = {&args};
  PBG_CUDA(cudaLaunchCooperativeKernel((const void*)bfs_lean<MODE>, dim3(g), dim3(1024), params, 0, s));
  return PBG_OK;
}

template <int MODE, int BLOCK>
int launch_shape(const BfsArgs& a, int num_sms, cudaStream_t s) {
  static std::mutex mu;
  static int grid = 0, dev_of = -1;
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  int g;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev_of != dev) {
      int per_sm = 0;
      PBG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_persistent<MODE, BLOCK>, BLOCK, 0));
      if (per_sm < 1) return fail(PBG_ERR_CUDA, "BFS kernel cannot be resident with this block size");
      grid = per_sm * num_sms;
      dev_of = dev;
    }
    g = grid;
  }
  BfsArgs args = a;
  void* params[] = {&args};
  PBG_CUDA(cudaLaunchCooperativeKernel((const void*)bfs_persistent<MODE, BLOCK>, dim3(g), dim3(BLOCK), params, 0, s));
  return PBG_OK;
}

template <int MODE>
int launch_mode(const BfsArgs& a, int block, int num_sms, cudaStream_t s) {
  if (block == 256) return launch_shape<MODE, 256>(a, num_sms, s);
  if (block == 1024) return launch_shape<MODE, 1024>(a, num_sms, s);
  return launch_shape<MODE, 512>(a, num_sms, s);
}

}  // namespace

void resolve_opts(const pbg_bfs_opts* in, pbg_bfs_opts* o) {
  if (in)
    *o = *in;
  else
    pbg_bfs_opts_default(o);
  if (o->alpha == 0) o->alpha = 20;
  if (o->beta == 0) o->beta = 20;
  if (o->block_threads == 0) o->block_threads = 1024;
  if (o->chunk_min_degree == 0) o->chunk_min_degree = 32;
}

void resolve_graph_opts(const pbg_graph* g, const pbg_bfs_opts* in, bool multi, pbg_bfs_opts* o) {
  if (!in && g && (multi ? g->has_tuned_multi : g->has_tuned))
    resolve_opts(multi ? &g->tuned_multi : &g->tuned, o);
  else
    resolve_opts(in, o);
}

int bfs_ensure_workspace(pbg_graph* g, const pbg_bfs_opts& o) {
  BfsWorkspace& w = g->ws;
  if (w.ready && w.big_min_degree <= o.chunk_min_degree) return PBG_OK;
  bfs_free_workspace(g);
  const size_t n = g->n ? g->n : 1;
  const uint32_t big_cap = (uint32_t)std::min<uint64_t>(n, g->m / o.chunk_min_degree + 1);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaMalloc(&w.bm[i], sizeof(uint32_t) * g->nwords);
    if (e == cudaSuccess) e = cudaMalloc(&w.q[i], sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&w.qr[i], sizeof(uint2) * n);
    if (e == cudaSuccess) e = cudaMalloc(&w.qbig[i], sizeof(uint4) * big_cap);
  }
  if (e == cudaSuccess) e = cudaMalloc(&w.ctrl, sizeof(BfsCtrl));
  if (e == cudaSuccess) e = cudaMemset(w.ctrl, 0, sizeof(BfsCtrl));
  if (e == cudaSuccess && !w.ev0) e = cudaEventCreate(&w.ev0);
  if (e == cudaSuccess && !w.ev1) e = cudaEventCreate(&w.ev1);
  if (e != cudaSuccess) {
    bfs_free_workspace(g);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA,
                std::string("BFS workspace: ") + cudaGetErrorString(e));
  }
  w.big_cap = big_cap;
  w.big_min_degree = o.chunk_min_degree;
  w.ready = true;
  return PBG_OK;
}

void bfs_free_workspace(pbg_graph* g) {
  BfsWorkspace& w = g->ws;
  for (int i = 0; i < 2; i++) {
    cudaFree(w.bm[i]);
    cudaFree(w.q[i]);
    cudaFree(w.qr[i]);
    w.qr[i] = nullptr;
    cudaFree(w.qbig[i]);
    w.bm[i] = nullptr;
    w.q[i] = nullptr;
    w.qbig[i] = nullptr;
  }
  cudaFree(w.ctrl);
  w.ctrl = nullptr;
  cudaFree(w.parent);
  cudaFree(w.level);
  w.parent = nullptr;
  w.level = nullptr;
  w.ready = false;
}

// Launches the persistent kernel on caller-provided state arrays (used by the
// allocation-free entry point in noalloc.cu; the handle path above builds the
// same arguments from its workspace).
int bfs_launch_on(const BfsOnArgs& r, const pbg_bfs_opts& o, int num_sms, cudaStream_t s) {
  BfsArgs a;
  a.offsets = r.offsets;
  a.edges = r.edges;
  a.iso = r.iso;
  a.parent = r.parent;
  a.level = r.level;
  a.bm0 = r.bm0;
  a.bm1 = r.bm1;
  a.q0 = r.q0;
  a.q1 = r.q1;
  a.qr0 = r.qr0;
  a.qr1 = r.qr1;
  a.qb0 = r.qb0;
  a.qb1 = r.qb1;
  a.ctrl = r.ctrl;
  a.m = r.m;
  a.n = r.n;
  a.nwords = r.nwords;
  a.big_cap = r.big_cap;
  a.src = r.src;
  a.alpha = o.alpha;
  a.beta = o.beta;
  a.policy = o.direction;
  a.chunk_deg = o.chunk_min_degree;
  a.symmetric = r.symmetric;
  switch (o.parent_mode) {
    case PBG_PARENT_ANY: return launch_mode<MODE_ANY>(a, (int)o.block_threads, num_sms, s);
    case PBG_PARENT_MIN: return launch_mode<MODE_MIN>(a, (int)o.block_threads, num_sms, s);
    default: return launch_mode<MODE_MAX>(a, (int)o.block_threads, num_sms, s);
  }
}

int bfs_launch(pbg_graph* g, uint32_t src, const pbg_bfs_opts& o, uint32_t* d_parent, uint32_t* d_level,
               cudaStream_t s) {
  if (o.parent_mode > PBG_PARENT_MAX) return fail(PBG_ERR_ARG, "unknown parent_mode");
  if (o.direction > PBG_DIR_BOTTOMUP) return fail(PBG_ERR_ARG, "unknown direction policy");
  if (o.direction == PBG_DIR_BOTTOMUP && !(g->flags & PBG_GRAPH_SYMMETRIC))
    return fail(PBG_ERR_ARG, "bottom-up needs a symmetric graph");
  if (o.block_threads != 256 && o.block_threads != 512 && o.block_threads != 1024)
    return fail(PBG_ERR_ARG, "block_threads must be 256, 512 or 1024");
  if (o.chunk_min_degree < 1) return fail(PBG_ERR_ARG, "chunk_min_degree must be >= 1");
  int rc = bfs_ensure_workspace(g, o);
  if (rc) return rc;
  BfsWorkspace& w = g->ws;
  BfsArgs a;
  a.offsets = g->d_offsets;
  a.edges = g->d_edges;
  a.iso = g->d_iso;
  a.parent = d_parent;
  a.level = d_level;
  a.bm0 = w.bm[0];
  a.bm1 = w.bm[1];
  a.q0 = w.q[0];
  a.q1 = w.q[1];
  a.qr0 = w.qr[0];
  a.qr1 = w.qr[1];
  a.qb0 = w.qbig[0];
  a.qb1 = w.qbig[1];
  a.ctrl = w.ctrl;
  a.m = g->m;
  a.n = g->n;
  a.nwords = g->nwords;
  a.big_cap = w.big_cap;
  a.src = src;
  a.alpha = o.alpha;
  a.beta = o.beta;
  a.policy = o.direction;
  a.chunk_deg = o.chunk_min_degree;
  a.symmetric = (g->flags & PBG_GRAPH_SYMMETRIC) ? 1u : 0u;
  PBG_CUDA(cudaMemsetAsync(w.ctrl, 0, sizeof(BfsCtrl), s));
  PBG_CUDA(cudaEventRecord(w.ev0, s));
  if (g->max_degree < o.chunk_min_degree) {  // every list short: no chunk queue (bfs_lean)
    switch (o.parent_mode) {
      case PBG_PARENT_ANY: rc = launch_lean<MODE_ANY>(a, g->num_sms, s); break;
      case PBG_PARENT_MIN: rc = launch_lean<MODE_MIN>(a, g->num_sms, s); break;
      default: rc = launch_lean<MODE_MAX>(a, g->num_sms, s); break;
    }
  } else {
    switch (o.parent_mode) {
      case PBG_PARENT_ANY: rc = launch_mode<MODE_ANY>(a, (int)o.block_threads, g->num_sms, s); break;
      case PBG_PARENT_MIN: rc = launch_mode<MODE_MIN>(a, (int)o.block_threads, g->num_sms, s); break;
      default: rc = launch_mode<MODE_MAX>(a, (int)o.block_threads, g->num_sms, s); break;
    }
  }
  if (rc) return rc;
  PBG_CUDA(cudaEventRecord(w.ev1, s));
  g->stats_pending = true;
  return PBG_OK;
}

int bfs_read_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count) {
  if (!g->ws.ready) return fail(PBG_ERR_STATE, "no BFS has run on this graph");
  int rc = bfs_read_stats(g, nullptr);
  if (rc && rc != PBG_ERR_TIMEOUT && rc != PBG_ERR_STATE) return rc;
  BfsCtrl* c = new BfsCtrl;
  cudaError_t e = cudaMemcpy(c, g->ws.ctrl, sizeof(BfsCtrl), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "trace copy");
  }
  uint32_t nl = std::min<uint32_t>(c->levels, PBG_TRACE_LEVELS);
  uint32_t k = std::min(nl, cap);
  for (uint32_t L = 0; L < k; L++) {
    out[L].level = L;
    out[L].bottom_up = c->t_bu[L];
    out[L].frontier = c->t_nf[L];
    out[L].frontier_degree = c->t_deg[L];
    out[L].ms = (c->t_ns[L + 1] - c->t_ns[L]) * 1e-6;
  }
  if (count) *count = k;
  delete c;
  return PBG_OK;
}

int bfs_read_stats(pbg_graph* g, pbg_bfs_stats* st) {
  if (!g->ws.ready) return fail(PBG_ERR_STATE, "no BFS has run on this graph");
  if (g->stats_pending) {
    BfsCtrl c;
    PBG_CUDA(cudaEventSynchronize(g->ws.ev1));
    PBG_CUDA(cudaMemcpy(&c, g->ws.ctrl, sizeof(BfsCtrl), cudaMemcpyDeviceToHost));
    pbg_bfs_stats& s = g->last;
    s.levels = c.levels;
    s.topdown_levels = c.td_levels;
    s.bottomup_levels = c.bu_levels;
    s.error = c.sync.error;
    s.visited = c.visited;
    s.edges_reached = c.edges_reached;
    s.bottomup_mask = c.bu_mask;
    float ms = 0.f;
    PBG_CUDA(cudaEventElapsedTime(&ms, g->ws.ev0, g->ws.ev1));
    s.device_ms = ms;
    s.init_ms = (c.levels > 0 && c.t_ns[0] > c.t_start) ? (float)((c.t_ns[0] - c.t_start) * 1e-6) : 0.f;
    s.kernel_ms = (c.t_end > c.t_start) ? (float)((c.t_end - c.t_start) * 1e-6) : 0.f;
    g->stats_pending = false;
  }
  if (st) *st = g->last;
  if (g->last.error & ERR_BARRIER_TIMEOUT) return fail(PBG_ERR_TIMEOUT, "BFS: a grid barrier wait ran out");
  if (g->last.error) return fail(PBG_ERR_STATE, "BFS: device error word set");
  return PBG_OK;
}

}  // namespace pbg
