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
//   planes  u64   MS_PLANES x n ring: the bits found at each of the last
//                 levels (plane of level L = frontier of level L); every few
//                 levels a flush expands them into the level rows, one byte
//                 per 32-vertex piece of a row, instead of each level writing
//                 scattered bytes
//   q0/q1   u32   queue of the frontier, kept only after a sparse push level
//   qb0/qb1 uint4 same for vertices with degree >= big_min_degree, in
//                 CHUNK-edge pieces (v, begin, end, first chunk)
//   levels  u8    [k][n], source-major
// Per graph: the pull chunk table (the tails of lists longer than
// MS_PULL_SERIAL in MS_PULL_CHUNK-edge pieces), shared by every job on it.
//
// Each level every job independently runs one of
//   pull (bottom-up): every v not yet reached by all the frontier's sources
//     ORs its neighbours' frontier masks, stopping once every missing live
//     bit is found (the bit-parallel form of edge_map_dense,
//     common/ligraLight.h:87-112); long lists are finished chunk by chunk by
//     all warps after a grid barrier;
//   sparse push (top-down, small frontiers): every frontier vertex u ORs
//     fr[u] & ~vis[v] into the next mask of each neighbour v with atomicOr;
//     the first writer queues v (edge_map_sparse, ligraLight.h:70-85); a
//     second phase folds the new bits into vis and writes the levels;
//   dense push (large frontiers): the frontier read in vertex order pushes
//     its whole masks with 64-bit reductions (no return value, no checks, no
//     queue); a dense fold then drops the bits each vertex had,
// chosen per job from its frontier out-degree against the out-degree of the
// vertices not yet reached by every source (decide).  Pull and dense push
// produce a dense frontier: only its size, out-degree and source bits are
// counted (per block, in shared memory), and a sparse push that follows reads
// it in vertex order.  Work of all jobs in a level is spread over all warps of
// the grid through a prefix sum of per-job tile counts, so graphs of uneven
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
constexpr uint32_t CHUNK = 256;  // edges per piece of a big-queue entry
constexpr unsigned long long BIG_SHIFT = 40;
constexpr unsigned long long BIG_MASK = (1ull << BIG_SHIFT) - 1;
enum : uint32_t { M_DONE = 0, M_PULL = 1, M_PUSH = 2, M_DPUSH = 3 };

struct MsParams {
  uint32_t policy, big_deg;
};

// ------------------------------------------------------------- source masks
// A job's masks are W 64-bit words per vertex (64 W sources), stored
// vertex-major (word i of vertex v at v * W + i): one vector load reads a
// vertex's mask (8, 16 or 32 bytes; sm_100 has 32-byte loads), one 32-byte
// sector and one cache lookup whatever W, so a job of 256 sources gathers
// its graph's neighbour masks for about the cost of one of 64.
template <int W>
struct Mask {
  unsigned long long w[W];
};

template <int W>
__device__ __forceinline__ Mask<W> mzero() {
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = 0;
  return m;
}
template <int W>
__device__ __forceinline__ Mask<W> mor(const Mask<W>& a, const Mask<W>& b) {
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = a.w[i] | b.w[i];
  return m;
}
template <int W>
__device__ __forceinline__ Mask<W> mandn(const Mask<W>& a, const Mask<W>& b) {  // a & ~b
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = a.w[i] & ~b.w[i];
  return m;
}
template <int W>
__device__ __forceinline__ bool many(const Mask<W>& a) {
  unsigned long long x = 0;
#pragma unroll
  for (int i = 0; i < W; i++) x |= a.w[i];
  return x != 0;
}
template <int W>
__device__ __forceinline__ bool meq(const Mask<W>& a, const Mask<W>& b) {
  unsigned long long x = 0;
#pragma unroll
  for (int i = 0; i < W; i++) x |= a.w[i] ^ b.w[i];
  return x == 0;
}
// every bit of need is in have
template <int W>
__device__ __forceinline__ bool mcov(const Mask<W>& have, const Mask<W>& need) {
  return !many(mandn(need, have));
}
template <int W>
__device__ __forceinline__ Mask<W> mld(const unsigned long long* p, size_t v) {
  Mask<W> m;
  if constexpr (W == 4) {  // one 32-byte load (the masks are 32-byte aligned)
    asm volatile("ld.global.v4.u64 {%0, %1, %2, %3}, [%4];"
                 : "=l"(m.w[0]), "=l"(m.w[1]), "=l"(m.w[2]), "=l"(m.w[3])
                 : "l"(p + v * 4));
  } else if constexpr (W == 2) {
    const ulonglong2 x = reinterpret_cast<const ulonglong2*>(p)[v];
    m.w[0] = x.x;
    m.w[1] = x.y;
  } else {
#pragma unroll
    for (int i = 0; i < W; i++) m.w[i] = p[v * W + i];
  }
  return m;
}
template <int W>
__device__ __forceinline__ Mask<W> mld_relaxed(const unsigned long long* p, size_t v) {
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = dev::ld_relaxed_u64(p + v * W + i);
  return m;
}
template <int W>
__device__ __forceinline__ void mst(unsigned long long* p, size_t v, const Mask<W>& m) {
  if constexpr (W == 4) {
    asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p + v * 4), "l"(m.w[0]), "l"(m.w[1]),
                 "l"(m.w[2]), "l"(m.w[3])
                 : "memory");
  } else if constexpr (W == 2) {
    reinterpret_cast<ulonglong2*>(p)[v] = make_ulonglong2(m.w[0], m.w[1]);
  } else {
#pragma unroll
    for (int i = 0; i < W; i++) p[v * W + i] = m.w[i];
  }
}
// atomicOr word by word; words of m that are 0 are read, not written.
// Returns the old mask.
template <int W>
__device__ __forceinline__ Mask<W> matomic_or(unsigned long long* p, size_t v, const Mask<W>& m) {
  Mask<W> o;
#pragma unroll
  for (int i = 0; i < W; i++)
    o.w[i] = m.w[i] ? atomicOr(p + v * W + i, m.w[i]) : dev::ld_relaxed_u64(p + v * W + i);
  return o;
}
// reduction (no return value) of the non-zero words
template <int W>
__device__ __forceinline__ void mred_or(unsigned long long* p, size_t v, const Mask<W>& m) {
#pragma unroll
  for (int i = 0; i < W; i++)
    if (m.w[i]) atomicOr(p + v * W + i, m.w[i]);
}
template <int W>
__device__ __forceinline__ Mask<W> mshfl(const Mask<W>& m, int src) {
  Mask<W> r;
#pragma unroll
  for (int i = 0; i < W; i++) r.w[i] = __shfl_sync(FULL, m.w[i], src);
  return r;
}
template <int W>
__device__ __forceinline__ Mask<W> warp_or(Mask<W> m) {
#pragma unroll
  for (int i = 0; i < W; i++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m.w[i] |= __shfl_xor_sync(FULL, m.w[i], o);
  return m;
}
template <int W>
__device__ __forceinline__ Mask<W> job_all(const MsJob& J) {
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = J.all[i];
  return m;
}

// Warp-collective append (as in bfs.cu); deg goes to a per-block shared
// accumulator of the job.  One-word jobs only: their sparse pushes queue the
// first writer of each target.
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

constexpr uint32_t SERIAL_MAX = MS_PULL_SERIAL;
constexpr int PCH_STEPS = MS_PULL_CHUNK / 32;
constexpr uint32_t NONE32 = 0xFFFFFFFFu;

// Per-block shared sums of one job for the frontier a dense level produces
// (no queue is written): vertices found, their out-degree, the out-degree of
// the ones now reached by every source, and the source bits found.  Flushed
// to the job's counters once per block and phase (flush_counts), so a level
// issues a few hundred global atomics, not one per tile.
template <int W>
struct Acc {
  unsigned long long* nf;
  unsigned long long* deg;
  unsigned long long* ddeg;
  unsigned long long* live;  // W words
};

template <int W>
__device__ __forceinline__ void acc_live(const Acc<W>& a, const Mask<W>& bits) {
#pragma unroll
  for (int i = 0; i < W; i++)
    if (bits.w[i]) atomicOr(a.live + i, bits.w[i]);
}

// Warp-collective: lanes with `found` add their vertex (degree deg; `full`
// = now reached by every source); `bits` is the OR of the lanes' new bits.
template <int W>
__device__ __forceinline__ void account_warp(bool found, bool full, uint32_t deg, const Mask<W>& bits,
                                             const Acc<W>& a) {
  const unsigned fm = __ballot_sync(FULL, found);
  if (fm == 0) return;
  unsigned long long d = found ? deg : 0u, dd = (found && full) ? deg : 0u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_xor_sync(FULL, d, o);
    dd += __shfl_xor_sync(FULL, dd, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(a.nf, (unsigned long long)__popc(fm));
    atomicAdd(a.deg, d);
    if (dd) atomicAdd(a.ddeg, dd);
    acc_live(a, bits);
  }
}

// Level bytes of one vertex: one store per new bit (scattered rows).
template <int W>
__device__ __forceinline__ void write_levels(uint8_t* levels, uint32_t n, uint32_t v, const Mask<W>& m,
                                             uint8_t lv) {
#pragma unroll
  for (int k = 0; k < W; k++) {
    unsigned long long bits = m.w[k];
    while (bits) {
      const int i = __ffsll((long long)bits) - 1;
      bits &= bits - 1;
      levels[(size_t)(64 * k + i) * n + v] = lv;
    }
  }
}

// Levels of a 32-vertex tile found at level lvl, for a job that writes its
// levels as it goes (J.direct; see MsJob): one store per row that any lane
// gained, each into a 32-byte piece of that row.  Jobs on planes leave them
// to the flushes.  Whole warp; v = the lane's vertex, wb = OR of the lanes'
// new bits.
template <int W>
__device__ __forceinline__ void tile_levels(const MsJob& J, uint32_t lvl, uint32_t v, const Mask<W>& nb,
                                            const Mask<W>& wb) {
  if (!J.direct) return;
#pragma unroll
  for (int k = 0; k < W; k++) {
    unsigned long long any = wb.w[k];
    while (any) {
      const int i = __ffsll((long long)any) - 1;
      any &= any - 1;
      if ((nb.w[k] >> i) & 1ull) J.levels[(size_t)(64 * k + i) * J.n + v] = (uint8_t)lvl;
    }
  }
}

// Pull for 32 consecutive vertices, one per lane.  `live` holds the source
// bits present in this level's frontier: only those can be found, so a
// vertex is done once it has every live bit (or never starts when it already
// has them).  Each lane ORs the frontier masks of its vertex's first
// MS_PULL_SERIAL neighbours, pull_step<W> at a time (independent loads),
// with that early exit; the rest of a longer list is left to
// pull_chunk_group, which runs after a grid barrier.  fnext is written for
// every vertex (the next frontier, dense); two-word jobs also write the
// frontier bitmap word of the tile (pull_chunk_group counts by it).  A warp
// pulls its tiles of a job (first, first + stride, ... < end) with the next
// tile's visited masks and offsets loaded while the current tile's lists are
// read.
template <int W>
__host__ __device__ constexpr int pull_step() {
  return W >= 4 ? 4 : 8;
}

template <int W>
struct PullHead {
  Mask<W> vv;
  uint32_t b, e;
};

// Per-warp shared state of a range walk (range_push).
template <int W>
struct RangeShared {
  uint32_t start[32];
  uint32_t begin[32];
  Mask<W> m[32];
};

template <int W>
__device__ __forceinline__ PullHead<W> pull_head(const MsJob& J, uint32_t tile, uint32_t end) {
  PullHead<W> h{job_all<W>(J), 0u, 0u};
  const uint32_t v = tile * 32 + (threadIdx.x & 31);
  if (tile < end && v < J.n) {
    h.vv = mld<W>(J.vis, v);
    h.b = __ldg(J.offsets + v);
    h.e = __ldg(J.offsets + v + 1);
  }
  return h;
}

template <int W>
__device__ void pull_tiles(const MsJob& J, uint32_t first, uint32_t stride, uint32_t end,
                           const unsigned long long* fcur, unsigned long long* fnext, uint32_t lvl,
                           const Mask<W>& live, const Acc<W>& a) {
  constexpr int STEP = pull_step<W>();
  const int lane = threadIdx.x & 31;
  const Mask<W> all = job_all<W>(J);
  PullHead<W> h = pull_head<W>(J, first, end);
  for (uint32_t tile = first; tile < end; tile += stride) {
    const PullHead<W> nh = pull_head<W>(J, tile + stride, end);
    const uint32_t v = tile * 32 + lane;
    const bool active = v < J.n;
    const Mask<W> vv = h.vv;
    const uint32_t b = h.b;
    const uint32_t e = mcov(vv, live) ? b : h.e;
    Mask<W> acc = mzero<W>();
    const uint32_t es = (e - b > SERIAL_MAX) ? b + SERIAL_MAX : e;
    // the list in aligned 4-edge groups, one 16-byte load each (positions
    // before b or from es on are masked): a quarter of the L1 requests of
    // one load per edge
    for (uint32_t j0 = (es > b) ? (b & ~3u) : es; j0 < es && !mcov(mor(acc, vv), live); j0 += STEP) {
      uint32_t u[STEP];
#pragma unroll
      for (int q = 0; q < STEP / 4; q++) {
        uint4 x = make_uint4(NONE32, NONE32, NONE32, NONE32);
        if (j0 + 4 * q < es) x = __ldg(reinterpret_cast<const uint4*>(J.edges + j0 + 4 * q));
        u[4 * q] = x.x;
        u[4 * q + 1] = x.y;
        u[4 * q + 2] = x.z;
        u[4 * q + 3] = x.w;
      }
#pragma unroll
      for (int i = 0; i < STEP; i++)
        if (j0 + i < b || j0 + i >= es) u[i] = NONE32;
      Mask<W> f[STEP];
#pragma unroll
      for (int i = 0; i < STEP; i++) f[i] = (u[i] != NONE32) ? mld<W>(fcur, u[i]) : mzero<W>();
#pragma unroll
      for (int i = 0; i < STEP; i++) acc = mor(acc, f[i]);
    }
    const Mask<W> nb = mandn(acc, vv);
    const bool found = active && many(nb);
    if (found) mst<W>(J.vis, v, mor(vv, nb));
    if (active) mst<W>(fnext, v, nb);
    if (W > 1) {
      const unsigned fw = __ballot_sync(FULL, found);
      if (lane == 0 && tile * 32 < J.n) J.fbits[tile] = fw;
    }
    const Mask<W> wb = warp_or(nb);
    if (many(wb)) {
      account_warp<W>(found, meq(mor(vv, nb), all), e - b, wb, a);
      tile_levels<W>(J, lvl, v, nb, wb);
    }
    h = nh;
  }
}

// Pull over 32 consecutive entries of the graph's pull chunk table (the
// tails of lists longer than MS_PULL_SERIAL).  Each lane checks one chunk's
// vertex; the warp then pulls, one after another, every chunk whose vertex
// still misses a live bit, 32 edges a step with MS_PULL_CHUNK / 32
// independent loads per lane, and the lane of the chunk keeps the bits
// found.  At the end all lanes claim their bits at once: several chunks of
// one vertex run on different warps, so new bits are claimed with atomicOr
// on vis (word by word; each bit has one claimer) and the vertex is counted
// by whoever first makes it part of the next frontier (one-word jobs: the
// first to make its next mask non-zero; two-word jobs: the first to set its
// bit in the frontier bitmap, which pull_tiles wrote for the level).
template <int W>
__device__ void pull_chunk_group(const MsJob& J, uint32_t group, const unsigned long long* fcur,
                                 unsigned long long* fnext, uint32_t lvl, const Mask<W>& live, const Acc<W>& a) {
  const int lane = threadIdx.x & 31;
  const uint32_t c = group * 32 + lane;
  uint4 ent = make_uint4(0, 0, 0, 0);
  Mask<W> have = live;
  if (c < J.npc) {
    ent = J.pchunks[c];
    have = mld_relaxed<W>(J.vis, ent.x);
  }
  unsigned mm = __ballot_sync(FULL, !mcov(have, live));
  if (mm == 0) return;
  Mask<W> mine = mzero<W>();
  uint32_t prev_v = NONE32;
  Mask<W> prev_have = mzero<W>();
  while (mm) {
    const int l = __ffs(mm) - 1;
    mm &= mm - 1;
    const uint32_t v = __shfl_sync(FULL, ent.x, l);
    const uint32_t cb = __shfl_sync(FULL, ent.y, l);
    const uint32_t ce = __shfl_sync(FULL, ent.z, l);
    Mask<W> h = mshfl(have, l);
    if (v == prev_v) h = mor(h, prev_have);  // bits this warp found in the vertex's earlier chunks
    if (mcov(h, live)) continue;             // warp-uniform
    uint32_t u[PCH_STEPS];
#pragma unroll
    for (int i = 0; i < PCH_STEPS; i++) {
      const uint32_t j = cb + i * 32 + lane;
      u[i] = (j < ce) ? __ldg(J.edges + j) : NONE32;
    }
    Mask<W> acc = mzero<W>();
#pragma unroll
    for (int i = 0; i < PCH_STEPS; i++)
      if (u[i] != NONE32) acc = mor(acc, mld<W>(fcur, u[i]));
    const Mask<W> nb = mandn(warp_or(acc), h);
    if (lane == l) mine = nb;
    prev_v = v;
    prev_have = mor(h, nb);
  }
  bool first = false, full = false;
  Mask<W> nw = mzero<W>();
  if (many(mine)) {
    const uint32_t v = ent.x;
    const Mask<W> old = matomic_or<W>(J.vis, v, mine);
    nw = mandn(mine, old);
    if (many(nw)) {
      if (W == 1) {
        first = atomicOr(fnext + v, nw.w[0]) == 0;
      } else {
        mred_or<W>(fnext, v, nw);
        const uint32_t bit = 1u << (v & 31);
        first = (atomicOr(J.fbits + v / 32, bit) & bit) == 0;
      }
      full = meq(mor(old, mine), job_all<W>(J));
      if (J.direct) write_levels<W>(J.levels, J.n, v, nw, (uint8_t)lvl);
    }
  }
  const unsigned fm = __ballot_sync(FULL, first);
  unsigned long long d = first ? ent.w : 0u, dd = full ? ent.w : 0u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_xor_sync(FULL, d, o);
    dd += __shfl_xor_sync(FULL, dd, o);
  }
  const Mask<W> bits = warp_or(nw);
  if (lane == 0) {
    if (fm) {
      atomicAdd(a.nf, (unsigned long long)__popc(fm));
      atomicAdd(a.deg, d);
    }
    if (dd) atomicAdd(a.ddeg, dd);
    acc_live(a, bits);
  }
}

// Push steps.  PM_SPARSE (one-word jobs, small frontiers): the bits a
// target lacks go in with atomicOr and the first writer of the level queues
// it (sparse_push_run).  PM_DENSE (large frontiers): the whole mask goes into
// each neighbour's next mask with reductions (no return value, no visited
// check, no queueing); fold_tiles then removes the bits a vertex already had.
// PM_CHECKED (two-word jobs' small frontiers): like PM_DENSE, but only the
// bits the target lacks are sent (read of its visited mask first), and
// nothing when it lacks none; fold_tiles then builds the frontier counts (a
// two-word first-writer test would need a 128-bit atomic).
enum : int { PM_SPARSE = 0, PM_DENSE = 1, PM_CHECKED = 2 };

// Sparse push of SP_RUN edges per lane (edge index NONE32 = none), with the
// SP_RUN loads of each step independent: the edges, then the neighbours'
// visited masks, then the claims (atomicOr of the bits v lacks; the first
// writer of the level queues v), then the winners' degrees; then one warp
// append per step.
constexpr int SP_RUN = 4;

__device__ __forceinline__ void sparse_push_run(const MsJob& J, unsigned long long* fnext, LevelSlot* out,
                                                uint32_t* qout, uint4* qbout, const uint32_t* jj,
                                                const Mask<1>* ff, uint32_t big_deg, unsigned long long* s_deg) {
  uint32_t u[SP_RUN];
#pragma unroll
  for (int s2 = 0; s2 < SP_RUN; s2++) u[s2] = (jj[s2] != NONE32) ? __ldg(J.edges + jj[s2]) : NONE32;
  unsigned long long vv[SP_RUN];
#pragma unroll
  for (int s2 = 0; s2 < SP_RUN; s2++) vv[s2] = (u[s2] != NONE32) ? J.vis[u[s2]] : ~0ull;
  bool win[SP_RUN];
#pragma unroll
  for (int s2 = 0; s2 < SP_RUN; s2++) {
    const unsigned long long mb = ff[s2].w[0] & ~vv[s2];
    // first writer of this level: the target plane may still hold bits of an
    // older level, all of them already in vis
    win[s2] = mb != 0 && (atomicOr(fnext + u[s2], mb) & ~vv[s2]) == 0;
  }
  uint32_t b[SP_RUN], e[SP_RUN];
#pragma unroll
  for (int s2 = 0; s2 < SP_RUN; s2++) {
    b[s2] = e[s2] = 0;
    if (win[s2]) {
      b[s2] = __ldg(J.offsets + u[s2]);
      e[s2] = __ldg(J.offsets + u[s2] + 1);
    }
  }
#pragma unroll
  for (int s2 = 0; s2 < SP_RUN; s2++) ms_emit(J, out, qout, qbout, win[s2], u[s2], b[s2], e[s2], ~0ull, big_deg, s_deg);
}

// RUN edges per lane of a reduction push (PM_DENSE or PM_CHECKED), the RUN
// edge loads (and visited-mask loads) of a step independent.
template <int PM, int W, int RUN>
__device__ __forceinline__ void red_push_run(const MsJob& J, unsigned long long* fnext, const uint32_t* jj,
                                             const Mask<W>* ff) {
  uint32_t u[RUN];
#pragma unroll
  for (int s2 = 0; s2 < RUN; s2++) u[s2] = (jj[s2] != NONE32) ? __ldg(J.edges + jj[s2]) : NONE32;
  if (PM == PM_CHECKED) {
    Mask<W> vv[RUN];
#pragma unroll
    for (int s2 = 0; s2 < RUN; s2++) vv[s2] = (u[s2] != NONE32) ? mld<W>(J.vis, u[s2]) : ff[s2];
#pragma unroll
    for (int s2 = 0; s2 < RUN; s2++)
      if (u[s2] != NONE32) mred_or<W>(fnext, u[s2], mandn(ff[s2], vv[s2]));
  } else {
#pragma unroll
    for (int s2 = 0; s2 < RUN; s2++)
      if (u[s2] != NONE32) mred_or<W>(fnext, u[s2], ff[s2]);
  }
}

template <int PM, int W>
__host__ __device__ constexpr int push_run() {
  return PM == PM_SPARSE ? SP_RUN : (PM == PM_CHECKED || W >= 4) ? 4 : 8;
}

// Push over a tile of 32 frontier vertices: 32 consecutive vertices (the
// frontier read in vertex order, FROM_QUEUE false; lists capped at
// MS_PULL_SERIAL, the tails come from the pull chunk table, vchunk_push) or
// 32 entries of the frontier queue (lists shorter than the big-vertex
// threshold).  The warp walks the tile's lists as one range of positions:
// each lane takes RUN consecutive positions, finds the owner of the first by
// binary search over the per-vertex starts in shared memory and steps to the
// next owner as positions cross its start (vertex-order lists are contiguous
// in the CSR, so those edge loads are nearly coalesced).
template <int PM, bool FROM_QUEUE, int W>
__device__ void range_push(const MsJob& J, uint32_t tile, unsigned long long nq, const uint32_t* qin,
                           const unsigned long long* fcur, unsigned long long* fnext, RangeShared<W>& sh,
                           LevelSlot* out, uint32_t* qout, uint4* qbout, uint32_t big_deg,
                           unsigned long long* s_deg) {
  static_assert(PM != PM_SPARSE || W == 1, "queued sparse pushes are one-word only");
  constexpr int RUN = push_run<PM, W>();
  const int lane = threadIdx.x & 31;
  Mask<W> f = mzero<W>();
  uint32_t b = 0, e = 0;
  if (FROM_QUEUE) {
    const unsigned long long idx = (unsigned long long)tile * 32 + lane;
    if (idx < nq) {
      const uint32_t u = qin[idx];
      f = mld<W>(fcur, u);
      b = __ldg(J.offsets + u);
      e = __ldg(J.offsets + u + 1);
    }
  } else {
    const uint32_t v = tile * 32 + lane;
    if (v < J.n) {
      f = mld<W>(fcur, v);
      if (many(f)) {
        b = __ldg(J.offsets + v);
        e = __ldg(J.offsets + v + 1);
      }
    }
  }
  const uint32_t d = FROM_QUEUE ? e - b : min(e - b, SERIAL_MAX);
  uint32_t x = d;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  const uint32_t total = __shfl_sync(FULL, x, 31);
  if (total == 0) return;  // warp-uniform
  sh.start[lane] = x - d;
  sh.begin[lane] = b;
  sh.m[lane] = f;
  __syncwarp();
  for (uint32_t base = 0; base < total; base += 32 * RUN) {
    const uint32_t p0 = base + lane * RUN;
    int own = 0;
    uint32_t nxt = total;
    if (p0 < total) {
#pragma unroll
      for (int step = 16; step > 0; step >>= 1)
        if (sh.start[own + step] <= p0) own += step;
      nxt = (own < 31) ? sh.start[own + 1] : total;
    }
    uint32_t jj[RUN];
    Mask<W> ff[RUN];
#pragma unroll
    for (int s2 = 0; s2 < RUN; s2++) {
      const uint32_t ps = p0 + s2;
      jj[s2] = NONE32;
      ff[s2] = mzero<W>();
      if (ps < total) {
        while (ps >= nxt) {
          own++;
          nxt = (own < 31) ? sh.start[own + 1] : total;
        }
        jj[s2] = sh.begin[own] + (ps - sh.start[own]);
        ff[s2] = sh.m[own];
      }
    }
    if constexpr (PM == PM_SPARSE)
      sparse_push_run(J, fnext, out, qout, qbout, jj, ff, big_deg, s_deg);
    else
      red_push_run<PM, W, RUN>(J, fnext, jj, ff);
  }
  __syncwarp();
}

// Push of one chunk [cb, ce) of a frontier vertex with mask f, by the whole
// warp, 32 * RUN edges a step.
template <int PM, int W>
__device__ __forceinline__ void chunk_push(const MsJob& J, uint32_t cb, uint32_t ce, const Mask<W>& f,
                                           unsigned long long* fnext, LevelSlot* out, uint32_t* qout,
                                           uint4* qbout, uint32_t big_deg, unsigned long long* s_deg) {
  constexpr int RUN = (PM == PM_DENSE && W < 4) ? PCH_STEPS : 4;
  const int lane = threadIdx.x & 31;
  for (uint32_t j0 = cb; j0 < ce; j0 += 32 * RUN) {
    uint32_t jj[RUN];
    Mask<W> ff[RUN];
#pragma unroll
    for (int i = 0; i < RUN; i++) {
      const uint32_t j = j0 + i * 32 + lane;
      jj[i] = (j < ce) ? j : NONE32;
      ff[i] = f;
    }
    if constexpr (PM == PM_SPARSE)
      sparse_push_run(J, fnext, out, qout, qbout, jj, ff, big_deg, s_deg);
    else
      red_push_run<PM, W, RUN>(J, fnext, jj, ff);
  }
}

// Push of list tails: 32 entries of the pull chunk table per warp; every
// chunk whose vertex is in the frontier is pushed by the whole warp.
template <int PM, int W>
__device__ void vchunk_push(const MsJob& J, uint32_t group, const unsigned long long* fcur, unsigned long long* fnext,
                            LevelSlot* out, uint32_t* qout, uint4* qbout, uint32_t big_deg,
                            unsigned long long* s_deg) {
  const int lane = threadIdx.x & 31;
  const uint32_t c = group * 32 + lane;
  uint4 ent = make_uint4(0, 0, 0, 0);
  Mask<W> f = mzero<W>();
  if (c < J.npc) {
    ent = J.pchunks[c];
    f = mld<W>(fcur, ent.x);
  }
  unsigned mm = __ballot_sync(FULL, many(f));
  while (mm) {
    const int l = __ffs(mm) - 1;
    mm &= mm - 1;
    const uint32_t cb = __shfl_sync(FULL, ent.y, l);
    const uint32_t ce = __shfl_sync(FULL, ent.z, l);
    chunk_push<PM, W>(J, cb, ce, mshfl(f, l), fnext, out, qout, qbout, big_deg, s_deg);
  }
}

// Push of the CHUNK-edge pieces c0 .. c1 - 1 of big frontier vertices (the
// big queue): one binary search for the entry owning c0, then forward.
template <int PM, int W>
__device__ void qchunk_push(const MsJob& J, uint32_t c0, uint32_t c1, const uint4* qbin, uint32_t nbig,
                            const unsigned long long* fcur, unsigned long long* fnext, LevelSlot* out,
                            uint32_t* qout, uint4* qbout, uint32_t big_deg, unsigned long long* s_deg) {
  uint32_t lo = 0, hi = nbig - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (qbin[mid].w <= c0)
      lo = mid;
    else
      hi = mid - 1;
  }
  uint4 ent = qbin[lo];
  uint32_t next_first = (lo + 1 < nbig) ? qbin[lo + 1].w : 0xFFFFFFFFu;
  Mask<W> f = mld<W>(fcur, ent.x);
  for (uint32_t c = c0; c < c1; c++) {
    while (c >= next_first) {
      lo++;
      ent = qbin[lo];
      next_first = (lo + 1 < nbig) ? qbin[lo + 1].w : 0xFFFFFFFFu;
      f = mld<W>(fcur, ent.x);
    }
    const uint32_t cb = ent.y + (c - ent.w) * CHUNK;
    chunk_push<PM, W>(J, cb, min(ent.z, cb + CHUNK), f, fnext, out, qout, qbout, big_deg, s_deg);
  }
}

// Fold of a level's new plane, 32 consecutive vertices per warp, after a
// dense push (or a push into a plane still holding an older level): each
// mask loses the bits its vertex already had (reductions and older levels),
// the rest go into vis.  COUNT: the level built no queue, so the frontier's
// size and out-degree are counted here.  A warp folds its tiles (first,
// first + stride, ... < end) with every load of the next tile issued before
// the current one is worked.
template <int W>
struct FoldHead {
  Mask<W> x, vv;
  uint32_t b, e;
};

template <int W>
__device__ __forceinline__ FoldHead<W> fold_head(const MsJob& J, const unsigned long long* fnext, uint32_t tile,
                                                 uint32_t end) {
  FoldHead<W> h{mzero<W>(), mzero<W>(), 0u, 0u};
  const uint32_t v = tile * 32 + (threadIdx.x & 31);
  if (tile < end && v < J.n) {
    h.x = mld<W>(fnext, v);
    h.vv = mld<W>(J.vis, v);
    h.b = __ldg(J.offsets + v);
    h.e = __ldg(J.offsets + v + 1);
  }
  return h;
}

template <bool COUNT, int W>
__device__ void fold_tiles(const MsJob& J, uint32_t first, uint32_t stride, uint32_t end, unsigned long long* fnext,
                           uint32_t lvl, const Acc<W>& a) {
  const int lane = threadIdx.x & 31;
  const Mask<W> all = job_all<W>(J);
  FoldHead<W> h = fold_head<W>(J, fnext, first, end);
  for (uint32_t tile = first; tile < end; tile += stride) {
    const FoldHead<W> nh = fold_head<W>(J, fnext, tile + stride, end);
    const uint32_t v = tile * 32 + lane;
    const Mask<W> nb = mandn(h.x, h.vv);
    if (v < J.n) {
      if (!meq(nb, h.x)) mst<W>(fnext, v, nb);
      if (many(nb)) mst<W>(J.vis, v, mor(h.vv, nb));
    }
    const Mask<W> wb = warp_or(nb);
    if (many(wb)) {
      tile_levels<W>(J, lvl, v, nb, wb);
      const bool full = many(nb) && meq(mor(h.vv, nb), all);
      if (COUNT) {
        account_warp<W>(many(nb), full, h.e - h.b, wb, a);
      } else {
        unsigned long long dd = full ? h.e - h.b : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(FULL, dd, o);
        if (lane == 0) {
          acc_live(a, wb);
          if (dd) atomicAdd(a.ddeg, dd);
        }
      }
    }
    h = nh;
  }
}

// Flush: the planes of levels F..M (M - F < MS_PLANES <= 8) of 32
// consecutive vertices expanded into the level rows, word by word of the
// masks (64 rows each).  Each lane turns its vertex's planes into three
// bit-sliced code masks (bit b of row i = bit b of the level - F that found
// source i) and a mask of the sources it did not reach, and builds the bytes
// of four rows at a time in one 32-bit word: F + code where reached, and
// F + (255 - F) = 255 where not (each byte's sum stays below 256, so the
// additions of the four bytes never carry into each other); a 4 x 4 byte
// transpose across each group of four lanes (two shuffles) leaves every lane
// with four consecutive vertices of one row, so one 32-bit store per lane
// writes four 32-byte row pieces.  The first flush (F = 0) writes every row
// (255 = not reached yet): the rows need no other initialisation.  Later
// flushes merge only the bytes of vertices that gained the row's bit.
__device__ __forceinline__ uint32_t spread4(uint32_t x) {  // bit b of a nibble -> bit 8b
  return (x * 0x00204081u) & 0x01010101u;  // x + x<<7 + x<<14 + x<<21: no overlapping bits
}

// 4 x 4 byte transpose across each group of four lanes: lane p of a group
// ends with byte p of the group's four words.  s1/s2: the lane's selectors.
__device__ __forceinline__ uint32_t transpose4(uint32_t w, uint32_t s1, uint32_t s2) {
  const uint32_t a = __byte_perm(w, __shfl_xor_sync(FULL, w, 2), s1);
  return __byte_perm(a, __shfl_xor_sync(FULL, a, 1), s2);
}

// A warp flushes its tiles (first, first + stride, ... < end).  The loops
// over the four-row words stay rolled: the function is called out of line,
// and a smaller register footprint here keeps the kernel's other phases
// from spilling around the call.
template <int W>
__device__ __noinline__ void flush_tiles(const MsJob& J, uint32_t first, uint32_t stride, uint32_t end, uint32_t F,
                                         uint32_t M) {
  static_assert(MS_PLANES <= 8, "three code bits");
  const int lane = threadIdx.x & 31, p = lane & 3;
  const uint32_t s1 = (p < 2) ? 0x5410u : 0x3276u, s2 = (p & 1) ? 0x3715u : 0x6240u;
  const uint32_t fb = F * 0x01010101u, c255 = 255u - F;
  const bool wide_n = (J.n & 3) == 0, first_flush = F == 0;
  const size_t step = (size_t)4 * J.n;
  for (uint32_t tile = first; tile < end; tile += stride) {
    const uint32_t v = tile * 32 + lane;
    const bool active = v < J.n;
    const uint32_t vb = tile * 32 + (lane & ~3);
    const bool wide = wide_n && vb + 3 < J.n;
    for (int k = 0; k < W && 64u * k < J.k; k++) {
      unsigned long long any = 0, c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
      for (uint32_t q = 0; q < MS_PLANES; q++) {
        const unsigned long long m =
            (active && F + q <= M) ? J.planes[((size_t)((F + q) % MS_PLANES) * J.n + v) * W + k] : 0ull;
        any |= m;
        if (q & 1) c0 |= m;
        if (q & 2) c1 |= m;
        if (q & 4) c2 |= m;
      }
      const uint32_t nrows = min(64u, J.k - 64u * k);
      const unsigned long long rows = first_flush ? ~0ull : warp_or(Mask<1>{{any}}).w[0];
      uint8_t* dst = J.levels + (size_t)(64 * k + p) * J.n + vb;
#pragma unroll 1
      for (int half = 0; half < 2; half++) {
        const uint32_t xn = ~(uint32_t)(any >> (32 * half)), x0 = (uint32_t)(c0 >> (32 * half)),
                       x1 = (uint32_t)(c1 >> (32 * half)), x2 = (uint32_t)(c2 >> (32 * half));
        const uint32_t r32 = (uint32_t)(rows >> (32 * half));
#pragma unroll 1
        for (uint32_t w = 0; w < 8; w++, dst += step) {
          const uint32_t row0 = 32 * half + 4 * w;
          if (row0 >= nrows) break;  // warp-uniform
          const uint32_t sh = 4 * w;
          if (((r32 >> sh) & 0xFu) == 0) continue;  // warp-uniform: no lane gained these four rows
          const uint32_t un = spread4((xn >> sh) & 0xFu);  // sources not reached in these planes
          // reached bytes: F + code; the others F + (255 - F) = 255 (no carries between bytes)
          const uint32_t val = transpose4(spread4((x0 >> sh) & 0xFu) + (spread4((x1 >> sh) & 0xFu) << 1) +
                                              (spread4((x2 >> sh) & 0xFu) << 2) + fb + un * c255,
                                          s1, s2);
          if (first_flush) {
            if (row0 + p >= nrows) continue;
            if (wide) {
              *reinterpret_cast<uint32_t*>(dst) = val;
            } else {
#pragma unroll
              for (uint32_t b2 = 0; b2 < 4; b2++)
                if (vb + b2 < J.n) dst[b2] = (uint8_t)(val >> (8 * b2));
            }
            continue;
          }
          const uint32_t got = transpose4(~(un * 0xFFu), s1, s2);
          if (row0 + p >= nrows || got == 0) continue;
          if (wide) {
            uint32_t* d4 = reinterpret_cast<uint32_t*>(dst);
            *d4 = (got == 0xFFFFFFFFu) ? val : ((*d4 & ~got) | (val & got));
          } else {
#pragma unroll
            for (uint32_t b2 = 0; b2 < 4; b2++)
              if (vb + b2 < J.n && ((got >> (8 * b2)) & 0xFFu)) dst[b2] = (uint8_t)(val >> (8 * b2));
          }
        }
      }
    }
  }
}

// Direction for a job's next level.  With many sources a vertex rarely
// finds every missing bit early, so a pull reads about the out-edges of the
// vertices not yet reached by all sources (rem) and a push those of the
// frontier (fdeg); a pushed edge costs about PUSH_EDGE_COST pulled ones (a
// random 64-bit reduction, piling up on hubs, against a random load).  Pull
// when rem * alpha <= fdeg * beta * PUSH_EDGE_COST (the job's alpha and beta:
// 20 and 20 by default, or the graph's tuned ones).  A push whose frontier
// degree reaches n/2 runs dense.
constexpr unsigned long long PUSH_EDGE_COST = 2;

__device__ __forceinline__ uint32_t decide(const MsJob& J, const MsParams& p, unsigned long long nf,
                                           unsigned long long fdeg, unsigned long long done_deg) {
  if (nf == 0) return M_DONE;
  const uint32_t push = (fdeg >= J.n / 2) ? M_DPUSH : M_PUSH;
  if (p.policy == PBG_DIR_TOPDOWN || !J.symmetric) return push;
  if (p.policy == PBG_DIR_BOTTOMUP) return M_PULL;
  const unsigned long long rem = J.m - min(done_deg, J.m);
  return (rem * J.alpha <= fdeg * J.beta * PUSH_EDGE_COST) ? M_PULL : push;
}

// Work of a phase: batches of batch_tiles() tiles.  Warp w works batch w
// first; when there are more batches than warps, a warp that is done takes
// the next one from the grid-wide counter sync->work (asking for the one
// after while working).  The counter is never reset: a warp stops at its
// first grab past the end, so such a phase consumes exactly nbat - warps
// valid grabs plus one per warp = nbat counts, and every block knows where
// the next phase starts (wbase).  Fixed first batches keep the warps from all
// hitting the counter at once when a phase starts.
__device__ __forceinline__ unsigned long long batch_tiles(unsigned long long total, uint32_t nwarps) {
  return total >= 16ull * nwarps ? 4ull : 1ull;
}

__device__ __forceinline__ unsigned long long grab_batch(dev::GridSync* sync, unsigned long long wbase) {
  unsigned long long g = 0;
  if ((threadIdx.x & 31) == 0) g = atomicAdd(&sync->work, 1ull);
  return __shfl_sync(FULL, g, 0) - wbase;
}

template <int W>
__device__ __forceinline__ unsigned long long* plane_of(const MsJob& J, uint32_t level) {
  return J.planes + (size_t)(level % MS_PLANES) * J.n * W;
}

__device__ __forceinline__ void zero_words(unsigned long long* pl, unsigned long long words, unsigned long long tid,
                                           unsigned long long nth) {
  uint4* p4 = reinterpret_cast<uint4*>(pl);  // callers' arrays are 16-byte aligned when words is even
  if ((words & 1) == 0) {
    for (unsigned long long i = tid; i < words / 2; i += nth) p4[i] = make_uint4(0, 0, 0, 0);
  } else {
    for (unsigned long long i = tid; i < words; i += nth) pl[i] = 0;
  }
}

__device__ __forceinline__ uint32_t find_job(const unsigned long long* ends, uint32_t njobs, unsigned long long t) {
  uint32_t lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (ends[mid] > t)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// Per-block sums into the jobs' counters (after a __syncthreads); the shared
// sums restart at zero.
template <int W>
__device__ __forceinline__ void flush_counts(const MsJob* jobs, uint32_t njobs, uint32_t L, unsigned long long* s_nf,
                                             unsigned long long* s_deg, unsigned long long* s_ddeg,
                                             unsigned long long* s_lnext) {
  for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
    MsJobCtrl* c = jobs[j].ctrl;
    LevelSlot* o = &c->slot[(L + 1) % 3];
    if (s_nf[j]) atomicAdd(&o->nmain, s_nf[j]);
    if (s_deg[j]) atomicAdd(&o->deg, s_deg[j]);
#pragma unroll
    for (int k = 0; k < W; k++) {
      if (s_lnext[j * W + k]) atomicOr(&c->live[(L + 1) % 3][k], s_lnext[j * W + k]);
      s_lnext[j * W + k] = 0;
    }
    if (s_ddeg[j]) atomicAdd(&c->done_deg, s_ddeg[j]);
    s_nf[j] = 0;
    s_deg[j] = 0;
    s_ddeg[j] = 0;
  }
}

// Fold of a one-word sparse push into a clean plane, over the queue it
// built: the new masks go into vis (and the levels, for direct jobs), with
// the next frontier's live bits and reached out-degree summed per block.
__device__ void queue_fold(const MsJob& J, uint32_t L, const unsigned long long* fnext, unsigned long long tid,
                           unsigned long long nth, unsigned long long* s_lnext, unsigned long long* s_ddeg) {
  const uint32_t* qout = (L & 1) ? J.q0 : J.q1;
  const uint4* qbout = (L & 1) ? J.qb0 : J.qb1;
  const LevelSlot* o = &J.ctrl->slot[(L + 1) % 3];
  const unsigned long long onm = dev::ld_relaxed_u64(&o->nmain);
  const unsigned long long onb = min(dev::ld_relaxed_u64(&o->big) >> BIG_SHIFT, (unsigned long long)J.big_cap);
  unsigned long long seen = 0, dd = 0;
  for (unsigned long long i = tid; i < onm + onb; i += nth) {
    uint32_t v, b = 0, e = 0;
    if (i < onm) {
      v = qout[i];
    } else {
      const uint4 q = qbout[i - onm];
      v = q.x;
      b = q.y;
      e = q.z;
    }
    const unsigned long long nb = fnext[v];
    const unsigned long long vv = J.vis[v];
    J.vis[v] = vv | nb;
    if (J.direct) write_levels<1>(J.levels, J.n, v, Mask<1>{{nb}}, (uint8_t)(L + 1));
    seen |= nb;
    if ((vv | nb) == J.all[0]) {
      if (i < onm) {
        b = __ldg(J.offsets + v);
        e = __ldg(J.offsets + v + 1);
      }
      dd += e - b;
    }
  }
  seen = warp_or(Mask<1>{{seen}}).w[0];  // the next frontier's live source bits
#pragma unroll
  for (int o2 = 16; o2 > 0; o2 >>= 1) dd += __shfl_xor_sync(FULL, dd, o2);
  if ((threadIdx.x & 31) == 0) {
    if (seen) atomicOr(s_lnext, seen);
    if (dd) atomicAdd(s_ddeg, dd);
  }
}

template <int W>
__device__ __forceinline__ Mask<W> live_of(const unsigned long long* s_live, uint32_t j) {
  Mask<W> m;
#pragma unroll
  for (int i = 0; i < W; i++) m.w[i] = s_live[j * W + i];
  return m;
}

// One-word jobs: two blocks per SM (64 registers); two- and four-word jobs
// carry more mask registers and run one block per SM (128 registers; four-word
// jobs pull and push 4 edges a step instead of 8).
template <int W>
__global__ void __launch_bounds__(512, W == 1 ? 2 : 1) ms_persistent(const MsJob* __restrict__ jobs, uint32_t njobs, MsParams p,
                                                     dev::GridSync* sync) {
  __shared__ uint32_t s_mode[MS_MAX_JOBS];    // this level's mode (the previous one's in the decision)
  __shared__ uint8_t s_done[MS_MAX_JOBS];
  __shared__ uint8_t s_dense_in[MS_MAX_JOBS];  // the frontier has no queue (a dense level produced it)
  __shared__ uint8_t s_fold[MS_MAX_JOBS];      // phase B: 0 none, 1 queue fold, 2 dense fold (counted), 3 dense fold
  __shared__ uint8_t s_final[MS_MAX_JOBS];     // the job's last flush is done
  __shared__ uint32_t s_flushed[MS_MAX_JOBS];  // first level whose plane is not flushed yet
  __shared__ uint32_t s_flush_to[MS_MAX_JOBS];  // this level's flush: planes s_flushed .. s_flush_to
  __shared__ unsigned long long s_fl_end[MS_MAX_JOBS];  // prefix of flush tiles
  __shared__ unsigned long long s_tile_end[MS_MAX_JOBS];
  __shared__ unsigned long long s_pc_end[MS_MAX_JOBS];  // prefix of pull chunk groups
  __shared__ unsigned long long s_nmain[MS_MAX_JOBS];
  __shared__ uint32_t s_nbig[MS_MAX_JOBS];
  __shared__ unsigned long long s_live[MS_MAX_JOBS * W];  // source bits in the job's current frontier
  __shared__ unsigned long long s_nf[MS_MAX_JOBS];
  __shared__ unsigned long long s_deg[MS_MAX_JOBS];
  __shared__ unsigned long long s_ddeg[MS_MAX_JOBS];
  __shared__ unsigned long long s_lnext[MS_MAX_JOBS * W];
  __shared__ unsigned long long s_total;
  __shared__ unsigned long long s_pc_total;
  __shared__ unsigned long long s_fl_total;
  __shared__ int s_any_fold;
  __shared__ RangeShared<W> s_range[16];  // one per warp (512 threads)

  unsigned long long bar_epoch = 0;  // barriers passed (thread 0's count matters)
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
  const uint32_t gwarp = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;  // round-robin over blocks first
  const uint32_t nwarps = (uint32_t)(nth >> 5);

  // ---- init: visited masks and the first two planes to zero (on planes,
  // the first flush writes every level row)
  for (uint32_t j = 0; j < njobs; j++) {
    const MsJob& J = jobs[j];
    zero_words(J.vis, (unsigned long long)J.n * W, tid, nth);
    zero_words(J.planes, 2ull * J.n * W, tid, nth);  // planes of levels 0 and 1; the others the level before their use
    if (J.direct) {  // levels written as found: 255 until then
      const unsigned long long nb = (unsigned long long)J.k * J.n;
      uint4* lv4 = reinterpret_cast<uint4*>(J.levels);
      const uint4 ff = make_uint4(FULL, FULL, FULL, FULL);
      for (unsigned long long i = tid; i < nb / 16; i += nth) lv4[i] = ff;
      for (unsigned long long i = (nb / 16) * 16 + tid; i < nb; i += nth) J.levels[i] = 255;
    }
  }
  if (!dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch)) return;
  // ---- sources: one thread per job.
  if (blockIdx.x == 0) {
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const MsJob& J = jobs[j];
      LevelSlot* s0 = &J.ctrl->slot[0];
      for (uint32_t i = 0; i < J.k; i++) {
        const uint32_t s = J.srcs[i];
        const unsigned long long bit = 1ull << (i & 63);
        const Mask<W> old = mld<W>(J.planes, s);  // plane of level 0
        J.planes[(size_t)s * W + i / 64] |= bit;
        J.vis[(size_t)s * W + i / 64] |= bit;
        if (J.direct) J.levels[(size_t)i * J.n + s] = 0;
        J.ctrl->live[0][i / 64] |= bit;
        if (!many(old)) {
          // every source goes to the chunked queue, so level 0's few lists
          // are spread over many warps
          const uint32_t b = __ldg(J.offsets + s), e = __ldg(J.offsets + s + 1);
          const unsigned long long nch = (e - b + CHUNK - 1) / CHUNK;
          const unsigned long long slot = s0->big >> BIG_SHIFT;
          J.qb0[slot] = make_uint4(s, b, e, (uint32_t)(s0->big & BIG_MASK));
          s0->big += (1ull << BIG_SHIFT) | nch;
          s0->deg += e - b;
        }
      }
    }
  }
  for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
    s_mode[j] = M_PUSH;  // the sources form a queue
    s_done[j] = 0;
    s_dense_in[j] = 0;
    s_final[j] = 0;
    s_flushed[j] = 0;
    s_nf[j] = s_deg[j] = s_ddeg[j] = 0;
#pragma unroll
    for (int q = 0; q < W; q++) s_lnext[j * W + q] = 0;
  }
  bool ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);

  unsigned long long wbase = 0;  // work counter at the start of the current phase
  uint32_t L = 0;
  while (ok) {
    // ---- per-job decision (every block computes the same)
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const MsJob& J = jobs[j];
      // a frontier without a queue: after a pull or a dense push, and for
      // two-word jobs after any level but the sources' (they queue nothing)
      if (!s_done[j])
        s_dense_in[j] = (W > 1) ? (L > 0 ? 1 : 0) : ((s_mode[j] == M_PULL || s_mode[j] == M_DPUSH) ? 1 : 0);
      const LevelSlot* in = &J.ctrl->slot[L % 3];
      const unsigned long long nmain = dev::ld_relaxed_u64(&in->nmain);
      const unsigned long long big = dev::ld_relaxed_u64(&in->big);
      const unsigned long long fdeg = dev::ld_relaxed_u64(&in->deg);
      const uint32_t nbig = (uint32_t)(big >> BIG_SHIFT);
      uint32_t mode =
          s_done[j] ? M_DONE : decide(J, p, nmain + nbig, fdeg, dev::ld_relaxed_u64(&J.ctrl->done_deg));
      if (mode != M_DONE && (L + 1 >= 255 || nbig > J.big_cap || nmain > J.n)) {
        if (blockIdx.x == 0) atomicOr(&J.ctrl->error, L + 1 >= 255 ? MS_ERR_OVERFLOW : MS_ERR_QUEUE);
        mode = M_DONE;
      }
      if (blockIdx.x == 0 && !s_done[j] && L <= MS_TRACE_LEVELS) {
        J.ctrl->t_ns[L] = dev::globaltimer();
        if (mode != M_DONE && L < MS_TRACE_LEVELS) {
          J.ctrl->t_nf[L] = nmain + nbig;
          J.ctrl->t_deg[L] = fdeg;
          J.ctrl->t_pull[L] = mode == M_PULL ? 1u : (mode == M_DPUSH ? 2u : 0u);
        }
      }
      if (mode == M_DONE && !s_done[j]) {
        s_done[j] = 1;
        if (blockIdx.x == 0) J.ctrl->levels = L;
      }
      s_mode[j] = mode;
      s_nmain[j] = nmain;
      s_nbig[j] = nbig;
#pragma unroll
      for (int q = 0; q < W; q++) s_live[j * W + q] = dev::ld_relaxed_u64(&J.ctrl->live[L % 3][q]);
      const unsigned long long vt = (J.n + 31) / 32, ct = (J.npc + 31) / 32;
      if (mode == M_PULL)
        s_tile_end[j] = vt;
      else if ((mode == M_DPUSH || mode == M_PUSH) && s_dense_in[j])
        s_tile_end[j] = vt + ct;
      else if (mode == M_DPUSH || mode == M_PUSH)
        s_tile_end[j] = (nmain + 31) / 32 + (big & BIG_MASK);
      else
        s_tile_end[j] = 0;
      s_pc_end[j] = (mode == M_PULL) ? ct : 0;
      // flush planes s_flushed .. L when this level's target plane still
      // holds an unflushed one, or when the job has just ended
      bool fl = false;
      if (!s_final[j] && !J.direct) {
        if (mode == M_DONE) {
          fl = true;
          s_final[j] = 1;
        } else {
          fl = L + 1 >= MS_PLANES && L + 1 - MS_PLANES >= s_flushed[j];
        }
      }
      s_flush_to[j] = L;
      s_fl_end[j] = fl ? vt : 0;
      if (blockIdx.x == 0 && mode != M_DONE) {
        J.ctrl->slot[(L + 2) % 3] = LevelSlot{0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < W; q++) J.ctrl->live[(L + 2) % 3][q] = 0;
        if (mode == M_PULL)
          J.ctrl->pull_levels++;
        else
          J.ctrl->push_levels++;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long acc = 0, pacc = 0, facc = 0;
      for (uint32_t j = 0; j < njobs; j++) {
        acc += s_tile_end[j];
        s_tile_end[j] = acc;
        pacc += s_pc_end[j];
        s_pc_end[j] = pacc;
        facc += s_fl_end[j];
        s_fl_end[j] = facc;
      }
      s_total = acc;
      s_pc_total = pacc;
      s_fl_total = facc;
    }
    __syncthreads();
    const unsigned long long total = s_total;

    // ---- flush: the planes of levels s_flushed .. L into the level rows
    const unsigned long long fl_total = s_fl_total;
    if (fl_total) {
      for (unsigned long long t = gwarp; t < fl_total; t += nwarps) {
        // all of this warp's tiles of the job, then on past its end
        const uint32_t j = find_job(s_fl_end, njobs, t);
        const unsigned long long t0 = j ? s_fl_end[j - 1] : 0;
        const uint32_t lt = (uint32_t)(t - t0), end = (uint32_t)(s_fl_end[j] - t0);
        flush_tiles<W>(jobs[j], lt, nwarps, end, s_flushed[j], s_flush_to[j]);
        t += (unsigned long long)((end - 1 - lt) / nwarps) * nwarps;
      }
      ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
      for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x)
        if (s_fl_end[j] != (j ? s_fl_end[j - 1] : 0)) s_flushed[j] = s_flush_to[j] + 1;
      __syncthreads();
      if (!ok) break;
    }
    if (total == 0) break;

    // ---- phase A: all jobs' tiles over all warps (batches: first one per
    // warp fixed, the rest from the grid-wide counter; see grab_batch)
    {
      auto run = [&](unsigned long long t, unsigned long long tb_end) {
        while (t < tb_end) {
          const uint32_t j = find_job(s_tile_end, njobs, t);
          const unsigned long long t0 = j ? s_tile_end[j - 1] : 0;
          const uint32_t lt = (uint32_t)(t - t0);
          const MsJob& J = jobs[j];
          const unsigned long long* fcur = plane_of<W>(J, L);
          unsigned long long* fnext = plane_of<W>(J, L + 1);
          const uint32_t mode = s_mode[j];
          if (mode == M_PULL) {
            // the batch's tiles of this job in one pipelined run
            const unsigned long long stop = min(tb_end, s_tile_end[j]);
            pull_tiles<W>(J, lt, 1, (uint32_t)(stop - t0), fcur, fnext, L + 1, live_of<W>(s_live, j),
                       Acc<W>{&s_nf[j], &s_deg[j], &s_ddeg[j], &s_lnext[j * W]});
            t = stop;
            continue;
          }
          uint32_t* qout = (L & 1) ? J.q0 : J.q1;
          uint4* qbout = (L & 1) ? J.qb0 : J.qb1;
          LevelSlot* out = &J.ctrl->slot[(L + 1) % 3];
          const uint32_t vt = (J.n + 31) / 32;
          RangeShared<W>& sh = s_range[threadIdx.x >> 5];
          // two-word jobs have no queued sparse push: their small pushes are checked reductions
          constexpr int PMS = (W == 1) ? PM_SPARSE : PM_CHECKED;
          if (s_dense_in[j]) {  // the frontier in vertex order
            if (mode == M_DPUSH) {
              if (lt < vt)
                range_push<PM_DENSE, false, W>(J, lt, 0, nullptr, fcur, fnext, sh, out, qout, qbout, p.big_deg,
                                               &s_deg[j]);
              else
                vchunk_push<PM_DENSE, W>(J, lt - vt, fcur, fnext, out, qout, qbout, p.big_deg, &s_deg[j]);
            } else {
              if (lt < vt)
                range_push<PMS, false, W>(J, lt, 0, nullptr, fcur, fnext, sh, out, qout, qbout, p.big_deg,
                                          &s_deg[j]);
              else
                vchunk_push<PMS, W>(J, lt - vt, fcur, fnext, out, qout, qbout, p.big_deg, &s_deg[j]);
            }
          } else {  // the frontier queue
            const uint32_t* qin = (L & 1) ? J.q1 : J.q0;
            const uint4* qbin = (L & 1) ? J.qb1 : J.qb0;
            const uint32_t main_tiles = (uint32_t)((s_nmain[j] + 31) / 32);
            if (lt >= main_tiles) {
              // the run's chunks of this job's big queue together
              const unsigned long long stop = min(tb_end, s_tile_end[j]);
              const uint32_t c0 = lt - main_tiles, c1 = (uint32_t)(stop - t0) - main_tiles;
              if (mode == M_DPUSH)
                qchunk_push<PM_DENSE, W>(J, c0, c1, qbin, s_nbig[j], fcur, fnext, out, qout, qbout, p.big_deg,
                                         &s_deg[j]);
              else
                qchunk_push<PMS, W>(J, c0, c1, qbin, s_nbig[j], fcur, fnext, out, qout, qbout, p.big_deg,
                                    &s_deg[j]);
              t = stop;
              continue;
            }
            if (mode == M_DPUSH)
              range_push<PM_DENSE, true, W>(J, lt, s_nmain[j], qin, fcur, fnext, sh, out, qout, qbout, p.big_deg,
                                            &s_deg[j]);
            else
              range_push<PMS, true, W>(J, lt, s_nmain[j], qin, fcur, fnext, sh, out, qout, qbout, p.big_deg,
                                       &s_deg[j]);
          }
          t++;
        }
      };
      const unsigned long long wg = batch_tiles(total, nwarps);
      const unsigned long long nbat = (total + wg - 1) / wg;
      if (wg == 1) {  // small phase: tiles round-robin over the warps
        for (unsigned long long t = gwarp; t < total; t += nwarps) {
          const uint32_t j = find_job(s_tile_end, njobs, t);
          if (s_mode[j] == M_PULL) {  // all of this warp's tiles of the job, pipelined
            const MsJob& J = jobs[j];
            const unsigned long long t0 = j ? s_tile_end[j - 1] : 0;
            const uint32_t lt = (uint32_t)(t - t0), end = (uint32_t)(s_tile_end[j] - t0);
            pull_tiles<W>(J, lt, nwarps, end, plane_of<W>(J, L), plane_of<W>(J, L + 1), L + 1, live_of<W>(s_live, j),
                       Acc<W>{&s_nf[j], &s_deg[j], &s_ddeg[j], &s_lnext[j * W]});
            t += (unsigned long long)((end - 1 - lt) / nwarps) * nwarps;
            continue;
          }
          run(t, t + 1);
        }
      } else {
        run(gwarp * wg, min(gwarp * wg + wg, total));
        unsigned long long cur = nwarps + grab_batch(sync, wbase);
        while (cur < nbat) {
          const unsigned long long nxt = nwarps + grab_batch(sync, wbase);
          run(cur * wg, min(cur * wg + wg, total));
          cur = nxt;
        }
        wbase += nbat;
      }
    }
    // the plane of level L + 2 is used for the first time next level: zero it
    // now (from then on planes are reused and their old bits are in vis)
    if (L + 2 < MS_PLANES)
      for (uint32_t j = 0; j < njobs; j++)
        if (s_mode[j] != M_DONE) zero_words(plane_of<W>(jobs[j], L + 2), (unsigned long long)jobs[j].n * W, tid, nth);
    __syncthreads();
    flush_counts<W>(jobs, njobs, L, s_nf, s_deg, s_ddeg, s_lnext);
    ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
    if (!ok) break;

    // ---- phase A2: the tails of long lists of pull jobs, over all warps
    const unsigned long long pc_total = s_pc_total;
    if (pc_total) {
      auto run = [&](unsigned long long t, unsigned long long tb_end) {
        for (; t < tb_end; t++) {
          const uint32_t j = find_job(s_pc_end, njobs, t);
          const MsJob& J = jobs[j];
          pull_chunk_group<W>(J, (uint32_t)(t - (j ? s_pc_end[j - 1] : 0)), plane_of<W>(J, L), plane_of<W>(J, L + 1), L + 1,
                           live_of<W>(s_live, j), Acc<W>{&s_nf[j], &s_deg[j], &s_ddeg[j], &s_lnext[j * W]});
        }
      };
      const unsigned long long wg = batch_tiles(pc_total, nwarps);
      const unsigned long long nbat = (pc_total + wg - 1) / wg;
      if (wg == 1) {
        for (unsigned long long t = gwarp; t < pc_total; t += nwarps) run(t, t + 1);
      } else {
        run(gwarp * wg, min(gwarp * wg + wg, pc_total));
        unsigned long long cur = nwarps + grab_batch(sync, wbase);
        while (cur < nbat) {
          const unsigned long long nxt = nwarps + grab_batch(sync, wbase);
          run(cur * wg, min(cur * wg + wg, pc_total));
          cur = nxt;
        }
        wbase += nbat;
      }
      __syncthreads();
      flush_counts<W>(jobs, njobs, L, s_nf, s_deg, s_ddeg, s_lnext);
      ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
      if (!ok) break;
    }

    // ---- phase B: a push folds its new plane into vis: a one-word sparse
    // push into a clean plane over its queue, a dense push (or a sparse push
    // into a plane that still holds an older level) over every vertex
    // (fold_tiles); two-word pushes built no queue, so their fold counts the
    // frontier.
    if (threadIdx.x == 0) s_any_fold = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < njobs; j += blockDim.x) {
      const uint32_t mode = s_mode[j];
      const bool reused = L + 1 >= MS_PLANES;  // the target plane held level L + 1 - MS_PLANES
      uint8_t f = 0;
      if (mode == M_PUSH)
        f = (W > 1) ? 2 : (reused ? 3 : 1);
      else if (mode == M_DPUSH)
        f = 2;
      s_fold[j] = f;
      if (f) s_any_fold = 1;
    }
    __syncthreads();
    if (s_any_fold) {
      for (uint32_t j = 0; j < njobs; j++) {
        const MsJob& J = jobs[j];
        unsigned long long* fnext = plane_of<W>(J, L + 1);
        const uint8_t f = s_fold[j];
        const Acc<W> a{&s_nf[j], &s_deg[j], &s_ddeg[j], &s_lnext[j * W]};
        if constexpr (W == 1) {
          if (f == 1) queue_fold(J, L, fnext, tid, nth, &s_lnext[j], &s_ddeg[j]);
        }
        if (f == 2) {
          fold_tiles<true, W>(J, gwarp, nwarps, (J.n + 31) / 32, fnext, L + 1, a);
        } else if (f == 3) {
          fold_tiles<false, W>(J, gwarp, nwarps, (J.n + 31) / 32, fnext, L + 1, a);
        }
      }
      __syncthreads();
      flush_counts<W>(jobs, njobs, L, s_nf, s_deg, s_ddeg, s_lnext);
      ok = dev::grid_barrier(sync, MS_ERR_TIMEOUT, bar_epoch);
    }
    L++;
  }
}

std::mutex g_grid_mu;
int g_grid_dev[5] = {-1, -1, -1, -1, -1}, g_grid[5] = {0, 0, 0, 0, 0};  // by mask words (1, 2, 4)

const void* kernel_for(uint32_t words) {
  return words > 2 ? (const void*)ms_persistent<4>
                   : words > 1 ? (const void*)ms_persistent<2> : (const void*)ms_persistent<1>;
}

}  // namespace

int ms_full_grid(int num_sms, uint32_t words) {
  const int w = words > 2 ? 4 : words > 1 ? 2 : 1;
  std::lock_guard<std::mutex> lk(g_grid_mu);
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_grid_dev[w] != dev) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_for(w), 512, 0);
    if (e != cudaSuccess || per_sm < 1) return -1;
    g_grid[w] = per_sm * num_sms;
    g_grid_dev[w] = dev;
  }
  return g_grid[w];
}

int ms_launch(const MsJob* d_jobs, uint32_t njobs, const pbg_bfs_opts& o, dev::GridSync* d_sync, int num_sms,
              cudaStream_t s, int max_blocks, uint32_t words) {
  int grid = ms_full_grid(num_sms, words);
  if (grid < 1) return fail(PBG_ERR_CUDA, "multi-source kernel cannot be resident");
  if (max_blocks > 0 && max_blocks < grid) grid = max_blocks;
  MsParams p{o.direction, ms_big_degree(o)};
  void* params[] = {(void*)&d_jobs, &njobs, &p, &d_sync};
  PBG_CUDA(cudaLaunchCooperativeKernel(kernel_for(words), dim3(grid), dim3(512), params, 0, s));
  return PBG_OK;
}

}  // namespace pbg
