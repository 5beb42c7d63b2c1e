// mis.cu -- maximal independent set on a resident graph (sm_100a): the
// frontier engine of the BFS path reused for PBBS's maximalIndependentSet
// benchmark (benchmarks/maximalIndependentSet/bench/MIS.h:8).
//
// The set computed is the one serialMIS returns
// (maximalIndependentSet/serialMIS/MIS.C:33-47): vertices are taken in id
// order and v joins unless a vertex already in the set is among its
// neighbours (a self loop keeps v out).  That greedy set is the unique one
// in which
//     v is in  <=>  no out-neighbour u < v is in, and v has no self loop,
// and this rule can be evaluated in parallel rounds: v is decided OUT as soon
// as one earlier neighbour is IN, IN as soon as every earlier neighbour is
// OUT, and waits otherwise.  Decisions are final and correct whatever the
// order in which other vertices were decided, so threads may read flags that
// others are writing in the same round; the smallest undecided vertex always
// decides, so the rounds end.  The result is deterministic and bit-exact with
// serialMIS, and a valid maximal independent set on symmetric graphs (the
// test of MISCheck.C:39-66), the contract of the nondeterministic ndMIS
// (ndMIS/MIS.C:41-80) as well.
//
// One persistent cooperative launch: round 0 walks every vertex; an
// undecided vertex goes to the next round's queue with a cursor, the position
// of its first undecided earlier neighbour (everything before it is known to
// be out of the set), so no edge is read again once passed, and a walk stops
// at the step where it meets an undecided neighbour.  Each lane walks the
// first entries of its list itself (round 0: 8 entries, 2 loads a step: most
// walks end at their first or second entry, and wider steps only add L1
// requests; later rounds: 16 entries, 4 a step); a list still clear after
// those is walked on by the whole warp, 32 a step.  A queue entry carries (vertex, cursor,
// list end); each warp collects its requeued entries in shared memory and
// appends them with one atomic per WQ entries.  One grid barrier per round
// (bounded, device_util.cuh).  When the graph's lists are ascending (checked
// once per graph), a walk stops at the first neighbour above v.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "device_util.cuh"
#include "internal.cuh"

namespace pbg {
namespace {

using dev::FULL;
// Round 0 walks every list from its start: most walks end at the first or
// second entry.  Later rounds resume walks that already passed their first
// undecided neighbour and run longer, so they take wider steps and a longer
// lane share.
constexpr int MK = 2;                   // round 0: loads per lane per step
constexpr int MK_LATER = 4;             // later rounds
constexpr uint8_t UNDECIDED = 0, IN_SET = 1, OUT_SET = 2;
constexpr uint8_t MORE = 3;      // walk result: clear so far, list goes on past the lane's share
constexpr uint32_t LANE_SHARE = 8;        // round 0: entries a lane walks before the warp takes over
constexpr uint32_t LANE_SHARE_LATER = 16; // later rounds

struct MisArgs {
  const uint32_t* __restrict__ offsets;
  const uint32_t* __restrict__ edges;
  uint8_t* flags;
  uint32_t* q0;
  uint32_t* q1;
  uint2* c0;  // (cursor, list end) of each queue entry
  uint2* c1;
  BfsCtrl* ctrl;
  uint32_t n;
  uint32_t sorted;
};

// A neighbour's flag, through L1.  A flag changes once per call, from
// UNDECIDED to its final value (the kernel's fill and a grid barrier come
// before the first read, and the barrier's acquire leaves no older line in
// L1), so a line cached earlier in the round holds either the final value or
// an UNDECIDED that only makes the reader wait a round.  Hub flags, read by
// many lists on one SM, then come from L1 instead of L2: 28-34% faster on
// rMat than reading every flag from L2.
__device__ __forceinline__ uint8_t ld_flag(const uint8_t* p) {
  uint16_t v;
  asm volatile("ld.global.ca.u8 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
  return (uint8_t)v;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Lane-serial walk of v's list from position j, up to LS entries, MKS loads
// a step.
// Returns OUT_SET; UNDECIDED with *cur set to the first undecided earlier
// neighbour; IN_SET when the list is clear to its end (or to a larger
// neighbour in an ascending list); MORE with *cur at the first entry not
// walked when the share is clear and the list goes on.
template <uint32_t LS, int MKS>
__device__ __forceinline__ uint8_t walk_lane(const MisArgs& a, uint32_t v, uint32_t j, uint32_t e, uint32_t* cur) {
  const uint32_t end = min(e, j + LS);
  uint32_t first_wait = e;
  bool stop = false;
  for (; j < end; j += MKS) {
    uint32_t u[MKS];
#pragma unroll
    for (int i = 0; i < MKS; i++) u[i] = (j + i < end) ? __ldg(a.edges + j + i) : v + 1;
    uint8_t f[MKS];
#pragma unroll
    for (int i = 0; i < MKS; i++) f[i] = (u[i] < v) ? ld_flag(a.flags + u[i]) : OUT_SET;
#pragma unroll
    for (int i = 0; i < MKS; i++) {
      if (j + i >= end) break;
      if (u[i] == v || f[i] == IN_SET) return OUT_SET;  // a self loop, or an earlier neighbour in the set
      if (u[i] < v && f[i] == UNDECIDED && first_wait == e) first_wait = j + i;
      if (u[i] > v && a.sorted) stop = true;
    }
    // A step with an undecided neighbour ends the walk: the rest of the list
    // is read when that neighbour has decided (mostly OUT), not now, when
    // nearly everything is still undecided (round 0 would walk every list).
    if (stop || first_wait < e) break;
  }
  if (first_wait < e) {
    *cur = first_wait;
    return UNDECIDED;
  }
  if (!stop && end < e) {
    *cur = end;
    return MORE;
  }
  return IN_SET;
}

// Warp-cooperative walk of one long list (every lane calls it with the same
// v, j, e).
__device__ __forceinline__ uint8_t walk_warp(const MisArgs& a, uint32_t v, uint32_t j, uint32_t e, uint32_t* cur) {
  const int lane = threadIdx.x & 31;
  uint32_t first_wait = e;
  for (uint32_t j0 = j; j0 < e; j0 += 32) {
    const uint32_t p = j0 + lane;
    uint32_t u = v + 1;
    uint8_t f = OUT_SET;
    if (p < e) {
      u = __ldg(a.edges + p);
      if (u < v) f = ld_flag(a.flags + u);
    }
    const bool out = p < e && (u == v || f == IN_SET);
    if (__any_sync(FULL, out)) return OUT_SET;
    const unsigned w = __ballot_sync(FULL, p < e && u < v && f == UNDECIDED);
    if (w && first_wait == e) first_wait = j0 + __ffs(w) - 1;
    if (first_wait < e) break;  // as in walk_lane: resume at the first undecided neighbour
    if (a.sorted && __any_sync(FULL, p < e && u > v)) break;
  }
  if (first_wait < e) {
    *cur = first_wait;
    return UNDECIDED;
  }
  return IN_SET;
}

constexpr uint32_t WQ = 64;  // entries of a warp's requeue buffer in shared memory

// Appends a warp's buffered entries to the next round's queue (one atomic).
__device__ __forceinline__ void wq_flush(const uint32_t* wv, const uint2* wc, uint32_t nbuf, LevelSlot* out,
                                         uint32_t* qout, uint2* cout_) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
  uint32_t base = 0;
  if (lane == 0) base = (uint32_t)atomicAdd(&out->nmain, (unsigned long long)nbuf);
  base = __shfl_sync(FULL, base, 0);
  for (uint32_t i = lane; i < nbuf; i += 32) {
    qout[base + i] = wv[i];
    cout_[base + i] = wc[i];
  }
  __syncwarp();
}

// One queue entry per lane (valid when `have`): decide it or requeue it.
// Every lane walks its own list first (most walks end within a few
// entries); the lists still clear after a lane's share are walked by the
// whole warp, one after another.
template <uint32_t LS, int MKS>
__device__ __forceinline__ void decide(const MisArgs& a, uint32_t v, uint32_t j, uint32_t e, bool have,
                                       LevelSlot* out, uint32_t* qout, uint2* cout_,
                                       unsigned long long& in_count, uint32_t* wv, uint2* wc, uint32_t& nbuf) {
  const int lane = threadIdx.x & 31;
  uint8_t res = UNDECIDED;
  uint32_t cur = j;
  if (have) res = walk_lane<LS, MKS>(a, v, j, e, &cur);
  unsigned lm = __ballot_sync(FULL, res == MORE);
  while (lm) {
    const int l = __ffs(lm) - 1;
    lm &= lm - 1;
    const uint32_t lv = __shfl_sync(FULL, v, l), lj = __shfl_sync(FULL, cur, l), le = __shfl_sync(FULL, e, l);
    uint32_t lc = lj;
    const uint8_t r = walk_warp(a, lv, lj, le, &lc);
    if (lane == l) {
      res = r;
      cur = lc;
    }
  }
  if (have && res != UNDECIDED) {
    a.flags[v] = res;
    if (res == IN_SET) in_count++;
  }
  // requeue the undecided with their cursors, through the warp's buffer
  const bool wait = have && res == UNDECIDED;
  const uint32_t incl = warp_incl_scan(wait ? 1u : 0u);
  const uint32_t tot = __shfl_sync(FULL, incl, 31);
  if (tot == 0) return;
  if (nbuf + tot > WQ) {
    wq_flush(wv, wc, nbuf, out, qout, cout_);
    nbuf = 0;
  }
  if (wait) {
    wv[nbuf + incl - 1] = v;
    wc[nbuf + incl - 1] = make_uint2(cur, e);
  }
  nbuf += tot;
  __syncwarp();
}

// Two blocks per SM at <= 40 registers (no spills): 48 resident warps a SM
// instead of 32 hide more of each walk's load latency (11% on rMat 2^24
// against one 1024-thread block; 1024 x 2 at 32 registers spills and 512 x 3
// or 4 are slower).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 2) mis_persistent(MisArgs a) {
  BfsCtrl* c = a.ctrl;
  __shared__ unsigned long long bar_epoch;
  __shared__ unsigned long long s_q;
  __shared__ uint32_t s_wv[BLOCK / 32][WQ];
  __shared__ uint2 s_wc[BLOCK / 32][WQ];
  uint32_t* wv = s_wv[threadIdx.x >> 5];
  uint2* wc = s_wc[threadIdx.x >> 5];
  if (threadIdx.x == 0) bar_epoch = 0;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) c->t_start = dev::globaltimer();
  // ---- init: every vertex undecided
  {
    const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long v = tid; v < a.n; v += nth) a.flags[v] = UNDECIDED;
    if (tid == 0)
      for (int s = 0; s < 3; s++) c->slot[s] = LevelSlot{0, 0, 0, 0};
  }
  bool ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
  unsigned long long in_count = 0;
  uint32_t r = 0;
  unsigned long long nq = a.n;  // round 0: every vertex, from the start of its list
  while (ok && nq > 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && r < PBG_TRACE_LEVELS) {
      c->t_ns[r] = dev::globaltimer();
      c->t_nf[r] = nq;
    }
    if (r >= a.n + 1) {  // cannot happen: the smallest undecided vertex decides every round
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->sync.error, ERR_LEVEL_LIMIT);
      break;
    }
    LevelSlot* out = &c->slot[(r + 1) % 3];
    const uint32_t* qin = (r & 1) ? a.q1 : a.q0;
    const uint2* cin = (r & 1) ? a.c1 : a.c0;
    uint32_t* qout = (r & 1) ? a.q0 : a.q1;
    uint2* cout_ = (r & 1) ? a.c0 : a.c1;
    if (blockIdx.x == 0 && threadIdx.x == 0) c->slot[(r + 2) % 3] = LevelSlot{0, 0, 0, 0};
    const unsigned long long tiles = (nq + 31) / 32;
    uint32_t nbuf = 0;
    for (unsigned long long t = gw; t < tiles; t += tw) {
      const unsigned long long idx = t * 32 + lane;
      const bool have = idx < nq;
      uint32_t v = 0, j = 0, e = 0;
      if (have) {
        if (r == 0) {
          v = (uint32_t)idx;
          j = __ldg(a.offsets + v);
          e = __ldg(a.offsets + v + 1);
        } else {
          v = qin[idx];
          const uint2 ce = cin[idx];
          j = ce.x;
          e = ce.y;
        }
      }
      if (r == 0)
        decide<LANE_SHARE, MK>(a, v, j, e, have, out, qout, cout_, in_count, wv, wc, nbuf);
      else
        decide<LANE_SHARE_LATER, MK_LATER>(a, v, j, e, have, out, qout, cout_, in_count, wv, wc, nbuf);
    }
    if (nbuf) wq_flush(wv, wc, nbuf, out, qout, cout_);
    nbuf = 0;
    r++;
    ok = dev::grid_barrier(&c->sync, ERR_BARRIER_TIMEOUT, bar_epoch);
    if (!ok) break;
    if (threadIdx.x == 0) s_q = dev::ld_relaxed_u64(&out->nmain);
    __syncthreads();
    nq = s_q;
    __syncthreads();
  }
  const unsigned long long bin = dev::block_sum(in_count);
  if (threadIdx.x == 0 && bin) atomicAdd(&c->visited, bin);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->levels = r;
    c->t_end = dev::globaltimer();
    if (r <= PBG_TRACE_LEVELS) c->t_ns[r] = c->t_end;
  }
}

// One warp per vertex: is every list ascending?  (bad set when one is not)
__global__ void k_lists_sorted(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg, uint32_t n,
                               unsigned* bad) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = w; v < n; v += nw) {
    const uint32_t b = off[v], e = off[v + 1];
    bool unsorted = false;
    for (uint32_t j = b + 1 + lane; j < e; j += 32) unsorted |= edg[j - 1] > edg[j];
    if (__any_sync(FULL, unsorted)) {
      if (lane == 0) atomicOr(bad, 1u);
    }
  }
}

constexpr int MIS_BLOCK = 768;

int mis_grid(int num_sms, int* grid_out) {
  static std::mutex mu;
  static int grid = 0, dev_of = -1;
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev_of != dev) {
    int per_sm = 0;
    PBG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mis_persistent<MIS_BLOCK>, MIS_BLOCK, 0));
    if (per_sm < 1) return fail(PBG_ERR_CUDA, "MIS kernel cannot be resident");
    grid = per_sm * num_sms;
    dev_of = dev;
  }
  *grid_out = grid;
  return PBG_OK;
}

// Whether every list of g is ascending, found once per graph.
int lists_sorted(pbg_graph* g, uint32_t* sorted) {
  if (g->lists_sorted >= 0) {
    *sorted = (uint32_t)g->lists_sorted;
    return PBG_OK;
  }
  unsigned* d_bad = nullptr;
  unsigned bad = 0;
  PBG_CUDA(cudaMalloc(&d_bad, sizeof(unsigned)));
  cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), g->stream);
  if (e == cudaSuccess) {
    k_lists_sorted<<<grid_for((uint64_t)g->n * 32, g->num_sms), 256, 0, g->stream>>>(g->d_offsets, g->d_edges, g->n,
                                                                                      d_bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(d_bad);
  if (e != cudaSuccess) return cuda_fail(e, "list order check");
  g->lists_sorted = bad ? 0 : 1;
  *sorted = (uint32_t)g->lists_sorted;
  return PBG_OK;
}

}  // namespace

int mis_launch(pbg_graph* g, uint8_t* d_flags, cudaStream_t s) {
  pbg_bfs_opts o;
  resolve_opts(nullptr, &o);
  int rc = bfs_ensure_workspace(g, o);  // the BFS queues and control block serve the rounds
  if (rc) return rc;
  uint32_t sorted = 0;
  rc = lists_sorted(g, &sorted);
  if (rc) return rc;
  int grid = 0;
  rc = mis_grid(g->num_sms, &grid);
  if (rc) return rc;
  if (!g->mis_ctrl) {
    cudaError_t e = cudaMalloc(&g->mis_ctrl, sizeof(BfsCtrl));
    if (e == cudaSuccess && !g->mis_ev0) e = cudaEventCreate(&g->mis_ev0);
    if (e == cudaSuccess && !g->mis_ev1) e = cudaEventCreate(&g->mis_ev1);
    if (e != cudaSuccess) {
      cudaFree(g->mis_ctrl);
      g->mis_ctrl = nullptr;
      return cuda_fail(e, "MIS control block");
    }
  }
  BfsWorkspace& w = g->ws;
  MisArgs a;
  a.offsets = g->d_offsets;
  a.edges = g->d_edges;
  a.flags = d_flags;
  a.q0 = w.q[0];
  a.q1 = w.q[1];
  // the (begin, end) arrays of the BFS queues hold (cursor, list end)
  a.c0 = w.qr[0];
  a.c1 = w.qr[1];
  a.ctrl = g->mis_ctrl;
  a.n = g->n;
  a.sorted = sorted;
  PBG_CUDA(cudaMemsetAsync(g->mis_ctrl, 0, sizeof(BfsCtrl), s));
  PBG_CUDA(cudaEventRecord(g->mis_ev0, s));
  void* params[] = {&a};
  PBG_CUDA(cudaLaunchCooperativeKernel((const void*)mis_persistent<MIS_BLOCK>, dim3(grid), dim3(MIS_BLOCK), params,
                                       0, s));
  PBG_CUDA(cudaEventRecord(g->mis_ev1, s));
  g->mis_pending = true;
  return PBG_OK;
}

int mis_read_stats(pbg_graph* g, pbg_mis_stats* st) {
  if (!g->mis_ctrl || !g->mis_ran) return fail(PBG_ERR_STATE, "no MIS has run on this graph");
  if (g->mis_pending) {
    BfsCtrl c;
    PBG_CUDA(cudaEventSynchronize(g->mis_ev1));
    PBG_CUDA(cudaMemcpy(&c, g->mis_ctrl, sizeof(BfsCtrl), cudaMemcpyDeviceToHost));
    pbg_mis_stats& m = g->mis_last;
    m.rounds = c.levels;
    m.error = c.sync.error;
    m.in_set = c.visited;
    float ms = 0.f;
    PBG_CUDA(cudaEventElapsedTime(&ms, g->mis_ev0, g->mis_ev1));
    m.device_ms = ms;
    m.kernel_ms = (c.t_end > c.t_start) ? (float)((c.t_end - c.t_start) * 1e-6) : 0.f;
    g->mis_pending = false;
  }
  if (st) *st = g->mis_last;
  if (g->mis_last.error & ERR_BARRIER_TIMEOUT) return fail(PBG_ERR_TIMEOUT, "MIS: a grid barrier wait ran out");
  if (g->mis_last.error) return fail(PBG_ERR_STATE, "MIS: device error word set");
  return PBG_OK;
}

// Per-round trace of the last MIS: the vertices each round walked and its
// device time.
int mis_read_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count) {
  int rc = mis_read_stats(g, nullptr);
  if (rc && rc != PBG_ERR_TIMEOUT && rc != PBG_ERR_STATE) return rc;
  if (!g->mis_ctrl || !g->mis_ran) return fail(PBG_ERR_STATE, "no MIS has run on this graph");
  BfsCtrl* c = new BfsCtrl;
  cudaError_t e = cudaMemcpy(c, g->mis_ctrl, sizeof(BfsCtrl), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "trace copy");
  }
  const uint32_t k = std::min(std::min<uint32_t>(c->levels, PBG_TRACE_LEVELS), cap);
  for (uint32_t r = 0; r < k; r++) {
    out[r].level = r;
    out[r].bottom_up = 0;
    out[r].frontier = c->t_nf[r];
    out[r].frontier_degree = 0;
    out[r].ms = (c->t_ns[r + 1] - c->t_ns[r]) * 1e-6;
  }
  if (count) *count = k;
  delete c;
  return PBG_OK;
}

}  // namespace pbg

using namespace pbg;

extern "C" int pbg_mis_device(pbg_graph* g, uint8_t* d_flags, void* stream) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  if (!d_flags) return fail(PBG_ERR_ARG, "d_flags is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = mis_launch(g, d_flags, s);
  if (rc) return rc;
  g->mis_ran = true;
  return PBG_OK;
}

extern "C" int pbg_mis(pbg_graph* g, uint8_t* flags_out, pbg_mis_stats* st) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  if (!flags_out) return fail(PBG_ERR_ARG, "flags_out is NULL");
  if (!g->mis_flags) {
    cudaError_t e = cudaMalloc(&g->mis_flags, (size_t)g->n + 16);
    if (e != cudaSuccess) {
      g->mis_flags = nullptr;
      return cuda_fail(e, "MIS flags");
    }
  }
  int rc = mis_launch(g, g->mis_flags, g->stream);
  if (rc) return rc;
  g->mis_ran = true;
  PBG_CUDA(cudaMemcpyAsync(flags_out, g->mis_flags, g->n, cudaMemcpyDeviceToHost, g->stream));
  PBG_CUDA(cudaStreamSynchronize(g->stream));
  pbg_mis_stats tmp;
  return mis_read_stats(g, st ? st : &tmp);
}

extern "C" int pbg_mis_stats_get(pbg_graph* g, pbg_mis_stats* st) {
  if (!g || !st) return fail(PBG_ERR_ARG, "NULL argument");
  return mis_read_stats(g, st);
}

extern "C" int pbg_mis_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count) {
  if (!g || (!out && cap)) return fail(PBG_ERR_ARG, "NULL argument");
  return mis_read_trace(g, out, cap, count);
}
