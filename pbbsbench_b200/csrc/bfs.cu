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
//   q[2]    u32[n]                     frontier queues (vertices with deg < big_min_degree)
//   qbig[2] uint4[big_cap]             (v, begin, end, first chunk) of vertices with
//                                      deg >= big_min_degree, split in CHUNK-edge pieces
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
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "internal.cuh"

namespace pbg {
namespace {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr uint32_t CHUNK = 1024;                  // edges per big-vertex chunk
constexpr unsigned long long BIG_SHIFT = 40;
constexpr unsigned long long BIG_MASK = (1ull << BIG_SHIFT) - 1;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;  // 2 s

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
  uint32_t warp_deg;
  uint32_t big_deg;
  uint32_t symmetric;
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

// Grid-wide barrier for a cooperative launch.  Thread 0 of each block
// arrives with a release (fence + atomic) and waits with acquire loads on the
// generation word, bounded by BARRIER_TIMEOUT_NS.  Returns false if the wait
// ran out or another block reported an error.
__device__ bool grid_barrier(BfsCtrl* c) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned gen = ld_acquire_u32(&c->bar_gen);
    __threadfence();
    unsigned arrived = atomicAdd(&c->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&c->bar_count, 0u);
      __threadfence();
      atomicAdd(&c->bar_gen, 1u);
      (void)ld_acquire_u32(&c->bar_gen);
    } else {
      unsigned long long t0 = globaltimer();
      unsigned spins = 0;
      while (ld_acquire_u32(&c->bar_gen) == gen) {
        if (++spins > 8) __nanosleep(32);
        if ((spins & 255) == 0) {
          if (ld_acquire_u32(&c->error) != 0) {
            ok = 0;
            break;
          }
          if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
            atomicOr(&c->error, ERR_BARRIER_TIMEOUT);
            ok = 0;
            break;
          }
        }
      }
    }
    if (ok && ld_acquire_u32(&c->error) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

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
    int nw = blockDim.x >> 5;
    r = (lane < nw) ? s_part[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(FULL, r, o);
  }
  return r;  // valid in thread 0
}

// Warp-collective append of the lanes with win == true to the next frontier.
// [b, e) is the winner's adjacency range.  Vertices with degree >= big_deg go
// to the big queue with their chunk range; the rest are compacted with one
// ballot/popc and one atomic per warp.  Positions >= cap are counted but not
// written (bottom-up writes its queue only while it can still be used).
__device__ __forceinline__ void emit(const BfsArgs& a, LevelSlot* out, uint32_t* qout, uint4* qbout,
                                     bool win, uint32_t v, uint32_t b, uint32_t e, unsigned long long cap,
                                     unsigned long long& degacc) {
  const unsigned wm = __ballot_sync(FULL, win);
  if (wm == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t deg = e - b;
  const bool big = win && deg >= a.big_deg;
  if (win) degacc += deg;
  const unsigned mm = __ballot_sync(FULL, win && !big);
  if (mm) {
    const int leader = __ffs(mm) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&out->nmain, (unsigned long long)__popc(mm));
    base = __shfl_sync(FULL, base, leader);
    if (win && !big) {
      unsigned long long pos = base + __popc(mm & ((1u << lane) - 1u));
      if (pos < cap) qout[pos] = v;
    }
  }
  if (big) {
    const uint32_t nch = (deg + CHUNK - 1) / CHUNK;
    unsigned long long old = atomicAdd(&out->big, (1ull << BIG_SHIFT) | nch);
    uint32_t slot = (uint32_t)(old >> BIG_SHIFT);
    if (slot < a.big_cap)
      qbout[slot] = make_uint4(v, b, e, (uint32_t)(old & BIG_MASK));
    else
      atomicOr(&a.ctrl->error, ERR_QUEUE);
  }
}

// Top-down claim of v by u.  Returns true for the one thread that enqueues v.
template <int MODE>
__device__ __forceinline__ bool td_claim(const BfsArgs& a, const uint32_t* vis, uint32_t* claim, uint32_t u,
                                         uint32_t v, uint32_t next_level) {
  const uint32_t bit = 1u << (v & 31);
  const uint32_t wi = v >> 5;
  if (vis[wi] & bit) return false;
  if (MODE == MODE_ANY) {
    uint32_t old = atomicOr(claim + wi, bit);
    if (old & bit) return false;
    a.parent[v] = u;
  } else {
    if (MODE == MODE_MIN)
      atomicMin(a.parent + v, u);
    else
      atomicMax(reinterpret_cast<int*>(a.parent) + v, (int)u);
    if (claim[wi] & bit) return false;
    uint32_t old = atomicOr(claim + wi, bit);
    if (old & bit) return false;
  }
  if (a.level) a.level[v] = next_level;
  return true;
}

// Expands the lanes' edges [j, ...) warp-synchronously: one edge per lane.
template <int MODE>
__device__ __forceinline__ void td_edge(const BfsArgs& a, const uint32_t* vis, uint32_t* claim, LevelSlot* out,
                                        uint32_t* qout, uint4* qbout, bool act, uint32_t u, uint32_t j,
                                        uint32_t next_level, unsigned long long& degacc) {
  uint32_t v = act ? __ldg(a.edges + j) : 0u;
  bool win = act && td_claim<MODE>(a, vis, claim, u, v, next_level);
  uint32_t b = 0, e = 0;
  if (win) {
    b = __ldg(a.offsets + v);
    e = __ldg(a.offsets + v + 1);
  }
  emit(a, out, qout, qbout, win, v, b, e, ~0ull, degacc);
}

// Big vertices: every warp of the grid takes CHUNK-edge pieces; the owner of
// piece c is found by binary search on the entries' first-chunk index.
template <int MODE>
__device__ void td_big(const BfsArgs& a, const uint4* qbin, uint32_t nbig, uint32_t nchunks, const uint32_t* vis,
                       uint32_t* claim, LevelSlot* out, uint32_t* qout, uint4* qbout, uint32_t next_level,
                       unsigned long long& degacc) {
  if (nbig == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = gw; c < nchunks; c += tw) {
    uint32_t lo = 0, hi = nbig - 1;
    while (lo < hi) {
      uint32_t mid = (lo + hi + 1) >> 1;
      if (qbin[mid].w <= c)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint4 ent = qbin[lo];
    const uint32_t u = ent.x;
    const uint32_t cb = ent.y + (c - ent.w) * CHUNK;
    const uint32_t ce = min(ent.z, cb + CHUNK);
    if (MODE != MODE_ANY && c == ent.w && lane == 0) atomicOr(claim + (u >> 5), 1u << (u & 31));
    for (uint32_t j0 = cb; j0 < ce; j0 += 32) {
      uint32_t j = j0 + lane;
      td_edge<MODE>(a, vis, claim, out, qout, qbout, j < ce, u, j, next_level, degacc);
    }
  }
}

// Main queue: tiles of blockDim entries.  deg < warp_deg: the owning thread
// walks its list (all lanes step together so the append stays warp-wide);
// warp_deg <= deg < big_deg: the warp walks the list 32 edges at a time.
template <int MODE>
__device__ void td_main(const BfsArgs& a, const uint32_t* qin, unsigned long long nmain, const uint32_t* vis,
                        uint32_t* claim, LevelSlot* out, uint32_t* qout, uint4* qbout, uint32_t next_level,
                        unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < nmain; base += stride) {
    const unsigned long long idx = base + threadIdx.x;
    const bool have = idx < nmain;
    uint32_t u = 0, b = 0, e = 0;
    if (have) {
      u = qin[idx];
      b = __ldg(a.offsets + u);
      e = __ldg(a.offsets + u + 1);
      if (MODE != MODE_ANY) atomicOr(claim + (u >> 5), 1u << (u & 31));
    }
    const uint32_t deg = e - b;
    const bool med = have && deg >= a.warp_deg;
    const uint32_t sdeg = (have && !med) ? deg : 0u;
    const uint32_t maxd = __reduce_max_sync(FULL, sdeg);
    for (uint32_t j = 0; j < maxd; j++)
      td_edge<MODE>(a, vis, claim, out, qout, qbout, j < sdeg, u, b + j, next_level, degacc);
    unsigned mm = __ballot_sync(FULL, med);
    while (mm) {
      const int l = __ffs(mm) - 1;
      mm &= mm - 1;
      const uint32_t uu = __shfl_sync(FULL, u, l);
      const uint32_t bb = __shfl_sync(FULL, b, l);
      const uint32_t ee = __shfl_sync(FULL, e, l);
      for (uint32_t j0 = bb; j0 < ee; j0 += 32) {
        const uint32_t j = j0 + lane;
        td_edge<MODE>(a, vis, claim, out, qout, qbout, j < ee, uu, j, next_level, degacc);
      }
    }
  }
}

// Bottom-up over bitmap words: one warp per word, one lane per vertex.
template <int MODE>
__device__ void bu_level(const BfsArgs& a, const uint32_t* vin, uint32_t* vout, LevelSlot* out, uint32_t* qout,
                         uint4* qbout, uint32_t next_level, unsigned long long cap, unsigned long long& degacc) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t tw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t w = gw; w < a.nwords; w += tw) {
    const uint32_t word = vin[w];
    if (word == FULL) {
      if (lane == 0) vout[w] = word;
      continue;
    }
    const uint32_t v = w * 32 + lane;
    const bool unv = !((word >> lane) & 1u);  // padding bits past n are set
    bool found = false;
    uint32_t p = 0, b = 0, e = 0;
    if (unv) {
      b = __ldg(a.offsets + v);
      e = __ldg(a.offsets + v + 1);
      if (MODE == MODE_MAX) {
        for (uint32_t j = e; j > b;) {
          --j;
          const uint32_t u = __ldg(a.edges + j);
          if ((vin[u >> 5] >> (u & 31)) & 1u) {
            found = true;
            p = u;
            break;
          }
        }
      } else {
        for (uint32_t j = b; j < e; j++) {
          const uint32_t u = __ldg(a.edges + j);
          if ((vin[u >> 5] >> (u & 31)) & 1u) {
            found = true;
            p = u;
            break;
          }
        }
      }
    }
    const unsigned nb = __ballot_sync(FULL, found);
    if (lane == 0) vout[w] = word | nb;
    if (found) {
      a.parent[v] = p;
      if (a.level) a.level[v] = next_level;
    }
    emit(a, out, qout, qbout, found, v, b, e, cap, degacc);
  }
}

template <int MODE>
__global__ void __launch_bounds__(1024) bfs_persistent(BfsArgs a) {
  BfsCtrl* c = a.ctrl;
  __shared__ unsigned long long s_in[3];

  // ---- init: parent/level = NONE, bitmaps = degree-0 + padding bits, source.
  {
    const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = tid; i < a.n; i += nth) {
      a.parent[i] = (i == a.src) ? a.src : PBG_NONE;
      if (a.level) a.level[i] = (i == a.src) ? 0u : PBG_NONE;
    }
    const uint32_t sw = a.src >> 5, sbit = 1u << (a.src & 31);
    for (unsigned long long w = tid; w < a.nwords; w += nth) {
      uint32_t x = a.iso[w];
      a.bm0[w] = (w == sw) ? (x | sbit) : x;
      a.bm1[w] = (MODE == MODE_ANY && w == sw) ? (x | sbit) : x;
    }
    if (tid == 0) {
      const uint32_t b = __ldg(a.offsets + a.src), e = __ldg(a.offsets + a.src + 1);
      const uint32_t deg = e - b;
      for (int s = 0; s < 3; s++) c->slot[s] = LevelSlot{0, 0, 0, 0};
      if (deg >= a.big_deg) {
        a.qb0[0] = make_uint4(a.src, b, e, 0u);
        c->slot[0].big = (1ull << BIG_SHIFT) | ((deg + CHUNK - 1) / CHUNK);
      } else {
        a.q0[0] = a.src;
        c->slot[0].nmain = 1;
      }
      c->slot[0].deg = deg;
    }
  }
  bool ok = grid_barrier(c);

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
    const unsigned long long nmain = s_in[0], big = s_in[1], fdeg = s_in[2];
    __syncthreads();
    const uint32_t nbig = (uint32_t)(big >> BIG_SHIFT);
    const uint32_t nchunks = (uint32_t)(big & BIG_MASK);
    const unsigned long long nf = nmain + nbig;
    if (nf == 0) break;
    if (L >= a.n) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->error, ERR_LEVEL_LIMIT);
      break;
    }
    if (nbig > a.big_cap || nmain > a.n) {  // cannot happen: each vertex enters one frontier once
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->error, ERR_QUEUE);
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
    uint32_t* qout = (L & 1) ? a.q0 : a.q1;
    uint4* qbin = (L & 1) ? a.qb1 : a.qb0;
    uint4* qbout = (L & 1) ? a.qb0 : a.qb1;
    uint32_t* bcur = cur ? a.bm1 : a.bm0;
    uint32_t* both = cur ? a.bm0 : a.bm1;
    unsigned long long degacc = 0;
    if (bu) {
      const unsigned long long cap =
          (a.policy == PBG_DIR_AUTO) ? (unsigned long long)(a.n / a.beta) : (unsigned long long)a.n;
      bu_level<MODE>(a, bcur, both, out, qout, qbout, L + 1, cap, degacc);
      cur ^= 1u;
    } else {
      uint32_t* claim = (MODE == MODE_ANY) ? bcur : both;
      td_big<MODE>(a, qbin, nbig, nchunks, bcur, claim, out, qout, qbout, L + 1, degacc);
      td_main<MODE>(a, qin, nmain, bcur, claim, out, qout, qbout, L + 1, degacc);
      if (MODE != MODE_ANY) cur ^= 1u;
    }
    const unsigned long long bsum = block_sum(degacc);
    if (threadIdx.x == 0 && bsum) atomicAdd(&out->deg, bsum);
    prev_bu = bu;
    L++;
    ok = grid_barrier(c);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->levels = L;
    c->td_levels = tdl;
    c->bu_levels = bul;
    c->final_bm = cur;
    c->visited = visited;
    c->edges_reached = reached;
    c->bu_mask = bumask;
  }
}

struct KernelShape {
  int grid[3] = {0, 0, 0};  // per block size index (256, 512, 1024)
};

int block_index(int block) { return block == 256 ? 0 : (block == 512 ? 1 : 2); }

template <int MODE>
int launch_mode(const BfsArgs& a, int block, int num_sms, cudaStream_t s) {
  static std::mutex mu;
  static int grids[3] = {0, 0, 0};
  static int dev_of[3] = {-1, -1, -1};
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  const int bi = block_index(block);
  int grid;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev_of[bi] != dev) {
      int per_sm = 0;
      PBG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_persistent<MODE>, block, 0));
      if (per_sm < 1) return fail(PBG_ERR_CUDA, "BFS kernel cannot be resident with this block size");
      grids[bi] = per_sm * num_sms;
      dev_of[bi] = dev;
    }
    grid = grids[bi];
  }
  BfsArgs args = a;
  void* params[] = {&args};
  PBG_CUDA(cudaLaunchCooperativeKernel((const void*)bfs_persistent<MODE>, dim3(grid), dim3(block), params, 0, s));
  return PBG_OK;
}

}  // namespace

void resolve_opts(const pbg_bfs_opts* in, pbg_bfs_opts* o) {
  if (in)
    *o = *in;
  else
    pbg_bfs_opts_default(o);
  if (o->alpha == 0) o->alpha = 20;
  if (o->beta == 0) o->beta = 20;
  if (o->block_threads == 0) o->block_threads = 512;
  if (o->warp_min_degree == 0) o->warp_min_degree = 32;
  if (o->big_min_degree == 0) o->big_min_degree = 4096;
}

int bfs_ensure_workspace(pbg_graph* g, const pbg_bfs_opts& o) {
  BfsWorkspace& w = g->ws;
  if (w.ready && w.big_min_degree <= o.big_min_degree) return PBG_OK;
  bfs_free_workspace(g);
  const size_t n = g->n ? g->n : 1;
  const uint32_t big_cap = (uint32_t)std::min<uint64_t>(n, g->m / o.big_min_degree + 1);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaMalloc(&w.bm[i], sizeof(uint32_t) * g->nwords);
    if (e == cudaSuccess) e = cudaMalloc(&w.q[i], sizeof(uint32_t) * n);
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
  w.big_min_degree = o.big_min_degree;
  w.ready = true;
  return PBG_OK;
}

void bfs_free_workspace(pbg_graph* g) {
  BfsWorkspace& w = g->ws;
  for (int i = 0; i < 2; i++) {
    cudaFree(w.bm[i]);
    cudaFree(w.q[i]);
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

int bfs_launch(pbg_graph* g, uint32_t src, const pbg_bfs_opts& o, uint32_t* d_parent, uint32_t* d_level,
               cudaStream_t s) {
  if (o.parent_mode > PBG_PARENT_MAX) return fail(PBG_ERR_ARG, "unknown parent_mode");
  if (o.direction > PBG_DIR_BOTTOMUP) return fail(PBG_ERR_ARG, "unknown direction policy");
  if (o.direction == PBG_DIR_BOTTOMUP && !(g->flags & PBG_GRAPH_SYMMETRIC))
    return fail(PBG_ERR_ARG, "bottom-up needs a symmetric graph");
  if (o.block_threads != 256 && o.block_threads != 512 && o.block_threads != 1024)
    return fail(PBG_ERR_ARG, "block_threads must be 256, 512 or 1024");
  if (o.warp_min_degree < 1 || o.big_min_degree < o.warp_min_degree)
    return fail(PBG_ERR_ARG, "need 1 <= warp_min_degree <= big_min_degree");
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
  a.warp_deg = o.warp_min_degree;
  a.big_deg = o.big_min_degree;
  a.symmetric = (g->flags & PBG_GRAPH_SYMMETRIC) ? 1u : 0u;
  PBG_CUDA(cudaMemsetAsync(w.ctrl, 0, sizeof(BfsCtrl), s));
  PBG_CUDA(cudaEventRecord(w.ev0, s));
  switch (o.parent_mode) {
    case PBG_PARENT_ANY: rc = launch_mode<MODE_ANY>(a, (int)o.block_threads, g->num_sms, s); break;
    case PBG_PARENT_MIN: rc = launch_mode<MODE_MIN>(a, (int)o.block_threads, g->num_sms, s); break;
    default: rc = launch_mode<MODE_MAX>(a, (int)o.block_threads, g->num_sms, s); break;
  }
  if (rc) return rc;
  PBG_CUDA(cudaEventRecord(w.ev1, s));
  g->stats_pending = true;
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
    s.error = c.error;
    s.visited = c.visited;
    s.edges_reached = c.edges_reached;
    s.bottomup_mask = c.bu_mask;
    float ms = 0.f;
    PBG_CUDA(cudaEventElapsedTime(&ms, g->ws.ev0, g->ws.ev1));
    s.device_ms = ms;
    g->stats_pending = false;
  }
  if (st) *st = g->last;
  if (g->last.error & ERR_BARRIER_TIMEOUT) return fail(PBG_ERR_TIMEOUT, "BFS: a grid barrier wait ran out");
  if (g->last.error) return fail(PBG_ERR_STATE, "BFS: device error word set");
  return PBG_OK;
}

}  // namespace pbg
