// check.cu -- the BFS checker on the device.
//
// pbg_bfs_check restates checkBFS (benchmarks/breadthFirstSearch/bench/
// BFSCheck.C:39-90): levels by pointer doubling on the parent tree
// (level_number, :39-56: (0, v) for a root or an unreached vertex, else
// (1, parent); (c, p) <- (c + c[p], p[p]) until nothing changes; a vertex
// whose root has no parent gets level n), then every vertex but the start
// must have level = (minimum neighbour level) + 1, or level n with every
// neighbour at level n, and the start must be its own parent (:66-78).  The
// reference loops until a fixed point; its counts are 32-bit and wrap, so
// even a cycle in the parent array settles (its counts reach 0 after about
// 33 doublings) and the predicate then finds a failing vertex.  Here the
// counts wrap the same way and the doubling stops after MAX_ROUNDS rounds;
// one that has not settled by then fails with bad vertex n.  PBG_CHECK_EDGES
// adds the
// edge test: each parent must be a neighbour of its vertex (found during the
// same neighbour scan).  pbg_levels_check applies the same level predicate
// to uint8 level rows (255 = unreached) of batched searches.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.cuh"
#include "msbfs.cuh"

using namespace pbg;

namespace {

using dev::FULL;
constexpr uint32_t SERIAL = 64;
static_assert(SERIAL == MS_PULL_SERIAL, "list tails are the pull chunk table's pieces");
constexpr uint32_t MAX_ROUNDS = 64;  // doubling rounds (a valid tree of depth d settles in log2 d + 1)

// Also records the smallest vertex whose parent is neither PBG_NONE nor a
// vertex (checked before anything else, as the oracle does).
__global__ void jump_init(const uint32_t* __restrict__ parent, uint32_t n, uint32_t* __restrict__ cnt,
                          uint32_t* __restrict__ ptr, uint32_t* bad_parent) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t p = parent[v];
    if (p != PBG_NONE && p >= n) atomicMin(bad_parent, v);
    const bool root = p == PBG_NONE || p == v || p >= n;
    cnt[v] = root ? 0u : 1u;
    ptr[v] = root ? v : p;
  }
}

// One doubling round; *changed is set when any pair moves.
__global__ void jump_step(const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ ptr, uint32_t n,
                          uint32_t* __restrict__ cnt2, uint32_t* __restrict__ ptr2, unsigned* changed) {
  bool moved = false;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t p = ptr[v];
    const uint32_t c = cnt[v] + cnt[p];
    const uint32_t q = ptr[p];
    cnt2[v] = c;
    ptr2[v] = q;
    moved |= (c != cnt[v] || q != p);
  }
  if (__any_sync(FULL, moved) && (threadIdx.x & 31) == 0) atomicOr(changed, 1u);
}

// Level of each vertex from the settled pairs (n = unreached tree).
__global__ void jump_finish(const uint32_t* __restrict__ parent, const uint32_t* __restrict__ cnt,
                            const uint32_t* __restrict__ ptr, uint32_t n, uint32_t* __restrict__ level) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    level[v] = (parent[ptr[v]] == PBG_NONE) ? n : cnt[v];
}

// Level of vertex v in row r: uint32 levels (lv32, n = unreached) or uint8
// rows (lv8, 255 = unreached, mapped to n).
struct Levels {
  const uint32_t* lv32;
  const uint8_t* lv8;
  uint32_t n;
  __device__ __forceinline__ uint32_t at(uint32_t r, uint32_t v) const {
    if (lv32) return lv32[v];
    const uint8_t x = lv8[(size_t)r * n + v];
    return x == 255 ? n : x;
  }
};

// The neighbour minimum over the tails of lists longer than SERIAL (the
// graph's pull chunk table: (vertex, first, end, degree) pieces of
// MS_PULL_CHUNK edges), one warp a piece, any warp of the grid: tmin[v]
// (initially all ones) takes the smallest level with atomicMin, tadj[v] is
// set when the piece holds v's parent.  A hub's list is then spread over the
// grid instead of walked by the one warp that holds the vertex.
__global__ void check_tails(const uint4* __restrict__ chunks, uint32_t nchunks, const uint32_t* __restrict__ edges,
                            const uint32_t* __restrict__ level, const uint32_t* __restrict__ parent,
                            uint32_t* __restrict__ tmin, uint8_t* __restrict__ tadj) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nchunks; c += nw) {
    const uint4 ent = chunks[c];
    const uint32_t pv = parent[ent.x];
    uint32_t m = 0xFFFFFFFFu;
    bool adj = false;
#pragma unroll
    for (uint32_t k = 0; k < MS_PULL_CHUNK / 32; k++) {
      const uint32_t j = ent.y + k * 32 + lane;
      if (j < ent.z) {
        const uint32_t u = edges[j];
        m = min(m, level[u]);
        adj |= (u == pv);
      }
    }
    m = __reduce_min_sync(FULL, m);
    adj = __any_sync(FULL, adj);
    if (lane == 0) {
      if (m != 0xFFFFFFFFu) atomicMin(tmin + ent.x, m);
      if (adj) tadj[ent.x] = 1;
    }
  }
}

// The predicate for 32 consecutive vertices of row r per warp: neighbour
// minimum by one lane for the first SERIAL neighbours, the rest of longer
// lists from check_tails' tmin/tadj when given (one row), else by the whole
// warp; the smallest failing (row, vertex) goes into
// *bad as (row << 32 | vertex), with the level and neighbour minimum.
__global__ void check_rows(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edges, Levels L,
                           const uint32_t* __restrict__ srcs, uint32_t rows, const uint32_t* __restrict__ parent,
                           uint32_t check_edges, unsigned long long* bad, uint32_t* bad_info,
                           const uint32_t* __restrict__ tmin, const uint8_t* __restrict__ tadj) {
  const uint32_t n = L.n;
  const int lane = threadIdx.x & 31;
  const unsigned long long tiles = (unsigned long long)rows * ((n + 31) / 32);
  const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  for (unsigned long long t = (unsigned long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < tiles;
       t += nw) {
    const uint32_t r = (uint32_t)(t / ((n + 31) / 32));
    const uint32_t v = (uint32_t)(t % ((n + 31) / 32)) * 32 + lane;
    const bool active = v < n;
    const uint32_t src = srcs[r];
    uint32_t b = 0, e = 0, lv = n, pv = PBG_NONE;
    if (active) {
      b = off[v];
      e = off[v + 1];
      lv = L.at(r, v);
      if (parent) pv = parent[v];
    }
    uint32_t mn = n;
    bool padj = false;
    const uint32_t es = (e - b > SERIAL) ? b + SERIAL : e;
#pragma unroll 4
    for (uint32_t j = b; j < es; j++) {
      const uint32_t u = edges[j];
      mn = min(mn, L.at(r, u));
      padj |= (u == pv);
    }
    if (tmin && e - b > SERIAL) {
      mn = min(mn, tmin[v]);  // all ones when no tail piece saw a smaller level
      padj |= tadj[v] != 0;
    }
    unsigned big = tmin ? 0u : __ballot_sync(FULL, e - b > SERIAL);
    while (big) {
      const int l = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bb = __shfl_sync(FULL, b, l) + SERIAL, ee = __shfl_sync(FULL, e, l);
      const uint32_t pl = __shfl_sync(FULL, pv, l);
      uint32_t m2 = n;
      bool a2 = false;
      for (uint32_t j = bb + lane; j < ee; j += 32) {
        const uint32_t u = edges[j];
        m2 = min(m2, L.at(r, u));
        a2 |= (u == pl);
      }
      m2 = __reduce_min_sync(FULL, m2);
      a2 = __any_sync(FULL, a2);
      if (lane == l) {
        mn = min(mn, m2);
        padj |= a2;
      }
    }
    bool ok = true;
    if (active) {
      if (v == src) {
        ok = parent ? (pv == v) : (lv == 0);
      } else {
        ok = (lv == n && mn == n) || (mn < n && lv == mn + 1);
        if (ok && check_edges && parent && pv != PBG_NONE) ok = padj;
      }
    }
    if (!ok) {
      const unsigned long long key = ((unsigned long long)r << 32) | v;
      const unsigned long long old = atomicMin(bad, key);
      if (key < old) {
        bad_info[0] = lv;
        bad_info[1] = mn;
      }
    }
  }
}

int grid_for(uint32_t n) { return (int)std::min<uint64_t>((n + 255) / 256, 148 * 16); }

// Scratch of at least `bytes` for a check on g, kept on the handle for later
// checks (a larger request replaces it; every check waits for its kernels
// before returning, so none is still using the old one).
int check_scratch(pbg_graph* g, size_t bytes, void** out) {
  if (g->check_bytes < bytes) {
    cudaFree(g->check_buf);
    g->check_buf = nullptr;
    g->check_bytes = 0;
    const cudaError_t e = cudaMalloc(&g->check_buf, bytes);
    if (e != cudaSuccess) {
      g->check_buf = nullptr;
      cudaGetLastError();
      return fail(e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA,
                  std::string("check scratch: ") + cudaGetErrorString(e));
    }
    g->check_bytes = bytes;
  }
  *out = g->check_buf;
  return PBG_OK;
}

int run_check(pbg_graph* g, Levels L, const uint32_t* d_srcs, uint32_t rows, const uint32_t* d_parent,
              uint32_t check_edges, pbg_check_result* res, cudaStream_t s, unsigned long long* d_bad,
              const uint32_t* tmin = nullptr, const uint8_t* tadj = nullptr) {
  uint32_t* info = reinterpret_cast<uint32_t*>(d_bad + 1);
  PBG_CUDA(cudaMemsetAsync(d_bad, 0xFF, sizeof(unsigned long long), s));
  PBG_CUDA(cudaMemsetAsync(info, 0, 2 * sizeof(uint32_t), s));
  const unsigned long long tiles = (unsigned long long)rows * ((g->n + 31) / 32);
  const int blocks = (int)std::min<unsigned long long>((tiles + 7) / 8, 148ull * 8);
  check_rows<<<std::max(blocks, 1), 256, 0, s>>>(g->d_offsets, g->d_edges, L, d_srcs, rows, d_parent, check_edges,
                                                  d_bad, info, tmin, tadj);
  PBG_CUDA(cudaGetLastError());
  unsigned long long h[2];
  PBG_CUDA(cudaMemcpyAsync(h, d_bad, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  const uint32_t* hi = reinterpret_cast<const uint32_t*>(&h[1]);
  if (h[0] == ~0ull) {
    res->bad_vertex = PBG_NONE;
    res->row = 0;
    res->level = 0;
    res->min_neighbor_level = 0;
  } else {
    res->bad_vertex = (uint32_t)(h[0] & 0xFFFFFFFFu);
    res->row = (uint32_t)(h[0] >> 32);
    res->level = hi[0];
    res->min_neighbor_level = hi[1];
  }
  return PBG_OK;
}

}  // namespace

extern "C" int pbg_bfs_check(pbg_graph* g, uint32_t src, const uint32_t* d_parent, uint32_t flags,
                             pbg_check_result* res) {
  if (!g || !d_parent || !res) return fail(PBG_ERR_ARG, "NULL argument");
  if (src >= g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  if (flags & ~PBG_CHECK_EDGES) return fail(PBG_ERR_ARG, "unknown check flags");
  const uint32_t n = g->n;
  cudaStream_t s = g->stream;
  int rc = ms_pull_chunks(g);  // the tails of lists longer than SERIAL, in pieces
  if (rc) return rc;
  // cnt, ptr, cnt2, ptr2, level, tmin (n each), the source; the result words;
  // tadj (n bytes)
  const size_t words = 6 * (size_t)n + 1;
  const size_t head = (sizeof(uint32_t) * words + 15) & ~15ull;
  const size_t tail = head + 4 * sizeof(unsigned long long);
  void* sp = nullptr;
  rc = check_scratch(g, tail + n, &sp);
  if (rc) return rc;
  uint32_t* cnt = static_cast<uint32_t*>(sp);
  uint32_t* ptr = cnt + n;
  uint32_t* cnt2 = ptr + n;
  uint32_t* ptr2 = cnt2 + n;
  uint32_t* level = ptr2 + n;
  uint32_t* tmin = level + n;
  uint32_t* d_src = tmin + n;
  uint8_t* tadj = static_cast<uint8_t*>(sp) + tail;
  unsigned long long* d_bad = reinterpret_cast<unsigned long long*>(static_cast<char*>(sp) + head);
  unsigned* changed = reinterpret_cast<unsigned*>(d_bad + 2);
  uint32_t* bad_parent = reinterpret_cast<uint32_t*>(d_bad + 3);
  PBG_CUDA(cudaMemcpyAsync(d_src, &src, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  PBG_CUDA(cudaMemsetAsync(bad_parent, 0xFF, sizeof(uint32_t), s));
  const int grid = grid_for(n);
  jump_init<<<grid, 256, 0, s>>>(d_parent, n, cnt, ptr, bad_parent);
  PBG_CUDA(cudaGetLastError());
  uint32_t hbp = PBG_NONE;
  PBG_CUDA(cudaMemcpyAsync(&hbp, bad_parent, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  if (hbp != PBG_NONE) {
    *res = pbg_check_result{hbp, 0, n, n};
    return PBG_OK;
  }
  bool settled = false;
  for (uint32_t i = 0; i < MAX_ROUNDS && !settled; i++) {
    PBG_CUDA(cudaMemsetAsync(changed, 0, sizeof(unsigned), s));
    jump_step<<<grid, 256, 0, s>>>(cnt, ptr, n, cnt2, ptr2, changed);
    PBG_CUDA(cudaGetLastError());
    unsigned h = 0;
    PBG_CUDA(cudaMemcpyAsync(&h, changed, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    std::swap(cnt, cnt2);
    std::swap(ptr, ptr2);
    settled = (h == 0);
  }
  if (!settled) {  // a cycle in the parent array
    *res = pbg_check_result{n, 0, n, n};
    return PBG_OK;
  }
  jump_finish<<<grid, 256, 0, s>>>(d_parent, cnt, ptr, n, level);
  PBG_CUDA(cudaGetLastError());
  PBG_CUDA(cudaMemsetAsync(tmin, 0xFF, sizeof(uint32_t) * n, s));
  PBG_CUDA(cudaMemsetAsync(tadj, 0, n, s));
  if (g->n_pull_chunks) {
    const int tb = (int)std::min<uint64_t>(((uint64_t)g->n_pull_chunks + 7) / 8, 148 * 16);
    check_tails<<<tb, 256, 0, s>>>(g->d_pull_chunks, g->n_pull_chunks, g->d_edges, level, d_parent, tmin, tadj);
    PBG_CUDA(cudaGetLastError());
  }
  return run_check(g, Levels{level, nullptr, n}, d_src, 1, d_parent, (flags & PBG_CHECK_EDGES) ? 1u : 0u, res, s,
                   d_bad, tmin, tadj);
}

extern "C" int pbg_levels_check(pbg_graph* g, const uint32_t* srcs, uint32_t rows, const uint8_t* d_levels,
                                pbg_check_result* res) {
  if (!g || !srcs || !d_levels || !res) return fail(PBG_ERR_ARG, "NULL argument");
  if (rows < 1) return fail(PBG_ERR_ARG, "rows must be >= 1");
  for (uint32_t i = 0; i < rows; i++)
    if (srcs[i] >= g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  cudaStream_t s = g->stream;
  const size_t head = (sizeof(uint32_t) * rows + 15) & ~15ull;
  void* sp = nullptr;
  const int rc = check_scratch(g, head + 2 * sizeof(unsigned long long), &sp);
  if (rc) return rc;
  uint32_t* d_srcs = static_cast<uint32_t*>(sp);
  unsigned long long* d_bad = reinterpret_cast<unsigned long long*>(static_cast<char*>(sp) + head);
  PBG_CUDA(cudaMemcpyAsync(d_srcs, srcs, sizeof(uint32_t) * rows, cudaMemcpyHostToDevice, s));
  return run_check(g, Levels{nullptr, d_levels, g->n}, d_srcs, rows, nullptr, 0, res, s, d_bad);
}
