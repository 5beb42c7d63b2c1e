// graph.cu -- device-resident CSR graphs: upload, validation, and the seeded
// synthetic generators built on the device.
//
// CSR as graph<int,uint> (common/graph.h:104-152): offsets u32[n+1] with
// offsets[n] = m, edges u32[m].  Degrees are offsets[v+1] - offsets[v]; the
// reference's optional degrees[] (graph.h:130-133) is not stored.
//
// Generators restate testData/graphData/{rMatGraph,gridGraph,randLocalGraph}.C
// with SplitMix64's output mix as the hash (parlay::hash64 is unavailable),
// and build the symmetric CSR as common/graphUtils.h:54-94 does: drop self
// loops, add reversed edges, sort by (u, v), drop duplicates, count, scan.
// The sort is cub::DeviceRadixSort over packed (u << shift | v) keys.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "internal.cuh"

namespace pbg {
namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

uint32_t prob_threshold(double p) {
  double t = p * 2147483648.0 + 0.5;
  if (t < 0) t = 0;
  if (t > 4294967295.0) t = 4294967295.0;
  return (uint32_t)t;
}

uint32_t ceil_log2(uint64_t x) {
  uint32_t r = 0;
  while ((1ull << r) < x) r++;
  return r;
}

// Bitmap of vertices that can never be reached or scanned: degree-0 vertices
// of a symmetric graph, and the padding bits past n.
__global__ void k_iso_bitmap(const uint32_t* __restrict__ off, uint32_t n, uint32_t nwords, int symmetric,
                             uint32_t* __restrict__ iso) {
  uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwords) return;
  uint32_t x = 0;
  for (int b = 0; b < 32; b++) {
    uint64_t v = (uint64_t)w * 32 + b;
    if (v >= n)
      x |= 1u << b;
    else if (symmetric && off[v] == off[v + 1])
      x |= 1u << b;
  }
  iso[w] = x;
}

// Validation: offsets[0] = 0, non-decreasing, offsets[n] = m, edges < n.
// bad[0]: error bits; bad[1]: the largest degree.
__global__ void k_validate(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg, uint32_t n,
                           uint64_t m, unsigned* bad) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  uint32_t md = 0;
  for (uint64_t v = tid; v < n; v += nth) {
    const uint32_t b = off[v], e = off[v + 1];
    if (b > e)
      atomicOr(bad, 1u);
    else
      md = max(md, e - b);
  }
  md = __reduce_max_sync(0xFFFFFFFFu, md);
  if ((threadIdx.x & 31) == 0 && md) atomicMax(bad + 1, md);
  if (tid == 0 && (off[0] != 0 || (uint64_t)off[n] != m)) atomicOr(bad, 2u);
  for (uint64_t i = tid; i < m; i += nth)
    if (edg[i] >= n) atomicOr(bad, 4u);
}

// rMat draw for edge i (rMatGraph.C:53-69): start/stride keys from i and the
// seed hash, one 31-bit draw per level, top level first.
__global__ void k_gen_rmat(uint64_t m, uint64_t h, uint32_t logn, uint32_t ta, uint32_t tab, uint32_t tabc,
                           uint32_t shift, uint64_t sentinel, uint64_t* __restrict__ keys) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < m; i += nth) {
    const uint64_t rs = mix64((2 * i) * h);
    const uint64_t st = mix64((2 * i + 1) * h);
    uint32_t u = 0, v = 0;
    for (uint32_t k = 0; k < logn; k++) {
      const uint32_t half = 1u << (logn - 1 - k);
      const uint32_t r = (uint32_t)(mix64(rs + (uint64_t)k * st) & 0x7FFFFFFFu);
      if (r < ta) {
      } else if (r < tab) {
        v += half;
      } else if (r < tabc) {
        u += half;
      } else {
        u += half;
        v += half;
      }
    }
    if (u == v) {
      keys[2 * i] = sentinel;
      keys[2 * i + 1] = sentinel;
    } else {
      keys[2 * i] = ((uint64_t)u << shift) | v;
      keys[2 * i + 1] = ((uint64_t)v << shift) | u;
    }
  }
}

__device__ __forceinline__ uint32_t relabel(const uint32_t* perm, uint32_t x) { return perm ? perm[x] : x; }

// 3-D torus (gridGraph.C:57-72): vertex l = (i*dn + j)*dn + k, edges to the
// +1 neighbour along each axis with wraparound; optional relabelling.
__global__ void k_gen_torus(uint32_t dn, const uint32_t* __restrict__ perm, uint32_t shift, uint64_t sentinel,
                            uint64_t* __restrict__ keys) {
  const uint64_t nn = (uint64_t)dn * dn * dn;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t l = tid; l < nn; l += nth) {
    const uint64_t i = l / ((uint64_t)dn * dn), j = (l / dn) % dn, k = l % dn;
    uint64_t nb[3] = {(((i + 1) % dn) * dn + j) * dn + k, (i * dn + (j + 1) % dn) * dn + k,
                      (i * dn + j) * dn + (k + 1) % dn};
    const uint32_t u = relabel(perm, (uint32_t)l);
    for (int d = 0; d < 3; d++) {
      const uint32_t v = relabel(perm, (uint32_t)nb[d]);
      const uint64_t o = 6 * l + 2 * d;
      if (u == v) {
        keys[o] = sentinel;
        keys[o + 1] = sentinel;
      } else {
        keys[o] = ((uint64_t)u << shift) | v;
        keys[o + 1] = ((uint64_t)v << shift) | u;
      }
    }
  }
}

// Random-local: `deg` out-edges of vertex i at (i + off) mod n, off uniform in
// [-w, w], redrawn (by rehashing) while it lands on i (randLocalGraph.C:46-57).
__global__ void k_gen_randlocal(uint32_t n, uint32_t deg, uint32_t w, uint64_t hs, uint32_t shift,
                                uint64_t sentinel, uint64_t* __restrict__ keys) {
  const uint64_t total = (uint64_t)n * deg;
  const uint64_t span = 2 * (uint64_t)w + 1;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t t = tid; t < total; t += nth) {
    const uint64_t i = t / deg;
    uint64_t x = mix64(hs + t);
    uint32_t j = 0;
    for (;;) {
      const int64_t offv = (int64_t)(x % span) - (int64_t)w;
      int64_t q = ((int64_t)i + offv) % (int64_t)n;
      if (q < 0) q += n;
      j = (uint32_t)q;
      if (j != i) break;
      x = mix64(x);
    }
    keys[2 * t] = ((uint64_t)i << shift) | j;
    keys[2 * t + 1] = ((uint64_t)j << shift) | i;
  }
}

__global__ void k_perm_keys(uint32_t n, uint64_t hs, uint64_t* __restrict__ keys) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < n; i += nth) keys[i] = (mix64(hs + i) & 0xFFFFFFFF00000000ull) | i;
}

__global__ void k_perm_scatter(uint32_t n, const uint64_t* __restrict__ sorted, uint32_t* __restrict__ new_id) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t p = tid; p < n; p += nth) new_id[(uint32_t)(sorted[p] & 0xFFFFFFFFu)] = (uint32_t)p;
}

// Symmetry test: lists ascending and every (u, v) has (v, u).  bad |= 1 on
// an unsorted list, 2 on a missing reverse edge.
__global__ void k_symmetric(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg, uint32_t n,
                            unsigned* bad) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u = tid; u < n; u += nth) {
    const uint32_t b = off[u], e = off[u + 1];
    for (uint32_t j = b; j < e; j++) {
      const uint32_t v = edg[j];
      if (j > b && edg[j - 1] > v) {
        atomicOr(bad, 1u);
        return;
      }
      uint32_t lo = off[v], hi = off[v + 1];
      while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (edg[mid] < u)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo == off[v + 1] || edg[lo] != u) {
        atomicOr(bad, 2u);
        return;
      }
    }
  }
}

// Sorted unique keys -> CSR.  offsets[v] = index of the first key with
// source >= v; edges[i] = low part of key i.
__global__ void k_keys_to_csr(const uint64_t* __restrict__ keys, uint64_t m, uint32_t n, uint32_t shift,
                              uint32_t* __restrict__ off, uint32_t* __restrict__ edg) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t vmask = (1ull << shift) - 1;
  for (uint64_t i = tid; i <= m; i += nth) {
    const uint64_t u = (i < m) ? (keys[i] >> shift) : n;
    const uint64_t pu = (i == 0) ? 0 : ((keys[i - 1] >> shift) + 1);
    for (uint64_t w = pu; w <= u && w <= n; w++) off[w] = (uint32_t)i;
    if (i < m) edg[i] = (uint32_t)(keys[i] & vmask);
  }
}

}  // namespace

int grid_for(uint64_t work, int num_sms) {
  uint64_t g = (work + 255) / 256;
  uint64_t cap = (uint64_t)num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int new_handle(uint32_t n, uint64_t m, uint32_t flags, pbg_graph** out) {
  if (!out) return fail(PBG_ERR_ARG, "out is NULL");
  if (n == 0) return fail(PBG_ERR_ARG, "graph has no vertices");
  if (n > PBG_MAX_VERTICES)
    return fail(PBG_ERR_ARG, "n must be below 2^31: vertex ids are int (bench/BFS.h:5)");
  if (m > 0xFFFFFFFFull) return fail(PBG_ERR_ARG, "m must fit in 32 bits (uint offsets)");
  pbg_graph* g = new pbg_graph();
  g->n = n;
  g->m = m;
  g->flags = flags;
  g->nwords = (uint32_t)((((uint64_t)n + 31) / 32 + 31) / 32 * 32);
  cudaError_t e = cudaGetDevice(&g->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_offsets, sizeof(uint32_t) * ((uint64_t)n + 1));
  // 4 ids of padding: 16-byte loads of aligned 4-edge groups may cover up to
  // 3 ids past the last list
  if (e == cudaSuccess) e = cudaMalloc(&g->d_edges, sizeof(uint32_t) * (m + 4));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_iso, sizeof(uint32_t) * g->nwords);
  if (e != cudaSuccess) {
    cudaFree(g->d_offsets);
    cudaFree(g->d_edges);
    cudaFree(g->d_iso);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA,
                std::string("graph allocation: ") + cudaGetErrorString(e));
  }
  *out = g;
  return PBG_OK;
}

// Validates the CSR now on the device and derives the degree-0 bitmap.
int finish_graph(pbg_graph* g) {
  unsigned* d_bad = nullptr;
  unsigned bad[2] = {0, 0};
  PBG_CUDA(cudaMalloc(&d_bad, 2 * sizeof(unsigned)));
  cudaError_t e = cudaMemsetAsync(d_bad, 0, 2 * sizeof(unsigned), g->stream);
  if (e == cudaSuccess) {
    k_validate<<<grid_for(g->m > g->n ? g->m : g->n, g->num_sms), 256, 0, g->stream>>>(g->d_offsets, g->d_edges,
                                                                                        g->n, g->m, d_bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(bad, d_bad, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(d_bad);
  if (e != cudaSuccess) return cuda_fail(e, "graph validation");
  if (bad[0] & 2u) return fail(PBG_ERR_ARG, "offsets[0] must be 0 and offsets[n] must equal m");
  if (bad[0] & 1u) return fail(PBG_ERR_ARG, "offsets must be non-decreasing");
  if (bad[0] & 4u) return fail(PBG_ERR_ARG, "an edge target is >= n");
  g->max_degree = bad[1];
  if (g->flags & PBG_GRAPH_DETECT_SYMMETRIC) {
    unsigned sbad = 0;
    PBG_CUDA(cudaMalloc(&d_bad, sizeof(unsigned)));
    e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), g->stream);
    if (e == cudaSuccess) {
      k_symmetric<<<grid_for(g->n, g->num_sms), 256, 0, g->stream>>>(g->d_offsets, g->d_edges, g->n, d_bad);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sbad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    cudaFree(d_bad);
    if (e != cudaSuccess) return cuda_fail(e, "symmetry test");
    g->flags = (g->flags & ~PBG_GRAPH_DETECT_SYMMETRIC) | (sbad == 0 ? PBG_GRAPH_SYMMETRIC : 0u);
  }
  k_iso_bitmap<<<(g->nwords + 255) / 256, 256, 0, g->stream>>>(g->d_offsets, g->n, g->nwords,
                                                                (g->flags & PBG_GRAPH_SYMMETRIC) ? 1 : 0, g->d_iso);
  PBG_CUDA(cudaGetLastError());
  PBG_CUDA(cudaStreamSynchronize(g->stream));
  return PBG_OK;
}

namespace {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
  template <class T>
  T* as() {
    return static_cast<T*>(p);
  }
};

// Sort 2*m packed keys, drop duplicates and sentinels, build the CSR into g.
int keys_to_graph(uint64_t* keys, uint64_t nkeys, uint32_t n, uint32_t shift, uint64_t sentinel,
                  pbg_graph** out, cudaStream_t s, int num_sms) {
  DevBuf sorted, uniq, nsel, tmp;
  PBG_CUDA(sorted.alloc(sizeof(uint64_t) * nkeys));
  PBG_CUDA(uniq.alloc(sizeof(uint64_t) * nkeys));
  PBG_CUDA(nsel.alloc(sizeof(unsigned long long)));
  const int end_bit = (int)std::min<uint32_t>(64, 2 * shift + 1);
  size_t t1 = 0, t2 = 0;
  PBG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, t1, keys, sorted.as<uint64_t>(), nkeys, 0, end_bit, s));
  PBG_CUDA(cub::DeviceSelect::Unique(nullptr, t2, sorted.as<uint64_t>(), uniq.as<uint64_t>(),
                                     nsel.as<unsigned long long>(), nkeys, s));
  PBG_CUDA(tmp.alloc(std::max(t1, t2)));
  size_t tb = std::max(t1, t2);
  PBG_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, keys, sorted.as<uint64_t>(), nkeys, 0, end_bit, s));
  tb = std::max(t1, t2);
  PBG_CUDA(cub::DeviceSelect::Unique(tmp.p, tb, sorted.as<uint64_t>(), uniq.as<uint64_t>(),
                                     nsel.as<unsigned long long>(), nkeys, s));
  unsigned long long nu = 0;
  PBG_CUDA(cudaMemcpyAsync(&nu, nsel.p, sizeof(nu), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  uint64_t m = nu;
  if (m > 0) {
    uint64_t last = 0;
    PBG_CUDA(cudaMemcpy(&last, uniq.as<uint64_t>() + (m - 1), sizeof(last), cudaMemcpyDeviceToHost));
    if (last == sentinel) m--;
  }
  pbg_graph* g = nullptr;
  int rc = new_handle(n, m, PBG_GRAPH_SYMMETRIC, &g);
  if (rc) return rc;
  k_keys_to_csr<<<grid_for(m + 1, num_sms), 256, 0, g->stream>>>(uniq.as<uint64_t>(), m, n, shift, g->d_offsets,
                                                                  g->d_edges);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess && m == 0) e = cudaMemset(g->d_offsets, 0, sizeof(uint32_t) * ((uint64_t)n + 1));
  if (e != cudaSuccess) {
    pbg_graph_free(g);
    return cuda_fail(e, "CSR build");
  }
  rc = finish_graph(g);
  if (rc) {
    pbg_graph_free(g);
    return rc;
  }
  *out = g;
  return PBG_OK;
}

}  // namespace
}  // namespace pbg

using namespace pbg;

extern "C" int pbg_graph_upload(const uint32_t* offsets, const uint32_t* edges, uint32_t n, uint64_t m,
                                uint32_t flags, pbg_graph** out) {
  if (!offsets || (m && !edges)) return fail(PBG_ERR_ARG, "offsets/edges is NULL");
  if (!out) return fail(PBG_ERR_ARG, "out is NULL");
  pbg_graph* g = nullptr;
  int rc = new_handle(n, m, flags, &g);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(g->d_offsets, offsets, sizeof(uint32_t) * ((uint64_t)n + 1),
                                  cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(g->d_edges, edges, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, g->stream);
  if (e != cudaSuccess) {
    pbg_graph_free(g);
    return cuda_fail(e, "graph upload");
  }
  rc = finish_graph(g);
  if (rc) {
    pbg_graph_free(g);
    return rc;
  }
  *out = g;
  return PBG_OK;
}

extern "C" int pbg_graph_upload_device(const uint32_t* d_offsets, const uint32_t* d_edges, uint32_t n, uint64_t m,
                                       uint32_t flags, pbg_graph** out) {
  if (!d_offsets || (m && !d_edges)) return fail(PBG_ERR_ARG, "offsets/edges is NULL");
  if (!out) return fail(PBG_ERR_ARG, "out is NULL");
  pbg_graph* g = nullptr;
  int rc = new_handle(n, m, flags, &g);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(g->d_offsets, d_offsets, sizeof(uint32_t) * ((uint64_t)n + 1),
                                  cudaMemcpyDeviceToDevice, g->stream);
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(g->d_edges, d_edges, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, g->stream);
  if (e != cudaSuccess) {
    pbg_graph_free(g);
    return cuda_fail(e, "graph upload");
  }
  rc = finish_graph(g);
  if (rc) {
    pbg_graph_free(g);
    return rc;
  }
  *out = g;
  return PBG_OK;
}

extern "C" int pbg_graph_generate(const pbg_gen_params* p, pbg_graph** out) {
  if (!p || !out) return fail(PBG_ERR_ARG, "NULL argument");
  uint64_t n = 0, nkeys = 0;
  if (p->kind == PBG_GEN_RMAT) {
    if (p->logn < 1 || p->logn > 30) return fail(PBG_ERR_ARG, "rmat: logn must be in [1, 30]");
    if (!(p->a >= 0 && p->b >= 0 && p->c >= 0 && p->a + p->b + p->c <= 1.0))
      return fail(PBG_ERR_ARG, "rmat: a + b + c must be <= 1 (rMatGraph.C:44-47)");
    n = 1ull << p->logn;
    nkeys = 2 * p->samples;
  } else if (p->kind == PBG_GEN_TORUS3D) {
    if (p->dn < 1) return fail(PBG_ERR_ARG, "torus: dn must be >= 1");
    n = (uint64_t)p->dn * p->dn * p->dn;
    nkeys = 6 * n;
  } else if (p->kind == PBG_GEN_RANDLOCAL) {
    if (p->n < 2) return fail(PBG_ERR_ARG, "randlocal: n must be >= 2");
    if (p->window < 1) return fail(PBG_ERR_ARG, "randlocal: window must be >= 1");
    n = p->n;
    nkeys = 2ull * p->n * p->degree;
  } else {
    return fail(PBG_ERR_ARG, "unknown generator kind");
  }
  if (n > PBG_MAX_VERTICES)
    return fail(PBG_ERR_ARG, "n must be below 2^31: vertex ids are int (bench/BFS.h:5)");
  const uint32_t shift = std::max<uint32_t>(1, ceil_log2(n));
  if (2 * shift + 1 > 64) return fail(PBG_ERR_ARG, "graph too large for packed keys");
  const uint64_t sentinel = 1ull << (2 * shift);

  int dev = 0, num_sms = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  PBG_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t s = nullptr;
  PBG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};

  DevBuf keys, perm;
  cudaError_t e = keys.alloc(sizeof(uint64_t) * nkeys);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PBG_ERR_OOM, "generator: key buffer allocation failed");
  }
  const int grid = grid_for(nkeys / 2 + 1, num_sms);
  if (p->kind == PBG_GEN_RMAT) {
    const uint64_t h = mix64(p->seed);
    k_gen_rmat<<<grid, 256, 0, s>>>(p->samples, h, p->logn, prob_threshold(p->a), prob_threshold(p->a + p->b),
                                    prob_threshold(p->a + p->b + p->c), shift, sentinel, keys.as<uint64_t>());
  } else if (p->kind == PBG_GEN_TORUS3D) {
    if (p->permute) {
      DevBuf pk, ps, tmp;
      PBG_CUDA(pk.alloc(sizeof(uint64_t) * n));
      PBG_CUDA(ps.alloc(sizeof(uint64_t) * n));
      PBG_CUDA(perm.alloc(sizeof(uint32_t) * n));
      k_perm_keys<<<grid_for(n, num_sms), 256, 0, s>>>((uint32_t)n, mix64(p->perm_seed), pk.as<uint64_t>());
      size_t tb = 0;
      PBG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, pk.as<uint64_t>(), ps.as<uint64_t>(), n, 0, 64, s));
      PBG_CUDA(tmp.alloc(tb));
      PBG_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, pk.as<uint64_t>(), ps.as<uint64_t>(), n, 0, 64, s));
      k_perm_scatter<<<grid_for(n, num_sms), 256, 0, s>>>((uint32_t)n, ps.as<uint64_t>(), perm.as<uint32_t>());
      PBG_CUDA(cudaGetLastError());
      PBG_CUDA(cudaStreamSynchronize(s));
    }
    k_gen_torus<<<grid, 256, 0, s>>>(p->dn, perm.as<uint32_t>(), shift, sentinel, keys.as<uint64_t>());
  } else {
    k_gen_randlocal<<<grid, 256, 0, s>>>(p->n, p->degree, p->window, mix64(p->seed), shift, sentinel,
                                         keys.as<uint64_t>());
  }
  PBG_CUDA(cudaGetLastError());
  return keys_to_graph(keys.as<uint64_t>(), nkeys, (uint32_t)n, shift, sentinel, out, s, num_sms);
}

extern "C" int pbg_graph_info(const pbg_graph* g, uint32_t* n, uint64_t* m, const uint32_t** d_offsets,
                              const uint32_t** d_edges) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (d_offsets) *d_offsets = g->d_offsets;
  if (d_edges) *d_edges = g->d_edges;
  return PBG_OK;
}

extern "C" int pbg_graph_flags(const pbg_graph* g, uint32_t* flags) {
  if (!g || !flags) return fail(PBG_ERR_ARG, "NULL argument");
  *flags = g->flags;
  return PBG_OK;
}

extern "C" int pbg_graph_download(const pbg_graph* g, uint32_t* offsets, uint32_t* edges) {
  if (!g || !offsets) return fail(PBG_ERR_ARG, "NULL argument");
  PBG_CUDA(cudaMemcpyAsync(offsets, g->d_offsets, sizeof(uint32_t) * ((uint64_t)g->n + 1), cudaMemcpyDeviceToHost,
                           g->stream));
  if (g->m && edges)
    PBG_CUDA(cudaMemcpyAsync(edges, g->d_edges, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  PBG_CUDA(cudaStreamSynchronize(g->stream));
  return PBG_OK;
}

extern "C" int pbg_graph_free(pbg_graph* g) {
  if (!g) return PBG_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  bfs_free_workspace(g);
  pbg_msbfs_free(g->ms_ws);
  pbg_batch_free(g->ms_batch);
  if (g->ws.ev0) cudaEventDestroy(g->ws.ev0);
  if (g->ws.ev1) cudaEventDestroy(g->ws.ev1);
  cudaFree(g->d_offsets);
  cudaFree(g->d_edges);
  cudaFree(g->d_iso);
  cudaFree(g->d_pull_chunks);
  cudaFree(g->mis_flags);
  cudaFree(g->mis_ctrl);
  cudaFree(g->check_buf);
  if (g->mis_ev0) cudaEventDestroy(g->mis_ev0);
  if (g->mis_ev1) cudaEventDestroy(g->mis_ev1);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return PBG_OK;
}
