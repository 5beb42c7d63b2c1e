// noalloc.cu -- pbg_bfs_noalloc: the single-source BFS for callers that
// cannot allocate device memory.  Has no counterpart in the reference.
//
// The caller owns the CSR and the outputs.  Everything else the persistent
// kernel needs (visited bitmaps, the degree-0 bitmap, frontier queues and
// their adjacency ranges, chunk queues, counters and the barrier, a
// validation word) is carved out of ONE
// file-scope device array, g_scratch, of PBG_NOALLOC_SCRATCH_BYTES.  The array
// is sized for n <= PBG_NOALLOC_MAX_VERTICES and m <= PBG_NOALLOC_MAX_EDGES
// with the default chunk threshold (32).  This file calls no cudaMalloc,
// cudaFree or allocating library routine; host-side results (the validation
// word, the error word) are read into local variables.
//
// In host code the name g_scratch is only a host-side stand-in for the
// device array: passing it to a kernel would fault, or silently touch the
// wrong memory where the GPU can reach host memory.  The first call on a
// device does its set-up there, with that device current: it reads the SM
// count and looks up the array's device address with cudaGetSymbolAddress
// (which loads this module on the device), so that first call should come
// before any stream capture.  Every later call looks the address up again
// (a host-side query: no allocation, no device work), so a context that was
// torn down and created again (cudaDeviceReset) never gets a stale address.
// All calls share the array and it keeps the last call's contents, so every
// call clears what must start at zero (counters, barrier) and the kernel
// rewrites the bitmaps; calls that overlap on the GPU race.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "internal.cuh"

namespace pbg {
namespace {

constexpr uint32_t NA_CHUNK_MIN_DEGREE = 32;  // the default chunk threshold the queues are sized for
constexpr size_t NA_WORDS = (((size_t)PBG_NOALLOC_MAX_VERTICES + 31) / 32 + 31) / 32 * 32;
constexpr size_t NA_BIG_CAP = (size_t)PBG_NOALLOC_MAX_EDGES / NA_CHUNK_MIN_DEGREE + 1 < PBG_NOALLOC_MAX_VERTICES
                                  ? (size_t)PBG_NOALLOC_MAX_EDGES / NA_CHUNK_MIN_DEGREE + 1
                                  : (size_t)PBG_NOALLOC_MAX_VERTICES;
constexpr size_t round256(size_t x) { return (x + 255) / 256 * 256; }

// Byte offsets of the pieces inside the array.
constexpr size_t OFF_BM0 = 0;
constexpr size_t OFF_BM1 = OFF_BM0 + round256(4 * NA_WORDS);
constexpr size_t OFF_ISO = OFF_BM1 + round256(4 * NA_WORDS);
constexpr size_t OFF_Q0 = OFF_ISO + round256(4 * NA_WORDS);
constexpr size_t OFF_Q1 = OFF_Q0 + round256(4 * (size_t)PBG_NOALLOC_MAX_VERTICES);
constexpr size_t OFF_QR0 = OFF_Q1 + round256(4 * (size_t)PBG_NOALLOC_MAX_VERTICES);
constexpr size_t OFF_QR1 = OFF_QR0 + round256(8 * (size_t)PBG_NOALLOC_MAX_VERTICES);
constexpr size_t OFF_QB0 = OFF_QR1 + round256(8 * (size_t)PBG_NOALLOC_MAX_VERTICES);
constexpr size_t OFF_QB1 = OFF_QB0 + round256(16 * NA_BIG_CAP);
constexpr size_t OFF_CTRL = OFF_QB1 + round256(16 * NA_BIG_CAP);
constexpr size_t OFF_BAD = OFF_CTRL + round256(sizeof(BfsCtrl));
constexpr size_t NA_USED = OFF_BAD + 256;
static_assert(NA_USED <= PBG_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds PBG_NOALLOC_SCRATCH_BYTES");

static __device__ __align__(256) unsigned char g_scratch[PBG_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
int g_sms[MAX_DEVICES] = {};  // set-up done on a device once its SM count is known

// Device address of g_scratch on `dev` (the current device).  The SM count
// is read once per device; the address is looked up on every call, since it
// belongs to the current context.
int scratch_on(int dev, unsigned char** out, int* sms) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
  if (!p) return fail(PBG_ERR_CUDA, "cudaGetSymbolAddress(scratch) returned NULL");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_sms[dev]) {
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "multiprocessor count");
    g_sms[dev] = n;
  }
  *out = static_cast<unsigned char*>(p);
  *sms = g_sms[dev];
  return PBG_OK;
}

__global__ void na_validate(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg, uint32_t n,
                            unsigned long long m, unsigned* bad) {
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long v = tid; v < n; v += nth)
    if (off[v] > off[v + 1]) atomicOr(bad, 1u);
  if (tid == 0 && (off[0] != 0 || (unsigned long long)off[n] != m)) atomicOr(bad, 2u);
  for (unsigned long long i = tid; i < m; i += nth)
    if (edg[i] >= n) atomicOr(bad, 4u);
}

__global__ void na_iso(const uint32_t* __restrict__ off, uint32_t n, uint32_t nwords, int symmetric,
                       uint32_t* __restrict__ iso) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwords) return;
  uint32_t x = 0;
  for (int b = 0; b < 32; b++) {
    const unsigned long long v = (unsigned long long)w * 32 + b;
    if (v >= n)
      x |= 1u << b;
    else if (symmetric && off[v] == off[v + 1])
      x |= 1u << b;
  }
  iso[w] = x;
}

}  // namespace
}  // namespace pbg

using namespace pbg;

extern "C" int pbg_bfs_noalloc(const uint32_t* d_offsets, const uint32_t* d_edges, uint32_t n, uint64_t m,
                               uint32_t flags, uint32_t src, uint32_t parent_mode, uint32_t* d_parent,
                               uint32_t* d_level, void* stream) {
  if (!d_offsets || (m && !d_edges) || !d_parent) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: NULL argument");
  if (n == 0 || n > PBG_NOALLOC_MAX_VERTICES)
    return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: n must be in [1, PBG_NOALLOC_MAX_VERTICES = 2^20]");
  if (m > PBG_NOALLOC_MAX_EDGES) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: m exceeds PBG_NOALLOC_MAX_EDGES = 2^24");
  if (src >= n) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: source vertex out of range");
  if (parent_mode > PBG_PARENT_MAX) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: unknown parent_mode");
  if (flags & ~PBG_GRAPH_SYMMETRIC) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: flags must be 0 or PBG_GRAPH_SYMMETRIC");
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: device ordinal too large");
  unsigned char* base = nullptr;
  int sms = 0;
  int rc = scratch_on(dev, &base, &sms);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // validate the CSR (its result is read into a local variable)
  unsigned* d_bad = reinterpret_cast<unsigned*>(base + OFF_BAD);
  PBG_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s));
  const unsigned long long work = (m > n) ? m : n;
  unsigned long long blocks = (work + 255) / 256;
  if (blocks > (unsigned long long)sms * 16) blocks = (unsigned long long)sms * 16;
  na_validate<<<(unsigned)(blocks ? blocks : 1), 256, 0, s>>>(d_offsets, d_edges, n, m, d_bad);
  PBG_CUDA(cudaGetLastError());
  unsigned bad = 0;
  PBG_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  if (bad & 2u) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: offsets[0] must be 0 and offsets[n] must equal m");
  if (bad & 1u) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: offsets must be non-decreasing");
  if (bad & 4u) return fail(PBG_ERR_ARG, "pbg_bfs_noalloc: an edge target is >= n");

  const uint32_t nwords = (uint32_t)((((uint64_t)n + 31) / 32 + 31) / 32 * 32);
  BfsOnArgs r;
  r.offsets = d_offsets;
  r.edges = d_edges;
  r.iso = reinterpret_cast<uint32_t*>(base + OFF_ISO);
  r.parent = d_parent;
  r.level = d_level;
  r.bm0 = reinterpret_cast<uint32_t*>(base + OFF_BM0);
  r.bm1 = reinterpret_cast<uint32_t*>(base + OFF_BM1);
  r.q0 = reinterpret_cast<uint32_t*>(base + OFF_Q0);
  r.q1 = reinterpret_cast<uint32_t*>(base + OFF_Q1);
  r.qr0 = reinterpret_cast<uint2*>(base + OFF_QR0);
  r.qr1 = reinterpret_cast<uint2*>(base + OFF_QR1);
  r.qb0 = reinterpret_cast<uint4*>(base + OFF_QB0);
  r.qb1 = reinterpret_cast<uint4*>(base + OFF_QB1);
  r.ctrl = reinterpret_cast<BfsCtrl*>(base + OFF_CTRL);
  r.m = m;
  r.n = n;
  r.nwords = nwords;
  const uint64_t cap = m / NA_CHUNK_MIN_DEGREE + 1;
  r.big_cap = (uint32_t)(cap < n ? cap : n);
  r.src = src;
  r.symmetric = (flags & PBG_GRAPH_SYMMETRIC) ? 1u : 0u;

  na_iso<<<(nwords + 255) / 256, 256, 0, s>>>(d_offsets, n, nwords, r.symmetric, const_cast<uint32_t*>(r.iso));
  PBG_CUDA(cudaGetLastError());
  // counters and barrier start at zero; the kernel initialises the rest
  PBG_CUDA(cudaMemsetAsync(r.ctrl, 0, sizeof(BfsCtrl), s));
  pbg_bfs_opts o;
  pbg_bfs_opts_default(&o);
  o.parent_mode = parent_mode;
  resolve_opts(&o, &o);
  o.chunk_min_degree = NA_CHUNK_MIN_DEGREE;
  rc = bfs_launch_on(r, o, sms, s);
  if (rc) return rc;
  unsigned err = 0;
  PBG_CUDA(cudaMemcpyAsync(&err, &r.ctrl->sync.error, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  if (err & ERR_BARRIER_TIMEOUT) return fail(PBG_ERR_TIMEOUT, "pbg_bfs_noalloc: a grid barrier wait ran out");
  if (err) return fail(PBG_ERR_STATE, "pbg_bfs_noalloc: device error word set");
  return PBG_OK;
}
