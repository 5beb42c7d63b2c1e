// msbfs_api.cu -- host side of the batched multi-source BFS: job
// workspaces, batch objects (descriptor staging + barrier), the fused launch
// and the one-graph convenience call.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <set>

#include "internal.cuh"
#include "msbfs.cuh"

using namespace pbg;

namespace {

// Entries of the big-vertex queue: the vertices of degree >= big_deg of a
// sparse push frontier, and the (distinct) sources of level 0.
uint32_t big_cap_for(const pbg_graph* g, uint32_t big_deg) {
  const uint64_t cap = std::max<uint64_t>(g->m / std::max(big_deg, 1u) + 1, MS_MAX_SOURCES);
  return (uint32_t)std::min<uint64_t>(g->n, cap);
}

__global__ void pull_chunk_count(const uint32_t* __restrict__ off, uint32_t n, uint32_t* __restrict__ cnt) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    const uint32_t d = off[v + 1] - off[v];
    cnt[v] = d > MS_PULL_SERIAL ? (d - MS_PULL_SERIAL + MS_PULL_CHUNK - 1) / MS_PULL_CHUNK : 0u;
  } else if (v == n) {
    cnt[n] = 0;
  }
}

__global__ void pull_chunk_fill(const uint32_t* __restrict__ off, uint32_t n, const uint32_t* __restrict__ start,
                                uint4* __restrict__ out) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint32_t s = start[v], c = start[v + 1] - s, b = off[v] + MS_PULL_SERIAL, e = off[v + 1];
  for (uint32_t i = 0; i < c; i++) {
    const uint32_t cb = b + i * MS_PULL_CHUNK;
    out[s + i] = make_uint4(v, cb, min(e, cb + MS_PULL_CHUNK), e - off[v]);
  }
}

std::mutex g_pc_mu;

}  // namespace

int pbg::ms_pull_chunks(pbg_graph* g) {
  std::lock_guard<std::mutex> lk(g_pc_mu);
  if (g->pull_chunks_built) return PBG_OK;
  const uint32_t n = g->n;
  uint32_t* cnt = nullptr;
  void* tmp = nullptr;
  size_t tb = 0;
  cudaStream_t s = g->stream;
  auto done = [&](int rc) {
    cudaFree(cnt);
    cudaFree(tmp);
    return rc;
  };
  PBG_CUDA(cudaMalloc(&cnt, sizeof(uint32_t) * 2 * ((size_t)n + 1)));
  uint32_t* start = cnt + n + 1;
  const uint32_t blocks = (n + 1 + 255) / 256;
  pull_chunk_count<<<blocks, 256, 0, s>>>(g->d_offsets, n, cnt);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, start, n + 1, s);
  if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, start, n + 1, s);
  uint32_t total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, start + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && total) e = cudaMalloc(&g->d_pull_chunks, sizeof(uint4) * (size_t)total);
  if (e == cudaSuccess && total) {
    pull_chunk_fill<<<(n + 255) / 256, 256, 0, s>>>(g->d_offsets, n, start, g->d_pull_chunks);
    e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    cudaFree(g->d_pull_chunks);
    g->d_pull_chunks = nullptr;
    cudaGetLastError();
    return done(cuda_fail(e, "pull chunk table"));
  }
  g->n_pull_chunks = total;
  g->pull_chunks_built = true;
  return done(PBG_OK);
}

namespace {
uint32_t words_for(uint32_t max_sources) { return max_sources > 128 ? 4u : max_sources > 64 ? 2u : 1u; }
}  // namespace

extern "C" uint64_t pbg_msbfs_bytes_k(const pbg_graph* g, const pbg_bfs_opts* opts, uint32_t max_sources) {
  if (!g || max_sources < 1 || max_sources > MS_MAX_SOURCES) return 0;
  pbg_bfs_opts o;
  resolve_opts(opts, &o);
  const uint64_t n = g->n, w = words_for(max_sources);
  return (1 + MS_PLANES) * 8 * w * n + (w > 1 ? 4 * ((n + 31) / 32) : 0) + 2 * 4 * n +
         2 * 16ull * big_cap_for(g, ms_big_degree(o)) + sizeof(MsJobCtrl);
}

extern "C" uint64_t pbg_msbfs_bytes(const pbg_graph* g, const pbg_bfs_opts* opts) {
  return pbg_msbfs_bytes_k(g, opts, 64);
}

extern "C" int pbg_msbfs_create(pbg_graph* g, const pbg_bfs_opts* opts, pbg_msbfs** out) {
  return pbg_msbfs_create_k(g, opts, 64, out);
}

extern "C" int pbg_msbfs_create_k(pbg_graph* g, const pbg_bfs_opts* opts, uint32_t max_sources, pbg_msbfs** out) {
  if (!g || !out) return fail(PBG_ERR_ARG, "NULL argument");
  if (max_sources < 1 || max_sources > MS_MAX_SOURCES) return fail(PBG_ERR_ARG, "max_sources must be in [1, 256]");
  pbg_bfs_opts o;
  resolve_opts(opts, &o);
  int rc = ms_pull_chunks(g);
  if (rc) return rc;
  pbg_msbfs* w = new pbg_msbfs();
  w->g = g;
  w->words = words_for(max_sources);
  w->big_min_degree = o.chunk_min_degree;
  w->big_cap = big_cap_for(g, ms_big_degree(o));
  const size_t n = g->n;
  cudaError_t e = cudaMalloc(&w->vis, 8 * n * w->words);
  if (e == cudaSuccess) e = cudaMalloc(&w->planes, 8 * n * w->words * MS_PLANES);
  if (e == cudaSuccess && w->words > 1) e = cudaMalloc(&w->fbits, 4 * ((n + 31) / 32));
  if (e == cudaSuccess) e = cudaMalloc(&w->q0, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&w->q1, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&w->qb0, 16 * (size_t)w->big_cap);
  if (e == cudaSuccess) e = cudaMalloc(&w->qb1, 16 * (size_t)w->big_cap);
  if (e == cudaSuccess) e = cudaMalloc(&w->ctrl, sizeof(MsJobCtrl));
  if (e != cudaSuccess) {
    pbg_msbfs_free(w);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA,
                std::string("multi-source workspace: ") + cudaGetErrorString(e));
  }
  *out = w;
  return PBG_OK;
}

extern "C" int pbg_msbfs_free(pbg_msbfs* w) {
  if (!w) return PBG_OK;
  cudaFree(w->vis);
  cudaFree(w->planes);
  cudaFree(w->fbits);
  cudaFree(w->q0);
  cudaFree(w->q1);
  cudaFree(w->qb0);
  cudaFree(w->qb1);
  cudaFree(w->ctrl);
  cudaFree(w->levels);
  delete w;
  return PBG_OK;
}

extern "C" int pbg_batch_create(uint32_t max_jobs, pbg_batch** out) {
  if (!out || max_jobs < 1 || max_jobs > MS_MAX_JOBS) return fail(PBG_ERR_ARG, "max_jobs must be in [1, 128]");
  pbg_batch* b = new pbg_batch();
  b->max_jobs = max_jobs;
  cudaError_t e = cudaGetDevice(&b->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_jobs, sizeof(MsJob) * max_jobs);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_jobs, sizeof(MsJob) * max_jobs);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_srcs, sizeof(uint32_t) * MS_MAX_SOURCES * max_jobs);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_srcs, sizeof(uint32_t) * MS_MAX_SOURCES * max_jobs);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_sync, sizeof(dev::GridSync));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e != cudaSuccess) {
    pbg_batch_free(b);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA,
                std::string("batch: ") + cudaGetErrorString(e));
  }
  *out = b;
  return PBG_OK;
}

extern "C" int pbg_batch_free(pbg_batch* b) {
  if (!b) return PBG_OK;
  if (b->staged) cudaEventSynchronize(b->staged);
  if (b->ev1) cudaEventSynchronize(b->ev1);
  cudaFree(b->d_jobs);
  cudaFreeHost(b->h_jobs);
  cudaFree(b->d_srcs);
  cudaFreeHost(b->h_srcs);
  cudaFree(b->d_sync);
  if (b->staged) cudaEventDestroy(b->staged);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
  return PBG_OK;
}

extern "C" int pbg_bfs_batch(pbg_batch* b, const pbg_batch_job* jobs, uint32_t njobs, const pbg_bfs_opts* opts,
                             void* stream) {
  return batch_launch(b, jobs, njobs, opts, static_cast<cudaStream_t>(stream), 0);
}

int pbg::batch_launch(pbg_batch* b, const pbg_batch_job* jobs, uint32_t njobs, const pbg_bfs_opts* opts,
                      cudaStream_t s, int max_blocks) {
  if (!b || !jobs) return fail(PBG_ERR_ARG, "NULL argument");
  if (njobs < 1 || njobs > b->max_jobs) return fail(PBG_ERR_ARG, "njobs out of range for this batch");
  pbg_bfs_opts o;
  resolve_opts(opts, &o);
  if (o.direction > PBG_DIR_BOTTOMUP) return fail(PBG_ERR_ARG, "unknown direction policy");
  if (o.chunk_min_degree < 1) return fail(PBG_ERR_ARG, "chunk_min_degree must be >= 1");
  std::set<const pbg_msbfs*> seen;
  const uint32_t words = (jobs && jobs[0].ws) ? jobs[0].ws->words : 1;
  for (uint32_t j = 0; j < njobs; j++) {
    const pbg_batch_job& J = jobs[j];
    if (!J.ws || !J.ws->g || !J.srcs || !J.d_levels) return fail(PBG_ERR_ARG, "job has a NULL field");
    if (J.k < 1 || J.k > 64 * J.ws->words)
      return fail(PBG_ERR_ARG, "a job needs 1 .. (the workspace's max_sources) sources");
    if (J.ws->words != words)
      return fail(PBG_ERR_ARG, "one launch takes workspaces of one size class (up to 64, 128 or 256 sources)");
    if (reinterpret_cast<uintptr_t>(J.d_levels) % 16) return fail(PBG_ERR_ARG, "d_levels must be 16-byte aligned");
    if (!seen.insert(J.ws).second) return fail(PBG_ERR_ARG, "a workspace appears twice in one launch");
    if (J.ws->g->device != b->device) return fail(PBG_ERR_ARG, "job graph on another device");
    if (o.chunk_min_degree < J.ws->big_min_degree)
      return fail(PBG_ERR_ARG, "chunk_min_degree below the one the workspace was sized for");
    if (o.direction == PBG_DIR_BOTTOMUP && !(J.ws->g->flags & PBG_GRAPH_SYMMETRIC))
      return fail(PBG_ERR_ARG, "bottom-up needs a symmetric graph");
    for (uint32_t i = 0; i < J.k; i++)
      if (J.srcs[i] >= J.ws->g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  }
  // the pinned staging buffers are reused: wait until the previous launch's
  // copies out of them have been done
  PBG_CUDA(cudaEventSynchronize(b->staged));
  for (uint32_t j = 0; j < njobs; j++) {
    const pbg_batch_job& J = jobs[j];
    pbg_msbfs* w = J.ws;
    pbg_graph* g = w->g;
    std::memcpy(b->h_srcs + MS_MAX_SOURCES * j, J.srcs, sizeof(uint32_t) * J.k);
    MsJob& d = b->h_jobs[j];
    d.offsets = g->d_offsets;
    d.edges = g->d_edges;
    d.m = g->m;
    for (uint32_t q = 0; q < 4; q++) {
      const uint32_t kq = (J.k > 64 * q) ? std::min<uint32_t>(J.k - 64 * q, 64) : 0;
      d.all[q] = (kq == 64) ? ~0ull : ((1ull << kq) - 1);
    }
    d.n = g->n;
    d.k = J.k;
    d.symmetric = (g->flags & PBG_GRAPH_SYMMETRIC) ? 1u : 0u;
    d.big_cap = w->big_cap;
    d.vis = w->vis;
    d.planes = w->planes;
    d.fbits = w->fbits;
    d.q0 = w->q0;
    d.q1 = w->q1;
    d.qb0 = w->qb0;
    d.qb1 = w->qb1;
    d.levels = J.d_levels;
    d.srcs = b->d_srcs + MS_MAX_SOURCES * j;
    d.ctrl = w->ctrl;
    d.pchunks = g->d_pull_chunks;
    d.npc = g->n_pull_chunks;
    d.direct = ms_direct_levels(g->n, g->m);
    pbg_bfs_opts jo;  // the switch: the call's options, else the graph's tuned ones
    resolve_graph_opts(g, opts, true, &jo);
    d.alpha = jo.alpha;
    d.beta = jo.beta;
    w->last_k = J.k;
    PBG_CUDA(cudaMemsetAsync(w->ctrl, 0, sizeof(MsJobCtrl), s));
  }
  PBG_CUDA(cudaMemcpyAsync(b->d_srcs, b->h_srcs, sizeof(uint32_t) * MS_MAX_SOURCES * njobs, cudaMemcpyHostToDevice,
                           s));
  PBG_CUDA(cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(MsJob) * njobs, cudaMemcpyHostToDevice, s));
  PBG_CUDA(cudaEventRecord(b->staged, s));
  PBG_CUDA(cudaMemsetAsync(b->d_sync, 0, sizeof(dev::GridSync), s));
  PBG_CUDA(cudaEventRecord(b->ev0, s));
  int rc = ms_launch(b->d_jobs, njobs, o, b->d_sync, b->num_sms, s, max_blocks, words);
  if (rc) return rc;
  PBG_CUDA(cudaEventRecord(b->ev1, s));
  b->pending = true;
  return PBG_OK;
}

extern "C" int pbg_batch_job_stats(pbg_batch* b, pbg_msbfs* ws, pbg_batch_stats* st) {
  if (!b || !ws || !st) return fail(PBG_ERR_ARG, "NULL argument");
  PBG_CUDA(cudaEventSynchronize(b->ev1));
  MsJobCtrl c;
  dev::GridSync gs;
  PBG_CUDA(cudaMemcpy(&c, ws->ctrl, sizeof(c), cudaMemcpyDeviceToHost));
  PBG_CUDA(cudaMemcpy(&gs, b->d_sync, sizeof(gs), cudaMemcpyDeviceToHost));
  float ms = 0.f;
  PBG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  st->levels = c.levels;
  st->pull_levels = c.pull_levels;
  st->push_levels = c.push_levels;
  st->error = c.error | (gs.error ? MS_ERR_TIMEOUT : 0u);
  st->device_ms = ms;
  if (gs.error) return fail(PBG_ERR_TIMEOUT, "multi-source BFS: a grid barrier wait ran out");
  if (c.error & MS_ERR_OVERFLOW) return fail(PBG_ERR_OVERFLOW, "multi-source BFS: a level does not fit in uint8");
  if (c.error) return fail(PBG_ERR_STATE, "multi-source BFS: device error word set");
  return PBG_OK;
}

extern "C" int pbg_batch_job_trace(pbg_batch* b, pbg_msbfs* ws, pbg_level_trace* out, uint32_t cap,
                                   uint32_t* count) {
  if (!b || !ws || !count || (cap && !out)) return fail(PBG_ERR_ARG, "NULL argument");
  PBG_CUDA(cudaEventSynchronize(b->ev1));
  MsJobCtrl c;
  PBG_CUDA(cudaMemcpy(&c, ws->ctrl, sizeof(c), cudaMemcpyDeviceToHost));
  const uint32_t nl = std::min<uint32_t>(c.levels, MS_TRACE_LEVELS);
  uint32_t k = 0;
  for (; k < nl && k < cap; k++) {
    out[k].level = k;
    out[k].bottom_up = c.t_pull[k];
    out[k].frontier = c.t_nf[k];
    out[k].frontier_degree = c.t_deg[k];
    out[k].ms = (c.t_ns[k + 1] - c.t_ns[k]) * 1e-6;
  }
  *count = k;
  return PBG_OK;
}

extern "C" int pbg_bfs_multi_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count) {
  if (!g) return fail(PBG_ERR_ARG, "NULL argument");
  if (!g->ms_ws || !g->ms_batch) return fail(PBG_ERR_STATE, "no batched search has run on this graph");
  return pbg_batch_job_trace(g->ms_batch, g->ms_ws, out, cap, count);
}

extern "C" int pbg_bfs_multi(pbg_graph* g, const uint32_t* srcs, uint32_t k, const pbg_bfs_opts* opts,
                             uint8_t* levels_out, pbg_batch_stats* st) {
  if (!g || !srcs || !levels_out) return fail(PBG_ERR_ARG, "NULL argument");
  if (k < 1 || k > MS_MAX_SOURCES) return fail(PBG_ERR_ARG, "k must be in [1, 256]");
  pbg_bfs_opts o;
  resolve_graph_opts(g, opts, true, &o);
  if (g->ms_ws && (g->ms_ws->big_min_degree > o.chunk_min_degree || g->ms_ws->words != words_for(k))) {
    pbg_msbfs_free(g->ms_ws);
    g->ms_ws = nullptr;
  }
  int rc;
  if (!g->ms_ws && (rc = pbg_msbfs_create_k(g, &o, k, &g->ms_ws))) return rc;
  if (!g->ms_batch && (rc = pbg_batch_create(1, &g->ms_batch))) return rc;
  pbg_msbfs* w = g->ms_ws;
  const size_t bytes = (size_t)k * g->n;
  if (w->levels_bytes < bytes) {
    cudaFree(w->levels);
    w->levels = nullptr;
    w->levels_bytes = 0;
    PBG_CUDA(cudaMalloc(&w->levels, (size_t)64 * w->words * g->n));
    w->levels_bytes = (size_t)64 * w->words * g->n;
  }
  pbg_batch_job job{w, srcs, k, w->levels};
  rc = pbg_bfs_batch(g->ms_batch, &job, 1, &o, g->stream);
  if (rc) return rc;
  PBG_CUDA(cudaMemcpyAsync(levels_out, w->levels, bytes, cudaMemcpyDeviceToHost, g->stream));
  PBG_CUDA(cudaStreamSynchronize(g->stream));
  pbg_batch_stats tmp;
  return pbg_batch_job_stats(g->ms_batch, w, st ? st : &tmp);
}
