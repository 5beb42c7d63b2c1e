// capi.cu -- the extern "C" entry points of include/pbbs_bfs.h that are not
// graph construction, and the thread-local error message.
#include <cuda_runtime.h>

#include <string>

#include "internal.cuh"

namespace pbg {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? PBG_ERR_OOM : PBG_ERR_CUDA;
}

}  // namespace pbg

using namespace pbg;

extern "C" const char* pbg_last_error(void) { return g_last_error.c_str(); }

extern "C" void pbg_bfs_opts_default(pbg_bfs_opts* o) {
  if (!o) return;
  o->parent_mode = PBG_PARENT_ANY;
  o->direction = PBG_DIR_AUTO;
  o->alpha = 20;
  o->beta = 20;
  o->block_threads = 0;
  o->chunk_min_degree = 0;
}

extern "C" int pbg_bfs_device(pbg_graph* g, uint32_t src, const pbg_bfs_opts* opts, uint32_t* d_parent,
                              uint32_t* d_level, void* stream) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  if (!d_parent) return fail(PBG_ERR_ARG, "d_parent is NULL");
  if (src >= g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  pbg_bfs_opts o;
  resolve_graph_opts(g, opts, false, &o);
  return bfs_launch(g, src, o, d_parent, d_level, static_cast<cudaStream_t>(stream));
}

extern "C" int pbg_bfs_stats_get(pbg_graph* g, pbg_bfs_stats* stats) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  return bfs_read_stats(g, stats);
}

extern "C" int pbg_bfs_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count) {
  if (!g || (!out && cap)) return fail(PBG_ERR_ARG, "NULL argument");
  return bfs_read_trace(g, out, cap, count);
}

extern "C" int pbg_bfs(pbg_graph* g, uint32_t src, const pbg_bfs_opts* opts, int32_t* parent_out,
                       uint32_t* level_out, pbg_bfs_stats* stats) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  if (src >= g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  pbg_bfs_opts o;
  resolve_graph_opts(g, opts, false, &o);
  int rc = bfs_ensure_workspace(g, o);
  if (rc) return rc;
  BfsWorkspace& w = g->ws;
  if (!w.parent) PBG_CUDA(cudaMalloc(&w.parent, sizeof(uint32_t) * g->n));
  if (level_out && !w.level) PBG_CUDA(cudaMalloc(&w.level, sizeof(uint32_t) * g->n));
  rc = bfs_launch(g, src, o, w.parent, level_out ? w.level : nullptr, g->stream);
  if (rc) return rc;
  if (parent_out)
    PBG_CUDA(cudaMemcpyAsync(parent_out, w.parent, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, g->stream));
  if (level_out)
    PBG_CUDA(cudaMemcpyAsync(level_out, w.level, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, g->stream));
  PBG_CUDA(cudaStreamSynchronize(g->stream));
  return bfs_read_stats(g, stats);
}
