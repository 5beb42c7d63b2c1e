// autotune.cu -- a small autotuner for the options of one resident graph.
//
// No reference counterpart: PBBS fixes its switch constants in the source
// (alpha = beta = 20, common/ligraLight.h:122,130) and its block sizes in
// the scheduler.  Here the CTA size, the degree from which a frontier list
// is cut into chunks, and the direction switch of the single-source search
// (or the switch of the batched search) are picked per graph by coordinate
// descent: each option in turn takes every candidate value with the others
// held, the fastest (summed device time over the caller's sample sources,
// after an untimed pass) is kept, and the sweep runs twice.  The result is
// stored on the graph and used by every call that passes no options.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "internal.cuh"
#include "msbfs.cuh"

using namespace pbg;

namespace {

struct Timer {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Timer() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// Single-source searches from every sample source: one untimed pass, then
// the device time of a second.
int time_single(pbg_graph* g, const std::vector<uint32_t>& srcs, const pbg_bfs_opts& o, uint32_t* d_parent,
                uint32_t* d_level, Timer& t, float* ms) {
  for (int pass = 0; pass < 2; pass++) {
    if (pass == 1) PBG_CUDA(cudaEventRecord(t.e0, g->stream));
    for (uint32_t s : srcs) {
      int rc = bfs_launch(g, s, o, d_parent, d_level, g->stream);
      if (rc) return rc;
    }
    if (pass == 1) PBG_CUDA(cudaEventRecord(t.e1, g->stream));
    PBG_CUDA(cudaStreamSynchronize(g->stream));
    int rc = bfs_read_stats(g, nullptr);
    if (rc) return rc;
  }
  PBG_CUDA(cudaEventElapsedTime(ms, t.e0, t.e1));
  return PBG_OK;
}

// One batched job of all sample sources: one untimed launch, then the device
// time of a second.
int time_multi(pbg_graph* g, const std::vector<uint32_t>& srcs, const pbg_bfs_opts& o, uint8_t* d_levels,
               float* ms) {
  pbg_batch_job job{g->ms_ws, srcs.data(), (uint32_t)srcs.size(), d_levels};
  for (int pass = 0; pass < 2; pass++) {
    int rc = batch_launch(g->ms_batch, &job, 1, &o, g->stream, 0);
    if (rc) return rc;
    PBG_CUDA(cudaStreamSynchronize(g->stream));
    pbg_batch_stats st;
    rc = pbg_batch_job_stats(g->ms_batch, g->ms_ws, &st);
    if (rc) return rc;
    *ms = st.device_ms;
  }
  return PBG_OK;
}

using Key = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;

}  // namespace

extern "C" int pbg_autotune(pbg_graph* g, const uint32_t* srcs, uint32_t nsrc, uint32_t flags, pbg_bfs_opts* inout,
                            pbg_tune_report* rep) {
  if (!g || !srcs) return fail(PBG_ERR_ARG, "NULL argument");
  const bool multi = (flags & PBG_TUNE_BATCHED) != 0;
  if (nsrc < 1 || nsrc > (multi ? MS_MAX_SOURCES : PBG_TUNE_MAX_SOURCES))
    return fail(PBG_ERR_ARG, multi ? "batched tuning takes 1..256 sources" : "tuning takes 1..16 sources");
  if (flags & ~(PBG_TUNE_BATCHED | PBG_TUNE_NO_STORE)) return fail(PBG_ERR_ARG, "unknown tuning flags");
  for (uint32_t i = 0; i < nsrc; i++)
    if (srcs[i] >= g->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  if (multi && !(g->flags & PBG_GRAPH_SYMMETRIC)) return fail(PBG_ERR_ARG, "batched tuning needs a symmetric graph");
  std::vector<uint32_t> src(srcs, srcs + nsrc);

  pbg_bfs_opts best;
  resolve_opts(nullptr, &best);
  if (inout) {  // the caller's parent mode and direction policy are kept
    best.parent_mode = inout->parent_mode;
    best.direction = inout->direction;
  }
  Timer t;
  PBG_CUDA(cudaEventCreate(&t.e0));
  PBG_CUDA(cudaEventCreate(&t.e1));
  uint32_t* d_parent = nullptr;
  uint32_t* d_level = nullptr;
  uint8_t* d_levels = nullptr;
  struct Free {
    void* p[3];
    ~Free() {
      for (void* q : p) cudaFree(q);
    }
  } bufs{};
  int rc = PBG_OK;
  if (multi) {
    // a workspace of the graph's narrower than the sample is replaced by
    // one of the sample's width (as pbg_bfs_multi does)
    if (g->ms_ws && 64 * g->ms_ws->words < nsrc) {
      pbg_msbfs_free(g->ms_ws);
      g->ms_ws = nullptr;
    }
    if (!g->ms_ws && (rc = pbg_msbfs_create_k(g, &best, std::max<uint32_t>(nsrc, 64), &g->ms_ws))) return rc;
    if (!g->ms_batch && (rc = pbg_batch_create(1, &g->ms_batch))) return rc;
    PBG_CUDA(cudaMalloc(&d_levels, (size_t)nsrc * g->n));
    bufs.p[2] = d_levels;
  } else {
    PBG_CUDA(cudaMalloc(&d_parent, sizeof(uint32_t) * g->n));
    bufs.p[0] = d_parent;
    PBG_CUDA(cudaMalloc(&d_level, sizeof(uint32_t) * g->n));
    bufs.p[1] = d_level;
  }

  std::map<Key, float> seen;
  uint32_t evals = 0;
  auto eval = [&](const pbg_bfs_opts& o, float* ms) -> int {
    const Key k{o.block_threads, o.chunk_min_degree, o.alpha, o.beta};
    auto it = seen.find(k);
    if (it != seen.end()) {
      *ms = it->second;
      return PBG_OK;
    }
    int r = multi ? time_multi(g, src, o, d_levels, ms) : time_single(g, src, o, d_parent, d_level, t, ms);
    if (r) return r;
    seen[k] = *ms;
    evals++;
    return PBG_OK;
  };

  float best_ms = 0.f;
  if ((rc = eval(best, &best_ms))) return rc;
  const float default_ms = best_ms;
  struct Axis {
    uint32_t pbg_bfs_opts::*field;
    std::vector<uint32_t> values;
  };
  std::vector<Axis> axes;
  if (multi) {
    // the batched switch only: pull when rem * alpha <= fdeg * beta * 2
    axes.push_back({&pbg_bfs_opts::alpha, {2, 5, 10, 20, 40, 80}});
  } else {
    axes.push_back({&pbg_bfs_opts::block_threads, {256, 512, 1024}});
    axes.push_back({&pbg_bfs_opts::chunk_min_degree, {16, 32, 64, 128, 256}});
    axes.push_back({&pbg_bfs_opts::alpha, {5, 10, 20, 40}});
    axes.push_back({&pbg_bfs_opts::beta, {5, 10, 20, 40}});
  }
  for (int round = 0; round < 2; round++) {
    for (const Axis& ax : axes) {
      for (uint32_t v : ax.values) {
        pbg_bfs_opts o = best;
        o.*ax.field = v;
        float ms = 0.f;
        if ((rc = eval(o, &ms))) return rc;
        if (ms < best_ms) {
          best_ms = ms;
          best = o;
        }
      }
    }
  }
  if (!(flags & PBG_TUNE_NO_STORE)) {
    if (multi) {
      g->tuned_multi = best;
      g->has_tuned_multi = true;
    } else {
      g->tuned = best;
      g->has_tuned = true;
    }
  }
  if (inout) *inout = best;
  if (rep) {
    rep->evaluations = evals;
    rep->default_ms = default_ms;
    rep->best_ms = best_ms;
  }
  return PBG_OK;
}

extern "C" int pbg_autotune_clear(pbg_graph* g) {
  if (!g) return fail(PBG_ERR_ARG, "graph is NULL");
  g->has_tuned = false;
  g->has_tuned_multi = false;
  return PBG_OK;
}
