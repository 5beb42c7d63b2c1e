// server.cu -- continuous-batching BFS service (pbg_server_*).  No reference
// counterpart: PBBS answers one source per BFS() call.
//
// One scheduler thread owns all CUDA work.  Each scheduling round it
//   1. retires launches whose completion callback has fired: job statistics
//      and checksums were copied to pinned memory on the launch's stream, so
//      retiring needs no synchronising call; results are posted and the job
//      slots and the launch slot are freed;
//   2. admits pending queries into jobs (one job per graph, up to max_sources
//      of that graph's queries in arrival order, each job needing a free
//      pre-allocated slot of that graph; graphs are served oldest request
//      first, and a launch only takes graphs within a factor of four in edge
//      count of its first job's) and, while a launch slot is free, enqueues a fused launch of
//      those jobs on that slot's stream, followed by the checksum kernel, the
//      copies to pinned memory and a host callback.
// Launch slots run on their own streams with 1/streams of the resident
// blocks, so several fused launches are on the GPU at once.  Queries that
// arrive while launches run wait only for the next free slot (continuous
// batching at launch granularity); a graph's queries beyond its free job
// slots wait for one to be retired (admission by the memory budget).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"
#include "msbfs.cuh"

using namespace pbg;

namespace {

using clock_t_ = std::chrono::steady_clock;

struct Request {
  uint64_t id;
  uint32_t graph;
  uint32_t src;
  uint8_t* host_out;
  double t_submit;
};

struct JobSlot {
  uint32_t graph = 0;
  uint32_t width = 64;  // queries per job on this slot's graph
  pbg_msbfs* ws = nullptr;
  uint8_t* d_levels = nullptr;  // width rows of n bytes
  bool busy = false;
};

struct Job {
  JobSlot* slot;
  std::vector<Request> reqs;
  std::vector<uint32_t> srcs;
};

struct LaunchSlot {
  pbg_server* server = nullptr;
  cudaStream_t stream = nullptr;
  pbg_batch* batch = nullptr;
  int max_blocks = 0;  // set per launch: the share of the resident blocks of its mask width
  bool busy = false;
  std::atomic<int> done{0};
  double t_launch = 0, t_done = 0;
  std::vector<Job> jobs;
  uint64_t* d_hash = nullptr;   // max_jobs * 64
  uint64_t* h_hash = nullptr;   // pinned
  MsJobCtrl* h_ctrl = nullptr;  // pinned, max_jobs
  dev::GridSync* h_sync = nullptr;
  int rc = PBG_OK;
};

}  // namespace

struct pbg_server {
  std::vector<pbg_graph*> graphs;
  pbg_server_config cfg{};
  std::vector<std::unique_ptr<JobSlot>> slots;
  std::vector<std::vector<JobSlot*>> by_graph;
  std::vector<std::unique_ptr<LaunchSlot>> launches;
  std::mutex mu;
  std::condition_variable cv;       // scheduler wake-ups
  std::condition_variable cv_done;  // results / drain waiters
  std::vector<std::deque<Request>> pending;  // per graph, arrival order
  size_t npending = 0;
  std::deque<pbg_query_result> done_q;
  uint64_t next_id = 1;
  uint64_t submitted = 0, completed = 0, nlaunches = 0, njobs = 0;
  uint32_t inflight = 0, max_inflight = 0;
  uint64_t slot_bytes = 0;
  uint64_t budget_bytes = 0;  // hbm_budget_bytes clamped to the free HBM at create
  uint64_t free_bytes = 0;    // free device memory at create
  std::vector<uint32_t> width;  // queries per job, per graph
  int full_grid[5] = {0, 0, 0, 0, 0};  // resident blocks of the batched kernel, by mask words (1, 2, 4)
  bool stop = false;
  int replaying = 0;
  std::thread sched;
  std::vector<std::thread> replayers;
  clock_t_::time_point t0 = clock_t_::now();

  double now_us() const { return std::chrono::duration<double, std::micro>(clock_t_::now() - t0).count(); }
};

namespace {

// Mask words per vertex of a job of `sources` queries (1, 2 or 4).
uint32_t words_of(uint32_t sources) { return sources > 128 ? 4u : sources > 64 ? 2u : 1u; }

void CUDART_CB on_launch_done(void* p) {
  LaunchSlot* L = static_cast<LaunchSlot*>(p);
  L->t_done = L->server->now_us();
  L->done.store(1, std::memory_order_release);
  L->server->cv.notify_one();
}

// Posts the results of a finished launch and frees its slots.  Called by the
// scheduler with the lock held; touches only pinned host memory.
void retire(pbg_server* S, LaunchSlot* L) {
  const uint32_t flags = S->cfg.flags;
  for (size_t j = 0; j < L->jobs.size(); j++) {
    Job& J = L->jobs[j];
    const MsJobCtrl& c = L->h_ctrl[j];
    uint32_t status = L->rc;
    if (status == PBG_OK) {
      if (L->h_sync->error)
        status = PBG_ERR_TIMEOUT;
      else if (c.error & MS_ERR_OVERFLOW)
        status = PBG_ERR_OVERFLOW;
      else if (c.error)
        status = PBG_ERR_STATE;
    }
    for (size_t i = 0; i < J.reqs.size(); i++) {
      pbg_query_result r{};
      r.id = J.reqs[i].id;
      r.graph = J.reqs[i].graph;
      r.src = J.reqs[i].src;
      r.status = status;
      r.levels = (L->rc == PBG_OK) ? c.levels : 0;
      r.checksum = (flags & PBG_SERVER_CHECKSUM && L->rc == PBG_OK) ? L->h_hash[MS_MAX_SOURCES * j + i] : 0;
      r.t_submit_us = J.reqs[i].t_submit;
      r.t_launch_us = L->t_launch;
      r.t_done_us = L->t_done;
      S->done_q.push_back(r);
      S->completed++;
    }
    J.slot->busy = false;
  }
  L->jobs.clear();
  L->busy = false;
  L->done.store(0, std::memory_order_relaxed);
  S->inflight--;
  S->cv_done.notify_all();
}

// Enqueues the launch of L->jobs on L's stream (lock not held).
int enqueue(pbg_server* S, LaunchSlot* L) {
  const uint32_t nj = (uint32_t)L->jobs.size();
  std::vector<pbg_batch_job> bj(nj);
  for (uint32_t j = 0; j < nj; j++) {
    Job& J = L->jobs[j];
    bj[j].ws = J.slot->ws;
    bj[j].srcs = J.srcs.data();
    bj[j].k = (uint32_t)J.srcs.size();
    bj[j].d_levels = J.slot->d_levels;
  }
  // the launch's share of the resident blocks of its mask width
  const uint32_t w = words_of(L->jobs[0].slot->width);
  L->max_blocks = std::max(1, S->full_grid[w] / (int)S->cfg.streams);
  // NULL options: every job takes its graph's tuned switch (pbg_autotune) or the defaults
  int rc = batch_launch(L->batch, bj.data(), nj, nullptr, L->stream, L->max_blocks);
  if (rc) return rc;
  for (uint32_t j = 0; j < nj; j++) {
    Job& J = L->jobs[j];
    const uint32_t n = S->graphs[J.slot->graph]->n;
    if (S->cfg.flags & PBG_SERVER_CHECKSUM) {
      rc = checksum_rows_u8(J.slot->d_levels, (uint32_t)J.srcs.size(), n, L->d_hash + MS_MAX_SOURCES * j,
                            L->stream);
      if (rc) return rc;
    }
    PBG_CUDA(cudaMemcpyAsync(L->h_ctrl + j, J.slot->ws->ctrl, sizeof(MsJobCtrl), cudaMemcpyDeviceToHost,
                             L->stream));
    for (size_t i = 0; i < J.reqs.size(); i++)
      if (J.reqs[i].host_out)
        PBG_CUDA(cudaMemcpyAsync(J.reqs[i].host_out, J.slot->d_levels + i * (size_t)n, n, cudaMemcpyDeviceToHost,
                                 L->stream));
  }
  if (S->cfg.flags & PBG_SERVER_CHECKSUM)
    PBG_CUDA(cudaMemcpyAsync(L->h_hash, L->d_hash, sizeof(uint64_t) * MS_MAX_SOURCES * nj, cudaMemcpyDeviceToHost,
                             L->stream));
  PBG_CUDA(cudaMemcpyAsync(L->h_sync, L->batch->d_sync, sizeof(dev::GridSync), cudaMemcpyDeviceToHost, L->stream));
  PBG_CUDA(cudaLaunchHostFunc(L->stream, on_launch_done, L));
  return PBG_OK;
}

// Takes pending requests into jobs for one launch (lock held): repeatedly
// the graph whose oldest pending request is oldest among graphs with a free
// job slot gets a job of up to its width (max_sources, or wide_sources for a
// small graph) of its requests; a launch takes jobs of one mask width, and
// no more than max_launch_edges of graph edges (at least one job).
// A fused launch ends with its slowest job, so a launch takes graphs within
// a factor of four in edge count of its first (oldest) job's graph: queries
// on small graphs do not wait behind jobs on large ones.
bool similar_size(uint64_t m, uint64_t m0) {
  const uint64_t a = std::max<uint64_t>(m, 1);
  return a <= 4 * m0 && m0 <= 4 * a;
}

void build_jobs(pbg_server* S, LaunchSlot* L) {
  const size_t ng = S->graphs.size();
  uint64_t m0 = 0;  // edges of the launch's first job's graph
  uint32_t w0 = 0;  // mask words of the launch's jobs
  uint64_t edges = 0;  // sum of the edge counts of the launch's jobs' graphs
  while (L->jobs.size() < S->cfg.max_jobs && S->npending) {
    size_t best = ng;
    JobSlot* best_slot = nullptr;
    for (size_t g = 0; g < ng; g++) {
      if (S->pending[g].empty()) continue;
      if (best < ng && S->pending[g].front().t_submit >= S->pending[best].front().t_submit) continue;
      if (m0 && (!similar_size(S->graphs[g]->m, m0) || words_of(S->width[g]) != w0)) continue;
      for (JobSlot* js : S->by_graph[g])
        if (!js->busy) {
          best = g;
          best_slot = js;
          break;
        }
    }
    if (best == ng) break;  // no graph with pending requests has a free job slot
    if (m0 && S->cfg.max_launch_edges && edges + S->graphs[best]->m > S->cfg.max_launch_edges) break;
    edges += S->graphs[best]->m;
    if (!m0) {
      m0 = std::max<uint64_t>(S->graphs[best]->m, 1);
      w0 = words_of(S->width[best]);
    }
    best_slot->busy = true;
    Job J;
    J.slot = best_slot;
    std::deque<Request>& q = S->pending[best];
    while (!q.empty() && J.reqs.size() < S->width[best]) {
      J.reqs.push_back(q.front());
      J.srcs.push_back(q.front().src);
      q.pop_front();
      S->npending--;
    }
    L->jobs.push_back(std::move(J));
  }
}

void scheduler(pbg_server* S) {
  cudaSetDevice(S->graphs[0]->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool any_busy = false;
    for (auto& L : S->launches) {
      if (L->busy && L->done.load(std::memory_order_acquire)) retire(S, L.get());
      any_busy |= L->busy;
    }
    if (S->stop && !any_busy) break;
    // admit into every free launch slot while pending requests can form jobs
    bool launched = false;
    for (auto& Lp : S->launches) {
      LaunchSlot* L = Lp.get();
      if (S->stop || L->busy || S->npending == 0) continue;
      build_jobs(S, L);
      if (L->jobs.empty()) break;  // no free job slot for any pending graph
      L->busy = true;
      L->t_launch = S->now_us();
      S->inflight++;
      S->max_inflight = std::max(S->max_inflight, S->inflight);
      S->nlaunches++;
      S->njobs += L->jobs.size();
      lk.unlock();
      L->rc = enqueue(S, L);
      if (L->rc != PBG_OK) cudaStreamSynchronize(L->stream);  // whatever was enqueued has finished
      lk.lock();
      if (L->rc != PBG_OK) {  // no callback will come: retire now with the error
        L->t_done = S->now_us();
        retire(S, L);
      }
      launched = true;
    }
    if (!launched)
      S->cv.wait_for(lk, std::chrono::microseconds(200), [&] {
        bool busy = false;
        for (auto& L : S->launches) {
          if (L->busy && L->done.load(std::memory_order_acquire)) return true;
          busy |= L->busy;
        }
        if (S->stop) return !busy;
        if (S->npending)
          for (auto& L : S->launches)
            if (!L->busy) return true;
        return false;
      });
  }
}

void free_server(pbg_server* S) {
  for (auto& L : S->launches) {
    if (L->stream) cudaStreamSynchronize(L->stream);
    pbg_batch_free(L->batch);
    cudaFree(L->d_hash);
    cudaFreeHost(L->h_hash);
    cudaFreeHost(L->h_ctrl);
    cudaFreeHost(L->h_sync);
    if (L->stream) cudaStreamDestroy(L->stream);
  }
  for (auto& js : S->slots) {
    pbg_msbfs_free(js->ws);
    cudaFree(js->d_levels);
  }
  delete S;
}

}  // namespace

extern "C" int pbg_server_create(pbg_graph* const* graphs, uint32_t ngraphs, const pbg_server_config* cfg,
                                 pbg_server** out) {
  if (!graphs || !cfg || !out || ngraphs == 0) return fail(PBG_ERR_ARG, "NULL argument or no graphs");
  if (cfg->max_sources < 1 || cfg->max_sources > MS_MAX_SOURCES) return fail(PBG_ERR_ARG, "max_sources in [1, 256]");
  if (cfg->wide_sources > MS_MAX_SOURCES) return fail(PBG_ERR_ARG, "wide_sources in [0, 256]");
  if (cfg->max_jobs < 1 || cfg->max_jobs > MS_MAX_JOBS) return fail(PBG_ERR_ARG, "max_jobs in [1, 128]");
  if (cfg->streams < 1 || cfg->streams > 16) return fail(PBG_ERR_ARG, "streams in [1, 16]");
  for (uint32_t g = 0; g < ngraphs; g++) {
    if (!graphs[g]) return fail(PBG_ERR_ARG, "NULL graph");
    if (graphs[g]->device != graphs[0]->device) return fail(PBG_ERR_ARG, "graphs on different devices");
  }
  pbg_bfs_opts o;
  pbg_bfs_opts_default(&o);
  std::vector<uint64_t> need(ngraphs);
  std::vector<uint32_t> width(ngraphs);
  uint64_t first = 0;
  for (uint32_t g = 0; g < ngraphs; g++) {
    width[g] = (cfg->wide_sources && graphs[g]->n <= cfg->wide_max_vertices) ? cfg->wide_sources : cfg->max_sources;
    need[g] = pbg_msbfs_bytes_k(graphs[g], &o, width[g]) + (uint64_t)width[g] * graphs[g]->n + 256;
    first += need[g];
  }
  if (first > cfg->hbm_budget_bytes) return fail(PBG_ERR_OOM, "hbm_budget_bytes is below one job slot per graph");
  // admission by free HBM: the slot budget is what the caller allows, at
  // most the device's free memory less a reserve and the launch slots' buffers
  int cur = 0;
  PBG_CUDA(cudaGetDevice(&cur));
  if (cur != graphs[0]->device) PBG_CUDA(cudaSetDevice(graphs[0]->device));
  size_t free_b = 0, total_b = 0;
  cudaError_t me = cudaMemGetInfo(&free_b, &total_b);
  if (cur != graphs[0]->device) cudaSetDevice(cur);
  if (me != cudaSuccess) return cuda_fail(me, "cudaMemGetInfo");
  const uint64_t launch_bytes = (uint64_t)cfg->streams * sizeof(uint64_t) * MS_MAX_SOURCES * cfg->max_jobs;
  const uint64_t reserve = PBG_SERVER_HBM_RESERVE + launch_bytes;
  const uint64_t avail = (uint64_t)free_b > reserve ? (uint64_t)free_b - reserve : 0;
  const uint64_t budget = std::min<uint64_t>(cfg->hbm_budget_bytes, avail);
  if (first > budget)
    return fail(PBG_ERR_OOM, "free HBM (" + std::to_string(free_b >> 20) + " MiB, less a " +
                                  std::to_string(reserve >> 20) + " MiB reserve) is below one job slot per graph");
  pbg_server* S = new pbg_server();
  S->cfg = *cfg;
  S->budget_bytes = budget;
  S->free_bytes = free_b;
  S->graphs.assign(graphs, graphs + ngraphs);
  S->by_graph.resize(ngraphs);
  S->pending.resize(ngraphs);
  S->width = width;
  // job slots: one per graph first, then round-robin while the budget lasts
  const uint32_t per_graph_cap = 2 * cfg->streams;
  auto add_slot = [&](uint32_t g) -> int {
    std::unique_ptr<JobSlot> js(new JobSlot());
    js->graph = g;
    js->width = width[g];
    int rc = pbg_msbfs_create_k(graphs[g], &o, width[g], &js->ws);
    if (rc) return rc;
    cudaError_t e = cudaMalloc(&js->d_levels, (size_t)width[g] * graphs[g]->n + 16);
    if (e != cudaSuccess) {
      pbg_msbfs_free(js->ws);
      return cuda_fail(e, "server level rows");
    }
    S->by_graph[g].push_back(js.get());
    S->slots.push_back(std::move(js));
    S->slot_bytes += need[g];
    return PBG_OK;
  };
  int rc = PBG_OK;
  for (uint32_t g = 0; g < ngraphs && !rc; g++) rc = add_slot(g);
  // more slots round-robin while the budget lasts; an allocation that fails
  // anyway (memory taken since the free-memory query) ends the growth
  for (bool grew = true; grew && !rc;) {
    grew = false;
    for (uint32_t g = 0; g < ngraphs && !rc; g++)
      if (S->by_graph[g].size() < per_graph_cap && S->slot_bytes + need[g] <= budget) {
        rc = add_slot(g);
        if (rc == PBG_ERR_OOM) {
          cudaGetLastError();
          rc = PBG_OK;
          grew = false;
          break;
        }
        grew = true;
      }
  }
  // launch slots
  for (uint32_t g = 0; g < ngraphs && !rc; g++) {
    const uint32_t w = words_of(width[g]);
    if (!S->full_grid[w]) S->full_grid[w] = ms_full_grid(graphs[0]->num_sms, w);
    if (S->full_grid[w] < 1) rc = fail(PBG_ERR_CUDA, "multi-source kernel cannot be resident");
  }
  for (uint32_t i = 0; i < cfg->streams && !rc; i++) {
    std::unique_ptr<LaunchSlot> L(new LaunchSlot());
    L->server = S;
    cudaError_t e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&L->d_hash, sizeof(uint64_t) * MS_MAX_SOURCES * cfg->max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&L->h_hash, sizeof(uint64_t) * MS_MAX_SOURCES * cfg->max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&L->h_ctrl, sizeof(MsJobCtrl) * cfg->max_jobs);
    if (e == cudaSuccess) e = cudaMallocHost(&L->h_sync, sizeof(dev::GridSync));
    if (e != cudaSuccess) rc = cuda_fail(e, "server launch slot");
    if (!rc) rc = pbg_batch_create(cfg->max_jobs, &L->batch);
    S->launches.push_back(std::move(L));
  }
  if (rc) {
    free_server(S);
    return rc;
  }
  S->sched = std::thread(scheduler, S);
  *out = S;
  return PBG_OK;
}

extern "C" int pbg_server_submit(pbg_server* S, uint32_t graph, uint32_t src, uint8_t* levels_out, uint64_t* id) {
  if (!S) return fail(PBG_ERR_ARG, "server is NULL");
  if (graph >= S->graphs.size()) return fail(PBG_ERR_ARG, "graph index out of range");
  if (src >= S->graphs[graph]->n) return fail(PBG_ERR_ARG, "source vertex out of range");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fail(PBG_ERR_STATE, "server is stopping");
    Request r{S->next_id++, graph, src, levels_out, S->now_us()};
    if (id) *id = r.id;
    S->pending[graph].push_back(r);
    S->npending++;
    S->submitted++;
  }
  S->cv.notify_one();
  return PBG_OK;
}

extern "C" int pbg_server_replay(pbg_server* S, const uint32_t* graph, const uint32_t* src, const double* arrival_us,
                                 uint32_t count) {
  if (!S || (count && (!graph || !src || !arrival_us))) return fail(PBG_ERR_ARG, "NULL argument");
  for (uint32_t i = 0; i < count; i++) {
    if (graph[i] >= S->graphs.size() || src[i] >= S->graphs[graph[i]]->n)
      return fail(PBG_ERR_ARG, "replay entry out of range");
    if (i && arrival_us[i] < arrival_us[i - 1]) return fail(PBG_ERR_ARG, "arrival times must be non-decreasing");
  }
  std::vector<uint32_t> g(graph, graph + count), s(src, src + count);
  std::vector<double> t(arrival_us, arrival_us + count);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fail(PBG_ERR_STATE, "server is stopping");
    S->replaying++;
  }
  S->replayers.emplace_back([S, g = std::move(g), s = std::move(s), t = std::move(t)]() {
    const double base = S->now_us();
    for (size_t i = 0; i < g.size(); i++) {
      const double due = base + t[i];
      const double now = S->now_us();
      if (due - now > 200) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)(due - now - 100)));
      while (S->now_us() < due) {
      }
      {
        std::lock_guard<std::mutex> lk(S->mu);
        Request r{S->next_id++, g[i], s[i], nullptr, S->now_us()};
        S->pending[g[i]].push_back(r);
        S->npending++;
        S->submitted++;
      }
      S->cv.notify_one();
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->replaying--;
    S->cv_done.notify_all();
  });
  return PBG_OK;
}

extern "C" int pbg_server_poll(pbg_server* S, pbg_query_result* out, uint32_t cap, uint32_t* count, int wait_ms) {
  if (!S || (!out && cap) || !count) return fail(PBG_ERR_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done_q.empty() && wait_ms > 0)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->done_q.empty(); });
  uint32_t k = 0;
  while (k < cap && !S->done_q.empty()) {
    out[k++] = S->done_q.front();
    S->done_q.pop_front();
  }
  *count = k;
  return PBG_OK;
}

extern "C" int pbg_server_drain(pbg_server* S, int timeout_ms) {
  if (!S) return fail(PBG_ERR_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                      [&] { return S->replaying == 0 && S->completed == S->submitted; });
  return ok ? PBG_OK : fail(PBG_ERR_TIMEOUT, "server drain timed out");
}

extern "C" int pbg_server_stats_get(pbg_server* S, pbg_server_stats* st) {
  if (!S || !st) return fail(PBG_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->launches = S->nlaunches;
  st->jobs = S->njobs;
  st->max_inflight = S->max_inflight;
  st->slots = (uint32_t)S->slots.size();
  st->slot_bytes = S->slot_bytes;
  st->budget_bytes = S->budget_bytes;
  st->free_bytes = S->free_bytes;
  return PBG_OK;
}

extern "C" int pbg_server_destroy(pbg_server* S) {
  if (!S) return PBG_OK;
  for (auto& t : S->replayers) t.join();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  S->sched.join();
  free_server(S);
  return PBG_OK;
}
