// internal.cuh -- shared declarations of the B200 BFS library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "device_util.cuh"
#include "pbbs_bfs.h"

#define PBG_NONE 0xFFFFFFFFu

namespace pbg {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define PBG_CUDA(call)                                  \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return pbg::cuda_fail(_e, #call); \
  } while (0)

// Device error word bits.
enum : uint32_t {
  ERR_BARRIER_TIMEOUT = 1u,  // a grid barrier wait ran out of its budget
  ERR_LEVEL_LIMIT = 2u,      // more levels than vertices (cannot happen on valid input)
  ERR_QUEUE = 4u,            // a frontier queue would overflow (cannot happen on valid input)
};

// ------------------------------------------------------- BFS control block
// One slot per frontier: the frontier produced at level L lives in slot
// (L + 1) % 3 (three slots so the next-but-one can be cleared while the
// current one is read and the next one written).
struct LevelSlot {
  unsigned long long nmain;  // entries in the main queue
  unsigned long long big;    // (entries << 40) | chunks, big-vertex queue
  unsigned long long deg;    // sum of degrees of the frontier
  unsigned long long pad;
};

struct BfsCtrl {
  LevelSlot slot[3];
  LevelSlot conv;  // queues rebuilt from the bitmap after a bottom-up level
  dev::GridSync sync;
  unsigned int levels;
  unsigned int td_levels;
  unsigned int bu_levels;
  unsigned int final_bm;
  unsigned int pad0;
  unsigned long long visited;
  unsigned long long edges_reached;
  unsigned long long bu_mask;
  unsigned long long t_start;  // kernel start (block 0)
  unsigned long long t_end;    // kernel end (block 0)
  // per-level trace written by block 0 at the start of each level
  unsigned long long t_ns[PBG_TRACE_LEVELS + 1];
  unsigned long long t_nf[PBG_TRACE_LEVELS];
  unsigned long long t_deg[PBG_TRACE_LEVELS];
  unsigned int t_bu[PBG_TRACE_LEVELS];
};

struct BfsWorkspace {
  uint32_t* bm[2] = {nullptr, nullptr};  // visited bitmaps, nwords each
  uint32_t* q[2] = {nullptr, nullptr};   // main frontier queues, n each
  uint2* qr[2] = {nullptr, nullptr};     // (begin, end) of each main queue entry
  uint4* qbig[2] = {nullptr, nullptr};   // big-vertex queues (v, begin, end, first chunk)
  uint32_t big_cap = 0;
  uint32_t big_min_degree = 0;           // the chunk threshold the chunk queues were sized for
  BfsCtrl* ctrl = nullptr;
  uint32_t* parent = nullptr;            // scratch outputs for host-buffer calls
  uint32_t* level = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool ready = false;
};

struct LaunchShape {
  int block = 0;
  int grid = 0;
};

}  // namespace pbg

struct pbg_graph {
  uint32_t n = 0;
  uint64_t m = 0;
  uint32_t flags = 0;
  uint32_t nwords = 0;        // bitmap words, rounded up to a multiple of 32
  uint32_t* d_offsets = nullptr;
  uint32_t* d_edges = nullptr;
  uint32_t* d_iso = nullptr;  // bitmap of degree-0 vertices (symmetric graphs)
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  pbg::BfsWorkspace ws;
  pbg_bfs_stats last{};
  bool stats_pending = false;
  pbg_msbfs* ms_ws = nullptr;    // for pbg_bfs_multi
  pbg_batch* ms_batch = nullptr;
  // Pull chunks of the batched search (built on first use): the tail of
  // every neighbour list longer than MS_PULL_SERIAL cut into MS_PULL_CHUNK
  // pieces, (vertex, first edge, end edge, vertex degree) each, in vertex
  // order.
  uint4* d_pull_chunks = nullptr;
  uint32_t n_pull_chunks = 0;
  bool pull_chunks_built = false;
  // options picked by pbg_autotune, used by calls that pass none
  pbg_bfs_opts tuned{};
  bool has_tuned = false;
  pbg_bfs_opts tuned_multi{};
  bool has_tuned_multi = false;
  // maximal independent set (mis.cu): whether every list is ascending (-1 =
  // not yet known), the flags buffer of host-output calls, the last run
  int lists_sorted = -1;
  uint8_t* mis_flags = nullptr;
  pbg::BfsCtrl* mis_ctrl = nullptr;  // its own control block and events: BFS statistics stay readable
  cudaEvent_t mis_ev0 = nullptr, mis_ev1 = nullptr;
  bool mis_pending = false;
  bool mis_ran = false;
  pbg_mis_stats mis_last{};
  // the largest degree (found when the graph is validated); below the chunk
  // degree, single-source searches run bfs_lean
  uint32_t max_degree = 0;
  // device check (check.cu): scratch kept between calls, grown when needed
  void* check_buf = nullptr;
  size_t check_bytes = 0;
};

namespace pbg {
// State arrays of one single-source search, for bfs_launch_on.
struct BfsOnArgs {
  const uint32_t* offsets;
  const uint32_t* edges;
  const uint32_t* iso;
  uint32_t* parent;
  uint32_t* level;
  uint32_t* bm0;
  uint32_t* bm1;
  uint32_t* q0;
  uint32_t* q1;
  uint2* qr0;
  uint2* qr1;
  uint4* qb0;
  uint4* qb1;
  BfsCtrl* ctrl;
  unsigned long long m;
  uint32_t n;
  uint32_t nwords;
  uint32_t big_cap;
  uint32_t src;
  uint32_t symmetric;
};
int bfs_launch_on(const BfsOnArgs& r, const pbg_bfs_opts& o, int num_sms, cudaStream_t s);
int bfs_ensure_workspace(pbg_graph* g, const pbg_bfs_opts& o);
void bfs_free_workspace(pbg_graph* g);
int bfs_launch(pbg_graph* g, uint32_t src, const pbg_bfs_opts& o, uint32_t* d_parent, uint32_t* d_level,
               cudaStream_t s);
int bfs_read_stats(pbg_graph* g, pbg_bfs_stats* st);
int bfs_read_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count);
void resolve_opts(const pbg_bfs_opts* in, pbg_bfs_opts* out);

// Graph handles (graph.cu): a grid of 256-thread blocks for `work` items
// (at most 16 blocks per SM); a new handle with device arrays for n + 1
// offsets and m edges; validation of the CSR now on the device (offsets
// from 0 to m, non-decreasing, edge targets < n), symmetry detection when
// asked, and the degree-0 bitmap.
int grid_for(uint64_t work, int num_sms);
int new_handle(uint32_t n, uint64_t m, uint32_t flags, pbg_graph** out);
int finish_graph(pbg_graph* g);
// `in`, or when it is NULL the graph's tuned options (pbg_autotune), else
// the defaults; multi: the batched search's.
void resolve_graph_opts(const pbg_graph* g, const pbg_bfs_opts* in, bool multi, pbg_bfs_opts* out);
}  // namespace pbg
