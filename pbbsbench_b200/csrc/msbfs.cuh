// msbfs.cuh -- structures of the batched multi-source BFS (msbfs.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_util.cuh"
#include "internal.cuh"

namespace pbg {

constexpr uint32_t MS_MAX_JOBS = 128;  // jobs in one fused launch
constexpr uint32_t MS_MAX_SOURCES = 256;  // up to four 64-bit mask words per vertex
// Pull: the first MS_PULL_SERIAL neighbours of a vertex are scanned by one
// lane; the rest of a longer list is pulled in MS_PULL_CHUNK-edge pieces
// spread over all warps of the grid (the graph's pull chunk table).
constexpr uint32_t MS_PULL_SERIAL = 64;
constexpr uint32_t MS_PULL_CHUNK = 256;
// Frontier planes per job: the new-bit masks of the last MS_PLANES levels,
// kept until they are expanded into the level rows (a flush writes each
// row's bytes of several levels at once).
constexpr uint32_t MS_PLANES = 8;

enum : uint32_t {
  MS_ERR_TIMEOUT = 1u,   // a grid barrier wait ran out
  MS_ERR_OVERFLOW = 2u,  // a level >= 255 would be needed (uint8 levels)
  MS_ERR_QUEUE = 4u,     // a frontier queue would overflow (cannot happen on valid input)
};

constexpr uint32_t MS_TRACE_LEVELS = 64;

// Per-job counters (device).
struct MsJobCtrl {
  LevelSlot slot[3];
  unsigned int levels;
  unsigned int pull_levels;
  unsigned int push_levels;
  unsigned int error;
  unsigned long long done_deg;  // out-degree sum of vertices reached by every source
  unsigned long long live[3][4];  // per level slot: the source bits of that frontier
  // per-level trace (first MS_TRACE_LEVELS levels), written by block 0 when
  // the level's direction is decided; t_ns[L + 1] ends level L
  unsigned long long t_ns[MS_TRACE_LEVELS + 1];
  unsigned long long t_nf[MS_TRACE_LEVELS];
  unsigned long long t_deg[MS_TRACE_LEVELS];
  unsigned int t_pull[MS_TRACE_LEVELS];
};

// Device descriptor of one job: a graph, up to 256 sources, its state arrays.
struct MsJob {
  const uint32_t* offsets;
  const uint32_t* edges;
  unsigned long long m;
  unsigned long long all[4];  // mask of the job's source bits (words 0 .. words - 1)
  uint32_t n;
  uint32_t k;
  uint32_t symmetric;
  uint32_t big_cap;
  unsigned long long* vis;
  unsigned long long* planes;  // MS_PLANES x n masks: plane of level L at (L % MS_PLANES) * n * words
  uint32_t* fbits;             // two-word jobs: frontier bitmap of the level a pull builds
  uint32_t* q0;
  uint32_t* q1;
  uint4* qb0;
  uint4* qb1;
  uint8_t* levels;
  const uint32_t* srcs;
  MsJobCtrl* ctrl;
  const uint4* pchunks;  // the graph's pull chunks (vertex, first edge, end edge, degree)
  uint32_t npc;
  // 1: levels written as they are found (sparse graphs, where a level's new
  // bits touch few rows of each 32-vertex piece); 0: kept in the planes and
  // expanded every MS_PLANES levels (dense graphs, where per-level writes
  // would rewrite most row pieces level after level).  See ms_direct_levels.
  uint32_t direct;
  uint32_t alpha, beta;  // the job's direction switch (decide in msbfs.cu)
};

// Degree from which a frontier vertex queued by a push goes to the chunked
// queue (pieces of MS CHUNK edges spread over all warps); shorter lists share
// 32-vertex tiles walked by one warp.
inline uint32_t ms_big_degree(const pbg_bfs_opts& o) { return o.chunk_min_degree > 128u ? o.chunk_min_degree : 128u; }

// Level-writing mode of a job on a graph of n vertices and m directed edges:
// direct below an average degree of 16.
inline uint32_t ms_direct_levels(uint64_t n, uint64_t m) { return m < 16 * n ? 1u : 0u; }

// words: mask words per vertex of the launch's jobs (1, 2 or 4).
int ms_full_grid(int num_sms, uint32_t words = 1);
// Builds g's pull chunk table once (synchronous; thread-safe).
int ms_pull_chunks(pbg_graph* g);
// max_blocks > 0 caps the grid, so several launches can be resident at once.
int ms_launch(const MsJob* d_jobs, uint32_t njobs, const pbg_bfs_opts& o, dev::GridSync* d_sync, int num_sms,
              cudaStream_t s, int max_blocks, uint32_t words);
int batch_launch(pbg_batch* b, const pbg_batch_job* jobs, uint32_t njobs, const pbg_bfs_opts* opts, cudaStream_t s,
                 int max_blocks);
int checksum_rows_u8(const uint8_t* d_levels, uint32_t rows, uint32_t n, uint64_t* d_out, cudaStream_t s);

}  // namespace pbg

// Workspace of one multi-source job on one graph.
struct pbg_msbfs {
  pbg_graph* g = nullptr;
  unsigned long long* vis = nullptr;
  unsigned long long* planes = nullptr;
  uint32_t* fbits = nullptr;
  uint32_t words = 1;  // mask words per vertex (1, 2 or 4): sources up to 64 * words
  uint32_t* q0 = nullptr;
  uint32_t* q1 = nullptr;
  uint4* qb0 = nullptr;
  uint4* qb1 = nullptr;
  uint32_t big_cap = 0;
  uint32_t big_min_degree = 0;
  pbg::MsJobCtrl* ctrl = nullptr;
  uint8_t* levels = nullptr;  // owned k*n buffer for host-output calls (lazily)
  size_t levels_bytes = 0;
  uint32_t last_k = 0;
};

// Descriptor arrays, staging and barrier of fused launches.
struct pbg_batch {
  uint32_t max_jobs = 0;
  int device = 0;
  int num_sms = 0;
  pbg::MsJob* d_jobs = nullptr;
  pbg::MsJob* h_jobs = nullptr;  // pinned
  uint32_t* d_srcs = nullptr;    // max_jobs * 64
  uint32_t* h_srcs = nullptr;    // pinned
  pbg::dev::GridSync* d_sync = nullptr;
  cudaEvent_t staged = nullptr;  // host staging buffers free again
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool pending = false;
};
