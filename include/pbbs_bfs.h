/*
 * pbbs_bfs.h -- C ABI of the B200 breadth-first-search library
 * (pbbsbench_b200/libpbbsbfs.so).
 *
 * It replaces the link-time plugin boundary of PBBS's breadthFirstSearch
 * benchmark,
 *     parlay::sequence<vertexId> BFS(vertexId start, const Graph& G, bool verbose)
 * (benchmarks/breadthFirstSearch/bench/BFS.h:11), with plain-C calls over the
 * same data: the CSR graph of common/graph.h:104-152 (offsets[n+1] with
 * offsets[n] = m, edges[m], 32-bit ids) and the parent array the benchmark
 * returns (-1 = unvisited, parent[start] = start; BFS.h:9-10).  The drop-in
 * BFS.C that implements BFS.h:11 on top of these calls is
 * pbbsbench_b200/dropin/gpuBFS/BFS.C.
 *
 * All entry points return an int status (PBG_OK = 0); pbg_last_error() gives
 * the calling thread's last message.  Calls on one graph handle are
 * serialised on that handle's CUDA stream; different handles may run
 * concurrently.  Everything runs on the CUDA device that is current when the
 * graph is created.
 */
#ifndef PBBS_BFS_H_
#define PBBS_BFS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
#define PBG_OK 0
#define PBG_ERR_ARG 1      /* bad argument (null handle, src >= n, ...) */
#define PBG_ERR_CUDA 2     /* a CUDA runtime call failed */
#define PBG_ERR_OOM 3      /* device allocation failed / HBM budget exceeded */
#define PBG_ERR_TIMEOUT 4  /* a bounded device-side wait ran out */
#define PBG_ERR_OVERFLOW 5 /* a level does not fit the output type */
#define PBG_ERR_STATE 6    /* call not valid in the handle's current state */

/* Message for the calling thread's most recent failed call ("" if none). */
const char* pbg_last_error(void);

/* ------------------------------------------------------------ graphs */
typedef struct pbg_graph pbg_graph;

/* Largest vertex count a graph handle accepts.  The reference's vertex ids
 * are int (bench/BFS.h:5, `typedef int vertexId`), so a graph has at most
 * 2^31 - 1 vertices; that also keeps PBG_NONE (0xFFFFFFFF) out of the id
 * range and lets the max-parent rule compare ids as signed ints.  Every
 * call that creates a handle returns PBG_ERR_ARG for a larger n. */
#define PBG_MAX_VERTICES 0x7FFFFFFFu

/* The graph is symmetric (every edge present in both directions).  Only then
 * may BFS run bottom-up, which scans N(v) as in-neighbours exactly as
 * edge_map_dense does (common/ligraLight.h:87-112). */
#define PBG_GRAPH_SYMMETRIC 1u
/* Decide symmetry on the device at upload: the graph is marked symmetric when
 * every adjacency list is ascending and every edge (u, v) has its reverse
 * (binary search in N(v)).  Otherwise it is searched top-down only. */
#define PBG_GRAPH_DETECT_SYMMETRIC 2u

/* Copies a host CSR graph into HBM; the library owns the device copy, the
 * caller keeps its arrays.  Replaces the graph<int,uint> the driver builds in
 * readGraphFromFile (common/graphIO.h:191-215) + G.addDegrees()
 * (bench/BFSTime.C:58-59); degrees are derived from offsets on the device. */
int pbg_graph_upload(const uint32_t* offsets, const uint32_t* edges, uint32_t n, uint64_t m,
                     uint32_t flags, pbg_graph** out);

/* Same, from device memory (the arrays are copied). */
int pbg_graph_upload_device(const uint32_t* d_offsets, const uint32_t* d_edges, uint32_t n,
                            uint64_t m, uint32_t flags, pbg_graph** out);

/* Seeded synthetic graphs built on the device (symmetrised, self loops and
 * duplicates removed, each adjacency list ascending: the construction of
 * common/graphUtils.h:54-94).  Kinds follow testData/graphData/. */
#define PBG_GEN_RMAT 1      /* rMatGraph.C:33-79: n = 2^logn, `samples` edge draws */
#define PBG_GEN_TORUS3D 2   /* gridGraph.C:53-72 (-d 3): n = dn^3, 3 edges per vertex */
#define PBG_GEN_RANDLOCAL 3 /* n vertices, `degree` out-edges at offsets in [-window, window] */
typedef struct pbg_gen_params {
  uint32_t kind;
  uint32_t logn;    /* RMAT */
  uint64_t samples; /* RMAT: number of edge draws */
  uint64_t seed;
  double a, b, c;   /* RMAT quadrant probabilities */
  uint32_t dn;      /* TORUS3D side */
  uint32_t n;       /* RANDLOCAL vertices */
  uint32_t degree;  /* RANDLOCAL out-edges per vertex */
  uint32_t window;  /* RANDLOCAL offset bound */
  uint32_t permute; /* nonzero: relabel vertices by a seeded random permutation (graphReorder) */
  uint64_t perm_seed;
} pbg_gen_params;
int pbg_graph_generate(const pbg_gen_params* p, pbg_graph** out);

/* n, m, and the device CSR arrays (owned by the handle). */
int pbg_graph_info(const pbg_graph* g, uint32_t* n, uint64_t* m, const uint32_t** d_offsets,
                   const uint32_t** d_edges);
/* The handle's PBG_GRAPH_* flags (after symmetry detection). */
int pbg_graph_flags(const pbg_graph* g, uint32_t* flags);
/* Copies the CSR back to host arrays of n+1 and m entries (edges may be NULL:
 * offsets only). */
int pbg_graph_download(const pbg_graph* g, uint32_t* offsets, uint32_t* edges);
/* Frees the device copy and every workspace attached to the handle. */
int pbg_graph_free(pbg_graph* g);

/* ------------------------------------------------------------ graph files */
/* Reads a PBBS AdjacencyGraph text file: the header word, n, m, n offsets, m
 * edges, tokens split by space, tab, LF, CR or NUL (the reader of
 * common/graphIO.h:191-215 with the tokens of common/IO.h:41-50,207-214).
 * The text after the header is parsed on the device straight into the CSR;
 * offsets[n] = m as in the reference.  Errors: a missing header, a token
 * count other than n + m after it ("bad input file: length = ..." as the
 * reference prints), a token that is not an unsigned decimal integer below
 * 2^32, and a CSR that fails validation.  flags as pbg_graph_upload. */
int pbg_graph_load_adj(const char* path, uint32_t flags, pbg_graph** out);
/* The same from text in host memory (len bytes). */
int pbg_graph_parse_adj(const char* text, uint64_t len, uint32_t flags, pbg_graph** out);
/* Writes g as AdjacencyGraph text, formatted on the device: the header
 * line, n, m, then one value per line (common/graphIO.h:79-104 with the
 * stream layout of common/IO.h:100-150). */
int pbg_graph_write_adj(const pbg_graph* g, const char* path);
/* Writes count values as a sequenceInt file, formatted on the device: the
 * output the BFS driver writes for the parent array (common/IO.h:198-203,
 * bench/BFSTime.C). */
int pbg_write_seq_int(const int32_t* values, uint64_t count, const char* path);
/* Binary CSR image: a 32-byte header ("PBGCSR01", n and m as uint64, the
 * symmetric flag, 0), then uint32 offsets[n + 1] and edges[m] as in memory.
 * Loading with flags 0 keeps the symmetric flag the file was saved with. */
int pbg_graph_save_bin(const pbg_graph* g, const char* path);
int pbg_graph_load_bin(const char* path, uint32_t flags, pbg_graph** out);

/* ----------------------------------------------------- single-source BFS */
/* Parent rule. */
#define PBG_PARENT_ANY 0 /* first claimer wins: backForwardBFS/BFS.C:45-48, simpleBFS/BFS.C:50-54 */
#define PBG_PARENT_MIN 1 /* smallest neighbour one level up (deterministic; atomicMin) */
#define PBG_PARENT_MAX 2 /* largest neighbour one level up: deterministicBFS/BFS.C:60-74 */

/* Direction policy. */
#define PBG_DIR_AUTO 0     /* direction-optimizing switch of ligraLight.h:114-136 */
#define PBG_DIR_TOPDOWN 1  /* every level top-down (simpleBFS / ndBFS) */
#define PBG_DIR_BOTTOMUP 2 /* every level bottom-up (symmetric graphs only) */

typedef struct pbg_bfs_opts {
  uint32_t parent_mode;     /* PBG_PARENT_* */
  uint32_t direction;       /* PBG_DIR_* */
  uint32_t alpha;           /* go bottom-up when |F| + sum deg(F) > m / alpha (ligraLight.h:122; 20) */
  uint32_t beta;            /* stay bottom-up while |F| > n / beta (ligraLight.h:130; 20) */
  uint32_t block_threads;   /* CTA size of the persistent kernel: 256, 512 or 1024 (0 = tuned) */
  uint32_t chunk_min_degree; /* top-down: degree from which a list is cut into 256-edge pieces that
                                whole warps expand anywhere in the grid; shorter lists are walked by
                                one thread each (0 = tuned, else 32).  When every list of the graph is
                                shorter, the search runs a kernel without the piece queue (same
                                results); block_threads is then 1024 whatever is asked. */
} pbg_bfs_opts;

/* Fills the defaults (ANY, AUTO, alpha = beta = 20, tuned sizes). */
void pbg_bfs_opts_default(pbg_bfs_opts* o);

typedef struct pbg_bfs_stats {
  uint32_t levels;          /* number of non-empty frontiers */
  uint32_t topdown_levels;
  uint32_t bottomup_levels;
  uint32_t error;           /* device error word (0 = none) */
  uint64_t visited;         /* reached vertices */
  uint64_t edges_reached;   /* sum of degrees of reached vertices (m_r) */
  uint64_t bottomup_mask;   /* bit L set: level L (< 64) ran bottom-up */
  float device_ms;          /* device time of the last pbg_bfs call (events) */
  float init_ms;            /* of which: kernel start to the first level (initialisation) */
  float kernel_ms;          /* kernel start to end as seen by the device clock */
} pbg_bfs_stats;

/* BFS from src.  parent_out (host, n entries, may be NULL) receives the
 * BFS.h:9-10 parent array (-1 unvisited, parent[src] = src); level_out (host,
 * n entries, may be NULL) receives BFS distances (0xFFFFFFFF unreached).
 * Blocks until the results are on the host.  stats may be NULL. */
int pbg_bfs(pbg_graph* g, uint32_t src, const pbg_bfs_opts* opts, int32_t* parent_out,
            uint32_t* level_out, pbg_bfs_stats* stats);

/* Same into device buffers (parent n entries required, level may be NULL),
 * enqueued on `stream` (a cudaStream_t; 0 is CUDA's default stream) without
 * synchronising.  Statistics of the run are read with pbg_bfs_stats_get after
 * the stream has been synchronised. */
int pbg_bfs_device(pbg_graph* g, uint32_t src, const pbg_bfs_opts* opts, uint32_t* d_parent,
                   uint32_t* d_level, void* stream);
int pbg_bfs_stats_get(pbg_graph* g, pbg_bfs_stats* stats);

/* Per-level trace of the last BFS on the handle (first PBG_TRACE_LEVELS
 * levels): the frontier size and out-degree that drove the direction switch,
 * the direction taken, and the level's device time.  The counterpart of the
 * reference's verbose "edge map sparse/dense: <size>" lines and phase timers
 * (common/ligraLight.h:71,88,115,126).  Call after the stream is synchronised. */
#define PBG_TRACE_LEVELS 256
typedef struct pbg_level_trace {
  uint32_t level;
  uint32_t bottom_up;
  uint64_t frontier;
  uint64_t frontier_degree;
  double ms;
} pbg_level_trace;
int pbg_bfs_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count);

/* ------------------------------------- single-source BFS without allocation */
/* Has no counterpart in the reference.  For callers that cannot call
 * cudaMalloc: code that runs where device allocation is not allowed or not
 * wanted, such as a latency-critical path that must not hit cudaMalloc's
 * implicit device-wide synchronisation, a process whose memory is capped or
 * pre-reserved by another framework's allocator, or a plugin that may only
 * touch the buffers its host hands it.  The caller passes the CSR (device
 * memory), the source and the output buffers; every scratch array lives in
 * one fixed file-scope device array of PBG_NOALLOC_SCRATCH_BYTES, which each
 * GPU holds from the first time the library's code for this call is loaded on
 * it until the process exits.  Limits: n <= PBG_NOALLOC_MAX_VERTICES and
 * m <= PBG_NOALLOC_MAX_EDGES; larger graphs are rejected with PBG_ERR_ARG.
 * The first call on a device does the set-up there (the SM count, and the
 * array's device address from cudaGetSymbolAddress, which loads the module),
 * so make that first call before any stream capture; later calls look the
 * address up again, which allocates nothing.  All calls share the array and
 * it keeps the last call's contents (each call clears what must start at
 * zero): calls whose work overlaps on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.
 * flags: PBG_GRAPH_SYMMETRIC or 0 (top-down only).  parent_mode as in
 * pbg_bfs_opts; d_level may be NULL.  The call validates the CSR, runs the
 * search on `stream` (0 = default stream) and waits for it; it returns the
 * search's status.  The results are those of pbg_bfs with the options of
 * pbg_bfs_opts_default() and this parent_mode; options tuned for a graph
 * handle (pbg_autotune) are not used. */
#define PBG_NOALLOC_MAX_VERTICES (1u << 20)
#define PBG_NOALLOC_MAX_EDGES (1u << 24)
#define PBG_NOALLOC_SCRATCH_BYTES (41u << 20)
int pbg_bfs_noalloc(const uint32_t* d_offsets, const uint32_t* d_edges, uint32_t n, uint64_t m, uint32_t flags,
                    uint32_t src, uint32_t parent_mode, uint32_t* d_parent, uint32_t* d_level, void* stream);

/* ------------------------------------------------ maximal independent set */
/* The frontier engine reused for PBBS's maximalIndependentSet benchmark,
 * whose plugin is
 *     parlay::sequence<char> maximalIndependentSet(Graph const& G)
 * (benchmarks/maximalIndependentSet/bench/MIS.h:8; flags 1 = in the set,
 * 2 = not).  The set is the one serialMIS returns
 * (maximalIndependentSet/serialMIS/MIS.C:33-47: vertices in id order, v in
 * unless an out-neighbour already in the set, a self loop keeping v out),
 * found in parallel rounds on the device and bit-exact with it; on
 * symmetric graphs it passes MISCheck (bench/MISCheck.C:39-66), the contract
 * of the nondeterministic ndMIS too.  Runs on any graph handle. */
typedef struct pbg_mis_stats {
  uint32_t rounds;   /* rounds of the persistent kernel (one grid barrier each) */
  uint32_t error;    /* device error word (0 = none) */
  uint64_t in_set;   /* vertices in the set */
  float device_ms;   /* device time of the last call (events) */
  float kernel_ms;   /* kernel start to end as seen by the device clock */
} pbg_mis_stats;
/* flags_out: host, n bytes (1 in the set, 2 not).  Blocks until the flags are
 * on the host; stats may be NULL. */
int pbg_mis(pbg_graph* g, uint8_t* flags_out, pbg_mis_stats* stats);
/* Same into device memory (n bytes), enqueued on `stream` without
 * synchronising; statistics with pbg_mis_stats_get after the stream is
 * synchronised. */
int pbg_mis_device(pbg_graph* g, uint8_t* d_flags, void* stream);
int pbg_mis_stats_get(pbg_graph* g, pbg_mis_stats* stats);
/* Per-round trace of the last MIS on the handle (first PBG_TRACE_LEVELS
 * rounds): `frontier` = the undecided vertices the round walked (n in round
 * 0), `ms` = the round's device time; bottom_up and frontier_degree are 0.
 * The reference's timers (common/time_loop.h) time whole calls only.  Call
 * after the stream is synchronised. */
int pbg_mis_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count);

/* ------------------------------------------------ batched multi-source BFS */
/* No reference counterpart: PBBS answers one source per BFS() call.  A job is
 * up to 256 sources on one resident graph, searched together with one
 * visited mask per vertex (one 64-bit word for up to 64 sources, two for up
 * to 128, four for up to 256: a pull gathers a wider mask for the same one
 * cache lookup per neighbour); many jobs (on graphs of any sizes) run in ONE fused
 * persistent launch.  Each source's result is its level array, uint8
 * per vertex (255 = unreached), identical to a single-source search from it;
 * a search that would need level 255 fails with PBG_ERR_OVERFLOW.
 * Options: direction AUTO picks, per job and level, pull when the out-degree
 * of the vertices not yet reached by every source, times alpha, is at most
 * twice the frontier's out-degree times beta (a pushed edge costs about two
 * pulled ones); TOPDOWN pushes and BOTTOMUP pulls every level.
 * chunk_min_degree sizes the big-vertex queues of sparse push levels. */
#define PBG_MAX_SOURCES 256
#define PBG_MAX_JOBS 128
typedef struct pbg_msbfs pbg_msbfs; /* device state of one job on one graph */
typedef struct pbg_batch pbg_batch; /* descriptors + barrier of fused launches */

/* Device bytes one job workspace for up to max_sources (1..256) sources takes
 * on g (for admission control); 0 for bad arguments. */
uint64_t pbg_msbfs_bytes_k(const pbg_graph* g, const pbg_bfs_opts* opts, uint32_t max_sources);
int pbg_msbfs_create_k(pbg_graph* g, const pbg_bfs_opts* opts, uint32_t max_sources, pbg_msbfs** out);
/* The same for up to 64 sources.  One fused launch takes workspaces of one
 * size class only (all up to 64, all up to 128, or all up to 256 sources). */
uint64_t pbg_msbfs_bytes(const pbg_graph* g, const pbg_bfs_opts* opts);
int pbg_msbfs_create(pbg_graph* g, const pbg_bfs_opts* opts, pbg_msbfs** out);
int pbg_msbfs_free(pbg_msbfs* ws);

int pbg_batch_create(uint32_t max_jobs, pbg_batch** out);
int pbg_batch_free(pbg_batch* b);

typedef struct pbg_batch_job {
  pbg_msbfs* ws;        /* distinct per job within one launch */
  const uint32_t* srcs; /* host array of k sources */
  uint32_t k;           /* 1 .. the workspace's max_sources (<= 256) */
  uint8_t* d_levels;    /* device, k * n bytes, 16-byte aligned: [source][vertex] */
} pbg_batch_job;

/* Enqueues one fused launch of all jobs on `stream` (0 = CUDA's default
 * stream).  The source arrays are staged before the call returns; results are
 * valid once the stream is synchronised.  A batch object must not be reused
 * before its previous launch has been staged (the call waits for that). */
int pbg_bfs_batch(pbg_batch* b, const pbg_batch_job* jobs, uint32_t njobs, const pbg_bfs_opts* opts,
                  void* stream);

typedef struct pbg_batch_stats {
  uint32_t levels;      /* levels of the job (deepest source + 1) */
  uint32_t pull_levels; /* levels run bottom-up (pull) */
  uint32_t push_levels; /* levels run top-down (push) */
  uint32_t error;       /* device error word of the job */
  float device_ms;      /* device time of the whole fused launch */
} pbg_batch_stats;
/* Per-job statistics of the last launch that used ws, launched through b. */
int pbg_batch_job_stats(pbg_batch* b, pbg_msbfs* ws, pbg_batch_stats* st);

/* Per-level trace of ws's job in the last launch through b (first 64
 * levels; fields as pbg_level_trace, bottom_up: 0 sparse push, 1 pull,
 * 2 dense push).  Blocks until that launch is done. */
int pbg_batch_job_trace(pbg_batch* b, pbg_msbfs* ws, pbg_level_trace* out, uint32_t cap, uint32_t* count);

/* Convenience: one job of k <= 256 sources on g, host output
 * levels_out[k * n]; blocks. */
int pbg_bfs_multi(pbg_graph* g, const uint32_t* srcs, uint32_t k, const pbg_bfs_opts* opts, uint8_t* levels_out,
                  pbg_batch_stats* st);

/* Per-level trace of the last pbg_bfs_multi on g. */
int pbg_bfs_multi_trace(pbg_graph* g, pbg_level_trace* out, uint32_t cap, uint32_t* count);

/* ------------------------------------------------------------------ checker */
/* The reference's check on the device.  pbg_bfs_check restates checkBFS
 * (benchmarks/breadthFirstSearch/bench/BFSCheck.C:39-90) for a device parent
 * array (PBG_NONE = unreached): levels by pointer doubling on the parent
 * tree, then the start must be its own parent and every other vertex must
 * sit one level below its lowest neighbour, or be unreached with every
 * neighbour unreached.  A parent that is neither PBG_NONE nor a vertex fails
 * first (smallest such vertex).  Doubling counts wrap at 32 bits as the
 * reference's do (so a parent cycle settles and fails the predicate); a
 * numbering still unsettled after 64 rounds fails with bad_vertex = n.
 * PBG_CHECK_EDGES also requires each parent to be a
 * neighbour of its vertex.  pbg_levels_check applies the level predicate to
 * `rows` uint8 level rows (row i from srcs[i], 255 = unreached) such as the
 * batched search writes.  Both block (graph's stream); bad_vertex = PBG_NONE
 * when everything holds, else the first failing (row, vertex) with its level
 * and lowest neighbour level (n = unreached).  Like the reference's check,
 * the level predicate reads a vertex's out-edges as its in-edges, so it
 * holds for symmetric graphs only; on a directed graph a correct search can
 * fail it. */
#define PBG_CHECK_EDGES 1u
typedef struct pbg_check_result {
  uint32_t bad_vertex;
  uint32_t row;
  uint32_t level;
  uint32_t min_neighbor_level;
} pbg_check_result;
int pbg_bfs_check(pbg_graph* g, uint32_t src, const uint32_t* d_parent, uint32_t flags, pbg_check_result* res);
int pbg_levels_check(pbg_graph* g, const uint32_t* srcs, uint32_t rows, const uint8_t* d_levels,
                     pbg_check_result* res);

/* ----------------------------------------------------------------- autotune */
/* No reference counterpart (PBBS fixes alpha = beta = 20 in
 * common/ligraLight.h:122,130).  Picks, for one resident graph, the options
 * of the single-source search (block_threads, chunk_min_degree, alpha, beta)
 * or with PBG_TUNE_BATCHED the switch of the batched search (alpha against
 * beta = 20), by coordinate descent over candidate values (two sweeps),
 * timing each candidate's device time summed over the sample sources after
 * an untimed pass.  The result is stored on the graph (unless
 * PBG_TUNE_NO_STORE) and used by pbg_bfs, pbg_bfs_device, pbg_bfs_multi,
 * pbg_bfs_batch and the server whenever they get no options.  inout (may be
 * NULL): its parent_mode and direction are kept; it receives the result.
 * The sample holds 1..PBG_TUNE_MAX_SOURCES sources, or 1..256 with
 * PBG_TUNE_BATCHED (one batched job; a batched workspace of the graph's that
 * is narrower than the sample is replaced by one as wide as the sample).
 * Blocks; runs on the graph's stream. */
#define PBG_TUNE_BATCHED 1u
#define PBG_TUNE_NO_STORE 2u
#define PBG_TUNE_MAX_SOURCES 16
typedef struct pbg_tune_report {
  uint32_t evaluations; /* distinct option sets timed */
  float default_ms;     /* device time of the defaults over the samples */
  float best_ms;        /* device time of the result */
} pbg_tune_report;
int pbg_autotune(pbg_graph* g, const uint32_t* srcs, uint32_t nsrc, uint32_t flags, pbg_bfs_opts* inout,
                 pbg_tune_report* rep);
/* Drops the graph's tuned options (calls without options use the defaults). */
int pbg_autotune_clear(pbg_graph* g);

/* --------------------------------------------------------- level checksums */
/* Order-free 64-bit checksum of each of `rows` uint8 level rows of n bytes
 * (row i at d_levels + i*n): the sum over the row's 8-byte little-endian words
 * w_j (bytes past n read as 0xFF) of mix64(w_j + (j+1) * 0x9E3779B97F4A7C15),
 * mix64 = SplitMix64's output function.  d_out: rows uint64 in device memory.
 * Lets served results be verified without moving them. */
int pbg_levels_checksum(const uint8_t* d_levels, uint32_t rows, uint32_t n, uint64_t* d_out, void* stream);
/* The same checksum of a uint32 level array mapped to bytes (>= 255 -> 255). */
int pbg_levels32_checksum(const uint32_t* d_levels, uint32_t n, uint64_t* d_out, void* stream);

/* ------------------------------------------------------------- BFS service */
/* No reference counterpart.  A continuous-batching service over
 * device-resident graphs: queries (graph, source) are admitted as job slots
 * and device memory free up, batched up to max_sources per graph into jobs,
 * and the jobs of all graphs run as fused multi-source launches (the batched
 * path above).  Up to `streams` launches are in flight at once, each on its
 * own stream with 1/streams of the GPU's resident blocks, so queries arriving
 * while others run start on the next free launch and their work overlaps on
 * the device.  Job slots (workspace + uint8 level rows) are pre-allocated per
 * graph within hbm_budget_bytes: admission is bounded by that budget.  A
 * query's result is its level array (optionally copied to a host buffer) and
 * its checksum (pbg_levels_checksum of its row). */
typedef struct pbg_server pbg_server;
#define PBG_SERVER_CHECKSUM 1u /* compute each query's level checksum */
/* Device memory a server leaves free when it sizes its job slots. */
#define PBG_SERVER_HBM_RESERVE (512ull << 20)
typedef struct pbg_server_config {
  /* Device memory for job slots (workspaces + level rows), at most.  At
   * create the server clamps it to the device's free memory (cudaMemGetInfo)
   * less PBG_SERVER_HBM_RESERVE and its launch slots' own buffers, so a
   * budget above what is free admits the job slots that fit instead of
   * failing; pbg_server_stats reports the budget it used. */
  uint64_t hbm_budget_bytes;
  uint32_t max_sources;      /* sources per job, 1..256 (above 64: two-word, above 128: four-word masks) */
  uint32_t max_jobs;         /* jobs per fused launch, 1..128 */
  uint32_t streams;          /* launches in flight, 1..16 */
  uint32_t flags;            /* PBG_SERVER_* */
  /* Optional wider jobs for small graphs: graphs of at most
   * wide_max_vertices vertices take up to wide_sources (1..256) queries per
   * job instead of max_sources; 0 = off.  A launch holds jobs of one mask
   * width, so such graphs are never fused with the others. */
  uint32_t wide_sources;
  uint32_t wide_max_vertices;
  /* A launch takes jobs while the edge counts of their graphs add up to at
   * most this (it always takes one); 0 = no limit.  Short launches keep the
   * launch slots interleaving: on a B200, 2^29 (two jobs on a 2^23-vertex,
   * 16n rMat graph) served the 8-graph stream at 9.95-10.2x plain launches,
   * against 8.5-9.4x without a limit. */
  uint64_t max_launch_edges;
} pbg_server_config;

typedef struct pbg_query_result {
  uint64_t id;
  uint32_t graph;
  uint32_t src;
  uint32_t status;    /* PBG_OK or an error code */
  uint32_t levels;    /* levels of the job the query ran in */
  uint64_t checksum;  /* level checksum (PBG_SERVER_CHECKSUM) */
  double t_submit_us; /* server clock: submitted, launched, results ready */
  double t_launch_us;
  double t_done_us;
} pbg_query_result;

typedef struct pbg_server_stats {
  uint64_t submitted;
  uint64_t completed;
  uint64_t launches;
  uint64_t jobs;
  uint32_t max_inflight; /* most launches seen in flight together */
  uint32_t slots;        /* job slots allocated within the budget */
  uint64_t slot_bytes;   /* device bytes those slots take */
  uint64_t budget_bytes; /* the slot budget used: hbm_budget_bytes clamped to free HBM */
  uint64_t free_bytes;   /* free device memory when the server was created */
} pbg_server_stats;

/* The graphs stay owned by the caller and must outlive the server. */
int pbg_server_create(pbg_graph* const* graphs, uint32_t ngraphs, const pbg_server_config* cfg,
                      pbg_server** out);
/* Thread-safe.  levels_out: NULL, or host memory of n(graph) bytes that
 * receives the query's uint8 levels before its result is posted. */
int pbg_server_submit(pbg_server* s, uint32_t graph, uint32_t src, uint8_t* levels_out, uint64_t* id);
/* Open-loop load: a server thread submits query i at arrival_us[i]
 * (microseconds after this call).  Arrays are copied. */
int pbg_server_replay(pbg_server* s, const uint32_t* graph, const uint32_t* src, const double* arrival_us,
                      uint32_t count);
/* Completed queries (up to cap), waiting up to wait_ms for the first. */
int pbg_server_poll(pbg_server* s, pbg_query_result* out, uint32_t cap, uint32_t* count, int wait_ms);
/* Waits until every submitted (and replayed) query has completed. */
int pbg_server_drain(pbg_server* s, int timeout_ms);
int pbg_server_stats_get(pbg_server* s, pbg_server_stats* st);
/* Finishes in-flight launches, then frees the server. */
int pbg_server_destroy(pbg_server* s);

#ifdef __cplusplus
}
#endif
#endif /* PBBS_BFS_H_ */
