// ref_glue.cpp -- C entry points onto the reference's own BFS code, compiled
// unmodified from the pbbsbench sources against the project parlay shim.
//
// TEST INFRASTRUCTURE: built by oracle/Makefile into oracle/_ref/libpbbsref.so,
// used by tests (to pin the C restatement in bfs_oracle.c and to check GPU
// parent arrays with the reference's own checkBFS) and by bench.py's
// CPU-baseline leg.  Never linked into the product library.
//
// Each BFS.C is compiled with -DBFS=<name> so the four implementations of
// benchmarks/breadthFirstSearch/bench/BFS.h:11 can live in one library, and
// bench/BFSCheck.C with -Dmain=pbbsref_bfscheck_main so its checkBFS
// (BFSCheck.C:59-90) and level_number (BFSCheck.C:39-56) can be called here.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "BFS.h"  // benchmarks/breadthFirstSearch/bench/BFS.h
#include "common/graph.h"

// The reference's graph reader (common/graphIO.h:191-215).  Its header
// defines non-inline globals, so it is not included a second time here; the
// instantiation for <vertexId, edgeId> comes from bench/BFSCheck.C, whose
// main reads its graph with it.
namespace benchIO {
template <class intV, class intE>
graph<intV, intE> readGraphFromFile(char* fname);
}

using vtx_seq = parlay::sequence<vertexId>;

parlay::sequence<vertexId> pbbsref_serialBFS(vertexId, const Graph&, bool);
parlay::sequence<vertexId> pbbsref_backForwardBFS(vertexId, const Graph&, bool);
parlay::sequence<vertexId> pbbsref_deterministicBFS(vertexId, const Graph&, bool);
parlay::sequence<vertexId> pbbsref_simpleBFS(vertexId, const Graph&, bool);
int checkBFS(size_t start, vtx_seq const& parents, Graph const& G);
vtx_seq level_number(vtx_seq const& parent);

namespace {
using bfs_fn = parlay::sequence<vertexId> (*)(vertexId, const Graph&, bool);

bfs_fn pick(int which) {
  switch (which) {
    case 0: return pbbsref_serialBFS;
    case 1: return pbbsref_backForwardBFS;
    case 2: return pbbsref_deterministicBFS;
    case 3: return pbbsref_simpleBFS;
    default: return nullptr;
  }
}

// Builds graph<int,uint> from CSR arrays and adds degrees, as BFSTime's main
// does before timing (bench/BFSTime.C:58-59).
Graph* make_graph(uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* edges) {
  auto off = parlay::sequence<edgeId>::from_function(n + 1, [&](size_t i) { return (edgeId)offsets[i]; });
  auto edg = parlay::sequence<vertexId>::from_function(m, [&](size_t i) { return (vertexId)edges[i]; });
  Graph* G = new Graph(std::move(off), std::move(edg), n);
  G->addDegrees();
  return G;
}
}  // namespace

extern "C" {

int pbbsref_num_workers(void) { return parlay::num_workers(); }

void* pbbsref_graph_new(uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* edges) {
  return make_graph(n, m, offsets, edges);
}

void pbbsref_graph_free(void* g) { delete static_cast<Graph*>(g); }

// The reference's graph reader (common/graphIO.h:191-215 with the tokens of
// common/IO.h:207-214), as BFSTime's main calls it (bench/BFSTime.C:58).  It
// aborts on a malformed file, so callers pass valid files only.
void* pbbsref_read_graph(const char* path) {
  return new Graph(benchIO::readGraphFromFile<vertexId, edgeId>(const_cast<char*>(path)));
}

// n and m of a graph; its arrays when the pointers are not NULL.
void pbbsref_graph_arrays(void* g, uint64_t* n, uint64_t* m, uint32_t* offsets, uint32_t* edges) {
  const Graph& G = *static_cast<Graph*>(g);
  *n = G.n;
  *m = G.m;
  if (offsets)
    for (size_t i = 0; i <= G.n; i++) offsets[i] = (uint32_t)G.offsets[i];
  if (edges)
    for (size_t i = 0; i < G.m; i++) edges[i] = (uint32_t)G.edges[i];
}

// which: 0 serialBFS, 1 backForwardBFS, 2 deterministicBFS, 3 simpleBFS.
int pbbsref_bfs_g(void* g, int which, uint32_t src, int32_t* parent_out) {
  bfs_fn f = pick(which);
  if (!f || !g) return -1;
  const Graph& G = *static_cast<Graph*>(g);
  vtx_seq p = f((vertexId)src, G, false);
  if (p.size() != G.numVertices()) return -2;
  std::memcpy(parent_out, p.data(), sizeof(int32_t) * p.size());
  return 0;
}

int pbbsref_bfs(int which, uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* edges,
                uint32_t src, int32_t* parent_out) {
  Graph* G = make_graph(n, m, offsets, edges);
  int rc = pbbsref_bfs_g(G, which, src, parent_out);
  delete G;
  return rc;
}

// The reference checker; returns its status (0 = ok, 1 = failed; it prints
// the first failing vertex on stdout).
int pbbsref_check_g(void* g, uint32_t start, const int32_t* parent) {
  const Graph& G = *static_cast<Graph*>(g);
  auto p = vtx_seq::from_function(G.numVertices(), [&](size_t i) { return (vertexId)parent[i]; });
  return checkBFS(start, p, G);
}

int pbbsref_check(uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* edges, uint32_t start,
                  const int32_t* parent) {
  Graph* G = make_graph(n, m, offsets, edges);
  int rc = pbbsref_check_g(G, start, parent);
  delete G;
  return rc;
}

// level_number of the reference checker: level per vertex, n for unreached.
void pbbsref_level_number(uint32_t n, const int32_t* parent, int32_t* level_out) {
  auto p = vtx_seq::from_function(n, [&](size_t i) { return (vertexId)parent[i]; });
  vtx_seq l = level_number(p);
  std::memcpy(level_out, l.data(), sizeof(int32_t) * n);
}

// Times `rounds` calls of one implementation after `warmup_s` seconds of
// untimed calls (common/time_loop.h:3-18).  Writes per-round seconds.
int pbbsref_time_bfs(void* g, int which, uint32_t src, int rounds, double warmup_s, double* secs_out) {
  bfs_fn f = pick(which);
  if (!f || !g) return -1;
  const Graph& G = *static_cast<Graph*>(g);
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  while (std::chrono::duration<double>(clk::now() - t0).count() < warmup_s) {
    vtx_seq p = f((vertexId)src, G, false);
  }
  for (int r = 0; r < rounds; r++) {
    auto a = clk::now();
    vtx_seq p = f((vertexId)src, G, false);
    auto b = clk::now();
    secs_out[r] = std::chrono::duration<double>(b - a).count();
  }
  return 0;
}
}
