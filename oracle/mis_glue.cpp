// mis_glue.cpp -- C entry points onto the reference's own maximal independent
// set code, compiled unmodified from the pbbsbench sources against the
// project parlay shim.
//
// TEST INFRASTRUCTURE: built by oracle/Makefile into oracle/_ref/libpbbsmis.so;
// used by tests (to pin the C restatement of serialMIS in bfs_oracle.c and to
// compare GPU flag arrays with the reference's own output) and by bench.py's
// CPU-baseline leg.  Never linked into the product library.  The reference's
// checker runs as its own binary (oracle/_ref/MISCheck) on files, as the
// benchmark's test harness runs it.
//
// Each MIS.C is compiled with -DmaximalIndependentSet=<name> so the
// implementations of benchmarks/maximalIndependentSet/bench/MIS.h:8 can live in
// one library.
#include <chrono>
#include <cstdint>
#include <cstring>

#include "MIS.h"  // benchmarks/maximalIndependentSet/bench/MIS.h: Graph = graph<uint, uint>
#include "common/graph.h"

parlay::sequence<char> pbbsref_serialMIS(Graph const& G);
parlay::sequence<char> pbbsref_ndMIS(Graph const& G);

namespace {
using mis_fn = parlay::sequence<char> (*)(Graph const&);

mis_fn pick(int which) {
  switch (which) {
    case 0: return pbbsref_serialMIS;
    case 1: return pbbsref_ndMIS;
    default: return nullptr;
  }
}
}  // namespace

extern "C" {

// graph<uint,uint> from CSR arrays, degrees added as MISTime's reader leaves
// them (readGraphFromFile fills offsets and edges; graph::operator[] reads
// degrees from offsets).
void* pbbsref_mis_graph_new(uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* edges) {
  auto off = parlay::sequence<edgeId>::from_function(n + 1, [&](size_t i) { return (edgeId)offsets[i]; });
  auto edg = parlay::sequence<vertexId>::from_function(m, [&](size_t i) { return (vertexId)edges[i]; });
  return new Graph(std::move(off), std::move(edg), n);
}

void pbbsref_mis_graph_free(void* g) { delete static_cast<Graph*>(g); }

// which: 0 serialMIS, 1 ndMIS.  flags_out[v]: 1 in the set, 2 not.
int pbbsref_mis_g(void* g, int which, uint8_t* flags_out) {
  mis_fn f = pick(which);
  if (!f || !g) return -1;
  const Graph& G = *static_cast<Graph*>(g);
  parlay::sequence<char> fl = f(G);
  if (fl.size() != G.n) return -2;
  std::memcpy(flags_out, fl.data(), fl.size());
  return 0;
}

// Times `rounds` calls after `warmup_s` seconds of untimed calls
// (common/time_loop.h:3-18).  Writes per-round seconds.
int pbbsref_time_mis(void* g, int which, int rounds, double warmup_s, double* secs_out) {
  mis_fn f = pick(which);
  if (!f || !g) return -1;
  const Graph& G = *static_cast<Graph*>(g);
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  while (std::chrono::duration<double>(clk::now() - t0).count() < warmup_s) {
    parlay::sequence<char> fl = f(G);
  }
  for (int r = 0; r < rounds; r++) {
    auto a = clk::now();
    parlay::sequence<char> fl = f(G);
    auto b = clk::now();
    secs_out[r] = std::chrono::duration<double>(b - a).count();
  }
  return 0;
}
}
