/*
 * bfs_oracle.c -- CPU restatement of PBBS breadthFirstSearch, used ONLY as a
 * test oracle.
 *
 * THIS FILE IS TEST INFRASTRUCTURE.  It is the checker for the CUDA library in
 * pbbsbench_b200/csrc: tests, the smoke entry point and the CPU-baseline leg of
 * bench.py may call it; the product path never does.  Parity of this
 * restatement is pinned against the reference's own BFS code compiled here
 * (oracle/Makefile -> oracle/_ref), see tests/test_oracle.py.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths are relative to the pbbsbench project root).
 *
 * Conventions
 *   - vertex ids are uint32; the reference's signed -1 "unvisited" parent is
 *     the bit pattern 0xFFFFFFFF (benchmarks/breadthFirstSearch/bench/BFS.h:4-10).
 *   - CSR: offsets[n+1] (uint32, offsets[n] = m) and edges[m] (uint32),
 *     as graph<int,uint> in common/graph.h:104-152.
 *   - levels: BFS distance from the source; unreached = 0xFFFFFFFF.
 *     (BFSCheck's level_number uses n for unreached; orc_level_number keeps
 *     that convention because it restates that function.)
 *
 * Generators use SplitMix64's output mix (Steele, Lea, Flood, "Fast
 * splittable pseudorandom number generators", OOPSLA 2014) as the hash
 * because parlay::hash64, which PBBS's generators use (common/dataGen.h:11-35),
 * lives in the unvendored parlaylib submodule.  The construction rules
 * (rMat recursion, torus wiring, symmetrise + dedup + sorted lists) follow
 * the reference; the bits of the graphs therefore differ from PBBS files.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_NONE 0xFFFFFFFFu

/* ------------------------------------------------------------------ hash */

/* SplitMix64 output function applied to x + golden gamma. */
uint64_t orc_hash64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

/* Integer threshold for a probability p: r31 < T  <=>  "r < p" with r a
 * 31-bit uniform draw.  Restates the double comparison of rMatRec
 * (testData/graphData/rMatGraph.C:58-61) in integers so that CPU and GPU
 * draw identical graphs. */
uint32_t orc_prob_threshold(double p) {
  double t = p * 2147483648.0 + 0.5;
  if (t < 0) t = 0;
  if (t > 4294967295.0) t = 4294967295.0;
  return (uint32_t)t;
}

/* ------------------------------------------------------------ generators */

/* rMat edge i (testData/graphData/rMatGraph.C:53-69): per edge a start and a
 * stride key, then one draw per recursion level, top level first. */
static inline void rmat_edge(uint64_t i, uint64_t h, uint32_t logn,
                             uint32_t ta, uint32_t tab, uint32_t tabc,
                             uint32_t* pu, uint32_t* pv) {
  uint64_t rs = orc_hash64((2 * i) * h);
  uint64_t st = orc_hash64((2 * i + 1) * h);
  uint32_t u = 0, v = 0;
  for (uint32_t k = 0; k < logn; k++) {
    uint32_t half = 1u << (logn - 1 - k);
    uint32_t r = (uint32_t)(orc_hash64(rs + (uint64_t)k * st) & 0x7FFFFFFFu);
    if (r < ta) {
    } else if (r < tab) {
      v += half;
    } else if (r < tabc) {
      u += half;
    } else {
      u += half;
      v += half;
    }
  }
  *pu = u;
  *pv = v;
}

/* m rMat samples on n = 2^logn vertices (rMatGraph.C:72-79). */
void orc_gen_rmat(uint32_t logn, uint64_t m, uint64_t seed, uint32_t ta,
                  uint32_t tab, uint32_t tabc, uint32_t* us, uint32_t* vs) {
  uint64_t h = orc_hash64(seed);
  for (uint64_t i = 0; i < m; i++) rmat_edge(i, h, logn, ta, tab, tabc, &us[i], &vs[i]);
}

/* 3-D torus, dn^3 vertices, 3 edges per vertex to the +1 neighbour along each
 * axis with wraparound (testData/graphData/gridGraph.C:53-72). */
void orc_gen_torus3d(uint32_t dn, uint32_t* us, uint32_t* vs) {
  uint64_t nn = (uint64_t)dn * dn * dn;
  for (uint64_t l = 0; l < nn; l++) {
    uint64_t i = l / ((uint64_t)dn * dn), j = (l / dn) % dn, k = l % dn;
    us[3 * l] = us[3 * l + 1] = us[3 * l + 2] = (uint32_t)l;
    vs[3 * l] = (uint32_t)((((i + 1) % dn) * dn + j) * dn + k);
    vs[3 * l + 1] = (uint32_t)((i * dn + (j + 1) % dn) * dn + k);
    vs[3 * l + 2] = (uint32_t)((i * dn + j) * dn + (k + 1) % dn);
  }
}

/* Random-local graph: vertex i gets `deg` out-neighbours (i + off) mod n with
 * off uniform in [-w, w] \ {0}; a draw that lands on i itself is redrawn, as
 * the do/while of testData/graphData/randLocalGraph.C:46-57 does.  (The
 * reference draws off from a heavy-tailed, dimension-dependent law; the
 * uniform window is the workload this library is measured on.) */
void orc_gen_randlocal(uint32_t n, uint32_t deg, uint32_t w, uint64_t seed,
                       uint32_t* us, uint32_t* vs) {
  uint64_t hs = orc_hash64(seed);
  uint64_t span = 2 * (uint64_t)w + 1;
  for (uint64_t i = 0; i < n; i++) {
    for (uint32_t k = 0; k < deg; k++) {
      uint64_t x = orc_hash64(hs + i * deg + k);
      uint32_t j;
      for (;;) {
        int64_t off = (int64_t)(x % span) - (int64_t)w;
        int64_t t = ((int64_t)i + off) % (int64_t)n;
        if (t < 0) t += n;
        j = (uint32_t)t;
        if (j != i) break;
        x = orc_hash64(x);
      }
      us[i * deg + k] = (uint32_t)i;
      vs[i * deg + k] = j;
    }
  }
}

/* ---------------------------------------------------------- radix sort */

static void radix_sort_u64(uint64_t* a, uint64_t* tmp, uint64_t m) {
  static uint64_t cnt[256];
  for (int shift = 0; shift < 64; shift += 8) {
    memset(cnt, 0, sizeof(cnt));
    for (uint64_t i = 0; i < m; i++) cnt[(a[i] >> shift) & 255]++;
    int skip = 0;
    for (int b = 0; b < 256; b++)
      if (cnt[b] == m) skip = 1;
    if (skip) continue;
    uint64_t s = 0;
    for (int b = 0; b < 256; b++) {
      uint64_t c = cnt[b];
      cnt[b] = s;
      s += c;
    }
    for (uint64_t i = 0; i < m; i++) tmp[cnt[(a[i] >> shift) & 255]++] = a[i];
    memcpy(a, tmp, m * sizeof(uint64_t));
  }
}

/* Random relabelling permutation: new id of vertex `old` is its rank when
 * vertices are ordered by (hash(seed) + old) mixed, ties by id.  Plays the role
 * of parlay::random_permutation in graphReorder (common/graphUtils.h:165-189). */
void orc_random_permutation(uint32_t n, uint64_t seed, uint32_t* new_id) {
  uint64_t hs = orc_hash64(seed);
  uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t* t = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  for (uint64_t i = 0; i < n; i++) k[i] = (orc_hash64(hs + i) & 0xFFFFFFFF00000000ull) | i;
  radix_sort_u64(k, t, n);
  for (uint64_t p = 0; p < n; p++) new_id[(uint32_t)(k[p] & 0xFFFFFFFFu)] = (uint32_t)p;
  free(k);
  free(t);
}

/* Symmetric CSR from an edge list: drop self loops, add every reversed edge,
 * sort by (u, v), remove duplicates, count per source, scan
 * (common/graphUtils.h:54-94).  Each adjacency list ends up ascending.
 * If relabel != NULL, endpoints are first mapped through it (graphReorder,
 * graphUtils.h:165-189).  Returns the number of directed edges written, or
 * UINT64_MAX if edges_cap is too small.  offsets has n+1 entries. */
uint64_t orc_csr_symmetric(uint32_t n, uint64_t m_in, const uint32_t* us,
                           const uint32_t* vs, const uint32_t* relabel,
                           uint32_t* offsets, uint32_t* edges, uint64_t edges_cap) {
  uint64_t cap = 2 * m_in ? 2 * m_in : 1;
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * cap);
  uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * cap);
  uint64_t k = 0;
  for (uint64_t i = 0; i < m_in; i++) {
    uint32_t u = us[i], v = vs[i];
    if (relabel) {
      u = relabel[u];
      v = relabel[v];
    }
    if (u == v) continue;
    key[k++] = ((uint64_t)u << 32) | v;
    key[k++] = ((uint64_t)v << 32) | u;
  }
  radix_sort_u64(key, tmp, k);
  uint64_t m = 0;
  for (uint64_t i = 0; i < k; i++)
    if (i == 0 || key[i] != key[i - 1]) key[m++] = key[i];
  if (m > edges_cap) {
    free(key);
    free(tmp);
    return UINT64_MAX;
  }
  memset(offsets, 0, sizeof(uint32_t) * ((uint64_t)n + 1));
  for (uint64_t i = 0; i < m; i++) {
    offsets[(key[i] >> 32) + 1]++;
    edges[i] = (uint32_t)(key[i] & 0xFFFFFFFFu);
  }
  for (uint64_t v = 0; v < n; v++) offsets[v + 1] += offsets[v];
  free(key);
  free(tmp);
  return m;
}

/* ------------------------------------------------------------------ BFS */

/* Sequential FIFO BFS (benchmarks/breadthFirstSearch/serialBFS/BFS.C:32-55):
 * the parent of a vertex is the first queue vertex that discovers it,
 * scanning each adjacency list in stored order.  parent[start] = start,
 * unvisited = 0xFFFFFFFF.  Returns the number of reached vertices. */
uint64_t orc_bfs_serial(uint32_t n, const uint32_t* offsets, const uint32_t* edges,
                        uint32_t start, uint32_t* parent) {
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (uint64_t i = 0; i < n; i++) parent[i] = ORC_NONE;
  uint64_t bot = 0, top = 1;
  q[0] = start;
  parent[start] = start;
  while (top > bot) {
    uint32_t v = q[bot++];
    for (uint32_t j = offsets[v]; j < offsets[v + 1]; j++) {
      uint32_t ngh = edges[j];
      if (parent[ngh] == ORC_NONE) {
        q[top++] = ngh;
        parent[ngh] = v;
      }
    }
  }
  free(q);
  return top;
}

/* BFS distances from start (unreached = 0xFFFFFFFF).  Returns the number of
 * levels (eccentricity + 1).  Same traversal as orc_bfs_serial. */
uint32_t orc_bfs_levels(uint32_t n, const uint32_t* offsets, const uint32_t* edges,
                        uint32_t start, uint32_t* level) {
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (uint64_t i = 0; i < n; i++) level[i] = ORC_NONE;
  uint64_t bot = 0, top = 1;
  q[0] = start;
  level[start] = 0;
  uint32_t maxl = 0;
  while (top > bot) {
    uint32_t v = q[bot++];
    uint32_t lv = level[v];
    if (lv > maxl) maxl = lv;
    for (uint32_t j = offsets[v]; j < offsets[v + 1]; j++) {
      uint32_t ngh = edges[j];
      if (level[ngh] == ORC_NONE) {
        q[top++] = ngh;
        level[ngh] = lv + 1;
      }
    }
  }
  free(q);
  return maxl + 1;
}

/* Deterministic parents.  which = 0: the smallest neighbour one level up
 * (the min-parent rule, no reference counterpart); which = 1: the largest
 * such neighbour, the rule deterministicBFS reaches through write_max with
 * std::less (benchmarks/breadthFirstSearch/deterministicBFS/BFS.C:60-74).
 * Candidates are found along out-edges u -> v with level[v] == level[u] + 1,
 * which is what a top-down round tries. */
void orc_bfs_det_parent(uint32_t n, const uint32_t* offsets, const uint32_t* edges,
                        uint32_t start, int which, uint32_t* parent) {
  uint32_t* level = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  orc_bfs_levels(n, offsets, edges, start, level);
  for (uint64_t i = 0; i < n; i++) parent[i] = ORC_NONE;
  for (uint64_t u = 0; u < n; u++) {
    if (level[u] == ORC_NONE) continue;
    for (uint32_t j = offsets[u]; j < offsets[u + 1]; j++) {
      uint32_t v = edges[j];
      if (v == start || level[v] != level[u] + 1) continue;
      if (parent[v] == ORC_NONE)
        parent[v] = (uint32_t)u;
      else if (which == 0 && u < parent[v])
        parent[v] = (uint32_t)u;
      else if (which == 1 && u > parent[v])
        parent[v] = (uint32_t)u;
    }
  }
  parent[start] = start;
  free(level);
}

/* level_number (benchmarks/breadthFirstSearch/bench/BFSCheck.C:39-56):
 * repeated pointer doubling over (count, ptr) pairs until a fixed point;
 * roots (parent == -1 or parent == self) have count 0; the result is the
 * count, or n when the chain ends at an unvisited vertex.  The reference
 * loops forever on a parent cycle; here the doubling is capped at 64 rounds
 * and a non-converged chain returns -1 (the caller reports a failed check). */
int orc_level_number(uint32_t n, const uint32_t* parent, uint32_t* level) {
  uint32_t* cnt = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* ptr = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* cnt2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* ptr2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (uint64_t i = 0; i < n; i++) {
    if (parent[i] == ORC_NONE || parent[i] == i) {
      cnt[i] = 0;
      ptr[i] = (uint32_t)i;
    } else {
      cnt[i] = 1;
      ptr[i] = parent[i];
    }
  }
  int converged = 0;
  for (int round = 0; round < 64 && !converged; round++) {
    converged = 1;
    for (uint64_t i = 0; i < n; i++) {
      uint32_t p = ptr[i];
      cnt2[i] = cnt[i] + cnt[p];
      ptr2[i] = ptr[p];
      if (cnt2[i] != cnt[i] || ptr2[i] != ptr[i]) converged = 0;
    }
    uint32_t* t;
    t = cnt; cnt = cnt2; cnt2 = t;
    t = ptr; ptr = ptr2; ptr2 = t;
  }
  for (uint64_t i = 0; i < n; i++) level[i] = (parent[ptr[i]] == ORC_NONE) ? n : cnt[i];
  free(cnt); free(ptr); free(cnt2); free(ptr2);
  return converged ? 0 : -1;
}

/* checkBFS (benchmarks/breadthFirstSearch/bench/BFSCheck.C:59-90) for any
 * start, strengthened: besides the reference's level predicate
 *   v == start ? parent[v] == v
 *              : (level[v] == n && minNgh == n) || level[v] == minNgh + 1
 * (minNgh = min level over v's out-neighbours, n for degree 0), a visited
 * v != start must have parent[v] among its neighbours (the reference never
 * checks edge existence).  Parent ids must be < n.  Returns -1 on success,
 * else the first failing vertex (n for a size/cycle failure).  check_edges = 0
 * gives the reference predicate alone. */
int64_t orc_check_bfs(uint32_t n, const uint32_t* offsets, const uint32_t* edges,
                      uint32_t start, const uint32_t* parent, int check_edges) {
  for (uint64_t i = 0; i < n; i++)
    if (parent[i] != ORC_NONE && parent[i] >= n) return (int64_t)i;
  uint32_t* level = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  if (orc_level_number(n, parent, level) != 0) {
    free(level);
    return (int64_t)n;
  }
  int64_t bad = -1;
  for (uint64_t v = 0; v < n && bad < 0; v++) {
    if (v == start) {
      if (parent[v] != v) bad = (int64_t)v;
      continue;
    }
    uint32_t mn = n;
    for (uint32_t j = offsets[v]; j < offsets[v + 1]; j++)
      if (level[edges[j]] < mn) mn = level[edges[j]];
    int ok = (level[v] == n && mn == n) || (level[v] == mn + 1);
    if (ok && check_edges && parent[v] != ORC_NONE) {
      int found = 0;
      for (uint32_t j = offsets[v]; j < offsets[v + 1] && !found; j++)
        if (edges[j] == parent[v]) found = 1;
      ok = found;
    }
    if (!ok) bad = (int64_t)v;
  }
  free(level);
  return bad;
}

/* Batched levels: k independent BFS runs, uint8 level per (source, vertex),
 * row-major [k][n], 255 = unreached.  Returns 0, or -1 if some level does not
 * fit in 8 bits (>= 255). */
int orc_bfs_levels_u8(uint32_t n, const uint32_t* offsets, const uint32_t* edges,
                      uint32_t k, const uint32_t* srcs, uint8_t* levels) {
  uint32_t* lv = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  int rc = 0;
  for (uint32_t s = 0; s < k; s++) {
    orc_bfs_levels(n, offsets, edges, srcs[s], lv);
    for (uint64_t i = 0; i < n; i++) {
      uint32_t l = lv[i];
      if (l != ORC_NONE && l >= 255) rc = -1;
      levels[(uint64_t)s * n + i] = (l == ORC_NONE || l >= 255) ? 255 : (uint8_t)l;
    }
  }
  free(lv);
  return rc;
}

/* ------------------------------------------------------------------ MIS */
/* Restates serialMIS (benchmarks/maximalIndependentSet/serialMIS/MIS.C:33-47):
 * vertices in id order; i joins the set (flag 1) unless a neighbour already
 * in the set is adjacent (flag 2).  The flag of i is set to 1 before its list
 * is scanned, so a self loop puts i out of the set, as in the reference.
 * flags: 1 in the set, 2 not in it (the reference's char flags). */
void orc_mis_serial(uint32_t n, const uint32_t* offsets, const uint32_t* edges, uint8_t* flags) {
  for (uint32_t i = 0; i < n; i++) flags[i] = 0;
  for (uint32_t i = 0; i < n; i++) {
    flags[i] = 1;
    for (uint32_t j = offsets[i]; j < offsets[i + 1]; j++) {
      if (flags[edges[j]] == 1) {
        flags[i] = 2;
        break;
      }
    }
  }
}

/* Restates checkMaximalIndependentSet (maximalIndependentSet/bench/
 * MISCheck.C:39-66): no vertex in the set has a neighbour in the set
 * (independence), and every vertex not in the set has one (maximality).
 * Returns -1 when valid, else the smallest bad vertex (as the reference's
 * minm reduction picks it). */
int64_t orc_check_mis(uint32_t n, const uint32_t* offsets, const uint32_t* edges, const uint8_t* flags) {
  for (uint32_t i = 0; i < n; i++) {
    int has = 0;
    for (uint32_t j = offsets[i]; j < offsets[i + 1]; j++) {
      if (flags[edges[j]] == 1) {
        has = 1;
        if (flags[i] == 1) return i;
      }
    }
    if (flags[i] != 1 && !has) return i;
  }
  return -1;
}
