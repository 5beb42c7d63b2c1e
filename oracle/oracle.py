"""CPU oracle for the BFS hot path -- TEST INFRASTRUCTURE ONLY.

Two layers, both checkers, never the product:

* ``liboracle.so`` (bfs_oracle.c): a plain-C restatement of the reference's
  BFS (serialBFS/BFS.C:32-55), its checker (bench/BFSCheck.C:39-90), the
  deterministic-parent rules (deterministicBFS/BFS.C:60-74 and the min-parent
  variant) and the seeded graph generators (testData/graphData/*.C rules).
* ``_ref/libpbbsref.so``: the reference's OWN sources (serialBFS, simpleBFS,
  backForwardBFS + common/ligraLight.h, deterministicBFS, bench/BFSCheck.C)
  compiled unmodified against the project parlay shim.  It pins the
  restatement (tests/test_oracle.py) and is the timed CPU
  baseline in bench.py.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes
import math
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NONE = 0xFFFFFFFF

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def reference_dir() -> str:
    """The reference checkout: $PBBS_REF, else a directory named `reference`
    beside this repository (it may not exist: only the oracle's build of the
    reference's own sources needs it)."""
    return os.environ.get("PBBS_REF") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and, with ref=True, the reference library when
    the reference sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(os.path.join(reference_dir(), "benchmarks", "breadthFirstSearch")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + reference_dir()], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_hash64.restype = ctypes.c_uint64
        L.orc_hash64.argtypes = [ctypes.c_uint64]
        L.orc_prob_threshold.restype = ctypes.c_uint32
        L.orc_prob_threshold.argtypes = [ctypes.c_double]
        L.orc_gen_rmat.restype = None
        L.orc_gen_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                   ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p]
        L.orc_gen_torus3d.restype = None
        L.orc_gen_torus3d.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        L.orc_gen_randlocal.restype = None
        L.orc_gen_randlocal.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                        _u32p, _u32p]
        L.orc_random_permutation.restype = None
        L.orc_random_permutation.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u32p]
        L.orc_csr_symmetric.restype = ctypes.c_uint64
        L.orc_csr_symmetric.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p, ctypes.c_void_p,
                                        _u32p, _u32p, ctypes.c_uint64]
        L.orc_bfs_serial.restype = ctypes.c_uint64
        L.orc_bfs_serial.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p]
        L.orc_bfs_levels.restype = ctypes.c_uint32
        L.orc_bfs_levels.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p]
        L.orc_bfs_det_parent.restype = None
        L.orc_bfs_det_parent.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, ctypes.c_int, _u32p]
        L.orc_level_number.restype = ctypes.c_int
        L.orc_level_number.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        L.orc_check_bfs.restype = ctypes.c_int64
        L.orc_check_bfs.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p, ctypes.c_int]
        L.orc_mis_serial.restype = None
        L.orc_mis_serial.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p]
        L.orc_check_mis.restype = ctypes.c_int64
        L.orc_check_mis.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p]
        L.orc_bfs_levels_u8.restype = ctypes.c_int
        L.orc_bfs_levels_u8.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p, _u8p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libpbbsref.so"))


def ref():
    """The reference's own BFS code (compiled from its sources)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libpbbsref.so")
        if not os.path.exists(path):
            raise FileNotFoundError("reference library not built: make -C oracle ref")
        R = ctypes.CDLL(path)
        R.pbbsref_num_workers.restype = ctypes.c_int
        R.pbbsref_graph_new.restype = ctypes.c_void_p
        R.pbbsref_graph_new.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p]
        R.pbbsref_graph_free.restype = None
        R.pbbsref_graph_free.argtypes = [ctypes.c_void_p]
        R.pbbsref_bfs_g.restype = ctypes.c_int
        R.pbbsref_bfs_g.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, _i32p]
        R.pbbsref_check_g.restype = ctypes.c_int
        R.pbbsref_check_g.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _i32p]
        R.pbbsref_level_number.restype = None
        R.pbbsref_level_number.argtypes = [ctypes.c_uint32, _i32p, _i32p]
        R.pbbsref_time_bfs.restype = ctypes.c_int
        R.pbbsref_time_bfs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_int,
                                       ctypes.c_double, _f64p]
        R.pbbsref_read_graph.restype = ctypes.c_void_p
        R.pbbsref_read_graph.argtypes = [ctypes.c_char_p]
        R.pbbsref_graph_arrays.restype = None
        R.pbbsref_graph_arrays.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p, ctypes.c_void_p]
        _ref = R
    return _ref


# ----------------------------------------------------------------- graphs

def prob_thresholds(a: float, b: float, c: float):
    """Integer thresholds (ta, tab, tabc) for the rMat quadrant draw."""
    L = lib()
    return (L.orc_prob_threshold(a), L.orc_prob_threshold(a + b), L.orc_prob_threshold(a + b + c))


def csr_symmetric(n: int, us: np.ndarray, vs: np.ndarray, relabel: np.ndarray | None = None):
    L = lib()
    m_in = len(us)
    offsets = np.zeros(n + 1, dtype=np.uint32)
    edges = np.zeros(max(1, 2 * m_in), dtype=np.uint32)
    rl = None
    if relabel is not None:
        relabel = np.ascontiguousarray(relabel, dtype=np.uint32)
        rl = relabel.ctypes.data_as(ctypes.c_void_p)
    m = L.orc_csr_symmetric(n, m_in, np.ascontiguousarray(us, np.uint32), np.ascontiguousarray(vs, np.uint32),
                            rl, offsets, edges, len(edges))
    return offsets, edges[:m].copy()


def rmat(logn: int, m: int, seed: int, a: float, b: float, c: float):
    """Symmetric rMat CSR (rMatGraph.C:33-79 + graphUtils.h:54-94)."""
    L = lib()
    us = np.empty(m, np.uint32)
    vs = np.empty(m, np.uint32)
    ta, tab, tabc = prob_thresholds(a, b, c)
    L.orc_gen_rmat(logn, m, seed, ta, tab, tabc, us, vs)
    return csr_symmetric(1 << logn, us, vs)


def torus3d(dn: int, perm_seed: int | None = None):
    """Symmetric 3-D torus CSR (gridGraph.C:53-72), optionally relabelled by a
    seeded random permutation (graphReorder, graphUtils.h:165-189)."""
    L = lib()
    n = dn ** 3
    us = np.empty(3 * n, np.uint32)
    vs = np.empty(3 * n, np.uint32)
    L.orc_gen_torus3d(dn, us, vs)
    rl = None
    if perm_seed is not None:
        rl = np.empty(n, np.uint32)
        L.orc_random_permutation(n, perm_seed, rl)
    return csr_symmetric(n, us, vs, rl)


def randlocal(n: int, deg: int, w: int, seed: int):
    L = lib()
    us = np.empty(n * deg, np.uint32)
    vs = np.empty(n * deg, np.uint32)
    L.orc_gen_randlocal(n, deg, w, seed, us, vs)
    return csr_symmetric(n, us, vs)


def random_permutation(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    lib().orc_random_permutation(n, seed, out)
    return out


# -------------------------------------------------------------------- BFS

def bfs_serial(offsets, edges, src: int) -> np.ndarray:
    n = len(offsets) - 1
    p = np.empty(n, np.uint32)
    lib().orc_bfs_serial(n, offsets, _nonempty(edges), src, p)
    return p


def bfs_levels(offsets, edges, src: int) -> np.ndarray:
    n = len(offsets) - 1
    lv = np.empty(n, np.uint32)
    lib().orc_bfs_levels(n, offsets, _nonempty(edges), src, lv)
    return lv


def bfs_det_parent(offsets, edges, src: int, which: str = "min") -> np.ndarray:
    n = len(offsets) - 1
    p = np.empty(n, np.uint32)
    lib().orc_bfs_det_parent(n, offsets, _nonempty(edges), src, 0 if which == "min" else 1, p)
    return p


def level_number(parent: np.ndarray):
    """BFSCheck's level_number: level per vertex, n for unreached; None on a
    parent cycle."""
    n = len(parent)
    lv = np.empty(n, np.uint32)
    rc = lib().orc_level_number(n, np.ascontiguousarray(parent, np.uint32), lv)
    return None if rc != 0 else lv


def check_bfs(offsets, edges, src: int, parent: np.ndarray, check_edges: bool = True) -> int:
    """-1 if parent is a valid BFS tree from src, else the first bad vertex."""
    n = len(offsets) - 1
    if len(parent) != n:
        return n
    return int(lib().orc_check_bfs(n, offsets, _nonempty(edges), src,
                                   np.ascontiguousarray(parent, np.uint32), 1 if check_edges else 0))


def mis_serial(offsets, edges) -> np.ndarray:
    """serialMIS's flags (1 in the set, 2 not): the greedy set in vertex order."""
    n = len(offsets) - 1
    out = np.empty(n, np.uint8)
    lib().orc_mis_serial(n, np.ascontiguousarray(offsets, np.uint32), _nonempty(edges), out)
    return out


def check_mis(offsets, edges, flags) -> int:
    """-1 if flags is a maximal independent set (MISCheck's test), else the
    smallest bad vertex."""
    n = len(offsets) - 1
    if len(flags) != n:
        return n
    return int(lib().orc_check_mis(n, np.ascontiguousarray(offsets, np.uint32), _nonempty(edges),
                                   np.ascontiguousarray(flags, np.uint8)))


def levels_u8(offsets, edges, srcs) -> np.ndarray:
    n = len(offsets) - 1
    srcs = np.ascontiguousarray(srcs, np.uint32)
    out = np.empty((len(srcs), n), np.uint8)
    rc = lib().orc_bfs_levels_u8(n, offsets, _nonempty(edges), len(srcs), srcs, out.reshape(-1))
    if rc != 0:
        raise OverflowError("a BFS level does not fit in uint8")
    return out


def _nonempty(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint32)
    return a if len(a) else np.zeros(1, np.uint32)


# ---------------------------------------------------- reference's own code

REF_SERIAL, REF_BACKFORWARD, REF_DETERMINISTIC, REF_SIMPLE = 0, 1, 2, 3


class RefGraph:
    """graph<int,uint> held by the reference library (degrees added, as
    bench/BFSTime.C:59 does)."""

    def __init__(self, offsets: np.ndarray, edges: np.ndarray):
        self.n = len(offsets) - 1
        self._R = ref()
        self._offsets = np.ascontiguousarray(offsets, np.uint32)
        self._edges = _nonempty(edges)
        self.h = self._R.pbbsref_graph_new(self.n, len(edges), self._offsets, self._edges)

    def bfs(self, src: int, which: int = REF_SERIAL) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        rc = self._R.pbbsref_bfs_g(self.h, which, src, out)
        if rc != 0:
            raise RuntimeError("reference BFS failed: %d" % rc)
        return out

    def check(self, src: int, parent: np.ndarray) -> int:
        """The reference checkBFS verdict (0 = ok)."""
        return self._R.pbbsref_check_g(self.h, src, np.ascontiguousarray(parent).view(np.int32))

    def time(self, src: int, which: int, rounds: int, warmup_s: float) -> np.ndarray:
        out = np.zeros(rounds, np.float64)
        self._R.pbbsref_time_bfs(self.h, which, src, rounds, warmup_s, out)
        return out

    def close(self):
        if self.h:
            self._R.pbbsref_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REF_SERIAL_MIS, REF_ND_MIS = 0, 1
_refmis = None


def refmis_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libpbbsmis.so"))


def refmis():
    """The reference's own maximal independent set code (serialMIS, ndMIS,
    MISCheck), compiled from its sources."""
    global _refmis
    if _refmis is None:
        path = os.path.join(HERE, "_ref", "libpbbsmis.so")
        if not os.path.exists(path):
            raise FileNotFoundError("reference MIS library not built: make -C oracle ref")
        R = ctypes.CDLL(path)
        R.pbbsref_mis_graph_new.restype = ctypes.c_void_p
        R.pbbsref_mis_graph_new.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p]
        R.pbbsref_mis_graph_free.restype = None
        R.pbbsref_mis_graph_free.argtypes = [ctypes.c_void_p]
        R.pbbsref_mis_g.restype = ctypes.c_int
        R.pbbsref_mis_g.argtypes = [ctypes.c_void_p, ctypes.c_int, _u8p]
        R.pbbsref_time_mis.restype = ctypes.c_int
        R.pbbsref_time_mis.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _f64p]
        _refmis = R
    return _refmis


class RefMisGraph:
    """graph<uint,uint> held by the reference MIS library."""

    def __init__(self, offsets: np.ndarray, edges: np.ndarray):
        self.n = len(offsets) - 1
        self._R = refmis()
        self._offsets = np.ascontiguousarray(offsets, np.uint32)
        self._edges = _nonempty(edges)
        self.h = self._R.pbbsref_mis_graph_new(self.n, len(edges), self._offsets, self._edges)

    def mis(self, which: int = REF_SERIAL_MIS) -> np.ndarray:
        out = np.empty(self.n, np.uint8)
        rc = self._R.pbbsref_mis_g(self.h, which, out)
        if rc != 0:
            raise RuntimeError("reference MIS failed: %d" % rc)
        return out

    def time(self, which: int, rounds: int, warmup_s: float) -> np.ndarray:
        out = np.zeros(rounds, np.float64)
        self._R.pbbsref_time_mis(self.h, which, rounds, warmup_s, out)
        return out

    def close(self):
        if self.h:
            self._R.pbbsref_mis_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_check_mis(offsets, edges, flags) -> int:
    """The reference's checker (oracle/_ref/MISCheck, bench/MISCheck.C) run on
    files, as the benchmark's harness runs it: 0 = ok."""
    import tempfile

    exe = os.path.join(HERE, "_ref", "MISCheck")
    with tempfile.TemporaryDirectory() as d:
        g, o = os.path.join(d, "g.adj"), os.path.join(d, "flags.seq")
        write_adjacency_graph(g, offsets, edges)
        write_sequence_int(o, np.asarray(flags, np.int32))
        r = subprocess.run([exe, g, o], capture_output=True, text=True, timeout=600)
    return r.returncode


def ref_level_number(parent: np.ndarray) -> np.ndarray:
    n = len(parent)
    out = np.empty(n, np.int32)
    ref().pbbsref_level_number(n, np.ascontiguousarray(parent).view(np.int32), out)
    return out


def ref_num_workers() -> int:
    return ref().pbbsref_num_workers()


# -------------------------------------------------------------- file IO

def write_adjacency_graph(path: str, offsets: np.ndarray, edges: np.ndarray) -> None:
    """AdjacencyGraph text format (docs/fileFormats/graph.md; written as
    graphIO.h:78-105 does): header, n, m, n offsets, m edges, one per line."""
    n = len(offsets) - 1
    with open(path, "w") as f:
        f.write("AdjacencyGraph\n%d\n%d\n" % (n, len(edges)))
        if n:
            f.write("\n".join(map(str, offsets[:-1].tolist())) + "\n")
        if len(edges):
            f.write("\n".join(map(str, edges.tolist())) + "\n")


def ref_read_graph(path: str):
    """(offsets, edges) as the reference's own reader returns them
    (common/graphIO.h:191-215; it aborts the process on a malformed file)."""
    R = ref()
    g = R.pbbsref_read_graph(os.fsencode(path))
    n, m = ctypes.c_uint64(), ctypes.c_uint64()
    R.pbbsref_graph_arrays(g, ctypes.byref(n), ctypes.byref(m), None, None)
    off = np.empty(n.value + 1, np.uint32)
    edg = np.empty(max(1, m.value), np.uint32)
    R.pbbsref_graph_arrays(g, ctypes.byref(n), ctypes.byref(m), off.ctypes.data, edg.ctypes.data)
    R.pbbsref_graph_free(g)
    return off, edg[: m.value]


# The token delimiters of common/IO.h:41-50 (is_space): space, tab, LF, CR,
# NUL (not VT or FF, which bytes.split() would also take).
_DELIMS = re.compile(rb"[ \t\n\r\x00]+")


def parse_adjacency_graph(text: bytes):
    """Restatement of readGraphFromFile (common/graphIO.h:191-215): tokens
    split on the delimiters of common/IO.h:41-50; header, n, m, n offsets, m
    edges; offsets[n] = m.  Raises ValueError where the reference aborts, and
    on tokens that are not unsigned decimal integers below 2^32."""
    toks = [t for t in _DELIMS.split(text) if t]
    if not toks or toks[0] != b"AdjacencyGraph":
        raise ValueError("missing header")
    n, m = int(toks[1]), int(toks[2])
    if len(toks) != n + m + 3:
        raise ValueError("bad input file: length = %d n+m+3 = %d" % (len(toks), n + m + 3))
    vals = []
    for t in toks[3:]:
        if not t.isdigit() or int(t) >= 1 << 32:
            raise ValueError("bad token %r" % t)
        vals.append(int(t))
    off = np.array(vals[:n] + [m], dtype=np.uint32)
    return off, np.array(vals[n:], dtype=np.uint32)


def write_sequence_int(path: str, values) -> None:
    """sequenceInt file as writeIntSeqToFile writes it (common/IO.h:100-150,
    198-203): the header line, then one value per line."""
    with open(path, "w") as f:
        f.write("sequenceInt\n")
        vals = np.asarray(values, dtype=np.int64)
        if len(vals):
            f.write("\n".join(map(str, vals.tolist())) + "\n")


def read_sequence_int(path: str) -> np.ndarray:
    """sequenceInt file (common/sequenceIO.h) -> int32 array."""
    with open(path) as f:
        toks = f.read().split()
    if not toks or toks[0] != "sequenceInt":
        raise ValueError("not a sequenceInt file: %s" % path)
    return np.array([int(t) for t in toks[1:]], dtype=np.int64).astype(np.int32)


def levels_checksum(row) -> int:
    """CPU restatement of the library's level checksum (csrc/checksum.cu):
    the row's bytes as little-endian 64-bit words w_j, the last padded with
    0xFF, summed as mix64(w_j + (j+1) * 0x9E3779B97F4A7C15) mod 2^64 with
    SplitMix64's output function."""
    row = np.ascontiguousarray(row, np.uint8)
    words = (len(row) + 7) // 8
    buf = np.full(words * 8, 0xFF, np.uint8)
    buf[: len(row)] = row
    with np.errstate(over="ignore"):
        x = buf.view("<u8") + (np.arange(1, words + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        x ^= x >> np.uint64(30)
        x *= np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(27)
        x *= np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
        return int(np.sum(x, dtype=np.uint64))


def u8_levels(lv32: np.ndarray) -> np.ndarray:
    """uint32 levels (0xFFFFFFFF unreached) as the uint8 rows of the batched
    path (>= 255 -> 255)."""
    return np.where(lv32 >= 255, 255, lv32).astype(np.uint8)


def gteps(m_reached: int, seconds: float) -> float:
    return (m_reached / 2.0) / seconds / 1e9 if seconds > 0 else math.inf
