"""pbbsbench_b200 -- PBBS breadthFirstSearch on one B200 (sm_100a).

Host-side mirror of the reference's plugin interface
(benchmarks/breadthFirstSearch/bench/BFS.h:4-11):

* ``Graph`` mirrors ``graph<int,uint>`` (common/graph.h:104-152): CSR
  ``offsets`` (n+1 uint32, offsets[n] = m) and ``edges`` (m uint32).
* ``BFS(start, G, verbose=False)`` returns the parent array of BFS.h:9-10
  (int32, -1 unvisited, parent[start] = start), exactly what the reference
  ``BFS`` returns.  The graph is uploaded to HBM once per Graph object and
  stays resident, as the C++ drop-in (dropin/gpuBFS/BFS.C) does.
* ``DeviceGraph`` is the resident handle (pbg_graph) with the full option set
  of the C ABI (parent rule, direction policy, device buffers, statistics).

All compute runs in libpbbsbfs.so (hand-written CUDA for sm_100a).  Nothing
here computes a BFS on the CPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _capi
from ._capi import (DIR_AUTO, DIR_BOTTOMUP, DIR_TOPDOWN, PARENT_ANY, PARENT_MAX, PARENT_MIN, BfsStats,
                    PbgError, build, check, default_opts, lib)

__all__ = ["Graph", "DeviceGraph", "MultiWorkspace", "Batch", "Server", "BFS", "levels_checksum_device",
           "levels32_checksum_device", "build", "lib", "PbgError", "rmat_graph", "torus3d_graph",
           "randlocal_graph", "PARENT_ANY", "PARENT_MIN", "PARENT_MAX", "DIR_AUTO", "DIR_TOPDOWN",
           "DIR_BOTTOMUP", "NONE"]

NONE = 0xFFFFFFFF


def _ptr(a) -> ctypes.c_void_p:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return ctypes.c_void_p(0)
    if isinstance(a, np.ndarray):
        return ctypes.c_void_p(a.ctypes.data)
    return ctypes.c_void_p(int(a.data_ptr()))


class Graph:
    """graph<int,uint> on the host: CSR offsets[n+1], edges[m] (uint32)."""

    def __init__(self, offsets, edges, symmetric: bool = True):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.edges = np.ascontiguousarray(edges, dtype=np.uint32)
        self.n = len(self.offsets) - 1
        self.m = len(self.edges)
        self.symmetric = symmetric
        self._dev = None

    def numVertices(self) -> int:  # noqa: N802 -- reference name (graph.h:117)
        return self.n

    def numEdges(self) -> int:  # noqa: N802 -- reference name (graph.h:118)
        return self.m

    def device(self) -> "DeviceGraph":
        """The resident device copy (uploaded on first use)."""
        if self._dev is None:
            self._dev = DeviceGraph.upload(self.offsets, self.edges, self.symmetric)
        return self._dev


class DeviceGraph:
    """A CSR graph resident in HBM (pbg_graph handle)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        n = ctypes.c_uint32()
        m = ctypes.c_uint64()
        po = ctypes.c_void_p()
        pe = ctypes.c_void_p()
        check(lib().pbg_graph_info(self._h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(po), ctypes.byref(pe)))
        self.n, self.m = n.value, m.value
        self.d_offsets, self.d_edges = po.value, pe.value

    @classmethod
    def upload(cls, offsets, edges, symmetric: bool = True) -> "DeviceGraph":
        h = ctypes.c_void_p()
        flags = _capi.GRAPH_SYMMETRIC if symmetric else 0
        if isinstance(offsets, np.ndarray):
            offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
            edges = np.ascontiguousarray(edges, dtype=np.uint32)
            if len(edges) == 0:
                edges = np.zeros(1, np.uint32)[:0]
            check(lib().pbg_graph_upload(_ptr(offsets), _ptr(edges), len(offsets) - 1, int(offsets[-1]), flags,
                                         ctypes.byref(h)))
        else:  # torch tensors on the device
            check(lib().pbg_graph_upload_device(_ptr(offsets), _ptr(edges), offsets.numel() - 1, edges.numel(),
                                                flags, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, params: _capi.GenParams) -> "DeviceGraph":
        h = ctypes.c_void_p()
        check(lib().pbg_graph_generate(ctypes.byref(params), ctypes.byref(h)))
        return cls(h)

    @staticmethod
    def _file_flags(symmetric) -> int:
        if symmetric is None:
            return _capi.GRAPH_DETECT_SYMMETRIC
        return _capi.GRAPH_SYMMETRIC if symmetric else 0

    @classmethod
    def load_adjacency(cls, path: str, symmetric: bool | None = None) -> "DeviceGraph":
        """A PBBS AdjacencyGraph text file (readGraphFromFile, common/graphIO.h:191-215),
        parsed on the device.  symmetric None: decided on the device."""
        h = ctypes.c_void_p()
        check(lib().pbg_graph_load_adj(os.fsencode(path), cls._file_flags(symmetric), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def parse_adjacency(cls, text: bytes, symmetric: bool | None = None) -> "DeviceGraph":
        """The same from AdjacencyGraph text in host memory."""
        buf = np.frombuffer(text, dtype=np.uint8) if len(text) else np.zeros(1, np.uint8)
        h = ctypes.c_void_p()
        check(lib().pbg_graph_parse_adj(_ptr(buf), len(text), cls._file_flags(symmetric), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load_binary(cls, path: str, symmetric: bool | None = False) -> "DeviceGraph":
        """A binary CSR image written by save_binary.  symmetric False keeps the
        file's flag; True forces it; None decides on the device."""
        h = ctypes.c_void_p()
        flags = 0 if symmetric is False else cls._file_flags(symmetric)
        check(lib().pbg_graph_load_bin(os.fsencode(path), flags, ctypes.byref(h)))
        return cls(h)

    def save_binary(self, path: str) -> None:
        check(lib().pbg_graph_save_bin(self._h, os.fsencode(path)))

    def write_adjacency(self, path: str) -> None:
        """AdjacencyGraph text (writeGraphToFile, common/graphIO.h:79-104), formatted on the device."""
        check(lib().pbg_graph_write_adj(self._h, os.fsencode(path)))

    def download(self):
        """(offsets, edges) back on the host."""
        off = np.empty(self.n + 1, np.uint32)
        edg = np.empty(max(1, self.m), np.uint32)
        check(lib().pbg_graph_download(self._h, _ptr(off), _ptr(edg)))
        return off, edg[: self.m]

    def download_offsets(self) -> np.ndarray:
        off = np.empty(self.n + 1, np.uint32)
        check(lib().pbg_graph_download(self._h, _ptr(off), ctypes.c_void_p(0)))
        return off

    def bfs(self, src: int, parent_mode: int = PARENT_ANY, direction: int = DIR_AUTO, levels: bool = False,
            parents: bool = True, **tune):
        """Host-buffer BFS (pbg_bfs).  Returns (parent int32 | None,
        level uint32 | None, stats dict)."""
        o = self._opts(False, parent_mode, direction, tune)
        par = np.empty(self.n, np.int32) if parents else None
        lv = np.empty(self.n, np.uint32) if levels else None
        st = BfsStats()
        check(lib().pbg_bfs(self._h, src, ctypes.byref(o), _ptr(par), _ptr(lv), ctypes.byref(st)))
        return par, lv, st.as_dict()

    def bfs_device(self, src: int, d_parent, d_level=None, stream=None, parent_mode: int = PARENT_ANY,
                   direction: int = DIR_AUTO, **tune) -> None:
        """Device-buffer BFS (pbg_bfs_device), asynchronous on `stream` (a raw
        cudaStream_t as int; None or 0 is CUDA's default stream)."""
        o = self._opts(False, parent_mode, direction, tune)
        check(lib().pbg_bfs_device(self._h, src, ctypes.byref(o), _ptr(d_parent), _ptr(d_level),
                                   ctypes.c_void_p(stream or 0)))

    def _opts(self, multi: bool, parent_mode: int, direction: int, tune: dict):
        """Options of a call: the graph's tuned ones (autotune) under the
        call's parent mode and direction, unless the call names any."""
        tuned = getattr(self, "_tuned_multi" if multi else "_tuned", None)
        if tuned and not tune:
            tune = {k: v for k, v in tuned.items() if k not in ("parent_mode", "direction")}
        return default_opts(parent_mode=parent_mode, direction=direction, **tune)

    def last_stats(self) -> dict:
        st = BfsStats()
        check(lib().pbg_bfs_stats_get(self._h, ctypes.byref(st)))
        return st.as_dict()

    def bfs_multi(self, srcs, parent_mode: int = PARENT_ANY, direction: int = DIR_AUTO, **tune):
        """Up to 64 sources in one batched search (pbg_bfs_multi).  Returns
        (levels uint8 [k][n], 255 = unreached; stats dict)."""
        srcs = np.ascontiguousarray(srcs, dtype=np.uint32)
        k = len(srcs)
        out = np.empty((k, self.n), np.uint8)
        o = self._opts(True, parent_mode, direction, tune)
        st = _capi.BatchStats()
        check(lib().pbg_bfs_multi(self._h, _ptr(srcs), k, ctypes.byref(o), _ptr(out), ctypes.byref(st)))
        return out, st.as_dict()

    def trace(self) -> list:
        """Per-level trace of the last BFS: direction, frontier size and
        out-degree, device ms."""
        return _read_trace(lib().pbg_bfs_trace, self._h)

    def autotune(self, srcs, batched: bool = False, store: bool = True, parent_mode: int = PARENT_ANY,
                 direction: int = DIR_AUTO):
        """Picks this graph's options by timing the sample sources
        (pbg_autotune): the single-source search's block size, chunk degree
        and switch, or with batched=True the batched search's switch.  Stored
        on the graph unless store=False; calls without options then use them.
        Returns (options dict, report dict)."""
        srcs = np.ascontiguousarray(srcs, dtype=np.uint32)
        o = default_opts(parent_mode=parent_mode, direction=direction)
        rep = _capi.TuneReport()
        flags = (_capi.TUNE_BATCHED if batched else 0) | (0 if store else _capi.TUNE_NO_STORE)
        check(lib().pbg_autotune(self._h, _ptr(srcs), len(srcs), flags, ctypes.byref(o), ctypes.byref(rep)))
        opts = {f: getattr(o, f) for f, _ in o._fields_}
        if store:
            setattr(self, "_tuned_multi" if batched else "_tuned", opts)
        return opts, rep.as_dict()

    def check(self, src: int, d_parent, edges: bool = True) -> dict:
        """The reference's BFS check on the device (pbg_bfs_check) of a
        device parent array (torch tensor, int32/uint32, -1 = unreached);
        bad_vertex = NONE when it is a valid BFS tree from src."""
        res = _capi.CheckResult()
        check(lib().pbg_bfs_check(self._h, src, _ptr(d_parent), _capi.CHECK_EDGES if edges else 0,
                                  ctypes.byref(res)))
        return res.as_dict()

    def levels_check(self, srcs, d_levels) -> dict:
        """The level predicate on uint8 level rows in device memory
        (pbg_levels_check): row i from srcs[i], 255 = unreached."""
        srcs = np.ascontiguousarray(srcs, dtype=np.uint32)
        res = _capi.CheckResult()
        check(lib().pbg_levels_check(self._h, _ptr(srcs), len(srcs), _ptr(d_levels), ctypes.byref(res)))
        return res.as_dict()

    def clear_tuning(self) -> None:
        check(lib().pbg_autotune_clear(self._h))
        self._tuned = self._tuned_multi = None

    def mis(self) -> tuple:
        """Maximal independent set (pbg_mis): the set serialMIS returns
        (vertices in id order).  Returns (uint8 flags, 1 in the set / 2 not;
        stats dict)."""
        flags = np.empty(self.n, np.uint8)
        st = _capi.MisStats()
        check(lib().pbg_mis(self._h, _ptr(flags), ctypes.byref(st)))
        return flags, st.as_dict()

    def mis_device(self, d_flags, stream=None) -> None:
        """pbg_mis_device into a device uint8 buffer of n entries, on `stream`."""
        check(lib().pbg_mis_device(self._h, _ptr(d_flags), ctypes.c_void_p(stream or 0)))

    def mis_stats(self) -> dict:
        st = _capi.MisStats()
        check(lib().pbg_mis_stats_get(self._h, ctypes.byref(st)))
        return st.as_dict()

    def mis_trace(self) -> list:
        """Per-round trace of the last MIS: vertices walked and device time
        of each round."""
        return _read_trace(lib().pbg_mis_trace, self._h)

    def trace_multi(self) -> list:
        """Per-level trace of the last bfs_multi (first 64 levels)."""
        return _read_trace(lib().pbg_bfs_multi_trace, self._h)

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            lib().pbg_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _read_trace(fn, *handles) -> list:
    buf = (_capi.LevelTrace * _capi.TRACE_LEVELS)()
    cnt = ctypes.c_uint32()
    check(fn(*handles, buf, _capi.TRACE_LEVELS, ctypes.byref(cnt)))
    dirs = {0: "top-down", 1: "bottom-up", 2: "top-down-dense"}
    return [{"level": t.level, "dir": dirs.get(t.bottom_up, str(t.bottom_up)), "frontier": t.frontier,
             "frontier_degree": t.frontier_degree, "ms": t.ms} for t in buf[: cnt.value]]


class MultiWorkspace:
    """Device state of one batched job (up to 64 sources) on a DeviceGraph."""

    def __init__(self, g: DeviceGraph, max_sources: int = 64, **tune):
        self.g = g
        h = ctypes.c_void_p()
        check(lib().pbg_msbfs_create_k(g.handle, ctypes.byref(default_opts(**tune)), max_sources, ctypes.byref(h)))
        self._h = h

    @staticmethod
    def bytes_needed(g: DeviceGraph, max_sources: int = 64, **tune) -> int:
        return int(lib().pbg_msbfs_bytes_k(g.handle, ctypes.byref(default_opts(**tune)), max_sources))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().pbg_msbfs_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Fused launches of many batched jobs (graphs of any sizes) at once."""

    def __init__(self, max_jobs: int = 8):
        h = ctypes.c_void_p()
        check(lib().pbg_batch_create(max_jobs, ctypes.byref(h)))
        self._h = h
        self._keep = None

    def launch(self, jobs, stream=None, **tune):
        """jobs: list of (MultiWorkspace, sources array, device uint8 tensor of
        k*n bytes).  Asynchronous on `stream` (raw cudaStream_t, None = 0)."""
        arr = (_capi.BatchJob * len(jobs))()
        keep = []
        for i, (ws, srcs, dlev) in enumerate(jobs):
            srcs = np.ascontiguousarray(srcs, dtype=np.uint32)
            keep.append(srcs)
            arr[i].ws = ws.handle
            arr[i].srcs = srcs.ctypes.data
            arr[i].k = len(srcs)
            arr[i].d_levels = int(dlev.data_ptr())
        o = default_opts(**tune)
        check(lib().pbg_bfs_batch(self._h, arr, len(jobs), ctypes.byref(o), ctypes.c_void_p(stream or 0)))
        self._keep = keep

    def job_stats(self, ws: MultiWorkspace) -> dict:
        st = _capi.BatchStats()
        check(lib().pbg_batch_job_stats(self._h, ws.handle, ctypes.byref(st)))
        return st.as_dict()

    def job_trace(self, ws: MultiWorkspace) -> list:
        """Per-level trace of ws's job in the last launch (first 64 levels)."""
        return _read_trace(lib().pbg_batch_job_trace, self._h, ws.handle)

    def close(self):
        if self._h:
            lib().pbg_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def levels_checksum_device(d_levels, rows: int, n: int, stream=None):
    """pbg_levels_checksum of `rows` uint8 rows of n bytes in a device tensor;
    returns a numpy uint64 array."""
    import torch

    out = torch.empty(max(1, rows), dtype=torch.int64, device=d_levels.device)
    check(lib().pbg_levels_checksum(_ptr(d_levels), rows, n, _ptr(out), ctypes.c_void_p(stream or 0)))
    torch.cuda.synchronize(d_levels.device)
    return out.cpu().numpy().view(np.uint64)[:rows]


def levels32_checksum_device(d_levels, n: int, stream=None) -> int:
    """pbg_levels32_checksum of a uint32 level array in a device tensor."""
    import torch

    out = torch.empty(1, dtype=torch.int64, device=d_levels.device)
    check(lib().pbg_levels32_checksum(_ptr(d_levels), n, _ptr(out), ctypes.c_void_p(stream or 0)))
    torch.cuda.synchronize(d_levels.device)
    return int(out.cpu().numpy().view(np.uint64)[0])


class Server:
    """Continuous-batching BFS service over resident graphs (pbg_server_*)."""

    def __init__(self, graphs, hbm_budget_bytes: int, max_sources: int = 64, max_jobs: int = 16, streams: int = 4,
                 checksum: bool = True, wide_sources: int = 0, wide_max_vertices: int = 0,
                 max_launch_edges: int = 0):
        self.graphs = list(graphs)
        arr = (ctypes.c_void_p * len(self.graphs))(*[g.handle.value for g in self.graphs])
        cfg = _capi.ServerConfig(hbm_budget_bytes=hbm_budget_bytes, max_sources=max_sources, max_jobs=max_jobs,
                                 streams=streams, flags=_capi.SERVER_CHECKSUM if checksum else 0,
                                 wide_sources=wide_sources, wide_max_vertices=wide_max_vertices,
                                 max_launch_edges=max_launch_edges)
        h = ctypes.c_void_p()
        check(lib().pbg_server_create(arr, len(self.graphs), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def submit(self, graph: int, src: int, levels_out: np.ndarray | None = None) -> int:
        qid = ctypes.c_uint64()
        check(lib().pbg_server_submit(self._h, graph, src, _ptr(levels_out), ctypes.byref(qid)))
        return qid.value

    def replay(self, graph, src, arrival_us) -> None:
        g = np.ascontiguousarray(graph, np.uint32)
        s = np.ascontiguousarray(src, np.uint32)
        t = np.ascontiguousarray(arrival_us, np.float64)
        check(lib().pbg_server_replay(self._h, _ptr(g), _ptr(s), _ptr(t), len(g)))

    def poll(self, cap: int = 4096, wait_ms: int = 0) -> list:
        buf = (_capi.QueryResult * cap)()
        cnt = ctypes.c_uint32()
        check(lib().pbg_server_poll(self._h, buf, cap, ctypes.byref(cnt), wait_ms))
        return [{f: getattr(r, f) for f, _ in r._fields_} for r in buf[: cnt.value]]

    def drain(self, timeout_ms: int = 600000) -> None:
        check(lib().pbg_server_drain(self._h, timeout_ms))

    def stats(self) -> dict:
        st = _capi.ServerStats()
        check(lib().pbg_server_stats_get(self._h, ctypes.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if self._h:
            lib().pbg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def BFS(start: int, G, verbose: bool = False) -> np.ndarray:  # noqa: N802 -- reference name (BFS.h:11)
    """parlay::sequence<vertexId> BFS(vertexId start, const Graph& G, bool verbose).

    Direction-optimizing BFS with first-claimer parents, the semantics of
    backForwardBFS (benchmarks/breadthFirstSearch/backForwardBFS/BFS.C:38-61).
    Returns int32 parents: -1 unvisited, parent[start] = start."""
    dev = G.device() if isinstance(G, Graph) else G
    par, _, st = dev.bfs(int(start))
    if verbose:
        print("BFS: levels = %d (top-down %d, bottom-up %d), visited = %d, device %.3f ms"
              % (st["levels"], st["topdown_levels"], st["bottomup_levels"], st["visited"], st["device_ms"]))
    return par


def maximalIndependentSet(G) -> np.ndarray:  # noqa: N802 -- reference name (MIS.h:8)
    """parlay::sequence<char> maximalIndependentSet(Graph const& G).

    The maximal independent set of benchmarks/maximalIndependentSet,
    computed on the device; the flags are the ones serialMIS returns
    (serialMIS/MIS.C:33-47): 1 in the set, 2 not."""
    dev = G.device() if isinstance(G, Graph) else G
    flags, _ = dev.mis()
    return flags


def write_int_sequence(path: str, values) -> None:
    """A sequenceInt file (writeIntSeqToFile, common/IO.h:198-203), formatted on the device:
    the parent output of the BFS driver."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    buf = v if len(v) else np.zeros(1, np.int32)
    check(lib().pbg_write_seq_int(_ptr(buf), len(v), os.fsencode(path)))


def rmat_graph(logn: int, samples: int, seed: int, a: float, b: float, c: float) -> DeviceGraph:
    """Symmetric rMat graph built on the device (rMatGraph.C:33-79)."""
    p = _capi.GenParams(kind=_capi.GEN_RMAT, logn=logn, samples=samples, seed=seed, a=a, b=b, c=c)
    return DeviceGraph.generate(p)


def torus3d_graph(dn: int, perm_seed: int | None = None) -> DeviceGraph:
    """Symmetric 3-D torus (gridGraph.C:53-72), optionally randomly relabelled."""
    p = _capi.GenParams(kind=_capi.GEN_TORUS3D, dn=dn, permute=0 if perm_seed is None else 1,
                        perm_seed=perm_seed or 0)
    return DeviceGraph.generate(p)


def randlocal_graph(n: int, degree: int, window: int, seed: int) -> DeviceGraph:
    """Symmetric random-local graph: `degree` out-edges per vertex at offsets
    uniform in [-window, window] (mod n)."""
    p = _capi.GenParams(kind=_capi.GEN_RANDLOCAL, n=n, degree=degree, window=window, seed=seed)
    return DeviceGraph.generate(p)
