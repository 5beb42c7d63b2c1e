"""ctypes declarations of include/pbbs_bfs.h and the in-tree build.

The library is built in-tree (pbbsbench_b200/libpbbsbfs.so) by ``build()``
with nvcc for sm_100a.  Loading fails loudly when it is missing: there is no
CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libpbbsbfs.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC"]
BUILD_DIR = os.path.join(PKG, "_build")

PBG_OK = 0
ERRORS = {1: "PBG_ERR_ARG", 2: "PBG_ERR_CUDA", 3: "PBG_ERR_OOM", 4: "PBG_ERR_TIMEOUT",
          5: "PBG_ERR_OVERFLOW", 6: "PBG_ERR_STATE"}

PARENT_ANY, PARENT_MIN, PARENT_MAX = 0, 1, 2
DIR_AUTO, DIR_TOPDOWN, DIR_BOTTOMUP = 0, 1, 2
GRAPH_SYMMETRIC = 1
GRAPH_DETECT_SYMMETRIC = 2
GEN_RMAT, GEN_TORUS3D, GEN_RANDLOCAL = 1, 2, 3


class PbgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s: %s" % (ERRORS.get(code, str(code)), msg))
        self.code = code


class BfsOpts(ctypes.Structure):
    _fields_ = [("parent_mode", ctypes.c_uint32), ("direction", ctypes.c_uint32),
                ("alpha", ctypes.c_uint32), ("beta", ctypes.c_uint32),
                ("block_threads", ctypes.c_uint32), ("chunk_min_degree", ctypes.c_uint32)]


class BfsStats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_uint32), ("topdown_levels", ctypes.c_uint32),
                ("bottomup_levels", ctypes.c_uint32), ("error", ctypes.c_uint32),
                ("visited", ctypes.c_uint64), ("edges_reached", ctypes.c_uint64),
                ("bottomup_mask", ctypes.c_uint64), ("device_ms", ctypes.c_float), ("init_ms", ctypes.c_float),
                ("kernel_ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class LevelTrace(ctypes.Structure):
    _fields_ = [("level", ctypes.c_uint32), ("bottom_up", ctypes.c_uint32), ("frontier", ctypes.c_uint64),
                ("frontier_degree", ctypes.c_uint64), ("ms", ctypes.c_double)]


TRACE_LEVELS = 256


class BatchJob(ctypes.Structure):
    _fields_ = [("ws", ctypes.c_void_p), ("srcs", ctypes.c_void_p), ("k", ctypes.c_uint32),
                ("d_levels", ctypes.c_void_p)]


class BatchStats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_uint32), ("pull_levels", ctypes.c_uint32), ("push_levels", ctypes.c_uint32),
                ("error", ctypes.c_uint32), ("device_ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


MAX_SOURCES = 256
MAX_JOBS = 128
SERVER_CHECKSUM = 1


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_sources", ctypes.c_uint32),
                ("max_jobs", ctypes.c_uint32), ("streams", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("wide_sources", ctypes.c_uint32), ("wide_max_vertices", ctypes.c_uint32),
                ("max_launch_edges", ctypes.c_uint64)]


class QueryResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("graph", ctypes.c_uint32), ("src", ctypes.c_uint32),
                ("status", ctypes.c_uint32), ("levels", ctypes.c_uint32), ("checksum", ctypes.c_uint64),
                ("t_submit_us", ctypes.c_double), ("t_launch_us", ctypes.c_double), ("t_done_us", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("jobs", ctypes.c_uint64), ("max_inflight", ctypes.c_uint32), ("slots", ctypes.c_uint32),
                ("slot_bytes", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64), ("free_bytes", ctypes.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


TUNE_BATCHED, TUNE_NO_STORE, TUNE_MAX_SOURCES = 1, 2, 16
CHECK_EDGES = 1


class CheckResult(ctypes.Structure):
    _fields_ = [("bad_vertex", ctypes.c_uint32), ("row", ctypes.c_uint32), ("level", ctypes.c_uint32),
                ("min_neighbor_level", ctypes.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class MisStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_uint32), ("error", ctypes.c_uint32), ("in_set", ctypes.c_uint64),
                ("device_ms", ctypes.c_float), ("kernel_ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class TuneReport(ctypes.Structure):
    _fields_ = [("evaluations", ctypes.c_uint32), ("default_ms", ctypes.c_float), ("best_ms", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


MAX_VERTICES = (1 << 31) - 1
SERVER_HBM_RESERVE = 512 << 20
NOALLOC_MAX_VERTICES = 1 << 20
NOALLOC_MAX_EDGES = 1 << 24


class GenParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("logn", ctypes.c_uint32), ("samples", ctypes.c_uint64),
                ("seed", ctypes.c_uint64), ("a", ctypes.c_double), ("b", ctypes.c_double),
                ("c", ctypes.c_double), ("dn", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("degree", ctypes.c_uint32), ("window", ctypes.c_uint32), ("permute", ctypes.c_uint32),
                ("perm_seed", ctypes.c_uint64)]


# (name, restype, argtypes) of every entry point declared in include/*.h.
_P = ctypes.c_void_p
_U32, _U64 = ctypes.c_uint32, ctypes.c_uint64
SIGNATURES = [
    ("pbg_last_error", ctypes.c_char_p, []),
    ("pbg_graph_upload", ctypes.c_int, [_P, _P, _U32, _U64, _U32, ctypes.POINTER(_P)]),
    ("pbg_graph_upload_device", ctypes.c_int, [_P, _P, _U32, _U64, _U32, ctypes.POINTER(_P)]),
    ("pbg_graph_generate", ctypes.c_int, [ctypes.POINTER(GenParams), ctypes.POINTER(_P)]),
    ("pbg_graph_info", ctypes.c_int, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_P),
                                      ctypes.POINTER(_P)]),
    ("pbg_graph_flags", ctypes.c_int, [_P, ctypes.POINTER(_U32)]),
    ("pbg_graph_download", ctypes.c_int, [_P, _P, _P]),
    ("pbg_graph_free", ctypes.c_int, [_P]),
    ("pbg_graph_load_adj", ctypes.c_int, [ctypes.c_char_p, _U32, ctypes.POINTER(_P)]),
    ("pbg_graph_parse_adj", ctypes.c_int, [_P, _U64, _U32, ctypes.POINTER(_P)]),
    ("pbg_graph_write_adj", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("pbg_write_seq_int", ctypes.c_int, [_P, _U64, ctypes.c_char_p]),
    ("pbg_graph_save_bin", ctypes.c_int, [_P, ctypes.c_char_p]),
    ("pbg_graph_load_bin", ctypes.c_int, [ctypes.c_char_p, _U32, ctypes.POINTER(_P)]),
    ("pbg_bfs_opts_default", None, [ctypes.POINTER(BfsOpts)]),
    ("pbg_bfs", ctypes.c_int, [_P, _U32, ctypes.POINTER(BfsOpts), _P, _P, ctypes.POINTER(BfsStats)]),
    ("pbg_bfs_device", ctypes.c_int, [_P, _U32, ctypes.POINTER(BfsOpts), _P, _P, _P]),
    ("pbg_bfs_stats_get", ctypes.c_int, [_P, ctypes.POINTER(BfsStats)]),
    ("pbg_bfs_trace", ctypes.c_int, [_P, ctypes.POINTER(LevelTrace), _U32, ctypes.POINTER(_U32)]),
    ("pbg_bfs_noalloc", ctypes.c_int, [_P, _P, _U32, _U64, _U32, _U32, _U32, _P, _P, _P]),
    ("pbg_msbfs_bytes", ctypes.c_uint64, [_P, ctypes.POINTER(BfsOpts)]),
    ("pbg_levels_checksum", ctypes.c_int, [_P, _U32, _U32, _P, _P]),
    ("pbg_levels32_checksum", ctypes.c_int, [_P, _U32, _P, _P]),
    ("pbg_server_create", ctypes.c_int, [ctypes.POINTER(_P), _U32, ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    ("pbg_server_submit", ctypes.c_int, [_P, _U32, _U32, _P, ctypes.POINTER(_U64)]),
    ("pbg_server_replay", ctypes.c_int, [_P, _P, _P, _P, _U32]),
    ("pbg_server_poll", ctypes.c_int, [_P, ctypes.POINTER(QueryResult), _U32, ctypes.POINTER(_U32), ctypes.c_int]),
    ("pbg_server_drain", ctypes.c_int, [_P, ctypes.c_int]),
    ("pbg_server_stats_get", ctypes.c_int, [_P, ctypes.POINTER(ServerStats)]),
    ("pbg_server_destroy", ctypes.c_int, [_P]),
    ("pbg_msbfs_create", ctypes.c_int, [_P, ctypes.POINTER(BfsOpts), ctypes.POINTER(_P)]),
    ("pbg_msbfs_create_k", ctypes.c_int, [_P, ctypes.POINTER(BfsOpts), _U32, ctypes.POINTER(_P)]),
    ("pbg_msbfs_bytes_k", ctypes.c_uint64, [_P, ctypes.POINTER(BfsOpts), _U32]),
    ("pbg_msbfs_free", ctypes.c_int, [_P]),
    ("pbg_batch_create", ctypes.c_int, [_U32, ctypes.POINTER(_P)]),
    ("pbg_batch_free", ctypes.c_int, [_P]),
    ("pbg_bfs_batch", ctypes.c_int, [_P, ctypes.POINTER(BatchJob), _U32, ctypes.POINTER(BfsOpts), _P]),
    ("pbg_batch_job_stats", ctypes.c_int, [_P, _P, ctypes.POINTER(BatchStats)]),
    ("pbg_bfs_multi", ctypes.c_int, [_P, _P, _U32, ctypes.POINTER(BfsOpts), _P, ctypes.POINTER(BatchStats)]),
    ("pbg_batch_job_trace", ctypes.c_int, [_P, _P, ctypes.POINTER(LevelTrace), _U32, ctypes.POINTER(_U32)]),
    ("pbg_bfs_multi_trace", ctypes.c_int, [_P, ctypes.POINTER(LevelTrace), _U32, ctypes.POINTER(_U32)]),
    ("pbg_mis", ctypes.c_int, [_P, _P, ctypes.POINTER(MisStats)]),
    ("pbg_mis_device", ctypes.c_int, [_P, _P, _P]),
    ("pbg_mis_stats_get", ctypes.c_int, [_P, ctypes.POINTER(MisStats)]),
    ("pbg_mis_trace", ctypes.c_int, [_P, ctypes.POINTER(LevelTrace), _U32, ctypes.POINTER(_U32)]),
    ("pbg_autotune", ctypes.c_int, [_P, _P, _U32, _U32, ctypes.POINTER(BfsOpts), ctypes.POINTER(TuneReport)]),
    ("pbg_autotune_clear", ctypes.c_int, [_P]),
    ("pbg_bfs_check", ctypes.c_int, [_P, _U32, _P, _U32, ctypes.POINTER(CheckResult)]),
    ("pbg_levels_check", ctypes.c_int, [_P, _P, _U32, _P, ctypes.POINTER(CheckResult)]),
]

_lib = None


def sources():
    return sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))


def build(verbose: bool = False, jobs: int | None = None) -> str:
    """Compile every CUDA source into pbbsbench_b200/libpbbsbfs.so for sm_100a.

    Each source is compiled to an object under pbbsbench_b200/_build/ in
    parallel (only when it, a header of csrc/ or include/, or the flags are
    newer than its object), then the objects are linked into the library."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = glob.glob(os.path.join(PKG, "csrc", "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    newest_dep = max([os.path.getmtime(h) for h in headers] + [os.path.getmtime(__file__)])
    jobs_to_run, objs = [], []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(newest_dep, os.path.getmtime(src)):
            jobs_to_run.append(["nvcc"] + NVCC_FLAGS + ["-I" + INCLUDE, "-c", "-o", obj, src])

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=jobs or min(len(jobs_to_run) or 1, os.cpu_count() or 4)) as ex:
        for cmd, res in zip(jobs_to_run, ex.map(run, jobs_to_run)):
            if res.returncode != 0:
                raise RuntimeError("nvcc failed: %s\n%s%s" % (" ".join(cmd), res.stdout, res.stderr))
    if jobs_to_run or not os.path.exists(LIB_PATH):
        link = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB_PATH] + objs
        if verbose:
            print(" ".join(link))
        subprocess.run(link, check=True)
    return LIB_PATH


def lib():
    """The loaded C-ABI library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("pbbsbench_b200: %s is missing; run pbbsbench_b200.build() "
                              "(nvcc, sm_100a). There is no CPU fallback." % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PBG_OK:
        raise PbgError(rc, lib().pbg_last_error().decode(errors="replace"))


def default_opts(**kw) -> BfsOpts:
    o = BfsOpts()
    lib().pbg_bfs_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        if v is not None:
            setattr(o, k, v)
    return o
