"""Argument checks of the C ABI, without a GPU.

The reference's BFS plugin (bench/BFS.h:11) has no error path: bad input
abort()s in its reader (common/graphIO.h:191-215).  The C ABI instead returns
PBG_ERR_ARG and leaves a message for the calling thread.  Every case below
returns at an argument check before the CUDA runtime is touched, so this file
runs on a machine without a GPU.  Where a device pointer must be non-NULL to
reach the check under test, a fake address stands in for it; each such call
returns before the address is used.  The last test runs the drop-in driver
on a machine without a GPU, where its first CUDA call fails, to show that
the product path fails loudly instead of falling back to the CPU.
"""
import ctypes
import os
import struct
import subprocess
import threading

import pytest

import pbbsbench_b200 as pb
from pbbsbench_b200 import _capi

ERR_ARG = 1
FAKE = ctypes.c_void_p(0x10000)  # never dereferenced: each call fails its checks first


def _err(rc, fragment):
    L = pb.lib()
    assert rc == ERR_ARG, (rc, L.pbg_last_error())
    msg = L.pbg_last_error().decode()
    assert fragment in msg, msg


def test_noalloc_limits_are_checked_before_any_device_call():
    L = pb.lib()
    N, M = _capi.NOALLOC_MAX_VERTICES, _capi.NOALLOC_MAX_EDGES
    f = L.pbg_bfs_noalloc
    _err(f(None, FAKE, 4, 4, 1, 0, 0, FAKE, None, None), "NULL argument")
    _err(f(FAKE, None, 4, 4, 1, 0, 0, FAKE, None, None), "NULL argument")
    _err(f(FAKE, FAKE, 4, 4, 1, 0, 0, None, None, None), "NULL argument")
    _err(f(FAKE, FAKE, 0, 0, 1, 0, 0, FAKE, None, None), "n must be in")
    _err(f(FAKE, FAKE, N + 1, 4, 1, 0, 0, FAKE, None, None), "n must be in")
    _err(f(FAKE, FAKE, N, M + 1, 1, 0, 0, FAKE, None, None), "m exceeds")
    _err(f(FAKE, FAKE, 4, 4, 1, 4, 0, FAKE, None, None), "source vertex out of range")
    _err(f(FAKE, FAKE, 4, 4, 1, 0, 3, FAKE, None, None), "unknown parent_mode")
    _err(f(FAKE, FAKE, 4, 4, 2, 0, 0, FAKE, None, None), "flags must be 0 or PBG_GRAPH_SYMMETRIC")


def test_graph_handles_reject_bad_shapes():
    L = pb.lib()
    h = ctypes.c_void_p()
    off = (ctypes.c_uint32 * 2)(0, 0)
    _err(L.pbg_graph_upload(off, None, 1, 3, 0, ctypes.byref(h)), "offsets/edges is NULL")
    _err(L.pbg_graph_upload(off, None, 0, 0, 0, ctypes.byref(h)), "graph has no vertices")
    _err(L.pbg_graph_upload(off, FAKE, 1, 1 << 32, 0, ctypes.byref(h)), "m must fit in 32 bits")
    _err(L.pbg_graph_upload(off, None, 1, 0, 0, None), "out is NULL")
    _err(L.pbg_graph_upload_device(FAKE, None, 1, 0, 0, None), "out is NULL")
    _err(L.pbg_graph_upload_device(None, None, 1, 0, 0, ctypes.byref(h)), "offsets/edges is NULL")
    _err(L.pbg_graph_generate(None, ctypes.byref(h)), "NULL argument")
    assert not h.value


def test_vertex_count_is_limited_to_int_ids(tmp_path):
    """The reference's vertex ids are int (bench/BFS.h:5): every call that
    creates a graph handle refuses n >= 2^31 before it touches the device."""
    L = pb.lib()
    h = ctypes.c_void_p()
    big = _capi.MAX_VERTICES + 1
    _err(L.pbg_graph_upload(FAKE, FAKE, big, 4, 0, ctypes.byref(h)), "n must be below 2^31")
    _err(L.pbg_graph_upload(FAKE, FAKE, 0xFFFFFFFF, 4, 0, ctypes.byref(h)), "n must be below 2^31")
    _err(L.pbg_graph_upload_device(FAKE, FAKE, big, 4, 0, ctypes.byref(h)), "n must be below 2^31")
    p = _capi.GenParams(kind=_capi.GEN_RMAT, logn=31, samples=4, a=0.5, b=0.1, c=0.1)
    _err(L.pbg_graph_generate(ctypes.byref(p), ctypes.byref(h)), "logn must be in [1, 30]")
    p = _capi.GenParams(kind=_capi.GEN_TORUS3D, dn=1291)  # 1291^3 > 2^31 - 1 >= 1290^3
    _err(L.pbg_graph_generate(ctypes.byref(p), ctypes.byref(h)), "n must be below 2^31")
    p = _capi.GenParams(kind=_capi.GEN_RANDLOCAL, n=big, degree=1, window=1)
    _err(L.pbg_graph_generate(ctypes.byref(p), ctypes.byref(h)), "n must be below 2^31")
    text = b"AdjacencyGraph\n2147483648\n0\n"
    buf = ctypes.create_string_buffer(text, len(text))
    _err(L.pbg_graph_parse_adj(buf, len(text), 0, ctypes.byref(h)), "n must be in [1, 2^31)")
    binf = tmp_path / "big.bin"
    binf.write_bytes(b"PBGCSR01" + struct.pack("<QQII", big, 0, 0, 0))
    _err(L.pbg_graph_load_bin(str(binf).encode(), 0, ctypes.byref(h)), "bad binary CSR header")
    assert not h.value


def test_handles_that_are_null_report():
    L = pb.lib()
    cases = [
        (L.pbg_bfs, (None, 0, None, None, None, None), "graph is NULL"),
        (L.pbg_bfs_device, (None, 0, None, FAKE, None, None), "graph is NULL"),
        (L.pbg_bfs_device, (FAKE, 0, None, None, None, None), "d_parent is NULL"),
        (L.pbg_bfs_check, (None, 0, FAKE, 0, None), "NULL argument"),
        (L.pbg_autotune, (None, FAKE, 1, 0, None, None), "NULL argument"),
        (L.pbg_autotune_clear, (None,), "graph is NULL"),
        (L.pbg_msbfs_create_k, (None, None, 64, ctypes.byref(ctypes.c_void_p())), "NULL argument"),
        (L.pbg_levels_checksum, (FAKE, 1, 8, None, None), "NULL argument"),
        (L.pbg_levels32_checksum, (None, 8, FAKE, None), "NULL argument"),
        (L.pbg_server_submit, (None, 0, 0, None, None), "server is NULL"),
        (L.pbg_server_drain, (None, 0), "server is NULL"),
    ]
    for fn, args, frag in cases:
        _err(fn(*args), frag)


def test_counts_out_of_range_report():
    L = pb.lib()
    out = ctypes.c_void_p()
    _err(L.pbg_msbfs_create_k(FAKE, None, 0, ctypes.byref(out)), "max_sources must be in [1, 256]")
    _err(L.pbg_msbfs_create_k(FAKE, None, _capi.MAX_SOURCES + 1, ctypes.byref(out)),
         "max_sources must be in [1, 256]")
    _err(L.pbg_batch_create(0, ctypes.byref(out)), "max_jobs must be in [1, 128]")
    _err(L.pbg_batch_create(_capi.MAX_JOBS + 1, ctypes.byref(out)), "max_jobs must be in [1, 128]")
    _err(L.pbg_levels_checksum(FAKE, 65536, 8, FAKE, None), "at most 65535 rows")
    src = (ctypes.c_uint32 * 1)(0)
    _err(L.pbg_autotune(FAKE, src, 0, 0, None, None), "tuning takes 1..16 sources")
    _err(L.pbg_autotune(FAKE, src, 17, 0, None, None), "tuning takes 1..16 sources")
    _err(L.pbg_autotune(FAKE, src, 0, _capi.TUNE_BATCHED, None, None), "batched tuning takes 1..256 sources")
    _err(L.pbg_autotune(FAKE, src, _capi.MAX_SOURCES + 1, _capi.TUNE_BATCHED, None, None),
         "batched tuning takes 1..256 sources")
    _err(L.pbg_autotune(FAKE, src, 1, 4, None, None), "unknown tuning flags")
    assert not out.value


def test_server_config_limits():
    L = pb.lib()
    graphs = (ctypes.c_void_p * 1)(FAKE.value)
    out = ctypes.c_void_p()

    def cfg(**kw):
        c = _capi.ServerConfig(hbm_budget_bytes=1 << 30, max_sources=64, max_jobs=16, streams=4)
        for k, v in kw.items():
            setattr(c, k, v)
        return c

    _err(L.pbg_server_create(graphs, 0, ctypes.byref(cfg()), ctypes.byref(out)), "no graphs")
    _err(L.pbg_server_create(graphs, 1, None, ctypes.byref(out)), "no graphs")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(max_sources=0)), ctypes.byref(out)), "max_sources in")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(max_sources=257)), ctypes.byref(out)), "max_sources in")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(wide_sources=257)), ctypes.byref(out)), "wide_sources")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(max_jobs=0)), ctypes.byref(out)), "max_jobs in")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(max_jobs=129)), ctypes.byref(out)), "max_jobs in")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(streams=0)), ctypes.byref(out)), "streams in")
    _err(L.pbg_server_create(graphs, 1, ctypes.byref(cfg(streams=17)), ctypes.byref(out)), "streams in")
    assert not out.value


# Header-level faults of an AdjacencyGraph text (the header word and the two
# counts, common/graphIO.h:197-201) are found on the host before the body is
# staged to the device.
HEADER_BAD = [
    (b"", "no AdjacencyGraph header"),
    (b" \n\t ", "no AdjacencyGraph header"),
    (b"AdjacencyGrap\n1\n0\n0\n", "missing header AdjacencyGraph"),
    (b"WeightedAdjacencyGraph\n1\n0\n0\n", "missing header AdjacencyGraph"),
    (b"AdjacencyGraph\nx\n0\n", "header value 1 is not a count"),
    (b"AdjacencyGraph\n2\n-1\n", "header value 2 is not a count"),
    (b"AdjacencyGraph\n99999999999999999999\n0\n", "header value 1 is not a count"),
    (b"AdjacencyGraph\n5\n", "the header has no value 2"),
    (b"AdjacencyGraph", "the header has no value 1"),
]


@pytest.mark.parametrize("text,frag", HEADER_BAD)
def test_text_header_faults_from_memory(text, frag):
    L = pb.lib()
    h = ctypes.c_void_p()
    buf = ctypes.create_string_buffer(text, len(text))
    _err(L.pbg_graph_parse_adj(buf, len(text), 0, ctypes.byref(h)), frag)
    assert not h.value


def test_files_that_cannot_be_read(tmp_path):
    L = pb.lib()
    h = ctypes.c_void_p()
    missing = str(tmp_path / "absent.adj").encode()
    _err(L.pbg_graph_load_adj(missing, 0, ctypes.byref(h)), "unable to open file")
    _err(L.pbg_graph_load_adj(None, 0, ctypes.byref(h)), "NULL argument")
    _err(L.pbg_graph_load_bin(missing, 0, ctypes.byref(h)), "unable to open file")
    _err(L.pbg_write_seq_int(None, 3, str(tmp_path / "s").encode()), "NULL argument")
    _err(L.pbg_write_seq_int(FAKE, 3, str(tmp_path / "no" / "dir" / "s").encode()), "unable to open file")

    short = tmp_path / "short.bin"
    short.write_bytes(b"PBGC")
    _err(L.pbg_graph_load_bin(str(short).encode(), 0, ctypes.byref(h)), "bad magic")
    wrong = tmp_path / "wrong.bin"
    wrong.write_bytes(b"NOTACSR!" + struct.pack("<QQII", 1, 0, 0, 0) + b"\0" * 8)
    _err(L.pbg_graph_load_bin(str(wrong).encode(), 0, ctypes.byref(h)), "bad magic")
    empty = tmp_path / "empty.bin"
    empty.write_bytes(b"PBGCSR01" + struct.pack("<QQII", 0, 0, 0, 0))
    _err(L.pbg_graph_load_bin(str(empty).encode(), 0, ctypes.byref(h)), "bad binary CSR header")
    sized = tmp_path / "sized.bin"
    # n = 2, m = 1 needs 3 offsets and 1 edge after the header; one id is missing
    sized.write_bytes(b"PBGCSR01" + struct.pack("<QQII", 2, 1, 0, 0) + struct.pack("<III", 0, 1, 1))
    _err(L.pbg_graph_load_bin(str(sized).encode(), 0, ctypes.byref(h)), "size does not match its header")
    assert not h.value


def test_error_messages_belong_to_the_calling_thread():
    L = pb.lib()
    _err(L.pbg_batch_create(0, ctypes.byref(ctypes.c_void_p())), "max_jobs")
    seen = {}

    def other():
        seen["before"] = L.pbg_last_error()
        L.pbg_autotune_clear(None)
        seen["after"] = L.pbg_last_error()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen["before"] == b""
    assert b"graph is NULL" in seen["after"]
    # this thread still holds its own message
    assert b"max_jobs" in L.pbg_last_error()


def test_python_wrapper_raises_with_the_code_and_message():
    L = pb.lib()
    with pytest.raises(pb.PbgError) as ei:
        _capi.check(L.pbg_batch_create(0, ctypes.byref(ctypes.c_void_p())))
    assert ei.value.code == ERR_ARG
    assert "PBG_ERR_ARG" in str(ei.value) and "max_jobs" in str(ei.value)


DROPIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "BFSTime_gpuBFS")


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in driver not built")
def test_dropin_fails_loudly_without_a_gpu(tmp_path):
    """The drop-in behind the reference's unmodified BFSTime driver has no
    CPU fallback: without a usable GPU it reports the failing call on stderr
    and aborts, which the PBBS runner counts as a failure
    (common/runTests.py:21-22), and writes no output file."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the drop-in runs in tests/test_bfs_gpu.py")
    from oracle import oracle as O

    off, edg = O.rmat(8, 10 * 256, 1, 0.5, 0.1, 0.1)
    gfile, ofile = str(tmp_path / "g.adj"), str(tmp_path / "out.seq")
    O.write_adjacency_graph(gfile, off, edg)
    r = subprocess.run([DROPIN, "-r", "1", "-o", ofile, gfile], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "gpuBFS: pbg_graph_upload failed (2)" in r.stderr
    assert not os.path.exists(ofile)


def test_python_bfs_fails_loudly_without_a_gpu():
    """pbbsbench_b200.BFS (the reference's BFS(start, G, verbose)) goes
    through the CUDA library only: without a usable GPU it raises."""
    import numpy as np
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; BFS runs in tests/test_bfs_gpu.py")
    G = pb.Graph(np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32))
    with pytest.raises(pb.PbgError) as ei:
        pb.BFS(0, G)
    assert ei.value.code == 2 and "PBG_ERR_CUDA" in str(ei.value)


def test_every_remaining_entry_point_rejects_null_handles(tmp_path):
    L = pb.lib()
    path = str(tmp_path / "x").encode()
    cnt = ctypes.c_uint32()
    cases = [
        (L.pbg_graph_info, (None, None, None, None, None), "graph is NULL"),
        (L.pbg_graph_flags, (FAKE, None), "NULL argument"),
        (L.pbg_graph_download, (None, FAKE, None), "NULL argument"),
        (L.pbg_graph_write_adj, (None, path), "NULL argument"),
        (L.pbg_graph_save_bin, (None, path), "NULL argument"),
        (L.pbg_bfs_trace, (None, None, 0, ctypes.byref(cnt)), "NULL argument"),
        (L.pbg_bfs_batch, (None, None, 1, None, None), "NULL argument"),
        (L.pbg_batch_job_stats, (None, FAKE, None), "NULL argument"),
        (L.pbg_batch_job_trace, (FAKE, FAKE, None, 0, None), "NULL argument"),
        (L.pbg_bfs_multi, (None, FAKE, 1, None, FAKE, None), "NULL argument"),
        (L.pbg_bfs_multi, (FAKE, FAKE, 0, None, FAKE, None), "k must be in [1, 256]"),
        (L.pbg_bfs_multi, (FAKE, FAKE, 257, None, FAKE, None), "k must be in [1, 256]"),
        (L.pbg_bfs_multi_trace, (None, None, 0, ctypes.byref(cnt)), "NULL argument"),
        (L.pbg_levels_check, (None, FAKE, 1, FAKE, None), "NULL argument"),
        (L.pbg_server_replay, (None, None, None, None, 0), "NULL argument"),
        (L.pbg_server_poll, (None, None, 0, ctypes.byref(cnt), 0), "NULL argument"),
        (L.pbg_server_stats_get, (None, None), "NULL argument"),
        (L.pbg_mis, (None, FAKE, None), "graph is NULL"),
        (L.pbg_mis, (FAKE, None, None), "flags_out is NULL"),
        (L.pbg_mis_device, (None, FAKE, None), "graph is NULL"),
        (L.pbg_mis_device, (FAKE, None, None), "d_flags is NULL"),
        (L.pbg_mis_stats_get, (None, None), "NULL argument"),
        (L.pbg_mis_trace, (None, None, 0, ctypes.byref(cnt)), "NULL argument"),
        (L.pbg_mis_trace, (FAKE, None, 4, ctypes.byref(cnt)), "NULL argument"),
    ]
    for fn, args, frag in cases:
        _err(fn(*args), frag)
    # releasing nothing succeeds; sizing nothing is 0
    for free in (L.pbg_graph_free, L.pbg_msbfs_free, L.pbg_batch_free, L.pbg_server_destroy):
        assert free(None) == 0
    assert L.pbg_msbfs_bytes(None, None) == 0 and L.pbg_msbfs_bytes_k(None, None, 64) == 0
    assert L.pbg_msbfs_bytes_k(FAKE, None, 0) == 0 and L.pbg_msbfs_bytes_k(FAKE, None, 257) == 0
    L.pbg_bfs_opts_default(None)
