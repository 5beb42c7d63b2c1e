"""pbg_bfs_noalloc: the single-source BFS for callers that cannot allocate
device memory (a latency-critical path that must not hit cudaMalloc's
device-wide synchronisation, a process whose memory another framework has
capped or reserved, a plugin that may only use the buffers it is handed).
It keeps its scratch in one fixed device array instead.

Checked through the C ABI against the allocating entry point (pbg_bfs): two
calls in a row on the same library instance, so the second call also shows
that the shared scratch left by the first does not leak into its result.
Collected last (file name), so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

import pbbsbench_b200 as pb
from pbbsbench_b200 import _capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(device)


def test_noalloc_matches_allocating_entry_point(cuda_device):
    import torch

    off, edg = O.rmat(16, 16 * 65536, 3, 0.57, 0.19, 0.19)
    n, m = len(off) - 1, len(edg)
    assert n <= _capi.NOALLOC_MAX_VERTICES and m <= _capi.NOALLOC_MAX_EDGES
    d_off, d_edg = _dev(off, cuda_device), _dev(edg, cuda_device)
    dg = pb.DeviceGraph.upload(off, edg)
    nz = np.nonzero(np.diff(off))[0]
    L = pb.lib()
    for src in (int(nz[0]), int(nz[len(nz) // 2])):  # two calls in a row
        for mode in (pb.PARENT_MIN, pb.PARENT_ANY):
            want_par, want_lv, _ = dg.bfs(src, parent_mode=mode, levels=True)
            d_par = torch.full((n,), 7, dtype=torch.int32, device=cuda_device)
            d_lv = torch.full((n,), 7, dtype=torch.int32, device=cuda_device)
            rc = L.pbg_bfs_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_edg.data_ptr()), n, m,
                                   _capi.GRAPH_SYMMETRIC, src, mode, ctypes.c_void_p(d_par.data_ptr()),
                                   ctypes.c_void_p(d_lv.data_ptr()), None)
            assert rc == 0, L.pbg_last_error()
            got_par = d_par.cpu().numpy().view(np.uint32)
            got_lv = d_lv.cpu().numpy().view(np.uint32)
            assert np.array_equal(got_lv, want_lv)  # levels: bit-exact
            if mode == pb.PARENT_MIN:
                assert np.array_equal(got_par, want_par.view(np.uint32))  # deterministic parents: bit-exact
            else:
                assert O.check_bfs(off, edg, src, got_par) == -1  # first-claimer parents: a valid BFS tree
    dg.close()


def test_noalloc_rejects_sizes_beyond_its_limit(cuda_device):
    import torch

    L = pb.lib()
    buf = torch.zeros(16, dtype=torch.int32, device=cuda_device)
    p = ctypes.c_void_p(buf.data_ptr())
    rc = L.pbg_bfs_noalloc(p, p, _capi.NOALLOC_MAX_VERTICES + 1, 0, 0, 0, 0, p, None, None)
    assert rc == _capi.PBG_OK + 1 and b"PBG_NOALLOC_MAX_VERTICES" in L.pbg_last_error()
    rc = L.pbg_bfs_noalloc(p, p, 4, _capi.NOALLOC_MAX_EDGES + 1, 0, 0, 0, p, None, None)
    assert rc == 1 and b"PBG_NOALLOC_MAX_EDGES" in L.pbg_last_error()
