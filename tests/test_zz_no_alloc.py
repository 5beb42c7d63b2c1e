"""pbg_bfs_noalloc: the single-source BFS for callers that cannot allocate
device memory (a latency-critical path that must not hit cudaMalloc's
device-wide synchronisation, a process whose memory another framework has
capped or reserved, a plugin that may only use the buffers it is handed).
It keeps its scratch in one fixed device array instead.

Checked through the C ABI, on the same library instance, two or more calls
in a row (so later calls also show that the shared scratch left by earlier
ones does not leak into their results):
* against the allocating entry point (pbg_bfs) on the same graph: levels
  and deterministic parents bit-exact;
* against the oracle (the sequential BFS of serialBFS/BFS.C:32-55 and the
  deterministic parent rules): levels bit-exact, MIN and MAX parents
  bit-exact, first-claimer (ANY) parents a valid BFS tree;
* on a symmetric rMat graph, on a directed graph (flags 0: top-down only,
  the degree-0 bitmap holds only its padding bits), and on a graph near
  PBG_NOALLOC_MAX_VERTICES / PBG_NOALLOC_MAX_EDGES with a hub adjacent to
  every vertex, where the fixed queue capacities of the scratch layout are
  used; one call passes d_level = NULL.
Collected last (file name), so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

import pbbsbench_b200 as pb
from pbbsbench_b200 import _capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RULE = {pb.PARENT_MIN: "min", pb.PARENT_MAX: "max"}


def _dev(a, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(device)


def _noalloc(d_off, d_edg, n, m, flags, src, mode, device, levels=True):
    import torch

    L = pb.lib()
    d_par = torch.full((n,), 7, dtype=torch.int32, device=device)
    d_lv = torch.full((n,), 7, dtype=torch.int32, device=device) if levels else None
    rc = L.pbg_bfs_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_edg.data_ptr()), n, m, flags,
                           src, mode, ctypes.c_void_p(d_par.data_ptr()),
                           ctypes.c_void_p(d_lv.data_ptr()) if levels else None, None)
    assert rc == 0, L.pbg_last_error()
    par = d_par.cpu().numpy().view(np.uint32)
    return par, (d_lv.cpu().numpy().view(np.uint32) if levels else None)


def _tree_ok(off, edg, src, par, lv):
    """Every reached vertex but src has a parent one level up joined to it by
    an out-edge (the reference's check without its symmetric-only level
    test), and unreached vertices have no parent."""
    n = len(off) - 1
    reached = lv != pb.NONE
    if not np.array_equal(reached, par != pb.NONE) or par[src] != src:
        return False
    v = np.nonzero(reached)[0]
    v = v[v != src]
    p = par[v].astype(np.int64)
    if np.any(p >= n) or np.any(lv[p] + 1 != lv[v]):
        return False
    keys = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64))) * n + edg.astype(np.int64)
    keys.sort()
    want = p * n + v
    pos = np.searchsorted(keys, want)
    return bool(np.all(pos < len(keys)) and np.all(keys[np.minimum(pos, len(keys) - 1)] == want))


def _check_against_both(dg, off, edg, flags, srcs, device, modes=(pb.PARENT_MIN, pb.PARENT_MAX, pb.PARENT_ANY)):
    n, m = len(off) - 1, len(edg)
    d_off, d_edg = _dev(off, device), _dev(edg, device)
    for src in srcs:
        want_lv = O.bfs_levels(off, edg, src)
        for mode in modes:
            got_par, got_lv = _noalloc(d_off, d_edg, n, m, flags, src, mode, device)
            ref_par, ref_lv, _ = dg.bfs(src, parent_mode=mode, levels=True,
                                        direction=pb.DIR_AUTO if flags else pb.DIR_TOPDOWN)
            assert np.array_equal(got_lv, want_lv)  # levels: bit-exact against the oracle
            assert np.array_equal(got_lv, ref_lv)  # and against pbg_bfs
            if mode in RULE:
                want_par = O.bfs_det_parent(off, edg, src, RULE[mode])
                assert np.array_equal(got_par, want_par)  # deterministic parents: bit-exact
                assert np.array_equal(got_par, ref_par.view(np.uint32))
            elif flags & _capi.GRAPH_SYMMETRIC:
                assert O.check_bfs(off, edg, src, got_par) == -1  # first-claimer parents: a valid BFS tree
            else:
                assert _tree_ok(off, edg, src, got_par, got_lv)


def test_noalloc_matches_allocating_entry_point(cuda_device):
    off, edg = O.rmat(16, 16 * 65536, 3, 0.57, 0.19, 0.19)
    assert len(off) - 1 <= _capi.NOALLOC_MAX_VERTICES and len(edg) <= _capi.NOALLOC_MAX_EDGES
    dg = pb.DeviceGraph.upload(off, edg)
    nz = np.nonzero(np.diff(off))[0]
    _check_against_both(dg, off, edg, _capi.GRAPH_SYMMETRIC, (int(nz[0]), int(nz[len(nz) // 2])), cuda_device)
    dg.close()


def test_noalloc_directed_graph(cuda_device):
    """flags 0: out-edges only, never bottom-up; duplicates and self loops kept."""
    rng = np.random.default_rng(11)
    n, m = 50000, 200000
    us = rng.integers(0, n, m).astype(np.uint32)
    vs = rng.integers(0, n, m).astype(np.uint32)
    order = np.lexsort((vs, us))
    us, vs = us[order], vs[order]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, us.astype(np.int64) + 1, 1)
    off = np.cumsum(off).astype(np.uint32)
    edg = vs.copy()
    dg = pb.DeviceGraph.upload(off, edg, symmetric=False)
    _check_against_both(dg, off, edg, 0, (0, 4321), cuda_device)
    dg.close()


def test_noalloc_near_its_limits(cuda_device):
    """n = PBG_NOALLOC_MAX_VERTICES, m close to PBG_NOALLOC_MAX_EDGES, and a
    hub joined to every vertex, so the big-list (chunk) queues and the
    frontier queues of the fixed layout fill up; the last call passes
    d_level = NULL."""
    logn = 20
    n = 1 << logn
    L = O.lib()
    samples = 6 * n
    us = np.empty(samples, np.uint32)
    vs = np.empty(samples, np.uint32)
    ta, tab, tabc = O.prob_thresholds(0.57, 0.19, 0.19)
    L.orc_gen_rmat(logn, samples, 21, ta, tab, tabc, us, vs)
    hub = np.uint32(12345)
    us = np.concatenate([us, np.full(n, hub, np.uint32)])
    vs = np.concatenate([vs, np.arange(n, dtype=np.uint32)])
    off, edg = O.csr_symmetric(n, us, vs)
    assert len(off) - 1 == _capi.NOALLOC_MAX_VERTICES
    assert (3 * _capi.NOALLOC_MAX_EDGES) // 4 < len(edg) <= _capi.NOALLOC_MAX_EDGES
    dg = pb.DeviceGraph.upload(off, edg)
    nz = np.nonzero(np.diff(off))[0]
    srcs = (int(hub), int(nz[len(nz) // 3]))
    _check_against_both(dg, off, edg, _capi.GRAPH_SYMMETRIC, srcs, cuda_device)
    d_off, d_edg = _dev(off, cuda_device), _dev(edg, cuda_device)
    par, _ = _noalloc(d_off, d_edg, n, len(edg), _capi.GRAPH_SYMMETRIC, srcs[1], pb.PARENT_MIN, cuda_device,
                      levels=False)
    assert np.array_equal(par, O.bfs_det_parent(off, edg, srcs[1], "min"))
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
