"""The device checker (pbg_bfs_check, pbg_levels_check) against the oracle's
restatement of checkBFS (BFSCheck.C:39-90).  Mistakes are planted in host
copies of parent arrays and level rows; the verdict (first bad vertex, or
none) must be the oracle's."""
import numpy as np
import pytest
import torch

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NONE = pb.NONE


def _gpu_verdict(dg, src, parent, edges=True):
    d = torch.from_numpy(np.ascontiguousarray(parent).view(np.int32)).cuda()
    r = dg.check(src, d, edges=edges)
    return r["bad_vertex"]


def _oracle_verdict(off, edg, src, parent, edges=True):
    b = O.check_bfs(off, edg, src, np.ascontiguousarray(parent).view(np.uint32), check_edges=edges)
    return NONE if b < 0 else b


@pytest.fixture(scope="module")
def graph():
    off, edg = O.rmat(14, 10 << 14, 21, 0.5, 0.1, 0.1)
    return off, edg


def test_valid_trees(cuda_device, graph):
    off, edg = graph
    dg = pb.DeviceGraph.upload(off, edg)
    for src in (0, 5, 999):
        for mode in (pb.PARENT_ANY, pb.PARENT_MIN, pb.PARENT_MAX):
            par, _, _ = dg.bfs(src, parent_mode=mode)
            assert _gpu_verdict(dg, src, par) == NONE
    dg.close()


def test_planted_mistakes(cuda_device, graph):
    off, edg = graph
    dg = pb.DeviceGraph.upload(off, edg)
    src = 0
    par, lv, _ = dg.bfs(src, levels=True)
    par = par.view(np.uint32).copy()
    lv = lv.copy()
    reached = np.nonzero((lv != NONE) & (np.arange(len(lv)) != src))[0]
    rng = np.random.default_rng(3)
    deep = reached[np.argsort(lv[reached])][-50:]
    cases = {}
    p = par.copy(); p[src] = int(deep[0]); cases["start not its own parent"] = p
    v = int(deep[-1]); p = par.copy(); p[v] = par[par[v]]; cases["parent two levels up"] = p
    v = int(deep[-2]); same = np.nonzero(lv == lv[par[v]])[0]
    nbrs = set(edg[off[v]:off[v + 1]].tolist())
    cand = [int(u) for u in same if int(u) not in nbrs]
    p = par.copy(); p[v] = cand[0]; cases["parent not a neighbour"] = p
    v = int(deep[-3]); p = par.copy(); p[v] = NONE; cases["reached reported unreached"] = p
    un = np.nonzero(lv == NONE)[0]
    if len(un):
        p = par.copy(); p[int(un[0])] = src; cases["unreached given a parent"] = p
    a, b = int(deep[-4]), int(deep[-5]); p = par.copy(); p[a] = b; p[b] = a; cases["cycle"] = p
    p = par.copy(); p[int(deep[-6])] = len(lv) + 7; cases["parent not a vertex"] = p
    for name, p in cases.items():
        for edges in (True, False):
            want = _oracle_verdict(off, edg, src, p, edges)
            got = _gpu_verdict(dg, src, p, edges)
            assert got == want, (name, edges, got, want)
            # only the edge test sees a non-neighbour parent at the right level
            if name != "parent not a neighbour" or edges:
                assert want != NONE, (name, edges)
    dg.close()


def test_levels_rows(cuda_device, graph):
    off, edg = graph
    dg = pb.DeviceGraph.upload(off, edg)
    n = dg.n
    srcs = np.array([0, 7, 123, 4096], np.uint32)
    lv, _ = dg.bfs_multi(srcs)
    d = torch.from_numpy(lv.reshape(-1)).cuda()
    assert dg.levels_check(srcs, d)["bad_vertex"] == NONE
    bad = lv.copy()
    v = int(np.nonzero(bad[2] == 3)[0][0])
    bad[2, v] = 5
    r = dg.levels_check(srcs, torch.from_numpy(bad.reshape(-1)).cuda())
    assert r["row"] == 2 and r["bad_vertex"] <= v
    bad = lv.copy()
    bad[1, srcs[1]] = 1
    r = dg.levels_check(srcs, torch.from_numpy(bad.reshape(-1)).cuda())
    assert r["row"] == 1 and r["bad_vertex"] <= srcs[1]
    dg.close()


def test_full_size_rmat24_tree(cuda_device):
    """The C3 graph: a parent tree from the device search checked on the
    device in well under a second."""
    dg = pb.rmat_graph(24, 1 << 28, 3, 0.57, 0.19, 0.19)
    off = dg.download_offsets()
    src = int(np.nonzero(np.diff(off))[0][0])
    par = torch.empty(dg.n, dtype=torch.int32, device="cuda")
    dg.bfs_device(src, par)
    torch.cuda.synchronize()
    assert dg.check(src, par)["bad_vertex"] == NONE
    dg.close()


def test_long_lists_checked_through_their_tails(cuda_device):
    """A vertex whose list is longer than the 64 entries one lane scans: its
    only neighbour one level up (its parent) sits in the list's tail, which
    the device check reads in pieces spread over the grid.  A correct tree
    passes only if the tail's minimum level and adjacency are used; a parent
    at the right level that is not a neighbour is caught by the edge test."""
    n, h, p, q = 1000, 999, 900, 950
    us = [0, p, 0] + [h] * 399
    vs = [p, h, q] + list(range(1, 400))
    off, edg = O.csr_symmetric(n, np.array(us, np.uint32), np.array(vs, np.uint32))
    assert off[h + 1] - off[h] == 400 and list(edg[off[h]:off[h + 1]]).index(p) == 399
    dg = pb.DeviceGraph.upload(off, edg)
    par, lv, _ = dg.bfs(0, levels=True)
    par = par.view(np.uint32).copy()
    assert par[h] == p and lv[h] == 2
    cases = {"valid": par}
    x = par.copy(); x[h] = q; cases["parent at the right level, not a neighbour"] = x
    x = par.copy(); x[p] = NONE; cases["the tail neighbour unreached"] = x
    for name, pp in cases.items():
        for edges in (True, False):
            want = _oracle_verdict(off, edg, 0, pp, edges)
            got = _gpu_verdict(dg, 0, pp, edges)
            assert got == want, (name, edges, got, want)
    assert _oracle_verdict(off, edg, 0, par, True) == NONE
    assert _oracle_verdict(off, edg, 0, cases["parent at the right level, not a neighbour"], True) == h
    assert _oracle_verdict(off, edg, 0, cases["parent at the right level, not a neighbour"], False) == NONE
    dg.close()
