"""Batched multi-source BFS (up to 64 sources per job, many jobs in one fused
launch): every source's uint8 level array bit-exact against an independent
sequential BFS from that source (serialBFS/BFS.C:32-55 distances)."""
import os

import numpy as np
import pytest

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "bfs_golden.npz")
DIRS = [pb.DIR_AUTO, pb.DIR_TOPDOWN, pb.DIR_BOTTOMUP]


def golden_cases():
    z = np.load(GOLDEN)
    for name in z["names"]:
        name = str(name)
        yield name, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name,case", list(golden_cases()))
def test_golden_graphs(cuda_device, name, case):
    off, edg = case["offsets"], case["edges"]
    n = len(off) - 1
    rng = np.random.default_rng(1)
    srcs = np.concatenate([case["srcs"], rng.integers(0, n, 20).astype(np.uint32), case["srcs"][:1]])
    dg = pb.DeviceGraph.upload(off, edg)
    want = O.levels_u8(off, edg, srcs)
    for d in DIRS:
        lv, st = dg.bfs_multi(srcs, direction=d)
        assert np.array_equal(lv, want), "direction %d" % d
        reached = want != 255
        assert st["levels"] == int(want[reached].max()) + 1
    dg.close()


@pytest.mark.parametrize("k", [1, 7, 63, 64])
@pytest.mark.parametrize("chunk", [1, 32, 2000])
def test_rmat_sources_and_bins(cuda_device, k, chunk):
    off, edg = O.rmat(13, 16 * 8192, 3, 0.57, 0.19, 0.19)
    n = len(off) - 1
    rng = np.random.default_rng(k)
    srcs = rng.integers(0, n, k).astype(np.uint32)
    srcs[0] = 0  # the biggest hub
    want = O.levels_u8(off, edg, srcs)
    dg = pb.DeviceGraph.upload(off, edg)
    for d in DIRS:
        lv, _ = dg.bfs_multi(srcs, direction=d, chunk_min_degree=chunk)
        assert np.array_equal(lv, want)
    dg.close()


def test_fused_launch_of_uneven_graphs(cuda_device):
    """Jobs on five graphs of different sizes and shapes in one launch."""
    import torch

    graphs = [O.rmat(10, 8 * 1024, 11, 0.57, 0.19, 0.19), O.torus3d(9, 2), O.randlocal(3000, 5, 50, 4),
              O.rmat(14, 16 * 16384, 12, 0.57, 0.19, 0.19), O.torus3d(4, None)]
    rng = np.random.default_rng(0)
    batch = pb.Batch(max_jobs=8)
    dgs, jobs, wants = [], [], []
    for off, edg in graphs:
        n = len(off) - 1
        dg = pb.DeviceGraph.upload(off, edg)
        ws = pb.MultiWorkspace(dg)
        k = int(rng.integers(1, 65))
        srcs = rng.integers(0, n, k).astype(np.uint32)
        dlev = torch.empty(k * n + 16, dtype=torch.uint8, device=cuda_device)
        dgs.append((dg, ws))
        jobs.append((ws, srcs, dlev))
        wants.append(O.levels_u8(off, edg, srcs))
    s = torch.cuda.Stream()
    batch.launch(jobs, stream=s.cuda_stream)
    s.synchronize()
    for (ws, srcs, dlev), want in zip(jobs, wants):
        k, n = want.shape
        got = dlev[: k * n].cpu().numpy().reshape(k, n)
        assert np.array_equal(got, want)
        st = batch.job_stats(ws)
        assert st["levels"] == int(want[want != 255].max()) + 1
    # the same batch object again, jobs in another order (staging reuse)
    batch.launch(jobs[::-1], stream=s.cuda_stream)
    s.synchronize()
    for (ws, srcs, dlev), want in zip(jobs, wants):
        k, n = want.shape
        assert np.array_equal(dlev[: k * n].cpu().numpy().reshape(k, n), want)
    batch.close()
    for dg, ws in dgs:
        ws.close()
        dg.close()


def test_level_overflow_is_reported(cuda_device):
    n = 300
    off, edg = O.csr_symmetric(n, np.arange(n - 1, dtype=np.uint32), np.arange(1, n, dtype=np.uint32))
    dg = pb.DeviceGraph.upload(off, edg)
    with pytest.raises(pb.PbgError, match="OVERFLOW"):
        dg.bfs_multi([0])
    lv, _ = dg.bfs_multi([150])  # depth 150 fits
    assert np.array_equal(lv, O.levels_u8(off, edg, [150]))
    dg.close()


def test_bad_batch_arguments(cuda_device):
    off, edg = O.torus3d(4, None)
    dg = pb.DeviceGraph.upload(off, edg)
    with pytest.raises(pb.PbgError):  # more than 256 sources
        dg.bfs_multi(np.arange(257, dtype=np.uint32) % 64)
    with pytest.raises(pb.PbgError):  # a source out of range
        dg.bfs_multi([64])
    ws = pb.MultiWorkspace(dg)  # sized for 64 sources
    batch = pb.Batch(max_jobs=1)
    import torch
    with pytest.raises(pb.PbgError):
        batch.launch([(ws, np.arange(65, dtype=np.uint32) % 64, torch.empty(65 * dg.n, dtype=torch.uint8, device="cuda"))])
    with pytest.raises(pb.PbgError):
        pb.MultiWorkspace(dg, max_sources=257)
    dg.close()


def test_c4_randlocal_64_sources_full_size(cuda_device):
    """randLocal n = 2^23, 5 out-neighbours within +-2^16, seed 4, 64 sources:
    every level array equal to a single-source search (the GPU path checked
    against the oracle above) and four of them against the oracle directly."""
    dg = pb.randlocal_graph(1 << 23, 5, 1 << 16, 4)
    n = dg.n
    rng = np.random.default_rng(4)
    srcs = rng.integers(0, n, 64).astype(np.uint32)
    lv, st = dg.bfs_multi(srcs)
    for i, s in enumerate(srcs):
        _, one, _ = dg.bfs(int(s), levels=True, parents=False)
        assert np.array_equal(lv[i], np.where(one == pb.NONE, 255, one).astype(np.uint8)), i
    off, edg = dg.download()
    for i in (0, 21, 42, 63):
        assert np.array_equal(lv[i], O.levels_u8(off, edg, srcs[i:i + 1])[0])
    dg.close()


def test_rmat18_64_sources_every_direction(cuda_device):
    """rMat n = 2^18, 16n samples (hubs of thousands of neighbours: the pull
    and dense-push chunk tails), 64 sources: every direction policy equal to
    the oracle."""
    off, edg = O.rmat(18, 16 << 18, 12, 0.57, 0.19, 0.19)
    n = len(off) - 1
    deg = np.diff(off)
    nz = np.nonzero(deg)[0]
    srcs = nz[np.random.default_rng(18).integers(0, len(nz), 64)].astype(np.uint32)
    srcs[0] = int(np.argmax(deg))
    want = O.levels_u8(off, edg, srcs)
    dg = pb.DeviceGraph.upload(off, edg)
    for d in DIRS:
        lv, st = dg.bfs_multi(srcs, direction=d)
        assert np.array_equal(lv, want), "direction %d" % d
        assert st["error"] == 0
    dg.close()


def _clique_path(blocks, size):
    """Cliques of `size` vertices joined in a path (last vertex of each to the
    first of the next): average degree about size, diameter about 2 * blocks."""
    adj = [[] for _ in range(blocks * size)]
    for b in range(blocks):
        base = b * size
        for i in range(size):
            for j in range(size):
                if i != j:
                    adj[base + i].append(base + j)
        if b + 1 < blocks:
            adj[base + size - 1].append(base + size)
            adj[base + size].append(base + size - 1)
    off = np.zeros(len(adj) + 1, np.uint32)
    off[1:] = np.cumsum([len(a) for a in adj])
    edg = np.array([v for a in adj for v in sorted(a)], np.uint32)
    return off, edg


@pytest.mark.parametrize("blocks", [3, 9, 40])
def test_dense_graph_many_levels(cuda_device, blocks):
    """A dense graph (average degree >= 16, so levels go through the planes
    and their flushes) with 5 to 80 levels: every flush window, first and
    later, against the oracle."""
    off, edg = _clique_path(blocks, 24)
    n = len(off) - 1
    assert len(edg) >= 16 * n
    rng = np.random.default_rng(blocks)
    srcs = rng.integers(0, n, 64).astype(np.uint32)
    srcs[0] = 0
    want = O.levels_u8(off, edg, srcs)
    dg = pb.DeviceGraph.upload(off, edg)
    for d in DIRS:
        lv, st = dg.bfs_multi(srcs, direction=d)
        assert np.array_equal(lv, want), "direction %d" % d
        assert st["levels"] == int(want[want != 255].max()) + 1
    dg.close()


@pytest.mark.parametrize("k", [65, 100, 128, 129, 200, 256])
def test_two_word_jobs_golden_and_rmat(cuda_device, k):
    """Jobs of 65..128 sources (two mask words per vertex) and 129..256 (four):
    every direction, on the golden graphs and on rMat 2^13 (16n), against the
    oracle."""
    rng = np.random.default_rng(k)
    for name, case in golden_cases():
        off, edg = case["offsets"], case["edges"]
        n = len(off) - 1
        srcs = rng.integers(0, n, k).astype(np.uint32)
        want = O.levels_u8(off, edg, srcs)
        dg = pb.DeviceGraph.upload(off, edg)
        for d in DIRS:
            lv, st = dg.bfs_multi(srcs, direction=d)
            assert np.array_equal(lv, want), (name, d)
        dg.close()
    off, edg = O.rmat(13, 16 * 8192, 3, 0.57, 0.19, 0.19)
    srcs = rng.integers(0, len(off) - 1, k).astype(np.uint32)
    srcs[0] = 0
    want = O.levels_u8(off, edg, srcs)
    dg = pb.DeviceGraph.upload(off, edg)
    for d in DIRS:
        lv, st = dg.bfs_multi(srcs, direction=d)
        assert np.array_equal(lv, want), d
        assert st["levels"] == int(want[want != 255].max()) + 1
    dg.close()


@pytest.mark.parametrize("kmax", [128, 256])
def test_two_word_jobs_dense_and_fused(cuda_device, kmax):
    """kmax-source jobs (two or four mask words) on a dense many-level graph
    (level planes, several flushes) and three graphs in one fused launch of
    workspaces of that width."""
    import torch

    off, edg = _clique_path(12, 24)
    srcs = np.random.default_rng(5).integers(0, len(off) - 1, kmax).astype(np.uint32)
    dg = pb.DeviceGraph.upload(off, edg)
    for d in DIRS:
        lv, _ = dg.bfs_multi(srcs, direction=d)
        assert np.array_equal(lv, O.levels_u8(off, edg, srcs)), d
    dg.close()
    graphs = [O.rmat(11, 16 * 2048, 12, 0.57, 0.19, 0.19), O.randlocal(4000, 5, 60, 4), _clique_path(5, 20)]
    dgs = [pb.DeviceGraph.upload(o, e) for o, e in graphs]
    wss = [pb.MultiWorkspace(g, max_sources=kmax) for g in dgs]
    batch = pb.Batch(max_jobs=4)
    jobs, wants = [], []
    for i, ((o, e), g, ws) in enumerate(zip(graphs, dgs, wss)):
        k = [kmax, 77, 100][i] if kmax == 128 else [256, 140, 200][i]
        s = np.random.default_rng(i).integers(0, g.n, k).astype(np.uint32)
        dl = torch.empty(k * g.n, dtype=torch.uint8, device="cuda")
        jobs.append((ws, s, dl))
        wants.append(O.levels_u8(o, e, s))
    batch.launch(jobs)
    torch.cuda.synchronize()
    for (ws, s, dl), want in zip(jobs, wants):
        assert np.array_equal(dl.cpu().numpy().reshape(len(s), -1), want)
        assert batch.job_stats(ws)["error"] == 0
    # one launch takes one size class
    ws64 = pb.MultiWorkspace(dgs[0])
    with pytest.raises(pb.PbgError):
        batch.launch([jobs[1], (ws64, jobs[0][1][:64], jobs[0][2])])


def _csr(n, pairs, symmetric=True):
    """CSR of an edge list (both directions when symmetric), lists ascending."""
    es = list(pairs) + ([(v, u) for u, v in pairs] if symmetric else [])
    es = sorted(set(es))
    off = np.zeros(n + 1, np.int64)
    for u, _ in es:
        off[u + 1] += 1
    off = np.cumsum(off).astype(np.uint32)
    return off, np.array([v for _, v in es], np.uint32)


@pytest.mark.parametrize("k", [1, 3, 64, 65, 200])
def test_batched_edge_cases(cuda_device, k):
    """One, two and four mask words on the shapes the level rows and planes
    handle specially.
    * n = 7: a partial 32-vertex tile, n not a multiple of 4 (byte stores),
      a self loop, an isolated vertex.
    * Duplicate sources and sources on isolated vertices.
    * A directed graph (pushes only; a pull is refused).
    * A dense graph of n = 1001, whose level planes are flushed.
    Every row is checked against the oracle's sequential BFS."""
    rng = np.random.default_rng(k)
    cases = []
    off, edg = _csr(7, [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 5)])
    cases.append((off, edg, True))
    pairs = [(int(u), int(v)) for u, v in zip(rng.integers(0, 500, 1500), rng.integers(0, 500, 1500))]
    cases.append(_csr(500, pairs, symmetric=False) + (False,))
    dense = [(int(u), int(v)) for u, v in zip(rng.integers(0, 1001, 12000), rng.integers(0, 1001, 12000)) if u != v]
    dense += [(i, i + 1) for i in range(0, 1000, 3)]
    cases.append(_csr(1001, dense) + (True,))
    for off, edg, sym in cases:
        n = len(off) - 1
        srcs = rng.integers(0, n, k).astype(np.uint32)
        if k >= 3:
            srcs[1] = srcs[0]  # a duplicate
        if n == 7:
            srcs[-1] = 6  # the isolated vertex
        want = O.levels_u8(off, edg, srcs)
        dg = pb.DeviceGraph.upload(off, edg, symmetric=sym)
        for d in (DIRS if sym else [pb.DIR_AUTO, pb.DIR_TOPDOWN]):
            lv, st = dg.bfs_multi(srcs, direction=d)
            assert np.array_equal(lv, want), (n, d)
        if not sym:
            with pytest.raises(pb.PbgError):
                dg.bfs_multi(srcs, direction=pb.DIR_BOTTOMUP)
        dg.close()
