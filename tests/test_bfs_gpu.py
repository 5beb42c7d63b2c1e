"""Parity of the CUDA BFS (through the C ABI) with the oracle.

* levels bit-exact against the sequential BFS (serialBFS/BFS.C:32-55) for every
  parent rule and direction policy;
* PARENT_ANY parents pass the strengthened checker (BFSCheck.C:59-90 plus edge
  existence) and, where built, the reference's own checkBFS;
* PARENT_MIN / PARENT_MAX parents bit-exact against the oracle's
  deterministic rules (MAX = deterministicBFS/BFS.C:60-74, checked against the
  reference's own output in the golden fixture).
"""
import ctypes
import os

import numpy as np
import pytest

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "bfs_golden.npz")
MODES = [pb.PARENT_ANY, pb.PARENT_MIN, pb.PARENT_MAX]
DIRS = [pb.DIR_AUTO, pb.DIR_TOPDOWN, pb.DIR_BOTTOMUP]


def golden_cases():
    z = np.load(GOLDEN)
    for name in z["names"]:
        name = str(name)
        yield name, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


def levels_of(off, edg, s):
    return O.bfs_levels(off, edg, s)


def check_run(dg, off, edg, s, mode, direction, **tune):
    par, lv, st = dg.bfs(s, parent_mode=mode, direction=direction, levels=True, **tune)
    want = levels_of(off, edg, s)
    assert np.array_equal(lv, want), "levels differ (src %d mode %d dir %d)" % (s, mode, direction)
    p = par.view(np.uint32)
    if mode == pb.PARENT_ANY:
        assert O.check_bfs(off, edg, s, p) == -1
    else:
        assert np.array_equal(p, O.bfs_det_parent(off, edg, s, "min" if mode == pb.PARENT_MIN else "max"))
    reached = want != O.NONE
    assert st["visited"] == int(reached.sum())
    assert st["edges_reached"] == int(np.diff(off.astype(np.int64))[reached].sum())
    assert st["levels"] == (int(want[reached].max()) + 1)
    return par, st


@pytest.mark.parametrize("name,case", list(golden_cases()))
def test_golden_graphs_all_modes(cuda_device, name, case):
    off, edg = case["offsets"], case["edges"]
    dg = pb.DeviceGraph.upload(off, edg, symmetric=True)
    for i, s in enumerate(case["srcs"]):
        s = int(s)
        for mode in MODES:
            for d in DIRS:
                par, _ = check_run(dg, off, edg, s, mode, d)
                if mode == pb.PARENT_MAX:
                    # the reference's own deterministicBFS output, bit-exact
                    assert np.array_equal(par, case["det_max_parent"][i])
    dg.close()


@pytest.mark.parametrize("chunk", [1, 8, 32, 300, 4096])
@pytest.mark.parametrize("block", [256, 1024])
def test_degree_bins_and_block_sizes(cuda_device, chunk, block):
    """Every list through both top-down bins: one thread per short list
    (deg < chunk) and 256-edge pieces over the grid (deg >= chunk, including
    lists of many pieces); 4096 makes every list thread-walked."""
    off, edg = O.rmat(13, 16 * 8192, 3, 0.57, 0.19, 0.19)
    dg = pb.DeviceGraph.upload(off, edg)
    for mode in MODES:
        check_run(dg, off, edg, 0, mode, pb.DIR_TOPDOWN, chunk_min_degree=chunk, block_threads=block)
        check_run(dg, off, edg, 5, mode, pb.DIR_AUTO, chunk_min_degree=chunk, block_threads=block)
    dg.close()


@pytest.mark.parametrize("kind", ["randlocal", "torus"])
def test_lean_and_chunked_kernels_agree(cuda_device, kind):
    """A graph whose lists are all shorter than the chunk degree runs the lean
    kernel (no chunk queue); the same graph with the chunk degree at its
    largest degree runs the chunked kernel.  Both equal the oracle (levels,
    MIN/MAX parents bit-exact, ANY parents checked) in every direction
    policy, with the same level counts and statistics."""
    if kind == "randlocal":
        off, edg = O.randlocal(1 << 14, 5, 256, 4)
    else:
        off, edg = O.torus3d(24, 7)
    dmax = int(np.diff(off.astype(np.int64)).max())
    dg = pb.DeviceGraph.upload(off, edg)
    keys = ("levels", "topdown_levels", "bottomup_levels", "visited", "edges_reached", "bottomup_mask")
    for mode in MODES:
        for d in DIRS:
            for s in (0, 17):
                _, lean = check_run(dg, off, edg, s, mode, d, chunk_min_degree=dmax + 1)
                _, chunked = check_run(dg, off, edg, s, mode, d, chunk_min_degree=dmax)
                assert {k: lean[k] for k in keys} == {k: chunked[k] for k in keys}
    dg.close()


def test_star_chunked_hub(cuda_device):
    n = 50000
    us = np.zeros(n - 1, np.uint32)
    vs = np.arange(1, n, dtype=np.uint32)
    off, edg = O.csr_symmetric(n, us, vs)
    dg = pb.DeviceGraph.upload(off, edg)
    for mode in MODES:
        for d in DIRS:
            for s in (0, 777):
                check_run(dg, off, edg, s, mode, d)
    dg.close()


def test_directed_graph_topdown_only(cuda_device):
    """A non-symmetric graph: the search follows out-edges and never runs
    bottom-up (which would read N(v) as in-neighbours)."""
    rng = np.random.default_rng(5)
    n, m = 3000, 12000
    us = rng.integers(0, n, m).astype(np.uint32)
    vs = rng.integers(0, n, m).astype(np.uint32)
    order = np.lexsort((vs, us))
    us, vs = us[order], vs[order]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, us.astype(np.int64) + 1, 1)
    off = np.cumsum(off).astype(np.uint32)
    edg = vs.copy()  # duplicates and self loops kept, as graphFromEdges does without -j
    dg = pb.DeviceGraph.upload(off, edg, symmetric=False)
    for mode in MODES:
        par, lv, st = dg.bfs(0, parent_mode=mode, levels=True)
        assert np.array_equal(lv, levels_of(off, edg, 0))
        assert st["bottomup_levels"] == 0
        if mode != pb.PARENT_ANY:
            assert np.array_equal(par.view(np.uint32),
                                  O.bfs_det_parent(off, edg, 0, "min" if mode == pb.PARENT_MIN else "max"))
    with pytest.raises(pb.PbgError):
        dg.bfs(0, direction=pb.DIR_BOTTOMUP)
    dg.close()


def test_single_vertex_and_empty_edges(cuda_device):
    off = np.zeros(2, np.uint32)
    edg = np.zeros(0, np.uint32)
    dg = pb.DeviceGraph.upload(off, edg)
    par, lv, st = dg.bfs(0, levels=True)
    assert par.tolist() == [0] and lv.tolist() == [0] and st["levels"] == 1
    dg.close()


def test_bad_inputs_are_rejected(cuda_device):
    off, edg = O.torus3d(4, None)
    dg = pb.DeviceGraph.upload(off, edg)
    with pytest.raises(pb.PbgError):
        dg.bfs(len(off) - 1)
    with pytest.raises(pb.PbgError):
        dg.bfs(0, block_threads=100)
    dg.close()
    bad = edg.copy()
    bad[3] = len(off) + 5
    with pytest.raises(pb.PbgError, match="edge target"):
        pb.DeviceGraph.upload(off, bad)
    bad_off = off.copy()
    bad_off[5] = bad_off[6] + 1  # decreasing offsets
    with pytest.raises(pb.PbgError, match="non-decreasing"):
        pb.DeviceGraph.upload(bad_off, edg)
    h = ctypes.c_void_p()
    rc = pb.lib().pbg_graph_upload(pb._ptr(off), pb._ptr(edg), len(off) - 1, len(edg) - 1, 1, ctypes.byref(h))
    assert rc == 1 and b"offsets[n]" in pb.lib().pbg_last_error()


def test_reference_checker_accepts_gpu_parents(cuda_device):
    if not O.ref_available():
        pytest.skip("reference library not built")
    off, edg = O.rmat(14, 10 * (1 << 14), 1, 0.5, 0.1, 0.1)
    G = O.RefGraph(off, edg)
    dg = pb.DeviceGraph.upload(off, edg)
    for s in (0, 9, 12345):
        for d in DIRS:
            par, _, _ = dg.bfs(s, direction=d)
            assert G.check(s, par) == 0
    dg.close()
    G.close()


@pytest.mark.parametrize("kind", ["rmat", "torus", "randlocal"])
def test_device_generators_match_oracle(cuda_device, kind):
    if kind == "rmat":
        dg = pb.rmat_graph(12, 16 * 4096, 3, 0.57, 0.19, 0.19)
        want = O.rmat(12, 16 * 4096, 3, 0.57, 0.19, 0.19)
    elif kind == "torus":
        dg = pb.torus3d_graph(10, perm_seed=2)
        want = O.torus3d(10, 2)
    else:
        dg = pb.randlocal_graph(5000, 5, 300, 4)
        want = O.randlocal(5000, 5, 300, 4)
    off, edg = dg.download()
    assert np.array_equal(off, want[0]) and np.array_equal(edg, want[1])
    dg.close()


def test_bfs_entry_point_mirrors_reference(cuda_device):
    off, edg = O.rmat(12, 10 * 4096, 1, 0.5, 0.1, 0.1)
    G = pb.Graph(off, edg)
    par = pb.BFS(0, G)
    assert par.dtype == np.int32 and len(par) == G.numVertices()
    assert par[0] == 0
    assert O.check_bfs(off, edg, 0, par.view(np.uint32)) == -1
    assert np.array_equal(O.level_number(par.view(np.uint32)), O.level_number(O.bfs_serial(off, edg, 0)))


def test_device_buffers_and_stream(cuda_device):
    import torch

    off, edg = O.torus3d(12, 2)
    dg = pb.DeviceGraph.upload(off, edg)
    n = len(off) - 1
    par = torch.empty(n, dtype=torch.int32, device=cuda_device)
    lv = torch.empty(n, dtype=torch.int32, device=cuda_device)
    s = torch.cuda.Stream()
    dg.bfs_device(3, par, lv, stream=s.cuda_stream)
    s.synchronize()
    st = dg.last_stats()
    assert np.array_equal(lv.cpu().numpy().view(np.uint32), levels_of(off, edg, 3))
    assert O.check_bfs(off, edg, 3, par.cpu().numpy().view(np.uint32)) == -1
    assert st["levels"] == int(lv.max().item()) + 1
    dg.close()


@pytest.mark.parametrize("cfg", ["c1_rmat20", "c2_torus160"])
def test_config_graphs_full_parity(cuda_device, cfg):
    """The two single-source benchmark graphs at full size: levels bit-exact
    against the sequential BFS on the downloaded CSR, parents checked."""
    if cfg == "c1_rmat20":
        dg = pb.rmat_graph(20, 10 * (1 << 20), 1, 0.5, 0.1, 0.1)
    else:
        dg = pb.torus3d_graph(160, perm_seed=2)
    off, edg = dg.download()
    want = levels_of(off, edg, 0)
    for mode in MODES:
        par, lv, st = dg.bfs(0, parent_mode=mode, levels=True)
        assert np.array_equal(lv, want)
        if mode == pb.PARENT_ANY:
            assert O.check_bfs(off, edg, 0, par.view(np.uint32)) == -1
        else:
            assert np.array_equal(par.view(np.uint32),
                                  O.bfs_det_parent(off, edg, 0, "min" if mode == pb.PARENT_MIN else "max"))
    if cfg == "c2_torus160":
        assert st["levels"] > 200
    dg.close()


@pytest.mark.slow
def test_c3_rmat24_levels_full_size(cuda_device):
    """rMat 2^24 / 2^28 samples (the direction-optimizing headline graph):
    levels bit-exact for two sources, min-parent bit-exact for one."""
    dg = pb.rmat_graph(24, 1 << 28, 3, 0.57, 0.19, 0.19)
    off, edg = dg.download()
    deg = np.diff(off.astype(np.int64))
    nz = np.nonzero(deg)[0]
    rng = np.random.default_rng(3)
    for s in [int(nz[i]) for i in rng.integers(0, len(nz), 2)]:
        want = levels_of(off, edg, s)
        par, lv, st = dg.bfs(s, levels=True)
        assert np.array_equal(lv, want)
        assert st["bottomup_levels"] >= 1
        assert O.check_bfs(off, edg, s, par.view(np.uint32)) == -1
    par, _, _ = dg.bfs(s, parent_mode=pb.PARENT_MIN)
    assert np.array_equal(par.view(np.uint32), O.bfs_det_parent(off, edg, s, "min"))
    dg.close()


DROPIN = os.path.join(os.path.dirname(O.__file__), "_ref", "BFSTime_gpuBFS")
CHECKER = os.path.join(os.path.dirname(O.__file__), "_ref", "BFSCheck")


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(CHECKER)), reason="drop-in driver not built")
def test_dropin_behind_reference_driver_and_checker(cuda_device, tmp_path):
    """The unmodified reference driver bench/BFSTime.C linked with the drop-in
    gpuBFS/BFS.C reads an AdjacencyGraph file, runs warm-up + timed rounds and
    writes the parent sequence; the reference's BFSCheck accepts it."""
    import subprocess

    off, edg = O.rmat(14, 12 * (1 << 14), 1, 0.55, 0.125, 0.125)
    gfile, ofile = str(tmp_path / "g.adj"), str(tmp_path / "out.seq")
    O.write_adjacency_graph(gfile, off, edg)
    r = subprocess.run([DROPIN, "-r", "3", "-o", ofile, gfile], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stderr == "", r.stderr
    times = [l for l in r.stdout.splitlines() if l.startswith("Parlay time: ")]
    assert len(times) == 3
    c = subprocess.run([CHECKER, gfile, ofile], capture_output=True, text=True, timeout=120)
    assert c.returncode == 0 and c.stdout.strip() == "", c.stdout
    par = O.read_sequence_int(ofile).view(np.uint32)
    assert O.check_bfs(off, edg, 0, par) == -1
