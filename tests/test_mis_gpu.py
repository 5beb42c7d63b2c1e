"""Parity of the device maximal independent set (pbg_mis) with the reference.

* flags bit-exact against the reference's own serialMIS
  (maximalIndependentSet/serialMIS/MIS.C:33-47), through the golden fixture
  made from it and through the oracle's restatement pinned to it;
* on symmetric graphs the set passes the MIS check (MISCheck.C:39-66, the
  oracle's restatement and the reference's own binary);
* the drop-in gpuMIS/MIS.C behind the unmodified bench/MISTime.C writes flags
  the reference's MISCheck accepts.
"""
import os
import subprocess

import numpy as np
import pytest

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mis_golden.npz")


def golden_cases():
    z = np.load(GOLDEN)
    for name in z["names"]:
        name = str(name)
        yield name, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


def check_graph(dg, off, edg, symmetric=True):
    flags, st = dg.mis()
    want = O.mis_serial(off, edg)
    assert np.array_equal(flags, want), "flags differ from serialMIS at %s" % np.nonzero(flags != want)[0][:5]
    assert st["in_set"] == int((want == 1).sum()) and st["error"] == 0 and st["rounds"] >= 1
    if symmetric:
        assert O.check_mis(off, edg, flags) == -1
    return flags, st


@pytest.mark.parametrize("name,case", list(golden_cases()))
def test_golden_graphs(cuda_device, name, case):
    off, edg = case["offsets"], case["edges"]
    dg = pb.DeviceGraph.upload(off, edg, symmetric=not name.startswith("directed"))
    flags, _ = dg.mis()
    assert np.array_equal(flags, case["serial_flags"])  # the reference's own serialMIS output
    dg.close()


@pytest.mark.parametrize("kind", ["rmat16", "torus40", "randlocal16", "rmat16_dense"])
def test_generated_graphs(cuda_device, kind):
    if kind == "rmat16":
        off, edg = O.rmat(16, 10 << 16, 3, 0.5, 0.1, 0.1)
    elif kind == "rmat16_dense":
        off, edg = O.rmat(16, 64 << 16, 9, 0.57, 0.19, 0.19)
    elif kind == "torus40":
        off, edg = O.torus3d(40, 2)
    else:
        off, edg = O.randlocal(1 << 16, 5, 256, 4)
    dg = pb.DeviceGraph.upload(off, edg)
    check_graph(dg, off, edg)
    check_graph(dg, off, edg)  # a second call on the same handle starts clean
    dg.close()


def test_unsorted_lists_and_directed_graph(cuda_device):
    """Lists in any order (the walk cannot stop at the first larger
    neighbour) and a directed graph with self loops and repeated edges."""
    off, edg = O.rmat(14, 12 << 14, 4, 0.57, 0.19, 0.19)
    rng = np.random.default_rng(3)
    shuffled = edg.copy()
    for v in range(len(off) - 1):
        rng.shuffle(shuffled[off[v]:off[v + 1]])
    dg = pb.DeviceGraph.upload(off, shuffled)
    check_graph(dg, off, shuffled)
    dg.close()
    n, m = 20000, 90000
    us = rng.integers(0, n, m).astype(np.uint32)
    vs = rng.integers(0, n, m).astype(np.uint32)
    us = np.concatenate([us, np.arange(0, n, 97, dtype=np.uint32)])  # self loops
    vs = np.concatenate([vs, np.arange(0, n, 97, dtype=np.uint32)])
    order = np.lexsort((vs, us))
    us, vs = us[order], vs[order]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, us.astype(np.int64) + 1, 1)
    off = np.cumsum(off).astype(np.uint32)
    dg = pb.DeviceGraph.upload(off, vs.copy(), symmetric=False)
    check_graph(dg, off, vs, symmetric=False)
    dg.close()


def test_edge_cases(cuda_device):
    # one vertex, no edges; isolated vertices; a star; a path in id order (the
    # longest chain of waits) and the same path relabelled at random
    for n, pairs in [(1, []), (7, [(2, 3)]), (5000, [(0, i) for i in range(1, 5000)]),
                     (3000, [(i, i + 1) for i in range(2999)])]:
        if pairs:
            us = np.array([p[0] for p in pairs], np.uint32)
            vs = np.array([p[1] for p in pairs], np.uint32)
            off, edg = O.csr_symmetric(n, us, vs)
        else:
            off, edg = np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32)
        dg = pb.DeviceGraph.upload(off, edg)
        check_graph(dg, off, edg)
        dg.close()
    n = 50000
    perm = O.random_permutation(n, 5)
    us = perm[np.arange(n - 1)]
    vs = perm[np.arange(1, n)]
    off, edg = O.csr_symmetric(n, us, vs)
    dg = pb.DeviceGraph.upload(off, edg)
    check_graph(dg, off, edg)
    dg.close()


@pytest.mark.parametrize("cfg", ["rmat20", "torus160", "rmat24"])
def test_benchmark_graphs_full_size(cuda_device, cfg):
    if cfg == "rmat20":
        dg = pb.rmat_graph(20, 10 << 20, 1, 0.5, 0.1, 0.1)
    elif cfg == "torus160":
        dg = pb.torus3d_graph(160, perm_seed=2)
    else:
        dg = pb.rmat_graph(24, 1 << 28, 3, 0.57, 0.19, 0.19)
    off, edg = dg.download()
    check_graph(dg, off, edg)
    dg.close()


def test_round_trace(cuda_device):
    """The per-round trace: round 0 walks every vertex, each later round
    walks the vertices left undecided by the one before (never more), one
    entry per round, and the rounds' times add up to the kernel's."""
    off, edg = O.rmat(16, 10 << 16, 3, 0.5, 0.1, 0.1)
    dg = pb.DeviceGraph.upload(off, edg)
    _, st = check_graph(dg, off, edg)
    tr = dg.mis_trace()
    assert len(tr) == st["rounds"] and tr[0]["frontier"] == dg.n
    walked = [t["frontier"] for t in tr]
    assert all(b <= a for a, b in zip(walked, walked[1:])) and walked[-1] >= 1
    assert all(t["ms"] >= 0 for t in tr)
    assert sum(t["ms"] for t in tr) <= st["kernel_ms"] + 1e-3
    dg.close()


def test_bfs_statistics_survive_an_mis_call(cuda_device):
    """A search's statistics stay readable after an MIS call on the same
    handle (each keeps its own control block)."""
    import torch

    off, edg = O.rmat(14, 10 << 14, 2, 0.5, 0.1, 0.1)
    dg = pb.DeviceGraph.upload(off, edg)
    par = torch.empty(dg.n, dtype=torch.int32, device=cuda_device)
    flags = torch.empty(dg.n, dtype=torch.uint8, device=cuda_device)
    dg.bfs_device(0, par, None)
    dg.mis_device(flags)
    torch.cuda.synchronize()
    st = dg.last_stats()
    want = O.bfs_levels(off, edg, 0)
    reached = want != O.NONE
    assert st["visited"] == int(reached.sum()) and st["levels"] == int(want[reached].max()) + 1
    ms = dg.mis_stats()
    assert ms["in_set"] == int((O.mis_serial(off, edg) == 1).sum())
    dg.close()


def test_device_buffers_and_python_entry_point(cuda_device):
    import torch

    off, edg = O.torus3d(20, 4)
    dg = pb.DeviceGraph.upload(off, edg)
    d = torch.full((dg.n,), 9, dtype=torch.uint8, device=cuda_device)
    s = torch.cuda.Stream()
    dg.mis_device(d, stream=s.cuda_stream)
    s.synchronize()
    st = dg.mis_stats()
    got = d.cpu().numpy()
    assert np.array_equal(got, O.mis_serial(off, edg)) and st["in_set"] == int((got == 1).sum())
    dg.close()
    G = pb.Graph(off, edg)
    assert np.array_equal(pb.maximalIndependentSet(G), O.mis_serial(off, edg))


DROPIN = os.path.join(os.path.dirname(O.__file__), "_ref", "MISTime_gpuMIS")
CHECKER = os.path.join(os.path.dirname(O.__file__), "_ref", "MISCheck")


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(CHECKER)), reason="drop-in driver not built")
def test_dropin_behind_reference_driver_and_checker(cuda_device, tmp_path):
    """The unmodified reference driver bench/MISTime.C linked with the drop-in
    gpuMIS/MIS.C reads an AdjacencyGraph file, runs warm-up + timed rounds and
    writes the flags; the reference's MISCheck accepts them, and they equal
    serialMIS's."""
    off, edg = O.rmat(14, 12 * (1 << 14), 1, 0.55, 0.125, 0.125)
    gfile, ofile = str(tmp_path / "g.adj"), str(tmp_path / "out.seq")
    O.write_adjacency_graph(gfile, off, edg)
    r = subprocess.run([DROPIN, "-r", "3", "-o", ofile, gfile], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stderr == "", r.stderr
    assert len([l for l in r.stdout.splitlines() if l.startswith("Parlay time: ")]) == 3
    c = subprocess.run([CHECKER, gfile, ofile], capture_output=True, text=True, timeout=120)
    assert c.returncode == 0 and c.stdout.strip() == "", c.stdout
    assert np.array_equal(O.read_sequence_int(ofile).astype(np.uint8), O.mis_serial(off, edg))
