"""The CPU oracle, pinned: against the committed golden vectors (outputs of
the reference's own BFS code) and, where the reference library is built,
against the reference run live.  No GPU."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "bfs_golden.npz")


def golden_cases():
    z = np.load(GOLDEN)
    for name in z["names"]:
        name = str(name)
        yield name, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name,case", list(golden_cases()))
def test_oracle_matches_golden(name, case):
    off, edg = case["offsets"], case["edges"]
    n = len(off) - 1
    for i, s in enumerate(case["srcs"]):
        s = int(s)
        # serialBFS parents bit-exact (serialBFS/BFS.C:32-55)
        assert np.array_equal(O.bfs_serial(off, edg, s), case["serial_parent"][i].view(np.uint32))
        # deterministicBFS = max-parent rule (deterministicBFS/BFS.C:60-74)
        assert np.array_equal(O.bfs_det_parent(off, edg, s, "max"), case["det_max_parent"][i].view(np.uint32))
        # level_number (BFSCheck.C:39-56), n = unreached
        lv = O.level_number(case["serial_parent"][i].view(np.uint32))
        assert np.array_equal(lv, case["levels"][i].view(np.uint32))
        # direct BFS distances agree with level_number
        d = O.bfs_levels(off, edg, s)
        ref_lv = case["levels"][i].astype(np.int64)
        assert np.array_equal(np.where(d == O.NONE, n, d).astype(np.int64), ref_lv)
        # the reference checker accepted backForwardBFS and simpleBFS outputs
        assert case["check_backforward"][i] == 0 and case["check_simple"][i] == 0
        # and the strengthened oracle check accepts the serial tree
        assert O.check_bfs(off, edg, s, case["serial_parent"][i].view(np.uint32)) == -1


def test_check_rejects_planted_errors():
    """Mistakes planted in oracle outputs, on the CPU: the checker finds them."""
    off, edg = O.rmat(10, 10 * 1024, 1, 0.5, 0.1, 0.1)
    p = O.bfs_serial(off, edg, 0)
    assert O.check_bfs(off, edg, 0, p) == -1
    lv = O.bfs_levels(off, edg, 0)
    # a parent two levels up: level predicate fails
    v = int(np.where(lv == 3)[0][0])
    bad = p.copy()
    bad[v] = 0
    assert O.check_bfs(off, edg, 0, bad) >= 0
    # a parent at the right level but not adjacent: only the edge test catches it
    lvl2 = np.where(lv == 2)[0]
    nbrs = set(edg[off[v]:off[v + 1]].tolist())
    cand = [int(u) for u in lvl2 if int(u) not in nbrs]
    bad = p.copy()
    bad[v] = cand[0]
    assert O.check_bfs(off, edg, 0, bad, check_edges=False) == -1
    assert O.check_bfs(off, edg, 0, bad, check_edges=True) == v
    # an unreached vertex marked visited
    iso = np.where(np.diff(off) == 0)[0]
    if len(iso):
        bad = p.copy()
        bad[int(iso[0])] = 0
        assert O.check_bfs(off, edg, 0, bad) >= 0
    # a parent cycle
    bad = p.copy()
    a, b = [int(x) for x in np.where(lv == 2)[0][:2]]
    bad[a], bad[b] = b, a
    assert O.check_bfs(off, edg, 0, bad) >= 0
    # wrong root
    bad = p.copy()
    bad[0] = O.NONE
    assert O.check_bfs(off, edg, 0, bad) >= 0


def test_generators_follow_construction_rules():
    for off, edg in [O.rmat(11, 20000, 7, 0.57, 0.19, 0.19), O.torus3d(6, 2), O.randlocal(3000, 5, 100, 4)]:
        n = len(off) - 1
        assert off[0] == 0 and off[-1] == len(edg)
        assert np.all(np.diff(off.astype(np.int64)) >= 0)
        u = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off))
        assert not np.any(u == edg)                       # no self loops
        key = u.astype(np.uint64) << 32 | edg
        assert np.all(np.diff(key.astype(np.int64)) > 0)  # sorted, no duplicates
        rev = np.sort(edg.astype(np.uint64) << 32 | u)
        assert np.array_equal(rev, key)                   # symmetric
    off, _ = O.torus3d(6, 2)
    assert np.all(np.diff(off) == 6)
    perm = O.random_permutation(1000, 2)
    assert np.array_equal(np.sort(perm), np.arange(1000, dtype=np.uint32))


def test_levels_u8():
    off, edg = O.torus3d(5, None)
    srcs = [0, 7, 100]
    lv = O.levels_u8(off, edg, srcs)
    for i, s in enumerate(srcs):
        d = O.bfs_levels(off, edg, s)
        assert np.array_equal(lv[i], np.where(d == O.NONE, 255, d).astype(np.uint8))


def test_levels_u8_boundary():
    """uint8 level rows hold levels 0..254 (255 = unreached); a search that
    reaches level 255 overflows, as the batched device search reports."""
    for n, fits in [(255, True), (256, False)]:
        off, edg = O.csr_symmetric(n, np.arange(n - 1, dtype=np.uint32), np.arange(1, n, dtype=np.uint32))
        if fits:
            lv = O.levels_u8(off, edg, [0])
            assert lv[0, -1] == 254 and np.array_equal(lv[0], np.arange(n, dtype=np.uint8))
        else:
            with pytest.raises(OverflowError):
                O.levels_u8(off, edg, [0])
            # from the middle the depth is 128: fits
            assert O.levels_u8(off, edg, [128]).max() == 128


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built (make -C oracle ref)")


@needs_ref
@pytest.mark.parametrize("logn,seed", [(12, 1), (13, 3)])
def test_oracle_vs_reference_live(logn, seed):
    off, edg = O.rmat(logn, 12 * (1 << logn), seed, 0.57, 0.19, 0.19)
    G = O.RefGraph(off, edg)
    for s in [0, 3, (1 << logn) - 1]:
        assert np.array_equal(G.bfs(s, O.REF_SERIAL).view(np.uint32), O.bfs_serial(off, edg, s))
        assert np.array_equal(G.bfs(s, O.REF_DETERMINISTIC).view(np.uint32), O.bfs_det_parent(off, edg, s, "max"))
        p = G.bfs(s, O.REF_BACKFORWARD).view(np.uint32)
        assert G.check(s, p) == 0 and O.check_bfs(off, edg, s, p) == -1
    G.close()


BIN = os.path.join(os.path.dirname(O.__file__), "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "BFSTime_serialBFS")), reason="reference binaries not built")
def test_reference_driver_and_checker_binaries():
    """The reference's own BFSTime driver and BFSCheck checker, on an
    AdjacencyGraph file written by the oracle."""
    off, edg = O.rmat(11, 10 * 2048, 1, 0.5, 0.1, 0.1)
    with tempfile.TemporaryDirectory() as d:
        gfile, ofile = os.path.join(d, "g.adj"), os.path.join(d, "out.seq")
        O.write_adjacency_graph(gfile, off, edg)
        r = subprocess.run([os.path.join(BIN, "BFSTime_serialBFS"), "-r", "1", "-o", ofile, gfile],
                           capture_output=True, text=True, check=True)
        assert "Parlay time" in r.stdout
        par = O.read_sequence_int(ofile).view(np.uint32)
        assert np.array_equal(par, O.bfs_serial(off, edg, 0))
        c = subprocess.run([os.path.join(BIN, "BFSCheck"), gfile, ofile], capture_output=True, text=True)
        assert c.returncode == 0 and c.stdout.strip() == ""
        bad = par.copy()
        lv = O.bfs_levels(off, edg, 0)
        bad[int(np.where(lv == 3)[0][0])] = 0
        with open(ofile, "w") as f:
            f.write("sequenceInt\n" + "\n".join(str(int(x)) for x in bad.view(np.int32)) + "\n")
        c = subprocess.run([os.path.join(BIN, "BFSCheck"), gfile, ofile], capture_output=True, text=True)
        assert c.returncode == 1 and "BFSCheck: failed" in c.stdout


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", [5, 6])
def test_oracle_vs_reference_live_directed(seed):
    """Directed graphs (no reverse edges; self loops and duplicates kept):
    serialBFS (serialBFS/BFS.C:32-55) and deterministicBFS
    (deterministicBFS/BFS.C:39-78) follow out-edges only, and the oracle's
    restatements agree with them bit for bit.  simpleBFS's parents form a
    BFS tree: the levels of its parent pointers are the oracle's distances
    and each parent has an out-edge to its child.  (The level check of
    bench/BFSCheck.C:39-90 reads out-edges as in-edges, so it holds on
    symmetric graphs only.)"""
    rng = np.random.default_rng(seed)
    n, m = 3000, 9000
    u = rng.integers(0, n, m)
    v = np.where(rng.random(m) < 0.7, (u + rng.integers(1, 40, m)) % n, rng.integers(0, n, m))
    order = np.lexsort((v, u))
    u, v = u[order], v[order]
    off = np.zeros(n + 1, np.uint32)
    np.add.at(off, u + 1, 1)
    off = np.cumsum(off).astype(np.uint32)
    edg = v.astype(np.uint32)
    G = O.RefGraph(off, edg)
    for s in [0, int(u[m // 2]), n - 1]:
        serial = G.bfs(s, O.REF_SERIAL).view(np.uint32)
        assert np.array_equal(serial, O.bfs_serial(off, edg, s))
        assert np.array_equal(G.bfs(s, O.REF_DETERMINISTIC).view(np.uint32), O.bfs_det_parent(off, edg, s, "max"))
        lv = O.bfs_levels(off, edg, s)
        assert np.array_equal(lv != O.NONE, serial != O.NONE)
        simple = G.bfs(s, O.REF_SIMPLE).view(np.uint32)
        assert np.array_equal(O.level_number(simple), np.where(lv == O.NONE, n, lv).astype(np.uint32))
        for w in np.nonzero((simple != O.NONE) & (np.arange(n) != s))[0]:
            p = simple[w]
            assert w in edg[off[p]:off[p + 1]]
    G.close()


# ------------------------------------------------------------------ MIS
MIS_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mis_golden.npz")


def mis_cases():
    z = np.load(MIS_GOLDEN)
    for name in z["names"]:
        name = str(name)
        yield name, {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name,case", list(mis_cases()))
def test_mis_oracle_matches_golden(name, case):
    """The restated serialMIS (serialMIS/MIS.C:33-47) equals the reference's
    own flags bit for bit; the restated checker (MISCheck.C:39-66) accepts
    them, and the reference's checker accepted ndMIS's set."""
    off, edg = case["offsets"], case["edges"]
    flags = O.mis_serial(off, edg)
    assert np.array_equal(flags, case["serial_flags"])
    if not name.startswith("directed"):  # an MIS (and its check) is defined on symmetric graphs
        assert O.check_mis(off, edg, flags) == -1
        assert int(case["check_nd"][0]) == 0


def test_mis_checker_catches_planted_faults():
    off, edg = O.rmat(11, 8 * 2048, 2, 0.5, 0.1, 0.1)
    flags = O.mis_serial(off, edg)
    v = int(np.nonzero(flags == 2)[0][0])
    nb = edg[off[v]:off[v + 1]]
    not_maximal = flags.copy()
    not_maximal[nb[flags[nb] == 1]] = 2  # v keeps no neighbour in the set
    assert O.check_mis(off, edg, not_maximal) != -1
    u = int(nb[flags[nb] == 1][0])
    not_independent = flags.copy()
    not_independent[v] = 1  # v and its neighbour u both in the set
    assert O.check_mis(off, edg, not_independent) == min(u, v)


@pytest.mark.skipif(not O.refmis_available(), reason="reference MIS library not built")
def test_mis_oracle_matches_reference_live():
    for off, edg in (O.rmat(16, 10 << 16, 5, 0.57, 0.19, 0.19), O.torus3d(30, 7), O.randlocal(60000, 4, 30, 3)):
        G = O.RefMisGraph(off, edg)
        assert np.array_equal(O.mis_serial(off, edg), G.mis(O.REF_SERIAL_MIS))
        G.close()
    # ndMIS (nondeterministic, and slow on the parlay shim: its lock-and-retry
    # loop spins around hubs) on a small graph: a valid set for both checkers
    off, edg = O.torus3d(10, 7)
    G = O.RefMisGraph(off, edg)
    nd = G.mis(O.REF_ND_MIS)
    G.close()
    assert O.check_mis(off, edg, nd) == -1
    assert O.ref_check_mis(off, edg, nd) == 0
