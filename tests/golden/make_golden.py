"""Generates tests/golden/bfs_golden.npz from the reference's OWN BFS code.

Run here (where the reference sources are present) after `make -C oracle ref`:
    python tests/golden/make_golden.py

For each small input graph it stores the CSR, the sources, and what the
reference computes on it:
  * serialBFS parents        (benchmarks/breadthFirstSearch/serialBFS/BFS.C:32-55)
  * deterministicBFS parents (deterministicBFS/BFS.C:39-78, max-parent rule)
  * level_number levels      (bench/BFSCheck.C:39-56; n = unreached)
  * checkBFS verdicts        (bench/BFSCheck.C:59-90) on backForwardBFS and simpleBFS
The CSR inputs come from the oracle's seeded generators (our construction of
the reference's generator rules) plus hand-made edge cases.  The fixture pins
oracle/bfs_oracle.c on machines without the reference (tests/test_oracle.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def csr_from_pairs(n, pairs, symmetric=True):
    us = np.array([p[0] for p in pairs], np.uint32)
    vs = np.array([p[1] for p in pairs], np.uint32)
    if symmetric:
        return O.csr_symmetric(n, us, vs)
    order = np.lexsort((vs, us))
    us, vs = us[order], vs[order]
    off = np.zeros(n + 1, np.uint32)
    np.add.at(off, us.astype(np.int64) + 1, 1)
    return np.cumsum(off, dtype=np.uint64).astype(np.uint32), vs


def cases():
    out = []
    off, edg = O.rmat(10, 10 * 1024, 1, 0.5, 0.1, 0.1)
    out.append(("rmat10_s1", off, edg, [0, 1, 17, 1000]))
    off, edg = O.rmat(12, 16 * 4096, 3, 0.57, 0.19, 0.19)
    out.append(("rmat12_s3", off, edg, [0, 2, 99, 4000]))
    off, edg = O.torus3d(8, 2)
    out.append(("torus8_perm2", off, edg, [0, 311]))
    off, edg = O.torus3d(5, None)
    out.append(("torus5", off, edg, [0, 62]))
    off, edg = O.randlocal(2048, 5, 64, 4)
    out.append(("randlocal2048", off, edg, [0, 1500]))
    n = 64
    off, edg = csr_from_pairs(n, [(i, i + 1) for i in range(n - 1)])
    out.append(("path64", off, edg, [0, 31, 63]))
    n = 6000
    off, edg = csr_from_pairs(n, [(0, i) for i in range(1, n)])
    out.append(("star6000", off, edg, [0, 5]))
    n = 40
    pairs = [(i, i + 1) for i in range(0, 19)] + [(i, i + 1) for i in range(20, 39)] + [(3, 3), (5, 6), (6, 5)]
    off, edg = csr_from_pairs(n, pairs)
    out.append(("two_components_selfloop", off, edg, [0, 25]))
    n = 10
    off, edg = csr_from_pairs(n, [(1, 2), (2, 3)])
    out.append(("isolated_source", off, edg, [0, 9, 1]))
    return out


def main():
    blobs = {}
    names = []
    for name, off, edg, srcs in cases():
        names.append(name)
        G = O.RefGraph(off, edg)
        n = len(off) - 1
        serial = np.stack([G.bfs(s, O.REF_SERIAL) for s in srcs])
        det = np.stack([G.bfs(s, O.REF_DETERMINISTIC) for s in srcs])
        levels = np.stack([O.ref_level_number(p) for p in serial])
        verdict_bf = np.array([G.check(s, G.bfs(s, O.REF_BACKFORWARD)) for s in srcs], np.int32)
        verdict_simple = np.array([G.check(s, G.bfs(s, O.REF_SIMPLE)) for s in srcs], np.int32)
        blobs[name + "/offsets"] = off
        blobs[name + "/edges"] = edg
        blobs[name + "/srcs"] = np.array(srcs, np.uint32)
        blobs[name + "/serial_parent"] = serial
        blobs[name + "/det_max_parent"] = det
        blobs[name + "/levels"] = levels
        blobs[name + "/check_backforward"] = verdict_bf
        blobs[name + "/check_simple"] = verdict_simple
        G.close()
        print("%-26s n=%6d m=%7d sources=%s" % (name, n, len(edg), srcs))
    blobs["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "bfs_golden.npz"), **blobs)


if __name__ == "__main__":
    main()
