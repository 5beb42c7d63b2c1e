"""Generates tests/golden/mis_golden.npz from the reference's OWN maximal
independent set code.

Run here (where the reference sources are present) after `make -C oracle ref`:
    python tests/golden/make_mis_golden.py

For each small input graph it stores the CSR and what the reference computes
on it:
  * serialMIS flags  (benchmarks/maximalIndependentSet/serialMIS/MIS.C:33-47;
                      1 in the set, 2 not)
  * the MISCheck verdict (bench/MISCheck.C:39-79, run as its own binary) on
    ndMIS's flags (ndMIS/MIS.C:41-80, nondeterministic), on the symmetric
    graphs without self loops only: ndMIS retries forever on a vertex with a
    self loop (it holds its own lock and then fails to take it again as a
    neighbour's), so the directed case stores -1 there
The CSR inputs come from the oracle's seeded generators plus hand-made edge
cases: a directed graph with self loops and repeated edges (serialMIS reads
out-edges only and puts a vertex with a self loop out of the set), a path, a
star and isolated vertices.  The fixture pins oracle/bfs_oracle.c's MIS
restatement on machines without the reference (tests/test_oracle.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import oracle as O  # noqa: E402
from make_golden import csr_from_pairs  # noqa: E402


def cases():
    out = []
    out.append(("rmat10_s1",) + tuple(O.rmat(10, 10 * 1024, 1, 0.5, 0.1, 0.1)))
    out.append(("rmat12_s3",) + tuple(O.rmat(12, 16 * 4096, 3, 0.57, 0.19, 0.19)))
    out.append(("torus8_perm2",) + tuple(O.torus3d(8, 2)))
    out.append(("randlocal2048",) + tuple(O.randlocal(2048, 5, 64, 4)))
    out.append(("path64",) + tuple(csr_from_pairs(64, [(i, i + 1) for i in range(63)])))
    out.append(("star3000",) + tuple(csr_from_pairs(3000, [(0, i) for i in range(1, 3000)])))
    out.append(("isolated10",) + tuple(csr_from_pairs(10, [(1, 2), (2, 3), (7, 8)])))
    rng = np.random.default_rng(12)
    n, m = 500, 2500
    pairs = [(int(a), int(b)) for a, b in zip(rng.integers(0, n, m), rng.integers(0, n, m))]
    pairs += [(5, 5), (9, 9), (40, 41), (40, 41)]
    out.append(("directed_selfloops",) + tuple(csr_from_pairs(n, pairs, symmetric=False)))
    return out


def main():
    blobs = {}
    names = []
    for name, off, edg in cases():
        names.append(name)
        G = O.RefMisGraph(off, edg)
        serial = G.mis(O.REF_SERIAL_MIS)
        verdict = -1
        if not name.startswith("directed"):
            verdict = O.ref_check_mis(off, edg, G.mis(O.REF_ND_MIS))
        G.close()
        blobs[name + "/offsets"] = off
        blobs[name + "/edges"] = edg
        blobs[name + "/serial_flags"] = serial
        blobs[name + "/check_nd"] = np.array([verdict], np.int32)
        print("%-22s n=%6d m=%7d in set %d" % (name, len(off) - 1, len(edg), int((serial == 1).sum())))
    blobs["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "mis_golden.npz"), **blobs)


if __name__ == "__main__":
    main()
