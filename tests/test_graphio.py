"""Graph files: the AdjacencyGraph text reader and writer, sequenceInt output
and the binary CSR image.

The oracle's text restatement (oracle.parse_adjacency_graph) is pinned to
the reference's own reader (common/graphIO.h:191-215, compiled from its
sources in oracle/_ref) on the CPU; the device parser and formatter are then
checked against both, byte for byte where text is written.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

# Texts that exercise the delimiters of common/IO.h:41-50 (space, tab, LF,
# CR, NUL), leading and trailing delimiters and leading zeros.
VARIANTS = [
    b"AdjacencyGraph\n3\n4\n0\n2\n3\n1\n2\n0\n0\n",
    b"AdjacencyGraph\r\n3\r\n4\r\n0\r\n2\r\n3\r\n1\r\n2\r\n0\r\n0\r\n",
    b"  \n\tAdjacencyGraph 3 4 0 2 3 1 2 0 0",
    b"AdjacencyGraph\x003\x004\x000\x00002\x003\x001\x0002\x000\x000\x00\x00\n",
    b"AdjacencyGraph\t\t3\t4\n\n\n0 \r 2\t3\n1 2 0 00000000000000000000\n   ",
]
EXPECTED = (np.array([0, 2, 3, 4], np.uint32), np.array([1, 2, 0, 0], np.uint32))

BAD = [
    (b"AdjacencyGrap\n1\n0\n0\n", "missing header"),
    (b"WeightedAdjacencyGraph\n1\n0\n0\n", "missing header"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n", "length = 5 n+m+3 = 6"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n1\n0\n", "length = 7 n+m+3 = 6"),
    (b"AdjacencyGraph\n2\n1\n0\n1x\n1\n", "not an unsigned decimal"),
    (b"AdjacencyGraph\n2\n1\n0\n-1\n1\n", "not an unsigned decimal"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n4294967296\n", "32 bits"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n12345678901\n", "32 bits"),
    (b"AdjacencyGraph\n2\n1\n1\n1\n0\n", "offsets[0] must be 0"),
    (b"AdjacencyGraph\n3\n2\n0\n2\n1\n1\n0\n", "non-decreasing"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n2\n", "edge target"),
    (b"AdjacencyGraph\n0\n0\n", "n must be"),
    (b"AdjacencyGraph\nx\n0\n", "not a count"),
    (b"AdjacencyGraph\n5\n", "has no value 2"),
    (b"", "no AdjacencyGraph header"),
]


def _ref_or_skip():
    if not O.ref_available():
        pytest.skip("reference library not built (make -C oracle ref)")


# ------------------------------------------------------------------ CPU


def test_oracle_parser_matches_reference_reader(tmp_path):
    _ref_or_skip()
    for i, text in enumerate(VARIANTS):
        p = tmp_path / ("v%d.adj" % i)
        p.write_bytes(text)
        off, edg = O.parse_adjacency_graph(text)
        r_off, r_edg = O.ref_read_graph(str(p))
        assert np.array_equal(off, EXPECTED[0]) and np.array_equal(edg, EXPECTED[1])
        assert np.array_equal(off, r_off) and np.array_equal(edg, r_edg)


def test_oracle_writer_is_read_back_by_reference(tmp_path):
    _ref_or_skip()
    off, edg = O.rmat(10, 8 * 1024, 5, 0.5, 0.1, 0.1)
    p = str(tmp_path / "g.adj")
    O.write_adjacency_graph(p, off, edg)
    r_off, r_edg = O.ref_read_graph(p)
    assert np.array_equal(off, r_off) and np.array_equal(edg, r_edg)
    assert np.array_equal(O.parse_adjacency_graph(open(p, "rb").read())[1], edg)


def test_oracle_parser_rejects_what_the_reference_rejects():
    for text, _ in BAD[:8]:
        with pytest.raises(ValueError):
            O.parse_adjacency_graph(text)


def test_oracle_sequence_int_round_trip(tmp_path):
    v = np.array([0, -1, 7, 2147483647, -2147483648, 10, 99, 100], np.int32)
    p = str(tmp_path / "s.txt")
    O.write_sequence_int(p, v)
    assert np.array_equal(O.read_sequence_int(p), v)


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
def test_parse_variants_match_oracle():
    import pbbsbench_b200 as pb

    for text in VARIANTS:
        g = pb.DeviceGraph.parse_adjacency(text)
        off, edg = g.download()
        assert np.array_equal(off, EXPECTED[0]) and np.array_equal(edg, EXPECTED[1]), text
        g.close()


@pytest.mark.gpu
def test_parse_errors_report():
    import pbbsbench_b200 as pb

    for text, msg in BAD:
        with pytest.raises(pb.PbgError) as ei:
            pb.DeviceGraph.parse_adjacency(text)
        assert msg in str(ei.value), (text, str(ei.value))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["rmat", "torus", "randlocal"])
def test_write_adjacency_is_byte_identical_to_oracle(tmp_path, kind):
    import pbbsbench_b200 as pb

    g = {"rmat": lambda: pb.rmat_graph(12, 10 * 4096, 1, 0.5, 0.1, 0.1),
         "torus": lambda: pb.torus3d_graph(12, 2),
         "randlocal": lambda: pb.randlocal_graph(5000, 5, 300, 4)}[kind]()
    off, edg = g.download()
    mine, want = str(tmp_path / "gpu.adj"), str(tmp_path / "oracle.adj")
    g.write_adjacency(mine)
    O.write_adjacency_graph(want, off, edg)
    assert open(mine, "rb").read() == open(want, "rb").read()
    # read back by the device parser and, where built, by the reference
    h = pb.DeviceGraph.load_adjacency(mine)
    off2, edg2 = h.download()
    assert np.array_equal(off2, off) and np.array_equal(edg2, edg)
    flags = ctypes.c_uint32()
    pb.check(pb.lib().pbg_graph_flags(h.handle, ctypes.byref(flags)))
    assert flags.value & pb._capi.GRAPH_SYMMETRIC  # detected on the device
    if O.ref_available():
        r_off, r_edg = O.ref_read_graph(mine)
        assert np.array_equal(r_off, off) and np.array_equal(r_edg, edg)
    h.close()
    g.close()


@pytest.mark.gpu
def test_load_spans_several_staging_pieces(tmp_path):
    """A text file of about 170 MB: more than two 64 MiB pinned pieces."""
    import pbbsbench_b200 as pb

    g = pb.rmat_graph(20, 10 << 20, 1, 0.5, 0.1, 0.1)
    p = str(tmp_path / "big.adj")
    g.write_adjacency(p)
    assert os.path.getsize(p) > 2 * (64 << 20)
    h = pb.DeviceGraph.load_adjacency(p, symmetric=True)
    a, b = g.download(), h.download()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    # the search on the loaded graph is the search on the original
    pa, la, _ = g.bfs(0, parent_mode=pb.PARENT_MIN, levels=True)
    pb_, lb, _ = h.bfs(0, parent_mode=pb.PARENT_MIN, levels=True)
    assert np.array_equal(pa, pb_) and np.array_equal(la, lb)
    h.close()
    g.close()


@pytest.mark.gpu
def test_binary_round_trip_and_checks(tmp_path):
    import pbbsbench_b200 as pb

    g = pb.rmat_graph(13, 16 * 8192, 3, 0.57, 0.19, 0.19)
    p = str(tmp_path / "g.bin")
    g.save_binary(p)
    off, edg = g.download()
    assert os.path.getsize(p) == 32 + 4 * (len(off) + len(edg))
    h = pb.DeviceGraph.load_binary(p)
    a, b = h.download()
    assert np.array_equal(a, off) and np.array_equal(b, edg)
    flags = ctypes.c_uint32()
    pb.check(pb.lib().pbg_graph_flags(h.handle, ctypes.byref(flags)))
    assert flags.value & pb._capi.GRAPH_SYMMETRIC  # kept from the file
    h.close()
    raw = open(p, "rb").read()
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(b"XXXXXXXX" + raw[8:])
    with pytest.raises(pb.PbgError, match="bad magic"):
        pb.DeviceGraph.load_binary(bad)
    open(bad, "wb").write(raw[:-4])
    with pytest.raises(pb.PbgError, match="size does not match"):
        pb.DeviceGraph.load_binary(bad)
    # a corrupted edge is caught by the validation every upload runs
    arr = bytearray(raw)
    arr[-4:] = (0xFFFFFFFF).to_bytes(4, "little")
    open(bad, "wb").write(bytes(arr))
    with pytest.raises(pb.PbgError, match="edge target"):
        pb.DeviceGraph.load_binary(bad)
    g.close()


@pytest.mark.gpu
def test_write_int_sequence_matches_oracle(tmp_path):
    import pbbsbench_b200 as pb

    rng = np.random.default_rng(7)
    v = np.concatenate([np.array([0, -1, 9, 10, 99, 100, 999999999, 1000000000, 2147483647, -2147483648,
                                  -10, -9], np.int32),
                        rng.integers(-2**31, 2**31, 100000, dtype=np.int64).astype(np.int32)])
    mine, want = str(tmp_path / "gpu.txt"), str(tmp_path / "oracle.txt")
    pb.write_int_sequence(mine, v)
    O.write_sequence_int(want, v)
    assert open(mine, "rb").read() == open(want, "rb").read()
    assert np.array_equal(O.read_sequence_int(mine), v)
    empty = str(tmp_path / "empty.txt")
    pb.write_int_sequence(empty, np.zeros(0, np.int32))
    assert open(empty, "rb").read() == b"sequenceInt\n"


@pytest.mark.gpu
def test_graph_without_edges(tmp_path):
    """m = 0: n offsets, all 0, and no edge tokens."""
    import pbbsbench_b200 as pb

    text = b"AdjacencyGraph\n3\n0\n0\n0\n0\n"
    off, edg = O.parse_adjacency_graph(text)
    g = pb.DeviceGraph.parse_adjacency(text)
    a, b = g.download()
    assert np.array_equal(a, off) and len(b) == 0 and list(a) == [0, 0, 0, 0]
    par, lv, _ = g.bfs(1, levels=True)
    assert list(par) == [-1, 1, -1]
    p = str(tmp_path / "e.adj")
    g.write_adjacency(p)
    assert open(p, "rb").read() == text
    g.close()


CHECKER = os.path.join(os.path.dirname(O.__file__), "_ref", "BFSCheck")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CHECKER), reason="reference checker not built (make -C oracle ref)")
def test_files_written_on_the_device_pass_the_reference_checker(tmp_path):
    """The whole file round trip of the driver, with every file written on the
    device: the graph (pbg_graph_write_adj) and the BFS parents
    (pbg_write_seq_int) are read by the reference's own BFSCheck binary
    (bench/BFSCheck.C), which accepts them."""
    import subprocess

    import pbbsbench_b200 as pb

    g = pb.rmat_graph(15, 12 << 15, 4, 0.55, 0.125, 0.125)
    gfile, pfile = str(tmp_path / "g.adj"), str(tmp_path / "p.seq")
    g.write_adjacency(gfile)
    h = pb.DeviceGraph.load_adjacency(gfile)
    par, _, _ = h.bfs(0)
    pb.write_int_sequence(pfile, par)
    c = subprocess.run([CHECKER, gfile, pfile], capture_output=True, text=True, timeout=120)
    assert c.returncode == 0 and c.stdout.strip() == "", c.stdout
    h.close()
    g.close()
