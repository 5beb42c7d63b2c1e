"""The autotuner (pbg_autotune): its picks come from the candidate sets, the
tuned configuration is never slower than the defaults on the samples it was
tuned on, and searches under tuned options keep exact results."""
import numpy as np
import pytest

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _graph():
    off, edg = O.rmat(16, 16 << 16, 10, 0.57, 0.19, 0.19)
    nz = np.nonzero(np.diff(off))[0]
    srcs = nz[np.random.default_rng(7).integers(0, len(nz), 8)].astype(np.uint32)
    return off, edg, srcs


def test_single_source_tuning(cuda_device):
    off, edg, srcs = _graph()
    dg = pb.DeviceGraph.upload(off, edg)
    opts, rep = dg.autotune(srcs[:4])
    assert opts["block_threads"] in (256, 512, 1024)
    assert opts["chunk_min_degree"] in (16, 32, 64, 128, 256)
    assert opts["alpha"] in (5, 10, 20, 40) and opts["beta"] in (5, 10, 20, 40)
    assert rep["evaluations"] >= 1 and rep["best_ms"] <= rep["default_ms"]
    want = O.levels_u8(off, edg, srcs)
    for i, s in enumerate(srcs):
        par, lv, st = dg.bfs(int(s), levels=True)  # runs on the tuned options
        assert np.array_equal(np.where(lv == pb.NONE, 255, lv).astype(np.uint8), want[i])
        assert O.check_bfs(off, edg, int(s), par) == -1
    dg.clear_tuning()
    dg.close()


def test_batched_tuning(cuda_device):
    off, edg, srcs = _graph()
    dg = pb.DeviceGraph.upload(off, edg)
    allsrc = np.concatenate([srcs, srcs + 1]).astype(np.uint32) % dg.n
    opts, rep = dg.autotune(allsrc, batched=True)
    assert opts["alpha"] in (2, 5, 10, 20, 40, 80)
    assert rep["best_ms"] <= rep["default_ms"]
    lv, st = dg.bfs_multi(allsrc)
    assert np.array_equal(lv, O.levels_u8(off, edg, allsrc))
    dg.close()


@pytest.mark.parametrize("k", [128, 256])
def test_batched_tuning_wide_masks(cuda_device, k):
    """Batched samples of 65..256 sources need two or four mask words: tuning
    replaces the graph's one-word workspace with one of the sample's width,
    and the searches that follow stay bit-exact against the oracle."""
    off, edg, _ = _graph()
    dg = pb.DeviceGraph.upload(off, edg)
    nz = np.nonzero(np.diff(off))[0]
    allsrc = nz[np.random.default_rng(k).integers(0, len(nz), k)].astype(np.uint32)
    opts, rep = dg.autotune(allsrc, batched=True)
    assert opts["alpha"] in (2, 5, 10, 20, 40, 80)
    assert rep["best_ms"] <= rep["default_ms"]
    lv, st = dg.bfs_multi(allsrc)
    assert np.array_equal(lv, O.levels_u8(off, edg, allsrc))
    lv64, _ = dg.bfs_multi(allsrc[:64])
    assert np.array_equal(lv64, O.levels_u8(off, edg, allsrc[:64]))
    dg.close()


def test_tuning_arguments(cuda_device):
    off, edg, srcs = _graph()
    dg = pb.DeviceGraph.upload(off, edg)
    with pytest.raises(pb.PbgError):
        dg.autotune(np.zeros(0, np.uint32))
    with pytest.raises(pb.PbgError):
        dg.autotune(np.zeros(17, np.uint32))
    with pytest.raises(pb.PbgError):
        dg.autotune(np.zeros(257, np.uint32), batched=True)
    with pytest.raises(pb.PbgError):
        dg.autotune([dg.n])
    dg.close()
