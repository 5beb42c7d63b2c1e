"""The continuous-batching BFS service (pbg_server_*): every query's uint8
levels equal an independent sequential BFS from its source, whether it ran
alone or in a mix of queries on several resident graphs; checksums match the
oracle's restatement; admission respects the device-memory budget."""
import numpy as np
import pytest

import pbbsbench_b200 as pb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_graphs(k=4, base=10):
    hosts, devs = [], []
    for i in range(k):
        off, edg = O.rmat(base + i, 16 << (base + i), 10 + i, 0.57, 0.19, 0.19)
        hosts.append((off, edg))
        devs.append(pb.DeviceGraph.upload(off, edg))
    return hosts, devs


def nonisolated(off, rng, count):
    nz = np.nonzero(np.diff(off))[0]
    return [int(nz[i]) for i in rng.integers(0, len(nz), count)]


def test_checksum_matches_oracle(cuda_device):
    import torch

    rng = np.random.default_rng(0)
    for n in (1, 7, 8, 9, 1000, 4099):
        rows = rng.integers(0, 256, (3, n)).astype(np.uint8)
        d = torch.from_numpy(rows.reshape(-1).copy()).to(cuda_device)
        got = pb.levels_checksum_device(d, 3, n)
        assert [int(x) for x in got] == [O.levels_checksum(r) for r in rows]
        lv32 = rng.integers(0, 400, n).astype(np.uint32)
        lv32[::5] = O.NONE
        d32 = torch.from_numpy(lv32.view(np.int32)).to(cuda_device)
        assert pb.levels32_checksum_device(d32, n) == O.levels_checksum(O.u8_levels(lv32))


@pytest.mark.parametrize("width", [64, 256, "wide", "capped"])
def test_mix_equals_alone_and_oracle(cuda_device, width):
    """64-source jobs (one mask word); 256-source jobs (four words), whose
    launches hold jobs of 129..256 queries and smaller ones; and 64-source
    jobs with 200-query jobs (four words) on the two smaller graphs, which
    run in launches of their own width; and 64-source jobs in launches capped
    at one largest-graph job's worth of edges."""
    hosts, devs = make_graphs()
    rng = np.random.default_rng(5)
    queries = []
    for _ in range(300 if width in (64, "capped") else 700):
        g = int(rng.integers(0, len(hosts)))
        queries.append((g, nonisolated(hosts[g][0], rng, 1)[0]))
    if width == "capped":  # launches of at most one largest-graph job's worth of edges
        srv = pb.Server(devs, hbm_budget_bytes=256 << 20, max_sources=64, max_jobs=8, streams=3,
                        max_launch_edges=devs[-1].m)
    elif width == "wide":
        srv = pb.Server(devs, hbm_budget_bytes=1024 << 20, max_sources=64, max_jobs=8, streams=3,
                        wide_sources=200, wide_max_vertices=len(hosts[1][0]) - 1)
    else:
        srv = pb.Server(devs, hbm_budget_bytes=(256 if width == 64 else 1024) << 20, max_sources=width, max_jobs=8,
                        streams=3)
    # in the mix: everything submitted at once
    mix = [np.empty(len(hosts[g][0]) - 1, np.uint8) for g, _ in queries]
    ids = [srv.submit(g, s, mix[i]) for i, (g, s) in enumerate(queries)]
    srv.drain()
    res = {r["id"]: r for r in srv.poll(cap=1000)}
    assert len(res) == len(queries)
    st = srv.stats()
    assert st["completed"] == len(queries) and st["launches"] >= 1
    # alone: one query at a time, the server idle otherwise
    for i, (g, s) in enumerate(queries[:40]):
        alone = np.empty_like(mix[i])
        srv.submit(g, s, alone)
        srv.drain()
        (r,) = srv.poll(cap=4)
        assert r["status"] == 0
        assert np.array_equal(alone, mix[i]), "query %d differs alone vs in the mix" % i
        assert r["checksum"] == res[ids[i]]["checksum"]
    for i, (g, s) in enumerate(queries):
        off, edg = hosts[g]
        want = O.u8_levels(O.bfs_levels(off, edg, s))
        assert res[ids[i]]["status"] == 0
        assert np.array_equal(mix[i], want), "query %d" % i
        assert res[ids[i]]["checksum"] == O.levels_checksum(want)
    srv.close()
    for d in devs:
        d.close()


def test_open_loop_replay_and_concurrency(cuda_device):
    hosts, devs = make_graphs(k=3, base=12)
    rng = np.random.default_rng(9)
    count = 2000
    graph = rng.integers(0, 3, count).astype(np.uint32)
    src = np.array([nonisolated(hosts[g][0], rng, 1)[0] for g in graph], np.uint32)
    arrival = np.cumsum(rng.exponential(1e6 / 20000.0, count))  # 20k queries/s Poisson
    srv = pb.Server(devs, hbm_budget_bytes=1 << 30, max_sources=64, max_jobs=8, streams=4)
    srv.replay(graph, src, arrival)
    srv.drain()
    res = srv.poll(cap=count + 10)
    assert len(res) == count and all(r["status"] == 0 for r in res)
    lat = np.array([r["t_done_us"] - r["t_submit_us"] for r in res])
    assert np.all(lat > 0)
    want = {}
    for r in res:  # every query against the oracle through its checksum
        key = (r["graph"], r["src"])
        if key not in want:
            off, edg = hosts[r["graph"]]
            want[key] = O.levels_checksum(O.u8_levels(O.bfs_levels(off, edg, r["src"])))
        assert r["checksum"] == want[key]
    srv.close()
    for d in devs:
        d.close()


def test_budget_admission(cuda_device):
    hosts, devs = make_graphs(k=2, base=10)
    with pytest.raises(pb.PbgError, match="budget"):
        pb.Server(devs, hbm_budget_bytes=1 << 10)
    # exactly one job slot of 4 sources per graph fits
    one = sum(int(pb.MultiWorkspace.bytes_needed(d)) + 4 * d.n + 256 for d in devs)
    srv = pb.Server(devs, hbm_budget_bytes=one, max_sources=4, max_jobs=4, streams=2)
    assert srv.stats()["slots"] == 2
    rng = np.random.default_rng(2)
    outs = []
    for i in range(50):  # 50 queries through 2 slots of 4 sources: many launches
        g = i % 2
        s = nonisolated(hosts[g][0], rng, 1)[0]
        outs.append((g, s, np.empty(len(hosts[g][0]) - 1, np.uint8)))
        srv.submit(g, s, outs[-1][2])
    srv.drain()
    assert srv.stats()["launches"] >= 50 // (2 * 4)
    for g, s, lv in outs:
        off, edg = hosts[g]
        assert np.array_equal(lv, O.u8_levels(O.bfs_levels(off, edg, s)))
    srv.close()
    for d in devs:
        d.close()


def test_bad_submissions(cuda_device):
    hosts, devs = make_graphs(k=1, base=10)
    srv = pb.Server(devs, hbm_budget_bytes=256 << 20)
    with pytest.raises(pb.PbgError):
        srv.submit(1, 0)
    with pytest.raises(pb.PbgError):
        srv.submit(0, 1 << 20)
    srv.close()
    devs[0].close()


def test_budget_above_free_hbm_admits_what_fits(cuda_device):
    """Admission by free HBM: a budget far above the device's memory is
    clamped at create to the free memory less PBG_SERVER_HBM_RESERVE (and the
    launch slots' buffers).  With most of the device taken by another
    allocation, the server still starts, with fewer job slots than its
    per-graph cap, and its results stay exact."""
    import torch

    hosts, devs = make_graphs(k=2, base=18)
    streams, max_jobs = 4, 4
    srv = pb.Server(devs, hbm_budget_bytes=1 << 62, max_sources=64, max_jobs=max_jobs, streams=streams)
    st = srv.stats()
    launch_bytes = streams * 8 * 256 * max_jobs
    assert 0 < st["budget_bytes"] <= st["free_bytes"] - pb._capi.SERVER_HBM_RESERVE - launch_bytes
    assert st["slot_bytes"] <= st["budget_bytes"] and st["slots"] == 2 * streams * len(devs)
    srv.close()

    need = sum(int(pb.MultiWorkspace.bytes_needed(d)) + 64 * d.n + 256 for d in devs)
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    hog_bytes = free - pb._capi.SERVER_HBM_RESERVE - launch_bytes - (5 * need) // 2
    assert hog_bytes > 0
    hog = torch.empty(hog_bytes, dtype=torch.uint8, device=cuda_device)
    try:
        srv = pb.Server(devs, hbm_budget_bytes=1 << 62, max_sources=64, max_jobs=max_jobs, streams=streams)
        st = srv.stats()
        assert st["budget_bytes"] < 4 * need
        assert len(devs) <= st["slots"] < 2 * streams * len(devs)
        rng = np.random.default_rng(3)
        outs = []
        for i in range(300):
            g = i % 2
            s = nonisolated(hosts[g][0], rng, 1)[0]
            outs.append((g, s, np.empty(len(hosts[g][0]) - 1, np.uint8)))
            srv.submit(g, s, outs[-1][2])
        srv.drain()
        res = srv.poll(cap=400)
        assert len(res) == 300 and all(r["status"] == 0 for r in res)
        for g, s, lv in outs:
            off, edg = hosts[g]
            assert np.array_equal(lv, O.u8_levels(O.bfs_levels(off, edg, s)))
        srv.close()
    finally:
        del hog
        torch.cuda.empty_cache()
    for d in devs:
        d.close()
