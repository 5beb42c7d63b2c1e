#!/usr/bin/env python3
"""Benchmark of the BFS hot path on B200.

Default run (no --workload): ONE JSON line.  Its headline (`value`) is the
direction-optimizing BFS on a symmetric rMat graph, n = 2^24 vertices, 2^28
edge draws, (a, b, c) = (.57, .19, .19), seed 3, deduplicated, uint32 CSR
resident in HBM; eight sources drawn uniformly (seed 3) from the vertices of
degree > 0.  Beside it, each with its own timed region and clock record:
    c1       plain BFS, rMat 2^20, 10n samples, (.5, .1, .1), seed 1, source 0
    c2       plain BFS, 3-D torus 160^3, ids permuted with seed 2, source 0
    batched  64 sources in one persistent launch (uint64 mask per vertex) on
             randLocal 2^23 (5 out-neighbours within +-2^16, seed 4), against
             64 back-to-back plain launches on the same GPU
    served   8 resident rMat graphs 2^16..2^23 (16n samples, seeds 10..17),
             100k queries (--queries), Poisson arrivals, continuous batching;
             p50/p99 latency, queries/s and back-to-back plain queries/s
(measured at N = 1; under torchrun only the headline runs, on every rank).

One headline step = one BFS from the next of the eight sources (first-claimer
parents, the semantics of backForwardBFS), with the library's default options
(with --autotune: the graph's options picked by pbg_autotune from four other
sources before any timing).  Between timed steps L2 is flushed by writing a
256 MiB buffer; each BFS is timed with CUDA events on its stream.

    value   GTEPS = sum over steps of (m_r / 2) / sum of device times
            (m_r = sum of degrees of the reached vertices, Graph500 style)
    e2e     the same metric through pbg_bfs() with host (pinned) output: the
            parent array (4n bytes) comes back to the host every step
    roofline  algorithmic bytes 4(n+1) + 4 m_r + 4n per BFS / device time,
            against MEASURED_PEAKS.json's HBM copy bandwidth

--impl reference runs the reference's own backForwardBFS (compiled from its
sources against the project parlay shim, oracle/_ref) on the host cores over
the same graph, with the same `config`.  Under torchrun every rank runs an
independent replica (BFS does not shard; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LOGN, SAMPLES, SEED = 24, 1 << 28, 3
A, B, C = 0.57, 0.19, 0.19
NSRC = 8
WORKLOAD = "rmat24_e28_dobfs"
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=24)
    p.add_argument("--warmup", type=int, default=4)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-rounds", type=int, default=0,
                   help="CPU baseline calls of the headline (0: the same --steps calls the reference arm makes)")
    p.add_argument("--logn", type=int, default=LOGN, help="smaller graphs for profiling captures")
    p.add_argument("--log-samples", type=int, default=28)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="default run: the headline only (no c1 / c2 / batched / served sub-objects)")
    p.add_argument("--trace", action="store_true", help="msbfs64/msbfs_rmat: per-level trace of a batch to stderr")
    p.add_argument("--block", type=int, default=0, help="CTA size of the persistent kernel (0 = tuned)")
    p.add_argument("--chunk", type=int, default=0, help="chunk_min_degree (0 = tuned)")
    p.add_argument("--autotune", action="store_true",
                   help="single-source workloads: first let the autotuner pick the graph's block size, chunk degree "
                        "and switch from 4 other sources (before any timing)")
    p.add_argument("--queries", type=int, default=100000, help="serve: number of queries")
    p.add_argument("--rate", type=float, default=0.0, help="serve: Poisson arrival rate (0 = 75%% of capacity)")
    p.add_argument("--max-jobs", type=int, default=16, help="serve: jobs per fused launch")
    p.add_argument("--streams", type=int, default=4, help="serve: launch slots (streams) on the GPU at once")
    p.add_argument("--serve-sources", type=int, default=64,
                   help="serve: queries per job (one source mask; 64 is the served configuration)")
    p.add_argument("--hbm-gb", type=int, default=48, help="serve: HBM budget for job slots, GiB")
    p.add_argument("--serve-max-launch-edges", type=int, default=1 << 29,
                   help="serve: a launch takes jobs while their graphs' edges add up to at most this (0: no limit)")
    p.add_argument("--serve-wide-sources", type=int, default=0,
                   help="serve: queries per job on the small graphs (0: off; see --serve-wide-max-logn)")
    p.add_argument("--serve-wide-max-logn", type=int, default=20,
                   help="serve: graphs of at most 2^this vertices take the wide jobs")
    p.add_argument("--sources", type=int, default=64,
                   help="msbfs64/msbfs_rmat: sources per batched job (1..256; above 64 the masks take two "
                        "words, above 128 four)")
    p.add_argument("--workload", default="all",
                   choices=["all", "rmat24", "rmat20", "torus160", "msbfs64", "msbfs_rmat", "serve", "io", "mis",
                            "check", "build"],
                   help="all (default): the headline rmat24 line with the c1, c2, batched and served "
                        "sub-objects; rmat24: the headline alone; rmat20 / torus160: the other single-source "
                        "graphs; msbfs64: --sources (64) sources batched on randLocal 2^logn (23 unless --logn); "
                        "msbfs_rmat: the same on the served rMat graph of n = 2^logn (23 unless --logn); serve: "
                        "the served request stream; io: AdjacencyGraph text file -> resident CSR; mis: maximal "
                        "independent set on the rMat graph of the headline (2^logn, 2^log_samples draws); "
                        "check: the device BFS check (pbg_bfs_check) of the headline searches' parents; "
                        "build: device construction of the headline graph into a resident CSR")
    return p.parse_args()


def pick_sources(deg: np.ndarray, k: int = NSRC, seed: int = SEED) -> list[int]:
    nz = np.nonzero(deg)[0]
    rng = np.random.default_rng(seed)
    return [int(nz[i]) for i in rng.integers(0, len(nz), k)]


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the CPU-baseline lines."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def traffic_per_launch():
    """dram bytes per BFS launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "bfs_persistent_rmat24_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """SM clocks and throttle reasons during the timed region: NVML read every
    2 ms from a background thread (one sample on entry and one on exit, so a
    timed region of a few milliseconds still has samples), the GPU found by
    the PCI bus id of the CUDA device; nvidia-smi -lms 100 where NVML is
    unavailable.  Reads only; changes no setting."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.nv = None
        self.samples = []  # (sm MHz, max MHz, reason bits)

    def _bus_id(self) -> str:
        """PCI bus id of the CUDA device (CUDA ordinals need not match
        nvidia-smi's or NVML's indices, e.g. under CUDA_VISIBLE_DEVICES)."""
        import torch
        pr = torch.cuda.get_device_properties(self.index)
        return "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(self._bus_id())

    def _sample(self):
        nv, h = self.nv
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        try:
            rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(sm), float(mx), int(rs)))

    def _loop(self):
        while not self.stop.wait(0.002):
            try:
                self._sample()
            except Exception:
                return

    def __enter__(self):
        import threading
        try:
            self.nv = self._nvml_handle()
            self._sample()
            self.stop = threading.Event()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nv = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", self._bus_id(), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.nv:
            self.stop.set()
            self.t.join(timeout=1)
            try:
                self._sample()
            except Exception:
                pass
            return
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for c, m, bits in self.samples:
            sm.append(c)
            mx = max(mx, m)
            reasons.update(nm for nm, b in self.BITS.items() if bits & b)
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    # NCCL reduces device tensors; gloo (the CPU tests of this plumbing) host ones
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def headline_config(n: int, m: int, sources, levels, world: int) -> dict:
    """The headline's `config`, identical in both arms (every value is a
    property of the graph, the sources and the search rule; run-specific
    figures such as build times live outside it)."""
    return {"workload": WORKLOAD, "n": n, "m_directed": m, "samples": SAMPLES, "abc": [A, B, C], "seed": SEED,
            "sources": list(sources), "levels": list(levels), "parent_rule": "first claimer (backForwardBFS)",
            "direction": "auto, alpha=beta=20 (ligraLight.h:122,130)",
            "l2": "inputs larger than L2 (2.2 GB CSR); the GPU arm also writes 256 MiB between timed steps",
            "parallelism": "replicas" if world > 1 else "single device", "graph_resident": True}


def single_source_graph(pb, which: str, args=None):
    """(graph, workload name, metric, sources, config extras) of a
    single-source workload: c1 (rMat 2^20), c2 (torus 160^3) or the headline
    (rMat 2^logn, 2^log_samples draws)."""
    if which == "torus160":
        dg = pb.torus3d_graph(160, perm_seed=2)
        return (dg, "torus160_perm2_bfs", "GTEPS (BFS, 3-D torus 160^3, ids permuted with seed 2)", [0],
                {"dn": 160, "perm_seed": 2})
    if which == "rmat20":
        dg = pb.rmat_graph(20, 10 << 20, 1, 0.5, 0.1, 0.1)
        return (dg, "rmat20_e10n_bfs", "GTEPS (BFS, rMat 2^20 / 10n samples, a=.5 b=c=.1)", [0],
                {"samples": 10 << 20, "abc": [0.5, 0.1, 0.1], "seed": 1})
    logn, lsamp = (args.logn, args.log_samples) if args else (LOGN, 28)
    samples = 1 << lsamp
    workload = WORKLOAD if (logn, samples) == (LOGN, SAMPLES) else "rmat%d_e%d_dobfs" % (logn, lsamp)
    dg = pb.rmat_graph(logn, samples, SEED, A, B, C)
    deg = np.diff(dg.download_offsets().astype(np.int64))
    return (dg, workload, "GTEPS (direction-optimizing BFS, rMat 2^%d / 2^%d samples)" % (logn, lsamp),
            pick_sources(deg), {"samples": samples, "abc": [A, B, C], "seed": SEED})


def measure_single(pb, dg, sources, steps, warmup, dev, world, local, tune=None, e2e=True, chunk=None):
    """Device-timed single-source searches (one persistent launch each, L2
    flushed between them, CUDA events on the launching stream), then the same
    searches end to end through pbg_bfs() into a pinned host parent array.
    `chunk`: the chunk degree the searches use (None: the named option or the
    library default), which decides the kernel: bfs_lean when every list is
    shorter, else bfs_persistent."""
    import ctypes as ct

    import torch

    tune = tune or {}
    n = dg.n
    chunk = chunk or tune.get("chunk_min_degree") or 32  # 32: the library's chunk degree when none is named
    max_deg = int(np.diff(dg.download_offsets().astype(np.int64)).max()) if n else 0
    kernel = "bfs_lean<ANY>" if max_deg < chunk else "bfs_persistent<ANY,%d>" % (tune.get("block_threads") or 1024)
    nsrc = len(sources)
    parent = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def one(i):
        dg.bfs_device(sources[i % nsrc], parent, None, stream=sptr, **tune)

    for i in range(warmup):
        flush.zero_()
        one(i)
    torch.cuda.synchronize()
    # per-source reached edges (a property of the graph and source)
    reached = {}
    trace0 = None
    for s in range(nsrc):
        dg.bfs_device(sources[s], parent, None, stream=sptr, **tune)
        torch.cuda.synchronize()
        reached[s] = dg.last_stats()
        if s == 0:
            trace0 = [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in t.items()} for t in dg.trace()]
    barrier(world)
    torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local) as clk:
        for i in range(steps):
            flush.zero_()
            evs[i][0].record(stream)
            one(i)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    times = [a.elapsed_time(b) / 1e3 for a, b in evs]
    total_s = sum(times)
    edges = sum(reached[i % nsrc]["edges_reached"] / 2.0 for i in range(steps))
    total_s_max = max_over_ranks(total_s, world)
    alg_bytes = [4 * (n + 1) + 4 * reached[i % nsrc]["edges_reached"] + 4 * n for i in range(steps)]
    achieved_gbs = sum(alg_bytes) / total_s / 1e9
    peak, peak_kind = peaks()

    # end to end through the public API with a pinned host parent buffer
    host_par = torch.empty(n, dtype=torch.int32, pin_memory=True)
    host_np = host_par.numpy()
    o = ct.byref(pb._capi.default_opts(**tune)) if tune else None  # None: the graph's own options
    st = pb._capi.BfsStats()
    e2e_times = []
    for i in range(max(2, min(warmup, 4)) if e2e else 0):
        pb._capi.check(pb.lib().pbg_bfs(dg.handle, sources[i % nsrc], o, ct.c_void_p(host_np.ctypes.data), None,
                                        ct.byref(st)))
    barrier(world)
    for i in range(steps if e2e else 0):
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        pb._capi.check(pb.lib().pbg_bfs(dg.handle, sources[i % nsrc], o, ct.c_void_p(host_np.ctypes.data), None,
                                        ct.byref(st)))
        e2e_times.append(time.perf_counter() - t)
    e2e_total = max_over_ranks(sum(e2e_times), world)
    e2e_gteps = world * edges / e2e_total / 1e9 if e2e_total > 0 else None
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return {
        "gteps": world * edges / total_s_max / 1e9, "total_s_max": total_s_max, "reached": reached,
        "trace0": trace0, "e2e_gteps": e2e_gteps, "clocks": clk.summary(),
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 4),
                     "peak_source": (peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                                     else "fallback 6.65 TB/s"),
                     "algorithmic_bytes_per_launch": int(statistics.mean(alg_bytes)), "kernel": kernel},
        "e2e": {"value": round(e2e_gteps, 3) if e2e_gteps else None, "unit": "GTEPS", "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 4 * n,
                "note": "pbg_bfs(): source id in, parent array (pinned host) out; CSR resident"},
    }


def sub_single(pb, which, args, dev, local) -> dict:
    """c1 / c2 sub-object of the default line: plain BFS from source 0."""
    t0 = time.perf_counter()
    dg, workload, metric, sources, extra = single_source_graph(pb, which)
    gen_s = time.perf_counter() - t0
    r = measure_single(pb, dg, sources, args.steps, args.warmup, dev, 1, local, e2e=not args.no_e2e)
    st = r["reached"][0]
    out = {"metric": metric, "value": round(r["gteps"], 3), "unit": "GTEPS",
           "ms_per_search": round(1e3 * r["total_s_max"] / args.steps, 4), "steps": args.steps,
           "warmup": args.warmup,
           "config": {"workload": workload, "n": dg.n, "m_directed": dg.m, **extra, "sources": sources,
                      "levels": st["levels"], "bottomup_levels": st["bottomup_levels"],
                      "l2": "flushed between timed steps (256 MiB write)"},
           "us_per_level": round(1e3 * 1e3 * r["total_s_max"] / args.steps / max(1, st["levels"]), 2),
           "roofline": r["roofline"], "e2e": r["e2e"], "gpu_launches": args.steps, "clocks": r["clocks"],
           "graph_build_s": round(gen_s, 2)}
    dg.close()
    return out


def cpu_baseline(dg, sources, reached, calls, warmup):
    """The reference's own backForwardBFS on the host cores (oracle/_ref), the
    same sample the reference arm times: `warmup` untimed calls, then `calls`
    timed calls cycling through all the sources."""
    try:
        from oracle import oracle as O

        if not O.ref_available():
            return {"value": None, "unit": "GTEPS", "cores": None, "kind": "reference", "cpu_model": cpu_model(),
                    "sample": "unavailable: oracle/_ref/libpbbsref.so not built"}
        off, edg = dg.download()
        G = O.RefGraph(off, edg)
        del edg
        nsrc = len(sources)
        for i in range(warmup):
            G.bfs(sources[i % nsrc], O.REF_BACKFORWARD)
        secs, edges = 0.0, 0.0
        for i in range(calls):
            t = G.time(sources[i % nsrc], O.REF_BACKFORWARD, 1, 0.0)
            secs += float(t[0])
            edges += reached[i % nsrc]["edges_reached"] / 2.0
        cores = O.ref_num_workers()
        G.close()
        return {"value": round(edges / secs / 1e9, 4), "unit": "GTEPS", "cores": cores, "kind": "reference",
                "cpu_model": cpu_model(),
                "sample": "backForwardBFS (reference source, parlay shim, OpenMP) on the same CSR: %d untimed calls, "
                          "then %d timed calls cycling through all %d sources (the reference arm's sample); "
                          "%.2f s timed" % (warmup, calls, nsrc, secs)}
    except Exception as e:  # the baseline is reported, never fatal
        return {"value": None, "unit": "GTEPS", "cores": None, "kind": "reference", "cpu_model": cpu_model(),
                "sample": "failed: %s" % e}


def measure_mis(pb, dg, args, local, host_csr=None) -> dict:
    """Maximal independent set on a resident graph (pbg_mis_device; the
    flags serialMIS returns): W untimed calls, K calls timed with CUDA events,
    then K end-to-end pbg_mis calls with the flags copied to pinned host
    memory; beside it the reference's serialMIS (compiled from its sources)
    on one host core, a bounded sample."""
    import ctypes as ct

    import torch

    dev = torch.device("cuda", local)
    flags = torch.empty(dg.n, dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        dg.mis_device(flags, stream=sp)
    stream.synchronize()
    st = dg.mis_stats()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream), ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            dg.mis_device(flags, stream=sp)
            ev[i][1].record(stream)
        stream.synchronize()
    t = sum(a.elapsed_time(b) for a, b in ev) / 1e3 / args.steps
    host = torch.empty(dg.n, dtype=torch.uint8, pin_memory=True).numpy()
    mst = pb._capi.MisStats()
    e2e = []
    for i in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pb._capi.check(pb.lib().pbg_mis(dg.handle, ct.c_void_p(host.ctypes.data), ct.byref(mst)))
        e2e.append(time.perf_counter() - t0)
    out = {"metric": "ms per maximal independent set (flags of serialMIS, bit-exact)", "value": round(1e3 * t, 4),
           "unit": "ms", "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
           "edges_per_s": round(dg.m / t, 1), "rounds": st["rounds"], "in_set": st["in_set"],
           "config": {"workload": "mis_rmat24_e28", "n": dg.n, "m_directed": dg.m,
                      "l2": "flushed between timed steps (256 MiB write)"},
           "e2e": {"value": round(1e3 * float(np.mean(e2e)), 4), "unit": "ms", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": dg.n, "note": "pbg_mis(): flags to pinned host memory; CSR resident"},
           "gpu_launches": args.steps, "kernel": "mis_persistent<768>", "clocks": clk.summary()}
    if host_csr is not None:
        try:
            from oracle import oracle as O

            if O.refmis_available():
                R = O.RefMisGraph(*host_csr)
                se = R.time(O.REF_SERIAL_MIS, 5, 1.0)
                R.close()
                # ndMIS is not timed: on the parlay shim its lock-and-retry
                # loop (ndMIS/MIS.C:52-76) took 37 s on rMat 2^14 and 441 s on
                # rMat 2^18 with 8 host threads
                out["cpu_baseline"] = {"value": round(1e3 * float(np.median(se)), 2), "unit": "ms",
                                       "kind": "reference", "cores": 1, "cpu_model": cpu_model(),
                                       "sample": "serialMIS (reference source) on the same CSR: median of 5 calls "
                                                 "after 1 s warm-up"}
        except Exception as e:  # the baseline is reported, never fatal
            out["cpu_baseline"] = {"value": None, "sample": "failed: %s" % e}
    return out


def run_ours(args):
    """Single-source workloads.  The default run (workload "all") prints the
    headline with the c1, c2, batched and served sub-objects."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    which = args.workload if args.workload in ("rmat20", "torus160") else "rmat24"
    t0 = time.perf_counter()
    dg, workload, metric, sources, extra = single_source_graph(pb, which, args)
    gen_s = time.perf_counter() - t0
    n, m = dg.n, dg.m
    nsrc = len(sources)

    # options named on the command line; none: the graph's tuned options
    # (after --autotune) or the defaults
    tune = {k: v for k, v in (("block_threads", args.block), ("chunk_min_degree", args.chunk)) if v}
    tuned = None
    if args.autotune:
        # the graph's options picked by the autotuner from 4 other sources, before any timing
        deg = np.diff(dg.download_offsets().astype(np.int64))
        opts, rep = dg.autotune(pick_sources(deg, 4, SEED + 100))
        tuned = {"block_threads": opts["block_threads"], "chunk_min_degree": opts["chunk_min_degree"],
                 "alpha": opts["alpha"], "beta": opts["beta"], "default_ms": round(rep["default_ms"], 4),
                 "best_ms": round(rep["best_ms"], 4)}
    r = measure_single(pb, dg, sources, args.steps, args.warmup, dev, world, local, tune, e2e=not args.no_e2e,
                       chunk=tuned["chunk_min_degree"] if tuned else None)
    reached = r["reached"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(dg, sources, reached, args.cpu_rounds or args.steps, args.warmup)
    levels = [reached[s]["levels"] for s in range(nsrc)]
    if workload == WORKLOAD and not tune and not tuned:
        config = headline_config(n, m, sources, levels, world)
    else:
        config = {"workload": workload, "n": n, "m_directed": m, **extra, "sources": sources, "levels": levels,
                  "autotuned": tuned, "options": tune or None,
                  "l2": "flushed between timed steps (256 MiB write)",
                  "parallelism": "replicas" if world > 1 else "single device", "graph_resident": True}
    roof = dict(r["roofline"])
    roof["traffic"] = traffic_per_launch() if workload == WORKLOAD else None
    line = {
        "metric": metric, "value": round(r["gteps"], 3), "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * r["total_s_max"] / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded %s generated on the device; no dataset)" %
                ("torus" if which == "torus160" else "rMat"),
        "config": config, "hbm_gbs": roof["achieved"], "roofline": roof, "e2e": r["e2e"],
        "gpu_launches": args.steps, "clocks": r["clocks"], "cpu_baseline": cpu,
        "graph_build_s": round(gen_s, 2),
        "bottomup_levels": [reached[s]["bottomup_levels"] for s in range(nsrc)],
        "init_ms": [round(reached[s]["init_ms"], 4) for s in range(nsrc)],
        "trace_first_source": r["trace0"],
    }
    if args.workload == "all" and world == 1 and not args.no_extras and workload == WORKLOAD:
        try:
            line["mis"] = measure_mis(pb, dg, args, local, dg.download() if not args.no_cpu_baseline else None)
        except Exception as e:  # a failing sub-measurement is reported, not hidden
            line["mis"] = {"error": "%s: %s" % (type(e).__name__, e)}
    dg.close()
    if args.workload == "all" and world == 1 and not args.no_extras:
        for key, fn in (("c1", lambda: sub_single(pb, "rmat20", args, dev, local)),
                        ("c2", lambda: sub_single(pb, "torus160", args, dev, local)),
                        ("batched", lambda: measure_batched(args, pb, dev, local, 64, False)),
                        ("served", lambda: measure_serve(args, pb, dev, local))):
            try:
                line[key] = fn()
            except Exception as e:  # a failing sub-measurement is reported, not hidden
                line[key] = {"error": "%s: %s" % (type(e).__name__, e)}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def measure_batched(args, pb, dev, local, K, rmat, world=1, trace=False) -> dict:
    """K sources on randLocal n = 2^23 (5 out-neighbours within +-2^16, seed
    4), or (rmat=True) on the served rMat graph of n = 2^logn (16n samples,
    (.57, .19, .19), seed 10 + logn - 16, sources uniform over non-isolated
    vertices): one batched launch (one uint64 mask word per vertex up to 64
    sources, two up to 128, four up to 256; uint8 levels) against K
    back-to-back plain single-source launches with level output, same GPU,
    same results (tests/test_msbfs_gpu.py checks they are identical)."""
    import ctypes as ct

    import torch

    if not 1 <= K <= pb._capi.MAX_SOURCES:
        raise SystemExit("--sources must be in 1..%d" % pb._capi.MAX_SOURCES)
    lg = args.logn if args.logn != LOGN else 23
    if rmat:
        dg = pb.rmat_graph(lg, 16 << lg, 10 + lg - 16, 0.57, 0.19, 0.19)
        nz = np.nonzero(np.diff(dg.download_offsets()))[0]
        srcs = nz[np.random.default_rng(lg).integers(0, len(nz), K)].astype(np.uint32)
    else:
        dg = pb.randlocal_graph(1 << lg, 5, 1 << 16, 4)
        srcs = np.random.default_rng(4).integers(0, dg.n, K).astype(np.uint32)
    n, m = dg.n, dg.m
    ws = pb.MultiWorkspace(dg, max_sources=K)
    batch = pb.Batch(max_jobs=1)
    dlev = torch.empty(K * n, dtype=torch.uint8, device=dev)
    level = torch.empty(n, dtype=torch.int32, device=dev)
    parent = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        batch.launch([(ws, srcs, dlev)], stream=sp)
    torch.cuda.synchronize()
    st = batch.job_stats(ws)
    if trace:
        for t in batch.job_trace(ws):
            print("level %3d %-15s frontier %10d out-degree %12d  %.3f ms" %
                  (t["level"], t["dir"], t["frontier"], t["frontier_degree"], t["ms"]), file=sys.stderr)
    # edges reached per source (on these graphs every source reaches its component)
    mr = []
    for s_ in srcs[:4]:
        dg.bfs_device(int(s_), parent, level, stream=sp)
        torch.cuda.synchronize()
        mr.append(dg.last_stats()["edges_reached"])
    m_r = int(np.mean(mr))
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            batch.launch([(ws, srcs, dlev)], stream=sp)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    t_batch = sum(a.elapsed_time(b) for a, b in ev) / 1e3 / args.steps
    # K plain single-source launches back to back (levels out), same sources
    plain = []
    with ClockSampler(local) as clk_plain:
        for rep in range(max(1, args.steps // 8)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for s_ in srcs:
                dg.bfs_device(int(s_), parent, level, stream=sp)
            e1.record(stream)
            torch.cuda.synchronize()
            plain.append(e0.elapsed_time(e1) / 1e3)
    t_plain = float(np.median(plain))
    t_batch_max = max_over_ranks(t_batch, world)
    qps = world * K / t_batch_max
    alg = 4 * (n + 1) + 4 * m_r + K * n
    peak, peak_kind = peaks()
    # end to end: pbg_bfs_multi with the K level arrays copied to host
    host = torch.empty(K * n, dtype=torch.uint8, pin_memory=True).numpy()
    o = pb._capi.default_opts()
    bst = pb._capi.BatchStats()
    srcs_c = np.ascontiguousarray(srcs)
    pb._capi.check(pb.lib().pbg_bfs_multi(dg.handle, ct.c_void_p(srcs_c.ctypes.data), K, ct.byref(o),
                                          ct.c_void_p(host.ctypes.data), ct.byref(bst)))
    e2e = []
    for i in range(max(2, args.steps // 4)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        pb._capi.check(pb.lib().pbg_bfs_multi(dg.handle, ct.c_void_p(srcs_c.ctypes.data), K, ct.byref(o),
                                              ct.c_void_p(host.ctypes.data), ct.byref(bst)))
        e2e.append(time.perf_counter() - t)
    e2e_q = world * K / max_over_ranks(float(np.mean(e2e)), world)
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    out = {
        "metric": "queries/s (%d-source batched BFS, %s, levels bit-exact)" %
                  (K, "rMat 2^%d 16n" % int(np.log2(n)) if rmat else "randLocal 2^%d" % int(np.log2(n))),
        "value": round(qps, 1), "unit": "queries/s", "steps": args.steps, "warmup": args.warmup,
        "ms_per_batch": round(1e3 * t_batch_max, 4),
        "config": dict(({"workload": "rmat%d_ms%d" % (int(np.log2(n)), K), "samples": 16 * n,
                         "abc": [0.57, 0.19, 0.19], "seed": 10 + int(np.log2(n)) - 16} if rmat else
                        {"workload": "randlocal%d_ms%d" % (int(np.log2(n)), K), "degree": 5, "window": 1 << 16,
                         "seed": 4}),
                       n=n, m_directed=m, sources=K, mask_words=(K + 63) // 64, levels=st["levels"],
                       pull_levels=st["pull_levels"], push_levels=st["push_levels"],
                       l2="flushed between timed steps (256 MiB write)"),
        "plain_back_to_back": {"ms_per_batch": round(1e3 * t_plain, 3), "queries_per_s": round(K / t_plain, 1),
                               "clocks": clk_plain.summary()},
        "speedup_vs_plain": round(t_plain / t_batch, 2),
        "roofline": {"bound": "hbm", "achieved": round(alg / t_batch / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(alg / t_batch / 1e9 / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": alg, "kernel": "ms_persistent<1>",
                     "peak_source": peak_kind},
        "e2e": {"value": round(e2e_q, 1), "unit": "queries/s", "h2d_bytes_per_step": K * 4,
                "d2h_bytes_per_step": K * n, "note": "pbg_bfs_multi(): %d level arrays to pinned host" % K},
        "gpu_launches": args.steps, "clocks": clk.summary(),
    }
    ws.close()
    batch.close()
    dg.close()
    return out


def run_msbfs(args):
    """--workload msbfs64 / msbfs_rmat: the batched measurement as its own line."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_batched(args, pb, dev, local, args.sources, args.workload == "msbfs_rmat", world,
                        trace=args.trace and rank == 0)
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": "queries/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_batch"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 masks / u8 levels",
                "data": "synthetic (seeded %s generated on the device)" %
                        ("rMat" if args.workload == "msbfs_rmat" else "randLocal")}
        line.update({k: v for k, v in r.items() if k not in line and k != "ms_per_batch"})
        print(json.dumps(line), flush=True)


def measure_serve(args, pb, dev, local) -> dict:
    """Served BFS request stream: 8 resident symmetric rMat graphs, n = 2^16 ..
    2^23, 16n samples, (.57, .19, .19), seeds 10..17; queries pick a graph
    uniformly and a non-isolated source uniformly; Poisson arrivals.  First a
    burst (all queries at t = 0) measures capacity, then an open-loop replay at
    the stated rate measures latency.  Every query of both runs is checked:
    its level checksum equals that of an independent single-source search."""
    import ctypes as ct

    import torch

    graphs = [pb.rmat_graph(lg, 16 << lg, 10 + i, A, B, C) for i, lg in enumerate(range(16, 24))]
    offs = [g.download_offsets() for g in graphs]
    rng = np.random.default_rng(5)
    Q = args.queries
    qg = rng.integers(0, len(graphs), Q).astype(np.uint32)
    qs = np.empty(Q, np.uint32)
    for gi in range(len(graphs)):
        nz = np.nonzero(np.diff(offs[gi]))[0]
        idx = np.nonzero(qg == gi)[0]
        qs[idx] = nz[rng.integers(0, len(nz), len(idx))]
    budget = args.hbm_gb << 30
    wide_n = (1 << args.serve_wide_max_logn) if args.serve_wide_sources else 0
    srv = pb.Server(graphs, hbm_budget_bytes=budget, max_sources=args.serve_sources, max_jobs=args.max_jobs,
                    streams=args.streams, wide_sources=args.serve_wide_sources, wide_max_vertices=wide_n,
                    max_launch_edges=args.serve_max_launch_edges)

    def run(arrival):
        srv.replay(qg, qs, arrival)
        srv.drain()
        res = []
        while len(res) < Q:
            res += srv.poll(cap=65536)
        return res

    def launches_of(res):
        groups = {}
        for r in res:
            groups.setdefault((r["t_launch_us"], r["t_done_us"]), []).append(r["graph"])
        sizes = np.array([len(v) for v in groups.values()])
        durs = np.array([k[1] - k[0] for k in groups])
        return {"launches": len(groups), "queries_per_launch_mean": round(float(sizes.mean()), 1),
                "launch_us_p50": round(float(np.percentile(durs, 50)), 1),
                "launch_us_p90": round(float(np.percentile(durs, 90)), 1)}

    run(np.zeros(Q))  # warm-up pass over the same stream
    with ClockSampler(local) as clk_burst:
        t0 = time.perf_counter()
        burst = run(np.zeros(Q))
        burst_s = time.perf_counter() - t0
    cap_qps = Q / burst_s
    rate = args.rate or round(0.75 * cap_qps, -2)
    arrival = np.cumsum(np.random.default_rng(6).exponential(1e6 / rate, Q))
    st0 = srv.stats()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        timed = run(arrival)
        wall = time.perf_counter() - t0
    lat = np.array([r["t_done_us"] - r["t_submit_us"] for r in timed])
    span_us = max(r["t_done_us"] for r in timed) - min(r["t_submit_us"] for r in timed)
    qps = Q / (span_us / 1e6)
    st = srv.stats()

    # every query of both runs against an independent single-source search
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream
    lvbuf = [torch.empty(g.n, dtype=torch.int32, device=dev) for g in graphs]
    pbuf = [torch.empty(g.n, dtype=torch.int32, device=dev) for g in graphs]
    pairs = sorted(set(zip(qg.tolist(), qs.tolist())))
    sums = torch.empty(len(pairs), dtype=torch.int64, device=dev)
    base = sums.data_ptr()
    for i, (g, s_) in enumerate(pairs):
        graphs[g].bfs_device(s_, pbuf[g], lvbuf[g], stream=sp)
        pb._capi.check(pb.lib().pbg_levels32_checksum(ct.c_void_p(lvbuf[g].data_ptr()), graphs[g].n,
                                                      ct.c_void_p(base + 8 * i), ct.c_void_p(sp)))
    stream.synchronize()
    sv = sums.cpu().numpy().view(np.uint64)
    want = {pr: int(sv[i]) for i, pr in enumerate(pairs)}
    bad = sum(1 for r in burst + timed if r["status"] != 0 or r["checksum"] != want[(r["graph"], r["src"])])

    # back-to-back plain single-source launches (levels out) on a sample
    sample = min(Q, 4000)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk_plain:
        e0.record(stream)
        for i in range(sample):
            g = int(qg[i])
            graphs[g].bfs_device(int(qs[i]), pbuf[g], lvbuf[g], stream=sp)
        e1.record(stream)
        stream.synchronize()
    plain_qps = sample / (e0.elapsed_time(e1) / 1e3)
    out = {
        "metric": "queries/s (served BFS, 8 resident rMat graphs 2^16..2^23, continuous batching%s)" %
                  ("" if args.serve_sources == 64 and not args.serve_wide_sources else
                   ", %d-source jobs%s" % (args.serve_sources, ", %d on graphs of <= 2^%d vertices" %
                                            (args.serve_wide_sources, args.serve_wide_max_logn)
                                            if args.serve_wide_sources else "")),
        "value": round(qps, 1), "unit": "queries/s", "queries": Q,
        "config": {"workload": "serve_rmat16to23", "queries": Q, "arrival": "Poisson",
                   "rate_qps": rate, "graphs_n": [g.n for g in graphs], "graphs_m": [g.m for g in graphs],
                   "max_sources": args.serve_sources, "max_jobs": args.max_jobs, "streams": args.streams,
                   "hbm_budget_bytes": budget, "max_launch_edges": args.serve_max_launch_edges,
                   "wide_sources": args.serve_wide_sources, "wide_max_vertices": wide_n},
        "latency_us": {"p50": round(float(np.percentile(lat, 50)), 1),
                       "p99": round(float(np.percentile(lat, 99)), 1), "max": round(float(lat.max()), 1)},
        "capacity_qps_burst": round(cap_qps, 1), "clocks_burst": clk_burst.summary(),
        "launch_shape_burst": launches_of(burst), "launch_shape_timed": launches_of(timed),
        "plain_back_to_back_qps": round(plain_qps, 1), "plain_sample_queries": sample,
        "clocks_plain": clk_plain.summary(),
        "speedup_vs_plain": round(qps / plain_qps, 2),
        "speedup_capacity_vs_plain": round(cap_qps / plain_qps, 2),
        "server": st, "verified_queries": len(burst) + len(timed), "mismatches": bad,
        "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 8,
                "d2h_bytes_per_step": 8, "note": "query (graph, source) in, level checksum out"},
        # the timed run's fused launches and one checksum launch per job
        "gpu_launches": (st["launches"] - st0["launches"]) + (st["jobs"] - st0["jobs"]),
        "clocks": clk.summary(), "wall_s": round(wall, 3),
    }
    srv.close()
    for g in graphs:
        g.close()
    return out


def run_serve(args):
    """--workload serve: the served measurement as its own line."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_serve(args, pb, dev, local)
    Q = args.queries
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": "queries/s", "n_gpus": world, "steps": Q,
                "warmup": Q, "ms_per_step": round(1e3 / r["value"], 5) if r["value"] else None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u64 masks / u8 levels", "data": "synthetic (seeded rMat on the device)"}
        line.update({k: v for k, v in r.items() if k not in line})
        print(json.dumps(line), flush=True)


def run_mis(args):
    """--workload mis: the maximal independent set measurement as its own line."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    dg = pb.rmat_graph(args.logn, 1 << args.log_samples, SEED, A, B, C)
    gen_s = time.perf_counter() - t0
    r = measure_mis(pb, dg, args, local, None if args.no_cpu_baseline else dg.download())
    r["config"]["workload"] = "mis_rmat%d_e%d" % (args.logn, args.log_samples)
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": "ms", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["value"], "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "u32 ids / u8 flags", "data": "synthetic (seeded rMat on the device)",
                "graph_build_s": round(gen_s, 2)}
        line.update({k: v for k, v in r.items() if k not in line})
        print(json.dumps(line), flush=True)
    dg.close()


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpbbsref.so not built"}))
        return
    t0 = time.perf_counter()
    off, edg = O.rmat(LOGN, SAMPLES, SEED, A, B, C)
    gen_s = time.perf_counter() - t0
    n = len(off) - 1
    deg = np.diff(off.astype(np.int64))
    sources = pick_sources(deg)
    G = O.RefGraph(off, edg)
    lv_edges, levels = {}, []
    for s in range(NSRC):
        lv = O.bfs_levels(off, edg, sources[s])
        lv_edges[s] = int(deg[lv != O.NONE].sum())
        levels.append(int(lv[lv != O.NONE].max()) + 1)  # BFS rounds, the GPU arm's `levels`
    m = len(edg)
    del edg
    for i in range(args.warmup):
        G.bfs(sources[i % NSRC], O.REF_BACKFORWARD)
    times, edges = [], 0.0
    for i in range(args.steps):
        t = G.time(sources[i % NSRC], O.REF_BACKFORWARD, 1, 0.0)
        times.append(float(t[0]))
        edges += lv_edges[i % NSRC] / 2.0
    total = sum(times)
    val = edges / total / 1e9
    cores = O.ref_num_workers()
    print(json.dumps({
        "impl": "reference",
        "metric": "GTEPS (direction-optimizing BFS, rMat 2^24 / 2^28 samples)",
        "value": round(val, 4), "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded rMat generated on the host; no dataset)",
        "config": headline_config(n, m, sources, levels, world),
        "graph_build_s": round(gen_s, 1),
        "cpu_baseline": {"value": round(val, 4), "unit": "GTEPS", "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": "backForwardBFS (reference source on the project parlay shim, OpenMP), "
                                   "%d untimed calls, then %d timed calls cycling through all %d sources" %
                                   (args.warmup, args.steps, NSRC)},
        "e2e": {"value": round(val, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)
    G.close()


def run_io(args):
    """Graph file input: the C1 graph (rMat 2^20, 10n samples) written as
    AdjacencyGraph text (formatted on the device), then loaded K times from
    the file into a resident, validated CSR (pbg_graph_load_adj: read through
    pinned pieces, copy, tokenise and parse on the device).  The CPU baseline
    is the reference's own reader (readGraphFromFile, common/graphIO.h:191-215,
    on the project parlay shim with OpenMP) on the same file."""
    import tempfile

    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    g = pb.rmat_graph(20, 10 << 20, 1, 0.5, 0.1, 0.1)
    n, m = g.n, g.m
    d = tempfile.mkdtemp(prefix="pbg_io_")
    path = os.path.join(d, "rmat20.adj")
    t = time.perf_counter()
    g.write_adjacency(path)
    t_write = time.perf_counter() - t
    size = os.path.getsize(path)
    ref_off, ref_edg = g.download()
    for _ in range(args.warmup):
        pb.DeviceGraph.load_adjacency(path, symmetric=True).close()
    barrier(world)
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        h = pb.DeviceGraph.load_adjacency(path, symmetric=True)
        times.append(time.perf_counter() - t)
        h.close()
    h = pb.DeviceGraph.load_adjacency(path, symmetric=True)
    off, edg = h.download()
    assert np.array_equal(off, ref_off) and np.array_equal(edg, ref_edg), "loaded graph differs"
    h.close()
    t_load = max_over_ranks(float(np.median(times)), world)
    # the same text from host memory (no file read): copy + parse + validation
    text = open(path, "rb").read()
    mem = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        pb.DeviceGraph.parse_adjacency(text, symmetric=True).close()
        if i >= args.warmup:
            mem.append(time.perf_counter() - t)
    t_mem = max_over_ranks(float(np.median(mem)), world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        if O.ref_available():
            R = O.ref()
            ts = []
            for _ in range(max(1, args.cpu_rounds)):
                t = time.perf_counter()
                gg = R.pbbsref_read_graph(os.fsencode(path))
                ts.append(time.perf_counter() - t)
                R.pbbsref_graph_free(gg)
            cpu = {"value": round(size / float(np.median(ts)) / 1e6, 1), "unit": "MB/s of text",
                   "cores": O.ref_num_workers(), "kind": "reference", "cpu_model": cpu_model(),
                   "sample": "readGraphFromFile on the same %d-byte file, median of %d" % (size, len(ts))}
    os.remove(path)
    os.rmdir(d)
    if rank == 0:
        mbs = world * size / t_load / 1e6
        print(json.dumps({
            "metric": "MB/s of AdjacencyGraph text loaded into a resident CSR (rMat 2^20 / 10n)",
            "value": round(mbs, 1), "unit": "MB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * t_load, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8 text -> u32 CSR", "data": "synthetic (seeded rMat written as text)",
            "config": {"workload": "io_rmat20", "n": n, "m_directed": m, "file_bytes": size,
                       "write_s": round(t_write, 3), "source": "file (page cache warm after the warm-up loads)"},
            "edges_per_s": round(world * m / t_load, 1),
            "from_host_memory": {"value": round(world * size / t_mem / 1e6, 1), "unit": "MB/s",
                                 "ms_per_step": round(1e3 * t_mem, 3),
                                 "note": "pbg_graph_parse_adj() on the file's bytes in pageable memory"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(mbs, 1), "unit": "MB/s", "h2d_bytes_per_step": size, "d2h_bytes_per_step": 8,
                    "note": "pbg_graph_load_adj(): file -> pinned pieces -> HBM -> CSR; the same number"},
            # per load: k_count_tokens, k_parse_tokens, k_validate, k_iso_bitmap (and CUB's scan)
            "gpu_launches": 4 * args.steps,
        }), flush=True)
    g.close()


def run_check(args):
    """The device check of BFS output (pbg_bfs_check: checkBFS's
    level_number by pointer doubling and the neighbour-minimum level test of
    bench/BFSCheck.C:39-90) on the parent arrays of the headline searches
    (rMat 2^logn, the headline's sources), device-resident parents, one
    synchronous call each; with the edge-existence test too; end to end with
    the parents copied from pinned host memory first.  The CPU baseline is the
    reference's own checkBFS (on the project parlay shim, OpenMP, all host
    cores) on the same CSR and parents, a bounded sample of sources."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dg, workload, _, sources, extra = single_source_graph(pb, "rmat24", args)
    n = dg.n
    par = torch.empty(n, dtype=torch.int32, device=dev)
    host = torch.empty(n, dtype=torch.int32, pin_memory=True)
    NONE = 0xFFFFFFFF

    def one(i, edges):
        r = dg.check(sources[i % len(sources)], par, edges=edges)
        assert r["bad_vertex"] == NONE, r

    for i in range(max(3, args.warmup)):
        dg.bfs_device(sources[i % len(sources)], par)
        torch.cuda.synchronize()
        one(i, False)
        one(i, True)
    barrier(world)
    lvl, edg, e2e = [], [], []
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            dg.bfs_device(sources[i % len(sources)], par)
            host.copy_(par)
            torch.cuda.synchronize()
            t = time.perf_counter()
            one(i, False)
            lvl.append(time.perf_counter() - t)
            t = time.perf_counter()
            one(i, True)
            edg.append(time.perf_counter() - t)
            t = time.perf_counter()
            par.copy_(host, non_blocking=True)
            one(i, False)
            e2e.append(time.perf_counter() - t)
    t_lvl = max_over_ranks(float(np.median(lvl)), world)
    t_edg = max_over_ranks(float(np.median(edg)), world)
    t_e2e = max_over_ranks(float(np.median(e2e)), world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        if O.ref_available():
            off, ed = dg.download()
            R = O.RefGraph(off, ed)
            ts = []
            for i in range(min(len(sources), max(2, args.cpu_rounds))):
                dg.bfs_device(sources[i], par)
                hp = par.cpu().numpy()
                t = time.perf_counter()
                rc = R.check(sources[i], hp)
                ts.append(time.perf_counter() - t)
                assert rc == 0, "reference checkBFS rejected a device BFS tree"
            R.close()
            cpu = {"value": round(1e3 * float(np.median(ts)), 2), "unit": "ms", "cores": O.ref_num_workers(),
                   "kind": "reference", "cpu_model": cpu_model(),
                   "sample": "checkBFS on the same CSR and parents, median of %d sources" % len(ts)}
    if rank == 0:
        print(json.dumps({
            "metric": "ms per BFS check (checkBFS level test on the device, rMat 2^%d)" % args.logn,
            "value": round(1e3 * t_lvl, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * t_lvl, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded rMat on the device)",
            "config": {"workload": "check_" + workload, "n": n, "m_directed": dg.m, **extra, "sources": sources},
            "with_edge_test_ms": round(1e3 * t_edg, 4),
            "e2e": {"value": round(1e3 * t_e2e, 4), "unit": "ms", "h2d_bytes_per_step": 4 * n,
                    "d2h_bytes_per_step": 16,
                    "note": "parents copied from pinned host memory, then pbg_bfs_check (level test)"},
            "cpu_baseline": cpu,
            # per check: jump_init, one jump_step per doubling round (4 here), jump_finish, check_rows
            "gpu_launches": 7 * args.steps,
            "clocks": clk.summary(),
        }), flush=True)
    dg.close()


def run_build(args):
    """Graph construction on the device (pbg_graph_generate: rMat draws
    (rMatGraph.C:33-79), symmetrise, sort, deduplicate (graphUtils.h:54-94),
    CSR, validation and the degree-0 bitmap) of the headline graph, rMat
    2^logn with 2^log_samples draws, into a resident CSR, K times; each
    graph is freed before the next.  The CPU baseline is the oracle's C
    restatement of the same construction (one core) on a bounded sample,
    rMat 2^20 with 2^24 draws; the reference's own generator needs parlay's
    hash and cannot be built here."""
    import torch

    import pbbsbench_b200 as pb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    samples = 1 << args.log_samples

    def one():
        return pb.rmat_graph(args.logn, samples, SEED, A, B, C)

    for _ in range(max(1, args.warmup)):
        one().close()
    barrier(world)
    ts = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            g = one()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t)
            n, m = g.n, g.m
            g.close()
    t_dev = max_over_ranks(float(np.median(ts)), world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        cs = 1 << 24
        t = time.perf_counter()
        O.rmat(20, cs, SEED, A, B, C)
        dt = time.perf_counter() - t
        cpu = {"value": round(cs / dt / 1e6, 2), "unit": "M draws/s", "cores": 1, "kind": "port",
               "cpu_model": cpu_model(),
               "sample": "the oracle's C construction of rMat 2^20 with 2^24 draws (%.1f s)" % dt}
    if rank == 0:
        v = world * samples / t_dev / 1e6
        print(json.dumps({
            "metric": "M rMat edge draws/s to a validated resident CSR (rMat 2^%d / 2^%d draws)"
                      % (args.logn, args.log_samples),
            "value": round(v, 1), "unit": "M draws/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * t_dev, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 keys -> u32 CSR",
            "data": "synthetic (seeded rMat on the device)",
            "config": {"workload": "build_rmat%d_e%d" % (args.logn, args.log_samples), "n": n, "m_directed": m,
                       "samples": samples, "abc": [A, B, C], "seed": SEED},
            "cpu_baseline": cpu,
            "e2e": {"value": round(v, 1), "unit": "M draws/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "note": "pbg_graph_generate(): the graph is built and kept in HBM; the same number"},
            # per graph: k_gen_rmat, k_keys_to_csr, k_validate, k_iso_bitmap (beside CUB's radix sort
            # and select, about 25 more launches)
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
        }), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("msbfs64", "msbfs_rmat"):
        run_msbfs(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "io":
        run_io(args)
    elif args.workload == "mis":
        run_mis(args)
    elif args.workload == "check":
        run_check(args)
    elif args.workload == "build":
        run_build(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
