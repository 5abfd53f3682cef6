"""Benchmark: decoded Mpixel/s of the HTJ2K tile-batch decode path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c1|c1i|c1c|c2|c3|c4] [--impl ours|reference]

A step is one decode of the whole workload batch.  Default workload: 256
tiles of 512x512 RGB8 (H&E-like, 5 levels, 64x64 code blocks, RCT), seeded
synthetic data; c1i is the same batch coded lossy (9/7, ICT, quantised),
c1c the same batch with classic (EBCOT) code blocks.
Prints one JSON line (rank 0):

  value        batched decode, codestreams resident in HBM (one plan: HT
               cleanup over all code blocks ordered by coded length, IDWT
               rounds, fused last level + RCT + pack), timed with CUDA events
               on the library's stream;
  plain_*      the plain per-tile path (one tile per call) on the same tiles;
  e2e          sgn_j2k_decode_tiles_to_device from pinned host codestreams:
               host parse, H2D copy, kernels, status read-back;
  roofline     dominant kernel: (codestream + output bytes) / its duration;
  cpu_baseline the oracle (C++ restatement of the reference CPU tile batch)
               on the host cores, bounded sample.

With --gpus N > 1 (torchrun) every rank decodes its own replica of the
workload (independent tiles, no data-path collective) and rank 0 reports the
total over the max per-rank time.
"""
import argparse
import json
import os
import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c1", choices=["c1", "c1i", "c1c", "c2", "c3", "c4"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape (profiling runs)")
    ap.add_argument("--pool", type=int, default=4096, help="c4: tiles in the serving pool")
    ap.add_argument("--rates", default="2000,5000,10000,20000,35000,50000,70000,90000,110000,130000,160000,200000",
                    help="c4: arrival rates, tiles/s")
    ap.add_argument("--seconds", type=float, default=1.0, help="c4: open-loop duration per rate")
    ap.add_argument("--slots", type=int, default=4, help="c4: batches in flight")
    ap.add_argument("--max-batch", type=int, default=512, help="c4: requests per batch")
    ap.add_argument("--max-batch-samples", type=int, default=96000000,
                    help="c4: decoded samples per batch (0: unbounded)")
    return ap.parse_args()


def build_workload(name):
    from signinum_b200 import encode

    if name == "c1":
        return encode.config1(), "rgb8"
    if name == "c1i":
        return encode.config1_irreversible(), "rgb8"
    if name == "c1c":
        return encode.config1_classic(), "rgb8"
    if name == "c2":
        return encode.config2(), "rgb8"
    return encode.config3(), "gray16"


WORKLOAD_CONFIG = {
    "c1": {"workload": "uniform batch: 256 tiles 512x512 RGB8, HTJ2K lossless 5/3, 5 levels, 64x64 code blocks, RCT",
           "tiles": 256},
    "c1i": {"workload": "uniform batch, lossy: 256 tiles 512x512 RGB8, HTJ2K irreversible 9/7 + ICT, scalar "
                    "expounded quantisation (relative step 1/256), 5 levels, 64x64 code blocks", "tiles": 256},
    "c1c": {"workload": "uniform batch, classic Tier-1: 256 tiles 512x512 RGB8, J2K lossless 5/3 with EBCOT (MQ) "
                    "code blocks, 5 levels, 64x64 code blocks, RCT", "tiles": 256},
    "c2": {"workload": "uneven batch: 1024 RGB8 tiles, sides 128..1024, 3..6 levels, 32x32/64x64 blocks, 20% near-blank",
           "tiles": 1024},
    "c3": {"workload": "high bit depth: 128 tiles 2048x2048 u16 gray, 6 levels, 64x64 code blocks",
           "tiles": 128},
}


class Clocks:
    """SM clock, power and clock-event reasons sampled from NVML (read-only
    queries) every millisecond during the timed region; each sample is also
    written to gpurun_out/clocks_<pid>.csv."""

    REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap")]

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.path = ROOT / "gpurun_out" / f"clocks_{os.getpid()}.csv"
        self.stop = None
        self.thread = None

    def _handle(self, nv):
        import torch

        try:
            prop = torch.cuda.get_device_properties(self.index)
            bus = f"{prop.pci_domain_id:08X}:{prop.pci_bus_id:02X}:{prop.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        nv, h = self.nv, self.h
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        try:
            power = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
        except Exception:
            power = float("nan")
        active = [name for name, attr in self.REASONS if reasons & getattr(nv, attr, 0)]
        self.rows.append((time.perf_counter(), sm, mx, power, active))

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h = self._handle(nv)
            self._sample()
        except Exception:
            self.nv = None
            return self
        self.stop = threading.Event()

        def loop():
            while not self.stop.is_set():
                try:
                    self._sample()
                except Exception:
                    pass
                self.stop.wait(0.001)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join()
        if self.nv:
            try:
                self._sample()
            except Exception:
                pass
            try:
                self.path.parent.mkdir(exist_ok=True)
                with open(self.path, "w") as f:
                    f.write("t_s,sm_mhz,sm_max_mhz,power_w,reasons\n")
                    for t, sm, mx, pw, act in self.rows:
                        f.write(f"{t:.6f},{sm},{mx},{pw:.1f},{'|'.join(act)}\n")
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[1] for r in self.rows]
        reasons = sorted({x for r in self.rows for x in r[4]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[2] for r in self.rows), "reasons": reasons,
                "samples": len(self.rows), "source": "NVML, 1 ms polling during the timed region"}


def cpu_baseline(tiles, fmt, budget_s=12.0):
    """The oracle's CPU tile batch (all host threads) over a bounded sample of
    the workload: whole passes over its tiles until about budget_s seconds."""
    from oracle import oracle

    cores = os.cpu_count() or 1
    # One single-threaded probe decode sizes the sample.
    t0 = time.perf_counter()
    oracle.decode(tiles[0].codestream, fmt)
    per_tile = max(time.perf_counter() - t0, 1e-4)
    k = int(max(1, min(len(tiles), budget_s * cores / per_tile)))
    sample = [t.codestream for t in tiles[:k]]
    px = sum(t.width * t.height for t in tiles[:k])
    passes, dt, ok = 0, 0.0, True
    while passes == 0 or dt < budget_s:
        t0 = time.perf_counter()
        outs, first = oracle.decode_batch(sample, fmt, workers=cores)
        dt += time.perf_counter() - t0
        ok = ok and first == -1
        passes += 1
    return {"value": passes * px / dt / 1e6, "unit": "Mpixel/s", "cores": cores, "kind": "port",
            "sample": f"first {k} of {len(tiles)} tiles of the workload, {passes} passes, {cores} threads; C++ "
                      "restatement of the reference CPU tile batch (Rust toolchain absent)",
            "seconds": dt, "ok": ok}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's tile batch."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, kind = build_workload(args.workload)
    fmt = 1 if kind == "rgb8" else 3
    from oracle import oracle

    cores = os.cpu_count() or 1
    # Each step: a bounded sample (~2 s of CPU work per step at one thread).
    t0 = time.perf_counter()
    oracle.decode(w.tiles[0].codestream, fmt)
    per_tile = max(time.perf_counter() - t0, 1e-4)
    k = int(max(1, min(len(w.tiles), 2.0 * cores / per_tile / max(args.steps, 1))))
    sample = [t.codestream for t in w.tiles[:k]]
    px = sum(t.width * t.height for t in w.tiles[:k])
    for _ in range(args.warmup):
        oracle.decode_batch(sample, fmt, workers=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, first = oracle.decode_batch(sample, fmt, workers=cores)
        times.append(time.perf_counter() - t0)
    ms = 1000.0 * float(np.mean(times))
    v = px / (ms / 1000.0) / 1e6
    line = {"impl": "reference", "metric": "decoded Mpixel/s", "value": v, "unit": "Mpixel/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)", "config": dict(WORKLOAD_CONFIG[args.workload], sample_tiles=k),
            "cpu_baseline": {"value": v, "unit": "Mpixel/s", "cores": cores, "kind": "port",
                             "sample": f"first {k} tiles of the workload per step, {cores} threads; C++ "
                                       "restatement of the reference CPU tile batch (Rust toolchain absent)"},
            "e2e": {"value": v, "unit": "Mpixel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Serving: open-loop Poisson arrivals over a resident pool of uneven tiles
    (60% full RGB8, 25% quarter resolution, 15% 256x256 region), continuous
    batching in the native server, p50/p99 latency and throughput per rate."""
    import ctypes
    import threading

    import torch

    from signinum_b200 import _native, encode
    from signinum_b200._native import SgnRequest, SgnServerResult
    from signinum_b200.server import Server

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pool = encode.config4_pool(args.pool).tiles
    coded = sum(len(t.codestream) for t in pool)
    from signinum_b200 import j2k_cuda

    ctx = j2k_cuda._Context.open(local)
    server = Server(ctx, device_budget_bytes=16 << 30, resident_capacity_bytes=coded + 64 * len(pool) + (1 << 20),
                    max_batch_tiles=args.max_batch, slots=args.slots, max_batch_samples=args.max_batch_samples)
    ids = [server.register(t.codestream) for t in pool]
    lib = _native.cuda_lib()
    h = server._h

    def make_requests(n, seed):
        rng = np.random.default_rng(seed)
        reqs, px = [], []
        for _ in range(n):
            i = int(rng.integers(len(pool)))
            t = pool[i]
            u = rng.uniform()
            r = SgnRequest(0, 0, 0, 0, 0, 1)
            if u < 0.60:
                px.append(t.width * t.height)
            elif u < 0.85:
                r.kind, r.downscale = 2, 4
                px.append(-(-t.width // 4) * -(-t.height // 4))
            else:
                side = min(256, t.width)
                r.kind, r.w, r.h = 1, side, side
                r.x = int(rng.integers(0, t.width - side + 1))
                r.y = int(rng.integers(0, t.height - side + 1))
                px.append(side * side)
            reqs.append((ids[i], r, i))
        return reqs, px

    def run(reqs, gaps, check=0):
        """Submits reqs at the given inter-arrival gaps (seconds), every request
        whose arrival time has passed going in with one sgn_server_submit_many
        call; returns latencies (ms), wall seconds from first submit to last
        result, and the parity of `check` sampled results against the oracle."""
        n = len(reqs)
        chunks = []
        done = threading.Event()
        keep = set(range(0, n, max(1, n // check))) if check else set()
        kept = {}
        first = []

        def poller():
            from signinum_b200._native import SgnSurface

            cap = 8192
            buf = (SgnServerResult * cap)()
            view = np.frombuffer(buf, dtype=np.dtype({
                "names": ["ticket", "status", "latency"],
                "formats": ["<u8", "<i4", "<f8"],
                "offsets": [SgnServerResult.ticket.offset, SgnServerResult.status.offset,
                            SgnServerResult.latency_ms.offset],
                "itemsize": ctypes.sizeof(SgnServerResult)}))
            cnt = ctypes.c_size_t()
            total = 0
            while total < n:
                lib.sgn_server_poll(h, buf, cap, ctypes.byref(cnt), 20)
                m = cnt.value
                if not m:
                    continue
                part = view[:m].copy()
                chunks.append(part)
                total += m
                if keep:
                    while not first:
                        pass
                    for j in np.nonzero(np.isin(part["ticket"] - first[0], list(keep)))[0]:
                        r = buf[int(j)]
                        if r.status != 0 or not r.surface.device_ptr:
                            continue
                        s = SgnSurface()
                        ctypes.pointer(s)[0] = r.surface
                        out = np.zeros(max(1, s.pitch_bytes * s.height), np.uint8)
                        lib.sgn_surface_download(ctx.handle, ctypes.byref(s), out.ctypes.data, out.nbytes,
                                                 s.pitch_bytes)
                        kept[int(r.ticket - first[0])] = out.tobytes()
                lib.sgn_server_results_release(h, buf, m)
            done.set()

        ids_arr = (ctypes.c_uint32 * n)(*[q[0] for q in reqs])
        req_arr = (SgnRequest * n)(*[q[1] for q in reqs])
        tick_arr = (ctypes.c_uint64 * n)()
        sub = ctypes.c_size_t()
        rsz = ctypes.sizeof(SgnRequest)
        th = threading.Thread(target=poller, daemon=True)
        sys.setswitchinterval(1e-4)  # the poller thread gets the interpreter often
        th.start()
        sched = np.cumsum(gaps)
        k = 0
        t0 = time.perf_counter()
        while k < n:
            j = int(np.searchsorted(sched, time.perf_counter() - t0, side="right"))
            if j <= k:
                continue
            rc = lib.sgn_server_submit_many(
                h, j - k, ctypes.cast(ctypes.addressof(ids_arr) + 4 * k, ctypes.POINTER(ctypes.c_uint32)), 1,
                ctypes.cast(ctypes.addressof(req_arr) + rsz * k, ctypes.POINTER(SgnRequest)),
                ctypes.cast(ctypes.addressof(tick_arr) + 8 * k, ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(sub))
            assert rc == 0 and sub.value == j - k, rc
            if not first:
                first.append(tick_arr[0])
            k = j
        done.wait(120)
        wall = time.perf_counter() - t0
        th.join(5)
        res = np.concatenate(chunks) if chunks else np.zeros(0)
        lat = res["latency"]
        assert len(res) == n and np.all(res["status"] == 0), "a request failed"
        ok = None
        if check:
            from oracle import oracle

            ok = len(kept) > 0
            for kk, b in kept.items():
                tid, r, i = reqs[kk]
                want, _, _ = oracle.decode(pool[i].codestream, 1, r.kind, (r.x, r.y, r.w, r.h), r.downscale)
                ok = ok and (want == b)
        return lat, wall, ok

    # Warm-up, then the closed-loop peak: every request submitted at once.
    warm, _ = make_requests(2000, 11)
    run(warm, np.zeros(len(warm)))
    peak_reqs, peak_px = make_requests(20000, 12)
    s0 = server.stats()
    with Clocks(local) as clk_peak:
        _, peak_wall, ok_peak = run(peak_reqs, np.zeros(len(peak_reqs)), check=16)
    peak_tps = len(peak_reqs) / peak_wall
    s1 = server.stats()

    def per_batch(a, b):
        nb = max(1, b["batches"] - a["batches"])
        return {"batches": b["batches"] - a["batches"], "tiles_per_batch": (b["completed"] - a["completed"]) / nb,
                "build_us": (b["build_us_total"] - a["build_us_total"]) / nb,
                "gpu_us": (b["gpu_us_total"] - a["gpu_us_total"]) / nb,
                "flight_us": (b["flight_us_total"] - a["flight_us_total"]) / nb}

    rates = [float(x) for x in args.rates.split(",") if x]
    per_rate = []
    for k, lam in enumerate(rates):
        n = int(max(200, min(lam * args.seconds, 40000)))
        reqs, px = make_requests(n, 100 + k)
        gaps = np.random.default_rng(200 + k).exponential(1.0 / lam, size=n)
        gaps[0] = 0.0
        sa = server.stats()
        with Clocks(local) as clk:
            lat, wall, ok = run(reqs, gaps, check=8)
        sb = server.stats()
        tps = n / wall
        per_rate.append({"rate_tiles_s": lam, "requests": n, "throughput_tiles_s": tps,
                         "throughput_mpix_s": sum(px) / wall / 1e6,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "max_ms": float(lat.max()), "parity_sample_ok": ok, "clocks": clk.summary(),
                         "per_batch": per_batch(sa, sb)})
    # Peak batched throughput: the larger of the closed-loop run and the best
    # rate the open-loop sweep sustained.
    peak_ref = max([peak_tps] + [r["throughput_tiles_s"] for r in per_rate])
    for r in per_rate:
        r["frac_of_peak"] = r["throughput_tiles_s"] / peak_ref
    st = server.stats()
    server.close()
    if rank == 0:
        best = [r for r in per_rate if r["p99_ms"] <= 5.0]
        line = {
            "metric": "serving: tiles/s and p50/p99 tile latency per arrival rate (continuous batching)",
            "value": max((r["throughput_tiles_s"] for r in best), default=None), "unit": "tiles/s",
            "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"serving pool of {len(pool)} uneven RGB8 tiles (sides 128..1024), requests 60% "
                                   "full RGB8 / 25% quarter resolution / 15% 256x256 region, Poisson arrivals, "
                                   "16 GiB admission budget, codestreams resident on the device",
                       "pool_coded_bytes": coded, "slots": args.slots, "max_batch_tiles": args.max_batch,
                       "max_batch_samples": args.max_batch_samples},
            "peak_tiles_s": peak_ref,
            "peak_closed_loop": {"throughput_tiles_s": peak_tps, "throughput_mpix_s": sum(peak_px) / peak_wall / 1e6,
                                 "requests": len(peak_reqs), "parity_sample_ok": ok_peak,
                                 "per_batch": per_batch(s0, s1),
                                 "clocks": clk_peak.summary()},
            "per_rate": per_rate,
            "server_stats": st,
        }
        print(json.dumps(line), flush=True)


def reduce_max(dist, x, device):
    """Max of a per-rank scalar over all ranks (the timed region's duration is
    the slowest replica's); identity without a process group."""
    if not dist:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, ms):
    """Whole-job rate (units/s, in millions) of `world` replicas that each
    processed units_per_rank in `ms` milliseconds (max over ranks)."""
    return world * units_per_rank / (ms / 1000.0) / 1e6


def traffic_for(workload, kernel):
    """dram bytes per launch of `kernel` from the committed ncu summary."""
    p = ROOT / "profiles" / "dram_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload and parts[1] == kernel:
            return float(parts[2])
    return None


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4":
        return run_serving(args)
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from signinum_b200 import j2k_cuda
    from signinum_b200.plan import Plan

    ctx = j2k_cuda._Context.open(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    w, kind = build_workload(args.workload)
    fmt = 1 if kind == "rgb8" else 3
    bpp = 3 if kind == "rgb8" else 2
    tiles = w.tiles
    n = len(tiles)
    pixels = w.pixels()
    coded = w.coded_bytes()
    out_bytes = sum(t.width * t.height * bpp for t in tiles)
    # Pinned, contiguous codestreams (16-byte aligned) for the H2D path.
    offs, pos = [], 0
    for t in tiles:
        offs.append(pos)
        pos += (len(t.codestream) + 15) & ~15
    pinned = torch.empty(pos, dtype=torch.uint8, pin_memory=True)
    host = pinned.numpy()
    for o, t in zip(offs, tiles):
        host[o:o + len(t.codestream)] = np.frombuffer(t.codestream, np.uint8)
    lens = [len(t.codestream) for t in tiles]

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(dist, x, "cuda")

    # ---- Batched, device-resident (value).
    plan = Plan(lens, fmt, ctx=ctx, contiguous=host, offsets=offs)
    # Launch shape chosen by the autotuner on this plan's data (untimed).
    tune = None if args.no_autotune else plan.autotune(5)
    # Per-stage breakdown with the tuned shape (events between stages; untimed).
    stages = [plan.execute_timed() for _ in range(3)]
    # Warm-up: the first execution runs eagerly, the second captures the plan
    # as a CUDA graph; timed steps replay the graph.
    for _ in range(args.warmup):
        plan.execute_async()
    st, per = plan.wait()
    assert st == 0, f"decode failed: {st}"
    barrier()
    with Clocks(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            plan.execute_async()
        ev1.record(stream)
        ev1.synchronize()
    barrier()
    batched_ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    stage = np.mean(np.array(stages), axis=0)  # VLC, MagSgn, refine, IDWT, pack, total
    launches = plan.launches * args.steps
    value = replica_throughput(world, pixels, batched_ms)
    # Parity spot check of the benchmark output against the oracle.
    check = None
    if rank == 0:
        from oracle import oracle

        idx = [0, n // 2, n - 1]
        check = all(plan.download(i) == oracle.decode(tiles[i].codestream, fmt)[0] for i in idx)

    # ---- Plain per-tile path (one tile per call), device-resident and e2e.
    plain = {}
    if not args.no_plain:
        tplans = [Plan([lens[i]], fmt, ctx=ctx, contiguous=host[offs[i]:offs[i] + ((lens[i] + 15) & ~15)],
                       offsets=[0]) for i in range(n)]
        for p in tplans[: min(8, n)]:
            p.execute_async()
            p.wait()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for p, (e0, e1) in zip(tplans, evs):
            e0.record(stream)
            p.execute_async()
            e1.record(stream)
            p.wait()
        a1.record(stream)
        a1.synchronize()
        lat = [e0.elapsed_time(e1) for e0, e1 in evs]
        plain_ms = max_over_ranks(a0.elapsed_time(a1))
        for p in tplans:
            p.destroy()
        # e2e plain: the drop-in call from pinned host memory, one tile per call.
        import ctypes

        from signinum_b200 import _native
        from signinum_b200._native import SgnRequest, SgnSurface

        lib = _native.cuda_lib()
        req = SgnRequest(0, 0, 0, 0, 0, 1)
        barrier()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        e2e_lat = []
        b0.record(stream)
        for i in range(n):
            s = SgnSurface()
            t0 = time.perf_counter()
            rc = lib.sgn_j2k_decode_to_device(ctx.handle, host.ctypes.data + offs[i], lens[i], fmt,
                                              ctypes.byref(req), 3, ctypes.byref(s))
            e2e_lat.append((time.perf_counter() - t0) * 1000.0)
            assert rc == 0
            lib.sgn_surface_free(ctx.handle, ctypes.byref(s))
        b1.record(stream)
        b1.synchronize()
        plain_e2e_ms = max_over_ranks(b0.elapsed_time(b1))
        plain = {"plain_mpix_s": world * pixels / (plain_ms / 1000.0) / 1e6,
                 "plain_tile_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                 "plain_e2e_mpix_s": world * pixels / (plain_e2e_ms / 1000.0) / 1e6,
                 "plain_e2e_tile_latency_ms": {"p50": float(np.percentile(e2e_lat, 50)),
                                               "p99": float(np.percentile(e2e_lat, 99))}}
        plain["batched_over_plain"] = value / plain["plain_mpix_s"]

    # ---- e2e batched: decode_tiles_to_device from pinned host buffers.
    import ctypes

    from signinum_b200 import _native
    from signinum_b200._native import SgnSurface

    lib = _native.cuda_lib()
    ptrs = (ctypes.c_void_p * n)(*[host.ctypes.data + o for o in offs])
    clens = (ctypes.c_size_t * n)(*lens)
    per_tile = (ctypes.c_int32 * n)()
    first = ctypes.c_size_t()

    def e2e_step():
        outs = (SgnSurface * n)()
        rc = lib.sgn_j2k_decode_tiles_to_device(ctx.handle, ptrs, clens, n, fmt, None, 3, outs, per_tile,
                                                ctypes.byref(first))
        assert rc == 0, rc
        return outs

    for _ in range(max(3, args.warmup)):
        outs = e2e_step()
        for i in range(n):
            lib.sgn_surface_free(ctx.handle, ctypes.byref(outs[i]))
    barrier()
    e2e_ms_list = []
    for _ in range(max(1, min(args.steps, 10))):
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        outs = e2e_step()
        c1.record(stream)
        c1.synchronize()
        e2e_ms_list.append(c0.elapsed_time(c1))
        for i in range(n):
            lib.sgn_surface_free(ctx.handle, ctypes.byref(outs[i]))
    e2e_ms = max_over_ranks(float(np.mean(e2e_ms_list)))
    e2e_val = world * pixels / (e2e_ms / 1000.0) / 1e6

    if rank == 0:
        names = ["ht_vlc_kernel", "ht_magsgn_kernel", "ht_refine_kernel", "idwt_level_kernel", "pack_kernel"]
        if args.workload == "c1i":
            names[3:] = ["idwt97_level_kernel", "pack97_kernel"]
        if args.workload == "c1c":
            names[2] = "classic_kernel"  # the classic blocks run in the refinement stage's slot
        dom = int(np.argmax(stage[:5]))
        peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
        peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
        algo = coded + out_bytes
        achieved = algo / (stage[dom] / 1000.0) / 1e9
        traffic = traffic_for(args.workload, names[dom])
        cpu = None if args.no_cpu else cpu_baseline(tiles, fmt)
        line = {
            "metric": "decoded Mpixel/s (batched persistent form; plain per-tile beside it)",
            "value": value, "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": batched_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32 (HT), f32 (9/7, ICT)" if args.workload == "c1i" else "int32", "data": "synthetic (seeded)",
            "config": dict(WORKLOAD_CONFIG[args.workload], parallelism=f"replicas{world}",
                           l2="inputs larger than L2 (coded + coefficient arenas), no flush",
                           coded_bytes=coded, output_bytes=out_bytes, pixels=pixels),
            "compressed_MB_s": world * coded / (batched_ms / 1000.0) / 1e6,
            "hbm_roofline_frac_path": (world * algo / (batched_ms / 1000.0) / 1e9) / peak,
            "stage_ms": {"ht_vlc": stage[0], "ht_magsgn": stage[1],
                         ("classic_blocks" if args.workload == "c1c" else "ht_refine"): stage[2], "idwt_levels": stage[3],
                         "last_level_pack": stage[4], "total": stage[5]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": names[dom],
                         "peak_source": "measured" if PEAKS.exists() else "fallback",
                         "algorithmic_bytes_per_launch": algo},
            "e2e": {"value": e2e_val, "unit": "Mpixel/s", "h2d_bytes_per_step": pos,
                    "d2h_bytes_per_step": 4 * n, "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "autotune": tune,
            "execution": "CUDA graph replay of the autotuned plan",
            "clocks": clk.summary(),
            "parity_spot_check": check,
        }
        line.update(plain)
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    plan.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
