"""Benchmark of the B200 transform-batch hot path: dense classify + exact plan + scatter of
N = 1e8 u32 keys into pooled output chunks (C = 8192), one whole-array batch per step.

  value   fused single-pass form (one classify->plan->scatter launch that also writes the chunk
          table and descriptors: gf_partition_fused_full_u32), inputs
          resident in HBM; particles/s summed over all ranks (weak scaling: every rank
          partitions its own 1e8 keys; the path has no exchange step, so no collective).
  plain   the reference's two-launch form (classify, host plan, scatter) on the same data.
  e2e     the same step through the C ABI from pinned host buffers: H2D of the keys, fused
          partition, D2H of the output chunks and descriptors, every step inside the timed
          region; a step's upload overlaps the previous step's download (full-duplex link).

``--impl reference`` times the reference algorithm's CPU restatement (the oracle's pool path:
per-tile histogram -> plan -> scatter, OpenMP over all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_KEYS = 100_000_000
CAPACITY = 8192
SEED = 42
HEADLINE_BINS = 64
HEADLINE_DIST = "uniform"
BYTES_PER_PARTICLE = 8  # read the 4-byte key once, write it once (algorithmic)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per key of one launch of the
# cooperative kernel, from an ncu capture of the 5e7-key case with B = 64 uniform keys (traffic
# grows in proportion to the keys, so it scales to a full launch); None for other workloads.
MEASURED_TRAFFIC_PER_KEY = {(64, "uniform"): 10.11}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--tile", type=int, default=4096)
    p.add_argument("--bins", type=int, default=HEADLINE_BINS)
    p.add_argument("--dist", default=HEADLINE_DIST)
    p.add_argument("--n", type=int, default=N_KEYS)
    p.add_argument("--no-sweep", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the other configurations' measurements")
    p.add_argument("--hash", type=int, default=0, metavar="K",
                   help="only run the device-planned hash partition of --n records over K keys (Zipf 1.2, "
                        "tiles of 2048) --steps times after --warmup batches and print its timing; for profiling")
    p.add_argument("--device-chain", type=int, default=0, metavar="NODES",
                   help="one run of the dense chain entirely on the device (gf_run_dense_chain_device) at N=--n, "
                        "B=--bins (profiling)")
    p.add_argument("--feedback-device-resident", action="store_true",
                   help="one particle_feedback run through the Flow device-resident at N=--n, C=8192 (profiling)")
    p.add_argument("--photon-device-resident", action="store_true",
                   help="one photon run through the Flow device-resident at N=--n (profiling)")
    p.add_argument("--flow-chain", type=int, default=0, metavar="NODES",
                   help="only run the dense chain of NODES partition nodes through the Flow on --n keys (--bins, "
                        "--dist, C=8192, P=16384, Q=8, partition groups) and print its counters; for profiling")
    return p.parse_args()


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.path, self.start = index, None, None, None

    def __enter__(self):
        import shutil
        try:
            self.path = f"/tmp/gf_clocks_{os.getpid()}.csv"
            self.f = open(self.path, "w")
            cmd = ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                   "-lms", "20"]
            if shutil.which("stdbuf"):  # one line per sample reaches the file at once
                cmd = ["stdbuf", "-oL"] + cmd
            self.proc = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def _lines(self):
        try:
            with open(self.path) as f:
                return f.readlines()
        except OSError:
            return []

    def begin(self, timeout=3.0):
        """Wait for the first sample, then count only the samples from here on."""
        if self.proc is None:
            return
        t = time.perf_counter()
        while not self._lines() and time.perf_counter() - t < timeout and self.proc.poll() is None:
            time.sleep(0.01)
        self.start = len(self._lines())

    def __exit__(self, *a):
        import signal
        if self.proc is not None:
            self.proc.send_signal(signal.SIGINT)  # lets nvidia-smi flush and exit
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self._lines()
        if self.start is not None and len(lines) > self.start:
            lines = lines[self.start:]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------------
# CPU arms (oracle = the reference algorithm restated in C; test infrastructure, used here only
# as the timed CPU baseline)
# ------------------------------------------------------------------------------------------------
def cpu_pool_pass(n, bins, dist, threads=0, reps=3):
    import numpy as np
    from oracle import oracle as O
    keys = O.generate_keys_u32(dist, SEED, n, bins, zipf_s=1.1, threads=threads)
    n_in = -(-n // CAPACITY)
    bound = O.output_chunk_bound(n, CAPACITY, bins)
    pool_in = np.zeros((n_in + bound) * CAPACITY, np.uint32)
    pool_in[:n] = keys
    fills = np.full(n_in, CAPACITY, np.uint32)
    fills[-1] = n - CAPACITY * (n_in - 1)
    tiles = O.flatten_tiles(np.arange(n_in, dtype=np.uint32), fills, 128)  # the reference's T = 128
    free = np.arange(n_in, n_in + bound, dtype=np.uint32)
    pool_out = pool_in.copy()
    bin_ids = np.zeros_like(pool_in)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.partition_pool_u32(pool_in, CAPACITY, tiles, bins, free, threads=threads, pool_out=pool_out,
                             bin_ids=bin_ids)
        times.append(time.perf_counter() - t0)
    return n / statistics.median(times), statistics.median(times)


class Ranks:
    """One process per device, as torchrun starts them: rank and world from the environment, a
    barrier and the max over ranks (NCCL on GPUs; gloo works the same way on CPU)."""

    def __init__(self, backend="nccl", device=None, timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_value(n_per_rank, world, ms):
    """Particles per second of the whole job: every rank partitions its own n_per_rank keys and the
    step takes the slowest rank's ms (weak scaling)."""
    return world * n_per_rank / (ms / 1e3)


REFERENCE_ARM_SECONDS = 90.0  # the reference arm's whole --steps/--warmup run stays near this


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    threads = O.cpu_threads()
    import numpy as np
    # each step is a bounded sample of the workload: size it from one probe step so that the whole
    # run of warmup + steps takes about REFERENCE_ARM_SECONDS
    probe = min(args.n, 1_000_000)
    pk = O.generate_keys_u32(args.dist, SEED, probe, args.bins, zipf_s=1.1, threads=threads)
    pn_in = -(-probe // CAPACITY)
    pbound = O.output_chunk_bound(probe, CAPACITY, args.bins)
    ppool = np.zeros((pn_in + pbound) * CAPACITY, np.uint32)
    ppool[:probe] = pk
    pfills = np.full(pn_in, CAPACITY, np.uint32)
    pfills[-1] = probe - CAPACITY * (pn_in - 1)
    ptiles = O.flatten_tiles(np.arange(pn_in, dtype=np.uint32), pfills, 128)
    pfree = np.arange(pn_in, pn_in + pbound, dtype=np.uint32)
    O.partition_pool_u32(ppool, CAPACITY, ptiles, args.bins, pfree, threads=threads, pool_out=ppool.copy())
    t0 = time.perf_counter()
    O.partition_pool_u32(ppool, CAPACITY, ptiles, args.bins, pfree, threads=threads, pool_out=ppool.copy())
    per_key = max((time.perf_counter() - t0) / probe, 1e-10)
    budget = REFERENCE_ARM_SECONDS / max(args.steps + args.warmup, 1)
    n = int(min(args.n, max(100_000, budget / per_key)))
    keys = O.generate_keys_u32(args.dist, SEED, n, args.bins, zipf_s=1.1, threads=threads)
    n_in = -(-n // CAPACITY)
    bound = O.output_chunk_bound(n, CAPACITY, args.bins)
    pool_in = np.zeros((n_in + bound) * CAPACITY, np.uint32)
    pool_in[:n] = keys
    fills = np.full(n_in, CAPACITY, np.uint32)
    fills[-1] = n - CAPACITY * (n_in - 1)
    tiles = O.flatten_tiles(np.arange(n_in, dtype=np.uint32), fills, 128)
    free = np.arange(n_in, n_in + bound, dtype=np.uint32)
    pool_out = pool_in.copy()
    bin_ids = np.zeros_like(pool_in)
    for _ in range(args.warmup):
        O.partition_pool_u32(pool_in, CAPACITY, tiles, args.bins, free, threads=threads, pool_out=pool_out,
                             bin_ids=bin_ids)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.partition_pool_u32(pool_in, CAPACITY, tiles, args.bins, free, threads=threads, pool_out=pool_out,
                             bin_ids=bin_ids)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    value = n / dt
    sample = (f"{n} of the workload's {args.n} u32 keys per step (B={args.bins} {args.dist}, C={CAPACITY}, "
              f"T=128 tiles; classify->plan->scatter over a chunk pool), sized so the run takes about "
              f"{REFERENCE_ARM_SECONDS:.0f} s")
    print(json.dumps({
        "impl": "reference", "metric": "particles/s", "value": value, "unit": "particles/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Philox keys)",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def workload_config(args):
    return {"workload": f"dense classify+plan+scatter, N={args.n:.0e} u32 keys, B={args.bins}, {args.dist}, "
                        f"C={CAPACITY}, one batch",
            "n": args.n, "bins": args.bins, "dist": args.dist, "capacity": CAPACITY, "tile": args.tile,
            "l2": (f"input and output {args.n * 4 / 1e6:.0f} MB each, "
                   + ("above the 126 MB L2: no flush" if args.n * 4 > 126e6 else "within L2"))}


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------
class DenseBench:
    """Device-resident setup of one whole-array batch (input chunks 0..n_in-1, a contiguous
    reservation of outputChunkBound chunks behind them)."""

    def __init__(self, n, bins, dist, tile, device):
        import numpy as np
        import torch
        from graphflow_b200 import capi
        from graphflow_b200.partition import ChunkPool, FusedPartition, PlainPartition
        self.torch, self.capi, self.np = torch, capi, np
        self.n, self.bins, self.dist, self.tile = n, bins, dist, tile
        self.n_in = -(-n // CAPACITY)
        self.bound = capi.output_chunk_bound(n, CAPACITY, bins)
        self.pool = ChunkPool(self.n_in + self.bound, CAPACITY, device=device)
        cdf = torch.from_numpy(capi.zipf_cdf(1.1, bins)).to(device) if dist == "zipf" else None
        capi.check(capi.lib().gf_generate_keys_u32(None, capi.DIST_NAMES[dist], SEED, 0, n, bins,
                                                   cdf.data_ptr() if cdf is not None else None,
                                                   self.pool.column.data_ptr()), "generate")
        self.fills = np.full(self.n_in, CAPACITY, np.uint32)
        self.fills[-1] = n - CAPACITY * (self.n_in - 1)
        self.chunks = np.arange(self.n_in, dtype=np.uint32)
        for _ in range(self.n_in):
            self.pool.free.popleft()
        self.fused = FusedPartition(self.pool, bins, tile_size=tile, max_batch_particles=n)
        tiles, self.d_tiles = self.fused._tiles(self.chunks, self.fills)
        self.n_tiles = len(tiles)
        reserved = np.arange(self.n_in, self.n_in + self.bound, dtype=np.uint32)
        self.fused.reserved[:self.bound].copy_(torch.from_numpy(reserved.view(np.int32)))
        self.plain = PlainPartition(self.pool, bins, tile_size=tile)
        torch.cuda.synchronize()

    def fused_step(self, stream):
        self.fused.enqueue(self.d_tiles, self.n_tiles, self.bound, stream)

    def plain_step(self, stream):
        totals, table, descs = self.plain.run(self.chunks, self.fills, stream)
        self.pool.release([int(c) for c in descs[:, 0]])

    def _gather(self, descs):
        """Output keys in descriptor (port) order and each key's port, on the device."""
        torch = self.torch
        d = torch.from_numpy(descs.astype(self.np.int64)).to(self.pool.column.device)
        rows = self.pool.column.view(-1, CAPACITY)[d[:, 0]]
        valid = torch.arange(CAPACITY, device=d.device)[None, :] < d[:, 1:2]
        return rows[valid], torch.repeat_interleave(d[:, 2], d[:, 1])

    def _expected(self):
        """The stable partition of the input keys by key mod B (a torch restatement on the device,
        not the product path): per-port totals and the keys in port order, input order inside a
        port."""
        torch = self.torch
        keys = self.pool.column[: self.n]
        port = (keys.to(torch.int64) & 0xFFFFFFFF) % self.bins
        order = torch.argsort(port, stable=True)
        return torch.bincount(port, minlength=self.bins), keys[order], port[order]

    def check(self, totals, descs, status, exact_order):
        """Every output slot of the batch against the expected partition: totals, each output
        chunk's port and fill (the plan), and each port's keys (the sequence for the fused form, the
        multiset for the plain form, whose in-port order is atomic order)."""
        np, torch = self.np, self.torch
        if status != 0 or int(np.asarray(totals, np.uint64).sum()) != self.n:
            return False
        exp_tot, exp_keys, exp_port = self._expected()
        if not np.array_equal(np.asarray(totals, np.int64), exp_tot.cpu().numpy()):
            return False
        got_keys, got_port = self._gather(descs)
        if got_keys.numel() != self.n or not torch.equal(got_port, exp_port):
            return False
        if exact_order:
            return bool(torch.equal(got_keys, exp_keys))
        m = 0xFFFFFFFF
        a = torch.sort((got_port << 32) | (got_keys.to(torch.int64) & m)).values
        b = torch.sort((exp_port << 32) | (exp_keys.to(torch.int64) & m)).values
        return bool(torch.equal(a, b))

    def check_fused(self):
        np = self.np
        r = int(self.fused.num_out.item())
        descs = self.fused.descs.cpu().numpy().view(np.uint32)[:3 * r].reshape(-1, 3)
        return self.check(self.fused.totals.cpu().numpy().view(np.uint32), descs, int(self.fused.status.item()), True)


def gpu_arm(args):
    import numpy as np
    import torch
    from graphflow_b200 import capi

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks("nccl", dev)
    world, rank = ranks.world, ranks.rank
    barrier, max_over_ranks = ranks.barrier, ranks.max

    stream = torch.cuda.Stream(device=dev)
    bench = DenseBench(args.n, args.bins, args.dist, args.tile, dev)

    # -------- fused (value) --------
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            bench.fused_step(stream)
    stream.synchronize()
    correct = bench.check_fused()
    k_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    k_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        clocks.begin()
        with torch.cuda.stream(stream):
            t_start.record(stream)
            for i in range(args.steps):
                # one step: the fused partition and its finish in one launch (+ the control-block reset)
                k_start[i].record(stream)
                capi.check(capi.lib().gf_partition_fused_full_u32(
                    stream.cuda_stream, bench.pool.ptr(), bench.pool.ptr(), CAPACITY, bench.pool.slots,
                    bench.d_tiles.data_ptr(), bench.n_tiles, args.tile, args.bins, capi.CLS_KEY_MOD,
                    bench.fused.reserved.data_ptr(), bench.bound, bench.fused.totals.data_ptr(),
                    bench.fused.port_chunks.data_ptr(), bench.fused.max_k, bench.fused.scratch.data_ptr(),
                    bench.fused.scratch_bytes, bench.fused.table.data_ptr(), bench.fused.descs.data_ptr(),
                    bench.fused.reserve_cap, bench.fused.num_out.data_ptr(), bench.fused.status.data_ptr()),
                    "fused")
                k_end[i].record(stream)
            t_end.record(stream)
        stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(t_start.elapsed_time(t_end) / args.steps)
    kernel_ms = statistics.mean(a.elapsed_time(b) for a, b in zip(k_start, k_end))
    correct &= bench.check_fused()
    value = whole_job_value(args.n, world, ms)

    # -------- the per-tile fused kernel (no bulk-copy pipeline) on the same data, for comparison --------
    capi.check(capi.lib().gf_set_tuning(b"fused_coop", 0), "tuning")
    with torch.cuda.stream(stream):
        for _ in range(3):
            bench.fused_step(stream)
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        v0.record(stream)
        for _ in range(20):
            bench.fused_step(stream)
        v1.record(stream)
    stream.synchronize()
    capi.check(capi.lib().gf_set_tuning(b"fused_coop", 1), "tuning")
    per_tile_ms = v0.elapsed_time(v1) / 20
    correct &= bench.check_fused()

    # -------- plain (reference's two-launch form) --------
    # every rank runs it: the max over ranks is a collective
    for _ in range(max(1, args.warmup // 2)):
        bench.plain_step(stream)
    stream.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(3, min(args.steps // 4, 100))
    p0.record(stream)
    for _ in range(reps):
        bench.plain_step(stream)
    p1.record(stream)
    stream.synchronize()
    plain_ms = max_over_ranks(p0.elapsed_time(p1) / reps)
    totals, _, pdescs = bench.plain.run(bench.chunks, bench.fills, stream)
    plain_correct = bench.check(totals, pdescs, 0, False)
    bench.pool.release([int(c) for c in pdescs[:, 0]])

    # -------- e2e through the C ABI from pinned host buffers --------
    host_keys = torch.empty(args.n, dtype=torch.int32, pin_memory=True)
    host_keys.copy_(bench.pool.column[: args.n].cpu())
    out_slots = bench.bound * CAPACITY
    host_out = torch.empty(out_slots, dtype=torch.int32, pin_memory=True)
    host_descs = torch.empty(3 * bench.fused.reserve_cap, dtype=torch.int32, pin_memory=True)
    host_small = torch.empty(2, dtype=torch.int32, pin_memory=True)
    out_view = bench.pool.column[bench.n_in * CAPACITY: bench.n_in * CAPACITY + out_slots]

    # Every step uploads its keys, runs the fused step and reads back its output, descriptors and
    # status. Consecutive steps overlap on the full-duplex host link: step k+1's upload (copy
    # stream) waits only for step k's kernel, which has finished reading the input chunks, and runs
    # while step k's download (compute stream) drains the output chunks; step k+1's kernel waits
    # for its upload and, in stream order, for step k's download.
    copy_stream = torch.cuda.Stream(device=dev)

    def e2e_steps(count, start):
        prev = start
        for _ in range(count):
            copy_stream.wait_event(prev)
            with torch.cuda.stream(copy_stream):
                bench.pool.column[: args.n].copy_(host_keys, non_blocking=True)
                up = torch.cuda.Event()
                up.record(copy_stream)
            stream.wait_event(up)
            with torch.cuda.stream(stream):
                bench.fused_step(stream)
                prev = torch.cuda.Event()
                prev.record(stream)
                host_out.copy_(out_view, non_blocking=True)
                host_descs.copy_(bench.fused.descs, non_blocking=True)
                host_small[0:1].copy_(bench.fused.num_out, non_blocking=True)
                host_small[1:2].copy_(bench.fused.status, non_blocking=True)

    warm = torch.cuda.Event()
    warm.record(stream)
    e2e_steps(2, warm)
    stream.synchronize()
    e_reps = max(3, min(args.steps // 4, 50))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps(e_reps, e0)
    e1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e_reps)
    correct &= int(host_small[1].item()) == 0

    # -------- sweep (fused, every B x distribution of the kernel-level config) --------
    sweep = []
    if not args.no_sweep:
        del bench
        torch.cuda.empty_cache()
        for b in (2, 8, 32, 64):
            for d in ("uniform", "zipf", "one_port", "round_robin"):
                sb = DenseBench(args.n, b, d, args.tile, dev)
                with torch.cuda.stream(stream):
                    for _ in range(2):
                        sb.fused_step(stream)
                    stream.synchronize()
                    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s0.record(stream)
                    for _ in range(5):
                        sb.fused_step(stream)
                    s1.record(stream)
                    stream.synchronize()
                sms = s0.elapsed_time(s1) / 5
                ok = sb.check_fused()
                sweep.append({"bins": b, "dist": d, "ms": round(sms, 4), "particles_per_s": args.n / (sms / 1e3),
                              "hbm_frac": round(args.n * BYTES_PER_PARTICLE / (sms / 1e3) / 1e9 /
                                                measured_peak()[0], 4), "correct": ok})
                del sb
                torch.cuda.empty_cache()

    peak, peak_kind = measured_peak()
    achieved = args.n * BYTES_PER_PARTICLE / (kernel_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import oracle as O
        threads = O.cpu_threads()
        sample_n = min(args.n, 20_000_000)
        v, t = cpu_pool_pass(sample_n, args.bins, args.dist, threads=threads)
        cpu = {"value": v, "unit": "particles/s", "cores": threads, "kind": "port",
               "sample": f"{sample_n:.0e} keys, same B/dist/C, median of 3 pool passes ({t:.3f} s)"}
    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        extra = other_configs(peak)
    ranks.close()
    if rank != 0:
        return
    line = {
        "metric": "particles/s", "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Philox keys)",
        "config": workload_config(args),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (MEASURED_TRAFFIC_PER_KEY[(args.bins, args.dist)] * args.n
                                 if (args.bins, args.dist) in MEASURED_TRAFFIC_PER_KEY and args.tile <= 4096 else None),
                     "traffic_source": "ncu, 5e7 keys, scaled", "peak_source": peak_kind,
                     "kernel": ("fused_partition_coop_bulk_kernel" if args.bins <= 16 else "fused_partition_coop_kernel"),
                     "kernel_ms": kernel_ms,
                     "algorithmic_bytes": f"{BYTES_PER_PARTICLE} B/particle"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * args.n / (e2e_ms / 1e3), "unit": "particles/s",
                "h2d_bytes_per_step": args.n * 4,
                "d2h_bytes_per_step": out_slots * 4 + 3 * 4 * bench_reserve_cap(args) + 8},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps,  # one fused_partition_coop_kernel launch per timed step
        "fused_per_tile_kernel": {"value": world * args.n / (per_tile_ms / 1e3), "ms_per_step": per_tile_ms},
        "plain": {"value": world * args.n / (plain_ms / 1e3), "ms_per_step": plain_ms, "correct": plain_correct,
                  "form": "classify, host plan, scatter"},
        # every output slot of the timed batch (and of every sweep case) against the stable partition
        "correct": bool(correct and plain_correct and all(e["correct"] for e in sweep)),
        "correct_check": "all slots vs a stable partition",
    }
    if sweep:
        fr = [e["hbm_frac"] for e in sweep]
        line["sweep"] = {"cases": len(sweep), "hbm_frac_min": min(fr), "hbm_frac_max": max(fr),
                         "ms_min": min(e["ms"] for e in sweep), "ms_max": max(e["ms"] for e in sweep),
                         "all_correct": all(e["correct"] for e in sweep)}
    if extra is not None:
        # the full record of the other configurations first, on its own line; the result line last
        print("# configs " + json.dumps({"sweep": sweep, "configs": extra}), flush=True)
        line["serving"] = extra.get("serving", {}).get("summary")
        chain = extra.get("dense_flow", {}).get("nodes4_device_chain")
        if chain:
            line["dense_chain_4nodes_1e8_on_device"] = {"particles_per_s": chain["particles_per_s"],
                                                        "all_chunks_free": chain["all_chunks_free"]}
    print(json.dumps(_compact(line), separators=(",", ":")), flush=True)


def _compact(obj, keep=("value", "ms_per_step")):
    """The result line with every float but the headline figures rounded to 4 significant digits,
    so that the whole line stays short."""
    def walk(x, top):
        if isinstance(x, dict):
            return {k: (v if top and k in keep else walk(v, False)) for k, v in x.items()}
        if isinstance(x, list):
            return [walk(v, False) for v in x]
        if isinstance(x, float) and x != 0.0 and math.isfinite(x):
            return float(f"{x:.4g}")
        return x
    return walk(obj, True)


# ------------------------------------------------------------------------------------------------
# The other configurations (bounded samples; each entry states its size)
# ------------------------------------------------------------------------------------------------
def _timed(f):
    import torch
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = f()
    torch.cuda.synchronize()
    return r, time.perf_counter() - t


def _cfg_particle_feedback():
    """particle_feedback: N = 1e6, seed 42, C = 1024, P = 4096, Q = 1, 64 visits; the sorted weight
    histogram must match the oracle's scalar model row for row and sum to N."""
    import numpy as np
    from graphflow_b200 import capi
    from oracle import oracle as O
    n = 1_000_000
    out = {"workload": "particle_feedback N=1e6 seed 42 C=1024 P=4096 Q=1 maxVisits=64"}
    (w, c, st), _ = _timed(lambda: capi.run_particle_feedback(42, n, chunk_capacity=1024, live_particles=4096,
                                                             batch_chunks=1, fused=True))
    out["flow_fused"] = {"seconds": st.seconds, "particles_per_s": n / st.seconds,
                         "partition_batches": st.partition_batches, "partition_launches": st.partition_launches,
                         "kernel_launches": st.kernel_launches, "form": "partition groups (B200 runner)"}
    capi.check(capi.lib().gf_set_tuning(b"group_partitions", 0), "tuning")
    try:
        (_, _, su), _ = _timed(lambda: capi.run_particle_feedback(42, n, chunk_capacity=1024, live_particles=4096,
                                                                 batch_chunks=1, fused=True))
    finally:
        capi.check(capi.lib().gf_set_tuning(b"group_partitions", 1), "tuning")
    out["flow_fused_one_node_per_partition"] = {"seconds": su.seconds, "particles_per_s": n / su.seconds,
                                                "partition_batches": su.partition_batches,
                                                "partition_launches": su.partition_launches}
    capi.check(capi.lib().gf_set_tuning(b"runner_batched", 0), "tuning")
    try:
        (w0, c0, st0), _ = _timed(lambda: capi.run_particle_feedback(42, n, chunk_capacity=1024, live_particles=4096,
                                                                    batch_chunks=1, fused=False))
    finally:
        capi.check(capi.lib().gf_set_tuning(b"runner_batched", 1), "tuning")
    out["flow_plain_reference_runner"] = {"seconds": st0.seconds, "particles_per_s": n / st0.seconds}
    threads = O.cpu_threads()
    ref, cpu_s = _timed(lambda: O.particle_scalar(42, n, 64, threads=threads))
    vals, counts = np.unique(w, return_counts=True)
    exp_vals, exp_counts = O.histogram_u32(ref[0])
    out["histogram_rows"] = int(len(vals))
    out["histogram_sum"] = int(counts.sum())
    out["histogram_matches_oracle"] = bool(np.array_equal(vals, exp_vals) and np.array_equal(counts, exp_counts))
    out["forms_identical"] = bool(np.array_equal(w, w0) and np.array_equal(c, c0))
    out["cpu_scalar_model"] = {"seconds": cpu_s, "particles_per_s": n / cpu_s, "cores": threads,
                               "kind": "port (tests/reference/ScalarModel.hpp restated: per-particle loop, no runner)"}
    # the reference's published configuration (docs/benchmarks.md:24-34: N=1e8, C=8192, P=16384,
    # Q=8, 1.3e7 particles/s on a V100) through the same Flow; its sorted weight,count rows must
    # hash to the SHA-256 the reference published
    import hashlib
    n8 = 100_000_000
    w8, _, st8 = capi.run_particle_feedback(42, n8, chunk_capacity=8192, live_particles=16384, batch_chunks=8)
    v8, c8 = O.histogram_u32(w8)
    text = "".join(f"{int(v)},{int(c)}\n" for v, c in zip(v8, c8))
    out["published_config_flow"] = {
        "workload": "particle_feedback N=1e8 seed 42 C=8192 P=16384 Q=8 maxVisits=64 through the Flow",
        "seconds": st8.seconds, "particles_per_s": n8 / st8.seconds, "partition_batches": st8.partition_batches,
        "kernel_launches": st8.kernel_launches, "histogram_rows": int(len(v8)),
        "histogram_sha256_matches_published": hashlib.sha256(text.encode()).hexdigest()
        == "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab",
        "reference_published_particles_per_s": 1.3e7}
    # the same Flow run device-resident (Tuning::deviceResident): Cfg1 and the published configuration
    capi.check(capi.lib().gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        capi.run_particle_feedback(42, 10_000, chunk_capacity=1024, live_particles=4096, batch_chunks=1)
        runs = [capi.run_particle_feedback(42, n, chunk_capacity=1024, live_particles=4096, batch_chunks=1)
                for _ in range(3)]
        runs8 = [capi.run_particle_feedback(42, n8, chunk_capacity=8192, live_particles=16384, batch_chunks=8)
                 for _ in range(3)]
    finally:
        capi.check(capi.lib().gf_set_tuning(b"device_resident", 0), "tuning")
    sd = sorted((r[2] for r in runs), key=lambda x: x.seconds)[1]
    wd8, _, sd8 = sorted(runs8, key=lambda r: r[2].seconds)[1]  # the median run of three
    vd, cd = O.histogram_u32(wd8)
    text_d = "".join(f"{int(v)},{int(c)}\n" for v, c in zip(vd, cd))
    out["flow_device_resident"] = {
        "seconds": sd.seconds, "particles_per_s": n / sd.seconds, "waves": sd.loop_iterations,
        "kernel_launches": sd.kernel_launches,
        "identical_to_host_runner": all(bool(np.array_equal(r[0], w) and np.array_equal(r[1], c)) for r in runs)}
    out["published_config_flow_device_resident"] = {
        "seconds": sd8.seconds, "particles_per_s": n8 / sd8.seconds, "waves": sd8.loop_iterations,
        "kernel_launches": sd8.kernel_launches, "peak_live_chunks": sd8.peak_live_chunks,
        "pool_chunks": sd8.pool_chunks,
        "histogram_sha256_matches_published": hashlib.sha256(text_d.encode()).hexdigest()
        == "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab"}
    return out


def _cfg_dense_flow():
    """The dense sweep through the public Flow: B = 64 uniform keys, C = 8192, P = 16384, Q = 8, at 1
    node and at 4 chained nodes. The 4-node chain runs with its partition nodes grouped (one
    multi-batch launch drains every node's ready batches) and, for comparison, with one runner node
    per partition node."""
    from graphflow_b200 import capi
    L = capi.lib()
    out = {"workload": "dense chain through Flow, B=64 uniform, C=8192 P=16384 Q=8 (records {u32 id, u32 key})"}

    def run(nodes, n, fused, batched, grouped=True):
        capi.check(L.gf_set_tuning(b"runner_batched", int(batched)), "tuning")
        capi.check(L.gf_set_tuning(b"group_partitions", int(grouped)), "tuning")
        try:
            _, st = capi.run_dense_chain(42, n, 64, nodes=nodes, dist="uniform", chunk_capacity=8192,
                                         live_particles=16384, batch_chunks=8, fused=fused, want_ports=False)
        finally:
            capi.check(L.gf_set_tuning(b"runner_batched", 1), "tuning")
            capi.check(L.gf_set_tuning(b"group_partitions", 1), "tuning")
        return {"n": n, "seconds": st.seconds, "particles_per_s": n / st.seconds,
                "partition_batches": st.partition_batches, "partition_launches": st.partition_launches,
                "kernel_launches": st.kernel_launches, "loop_iterations": st.loop_iterations}
    out["nodes1_fused_b200_runner"] = run(1, 100_000_000, True, True)
    out["nodes1_plain_reference_runner"] = run(1, 10_000_000, False, False)
    out["nodes4_grouped_b200_runner"] = run(4, 100_000_000, True, True, grouped=True)
    out["nodes4_per_node_b200_runner"] = run(4, 1_000_000, True, True, grouped=False)
    out["nodes4_plain_reference_runner"] = run(4, 200_000, False, False)
    # the same chain run entirely on the device (device-resident chunk pool, one launch per node,
    # no host round trip): device time over three runs, and the wall time of the whole call
    capi.check(L.gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        runs4 = [capi.run_dense_chain(42, 100_000_000, 64, nodes=4, dist="uniform", chunk_capacity=8192,
                                      live_particles=16384, batch_chunks=8, want_ports=False)[1] for _ in range(3)]
    finally:
        capi.check(L.gf_set_tuning(b"device_resident", 0), "tuning")
    st = sorted(runs4, key=lambda x: x.seconds)[1]  # the median run of three
    out["nodes4_flow_device_resident"] = {"n": 100_000_000, "seconds": st.seconds,
                                          "particles_per_s": 1e8 / st.seconds, "waves": st.loop_iterations,
                                          "kernel_launches": st.kernel_launches}
    runs = [capi.run_dense_chain_device(42, 100_000_000, 64, nodes=4, want_ports=False) for _ in range(3)]
    dev = sorted(r[3].loop_seconds for r in runs)[1]
    out["nodes4_device_chain"] = {"n": 100_000_000, "device_seconds": dev, "particles_per_s": 1e8 / dev,
                                  "wall_seconds": sorted(r[3].seconds for r in runs)[1],
                                  "kernel_launches": runs[0][3].kernel_launches,
                                  "pool_chunks": runs[0][2].num_chunks, "peak_live_chunks": runs[0][2].peak_live,
                                  "all_chunks_free": all(r[2].free_chunks == r[2].num_chunks for r in runs)}
    return out


def _cfg_hash(peak):
    """Hash partition of N = 1e8 16-byte records {u64 key, f32 weight, u32 tag}, keys over K values
    with Zipf(1.2) popularity; device-planned form (classify -> device plan -> scatter) vs the plain
    form (classify -> host plan -> scatter). Chunk capacity per K keeps the exact plan's chunk
    count (one partial chunk per non-empty port) within memory."""
    import ctypes
    import numpy as np
    import torch
    from graphflow_b200 import capi
    from graphflow_b200.hashpart import HashPartition, RecordPool
    from graphflow_b200.autotune import tune_hash
    n, salt, out = 100_000_000, 0x5EED, {}
    free_bytes = torch.cuda.mem_get_info()[0]
    tuned = {}
    for k in (1 << 10, 1 << 16, 1 << 20):
        # C and tile from the autotuner on a 2e7-record sample, among the capacities whose pool at the
        # full N fits in half the free device memory
        def pool_slots(c):
            return (-(-n // c) + capi.output_chunk_bound(n, c, k)) * c
        caps = tuple(c for c in (512, 1024, 2048, 4096, 8192)
                     if pool_slots(c) < (1 << 32) and pool_slots(c) * 16 <= free_bytes // 2)
        best, table = tune_hash(20_000_000, k, capacities=caps, tiles=(1024, 2048))
        tuned[k] = (best["capacity"], best["tile"])
        out[f"K{k}_autotune"] = {"chosen_C": best["capacity"], "chosen_tile": best["tile"], "sample_n": 20_000_000,
                                 "candidates_ms": {f"C{t['capacity']}_T{t['tile']}": round(t["ms"], 3)
                                                   for t in table if "ms" in t}}
        torch.cuda.empty_cache()
    for k in (1 << 10, 1 << 16, 1 << 20):
        cap, tile = tuned[k]
        for layout in (capi.LAYOUT_SOA, capi.LAYOUT_AOS):
            if layout == capi.LAYOUT_AOS and k != (1 << 16):
                continue
            n_in = -(-n // cap)
            bound = capi.output_chunk_bound(n, cap, k)
            pool = RecordPool(n_in + bound, cap, layout=layout)
            cdf = torch.from_numpy(capi.zipf_cdf(1.2, k)).cuda()
            capi.check(capi.lib().gf_generate_records16(None, 42, 0, n, cdf.data_ptr(), k, salt,
                                                        ctypes.byref(pool.cols), layout), "generate")
            fills = np.full(n_in, cap, np.uint32)
            fills[-1] = n - cap * (n_in - 1)
            chunks = np.arange(n_in, dtype=np.uint32)
            for _ in range(n_in):
                pool.free.popleft()
            part = HashPartition(pool, k, salt, tile_size=tile, form="device", max_batch_particles=n)
            tiles, d_tiles = part._tiles(chunks, fills)
            part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32).view(np.int32)))
            for _ in range(2):
                part.enqueue_device(d_tiles.data_ptr(), len(tiles), bound)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                part.enqueue_device(d_tiles.data_ptr(), len(tiles), bound)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 5
            name = f"K{k}_{'soa' if layout == capi.LAYOUT_SOA else 'aos'}_C{cap}_T{tile}"
            entry = {"device_form_ms": ms, "records_per_s": n / (ms / 1e3),
                     "hbm_frac": n * 32 / (ms / 1e3) / 1e9 / peak, "status": int(part.status.item())}
            if layout == capi.LAYOUT_SOA:
                plain = HashPartition(pool, k, salt, tile_size=tile, form="plain")
                descs = plain.run(list(chunks), list(fills))[2]
                pool.release([int(x) for x in descs[:, 0]])
                (_, _, descs), sec = _timed(lambda: plain.run(list(chunks), list(fills)))
                pool.release([int(x) for x in descs[:, 0]])
                entry["plain_form_ms_wall"] = sec * 1e3
                del plain
            out[name] = entry
            del pool, part
            torch.cuda.empty_cache()
    out["workload"] = ("hash partition, N=1e8 16-byte records, Zipf 1.2 over K keys; C and tile from the autotuner "
                       "(device-planned form on a 2e7-record sample)")
    return out


def _cfg_photon():
    """photon_scattering (weighted Henyey-Greenstein slab, FP32): the one-kernel transport at N = 1e8,
    the Flow graph at N = 1e6 (host runner, and device-resident: median of three runs), and the FP64
    CPU restatement at N = 1e5 (photons/s)."""
    from graphflow_b200 import capi
    from oracle import oracle as O
    p = capi.photon_params()
    out = {"workload": "slab L=1, mu_s=10, mu_a=0.1, g=0.9, roulette below 1e-4, 256-bin exit histograms, FP32"}
    capi.run_photon(42, 1_000_000, p, exec_mode=capi.EXEC_FUSED, records=False)
    r = capi.run_photon(42, 100_000_000, p, exec_mode=capi.EXEC_FUSED, records=False)
    out["transport_kernel_n1e8"] = {"seconds": r["stats"].seconds, "photons_per_s": 1e8 / r["stats"].seconds,
                                    "event_counts": [int(x) for x in r["event_counts"]]}
    r = capi.run_photon(42, 1_000_000, p, exec_mode=capi.EXEC_FLOW, records=False)
    out["flow_n1e6"] = {"seconds": r["stats"].seconds, "photons_per_s": 1e6 / r["stats"].seconds}
    capi.check(capi.lib().gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        runs = [capi.run_photon(42, 1_000_000, p, exec_mode=capi.EXEC_FLOW, records=False)["stats"]
                for _ in range(3)]
    finally:
        capi.check(capi.lib().gf_set_tuning(b"device_resident", 0), "tuning")
    sd = sorted(runs, key=lambda x: x.seconds)[1]
    out["flow_n1e6_device_resident"] = {"seconds": sd.seconds, "photons_per_s": 1e6 / sd.seconds,
                                        "waves": sd.loop_iterations, "kernel_launches": sd.kernel_launches}
    threads = O.cpu_threads()
    _, sec = _timed(lambda: O.photon_hg(42, 100_000, threads=threads))
    out["cpu_fp64_n1e5"] = {"seconds": sec, "photons_per_s": 1e5 / sec, "cores": threads, "kind": "port"}
    return out


def _cfg_serving():
    """Served mixed stream: whole-flow requests (particle_feedback; photon at 1/100 size; two-node
    dense chain, B in {2, 8, 32}), N log-uniform, Poisson arrivals, device memory cap 40 GB. The
    same streams three ways: the served form with continuous batching (up to 32 requests in
    flight), the served form one request at a time (max_inflight = 1: the same device-resident
    per-request work without batching) and the plain form (each request through the Flow, one at a
    time). The plain form runs the 256-request stream (N in [1e3, 1e5]) only; on the full
    4096-request stream (N in [1e3, 1e7]) it would take tens of minutes."""
    import numpy as np
    from graphflow_b200 import capi

    def summary(req, res, st):
        lat = res["done_s"] - req["arrival_s"]
        return {"requests": int(len(req)), "seconds": st.seconds, "flows_per_s": len(req) / st.seconds,
                "p50_latency_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_latency_ms": float(np.percentile(lat, 99) * 1e3),
                "peak_inflight": int(st.peak_inflight), "peak_bytes": int(st.peak_bytes),
                "all_ok": bool(np.all(res["status"] == 0))}

    def short(x):  # [flows/s, p50 ms, p99 ms]
        return [round(x["flows_per_s"], 1), round(x["p50_latency_ms"], 2), round(x["p99_latency_ms"], 2)]
    out = {"workload": "mixed flow requests, Poisson arrivals at 2000/s, memory cap 40 GB"}
    small = capi.make_requests(256, seed=7, n_min=1_000, n_max=100_000, rate_per_s=2000.0)
    s32, st32 = capi.serve(small, capi.SERVE_BATCHED, max_inflight=32)
    s1, st1 = capi.serve(small, capi.SERVE_BATCHED, max_inflight=1)
    pl, stp = capi.serve(small, capi.SERVE_PLAIN)
    out["stream256_n1e3_1e5"] = {
        "served_batched32": summary(small, s32, st32), "served_one_at_a_time": summary(small, s1, st1),
        "plain": summary(small, pl, stp),
        "results_identical": bool(np.array_equal(s32["digest"], pl["digest"]) and
                                  np.array_equal(s1["digest"], pl["digest"]))}
    full = capi.make_requests(4096, seed=8, n_min=1_000, n_max=10_000_000, rate_per_s=2000.0)
    f32, ft32 = capi.serve(full, capi.SERVE_BATCHED, max_inflight=32)
    f1, ft1 = capi.serve(full, capi.SERVE_BATCHED, max_inflight=1)
    out["stream4096_n1e3_1e7"] = {"served_batched32": summary(full, f32, ft32),
                                  "served_one_at_a_time": summary(full, f1, ft1),
                                  "results_identical": bool(np.array_equal(f32["digest"], f1["digest"]))}
    burst = full.copy()
    burst["arrival_s"] = 0.0
    b32, bt32 = capi.serve(burst, capi.SERVE_BATCHED, max_inflight=32)
    out["stream4096_all_at_once_batched32"] = summary(burst, b32, bt32)
    b1, bt1 = capi.serve(burst, capi.SERVE_BATCHED, max_inflight=1)
    out["stream4096_all_at_once_one_at_a_time"] = summary(burst, b1, bt1)
    sburst = small.copy()
    sburst["arrival_s"] = 0.0
    p32, pt32 = capi.serve(sburst, capi.SERVE_BATCHED, max_inflight=32)
    p1, pt1 = capi.serve(sburst, capi.SERVE_BATCHED, max_inflight=1)
    pp, ptp = capi.serve(sburst, capi.SERVE_PLAIN)
    pd, ptd = capi.serve(sburst, capi.SERVE_FLOW_DEVICE)
    out["stream256_all_at_once"] = {"served_batched32": summary(sburst, p32, pt32),
                                    "served_one_at_a_time": summary(sburst, p1, pt1),
                                    "plain": summary(sburst, pp, ptp),
                                    "flow_device_resident": summary(sburst, pd, ptd),
                                    "results_identical": bool(np.array_equal(p32["digest"], pp["digest"]) and
                                                              np.array_equal(p1["digest"], pp["digest"]) and
                                                              np.array_equal(pd["digest"], pp["digest"]))}
    a, b, c = (out["stream256_n1e3_1e5"][k] for k in ("served_batched32", "served_one_at_a_time", "plain"))
    d, e = (out["stream4096_n1e3_1e7"][k] for k in ("served_batched32", "served_one_at_a_time"))
    g, h = out["stream4096_all_at_once_batched32"], out["stream4096_all_at_once_one_at_a_time"]
    i, j, k2, fd = (out["stream256_all_at_once"][k]
                    for k in ("served_batched32", "served_one_at_a_time", "plain", "flow_device_resident"))
    # short keys: b32 = served with up to 32 requests in flight, one = served one request at a time,
    # plain = the Flow one request at a time, flowdev = the same Flow one request at a time run
    # device-resident; x_plain = b32 / plain, x_one = b32 / one (flows/s)
    out["summary"] = {
        "cols": "flows/s,p50 ms,p99 ms",
        "s256": {"b32": short(a), "one": short(b), "plain": short(c),
                 "x_plain": round(a["flows_per_s"] / c["flows_per_s"], 1),
                 "x_one": round(a["flows_per_s"] / b["flows_per_s"], 2)},
        "s4096": {"x_one": round(d["flows_per_s"] / e["flows_per_s"], 2)},
        "sat256": {"b32": short(i), "one": short(j), "plain": short(k2), "flowdev": short(fd),
                   "x_plain": round(i["flows_per_s"] / k2["flows_per_s"], 1),
                   "x_one": round(i["flows_per_s"] / j["flows_per_s"], 2)},
        "sat4096": {"x_one": round(g["flows_per_s"] / h["flows_per_s"], 2)},
        "identical": bool(out["stream256_n1e3_1e5"]["results_identical"] and
                          out["stream4096_n1e3_1e7"]["results_identical"] and
                          out["stream256_all_at_once"]["results_identical"])}
    return out


def _cfg_tuning_and_graphs():
    """The autotuner's choice of kernel and tile size for the headline batch (N = 1e8, B = 64
    uniform) and for a small batch (N = 1e6), and the step time of a CUDA-graph replay of the fused
    step (reset, partition, finish) against direct launches at both sizes."""
    import numpy as np
    import torch
    from graphflow_b200 import autotune, capi
    from graphflow_b200.partition import ChunkPool, FusedPartition
    out = {}
    for n in (100_000_000, 1_000_000):
        best, table = autotune.tune_fused_partition(n, 64, tiles=(2048, 4096, 8192), reps=5)
        out[f"fused_n{n}"] = {"best": best, "candidates": table}
        cap = 8192
        n_in = -(-n // cap)
        bound = capi.output_chunk_bound(n, cap, 64)
        pool = ChunkPool(n_in + bound, cap)
        capi.check(capi.lib().gf_generate_keys_u32(None, capi.DIST_UNIFORM, SEED, 0, n, 64, None, pool.ptr()), "gen")
        fills = np.full(n_in, cap, np.uint32)
        fills[-1] = n - cap * (n_in - 1)
        part = FusedPartition(pool, 64, tile_size=4096, max_batch_particles=n)
        tl, d_tiles = part._tiles(np.arange(n_in, dtype=np.uint32), fills)
        part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32).view(np.int32)))
        reps = 50
        direct = autotune._events_ms(lambda: [part.enqueue(d_tiles, len(tl), bound) for _ in range(reps)], 3) / reps
        graph = part.capture(d_tiles, len(tl), bound)
        replay = autotune._events_ms(lambda: [graph.replay() for _ in range(reps)], 3) / reps
        out[f"graph_n{n}"] = {"direct_step_ms": direct, "graph_replay_step_ms": replay,
                              "status": int(part.status.item())}
        del graph, part, pool
        torch.cuda.empty_cache()
    return out


def _cfg_kernel_workload():
    """The particle example's kernel workload through the Flow (KernelAxes.hpp runKernelAxes):
    N = 1e7 particles, one partition with B ports, every port into one sink; the fused form and the
    plain form with the shared-staging or the direct (one device atomic per particle) scatter, for
    the balanced and the one-hot distributions (the reference compares the scatter modes on one-hot,
    docs/benchmarks.md:105-108, on its CPU backend). One warm-up run per case, then five timed runs
    (median, min, max): whole runs from Flow construction to the final synchronisation."""
    import numpy as np
    from graphflow_b200 import capi
    n, out = 10_000_000, {"workload": "kernel workload through the Flow, N=1e7, C=8192, P=65536, Q=8, 5 runs"}
    summ = {}
    for bins in (64, 1024):
        for dist in ("balanced", "one-hot"):
            for form, fused, scatter in (("fused", True, "shared"), ("plain_shared", False, "shared"),
                                         ("plain_direct", False, "direct")):
                capi.run_kernel_axes(7, n, bins, dist, scatter, chunk_capacity=8192, live_particles=65536,
                                     batch_chunks=8, fused=fused)  # loads the configuration's kernels
                runs = []
                for _ in range(5):
                    _, st = capi.run_kernel_axes(7, n, bins, dist, scatter, chunk_capacity=8192,
                                                 live_particles=65536, batch_chunks=8, fused=fused)
                    runs.append((st.seconds, st.setup_seconds, st.loop_seconds))
                secs = [r[0] for r in runs]
                med = float(np.median(secs))
                worst = max(runs)
                key = f"B{bins}_{dist}_{form}"
                out[key] = {"seconds_median": med, "seconds_min": min(secs), "seconds_max": max(secs),
                            "particles_per_s": n / med, "partition_batches": st.partition_batches,
                            # host time of the slowest run: Flow built, scheduler loop, the rest
                            # (final synchronisation and teardown)
                            "slowest_setup_loop_rest_s": [worst[1], worst[2], worst[0] - worst[1] - worst[2]],
                            "median_loop_s": float(np.median([r[2] for r in runs]))}
                summ[key] = round(med * 1e3, 1)
    out["summary"] = {"ms_median": summ}
    return out


def _cfg_histogram(n=100_000_000, cpu=True):
    """The device histogram (ParticleTypes.hpp:206-219 histogramOf: sort + run-length encoding) of
    N = 1e8 u32 values: the particle_feedback final weights (the published 260 rows) and uniform
    values over the full 32-bit range (every 6-bit digit pass, ~1e8 rows). Device time with CUDA
    events, buffers allocated beforehand; the oracle's host sort + RLE on a 1e7 sample beside it."""
    import ctypes
    import time
    import numpy as np
    import torch
    from graphflow_b200 import capi
    from oracle import oracle as O
    L = capi.lib()
    w, _, _ = capi.run_particle_feedback_kernel(42, n, 64)
    gen = np.random.default_rng(SEED)
    uniform = gen.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    need = ctypes.c_uint64()
    capi.check(L.gf_histogram_scratch_bytes(n, ctypes.byref(need)), "scratch")
    scratch = torch.empty((need.value + 255) // 8 + 32, dtype=torch.int64, device="cuda")
    base = (scratch.data_ptr() + 255) & ~255
    rows_v = torch.empty(n, dtype=torch.int32, device="cuda")
    rows_c = torch.empty(n, dtype=torch.int64, device="cuda")
    small = torch.zeros(2, dtype=torch.int32, device="cuda")
    out = {"workload": f"histogramOf of N={n} u32 values on the device (radix passes of the stable "
                       "cooperative partition + run-length encoding)"}
    for name, vals in (("feedback_weights", w), ("uniform_u32", uniform)):
        d = torch.from_numpy(vals.view(np.int32)).cuda()
        stream = torch.cuda.current_stream()
        times = []
        for rep in range(4):
            small.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            capi.check(L.gf_histogram_u32(stream.cuda_stream, d.data_ptr(), n, base, need.value, rows_v.data_ptr(),
                                          rows_c.data_ptr(), small.data_ptr(), small[1:].data_ptr()), "histogram")
            e1.record(stream)
            torch.cuda.synchronize()
            if rep:
                times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        out[name] = {"ms": ms, "values_per_s": n / (ms / 1e3), "rows": int(small[0].item()),
                     "status": int(small[1].item())}
        del d
    if cpu:
        t = time.perf_counter()
        O.histogram_u32(uniform[:10_000_000])
        out["cpu_oracle_sort_rle_1e7_uniform"] = {"seconds": time.perf_counter() - t, "cores": 1, "kind": "port"}
    return out


def other_configs(peak):
    out = {}
    for name, f in (("particle_feedback", _cfg_particle_feedback), ("dense_flow", _cfg_dense_flow),
                    ("hash", lambda: _cfg_hash(peak)), ("photon", _cfg_photon), ("serving", _cfg_serving),
                    ("tuning_and_graphs", _cfg_tuning_and_graphs), ("histogram", _cfg_histogram),
                    ("kernel_workload", _cfg_kernel_workload)):
        try:
            out[name] = f()
        except Exception as e:  # reported, never silent
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def bench_reserve_cap(args):
    from graphflow_b200 import capi
    return capi.output_chunk_bound(args.n, CAPACITY, args.bins)


def hash_only(args):
    """One hash-partition workload (16-byte records in three columns, keys over args.hash values
    with Zipf(1.2) popularity, C = 8192 for K <= 4096, else 2048 (K <= 65536) or 512): warm-up
    batches, then timed batches of classify -> device plan -> scatter; prints one JSON line."""
    import ctypes
    import numpy as np
    import torch
    from graphflow_b200 import capi
    from graphflow_b200.hashpart import HashPartition, RecordPool
    n, k, salt = args.n, args.hash, 0x5EED
    cap = 8192 if k <= 4096 else (2048 if k <= 65536 else 512)
    n_in = -(-n // cap)
    bound = capi.output_chunk_bound(n, cap, k)
    pool = RecordPool(n_in + bound, cap, layout=capi.LAYOUT_SOA)
    cdf = torch.from_numpy(capi.zipf_cdf(1.2, k)).cuda()
    capi.check(capi.lib().gf_generate_records16(None, SEED, 0, n, cdf.data_ptr(), k, salt, ctypes.byref(pool.cols),
                                                capi.LAYOUT_SOA), "generate")
    fills = np.full(n_in, cap, np.uint32)
    fills[-1] = n - cap * (n_in - 1)
    for _ in range(n_in):
        pool.free.popleft()
    part = HashPartition(pool, k, salt, tile_size=2048, form="device", max_batch_particles=n)
    tiles, d_tiles = part._tiles(np.arange(n_in, dtype=np.uint32), fills)
    part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32).view(np.int32)))
    for _ in range(args.warmup):
        part.enqueue_device(d_tiles.data_ptr(), len(tiles), bound)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        part.enqueue_device(d_tiles.data_ptr(), len(tiles), bound)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"workload": f"hash partition, N={n} 16-byte records (SoA), Zipf 1.2 over K={k} keys, C={cap}, "
                                  "tiles of 2048", "ms_per_batch": ms, "records_per_s": n / (ms / 1e3),
                      "status": int(part.status.item())}))


def flow_chain_only(args):
    """One run of the dense chain through the Flow, for profiling its launches."""
    from graphflow_b200 import capi
    _, st = capi.run_dense_chain(SEED, args.n, args.bins, nodes=args.flow_chain, dist=args.dist, chunk_capacity=8192,
                                 live_particles=16384, batch_chunks=8, want_ports=False)
    print(json.dumps({"workload": f"dense chain through the Flow, {args.flow_chain} nodes, N={args.n}, B={args.bins}, "
                                  f"{args.dist}, C=8192 P=16384 Q=8", "seconds": st.seconds,
                      "partition_batches": st.partition_batches, "partition_launches": st.partition_launches,
                      "kernel_launches": st.kernel_launches, "sunk": st.sunk}))


def feedback_device_resident_only(args):
    """One particle_feedback run through the Flow device-resident (seed 42, C = 8192, 64 visits), for
    profiling its launches."""
    from graphflow_b200 import capi
    capi.check(capi.lib().gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        _, _, st = capi.run_particle_feedback(SEED, args.n, 64, chunk_capacity=8192, live_particles=16384,
                                              batch_chunks=8)
    finally:
        capi.check(capi.lib().gf_set_tuning(b"device_resident", 0), "tuning")
    print(json.dumps({"workload": f"particle_feedback through the Flow device-resident, N={args.n}, C=8192",
                      "seconds": st.seconds, "waves": st.loop_iterations, "kernel_launches": st.kernel_launches,
                      "partition_batches": st.partition_batches, "sunk": st.sunk}))


def photon_device_resident_only(args):
    """One photon_scattering run (weighted HG slab, FP32, seed 42) through the Flow device-resident,
    for profiling its launches."""
    from graphflow_b200 import capi
    p = capi.photon_params()
    capi.check(capi.lib().gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        st = capi.run_photon(SEED, args.n, p, exec_mode=capi.EXEC_FLOW, records=False)["stats"]
    finally:
        capi.check(capi.lib().gf_set_tuning(b"device_resident", 0), "tuning")
    print(json.dumps({"workload": f"photon slab through the Flow device-resident, N={args.n}",
                      "seconds": st.seconds, "waves": st.loop_iterations, "kernel_launches": st.kernel_launches,
                      "partition_batches": st.partition_batches, "sunk": st.sunk}))


def device_chain_only(args):
    """One run of the dense chain on the device (seed 42, C = 8192), for profiling its launches."""
    from graphflow_b200 import capi
    _, _, pool, st = capi.run_dense_chain_device(SEED, args.n, args.bins, nodes=args.device_chain, dist=args.dist,
                                                 want_ports=False)
    print(json.dumps({"workload": f"dense chain on the device, {args.device_chain} nodes, N={args.n}, B={args.bins}, "
                                  f"{args.dist}, C=8192", "device_seconds": st.loop_seconds,
                      "kernel_launches": st.kernel_launches, "pool_chunks": pool.num_chunks,
                      "peak_live_chunks": pool.peak_live}))


def main():
    args = parse()
    if args.device_chain:
        device_chain_only(args)
        return
    if args.feedback_device_resident:
        feedback_device_resident_only(args)
        return
    if args.photon_device_resident:
        photon_device_resident_only(args)
        return
    if args.flow_chain:
        flow_chain_only(args)
        return
    if args.hash:
        hash_only(args)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    gpu_arm(args)


if __name__ == "__main__":
    main()
