"""Autotuner of the hot path's launch shapes and batch sizes, measured on the GPU it runs on.

* ``tune_fused_partition``: kernel (cooperative count/plan/scatter or per-tile look-back) and tile
  size of one fused dense batch, on the batch's own size.
* ``tune_chain``: chunk capacity C and batch chunks Q of a dense chain through the Flow, on a
  sample of the flow's size (the Flow's cost is per batch, so a sample ranks C and Q correctly).
* ``tune_hash``: chunk capacity C and tile size of the device-planned hash partition.

Every candidate is measured (CUDA events or the Flow's own clock, median of repetitions); the
tuner returns the best candidate and the whole table. Results are cached per key for the process.
"""
from __future__ import annotations

import ctypes
import statistics

import numpy as np
import torch

from . import capi
from .hashpart import HashPartition, RecordPool
from .partition import ChunkPool, FusedPartition

_CACHE: dict = {}


def _events_ms(f, reps):
    f()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        f()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def tune_fused_partition(n, bins, dist="uniform", capacity=8192, tiles=(1024, 2048, 4096, 8192), reps=5, seed=42):
    """Best (kernel, tile size) for one fused batch of n u32 keys into `bins` ports."""
    key = ("fused", n, bins, dist, capacity, tuple(tiles))
    if key in _CACHE:
        return _CACHE[key]
    dev = torch.device("cuda", torch.cuda.current_device())
    n_in = -(-n // capacity)
    bound = capi.output_chunk_bound(n, capacity, bins)
    pool = ChunkPool(n_in + bound, capacity, device=dev)
    cdf = torch.from_numpy(capi.zipf_cdf(1.1, bins)).to(dev) if dist == "zipf" else None
    capi.check(capi.lib().gf_generate_keys_u32(None, capi.DIST_NAMES[dist], seed, 0, n, bins,
                                               cdf.data_ptr() if cdf is not None else None, pool.ptr()), "generate")
    fills = np.full(n_in, capacity, np.uint32)
    fills[-1] = n - capacity * (n_in - 1)
    table = []
    try:
        for tile in tiles:
            part = FusedPartition(pool, bins, tile_size=tile, max_batch_particles=n)
            tl, d_tiles = part._tiles(np.arange(n_in, dtype=np.uint32), fills)
            part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32)
                                                         .view(np.int32)))
            for coop in (1, 0):
                capi.check(capi.lib().gf_set_tuning(b"fused_coop", coop), "tuning")
                ms = _events_ms(lambda: part.enqueue(d_tiles, len(tl), bound), reps)
                status = int(part.status.item())
                # the cooperative kernel only takes tiles up to 4096 keys; it falls back otherwise
                kernel = "cooperative" if coop and tile <= 4096 and capacity >= 4096 and bins <= 64 else "per_tile"
                table.append({"kernel": kernel, "tile": tile, "ms": ms, "status": status})
            del part
    finally:
        capi.check(capi.lib().gf_set_tuning(b"fused_coop", 1), "tuning")
    best = min((t for t in table if t["status"] == 0), key=lambda t: t["ms"])
    _CACHE[key] = (best, table)
    return best, table


def tune_chain(bins, nodes, sample_n=1_000_000, capacities=(2048, 4096, 8192), batch_chunks=(2, 8, 32),
               live_particles=16384, reps=2, seed=42):
    """Best (C, Q) of a dense Flow chain, measured on sample_n particles."""
    key = ("chain", bins, nodes, sample_n, tuple(capacities), tuple(batch_chunks), live_particles)
    if key in _CACHE:
        return _CACHE[key]
    table = []
    for cap in capacities:
        for q in batch_chunks:
            secs = []
            for _ in range(reps):
                _, st = capi.run_dense_chain(seed, sample_n, bins, nodes=nodes, chunk_capacity=cap,
                                             live_particles=max(live_particles, cap), batch_chunks=q,
                                             want_ports=False)
                secs.append(st.seconds)
            table.append({"capacity": cap, "batch_chunks": q, "seconds": statistics.median(secs),
                          "particles_per_s": sample_n / statistics.median(secs)})
    best = min(table, key=lambda t: t["seconds"])
    _CACHE[key] = (best, table)
    return best, table


def tune_hash(n, k, zipf_s=1.2, capacities=(512, 2048, 8192), tiles=(1024, 2048), reps=3, salt=0x5EED, seed=42,
              layout=None):
    """Best (C, tile) of the device-planned hash partition of n records over k keys. Capacities whose
    exact plan (one partial chunk per non-empty port) would not fit in device memory are skipped."""
    layout = capi.LAYOUT_SOA if layout is None else layout
    key = ("hash", n, k, zipf_s, tuple(capacities), tuple(tiles), layout)
    if key in _CACHE:
        return _CACHE[key]
    free_bytes = torch.cuda.mem_get_info()[0]
    table = []
    for cap in capacities:
        n_in = -(-n // cap)
        bound = capi.output_chunk_bound(n, cap, k)
        if (n_in + bound) * cap * 16 > free_bytes // 2:
            table.append({"capacity": cap, "skipped": "pool would exceed half the free device memory"})
            continue
        pool = RecordPool(n_in + bound, cap, layout=layout)
        cdf = torch.from_numpy(capi.zipf_cdf(zipf_s, k)).cuda()
        capi.check(capi.lib().gf_generate_records16(None, seed, 0, n, cdf.data_ptr(), k, salt,
                                                    ctypes.byref(pool.cols), layout), "generate")
        fills = np.full(n_in, cap, np.uint32)
        fills[-1] = n - cap * (n_in - 1)
        for tile in tiles:
            part = HashPartition(pool, k, salt, tile_size=tile, form="device", max_batch_particles=n)
            tl, d_tiles = part._tiles(np.arange(n_in, dtype=np.uint32), fills)
            part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32)
                                                         .view(np.int32)))
            ms = _events_ms(lambda: part.enqueue_device(d_tiles.data_ptr(), len(tl), bound), reps)
            table.append({"capacity": cap, "tile": tile, "ms": ms, "status": int(part.status.item())})
            del part
        del pool
        torch.cuda.empty_cache()
    best = min((t for t in table if "ms" in t and t["status"] == 0), key=lambda t: t["ms"])
    _CACHE[key] = (best, table)
    return best, table
