"""Hash-bin partition of 16-byte records {u64 key, f32 weight, u32 tag} over a device chunk pool,
in SoA (three columns) or AoS (16-byte records) storage.

``HashPartition(..., form="plain")`` is the reference's two-launch form
(flow/Execution.hpp:1208-1502 with the host plan of :2520-2642); ``form="device"`` keeps the plan
on the device (classify without storing bins -> device plan from an outputChunkBound
reservation -> scatter that recomputes each bin from its key), so a batch needs no host round
trip and can be captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes as C
from collections import deque

import numpy as np
import torch

from . import capi
from .partition import BatchError, _stream_ptr, _u32


class RecordPool:
    """Fixed-layout pool of 16-byte records (SoA or AoS)."""

    def __init__(self, num_chunks, capacity, layout=capi.LAYOUT_SOA, device="cuda"):
        if num_chunks * capacity > 2**32:
            raise OverflowError("RecordPool: numChunks * chunkCapacity exceeds the 32-bit slot range")
        self.num_chunks, self.capacity, self.layout = num_chunks, capacity, layout
        slots = num_chunks * capacity
        if layout == capi.LAYOUT_SOA:
            self.key = torch.zeros(slots, dtype=torch.int64, device=device)
            self.weight = torch.zeros(slots, dtype=torch.float32, device=device)
            self.tag = torch.zeros(slots, dtype=torch.int32, device=device)
            self.cols = capi.Rec16Columns(self.key.data_ptr(), self.weight.data_ptr(), self.tag.data_ptr(), None)
        else:
            self.records = torch.zeros(slots * 4, dtype=torch.int32, device=device)
            self.cols = capi.Rec16Columns(None, None, None, self.records.data_ptr())
        self.free = deque(range(num_chunks))

    @property
    def slots(self):
        return self.num_chunks * self.capacity

    def acquire(self, n):
        if n > len(self.free):
            raise BatchError(f"chunk pool exhausted: {n} requested, {len(self.free)} free")
        return [self.free.popleft() for _ in range(n)]

    def release(self, chunks):
        self.free.extend(chunks)

    def host_slots(self, lo, hi):
        """(keys u64, weights f32, tags u32) of slots [lo, hi) copied to the host."""
        if self.layout == capi.LAYOUT_SOA:
            return (self.key[lo:hi].cpu().numpy().view(np.uint64), self.weight[lo:hi].cpu().numpy(),
                    self.tag[lo:hi].cpu().numpy().view(np.uint32))
        r = self.records[4 * lo:4 * hi].cpu().numpy().view(np.uint32).reshape(-1, 4)
        keys = r[:, 0].astype(np.uint64) | (r[:, 1].astype(np.uint64) << np.uint64(32))
        return keys, r[:, 2].copy().view(np.float32), r[:, 3].copy()

    def set_slots(self, lo, keys, weights, tags):
        n = len(keys)
        if self.layout == capi.LAYOUT_SOA:
            self.key[lo:lo + n].copy_(torch.from_numpy(np.asarray(keys, np.uint64).view(np.int64)))
            self.weight[lo:lo + n].copy_(torch.from_numpy(np.asarray(weights, np.float32)))
            self.tag[lo:lo + n].copy_(torch.from_numpy(np.asarray(tags, np.uint32).view(np.int32)))
        else:
            r = np.zeros((n, 4), np.uint32)
            k = np.asarray(keys, np.uint64)
            r[:, 0] = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            r[:, 1] = (k >> np.uint64(32)).astype(np.uint32)
            r[:, 2] = np.asarray(weights, np.float32).view(np.uint32)
            r[:, 3] = np.asarray(tags, np.uint32)
            self.records[4 * lo:4 * (lo + n)].copy_(torch.from_numpy(r.reshape(-1).view(np.int32)))


class HashPartition:
    def __init__(self, pool: RecordPool, bins: int, salt: int, tile_size: int = 1024, form: str = "plain",
                 max_batch_particles: int | None = None):
        if form not in ("plain", "device"):
            raise ValueError("form must be 'plain' or 'device'")
        self.pool, self.bins, self.salt, self.tile_size, self.form = pool, bins, salt, tile_size, form
        dev = (pool.key if pool.layout == capi.LAYOUT_SOA else pool.records).device
        self.dev = dev
        self.counts = torch.zeros(bins + 1, dtype=torch.int32, device=dev)
        self.next = torch.zeros(bins, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.bin_ids = torch.zeros(pool.slots, dtype=torch.int32, device=dev) if form == "plain" else None
        self.max_batch = max_batch_particles if max_batch_particles is not None else pool.slots
        self.reserve_cap = capi.output_chunk_bound(self.max_batch, pool.capacity, bins)
        if form == "device":
            self.reserved = torch.zeros(max(self.reserve_cap, 1), dtype=torch.int32, device=dev)
            self.table = torch.zeros(bins + max(self.reserve_cap, 1), dtype=torch.int32, device=dev)
            self.descs = torch.zeros(3 * max(self.reserve_cap, 1), dtype=torch.int32, device=dev)
            self.num_out = torch.zeros(1, dtype=torch.int32, device=dev)

    def _tiles(self, chunks, fills):
        tiles = capi.flatten_tiles(chunks, fills, self.tile_size)
        d = torch.from_numpy(tiles.view(np.int32).reshape(-1)).to(self.dev) if len(tiles) else None
        return tiles, d

    def enqueue_device(self, d_tiles, n_tiles, n_reserved, stream=None):
        """Device-planned batch: classify -> plan -> scatter, all stream-ordered."""
        s = _stream_ptr(stream)
        L = capi.lib()
        p = self.pool
        cols = C.byref(p.cols)
        self.counts.zero_()
        capi.check(L.gf_classify_hash_r16(s, cols, p.layout, p.capacity, p.slots, d_tiles, n_tiles, self.tile_size,
                                          self.bins, self.salt, None, self.counts.data_ptr(),
                                          self.status.data_ptr()), "hash classify")
        capi.check(L.gf_plan_device(s, self.counts.data_ptr(), self.bins, p.capacity, self.reserved.data_ptr(),
                                    n_reserved, self.table.data_ptr(), self.descs.data_ptr(), self.reserve_cap,
                                    self.num_out.data_ptr(), self.next.data_ptr(), self.status.data_ptr()),
                   "device plan")
        capi.check(L.gf_scatter_hash_r16(s, cols, cols, p.layout, p.capacity, p.slots, d_tiles, n_tiles,
                                         self.tile_size, self.bins, self.salt, None, self.table.data_ptr(),
                                         self.next.data_ptr(), self.counts.data_ptr(), self.status.data_ptr()),
                   "hash scatter")

    def run(self, chunks, fills, stream=None):
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            return self._run(chunks, fills, stream)

    def _run(self, chunks, fills, stream):
        n = int(np.sum(np.asarray(fills, np.uint64)))
        tiles, d_tiles = self._tiles(chunks, fills)
        dt = d_tiles.data_ptr() if d_tiles is not None else None
        s = _stream_ptr(stream)
        L = capi.lib()
        p = self.pool
        cols = C.byref(p.cols)
        self.status.zero_()
        if self.form == "device":
            bound = capi.checked_output_chunk_bound(n, p.capacity, self.bins)
            if bound > self.reserve_cap:
                raise BatchError("hash partition: batch exceeds the configured maximum")
            reserved = p.acquire(bound)
            if bound:
                self.reserved[:bound].copy_(torch.tensor(np.asarray(reserved, np.uint32).view(np.int32)))
            if len(tiles):
                self.enqueue_device(dt, len(tiles), bound, stream)
            else:
                self.counts.zero_()
                capi.check(L.gf_plan_device(s, self.counts.data_ptr(), self.bins, p.capacity,
                                            self.reserved.data_ptr(), bound, self.table.data_ptr(),
                                            self.descs.data_ptr(), self.reserve_cap, self.num_out.data_ptr(),
                                            self.next.data_ptr(), self.status.data_ptr()), "device plan")
            st = int(_u32(self.status)[0])
            counts = _u32(self.counts)
            if st != 0 or counts[self.bins] != 0:
                p.release(reserved)
                raise BatchError(f"hash partition: device status reports {capi.STATUS_NAMES.get(st, st)}")
            r = int(_u32(self.num_out)[0])
            totals = counts[:self.bins].copy()
            if int(totals.sum(dtype=np.uint64)) != n or not np.array_equal(_u32(self.next), totals):
                p.release(reserved)
                raise BatchError("hash partition: totals do not match the batch")
            table = _u32(self.table)[:self.bins + r].copy()
            descs = _u32(self.descs)[:3 * r].reshape(-1, 3).copy()
            p.release(reserved[r:])
            return totals, table, descs
        # plain: classify -> host plan -> scatter (reference structure)
        self.counts.zero_()
        if len(tiles):
            capi.check(L.gf_classify_hash_r16(s, cols, p.layout, p.capacity, p.slots, dt, len(tiles), self.tile_size,
                                              self.bins, self.salt, self.bin_ids.data_ptr(), self.counts.data_ptr(),
                                              self.status.data_ptr()), "hash classify")
        counts = _u32(self.counts)
        st = int(_u32(self.status)[0])
        if st != 0 or counts[self.bins] != 0:
            raise BatchError(f"hash classify: device status reports {capi.STATUS_NAMES.get(st, st)}")
        totals = counts[:self.bins].copy()
        if int(totals.sum(dtype=np.uint64)) != n:
            raise BatchError("hash classify: classified particle count does not match the batch")
        bin_base, fills_out, r = capi.plan_dense(totals, p.capacity)
        out_chunks = p.acquire(r)
        table = capi.build_dense_table(bin_base, out_chunks)
        d_table = torch.from_numpy(table.view(np.int32)).to(self.dev)
        self.next.zero_()
        if len(tiles):
            capi.check(L.gf_scatter_hash_r16(s, cols, cols, p.layout, p.capacity, p.slots, dt, len(tiles),
                                             self.tile_size, self.bins, self.salt, self.bin_ids.data_ptr(),
                                             d_table.data_ptr(), self.next.data_ptr(), self.counts.data_ptr(),
                                             self.status.data_ptr()), "hash scatter")
        st = int(_u32(self.status)[0])
        if st != 0 or _u32(self.counts)[self.bins] != 0 or not np.array_equal(_u32(self.next), totals):
            p.release(out_chunks)
            raise BatchError(f"hash scatter: finalise failed (status {capi.STATUS_NAMES.get(st, st)})")
        bins_of = np.repeat(np.arange(self.bins, dtype=np.uint32), (totals + p.capacity - 1) // p.capacity)
        descs = (np.stack([np.asarray(out_chunks, np.uint32), fills_out, bins_of], axis=1) if r
                 else np.zeros((0, 3), np.uint32))
        return totals, table, descs
