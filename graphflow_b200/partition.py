"""Host driver of one partition batch over a device chunk pool, mirroring the reference's
``PartitionStage`` (flow/Execution.hpp:2263-2772):

* ``launch``   flatten the batch's chunks into tile descriptors and enqueue classify
               (Execution.hpp:2363-2430);
* ``advance``  read the per-bin totals, check them, plan, take output chunks, enqueue scatter
               (planAndScatter, Execution.hpp:2520-2642);
* ``finalise`` check status, the status slot and next[b] == total[b] (Execution.hpp:2715-2725).

``PlainPartition`` is that two-launch form; ``FusedPartition`` replaces it with one fused launch
plus a device-side finish, taking output chunks from an ``outputChunkBound`` reservation.
Device memory is torch-allocated; every kernel runs through the C ABI (graphflow_b200.capi).
"""
from __future__ import annotations

import ctypes as C
from collections import deque

import numpy as np
import torch

from . import capi


class BatchError(RuntimeError):
    """Raised before any output of a failed batch is published (Execution.hpp:2527-2547)."""


def _u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class ChunkPool:
    """Fixed-layout pool of ``num_chunks`` chunks of ``capacity`` slots of one u32 column
    (core/ChunkPool.hpp; base(handle) = index * capacity)."""

    def __init__(self, num_chunks: int, capacity: int, device="cuda"):
        if capacity == 0 or num_chunks == 0:
            raise ValueError("ChunkPool: capacity and chunk count must be non-zero")
        if num_chunks * capacity > 2**32:
            raise OverflowError("ChunkPool: numChunks * chunkCapacity exceeds the 32-bit slot range")
        self.num_chunks, self.capacity = num_chunks, capacity
        self.column = torch.zeros(num_chunks * capacity, dtype=torch.int32, device=device)
        self.free = deque(range(num_chunks))

    @property
    def slots(self):
        return self.num_chunks * self.capacity

    def acquire(self, n: int = 1):
        if n > len(self.free):
            raise BatchError(f"chunk pool exhausted: {n} requested, {len(self.free)} free")
        return [self.free.popleft() for _ in range(n)]

    def release(self, chunks):
        self.free.extend(chunks)

    def ptr(self):
        return C.c_void_p(self.column.data_ptr())


class _Common:
    def __init__(self, pool: ChunkPool, bins: int, classifier: int = capi.CLS_KEY_MOD, tile_size: int = 4096):
        if tile_size not in capi.supported_tile_sizes():
            raise ValueError(f"tile size {tile_size} not in {capi.supported_tile_sizes()}")
        self.pool, self.bins, self.cls, self.tile_size = pool, bins, classifier, tile_size
        self.dev = pool.column.device
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)

    def _tiles(self, chunks, fills):
        tiles = capi.flatten_tiles(chunks, fills, self.tile_size)
        d = torch.from_numpy(tiles.view(np.int32).reshape(-1)).to(self.dev) if len(tiles) else None
        return tiles, d


class PlainPartition(_Common):
    """The reference's two-launch form: classify -> host plan -> scatter."""

    def __init__(self, pool, bins, classifier=capi.CLS_KEY_MOD, tile_size=4096, mode=capi.SCATTER_SHARED):
        super().__init__(pool, bins, classifier, tile_size)
        self.mode = mode
        self.bin_ids = torch.zeros(pool.slots, dtype=torch.int32, device=self.dev)
        self.counts = torch.zeros(bins + 1, dtype=torch.int32, device=self.dev)
        self.next = torch.zeros(bins, dtype=torch.int32, device=self.dev)
        self.classify_launches = 0
        self.scatter_launches = 0

    def run(self, chunks, fills, stream=None):
        """One batch. Returns (totals, table, output descriptors (chunk, fill, bin)). Every
        device operation of the batch, readbacks included, is ordered on `stream`."""
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            return self._run(chunks, fills, stream)

    def _run(self, chunks, fills, stream):
        n = int(np.sum(np.asarray(fills, np.uint64)))
        tiles, d_tiles = self._tiles(chunks, fills)
        s = _stream_ptr(stream)
        L = capi.lib()
        self.counts.zero_()
        self.status.zero_()
        if len(tiles):
            capi.check(L.gf_classify_dense_u32(s, self.pool.ptr(), self.pool.capacity, self.pool.slots,
                                               d_tiles.data_ptr(), len(tiles), self.tile_size, self.bins, self.cls,
                                               self.bin_ids.data_ptr(), self.counts.data_ptr(),
                                               self.status.data_ptr()), "classify")
            self.classify_launches += 1
        counts = _u32(self.counts)
        if int(_u32(self.status)[0]) != 0 or counts[self.bins] != 0:
            raise BatchError("partition classify: device status reports an invalid classifier result")
        totals = counts[:self.bins].copy()
        if int(totals.sum(dtype=np.uint64)) != n:
            raise BatchError("partition classify: classified particle count does not match the batch")
        bin_base, fills_out, r = capi.plan_dense(totals, self.pool.capacity)
        bound = capi.checked_output_chunk_bound(n, self.pool.capacity, self.bins)
        if r > bound:
            raise BatchError("partition plan: exact chunk count exceeds the reservation bound")
        out_chunks = self.pool.acquire(r)
        table = capi.build_dense_table(bin_base, out_chunks)
        d_table = torch.from_numpy(table.view(np.int32)).to(self.dev)
        self.next.zero_()
        if len(tiles):
            capi.check(L.gf_scatter_dense_u32(s, self.pool.ptr(), self.pool.ptr(), self.pool.capacity,
                                              self.pool.slots, d_tiles.data_ptr(), len(tiles), self.tile_size,
                                              self.bins, self.bin_ids.data_ptr(), d_table.data_ptr(),
                                              self.next.data_ptr(), self.counts.data_ptr(), self.mode,
                                              self.status.data_ptr()), "scatter")
            self.scatter_launches += 1
        # finalise (Execution.hpp:2715-2725)
        st = int(_u32(self.status)[0])
        if st != 0:
            self.pool.release(out_chunks)
            raise BatchError(f"partition scatter: device status reports {capi.STATUS_NAMES.get(st, st)}")
        if _u32(self.counts)[self.bins] != 0:
            self.pool.release(out_chunks)
            raise BatchError("partition scatter: device status reports a checked updater overflow")
        if not np.array_equal(_u32(self.next), totals):
            self.pool.release(out_chunks)
            raise BatchError("partition scatter: next[bin] does not match total[bin]")
        bins_of = np.repeat(np.arange(self.bins, dtype=np.uint32), (totals + self.pool.capacity - 1) //
                            self.pool.capacity)
        descs = np.stack([np.asarray(out_chunks, np.uint32), fills_out, bins_of], axis=1) if r else \
            np.zeros((0, 3), np.uint32)
        return totals, table, descs


class FusedPartition(_Common):
    """One fused classify -> scan -> scatter launch plus a device-side finish per batch."""

    def __init__(self, pool, bins, classifier=capi.CLS_KEY_MOD, tile_size=4096, max_batch_particles=None):
        super().__init__(pool, bins, classifier, tile_size)
        cap = pool.capacity
        self.max_batch = max_batch_particles if max_batch_particles is not None else pool.slots
        self.max_k = max(1, -(-self.max_batch // cap))
        self.max_tiles = max(1, -(-self.max_batch // min(tile_size, cap)) + pool.num_chunks)
        self.totals = torch.zeros(bins, dtype=torch.int32, device=self.dev)
        self.port_chunks = torch.zeros(bins * self.max_k, dtype=torch.int64, device=self.dev)
        self.scratch_bytes = capi.fused_scratch_bytes(self.max_tiles, bins)
        self.scratch = torch.zeros((self.scratch_bytes + 15) // 16 * 2, dtype=torch.int64, device=self.dev)
        self.reserve_cap = capi.output_chunk_bound(self.max_batch, cap, bins)
        self.reserved = torch.zeros(max(self.reserve_cap, 1), dtype=torch.int32, device=self.dev)
        self.table = torch.zeros(bins + max(self.reserve_cap, 1), dtype=torch.int32, device=self.dev)
        self.descs = torch.zeros(3 * max(self.reserve_cap, 1), dtype=torch.int32, device=self.dev)
        self.num_out = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.launches = 0
        self.combined = True

    def enqueue(self, d_tiles, n_tiles, n_reserved, stream=None, combined=None):
        """Enqueue the fused launch and the finish (no host synchronisation): one launch that
        does both (gf_partition_fused_full_u32), or with combined=False (default: the object's
        `combined` attribute, True) the two calls gf_partition_fused_u32 + gf_fused_finish."""
        s = _stream_ptr(stream)
        L = capi.lib()
        if self.combined if combined is None else combined:
            capi.check(L.gf_partition_fused_full_u32(
                s, self.pool.ptr(), self.pool.ptr(), self.pool.capacity, self.pool.slots,
                d_tiles.data_ptr() if n_tiles else None, n_tiles, self.tile_size, self.bins, self.cls,
                self.reserved.data_ptr(), n_reserved, self.totals.data_ptr(), self.port_chunks.data_ptr(), self.max_k,
                self.scratch.data_ptr(), self.scratch_bytes, self.table.data_ptr(), self.descs.data_ptr(),
                self.reserve_cap, self.num_out.data_ptr(), self.status.data_ptr()), "fused partition + finish")
            self.launches += 1
            return
        capi.check(L.gf_partition_fused_u32(s, self.pool.ptr(), self.pool.ptr(), self.pool.capacity, self.pool.slots,
                                            d_tiles.data_ptr() if n_tiles else None, n_tiles, self.tile_size,
                                            self.bins, self.cls, self.reserved.data_ptr(), n_reserved,
                                            self.totals.data_ptr(), self.port_chunks.data_ptr(), self.max_k,
                                            self.scratch.data_ptr(), self.scratch_bytes,
                                            self.status.data_ptr()), "fused partition")
        capi.check(L.gf_fused_finish(s, self.totals.data_ptr(), self.port_chunks.data_ptr(), self.bins,
                                     self.pool.capacity, self.max_k, self.scratch.data_ptr(), self.table.data_ptr(),
                                     self.descs.data_ptr(), self.reserve_cap, self.num_out.data_ptr(),
                                     self.status.data_ptr()), "fused finish")
        self.launches += 1

    def capture(self, d_tiles, n_tiles, n_reserved):
        """Captures one batch step (control-block reset, fused launch, device finish) into a CUDA
        graph for repeated replay on the same tiles, reservation and buffers. The launch epoch lives
        in device memory and advances on every replay, so a replay equals a direct launch."""
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=self.dev)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.enqueue(d_tiles, n_tiles, n_reserved, side)  # warm-up: kernel attributes, lazy loading
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=side):
            self.enqueue(d_tiles, n_tiles, n_reserved, side)
        torch.cuda.synchronize()
        return graph

    def run(self, chunks, fills, stream=None):
        """One batch on `stream`; returns (totals, table, output descriptors)."""
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            return self._run(chunks, fills, stream)

    def _run(self, chunks, fills, stream):
        n = int(np.sum(np.asarray(fills, np.uint64)))
        if n > self.max_batch:
            raise BatchError("fused partition: batch exceeds the configured maximum")
        tiles, d_tiles = self._tiles(chunks, fills)
        if len(tiles) > self.max_tiles:
            raise BatchError("fused partition: tile descriptor capacity exceeded")
        bound = capi.checked_output_chunk_bound(n, self.pool.capacity, self.bins)
        reserved = self.pool.acquire(bound)
        if bound:
            self.reserved[:bound].copy_(torch.tensor(np.asarray(reserved, np.uint32).view(np.int32)))
        self.status.zero_()
        self.enqueue(d_tiles, len(tiles), bound, stream)
        st = int(_u32(self.status)[0])
        r = int(_u32(self.num_out)[0])
        totals = _u32(self.totals).copy()
        if st != 0:
            self.pool.release(reserved)
            raise BatchError(f"fused partition: device status reports {capi.STATUS_NAMES.get(st, st)}")
        if int(totals.sum(dtype=np.uint64)) != n:
            self.pool.release(reserved)
            raise BatchError("fused partition: classified particle count does not match the batch")
        table = _u32(self.table)[:self.bins + r].copy()
        descs = _u32(self.descs)[:3 * r].reshape(-1, 3).copy()
        used = set(int(c) for c in table[self.bins:])
        if len(used) != r or not used.issubset(set(reserved)):
            self.pool.release(reserved)
            raise BatchError("fused partition: output chunks are not a subset of the reservation")
        self.pool.release([c for c in reserved if c not in used])
        return totals, table, descs
