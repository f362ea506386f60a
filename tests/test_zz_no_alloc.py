"""gf_partition_fused_u32_noalloc: the fused partition for callers that cannot allocate device
memory during the call (a runtime that owns all device memory through its own pool, or a path
that cannot afford cudaMalloc's device synchronisation). It must produce what the allocating
entry point (gf_partition_fused_u32 + gf_fused_finish with caller scratch) produces, exactly,
on consecutive calls that share its static scratch."""
import ctypes as C

import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_SIG = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
        C.c_int, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
        C.c_void_p, C.c_void_p]


def _noalloc():
    fn = capi.lib().gf_partition_fused_u32_noalloc
    fn.argtypes = _SIG
    fn.restype = C.c_int
    return fn


class _Case:
    """One batch: input chunks 0..n_in-1 of a pool, reservation behind them."""

    def __init__(self, n, capacity, bins, dist, seed):
        self.n, self.C, self.bins = n, capacity, bins
        self.keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
        self.n_in = -(-n // capacity)
        self.fills = [capacity] * (self.n_in - 1) + [n - capacity * (self.n_in - 1)]
        self.bound = capi.output_chunk_bound(n, capacity, bins)
        self.num_chunks = self.n_in + self.bound
        tiles = capi.flatten_tiles(np.arange(self.n_in, dtype=np.uint32), self.fills, 4096)
        self.n_tiles = len(tiles)
        self.tiles = torch.from_numpy(tiles.view(np.int32).reshape(-1)).cuda()
        self.reserved = torch.from_numpy(np.arange(self.n_in, self.num_chunks, dtype=np.uint32).view(np.int32)).cuda()
        self.max_k = -(-n // capacity)

    def buffers(self):
        pool = torch.zeros(self.num_chunks * self.C, dtype=torch.int32, device="cuda")
        pool[: self.n].copy_(torch.from_numpy(self.keys.view(np.int32)))
        out = dict(pool=pool,
                   totals=torch.zeros(self.bins, dtype=torch.int32, device="cuda"),
                   port=torch.zeros(self.bins * self.max_k, dtype=torch.int64, device="cuda"),
                   table=torch.zeros(self.bins + self.bound, dtype=torch.int32, device="cuda"),
                   descs=torch.zeros(3 * self.bound, dtype=torch.int32, device="cuda"),
                   num=torch.zeros(1, dtype=torch.int32, device="cuda"),
                   status=torch.zeros(1, dtype=torch.int32, device="cuda"))
        return out

    def args_in(self, b):
        return (None, b["pool"].data_ptr(), b["pool"].data_ptr(), self.C, self.num_chunks * self.C,
                self.tiles.data_ptr(), self.n_tiles, 4096, self.bins, capi.CLS_KEY_MOD, self.reserved.data_ptr(),
                self.bound, b["totals"].data_ptr(), b["port"].data_ptr(), self.max_k)

    def result(self, b):
        torch.cuda.synchronize()
        u = lambda t: t.cpu().numpy().view(np.uint32)  # noqa: E731
        r = int(u(b["num"])[0])
        descs = u(b["descs"])[: 3 * r].reshape(-1, 3)
        col = u(b["pool"])
        ports = [[] for _ in range(self.bins)]
        for chunk, fill, port in descs:
            ports[int(port)].append(col[int(chunk) * self.C: int(chunk) * self.C + int(fill)])
        seqs = [np.concatenate(p) if p else np.zeros(0, np.uint32) for p in ports]
        return int(u(b["status"])[0]), u(b["totals"]).copy(), u(b["table"])[: self.bins].copy(), descs[:, 1:].copy(), seqs


def _allocating(case):
    b = case.buffers()
    scratch_bytes = capi.fused_scratch_bytes(case.n_tiles, case.bins)
    scratch = torch.zeros((scratch_bytes + 15) // 8, dtype=torch.int64, device="cuda")
    L = capi.lib()
    capi.check(L.gf_partition_fused_u32(*case.args_in(b), scratch.data_ptr(), scratch_bytes, b["status"].data_ptr()),
               "fused")
    capi.check(L.gf_fused_finish(None, b["totals"].data_ptr(), b["port"].data_ptr(), case.bins, case.C, case.max_k,
                                 scratch.data_ptr(), b["table"].data_ptr(), b["descs"].data_ptr(), case.bound,
                                 b["num"].data_ptr(), b["status"].data_ptr()), "finish")
    return case.result(b)


def _static(case):
    b = case.buffers()
    rc = _noalloc()(*case.args_in(b), b["table"].data_ptr(), b["descs"].data_ptr(), case.bound, b["num"].data_ptr(),
                    b["status"].data_ptr())
    capi.check(rc, "noalloc: " + capi.last_error())
    return case.result(b)


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    cases = [_Case(300_007, 8192, 32, "uniform", 42), _Case(150_001, 1024, 8, "zipf", 7)]
    for case in cases:  # two calls in a row share the static scratch
        got = _static(case)
        exp = _allocating(case)
        assert got[0] == 0 and exp[0] == 0
        assert np.array_equal(got[1], exp[1])  # per-port totals
        assert np.array_equal(got[2], exp[2])  # binBase
        assert np.array_equal(got[3], exp[3])  # (fill, port) of every output chunk
        for a, e in zip(got[4], exp[4]):
            assert np.array_equal(a, e)        # every port's sequence, in order
        counts, _ = O.partition_stable_u32(case.keys, case.bins, want_order=False)
        assert np.array_equal(got[1], counts)


def test_noalloc_rejects_batches_beyond_its_scratch():
    L = capi.lib()
    rc = _noalloc()(None, None, None, 8192, 0, None, 200_000, 4096, 64, capi.CLS_KEY_MOD, None, 0, None, None, 1, None,
                    None, 0, None, None)
    assert rc == capi.GF_ERR_RANGE
    assert "static scratch" in capi.last_error()
    del L
