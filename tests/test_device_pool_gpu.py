"""Device-resident chunk pool (gf_device_pool_*) and the dense chain run entirely on the device with
it (gf_run_dense_chain_device).

The pool must hand out and take back chunks exactly as the host pool does (core/ChunkPool.hpp:
88-190 and core/ChunkLedger.hpp:33-150: the free list is filled S-1 .. 0 and popped from the back,
a release is pushed on the back; a release of a chunk that is not live fails), with the reservation
credits of sched/GraphRunner.hpp:1014-1037 (reserve a batch's outputChunkBound, keep what the plan
used, give the rest back). A Python restatement of that host pool is the model. The device chain
must give every particle the port of the Flow's chain and of the oracle's keys, per-node counts
bit-exact against the oracle, and leave every chunk free."""
import ctypes as C
import random

import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NO_CHUNK = 0xFFFFFFFF


class HostPoolModel:
    """The host pool's free list and liveness (core/ChunkPool.hpp:88-190)."""

    def __init__(self, s):
        self.free = list(range(s - 1, -1, -1))
        self.live = set()
        self.acquired = self.released = self.peak = 0
        self.s = s

    def acquire(self, k):
        if k > len(self.free):
            return None
        out = [self.free.pop() for _ in range(k)]
        self.live.update(out)
        self.acquired += k
        self.peak = max(self.peak, len(self.live))
        return out

    def settle(self, reserved, used, released):
        unused = reserved[used:]
        if any(c not in self.live for c in released) or len(set(released)) != len(released) or \
                set(unused) & set(released):
            return False
        for c in reversed(unused):   # back where they were: the first unused one is handed out next
            self.free.append(c)
            self.live.discard(c)
        self.acquired -= len(unused)
        for c in released:
            self.live.discard(c)
            self.free.append(c)
        self.released += len(released)
        return True


class DevicePool:
    def __init__(self, s):
        self.L = capi.lib()
        self.s = s
        nbytes = capi.device_pool_bytes(s)
        self.mem = torch.zeros((nbytes + 15) // 16 * 2, dtype=torch.int64, device="cuda")
        self.status = torch.zeros(1, dtype=torch.int32, device="cuda")
        capi.check(self.L.gf_device_pool_init(None, self.ptr, s), "pool init")

    @property
    def ptr(self):
        return self.mem.data_ptr()

    def acquire(self, k):
        ids = torch.zeros(max(k, 1), dtype=torch.int32, device="cuda")
        capi.check(self.L.gf_device_pool_acquire(None, self.ptr, k, ids.data_ptr(), self.status.data_ptr()),
                   "acquire")
        return [int(x) & 0xFFFFFFFF for x in ids[:k].cpu()]

    def settle(self, reserved, used, released, stride=1):
        res = torch.tensor([x if x < 2**31 else x - 2**32 for x in reserved] or [0], dtype=torch.int32,
                           device="cuda")
        flat = []
        for c in released:
            flat += [c] + [0] * (stride - 1)
        rel = torch.tensor([x if x < 2**31 else x - 2**32 for x in flat] or [0], dtype=torch.int32, device="cuda")
        capi.check(self.L.gf_device_pool_settle(None, self.ptr, res.data_ptr(), len(reserved), None, used,
                                                rel.data_ptr(), stride, None, len(released),
                                                self.status.data_ptr()), "settle")

    def stats(self):
        st = capi.DevicePoolStats()
        capi.check(self.L.gf_device_pool_read(None, self.ptr, C.byref(st)), "read")
        return st

    def take_status(self):
        v = int(self.status.item())
        self.status.zero_()
        return v


def test_fresh_pool_order_and_lifo_release():
    p = DevicePool(10)
    assert p.acquire(3) == [0, 1, 2]
    p.settle([0, 1, 2], 1, [])            # reservation of 3, one used: 1 and 2 go back in place
    assert p.acquire(2) == [1, 2]
    p.settle([], 0, [0, 2])               # released last = handed out first
    assert p.acquire(3) == [2, 0, 3]
    st = p.stats()
    assert (st.num_chunks, st.free_chunks, st.status) == (10, 6, 0)
    assert st.acquired == 6 and st.released == 2 and st.peak_live == 4
    assert p.take_status() == 0


def test_exhaustion_takes_nothing():
    p = DevicePool(4)
    assert p.acquire(3) == [0, 1, 2]
    assert p.acquire(2) == [NO_CHUNK, NO_CHUNK]
    assert p.take_status() == capi.GF_OVERFLOW
    st = p.stats()
    assert st.free_chunks == 1 and st.status == capi.GF_OVERFLOW
    assert p.acquire(1) == [3]


@pytest.mark.parametrize("released", [[5], [1, 1], [9], [1, 3]])
def test_bad_release_changes_nothing(released):
    """Not live (5), named twice, out of range, or one of the unused reservations (3)."""
    p = DevicePool(8)
    got = p.acquire(4)                   # 0 1 2 3: 0..1 used, 2..3 come back
    p.settle(got, 2, released)
    assert p.take_status() == capi.GF_INVALID
    st = p.stats()
    assert st.free_chunks == 4 and st.released == 0
    p.settle(got, 2, [0])                # the pool still works: the same settle without the bad name
    assert p.take_status() == 0
    assert p.acquire(4) == [0, 2, 3, 4]


def test_stale_reservation_is_rejected():
    p = DevicePool(8)
    a = p.acquire(3)
    p.acquire(1)                         # another acquisition in between: 'a' is no longer in front
    p.settle(a, 1, [])
    assert p.take_status() == capi.GF_INVALID


def test_pool_matches_host_model_on_random_operations():
    rng = random.Random(1234)
    s = 64
    p, m = DevicePool(s), HostPoolModel(s)
    live = []
    for step in range(300):
        if rng.random() < 0.55:
            k = rng.randint(0, 12)
            got, exp = p.acquire(k), m.acquire(k)
            if exp is None:
                assert got == [NO_CHUNK] * k and p.take_status() == capi.GF_OVERFLOW
                continue
            assert got == exp, step
            used = rng.randint(0, k)
            rel = rng.sample(live, rng.randint(0, min(len(live), 6))) if live else []
            ok = m.settle(exp, used, rel)
            p.settle(got, used, rel, stride=rng.choice([1, 3]))
            assert ok and p.take_status() == 0
            live = [c for c in live if c not in rel] + exp[:used]
        else:
            rel = rng.sample(live, rng.randint(0, min(len(live), 8))) if live else []
            assert m.settle([], 0, rel)
            p.settle([], 0, rel)
            assert p.take_status() == 0
            live = [c for c in live if c not in rel]
    st = p.stats()
    assert st.free_chunks == len(m.free) and st.acquired == m.acquired and st.released == m.released
    assert st.peak_live == m.peak and st.status == 0
    assert p.acquire(len(m.free)) == m.acquire(len(m.free))


def _expect(n, bins, nodes, dist, seed):
    keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
    return keys, ((keys >> np.uint32(8 * (nodes - 1))) % np.uint32(bins)).astype(np.uint32)


@pytest.mark.parametrize("n", [0, 1, 4097, 300_007])
@pytest.mark.parametrize("nodes,bins,dist", [(1, 2, "uniform"), (4, 8, "zipf"), (2, 32, "round_robin"),
                                             (4, 64, "uniform"), (3, 64, "one_port")])
def test_device_chain_matches_oracle(n, nodes, bins, dist):
    seed = 42
    port_of, totals, pool, st = capi.run_dense_chain_device(seed, n, bins, nodes=nodes, dist=dist)
    keys, exp = _expect(n, bins, nodes, dist, seed)
    assert np.array_equal(port_of, exp)
    for i in range(nodes):
        node_ports = (keys >> np.uint32(8 * i)) % np.uint32(bins)
        assert np.array_equal(totals[i], np.bincount(node_ports, minlength=bins)), i
    assert st.generated == n and st.sunk == n and st.partition_launches == nodes
    assert pool.status == 0 and pool.free_chunks == pool.num_chunks
    assert pool.acquired == pool.released
    bound = O.output_chunk_bound(n, 8192, bins)
    assert pool.num_chunks == max(-(-n // 8192), bound) + bound


def test_device_chain_equals_flow_chain():
    n, seed, bins, nodes = 500_009, 9, 32, 4
    dev, _, _, _ = capi.run_dense_chain_device(seed, n, bins, nodes=nodes, dist="zipf")
    flow, _ = capi.run_dense_chain(seed, n, bins, nodes=nodes, dist="zipf", chunk_capacity=8192,
                                   live_particles=16384, batch_chunks=8)
    assert np.array_equal(dev, flow)


def test_device_chain_argument_errors():
    with pytest.raises(capi.GfError):
        capi.run_dense_chain_device(1, 10, 5)
    with pytest.raises(capi.GfError):
        capi.run_dense_chain_device(1, 10, 8, nodes=5)


def test_device_chain_full_size_matches_oracle():
    """The 4-node chain of the dense sweep at its stated size (N = 1e8, B = 64 uniform, C = 8192)."""
    n, seed, bins, nodes = 100_000_000, 42, 64, 4
    port_of, totals, pool, st = capi.run_dense_chain_device(seed, n, bins, nodes=nodes)
    keys, exp = _expect(n, bins, nodes, "uniform", seed)
    assert np.array_equal(port_of, exp)
    for i in range(nodes):
        assert np.array_equal(totals[i], np.bincount((keys >> np.uint32(8 * i)) % np.uint32(bins),
                                                     minlength=bins)), i
    assert st.sunk == n and pool.free_chunks == pool.num_chunks and pool.status == 0
    print(f"device chain N=1e8, 4 nodes: {st.loop_seconds * 1e3:.2f} ms on the device, "
          f"{n / st.loop_seconds:.3e} particles/s, {st.seconds:.3f} s wall, peak live {pool.peak_live} "
          f"of {pool.num_chunks} chunks")
