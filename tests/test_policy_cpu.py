"""The device policy for the default C, P and T (core/DevicePolicy.hpp:344-614 makeDevicePolicy),
through gf_device_policy with explicit device properties (no GPU needed).

The pinned values are the reference's own (tests/unit/test_backend.cpp:134-340): an
accelerator-shaped device of 108 SMs with 24 GiB gets T = 128, a 3 GiB budget, C = 8192 and
P = 16384; with 2 GiB the budget is 256 MiB and C shrinks; explicit overrides are kept; impossible
overrides are rejected. With the Flow's accelerator ratio P/C = 8 the budget bisection halves C
and doubles the chunks in flight (DevicePolicy.hpp:45-53): C = 4096, P = 32768 on a B200 under the
reference's 3 GiB budget cap.
"""
import pytest

from graphflow_b200 import capi

GIB = 1 << 30
SLOT = 24  # payload bytes per slot the reference's policy charges by default


def _gpu(sms=108, mem=24 * GIB, grid=0x7FFFFFFF, smem=48 * 1024):
    return capi.DeviceProps(sms, 32, 1024, grid, smem, mem)


def _fits(p, slot=SLOT):
    return p.live_particles * p.chunk_capacity * slot <= p.budget_bytes


def test_policy_derives_the_budget_from_device_memory():
    high = capi.device_policy(100_000_000, _gpu(mem=24 * GIB))
    assert (high.tile_size, high.budget_bytes, high.chunk_capacity, high.live_particles) == (128, 3 * GIB, 8192, 16384)
    assert _fits(high) and high.live_explicit == 0
    low = capi.device_policy(100_000_000, _gpu(mem=2 * GIB))
    assert low.tile_size == 128 and low.budget_bytes == 256 << 20
    assert low.chunk_capacity < high.chunk_capacity and low.chunk_capacity % low.tile_size == 0 and _fits(low)


def test_policy_on_a_b200_with_the_flow_ratio():
    b200 = _gpu(sms=148, mem=183_359 << 20)
    p = capi.device_policy(100_000_000, b200, live_per_chunk=8)
    assert (p.chunk_capacity, p.live_particles, p.tile_size, p.budget_bytes) == (4096, 32768, 128, 3 * GIB)
    assert _fits(p)
    # {u32 id, u32 key} records: 8 C^2 x 8 B <= 3 GiB -> C = 7040 (a multiple of T), P = 8 C
    dense = capi.device_policy(100_000_000, b200, live_per_chunk=8, slot_bytes=8)
    assert (dense.chunk_capacity, dense.live_particles) == (7040, 56320) and _fits(dense, 8)
    # the published configuration passes C and P; the policy keeps them
    pub = capi.device_policy(100_000_000, b200, chunk_capacity=8192, live_particles=16384)
    assert (pub.chunk_capacity, pub.live_particles) == (8192, 16384)


def test_policy_caps_by_the_budget():
    low = capi.device_policy(4_000_000, _gpu(), budget_bytes=64 << 20)
    high = capi.device_policy(4_000_000, _gpu(), budget_bytes=GIB)
    assert low.budget_bytes == 64 << 20 and high.budget_bytes == GIB
    assert low.chunk_capacity < high.chunk_capacity
    assert low.chunk_capacity % low.tile_size == 0 and high.chunk_capacity % high.tile_size == 0
    assert _fits(low) and _fits(high)


def test_policy_keeps_explicit_overrides():
    d = _gpu()
    p = capi.device_policy(4096, d, chunk_capacity=256, live_particles=512, tile_size=64, budget_bytes=GIB)
    assert (p.chunk_capacity, p.live_particles, p.tile_size, p.live_explicit) == (256, 512, 64, 1) and _fits(p)
    odd = capi.device_policy(4096, d, chunk_capacity=100, tile_size=64, budget_bytes=GIB)
    assert (odd.chunk_capacity, odd.tile_size, odd.live_particles) == (100, 64, 200)   # P = min(N, 2C)
    t = capi.device_policy(4096, d, tile_size=32, budget_bytes=GIB)
    assert t.tile_size == 32 and t.chunk_capacity % 32 == 0
    assert capi.device_policy(4096, d, live_particles=100, budget_bytes=GIB).live_particles == 100
    # an explicit C squeezes the derived P instead of being rejected
    sq = capi.device_policy(100_000, d, chunk_capacity=8192, budget_bytes=8 << 20)
    assert sq.chunk_capacity == 8192 and sq.live_particles <= (8 << 20) // (8192 * SLOT) and _fits(sq)


@pytest.mark.parametrize("kw", [
    dict(n=1000, tile_size=1025),                                   # above maxThreadsPerBlock
    dict(n=1000, chunk_capacity=8193),                              # above the configured maximum
    dict(n=1000, live_particles=1001),                              # above N
    dict(n=1000, chunk_capacity=256, grid=1),                       # more tiles than the grid allows
    dict(n=4096, live_particles=512, budget_bytes=1024),            # budget below one tile
    dict(n=100_000, chunk_capacity=8192, live_particles=4096, budget_bytes=64 << 10),  # P x C over budget
])
def test_policy_rejects_impossible_requests(kw):
    kw = dict(kw)
    n, grid = kw.pop("n"), kw.pop("grid", 0x7FFFFFFF)
    kw.setdefault("budget_bytes", GIB)
    with pytest.raises(capi.GfError):
        capi.device_policy(n, _gpu(grid=grid), **kw)


@pytest.mark.parametrize("n", [0, 1, 127, 128, 4097, 1_000_000, 100_000_000])
def test_policy_invariants_across_run_sizes(n):
    p = capi.device_policy(n, _gpu())
    assert p.chunk_capacity % p.tile_size == 0 and p.live_particles <= n and _fits(p)
    assert (p.live_particles == 0) == (n == 0)
