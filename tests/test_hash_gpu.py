"""GPU parity of the hash-bin path (16-byte records, SoA and AoS) against the CPU oracle.

Mirrors tests/integration/test_hash_bins.cpp:286-685 of the reference (hash vs dense agreement,
sparse 4096 / 65536 bins): per-port counts and the exact plan are bit-exact; per-port record
multisets are bit-exact (in-port order is atomic order, as in the reference). Port counts up to
2^20 extend the reference's 65536-bin limit (core/Config.hpp:190).
"""
import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from graphflow_b200.hashpart import HashPartition, RecordPool
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SALT = 0x5EED5A17


def _device_records(n, k, s, layout, first_id=0):
    pool = RecordPool(1, max(n, 1), layout=layout)
    cdf = torch.from_numpy(capi.zipf_cdf(s, k)).cuda()
    capi.check(capi.lib().gf_generate_records16(None, 42, first_id, n, cdf.data_ptr(), k, SALT,
                                                __import__("ctypes").byref(pool.cols), layout), "generate")
    torch.cuda.synchronize()
    return pool.host_slots(0, n)


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
@pytest.mark.parametrize("k,s", [(1024, 0.8), (65536, 1.2), (2**20, 1.2)])
def test_record_source_matches_oracle(layout, k, s):
    n = 100_003
    gk, gw, gt = _device_records(n, k, s, layout, first_id=7)
    ek, ew, et = O.generate_records16(42, n, k, s, SALT, first_id=7)
    assert np.array_equal(gk, ek) and np.array_equal(gw.view(np.uint32), ew.view(np.uint32)) and np.array_equal(gt, et)


def _run(layout, form, n, k, s, capacity=8192, tile=1024, seed_shift=0):
    rng = np.random.default_rng(n + k + seed_shift)
    fills, left = [], n
    while left > 0:
        f = min(int(rng.integers(1, capacity + 1)), left)
        fills.append(f)
        left -= f
    n_in = len(fills)
    chunks = list(rng.permutation(n_in))
    bound = capi.output_chunk_bound(n, capacity, k)
    pool = RecordPool(n_in + bound + 2, capacity, layout=layout)
    keys, weights, tags = O.generate_records16(42, n, k, s, SALT)
    off = 0
    for c, f in zip(chunks, fills):
        pool.set_slots(int(c) * capacity, keys[off:off + f], weights[off:off + f], tags[off:off + f])
        off += f
    for c in chunks:
        pool.free.remove(int(c))
    part = HashPartition(pool, k, SALT, tile_size=tile, form=form, max_batch_particles=max(n, 1))
    totals, table, descs = part.run([int(c) for c in chunks], fills)
    counts, order = O.partition_stable_u64(keys, k, O.CLS_KEY_UNMIX, SALT)
    assert np.array_equal(totals, counts)
    base, ofills, r = O.plan_dense(counts, capacity)
    assert np.array_equal(table[:k], base) and len(descs) == r and np.array_equal(descs[:, 1], ofills)
    assert len(set(descs[:, 0].tolist())) == r and not (set(descs[:, 0].tolist()) & set(int(c) for c in chunks))
    # gather every output chunk once, then compare per-port record multisets through the tags
    got_tags = np.zeros(n, np.uint32)
    got_port = np.zeros(n, np.uint32)
    pos = 0
    for chunk, fill, b in descs:
        gk, gw, gt = pool.host_slots(int(chunk) * capacity, int(chunk) * capacity + int(fill))
        assert np.array_equal(gk, keys[gt]) and np.array_equal(gw.view(np.uint32), weights[gt].view(np.uint32))
        got_tags[pos:pos + fill] = gt
        got_port[pos:pos + fill] = b
        pos += fill
    assert pos == n
    exp_port = np.zeros(n, np.uint32)
    start = 0
    for b in np.nonzero(counts)[0]:
        exp_port[order[start:start + counts[b]]] = b
        start += counts[b]
    assert np.array_equal(np.sort(got_tags), np.arange(n, dtype=np.uint32))
    assert np.array_equal(got_port[np.argsort(got_tags)], exp_port)


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
@pytest.mark.parametrize("form", ["plain", "device"])
@pytest.mark.parametrize("k,s", [(1024, 0.8), (1024, 1.2), (65536, 0.8), (2**20, 1.2)])
def test_hash_partition_matches_oracle(layout, form, k, s):
    _run(layout, form, 150_001, k, s)


@pytest.mark.parametrize("form", ["plain", "device"])
@pytest.mark.parametrize("n", [0, 1, 17, 4097])
def test_hash_partition_small(form, n):
    _run(capi.LAYOUT_SOA, form, n, 4096, 1.2, capacity=127, tile=2048)


def test_hash_one_bin_per_particle_sparse():
    # tests/integration/test_hash_bins.cpp: sparse 65536 bins, every particle in its own bin
    _run(capi.LAYOUT_AOS, "device", 60_000, 65536, 0.0, capacity=64, tile=2048)


@pytest.mark.parametrize("k", [2048, 2049, 70_000])
@pytest.mark.parametrize("tile", [1024, 2048])
def test_hash_kernel_forms_at_their_boundaries(k, tile):
    """Port counts on both sides of the grouped scatter's limit (2048 ports: direct-indexed
    per-unit grouping) and of the per-record persistent form (above 65536 ports)."""
    _run(capi.LAYOUT_SOA, "device", 90_001, k, 1.1, tile=tile)


@pytest.mark.parametrize("form", ["plain", "device"])
@pytest.mark.parametrize("k", [1024, 2**20])
def test_hash_per_tile_kernels_agree(form, k):
    """The per-tile open-addressing kernels (tuning knob hash_persistent = 0) give the same
    counts, plan and per-port multisets as the persistent kernels."""
    try:
        capi.check(capi.lib().gf_set_tuning(b"hash_persistent", 0), "tuning")
        _run(capi.LAYOUT_AOS, form, 80_003, k, 1.2, tile=2048)
    finally:
        capi.check(capi.lib().gf_set_tuning(b"hash_persistent", 1), "tuning")
