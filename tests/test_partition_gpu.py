"""GPU parity of the dense partition path against the CPU oracle.

Mirrors the reference's dense-bin and batching tests (tests/integration/test_dense_bins.cpp,
test_batching.cpp:402-602, test_hash_bins.cpp:286-502 for id % B expectations):
per-port counts and the exact plan are bit-exact; per-port multisets are bit-exact for the
two-launch form (whose in-port order is atomic order, ScatterKernel.hpp:255-257) and per-port
sequences are bit-exact for the fused form (stable partition in input order).
"""
import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from graphflow_b200.partition import BatchError, ChunkPool, FusedPartition, PlainPartition
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DISTS = ["uniform", "zipf", "one_port", "round_robin"]


def _device_keys(dist, seed, n, bins, first_id=0):
    keys = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    cdf = None
    if dist == "zipf":
        cdf = torch.from_numpy(capi.zipf_cdf(1.1, bins)).cuda()
    capi.check(capi.lib().gf_generate_keys_u32(None, capi.DIST_NAMES[dist], seed, first_id, n, bins,
                                               cdf.data_ptr() if cdf is not None else None, keys.data_ptr()),
               "generate")
    torch.cuda.synchronize()
    return keys[:n].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("dist", DISTS)
@pytest.mark.parametrize("bins", [2, 64])
def test_key_source_matches_oracle(dist, bins):
    n = 300_001
    got = _device_keys(dist, 42, n, bins, first_id=5)
    exp = O.generate_keys_u32(dist, 42, n, bins, zipf_s=1.1, first_id=5)
    assert np.array_equal(got, exp)


def _fill_pool(pool, chunks, fills, keys):
    col = pool.column.cpu().numpy().view(np.uint32)
    off = 0
    for c, f in zip(chunks, fills):
        col[c * pool.capacity: c * pool.capacity + f] = keys[off: off + f]
        off += f
    pool.column.copy_(torch.from_numpy(col.view(np.int32)))


def _batch(n, capacity, rng, shuffle=True, ragged=True):
    """Chunk list and fills for n particles; ragged fills and shuffled chunk indices."""
    fills = []
    left = n
    while left > 0:
        f = capacity if not ragged else int(rng.integers(1, capacity + 1))
        f = min(f, left)
        fills.append(f)
        left -= f
    chunks = list(range(len(fills)))
    if shuffle:
        rng.shuffle(chunks)
    return chunks, fills


def _outputs(pool, table, descs, bins):
    col = pool.column.cpu().numpy().view(np.uint32)
    per_port = [[] for _ in range(bins)]
    for chunk, fill, b in descs:
        per_port[int(b)].append(col[int(chunk) * pool.capacity: int(chunk) * pool.capacity + int(fill)])
    return [np.concatenate(p) if p else np.zeros(0, np.uint32) for p in per_port]


def _check(pool, chunks, fills, keys, bins, result, exact_order, in_snapshot):
    totals, table, descs = result
    counts, order = O.partition_stable_u32(keys, bins)
    assert np.array_equal(totals, counts)
    base, ofills, r = O.plan_dense(counts, pool.capacity)
    assert np.array_equal(table[:bins], base)
    assert len(descs) == r
    assert np.array_equal(descs[:, 1], ofills)
    assert np.array_equal(descs[:, 2], np.repeat(np.arange(bins), (counts + pool.capacity - 1) // pool.capacity))
    assert np.array_equal(table[bins:], descs[:, 0])
    used = descs[:, 0].astype(np.int64)
    assert len(set(used.tolist())) == len(used)
    assert not (set(used.tolist()) & set(chunks))
    got = _outputs(pool, table, descs, bins)
    start = 0
    for b in range(bins):
        exp = keys[order[start:start + counts[b]]]
        start += counts[b]
        if exact_order:
            assert np.array_equal(got[b], exp), f"port {b}"
        else:
            assert np.array_equal(np.sort(got[b]), np.sort(exp)), f"port {b}"
    # inputs untouched
    col = pool.column.cpu().numpy().view(np.uint32)
    for c in chunks:
        assert np.array_equal(col[c * pool.capacity:(c + 1) * pool.capacity], in_snapshot[c])


def _run_case(kind, n, capacity, bins, dist, tile_size, seed=42, mode=capi.SCATTER_SHARED, ragged=True):
    rng = np.random.default_rng(seed + n + bins)
    chunks, fills = _batch(n, capacity, rng, ragged=ragged)
    n_in = len(chunks)
    bound = capi.output_chunk_bound(n, capacity, bins)
    pool = ChunkPool(n_in + bound + 3, capacity)
    keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
    _fill_pool(pool, chunks, fills, keys)
    for c in chunks:
        pool.free.remove(c)
    col = pool.column.cpu().numpy().view(np.uint32)
    snap = {c: col[c * capacity:(c + 1) * capacity].copy() for c in chunks}
    # the batch is the concatenation of the chunks in list order (tile order)
    if kind == "plain":
        part = PlainPartition(pool, bins, tile_size=tile_size, mode=mode)
    else:
        part = FusedPartition(pool, bins, tile_size=tile_size, max_batch_particles=max(n, 1))
    result = part.run(chunks, fills)
    _check(pool, chunks, fills, keys, bins, result, exact_order=(kind == "fused"), in_snapshot=snap)
    return part


@pytest.mark.parametrize("kind", ["plain", "fused"])
@pytest.mark.parametrize("dist", DISTS)
@pytest.mark.parametrize("bins", [2, 8, 32, 64])
def test_partition_matches_oracle(kind, dist, bins):
    _run_case(kind, 200_003, 8192, bins, dist, 4096)


@pytest.mark.parametrize("kind", ["plain", "fused"])
@pytest.mark.parametrize("n", [0, 1, 17, 4097])
@pytest.mark.parametrize("capacity", [127, 1024])
def test_partition_small_and_ragged(kind, n, capacity):
    _run_case(kind, n, capacity, 8, "uniform", 1024)


@pytest.mark.parametrize("tile_size", [1024, 2048, 4096, 8192])
def test_fused_tile_sizes_many_tiles(tile_size):
    # ~1000 tiles of look-back at the smallest tile size; full chunks
    _run_case("fused", 1_000_003, 8192, 32, "zipf", tile_size, ragged=False)


@pytest.mark.parametrize("combined", [True, False])
@pytest.mark.parametrize("coop", [1, 0])
@pytest.mark.parametrize("bins,capacity,tile_size,dist", [
    (1, 8192, 4096, "uniform"),        # one port: every tile one run
    (3, 4096, 4096, "uniform"),        # key mod 3 (division path); runs cross chunk boundaries often
    (17, 4100, 4096, "zipf"),          # capacity not a power of two, heavy skew
    (63, 4096, 2048, "round_robin"),   # a run in every port of every tile
    (64, 8192, 1024, "one_port"),
    (3, 1024, 4096, "uniform"),        # capacity below 4096: per-tile kernel
    (64, 8192, 8192, "uniform"),       # tiles above 4096: per-tile kernel
])
def test_fused_kernels_match_oracle(combined, coop, bins, capacity, tile_size, dist):
    """Both fused kernels (the cooperative count/plan/scatter kernel and the per-tile look-back
    kernel) give the oracle's counts, plan and per-port sequences; the cooperative kernel also
    takes the output chunks in plan order (table[B + f] = reserved[f]). Both forms of the finish:
    inside the partition launch (gf_partition_fused_full_u32) and as its own launch."""
    capi.check(capi.lib().gf_set_tuning(b"fused_coop", coop), "tuning")
    try:
        n = 250_007
        rng = np.random.default_rng(5)
        chunks, fills = _batch(n, capacity, rng)
        bound = capi.output_chunk_bound(n, capacity, bins)
        pool = ChunkPool(len(chunks) + bound + 3, capacity)
        keys = O.generate_keys_u32(dist, 11, n, bins, zipf_s=1.1)
        _fill_pool(pool, chunks, fills, keys)
        for ch in chunks:
            pool.free.remove(ch)
        col = pool.column.cpu().numpy().view(np.uint32)
        snap = {ch: col[ch * capacity:(ch + 1) * capacity].copy() for ch in chunks}
        expect_reserved = list(pool.free)[:bound]
        part = FusedPartition(pool, bins, tile_size=tile_size, max_batch_particles=n)
        part.combined = combined
        totals, table, descs = part.run(chunks, fills)
        _check(pool, chunks, fills, keys, bins, (totals, table, descs), exact_order=True, in_snapshot=snap)
        if coop and tile_size <= 4096 and capacity >= 4096:
            assert np.array_equal(table[bins:], np.asarray(expect_reserved[:len(descs)], np.uint32))
    finally:
        capi.check(capi.lib().gf_set_tuning(b"fused_coop", 1), "tuning")


def test_fused_many_tiles_per_cta_and_skew():
    """A batch large enough that every CTA of the cooperative grid owns many tiles, with all keys
    in one port (one output run per tile, thousands of output chunks in one port)."""
    _run_case("fused", 12_000_017, 8192, 8, "one_port", 4096, ragged=False)


def test_plain_direct_mode_matches_oracle():
    _run_case("plain", 100_000, 1024, 64, "uniform", 2048, mode=capi.SCATTER_DIRECT)


def test_plain_counts_one_classify_and_one_scatter_per_batch():
    # tests/integration/test_batching.cpp:402-450: a batch is two launches regardless of its chunks
    part = _run_case("plain", 50_000, 1024, 2, "round_robin", 1024)
    assert part.classify_launches == 1 and part.scatter_launches == 1


def test_fused_repeated_batches_share_scratch():
    rng = np.random.default_rng(3)
    capacity, bins = 1024, 8
    pool = ChunkPool(400, capacity)
    fused = FusedPartition(pool, bins, tile_size=1024, max_batch_particles=60_000)
    for it in range(4):
        n = int(rng.integers(1, 60_000))
        chunks = pool.acquire(-(-n // capacity))
        fills = [capacity] * (len(chunks) - 1) + [n - capacity * (len(chunks) - 1)]
        keys = O.generate_keys_u32("uniform", 100 + it, n, bins)
        _fill_pool(pool, chunks, fills, keys)
        col = pool.column.cpu().numpy().view(np.uint32)
        snap = {c: col[c * capacity:(c + 1) * capacity].copy() for c in chunks}
        res = fused.run(chunks, fills)
        _check(pool, chunks, fills, keys, bins, res, True, snap)
        pool.release(chunks)
        pool.release([int(c) for c in res[2][:, 0]])


def test_oversized_tile_sets_status_invalid():
    pool = ChunkPool(4, 2048)
    bins = 4
    counts = torch.zeros(bins + 1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    bin_ids = torch.zeros(pool.slots, dtype=torch.int32, device="cuda")
    tiles = torch.tensor([0, 0, 2048], dtype=torch.int32, device="cuda")  # count 2048 > tile size 1024
    capi.check(capi.lib().gf_classify_dense_u32(None, pool.ptr(), pool.capacity, pool.slots, tiles.data_ptr(), 1,
                                                1024, bins, capi.CLS_KEY_MOD, bin_ids.data_ptr(),
                                                counts.data_ptr(), status.data_ptr()), "classify")
    torch.cuda.synchronize()
    assert int(status.item()) == capi.GF_INVALID
    assert int(counts[:bins].sum().item()) == 0


def test_cooperative_scratch_reads_unpublished_to_the_per_tile_kernel():
    """A caller scratch serves the cooperative kernel, then the per-tile look-back kernel. The
    per-tile kernel reads the scratch as 64-bit (epoch, flag, value) descriptors and accepts a word
    whose flag bits (33..32) are non-zero and whose epoch is its own; whatever the cooperative
    kernel leaves there must carry flag 0. The first batch's port-1 total is 9 = 4 x 2 + 1, the
    flag-1 word of the next launch's epoch (2) in a layout that stored raw 32-bit totals."""
    capacity, bins = 8192, 2
    n_odd, n_even = 9, 300_000
    keys = np.concatenate([np.full(n_even, 4, np.uint32), np.full(n_odd, 7, np.uint32)])
    n_in = -(-keys.size // capacity)
    pool = ChunkPool(n_in + capi.output_chunk_bound(keys.size, capacity, bins) + 8, capacity)
    chunks = list(range(n_in))
    fills = [capacity] * (n_in - 1) + [keys.size - capacity * (n_in - 1)]
    _fill_pool(pool, chunks, fills, keys)
    for c in chunks:
        pool.free.remove(c)
    part = FusedPartition(pool, bins, tile_size=4096, max_batch_particles=8_000_000)
    part.scratch.zero_()
    totals, _, descs = part.run(chunks, fills)
    assert list(totals) == [n_even, n_odd]
    words = part.scratch.cpu().numpy().view(np.uint64)[8:]  # after the 64-byte control block
    assert not np.any(words & np.uint64(3 << 32)), "a cooperative word reads as a published descriptor"
    # the next batch on the same scratch runs the per-tile kernel (chunks of 1024 slots)
    pool2 = ChunkPool(400, 1024)
    part2 = FusedPartition(pool2, bins, tile_size=1024, max_batch_particles=200_003)
    assert part.scratch_bytes >= part2.scratch_bytes
    part2.scratch, part2.scratch_bytes = part.scratch, part.scratch_bytes
    k2 = O.generate_keys_u32("uniform", 5, 200_003, bins)
    chunks2 = pool2.acquire(-(-k2.size // 1024))
    fills2 = [1024] * (len(chunks2) - 1) + [k2.size - 1024 * (len(chunks2) - 1)]
    _fill_pool(pool2, chunks2, fills2, k2)
    col = pool2.column.cpu().numpy().view(np.uint32)
    snap = {c: col[c * 1024:(c + 1) * 1024].copy() for c in chunks2}
    _check(pool2, chunks2, fills2, k2, bins, part2.run(chunks2, fills2), True, snap)


def test_cooperative_barrier_wait_gives_up_under_a_short_limit():
    """Failure detection without a fault: with the poll budget of the waits between CTAs cut to
    one poll (tuning knob spin_limit), every CTA of the cooperative launch but the last to arrive
    gives up at the grid barrier. The batch reports GF_ERR_TIMEOUT, nothing is published (the
    reservation goes back to the pool), and with the default budget restored the next batch on the
    same scratch is exact."""
    n, capacity, bins = 4_000_003, 8192, 64
    keys = O.generate_keys_u32("uniform", 9, n, bins)
    n_in = -(-n // capacity)
    pool = ChunkPool(n_in + capi.output_chunk_bound(n, capacity, bins), capacity)
    chunks = list(range(n_in))
    fills = [capacity] * (n_in - 1) + [n - capacity * (n_in - 1)]
    _fill_pool(pool, chunks, fills, keys)
    for c in chunks:
        pool.free.remove(c)
    col = pool.column.cpu().numpy().view(np.uint32)
    snap = {c: col[c * capacity:(c + 1) * capacity].copy() for c in chunks}
    part = FusedPartition(pool, bins, tile_size=4096, max_batch_particles=n)
    free_before = len(pool.free)
    capi.check(capi.lib().gf_set_tuning(b"spin_limit", 1), "tuning")
    try:
        with pytest.raises(BatchError):
            part.run(chunks, fills)
        assert int(part.status.item()) == capi.GF_ERR_TIMEOUT
        assert len(pool.free) == free_before
    finally:
        capi.check(capi.lib().gf_set_tuning(b"spin_limit", 0), "tuning")
    _check(pool, chunks, fills, keys, bins, part.run(chunks, fills), True, snap)
