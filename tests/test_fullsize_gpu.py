"""GPU parity at the workloads' own sizes, against the oracle.

* Dense classify + plan + scatter of N = 1e8 u32 keys (B in {2, 8, 32, 64} x uniform, Zipf 1.1,
  one port, round robin; C = 8192, tiles of 4096, one whole-array batch): per-port counts and the
  exact plan (table, fills, bins) equal the oracle's; the fused form's per-port key sequences
  equal the oracle's stable partition; the plain two-launch form's per-port key multisets equal
  it (in-port order there is atomic order, as in the reference's ScatterKernel.hpp:255-257).
  Reference bar: tests/integration/test_dense_bins.cpp (multiset equality per bin).
* Hash classify + plan + scatter of N = 1e8 16-byte records {u64 key, f32 weight, u32 tag = id},
  Zipf 1.2 popularity over K in {2^10, 2^16, 2^20} keys, SoA and AoS, device-planned form:
  per-port counts and plan equal the oracle's, every output record is an input record (key and
  weight bits of its tag), and the per-port tag multisets equal the oracle's partition.
  Reference bar: tests/integration/test_hash_bins.cpp:286-502.
* photon_scattering, weighted Henyey-Greenstein slab in FP32 (N = 2e6) against the FP64 oracle:
  photon counts conserve N; the FP32 run's histograms equal the sums of its own per-photon exit
  records (FP32 accumulation, 5e-5 relative); and every one of the 2 x 256 exit-weight bins agrees
  with the oracle within
      |h32 - h64| <= 2e-4 h64 + k_i w_max,   k_i = the 1 - 1e-7 quantile of Poisson(2 f N_i),
  where f is the fraction of photons whose terminal event, scatter count or exit bin differs
  between the runs (FP32 rounding moves a photon across a bin edge or, rarely, flips a decision;
  required <= 1e-3), N_i the oracle's photon count in the bin and w_max the largest terminal
  weight. Photons that agree carry weights within 1e-4 relative (the 2e-4 term); a bin differs
  otherwise by the weights of the photons that moved in or out, whose number is Poisson with mean
  at most 2 f N_i.
The comparisons run on the device with torch (gathers, sorts, equality), fed by the oracle's
host results.
"""
import ctypes

import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from graphflow_b200.hashpart import HashPartition, RecordPool
from graphflow_b200.partition import ChunkPool, FusedPartition, PlainPartition
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 100_000_000
CAP = 8192
SALT = 0x5EED5A17


def _gather_u32(column, capacity, descs):
    """Concatenation, in descriptor (port) order, of the filled slots of the output chunks."""
    d = torch.from_numpy(descs.astype(np.int64)).cuda()
    rows = column.view(-1, capacity)[d[:, 0]]
    valid = torch.arange(capacity, device="cuda")[None, :] < d[:, 1:2]
    return rows[valid], torch.repeat_interleave(d[:, 2], d[:, 1])


def _check_plan(totals, table, descs, counts, capacity, bins, reserved):
    assert np.array_equal(totals, counts)
    base, ofills, r = O.plan_dense(counts, capacity)
    assert np.array_equal(table[:bins], base)
    assert len(descs) == r
    assert np.array_equal(descs[:, 1], ofills)
    assert np.array_equal(descs[:, 2], np.repeat(np.arange(bins), (counts + capacity - 1) // capacity))
    assert np.array_equal(table[bins:], descs[:, 0])
    used = descs[:, 0].astype(np.int64)
    assert len(np.unique(used)) == r and np.isin(used, reserved).all()


@pytest.fixture(scope="module")
def dense_keys():
    cache = {}

    def get(dist, bins):
        if (dist, bins) not in cache:
            cache.clear()
            cache[(dist, bins)] = O.generate_keys_u32(dist, 42, N, bins, zipf_s=1.1)
        return cache[(dist, bins)]
    return get


@pytest.mark.parametrize("kind", ["fused", "plain"])
@pytest.mark.parametrize("dist", ["uniform", "zipf", "one_port", "round_robin"])
@pytest.mark.parametrize("bins", [2, 8, 32, 64])
def test_dense_1e8_matches_oracle(dense_keys, kind, dist, bins):
    keys = dense_keys(dist, bins)
    n_in = -(-N // CAP)
    bound = capi.output_chunk_bound(N, CAP, bins)
    pool = ChunkPool(n_in + bound, CAP)
    pool.column[:N].copy_(torch.from_numpy(keys.view(np.int32)))
    chunks = list(range(n_in))
    fills = [CAP] * (n_in - 1) + [N - CAP * (n_in - 1)]
    for _ in range(n_in):
        pool.free.popleft()
    reserved = np.asarray(list(pool.free)[:bound], np.int64)
    if kind == "fused":
        part = FusedPartition(pool, bins, tile_size=4096, max_batch_particles=N)
    else:
        part = PlainPartition(pool, bins, tile_size=4096)
    totals, table, descs = part.run(chunks, fills)
    counts, order = O.partition_stable_u32(keys, bins)
    _check_plan(totals, table, descs, counts, CAP, bins, reserved)
    got, got_port = _gather_u32(pool.column, CAP, descs)
    assert got.numel() == N
    exp = torch.from_numpy(keys[order].view(np.int32)).cuda()
    if kind == "fused":
        assert torch.equal(got, exp)
    else:
        exp_port = torch.repeat_interleave(torch.arange(bins, device="cuda"), torch.from_numpy(
            counts.astype(np.int64)).cuda())
        assert torch.equal(got_port, exp_port)
        mask = 0xFFFFFFFF
        a = torch.sort((got_port << 32) | (got.to(torch.int64) & mask)).values
        b = torch.sort((exp_port << 32) | (exp.to(torch.int64) & mask)).values
        assert torch.equal(a, b)
    # the input chunks are untouched
    assert torch.equal(pool.column[:N], torch.from_numpy(keys.view(np.int32)).cuda())


HASH_CAPACITY = {1 << 10: 8192, 1 << 16: 2048, 1 << 20: 512}


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
@pytest.mark.parametrize("k", [1 << 10, 1 << 16, 1 << 20])
def test_hash_1e8_matches_oracle(layout, k):
    cap = HASH_CAPACITY[k]
    keys, weights, tags = O.generate_records16(42, N, k, 1.2, SALT)
    n_in = -(-N // cap)
    bound = capi.output_chunk_bound(N, cap, k)
    pool = RecordPool(n_in + bound, cap, layout=layout)
    pool.set_slots(0, keys, weights, tags)
    chunks = list(range(n_in))
    fills = [cap] * (n_in - 1) + [N - cap * (n_in - 1)]
    for _ in range(n_in):
        pool.free.popleft()
    reserved = np.asarray(list(pool.free)[:bound], np.int64)
    part = HashPartition(pool, k, SALT, tile_size=2048, form="device", max_batch_particles=N)
    totals, table, descs = part.run(chunks, fills)
    counts, order = O.partition_stable_u64(keys, k, O.CLS_KEY_UNMIX, SALT)
    _check_plan(totals, table, descs, counts, cap, k, reserved)
    d = torch.from_numpy(descs.astype(np.int64)).cuda()
    valid = torch.arange(cap, device="cuda")[None, :] < d[:, 1:2]
    if layout == capi.LAYOUT_SOA:
        got_key = pool.key.view(-1, cap)[d[:, 0]][valid]
        got_w = pool.weight.view(torch.int32).view(-1, cap)[d[:, 0]][valid]
        got_tag = pool.tag.view(-1, cap)[d[:, 0]][valid].to(torch.int64) & 0xFFFFFFFF
        in_key, in_w = pool.key[:N], pool.weight.view(torch.int32)[:N]
    else:
        rec = pool.records.view(-1, cap, 4)[d[:, 0]][valid]  # (N, 4) int32 words
        lo, hi = rec[:, 0].to(torch.int64) & 0xFFFFFFFF, rec[:, 1].to(torch.int64)
        got_key = lo | (hi << 32)
        got_w = rec[:, 2]
        got_tag = rec[:, 3].to(torch.int64) & 0xFFFFFFFF
        inr = pool.records.view(-1, 4)[:N]
        in_key = (inr[:, 0].to(torch.int64) & 0xFFFFFFFF) | (inr[:, 1].to(torch.int64) << 32)
        in_w = inr[:, 2]
    assert got_tag.numel() == N
    # every output record is the input record of its tag (tag = input position)
    assert torch.equal(got_key, in_key[got_tag]) and torch.equal(got_w, in_w[got_tag])
    got_port = torch.repeat_interleave(d[:, 2], d[:, 1])
    exp_port = torch.repeat_interleave(torch.arange(k, device="cuda"),
                                       torch.from_numpy(counts.astype(np.int64)).cuda())
    assert torch.equal(got_port, exp_port)
    exp = (exp_port << 32) | torch.from_numpy(order.astype(np.int64)).cuda()
    assert torch.equal(torch.sort((got_port << 32) | got_tag).values, exp)


def test_hash_k2e20_s08_matches_oracle():
    """K = 2^20 keys at Zipf 0.8 (a flat popularity: most ports hold a few records)."""
    n, k, cap = 2_000_003, 1 << 20, 512
    keys, weights, tags = O.generate_records16(42, n, k, 0.8, SALT)
    n_in = -(-n // cap)
    bound = capi.output_chunk_bound(n, cap, k)
    for layout in (capi.LAYOUT_SOA, capi.LAYOUT_AOS):
        pool = RecordPool(n_in + bound, cap, layout=layout)
        pool.set_slots(0, keys, weights, tags)
        for _ in range(n_in):
            pool.free.popleft()
        reserved = np.asarray(list(pool.free)[:bound], np.int64)
        part = HashPartition(pool, k, SALT, tile_size=2048, form="device", max_batch_particles=n)
        fills = [cap] * (n_in - 1) + [n - cap * (n_in - 1)]
        totals, table, descs = part.run(list(range(n_in)), fills)
        counts, order = O.partition_stable_u64(keys, k, O.CLS_KEY_UNMIX, SALT)
        _check_plan(totals, table, descs, counts, cap, k, reserved)
        got_tag = np.zeros(n, np.int64)
        got_port = np.zeros(n, np.int64)
        pos = 0
        for chunk, fill, b in descs:
            gk, gw, gt = pool.host_slots(int(chunk) * cap, int(chunk) * cap + int(fill))
            assert np.array_equal(gk, keys[gt]) and np.array_equal(gw.view(np.uint32), weights[gt].view(np.uint32))
            got_tag[pos:pos + fill] = gt
            got_port[pos:pos + fill] = b
            pos += fill
        assert pos == n
        exp = (np.repeat(np.arange(k, dtype=np.int64), counts) << 32) | order.astype(np.int64)
        assert np.array_equal(np.sort((got_port << 32) | got_tag), exp)


def _poisson_quantile(lam, tail=1e-7):
    """Smallest k with P(X > k) <= tail for X ~ Poisson(lam)."""
    k, pmf = 0, np.exp(-lam)
    cdf = pmf
    while 1.0 - cdf > tail:
        k += 1
        pmf *= lam / k
        cdf += pmf
    return k


def test_photon_fp32_exit_histograms_per_bin():
    n = 2_000_000
    p = capi.photon_params(model=capi.PHOTON_WEIGHTED, fp64=False)
    got = capi.run_photon(42, n, p, capi.EXEC_FUSED)
    refl, trans, ev, terms = O.photon_hg(42, n, O.hg_params(), want_terminals=True)
    assert int(got["event_counts"].sum()) == n and int(ev.sum()) == n
    nb = len(refl)
    b64 = np.minimum((terms["cos_exit"] * nb).astype(np.int64), nb - 1)
    b32 = np.minimum((got["cos_exit"] * nb).astype(np.int64), nb - 1)
    same = (got["event"] == terms["event"]) & (got["scatter_count"] == terms["scatter_count"]) & (b32 == b64)
    f = 1.0 - same.mean()
    assert f <= 1e-3
    w_ref = terms["weight"][same]
    assert np.all(np.abs(got["weight"][same] - w_ref) <= 1e-4 * w_ref)
    w_max = float(max(terms["weight"].max(), got["weight"].max()))
    for event, h32, h64 in ((2, got["refl"], refl), (1, got["trans"], trans)):
        s64, s32 = terms["event"] == event, got["event"] == event
        # each run's histogram is the sum of its photons' exit records
        assert np.allclose(np.bincount(b64[s64], weights=terms["weight"][s64], minlength=nb), h64, rtol=1e-12,
                           atol=1e-9)
        assert np.allclose(np.bincount(b32[s32], weights=got["weight"][s32], minlength=nb), h32, rtol=5e-5,
                           atol=1e-6)
        count = np.bincount(b64[s64], minlength=nb)
        k = np.array([_poisson_quantile(2.0 * f * c) for c in count])
        tol = 2e-4 * h64 + k * w_max
        assert np.all(np.abs(h32 - h64) <= tol), np.max(np.abs(h32 - h64) / tol)
