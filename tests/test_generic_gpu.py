"""The generic C ABI (gf_classify_dense, gf_scatter, gf_transform, gf_partition_fused over a
gf_columns descriptor with registered record, classifier, updater and transform ids) driven with
particle_feedback's 20-byte record {u64 id, u32 property, u32 weight, u32 visit}, in SoA (four
columns) and AoS (24-byte slots), against the oracle: the classifier draws are the oracle's keyed
Philox draws (rng/ParticleRng.hpp; ParticleFunctors.hpp FilterByProperty / SelectOutcome), the
per-port counts and plan are exact, the per-port record multisets (plain form) and sequences
(fused form) equal the stable partition of the oracle's bins, and the updaters and transforms
change exactly the fields the reference functors change."""
import ctypes as C

import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SEED, CAP, TILE = 42, 1024, 1024
PARTICLE = np.dtype([("id", "<u8"), ("property", "<u4"), ("weight", "<u4"), ("visit", "<u4"), ("pad", "<u4")])


class ParticlePool:
    """A device pool of particle records, SoA (four columns) or AoS (24-byte slots)."""

    def __init__(self, num_chunks, layout):
        self.num_chunks, self.layout = num_chunks, layout
        self.slots = num_chunks * CAP
        self.cols = capi.Columns()
        self.cols.record, self.cols.layout = capi.REC_PARTICLE, layout
        if layout == capi.LAYOUT_SOA:
            self.id = torch.zeros(self.slots, dtype=torch.int64, device="cuda")
            self.f32 = [torch.zeros(self.slots, dtype=torch.int32, device="cuda") for _ in range(3)]
            for i, t in enumerate([self.id] + self.f32):
                self.cols.column[i] = t.data_ptr()
        else:
            self.raw = torch.zeros(self.slots * 6, dtype=torch.int32, device="cuda")
            self.cols.column[0] = self.raw.data_ptr()

    def put(self, slot0, rec):
        n = len(rec)
        if self.layout == capi.LAYOUT_SOA:
            self.id[slot0:slot0 + n] = torch.from_numpy(rec["id"].view(np.int64))
            for t, f in zip(self.f32, ("property", "weight", "visit")):
                t[slot0:slot0 + n] = torch.from_numpy(rec[f].view(np.int32))
        else:
            self.raw[6 * slot0:6 * (slot0 + n)] = torch.from_numpy(rec.view(np.int32).reshape(-1))

    def get(self, slot0, n):
        out = np.zeros(n, PARTICLE)
        if self.layout == capi.LAYOUT_SOA:
            out["id"] = self.id[slot0:slot0 + n].cpu().numpy().view(np.uint64)
            for t, f in zip(self.f32, ("property", "weight", "visit")):
                out[f] = t[slot0:slot0 + n].cpu().numpy().view(np.uint32)
        else:
            out = self.raw[6 * slot0:6 * (slot0 + n)].cpu().numpy().view(PARTICLE).copy()
        return out


def _particles(n, rng):
    p = np.zeros(n, PARTICLE)
    p["id"] = rng.permutation(n).astype(np.uint64) + 1000
    p["property"] = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    p["weight"] = rng.integers(0, 5000, n).astype(np.uint32)
    p["weight"][:3] = 0xFFFFFFFF - 10  # a feedback step of these overflows
    p["visit"] = rng.integers(0, 70, n).astype(np.uint32)
    return p


def _batch(pool, parts, rng):
    """Ragged input chunks 0.. holding the particles in order; returns chunks, fills, tiles."""
    fills, left = [], len(parts)
    while left:
        f = min(int(rng.integers(1, CAP + 1)), left)
        fills.append(f)
        left -= f
    chunks = list(range(len(fills)))
    off = 0
    for c, f in zip(chunks, fills):
        pool.put(c * CAP, parts[off:off + f])
        off += f
    tiles = capi.flatten_tiles(chunks, fills, TILE)
    return chunks, fills, torch.from_numpy(tiles.view(np.int32).reshape(-1)).cuda(), len(tiles)


def _bins(parts, cls, purpose, max_visits=64):
    d = np.array([O.draw(SEED, int(i), int(v), purpose) for i, v in zip(parts["id"], parts["visit"])], np.uint64)
    if cls == capi.CLS_FEEDBACK_FILTER:
        return (d >= parts["property"]).astype(np.int64)
    return np.where(d < 0x80000000, 0, np.where(parts["visit"] < max_visits, 1, 2)).astype(np.int64)


def _params(purpose, max_visits=64, increment=1000):
    p = capi.FunctorParams()
    p.seed, p.purpose, p.max_visits, p.increment = SEED, purpose, max_visits, increment
    return p


def _records(pool, descs):
    got = [pool.get(int(c) * CAP, int(f)) for c, f, _ in descs]
    ports = np.repeat(descs[:, 2], descs[:, 1])
    return (np.concatenate(got) if got else np.zeros(0, PARTICLE)), ports


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
def test_select_and_feedback_update_plain_form(layout):
    """A/B of particle_feedback: classify (SelectOutcome), host plan, scatter with the feedback
    updater (UpdateWeight 1000); the three first particles overflow on feedback."""
    rng = np.random.default_rng(1)
    n, bins = 20_011, 3
    parts = _particles(n, rng)
    exp_bin = _bins(parts, capi.CLS_FEEDBACK_SELECT, 4)
    bound = capi.output_chunk_bound(n, CAP, bins)
    pool = ParticlePool(4 * n // CAP + bound + 64, layout)
    chunks, fills, tiles, n_tiles = _batch(pool, parts, rng)
    L = capi.lib()
    counts = torch.zeros(bins + 1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    bin_ids = torch.zeros(pool.slots, dtype=torch.int32, device="cuda")
    prm = _params(4)
    capi.check(L.gf_classify_dense(None, C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(), n_tiles, TILE, bins,
                                   capi.CLS_FEEDBACK_SELECT, C.byref(prm), bin_ids.data_ptr(), counts.data_ptr(),
                                   status.data_ptr()), "classify")
    totals = counts.cpu().numpy().view(np.uint32)
    assert int(status.item()) == 0 and totals[bins] == 0
    assert np.array_equal(totals[:bins], np.bincount(exp_bin, minlength=bins))
    base, ofills, r = capi.plan_dense(totals[:bins], CAP)
    out_chunks = np.arange(len(chunks) + 20, len(chunks) + 20 + r, dtype=np.uint32)
    table = torch.from_numpy(capi.build_dense_table(base, out_chunks).view(np.int32)).cuda()
    nxt = torch.zeros(bins, dtype=torch.int32, device="cuda")
    capi.check(L.gf_scatter(None, C.byref(pool.cols), C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(), n_tiles,
                            TILE, bins, bin_ids.data_ptr(), table.data_ptr(), nxt.data_ptr(), counts.data_ptr(),
                            capi.SCATTER_SHARED, capi.UPD_FEEDBACK, C.byref(prm), status.data_ptr()), "scatter")
    # the three overflowing feedback particles fail the batch with GF_OVERFLOW
    overflow = (exp_bin[:3] == 1).any()
    assert int(status.item()) == (capi.GF_OVERFLOW if overflow else 0)
    assert np.array_equal(nxt.cpu().numpy().view(np.uint32), totals[:bins])
    descs = np.stack([out_chunks, ofills, np.repeat(np.arange(bins), (totals[:bins] + CAP - 1) // CAP)], axis=1)
    got, ports = _records(pool, descs)
    exp = parts.copy()
    fb = (exp_bin == 1) & (exp["weight"] <= 0xFFFFFFFF - 1000)
    exp["weight"][fb] += 1000
    exp["visit"][fb] += 1
    for b in range(bins):
        g = np.sort(got[ports == b], order="id")
        e = np.sort(exp[exp_bin == b], order="id")
        assert np.array_equal(g[["id", "property", "weight", "visit"]], e[["id", "property", "weight", "visit"]])


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
def test_filter_fused_form_keeps_input_order(layout):
    """Filter of particle_feedback (FilterByProperty) through the generic fused partition: exact
    counts and plan, every port's records in input order, the outputs in reservation order."""
    rng = np.random.default_rng(2)
    n, bins = 30_007, 2
    parts = _particles(n, rng)
    exp_bin = _bins(parts, capi.CLS_FEEDBACK_FILTER, 2)
    bound = capi.output_chunk_bound(n, CAP, bins)
    pool = ParticlePool(4 * n // CAP + bound + 64, layout)
    chunks, fills, tiles, n_tiles = _batch(pool, parts, rng)
    L = capi.lib()
    reserved = torch.from_numpy(np.arange(len(chunks), len(chunks) + bound, dtype=np.uint32).view(np.int32)).cuda()
    totals = torch.zeros(bins, dtype=torch.int32, device="cuda")
    max_k = -(-n // CAP)
    port_chunks = torch.zeros(bins * max_k, dtype=torch.int64, device="cuda")
    sbytes = capi.fused_scratch_bytes(n_tiles, bins)
    scratch = torch.zeros((sbytes + 15) // 8, dtype=torch.int64, device="cuda")
    table = torch.zeros(bins + bound, dtype=torch.int32, device="cuda")
    descs = torch.zeros(3 * bound, dtype=torch.int32, device="cuda")
    num = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    prm = _params(2)
    capi.check(L.gf_partition_fused(None, C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(), n_tiles, bins,
                                    capi.CLS_FEEDBACK_FILTER, capi.UPD_NONE, C.byref(prm), reserved.data_ptr(), bound,
                                    totals.data_ptr(), port_chunks.data_ptr(), max_k, scratch.data_ptr(), sbytes,
                                    table.data_ptr(), descs.data_ptr(), bound, num.data_ptr(), status.data_ptr()),
               "fused")
    assert int(status.item()) == 0
    tot = totals.cpu().numpy().view(np.uint32)
    assert np.array_equal(tot, np.bincount(exp_bin, minlength=bins))
    base, ofills, r = capi.plan_dense(tot, CAP)
    assert int(num.item()) == r
    d = descs.cpu().numpy().view(np.uint32)[:3 * r].reshape(-1, 3)
    assert np.array_equal(d[:, 1], ofills) and np.array_equal(table.cpu().numpy().view(np.uint32)[:bins], base)
    got, ports = _records(pool, d)
    for b in range(bins):
        e = parts[exp_bin == b]
        assert np.array_equal(got[ports == b][["id", "property", "weight", "visit"]],
                              e[["id", "property", "weight", "visit"]])


def test_kernel_axis_classifier_and_bin_updater():
    """KernelAxes.hpp's balanced distribution (id % B) with the weight = bin updater, AoS."""
    rng = np.random.default_rng(3)
    n, bins = 12_345, 64
    parts = _particles(n, rng)
    pool = ParticlePool(4 * n // CAP + capi.output_chunk_bound(n, CAP, bins) + 64, capi.LAYOUT_AOS)
    chunks, fills, tiles, n_tiles = _batch(pool, parts, rng)
    L = capi.lib()
    counts = torch.zeros(bins + 1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    bin_ids = torch.zeros(pool.slots, dtype=torch.int32, device="cuda")
    prm = _params(2)
    capi.check(L.gf_classify_dense(None, C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(), n_tiles, TILE, bins,
                                   capi.CLS_ID_BALANCED, C.byref(prm), bin_ids.data_ptr(), counts.data_ptr(),
                                   status.data_ptr()), "classify")
    totals = counts.cpu().numpy().view(np.uint32)[:bins]
    exp_bin = (parts["id"] % bins).astype(np.int64)
    assert np.array_equal(totals, np.bincount(exp_bin, minlength=bins))
    base, ofills, r = capi.plan_dense(totals, CAP)
    out_chunks = np.arange(len(chunks) + 10, len(chunks) + 10 + r, dtype=np.uint32)
    table = torch.from_numpy(capi.build_dense_table(base, out_chunks).view(np.int32)).cuda()
    nxt = torch.zeros(bins, dtype=torch.int32, device="cuda")
    capi.check(L.gf_scatter(None, C.byref(pool.cols), C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(), n_tiles,
                            TILE, bins, bin_ids.data_ptr(), table.data_ptr(), nxt.data_ptr(), counts.data_ptr(),
                            capi.SCATTER_DIRECT, capi.UPD_SET_BIN, C.byref(prm), status.data_ptr()), "scatter")
    assert int(status.item()) == 0
    descs = np.stack([out_chunks, ofills, np.repeat(np.arange(bins), (totals + CAP - 1) // CAP)], axis=1)
    got, ports = _records(pool, descs)
    assert np.array_equal(got["weight"], ports.astype(np.uint32))
    assert np.array_equal(np.sort(got["id"]), np.sort(parts["id"]))
    assert np.array_equal(got["id"] % bins, ports)


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
def test_transform_dense_concatenation(layout):
    """TransformKernel semantics: input item i of tile t goes, transformed, to output position
    t.out_pos + i of the output chunk list (Execution.hpp:709-776)."""
    rng = np.random.default_rng(4)
    n = 9_001
    parts = _particles(n, rng)
    pool = ParticlePool(4 * n // CAP + 64, layout)
    chunks, fills, _, _ = _batch(pool, parts, rng)
    mt, pos = [], 0
    for c, f in zip(chunks, fills):
        for off in range(0, f, 256):
            cnt = min(256, f - off)
            mt.append((c, off, cnt, pos))
            pos += cnt
    tiles = torch.from_numpy(np.asarray(mt, np.uint32).view(np.int32).reshape(-1)).cuda()
    n_out = -(-n // CAP)
    out_chunks = np.arange(len(chunks) + 5, len(chunks) + 5 + n_out, dtype=np.uint32)
    d_out = torch.from_numpy(out_chunks.view(np.int32)).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L = capi.lib()
    inc = 20  # the three planted weights (2^32 - 11) overflow, every other weight does not
    for xf in (capi.XF_IDENTITY, capi.XF_ADD_WEIGHT):
        status.zero_()
        capi.check(L.gf_transform(None, C.byref(pool.cols), C.byref(pool.cols), CAP, pool.slots, tiles.data_ptr(),
                                  len(mt), d_out.data_ptr(), n_out, xf, C.byref(_params(0, increment=inc)),
                                  status.data_ptr()), "transform")
        got = np.concatenate([pool.get(int(c) * CAP, min(CAP, n - k * CAP)) for k, c in enumerate(out_chunks)])
        exp = parts.copy()
        if xf == capi.XF_ADD_WEIGHT:
            ok = exp["weight"] <= 0xFFFFFFFF - inc
            assert (~ok).sum() == 3
            exp["weight"][ok] += inc
            exp["visit"][ok] += 1
            assert int(status.item()) == capi.GF_OVERFLOW
            keep = ok
        else:
            assert int(status.item()) == 0
            keep = np.ones(n, bool)
        assert np.array_equal(got[keep][["id", "property", "weight", "visit"]],
                              exp[keep][["id", "property", "weight", "visit"]])


def test_unregistered_combinations_are_rejected():
    cols = capi.Columns()
    cols.record, cols.layout = capi.REC_U32, capi.LAYOUT_SOA
    buf = torch.zeros(4096, dtype=torch.int32, device="cuda")
    cols.column[0] = buf.data_ptr()
    L = capi.lib()
    prm = _params(0)
    # a record without a property field has no Filter classifier
    rc = L.gf_classify_dense(None, C.byref(cols), CAP, 4096, buf.data_ptr(), 1, TILE, 2, capi.CLS_FEEDBACK_FILTER,
                             C.byref(prm), buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert rc == capi.GF_ERR_ARGUMENT
    cols.record = 9
    rc = L.gf_classify_dense(None, C.byref(cols), CAP, 4096, buf.data_ptr(), 1, TILE, 2, capi.CLS_KEY_MOD,
                             C.byref(prm), buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert rc == capi.GF_ERR_ARGUMENT
