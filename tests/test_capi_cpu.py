"""CPU-side checks of the C ABI: the library loads, exports every symbol the public header
declares, and its host planning entry points agree with the oracle (no device work here)."""
import ctypes as C
import os

import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = capi.declared_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(L, name), name


@pytest.mark.parametrize("n,c,b", [(0, 128, 2), (1, 1, 2), (17, 127, 2), (128, 128, 2), (4097, 128, 2),
                                   (4097, 1, 2), (64, 128, 64), (1, 128, 64), (10**8, 8192, 64),
                                   (2**32 + 5, 8192, 2**20)])
def test_output_chunk_bound_matches_oracle(n, c, b):
    assert capi.output_chunk_bound(n, c, b) == O.output_chunk_bound(n, c, b)


def test_bound_errors():
    with pytest.raises(capi.GfError):
        capi.output_chunk_bound(4, 0, 2)
    with pytest.raises(capi.GfError):
        capi.output_chunk_bound(2**64 - 1, 1, 2)
    with pytest.raises(capi.GfError):
        capi.checked_output_chunk_bound(2**32 + 9, 1, 1)


def test_plan_matches_oracle_randomised():
    rng = np.random.default_rng(0)
    for _ in range(200):
        bins = int(rng.integers(1, 70))
        cap = int(rng.integers(1, 300))
        totals = rng.integers(0, 2000, bins).astype(np.uint32)
        a = capi.plan_dense(totals, cap)
        b = O.plan_dense(totals, cap)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_dense_table_layout():
    base, fills, r = capi.plan_dense([3, 0, 2], 2)
    assert capi.build_dense_table(base, [10, 11, 12]).tolist() == [0, 2, 2, 10, 11, 12]


def test_flatten_matches_oracle():
    rng = np.random.default_rng(1)
    for ts in (1024, 4096, 128):
        fills = rng.integers(0, 9000, 50).astype(np.uint32)
        chunks = rng.permutation(1000)[:50].astype(np.uint32)
        assert np.array_equal(capi.flatten_tiles(chunks, fills, ts), O.flatten_tiles(chunks, fills, ts))
    assert capi.tile_count(0, 128) == 0 and capi.tile_count(129, 128) == 2


def test_zipf_table_matches_oracle():
    for s, k in ((1.1, 64), (0.8, 1024), (1.2, 65536)):
        assert np.array_equal(capi.zipf_cdf(s, k), O.zipf_cdf(s, k))


def test_argument_errors_are_reported_not_thrown():
    L = capi.lib()
    assert L.gf_classify_dense_u32(None, None, 0, 0, None, 0, 1024, 4, 0, None, None, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_classify_dense_u32(None, None, 16, 0, None, 0, 1000, 4, 0, None, None, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_scatter_dense_u32(None, None, None, 16, 0, None, 0, 1024, 4, None, None, None, None, 7,
                                  None) == capi.GF_ERR_ARGUMENT
    # zero tiles is a valid empty batch: nothing is launched
    cnt = (C.c_uint32 * 5)()
    assert L.gf_classify_dense_u32(None, None, 16, 0, None, 0, 1024, 4, 0, None, C.addressof(cnt), None) == capi.GF_OK
    assert L.gf_partition_fused_u32(None, None, None, 16, 0, None, 0, 1024, 4, 0, None, 0, None, None, 0, None, 0,
                                    None) == capi.GF_ERR_ARGUMENT


def test_tuning_knobs():
    """Host-side knobs: names and ranges are checked; sink_batch_chunks takes 1..256."""
    L = capi.lib()
    assert L.gf_set_tuning(None, 1) == capi.GF_ERR_ARGUMENT
    assert L.gf_set_tuning(b"no_such_knob", 1) == capi.GF_ERR_ARGUMENT
    for bad in (0, 257, -1):
        assert L.gf_set_tuning(b"sink_batch_chunks", bad) == capi.GF_ERR_ARGUMENT
    try:
        for good in (1, 8, 256):
            assert L.gf_set_tuning(b"sink_batch_chunks", good) == capi.GF_OK
    finally:
        assert L.gf_set_tuning(b"sink_batch_chunks", 256) == capi.GF_OK
    for knob, default in ((b"device_resident", 0), (b"device_coop", 1), (b"fused_coop_bulk", 1)):
        assert L.gf_set_tuning(knob, 1 - default) == capi.GF_OK
        assert L.gf_set_tuning(knob, default) == capi.GF_OK


def test_device_pool_host_checks():
    """Device-resident pool: size formula (64-byte header, an id and a ledger word per chunk) and
    argument errors reported before any launch."""
    L = capi.lib()
    assert capi.device_pool_bytes(0) == 64 and capi.device_pool_bytes(1000) == 64 + 8 * 1000
    assert L.gf_device_pool_bytes(4, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_init(None, None, 4) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_init(None, 8, 4) == capi.GF_ERR_ARGUMENT          # not 16-byte aligned
    assert L.gf_device_pool_acquire(None, None, 1, None, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_acquire(None, 16, 1, None, None) == capi.GF_ERR_ARGUMENT  # k ids, no output
    assert L.gf_device_pool_settle(None, 16, None, 2, None, 0, None, 1, None, 0, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_settle(None, 16, None, 0, None, 0, None, 0, None, 0, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_settle(None, 16, None, 0, None, 0, None, 1, None, 3, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_device_pool_read(None, None, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_run_dense_chain_device(1, 10, 5, 1, 0, 1.1, None, None, None, None) == capi.GF_ERR_ARGUMENT
    assert L.gf_run_dense_chain_device(1, 10, 8, 5, 0, 1.1, None, None, None, None) == capi.GF_ERR_ARGUMENT


def test_every_documented_knob_is_accepted():
    """Each tuning knob the public header documents is a name gf_set_tuning accepts (set to its
    documented default here; spin_limit writes a device variable and is left to the GPU tests)."""
    import re
    header = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                               "graphflow_b200.h")).read()
    section = header[header.index("Process-wide tuning knobs"):header.index("gf_status gf_set_tuning")]
    knobs = re.findall(r'\*\s+"([a-z_]+)"\s+([0-9.]+)?', section)
    assert len(knobs) >= 9
    L = capi.lib()
    for name, default in knobs:
        if name == "spin_limit":
            continue
        m = re.search(r'"%s"\s+\S*\s*\(default (\d+)\)' % name, section) or \
            re.search(r'"%s"\s+(\d+)\s+\(default\)' % name, section)
        assert m, name
        assert L.gf_set_tuning(name.encode(), int(m.group(1))) == capi.GF_OK, name

