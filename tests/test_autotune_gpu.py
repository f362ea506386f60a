"""The autotuner (graphflow_b200.autotune): every candidate is measured on the GPU and the tuner
returns the fastest valid one; the tuned settings give the same results as any other (the
partition is exact whatever the shape)."""
import numpy as np
import pytest

from graphflow_b200 import autotune, capi

pytestmark = pytest.mark.gpu


def test_fused_partition_tuner_picks_the_fastest_valid_candidate():
    best, table = autotune.tune_fused_partition(600_000, 64, tiles=(1024, 4096, 8192), reps=3)
    valid = [t for t in table if t["status"] == 0]
    assert len(table) == 6 and len(valid) == 6
    assert best["ms"] == min(t["ms"] for t in valid)
    assert {t["kernel"] for t in table} == {"cooperative", "per_tile"}
    again, _ = autotune.tune_fused_partition(600_000, 64, tiles=(1024, 4096, 8192), reps=3)
    assert again is best  # cached per key


def test_chain_tuner_and_tuned_results_match():
    best, table = autotune.tune_chain(8, 2, sample_n=100_000, capacities=(1024, 4096), batch_chunks=(2, 8), reps=1)
    assert len(table) == 4 and best["seconds"] == min(t["seconds"] for t in table)
    a, _ = capi.run_dense_chain(3, 50_000, 8, nodes=2, chunk_capacity=best["capacity"],
                                batch_chunks=best["batch_chunks"], live_particles=16384)
    b, _ = capi.run_dense_chain(3, 50_000, 8, nodes=2, chunk_capacity=1024, batch_chunks=1, live_particles=4096)
    assert np.array_equal(a, b)


def test_hash_tuner():
    best, table = autotune.tune_hash(300_000, 1024, capacities=(1024, 4096), tiles=(1024, 2048), reps=2)
    timed = [t for t in table if "ms" in t]
    assert len(timed) == 4 and best["ms"] == min(t["ms"] for t in timed if t["status"] == 0)
