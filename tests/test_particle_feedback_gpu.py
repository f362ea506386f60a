"""particle_feedback through the C++ front end (Flow + GraphRunner + typed stages) on the GPU,
against the oracle's scalar model.

Mirrors tests/integration/test_particle_feedback.cpp:48-202 and :273-349 of the reference:
element-wise final weights, the sorted histogram, rows summing to N, the capped count, and no
particle left at the 0xDEADBEEF sentinel, across N, C, P, Q and seeds, plus the dense-path
variants (plain two-launch vs fused, SoA vs AoS storage).
"""
import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _check(seed, n, max_visits, **kw):
    w, capped, stats = capi.run_particle_feedback(seed, n, max_visits, **kw)
    ew, ecapped, encap = O.particle_scalar(seed, n, max_visits)
    assert not np.any(w == 0xDEADBEEF), "a particle never reached a sink"
    assert np.array_equal(w, ew)
    assert np.array_equal(capped.astype(np.uint8), ecapped)
    rows_w, rows_c = O.histogram_u32(w)
    erows_w, erows_c = O.histogram_u32(ew)
    assert np.array_equal(rows_w, erows_w) and np.array_equal(rows_c, erows_c)
    assert int(rows_c.sum()) == n
    assert stats.generated == n and stats.sunk == n
    return stats


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
@pytest.mark.parametrize("q", [1, 2, 8])
def test_feedback_matches_scalar_model(fused, layout, q):
    _check(42, 30_000, 64, chunk_capacity=1024, live_particles=4096, batch_chunks=q, fused=fused, layout=layout)


@pytest.mark.parametrize("n,c,p,seed", [(1, 1024, 4096, 42), (17, 128, 512, 7), (4097, 128, 1024, 3),
                                        (50_000, 8192, 16384, 42), (20_000, 64, 64, 11)])
def test_feedback_sizes_and_seeds(n, c, p, seed):
    _check(seed, n, 64, chunk_capacity=c, live_particles=p, batch_chunks=2)


def test_feedback_max_visits_zero():
    # tests/integration/test_particle_feedback.cpp:281-321: with maxVisits 0 every survivor is capped
    _check(5, 5_000, 0, chunk_capacity=256, live_particles=1024, batch_chunks=1)


def test_feedback_empty_run():
    w, capped, stats = capi.run_particle_feedback(42, 0, 64)
    assert w.size == 0 and stats.generated == 0


def test_feedback_config1_full():
    # particle_feedback, N=1e6, seed 42, C=1024, P=4096, Q=1, maxVisits 64
    stats = _check(42, 1_000_000, 64, chunk_capacity=1024, live_particles=4096, batch_chunks=1)
    assert stats.pool_chunks == 4096 + 8  # S = P + sum_nodes outputChunkBound(C, C, B): 2 + 3 + 3


def test_feedback_invalid_configuration_is_reported():
    """Configuration errors come back as GF_ERR_ARGUMENT before any device work (Config.hpp:233-349):
    Q = 0, and a pool of 2^32 or more slots."""
    for kw in (dict(batch_chunks=0), dict(chunk_capacity=1 << 20, live_particles=1 << 13)):
        with pytest.raises(capi.GfError) as e:
            capi.run_particle_feedback(42, 100_000, 64, **kw)
        assert e.value.code == capi.GF_ERR_ARGUMENT, kw


def test_feedback_default_chunk_and_live_counts_come_from_the_device_policy():
    """chunk_capacity = 0 and live_particles = 0 take the device policy's C and P (Flow's ratio 8);
    the results do not depend on them."""
    _check(11, 300_000, 64, chunk_capacity=0, live_particles=0, batch_chunks=4)


@pytest.mark.parametrize("n,seed,max_visits", [(1, 42, 64), (300_007, 42, 64), (100_000, 9, 0), (50_000, 3, 5)])
def test_per_particle_kernel_matches_flow_and_oracle(n, seed, max_visits):
    """The graph as one per-particle kernel gives the Flow run's weights and capped flags id for id."""
    w, capped, stats = capi.run_particle_feedback_kernel(seed, n, max_visits)
    ew, ecapped, _ = O.particle_scalar(seed, n, max_visits)
    assert np.array_equal(w, ew)
    assert np.array_equal(capped.astype(np.uint8), ecapped)
    fw, fcapped, _ = capi.run_particle_feedback(seed, n, max_visits, chunk_capacity=1024, live_particles=8192,
                                                batch_chunks=4)
    assert np.array_equal(w, fw) and np.array_equal(capped, fcapped)
    assert stats.sunk == n


def test_per_particle_kernel_reproduces_the_published_1e8_histogram():
    """N=1e8, seed 42, 64 visits on the GPU: the sorted weight,count rows hash to the SHA-256 the
    reference published for its own benchmark run (docs/benchmarks.md:32-34)."""
    import hashlib
    w, capped, stats = capi.run_particle_feedback_kernel(42, 100_000_000, 64)
    vals, counts = O.histogram_u32(w)
    text = "".join(f"{int(v)},{int(c)}\n" for v, c in zip(vals, counts))
    assert len(vals) == 260 and int(counts.sum()) == 100_000_000
    assert hashlib.sha256(text.encode()).hexdigest() == (
        "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab")


def test_flow_at_the_published_configuration_reproduces_the_published_histogram():
    """The whole Flow (runner, partition kernels, functors) at the reference's published
    configuration, N=1e8, C=8192, P=16384, Q=8, seed 42 (docs/benchmarks.md:24-34): the sorted
    weight,count rows hash to the published SHA-256."""
    import hashlib
    w, capped, stats = capi.run_particle_feedback(42, 100_000_000, 64, chunk_capacity=8192, live_particles=16384,
                                                  batch_chunks=8)
    vals, counts = O.histogram_u32(w)
    text = "".join(f"{int(v)},{int(c)}\n" for v, c in zip(vals, counts))
    assert stats.sunk == 100_000_000 and len(vals) == 260
    assert hashlib.sha256(text.encode()).hexdigest() == (
        "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab")
