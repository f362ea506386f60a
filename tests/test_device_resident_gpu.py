"""The Flow run device-resident (Tuning::deviceResident, C ABI knob device_resident): waves of whole
input lists on one stream with a device-resident chunk pool instead of the host runner's batches.

Every particle must get the result of the host runner and of the oracle (the reference's
integration tests check the same per-particle invariants: tests/integration/
test_particle_feedback.cpp:48-202, test_dense_bins.cpp), the run must end with every chunk back in
the pool, and the published N = 1e8 particle_feedback histogram must hash to the reference's
published SHA-256 (docs/benchmarks.md:32-34)."""
import contextlib
import hashlib

import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def device_resident():
    L = capi.lib()
    capi.check(L.gf_set_tuning(b"device_resident", 1), "tuning")
    try:
        yield
    finally:
        capi.check(L.gf_set_tuning(b"device_resident", 0), "tuning")


@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS, capi.LAYOUT_RECORD])
@pytest.mark.parametrize("n,c,seed", [(1_000_000, 1024, 42), (100_003, 4096, 7), (1, 1024, 3), (0, 1024, 1)])
def test_feedback_matches_oracle(layout, n, c, seed):
    with device_resident():
        w, capped, st = capi.run_particle_feedback(seed, n, 64, chunk_capacity=c, live_particles=4 * c,
                                                   batch_chunks=1, layout=layout)
    ew, ecapped, _ = O.particle_scalar(seed, n, 64)
    assert np.array_equal(w, ew)
    assert np.array_equal(capped.astype(np.uint8), ecapped)
    assert st.generated == n and st.sunk == n
    if n:
        assert st.loop_iterations > 1 and st.partition_batches > 0
        assert st.peak_live_chunks <= st.pool_chunks


@pytest.mark.parametrize("c", [1000, 3000, 2048])
def test_feedback_chunk_capacities_off_the_tile_size(c):
    """Chunk capacities that are not a multiple of the 1024-particle tile (a chunk's last tile is
    partial) and one that is."""
    n, seed = 150_001, 5
    with device_resident():
        w, capped, st = capi.run_particle_feedback(seed, n, 64, chunk_capacity=c, live_particles=4 * c,
                                                   batch_chunks=1)
    ew, ecapped, _ = O.particle_scalar(seed, n, 64)
    assert np.array_equal(w, ew) and np.array_equal(capped.astype(np.uint8), ecapped)
    assert st.sunk == n


def test_feedback_equals_host_runner():
    n, seed = 300_007, 11
    host = capi.run_particle_feedback(seed, n, 16, chunk_capacity=1024, live_particles=4096, batch_chunks=2)
    with device_resident():
        dev = capi.run_particle_feedback(seed, n, 16, chunk_capacity=1024, live_particles=4096, batch_chunks=2)
    assert np.array_equal(host[0], dev[0]) and np.array_equal(host[1], dev[1])


@pytest.mark.parametrize("nodes,bins,dist", [(1, 2, "uniform"), (4, 8, "zipf"), (2, 32, "round_robin"),
                                             (4, 64, "uniform"), (3, 64, "one_port")])
def test_dense_chain_matches_oracle(nodes, bins, dist):
    n, seed = 300_007, 42
    with device_resident():
        port_of, st = capi.run_dense_chain(seed, n, bins, nodes=nodes, dist=dist, chunk_capacity=8192)
    keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
    exp = ((keys >> np.uint32(8 * (nodes - 1))) % np.uint32(bins)).astype(np.uint32)
    assert np.array_equal(port_of, exp)
    assert st.sunk == n and st.partition_batches == nodes


@pytest.mark.parametrize("model,fp64", [(capi.PHOTON_ANALOG, True), (capi.PHOTON_WEIGHTED, False)])
def test_photon_flow_equals_fused_transport(model, fp64):
    n = 30_000
    p = capi.photon_params(model=model, sigma_s=10.0 if model else 2.0, sigma_a=0.1 if model else 0.5,
                           max_scatters=65535 if model else 64, fp64=fp64)
    with device_resident():
        a = capi.run_photon(42, n, p, capi.EXEC_FLOW, chunk_capacity=1024, live_particles=8192, batch_chunks=4)
    b = capi.run_photon(42, n, p, capi.EXEC_FUSED)
    for k in ("event", "scatter_count", "weight", "cos_exit", "position"):
        assert np.array_equal(a[k], b[k]), k
    assert a["stats"].generated == n and a["stats"].sunk == n
    # scatter -> propose flight -> advance and route run in one wave (transforms forward into the
    # same wave), so a photon takes one wave per scattering plus its first flight and its sink
    assert a["stats"].loop_iterations <= int(b["scatter_count"].max()) + 2


@pytest.mark.parametrize("bins,dist", [(64, "balanced"), (1024, "one-hot")])
def test_kernel_workload_equals_host_runner(bins, dist):
    n = 200_000
    host = capi.run_kernel_axes(3, n, bins, dist, chunk_capacity=8192, live_particles=65536, batch_chunks=8)
    with device_resident():
        dev = capi.run_kernel_axes(3, n, bins, dist, chunk_capacity=8192, live_particles=65536, batch_chunks=8)
    assert np.array_equal(host[0], dev[0])


def test_published_configuration_reproduces_the_published_histogram():
    """particle_feedback at N = 1e8, C = 8192, seed 42, run device-resident."""
    with device_resident():
        w, capped, st = capi.run_particle_feedback(42, 100_000_000, 64, chunk_capacity=8192, live_particles=16384,
                                                   batch_chunks=8)
    vals, counts = O.histogram_u32(w)
    text = "".join(f"{int(v)},{int(c)}\n" for v, c in zip(vals, counts))
    assert st.sunk == 100_000_000 and len(vals) == 260
    assert hashlib.sha256(text.encode()).hexdigest() == (
        "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab")
    print(f"device-resident particle_feedback N=1e8: {st.seconds:.3f} s, {1e8 / st.seconds:.3e} particles/s, "
          f"{st.loop_iterations} waves, {st.kernel_launches} launches, peak live {st.peak_live_chunks} of "
          f"{st.pool_chunks} chunks")


def test_kernel_workload_with_the_hash_path_runs_on_the_host_runner():
    """The device-resident mode runs the fused dense partition; the kernel workload's hash bin path
    keeps the host runner under the knob and gives the same ports."""
    n = 50_000
    host = capi.run_kernel_axes(3, n, 64, "balanced", bin_path="hash", fused=False)
    with device_resident():
        dev = capi.run_kernel_axes(3, n, 64, "balanced", bin_path="hash", fused=False)
    assert np.array_equal(host[0], dev[0]) and dev[1].partition_batches == host[1].partition_batches > 1


@pytest.mark.parametrize("n,c", [(50_001, 1024), (0, 1024)])
def test_set_transform_device_resident(n, c):
    """transform<Set<WeightTag, VisitTag>> on a Record payload, run device-resident (the transform
    is applied in place)."""
    with device_resident():
        weights, visits, st = capi.run_set_transform(7, n, 1234, chunk_capacity=c, live_particles=4 * c,
                                                     batch_chunks=1)
    assert st.sunk == n
    assert np.all(weights == 1234) and np.all(visits == 1)
    # the transform forwards into the sink's input of the same wave: one wave for the whole run
    assert st.loop_iterations == (1 if n else 0)
