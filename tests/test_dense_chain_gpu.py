"""The kernel-level dense sweep through the public Flow (gf_run_dense_chain): 1 and 4 chained
partition nodes between a key source and a sink, as the reference's Flow runs any partition graph
(flow/Flow.hpp:49-754, sched/GraphRunner.hpp). Every particle must reach the sink exactly once, in
the port its key selects at the last node, and the per-port counts are bit-exact against the
oracle's keys (tests/integration/test_dense_bins.cpp and test_batching.cpp check the same
invariants on the reference's own graphs)."""
import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _expect(n, bins, nodes, dist, seed):
    keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
    return ((keys >> np.uint32(8 * (nodes - 1))) % np.uint32(bins)).astype(np.uint32)


@pytest.mark.parametrize("nodes", [1, 4])
@pytest.mark.parametrize("bins,dist", [(2, "uniform"), (8, "zipf"), (32, "round_robin"), (64, "uniform"),
                                       (64, "one_port")])
def test_chain_ports_match_oracle(nodes, bins, dist):
    n, seed = 300_007, 42
    port_of, stats = capi.run_dense_chain(seed, n, bins, nodes=nodes, dist=dist, chunk_capacity=8192,
                                          live_particles=16384, batch_chunks=8)
    exp = _expect(n, bins, nodes, dist, seed)
    assert np.array_equal(port_of, exp)
    assert np.array_equal(np.bincount(port_of, minlength=bins), np.bincount(exp, minlength=bins))
    assert stats.generated == n and stats.sunk == n


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("layout", [capi.LAYOUT_SOA, capi.LAYOUT_AOS])
def test_chain_forms_and_layouts_agree(fused, layout):
    n, seed, bins, nodes = 123_457, 7, 8, 4
    port_of, stats = capi.run_dense_chain(seed, n, bins, nodes=nodes, dist="uniform", chunk_capacity=1024,
                                          live_particles=4096, batch_chunks=2, fused=fused, layout=layout)
    assert np.array_equal(port_of, _expect(n, bins, nodes, "uniform", seed))
    assert stats.sunk == n
    assert stats.partition_batches > 0


def test_chain_empty_and_argument_errors():
    port_of, stats = capi.run_dense_chain(1, 0, 8, nodes=2)
    assert len(port_of) == 0 and stats.sunk == 0
    with pytest.raises(capi.GfError):
        capi.run_dense_chain(1, 10, 5)          # port counts of the sweep only
    with pytest.raises(capi.GfError):
        capi.run_dense_chain(1, 10, 8, nodes=5)  # at most 4 chained nodes


def test_runner_options_give_identical_results():
    """The B200 runner options (sinks of up to sink_batch_chunks chunks, every idle node dispatched
    per iteration) and the reference runner's one-chunk sinks / one dispatch per iteration give the
    same results."""
    n, seed = 200_003, 3
    out = {}
    L = capi.lib()
    try:
        for on, sink in ((1, 256), (1, 8), (1, 1), (0, 256)):
            capi.check(L.gf_set_tuning(b"runner_batched", on), "tuning")
            capi.check(L.gf_set_tuning(b"sink_batch_chunks", sink), "tuning")
            ports, _ = capi.run_dense_chain(seed, n, 32, nodes=3, chunk_capacity=1024, live_particles=8192,
                                            batch_chunks=4)
            weights, capped, _ = capi.run_particle_feedback(seed, 50_000, chunk_capacity=1024, live_particles=4096,
                                                            batch_chunks=4)
            out[(on, sink)] = (ports, weights, capped)
    finally:
        capi.check(L.gf_set_tuning(b"runner_batched", 1), "tuning")
        capi.check(L.gf_set_tuning(b"sink_batch_chunks", 256), "tuning")
    first = out[(1, 256)]
    for key, res in out.items():
        for a, b in zip(first, res):
            assert np.array_equal(a, b), key
    assert np.array_equal(first[0], _expect(n, 32, 3, "uniform", seed))
