"""Partition groups: the fused partition nodes of one classifier type run as one runner node whose
launches drain every member's ready batches (batches of at most Q chunks per node, the reference's
per-node batches of sched/GraphRunner.hpp:985-1133) in one multi-batch kernel. Results must be the
ones the per-node runner gives, particle for particle, and the oracle's at full size."""
import time

import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _expect(n, bins, nodes, dist, seed):
    keys = O.generate_keys_u32(dist, seed, n, bins, zipf_s=1.1)
    return ((keys >> np.uint32(8 * (nodes - 1))) % np.uint32(bins)).astype(np.uint32)


def _chain(grouped, *args, **kw):
    L = capi.lib()
    capi.check(L.gf_set_tuning(b"group_partitions", int(grouped)), "tuning")
    try:
        return capi.run_dense_chain(*args, **kw)
    finally:
        capi.check(L.gf_set_tuning(b"group_partitions", 1), "tuning")


@pytest.mark.parametrize("nodes", [2, 3, 4])
@pytest.mark.parametrize("bins,dist,layout", [(8, "uniform", capi.LAYOUT_SOA), (64, "zipf", capi.LAYOUT_AOS),
                                              (32, "round_robin", capi.LAYOUT_SOA)])
def test_group_matches_per_node_runner(nodes, bins, dist, layout):
    n, seed = 200_003, 11
    kw = dict(nodes=nodes, dist=dist, chunk_capacity=2048, live_particles=8192, batch_chunks=4, layout=layout)
    grouped, gs = _chain(True, seed, n, bins, **kw)
    single, ss = _chain(False, seed, n, bins, **kw)
    assert np.array_equal(grouped, single)
    assert np.array_equal(grouped, _expect(n, bins, nodes, dist, seed))
    assert gs.sunk == n and ss.sunk == n
    # the per-node runner launches once per batch; the group drains several batches per launch
    assert ss.partition_launches == ss.partition_batches
    assert gs.partition_launches < gs.partition_batches


def test_group_feedback_graph_identical():
    """particle_feedback's processes A and B share classifier and updater types: grouped, their
    batches share launches; the weight histogram and capped flags do not change."""
    L = capi.lib()
    out = []
    for grouped in (1, 0):
        capi.check(L.gf_set_tuning(b"group_partitions", grouped), "tuning")
        try:
            out.append(capi.run_particle_feedback(42, 100_000, chunk_capacity=1024, live_particles=4096,
                                                  batch_chunks=2))
        finally:
            capi.check(L.gf_set_tuning(b"group_partitions", 1), "tuning")
    (wg, cg, sg), (ws, cs, ss) = out
    assert np.array_equal(wg, ws) and np.array_equal(cg, cs)
    assert sg.partition_launches < sg.partition_batches


def test_group_chain_full_size_matches_oracle():
    """The 4-node chain of the dense sweep at its stated size (N = 1e8, B = 64 uniform, C = 8192,
    P = 16384, Q = 8): every particle's final port equals the oracle's, and the per-port counts
    with it."""
    n, seed, bins = 100_000_000, 42, 64
    t0 = time.perf_counter()
    port_of, st = capi.run_dense_chain(seed, n, bins, nodes=4, dist="uniform", chunk_capacity=8192,
                                       live_particles=16384, batch_chunks=8)
    seconds = time.perf_counter() - t0
    exp = _expect(n, bins, 4, "uniform", seed)
    assert st.generated == n and st.sunk == n
    assert np.array_equal(np.bincount(port_of, minlength=bins), np.bincount(exp, minlength=bins))
    assert np.array_equal(port_of, exp)
    assert st.partition_launches < st.partition_batches
    print(f"4-node chain N=1e8: {seconds:.2f} s, {n / seconds:.3e} particles/s, "
          f"{st.partition_batches} batches in {st.partition_launches} partition launches")
