"""CUDA-graph replay of the fused batch step (control-block reset, fused partition, device
finish): every replay gives the direct launch's counts, plan and per-port sequences, with the
cooperative kernel and with the per-tile look-back kernel. The launch epoch lives in device memory
and advances per replay, which is what makes a captured step reusable."""
import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from graphflow_b200.partition import ChunkPool, FusedPartition
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _setup(n, bins, capacity, tile, dist):
    n_in = -(-n // capacity)
    bound = capi.output_chunk_bound(n, capacity, bins)
    pool = ChunkPool(n_in + bound, capacity)
    keys = O.generate_keys_u32(dist, 42, n, bins, zipf_s=1.1)
    pool.column[:n].copy_(torch.from_numpy(keys.view(np.int32)))
    fills = np.full(n_in, capacity, np.uint32)
    fills[-1] = n - capacity * (n_in - 1)
    part = FusedPartition(pool, bins, tile_size=tile, max_batch_particles=n)
    tiles, d_tiles = part._tiles(np.arange(n_in, dtype=np.uint32), fills)
    part.reserved[:bound].copy_(torch.from_numpy(np.arange(n_in, n_in + bound, dtype=np.uint32).view(np.int32)))
    torch.cuda.synchronize()
    return pool, part, d_tiles, len(tiles), bound, keys


def _outputs(pool, part, bins):
    torch.cuda.synchronize()
    u = lambda t: t.cpu().numpy().view(np.uint32)  # noqa: E731
    r = int(u(part.num_out)[0])
    descs = u(part.descs)[:3 * r].reshape(-1, 3)
    col = u(pool.column)
    seqs = [[] for _ in range(bins)]
    for chunk, fill, b in descs:
        seqs[int(b)].append(col[int(chunk) * pool.capacity: int(chunk) * pool.capacity + int(fill)])
    seqs = [np.concatenate(x) if x else np.zeros(0, np.uint32) for x in seqs]
    return int(u(part.status)[0]), u(part.totals).copy(), descs[:, 1:].copy(), seqs


@pytest.mark.parametrize("coop", [1, 0])
@pytest.mark.parametrize("bins,dist", [(64, "uniform"), (8, "zipf")])
def test_graph_replay_equals_direct_launch(coop, bins, dist):
    capi.check(capi.lib().gf_set_tuning(b"fused_coop", coop), "tuning")
    try:
        n = 2_000_003
        pool, part, d_tiles, n_tiles, bound, keys = _setup(n, bins, 8192, 4096, dist)
        part.enqueue(d_tiles, n_tiles, bound)
        direct = _outputs(pool, part, bins)
        graph = part.capture(d_tiles, n_tiles, bound)
        for _ in range(4):
            pool.column[bound * 0 + (-(-n // 8192)) * 8192:].zero_()  # wipe the output chunks
            graph.replay()
            got = _outputs(pool, part, bins)
            assert got[0] == 0 and np.array_equal(got[1], direct[1]) and np.array_equal(got[2], direct[2])
            for a, b in zip(got[3], direct[3]):
                assert np.array_equal(a, b)
        counts, order = O.partition_stable_u32(keys, bins)
        assert np.array_equal(direct[1], counts)
        start = 0
        for b in range(bins):
            assert np.array_equal(direct[3][b], keys[order[start:start + counts[b]]])
            start += counts[b]
    finally:
        capi.check(capi.lib().gf_set_tuning(b"fused_coop", 1), "tuning")
