"""The benchmark's multi-process plumbing on CPU: one process per rank as torchrun starts them
(RANK / WORLD_SIZE / MASTER_* from the environment, rendezvous on 127.0.0.1), a barrier, the max
over ranks of the step time, and the whole-job value. gloo stands in for NCCL; the GPU path uses
the same code with the nccl backend. Also the reference arm under a 2-rank launch: rank 0 prints
one line, the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    r = bench.Ranks("gloo", device=None, timeout_s=60)
    r.barrier()
    local_ms = 1.5 * (rank + 1)          # a slower rank sets the step time
    ms = r.max(local_ms)
    value = bench.whole_job_value(100_000_000, r.world, ms)
    r.barrier()
    r.close()
    out.put((rank, ms, value))


@pytest.mark.parametrize("world", [2, 3])
def test_max_over_ranks_and_whole_job_value(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = 1.5 * world
    for rank, ms, value in got:
        assert ms == pytest.approx(slowest)
        assert value == pytest.approx(world * 100_000_000 / (slowest / 1e3))


def test_single_process_needs_no_process_group():
    import bench
    r = bench.Ranks("gloo")
    assert r.world == 1 and r.max(2.5) == 2.5
    r.barrier()
    r.close()


def _reference_arm(rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "300000",
                           "--steps", "2", "--warmup", "1", "--gpus", str(world)], env=env, cwd=ROOT,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_rank0_prints_one_line_other_ranks_exit_quietly():
    p0 = _reference_arm(0, 2)
    assert p0.returncode == 0, p0.stderr
    lines = [l for l in p0.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    p1 = _reference_arm(1, 2)
    assert p1.returncode == 0 and p1.stdout.strip() == ""
