"""The host scheduler's failure paths on the CPU (no GPU touched): tests/cpp/runner_failures.cpp
runs graphflow::BasicGraphRunner with fake stages and a fake queue, the way the reference's
tests/integration/test_failure_paths.cpp drives its GraphRunner with a CPU device. Covered: stall
detection (SchedulerStallError after the stall timeout, per-node detail to the stall callback
only), a throwing launch, a throwing advance, lease-acquisition and event-enqueue failures
injected at the reference's FailurePoints, an unroutable output; every case must leave the chunk
ledger whole (each chunk released once, no lease left)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def runner_binary(tmp_path_factory):
    out = tmp_path_factory.mktemp("runner") / "runner_failures"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "graphflow_b200", "include", "graphflow"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "runner_failures.cpp"),
           os.path.join(ROOT, "graphflow_b200", "csrc", "gf_host.cpp"), "-o", str(out)]
    subprocess.run(cmd, check=True)
    return str(out)


def test_runner_failure_paths(runner_binary):
    r = subprocess.run([runner_binary], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
    assert r.stdout.count("\nok ") + r.stdout.startswith("ok ") >= 13
