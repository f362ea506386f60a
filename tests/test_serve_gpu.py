"""The request server (gf_serve): whole-flow requests of different sizes and topologies served one
at a time through the Flow (plain form) or with continuous batching (each admitted request's flow
on the device on its own stream, admitted while others run). A request's result must be the same
alone and in the mix, and in both forms: each result is reduced to an order-independent digest of
its per-particle outcome, checked here also against the per-particle outputs of the standalone
entry points."""
import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix64(v):
    v = v.astype(np.uint64)
    with np.errstate(over="ignore"):
        v ^= v >> np.uint64(30)
        v *= np.uint64(0xBF58476D1CE4E5B9)
        v ^= v >> np.uint64(27)
        v *= np.uint64(0x94D049BB133111EB)
        v ^= v >> np.uint64(31)
    return v


def _digest_feedback(weights, capped):
    ids = np.arange(len(weights), dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (ids * GOLDEN) ^ ((capped.astype(np.uint64) != 0).astype(np.uint64) << np.uint64(32) |
                              weights.astype(np.uint64))
    return int(_mix64(x).sum(dtype=np.uint64))


def _digest_port(port):
    ids = np.arange(len(port), dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (ids * GOLDEN) ^ (port.astype(np.uint64) << np.uint64(40))
    return int(_mix64(x).sum(dtype=np.uint64))


def _stream(count=18, seed=5, n_max=30_000):
    return capi.make_requests(count, seed=seed, n_min=1_000, n_max=n_max, rate_per_s=None, photon_scale=10)


def test_each_result_is_the_same_alone_in_the_mix_and_in_both_forms():
    req = _stream()
    mixed, st = capi.serve(req, capi.SERVE_BATCHED, max_inflight=8)
    plain, _ = capi.serve(req, capi.SERVE_PLAIN)
    flowdev, _ = capi.serve(req, capi.SERVE_FLOW_DEVICE)
    assert np.all(mixed["status"] == 0) and np.all(plain["status"] == 0) and np.all(flowdev["status"] == 0)
    assert np.array_equal(mixed["digest"], plain["digest"]) and np.array_equal(flowdev["digest"], plain["digest"])
    for i in range(len(req)):
        alone, _ = capi.serve(req[i:i + 1], capi.SERVE_BATCHED, max_inflight=1)
        assert alone["digest"][0] == mixed["digest"][i], f"request {i}"
    assert st.peak_inflight > 1  # requests overlapped on the device


def test_digests_match_the_standalone_entry_points():
    req = _stream(count=9, seed=11)
    res, _ = capi.serve(req, capi.SERVE_BATCHED, max_inflight=4)
    for r, out in zip(req, res):
        n = int(r["n"])
        if r["kind"] == capi.REQ_PARTICLE_FEEDBACK:
            w, c, _ = capi.run_particle_feedback_kernel(int(r["seed"]), n, 64)
            ew, ec, _ = O.particle_scalar(int(r["seed"]), n, 64)
            assert np.array_equal(w, ew)
            assert out["digest"] == _digest_feedback(w, c)
        elif r["kind"] == capi.REQ_DENSE_CHAIN:
            port, _ = capi.run_dense_chain(int(r["seed"]), n, int(r["bins"]), nodes=2, dist="uniform")
            assert out["digest"] == _digest_port(port)


def test_admission_respects_the_memory_cap():
    req = _stream(count=6, seed=3, n_max=20_000)
    big = capi.make_requests(1, seed=9)
    big["kind"] = capi.REQ_DENSE_CHAIN
    big["bins"] = 8
    big["n"] = 5_000_000  # two pool columns of 1847 chunks x 8192 slots: ~121 MB
    mix = np.concatenate([req, big])
    res, st = capi.serve(mix, capi.SERVE_BATCHED, memory_cap_bytes=64 << 20, max_inflight=4)
    assert np.all(res["status"][:-1] == 0)
    assert res["status"][-1] == capi.GF_ERR_RANGE  # larger than the cap: refused, never started
    assert st.peak_bytes <= 64 << 20


def test_arrivals_and_latencies_are_ordered():
    req = capi.make_requests(12, seed=21, n_min=1_000, n_max=20_000, rate_per_s=2_000.0, photon_scale=10)
    res, _ = capi.serve(req, capi.SERVE_BATCHED, max_inflight=4)
    assert np.all(res["admit_s"] >= req["arrival_s"] - 1e-6)
    assert np.all(res["done_s"] >= res["admit_s"])


def test_reused_device_memory_carries_no_state_between_requests():
    """Requests served one after another in the same device memory (one slot) give the digests
    they give alone: nothing a finished request left behind leaks into the next one."""
    req = capi.make_requests(40, seed=7, n_min=1_000, n_max=20_000, photon_scale=10)
    req["kind"] = capi.REQ_DENSE_CHAIN
    req["bins"] = np.resize(np.array([32, 2, 8], np.uint32), len(req))
    seq, _ = capi.serve(req, capi.SERVE_BATCHED, max_inflight=1)
    assert np.all(seq["status"] == 0)
    for i in (0, 13, 27, 39):
        alone, _ = capi.serve(req[i:i + 1], capi.SERVE_BATCHED, max_inflight=1)
        assert alone["digest"][0] == seq["digest"][i]
