"""Device histogram (gf_histogram_u32): the sorted (value, count) rows of a u32 column, the GPU form
of examples/particle_feedback/ParticleTypes.hpp:206-219 histogramOf (sort + run-length encoding),
bit-exact against the oracle's histogram and numpy, including the reference's published N=1e8
particle_feedback rows (docs/benchmarks.md:32-34)."""
import hashlib

import numpy as np
import pytest
import torch

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(v):
    return torch.from_numpy(np.ascontiguousarray(v, np.uint32).view(np.int32)).cuda()


@pytest.mark.parametrize("case", ["full_range", "narrow", "all_equal", "one_digit", "top_bits", "single",
                                  "empty", "two_values", "ragged_chunks"])
def test_histogram_matches_numpy(case):
    rng = np.random.default_rng(hash(case) % 2**32)
    n = {"single": 1, "empty": 0, "ragged_chunks": 8192 * 7 + 4095}.get(case, 1_000_003)
    if case == "full_range":
        v = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    elif case == "narrow":
        v = rng.integers(1000, 1300, n).astype(np.uint32)
    elif case == "all_equal":
        v = np.full(n, 0xDEADBEEF, np.uint32)
    elif case == "one_digit":
        v = rng.integers(0, 64, n).astype(np.uint32)
    elif case == "top_bits":
        v = (rng.integers(0, 4, n).astype(np.uint32) << np.uint32(30)) | np.uint32(5)
    elif case == "two_values":
        v = np.where(rng.random(n) < 0.5, 7, 4_000_000_000).astype(np.uint32)
    else:
        v = rng.integers(0, 2**20, n).astype(np.uint32)
    got_v, got_c = capi.histogram_u32(_dev(v))
    exp_v, exp_c = np.unique(v, return_counts=True)
    assert np.array_equal(got_v, exp_v)
    assert np.array_equal(got_c, exp_c.astype(np.uint64))


def test_histogram_of_feedback_weights_reproduces_the_published_1e8_rows():
    w, _, _ = capi.run_particle_feedback_kernel(42, 100_000_000, 64)
    vals, counts = capi.histogram_u32(_dev(w))
    ev, ec = O.histogram_u32(w)
    assert np.array_equal(vals, ev) and np.array_equal(counts, ec.astype(np.uint64))
    text = "".join(f"{int(a)},{int(b)}\n" for a, b in zip(vals, counts))
    assert hashlib.sha256(text.encode()).hexdigest() == (
        "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab")


def test_histogram_repeated_calls_share_nothing():
    rng = np.random.default_rng(1)
    for n in (300_000, 70_000, 1_000_000):
        v = rng.integers(0, 5000, n).astype(np.uint32)
        got_v, got_c = capi.histogram_u32(_dev(v))
        exp_v, exp_c = np.unique(v, return_counts=True)
        assert np.array_equal(got_v, exp_v) and np.array_equal(got_c, exp_c.astype(np.uint64))
