"""Named-attribute payloads (graphFlow::Record, flow/Attributes.hpp) through the Flow.

particle_feedback written the way the reference's example is (a Record of id, property, weight
and visit with one device column per attribute, functors reading particle[tag], the stream fields
from a StreamTraits specialisation) must give every particle the result of the struct-payload graph
and of the oracle's scalar model (tests/reference/ScalarModel.hpp). A transform restricted to
Set<WeightTag, VisitTag> (flow/Flow.hpp:235-242) changes exactly those attributes."""
import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("q", [1, 4])
def test_record_payload_matches_struct_payload(fused, q):
    n, seed = 100_003, 42
    kw = dict(chunk_capacity=1024, live_particles=4096, batch_chunks=q, fused=fused)
    wr, cr, sr = capi.run_particle_feedback(seed, n, layout=capi.LAYOUT_RECORD, **kw)
    ws, cs, ss = capi.run_particle_feedback(seed, n, layout=capi.LAYOUT_SOA, **kw)
    assert np.array_equal(wr, ws) and np.array_equal(cr, cs)
    assert sr.sunk == n and sr.generated == n


def test_record_payload_matches_scalar_model_at_config1():
    n, seed, max_visits = 1_000_000, 42, 64
    w, capped, st = capi.run_particle_feedback(seed, n, max_visits, chunk_capacity=1024, live_particles=4096,
                                               batch_chunks=1, layout=capi.LAYOUT_RECORD)
    ew, ecapped, _ = O.particle_scalar(seed, n, max_visits)
    assert np.array_equal(w, ew)
    assert np.array_equal(capped.astype(bool), ecapped.astype(bool))
    vals, counts = O.histogram_u32(w)
    assert int(counts.sum()) == n


@pytest.mark.parametrize("n,c,q", [(50_001, 1024, 1), (200_000, 4096, 3), (1, 1024, 1), (0, 1024, 1)])
def test_set_transform_changes_only_its_attributes(n, c, q):
    weights, visits, st = capi.run_set_transform(7, n, 1234, chunk_capacity=c, live_particles=4 * c,
                                                 batch_chunks=q)
    assert st.sunk == n
    assert np.all(weights == 1234) and np.all(visits == 1)
