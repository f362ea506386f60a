"""Bounded photon path traces (examples/photon_scattering/PhotonFunctors.hpp:201-234 TraceWriter,
recorded at :255 source, :364-369 every scatter and :401-406 the terminal event;
PhotonScattering.hpp:49-82, 158-174; PhotonOutput.hpp:131-146 the trace files).

Properties every trace has, checked on the oracle and on the GPU:
  * vertex 0 is the source at the origin heading +z with no scatter; vertices 1..k are the k
    scatters with scatter counts 1..k; the last is the terminal event (kind = event + 1) with the
    terminal record's scatter count, position and direction;
  * a photon keeps min(k + 2, V) vertices and is truncated exactly when k + 2 > V;
  * consecutive vertices lie on straight flights: vertex j+1 is on the ray from vertex j along
    vertex j's outgoing direction;
  * tracing does not change any history.
Tolerances: as the analog FP64 parity (>= 99.9 % of traced ids with the oracle's event and
scatter count, positions and directions within 1e-9 absolute where they agree); the Flow and the
fused kernel, and traced and untraced runs, are bit-identical.
"""
import csv
import ctypes as C

import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O

SLAB = dict(thickness=1.0, sigma_s=2.0, sigma_a=0.5)


def _check_trace(v, count, truncated, term_event, term_sc, term_pos, term_dir, V, thickness, exact=True):
    """One id's trace against its terminal record and the straight-flight rule."""
    k = int(term_sc)
    assert int(count) == min(k + 2, V)
    assert int(truncated) == int(k + 2 > V)
    rows = v[:int(count)]
    if len(rows) == 0:
        return
    assert rows[0]["kind"] == 0 and rows[0]["scatter_count"] == 0
    assert (rows[0]["x"], rows[0]["y"], rows[0]["z"], rows[0]["ux"], rows[0]["uy"], rows[0]["uz"]) == (0, 0, 0, 0, 0, 1)
    inner = rows[1:min(len(rows), k + 1)]
    assert np.all(inner["kind"] == 1)
    assert np.array_equal(inner["scatter_count"], np.arange(1, len(inner) + 1))
    if len(rows) == k + 2:
        last = rows[-1]
        assert last["kind"] == term_event + 1 and last["scatter_count"] == k
        pos = np.array([last["x"], last["y"], last["z"]])
        dirn = np.array([last["ux"], last["uy"], last["uz"]])
        if exact:
            assert np.array_equal(pos, term_pos) and np.array_equal(dirn, term_dir)
        else:
            assert np.allclose(pos, term_pos, atol=1e-9, rtol=0) and np.allclose(dirn, term_dir, atol=1e-9, rtol=0)
    p = np.stack([rows["x"], rows["y"], rows["z"]], axis=1)
    u = np.stack([rows["ux"], rows["uy"], rows["uz"]], axis=1)
    assert np.all(p[:, 2] >= -1e-12) and np.all(p[:, 2] <= thickness + 1e-12)
    assert np.allclose((u * u).sum(axis=1), 1.0, atol=1e-12)
    step = p[1:] - p[:-1]
    along = (step * u[:-1]).sum(axis=1)
    assert np.all(along >= -1e-12)
    assert np.allclose(step, along[:, None] * u[:-1], atol=1e-9, rtol=0)


# ---- oracle (CPU) ---------------------------------------------------------------------------

@pytest.mark.parametrize("isotropic", [True, False])
def test_oracle_trace_follows_its_own_histories(isotropic):
    n, M, V = 5_000, 400, 5
    exp = O.photon_analog(7, n, SLAB["thickness"], SLAB["sigma_s"], SLAB["sigma_a"], isotropic, 64)
    term, v, counts, trunc = O.photon_analog_traced(7, n, SLAB["thickness"], SLAB["sigma_s"], SLAB["sigma_a"],
                                                    isotropic, 64, M, V)
    assert np.array_equal(term, exp)  # tracing leaves the histories alone
    assert v.shape == (M, V) and trunc.any() and not trunc.all()
    for i in range(M):
        t = term[i]
        _check_trace(v[i], counts[i], trunc[i], int(t["event"]), t["scatter_count"],
                     np.array([t["x"], t["y"], t["z"]]), np.array([t["ux"], t["uy"], t["uz"]]), V, 1.0)


def test_oracle_trace_bounds():
    # M above N traces every id; V = 0 keeps no vertex and truncates every traced id
    term, v, counts, trunc = O.photon_analog_traced(1, 50, 1.0, 2.0, 0.5, True, 64, 1000, 4)
    assert counts.shape == (50,) and np.all(counts == np.minimum(term["scatter_count"] + 2, 4))
    term, v, counts, trunc = O.photon_analog_traced(1, 50, 1.0, 2.0, 0.5, True, 64, 10, 0)
    assert np.all(counts == 0) and np.all(trunc == 1)
    # vacuum: source and the far face
    term, v, counts, trunc = O.photon_analog_traced(1, 10, 2.0, 0.0, 0.0, False, 64, 10, 4)
    assert np.all(counts == 2) and np.all(v[:, 1]["kind"] == 2) and np.all(v[:, 1]["z"] == 2.0)


def test_traced_entry_rejects_an_offset_first_id():
    """A trace selects ids < M of a run that starts at id 0 (checked before any device work)."""
    p = capi.photon_params(model=capi.PHOTON_ANALOG, thickness=1.0, sigma_s=2.0, sigma_a=0.5, fp64=True)
    rc = capi.lib().gf_run_photon_traced(0, 5, 10, C.byref(p), capi.EXEC_FUSED, 0, 0, 1, *([None] * 9), None, 4, 8,
                                         None, None, None)
    assert rc == capi.GF_ERR_ARGUMENT


# ---- GPU ------------------------------------------------------------------------------------

def _params(isotropic, fp64=True, model=None):
    return capi.photon_params(model=capi.PHOTON_ANALOG if model is None else model, isotropic=isotropic,
                              max_scatters=64, fp64=fp64, **SLAB)


@pytest.mark.gpu
@pytest.mark.parametrize("isotropic", [True, False])
@pytest.mark.parametrize("exec_mode", ["fused", "flow"])
def test_gpu_trace_matches_the_oracle(isotropic, exec_mode):
    n, M, V = 20_000, 2_000, 6
    ex = capi.EXEC_FUSED if exec_mode == "fused" else capi.EXEC_FLOW
    got = capi.run_photon(42, n, _params(isotropic), ex, chunk_capacity=4096 if ex == capi.EXEC_FLOW else 8192,
                          batch_chunks=4, trace_photons=M, trace_vertices=V)
    term, v, counts, trunc = O.photon_analog_traced(42, n, SLAB["thickness"], SLAB["sigma_s"], SLAB["sigma_a"],
                                                    isotropic, 64, M, V)
    gv, gc, gt = got["trace_vertices"], got["trace_counts"], got["trace_truncated"]
    assert gv.shape == (M, V) and gt.any() and not gt.all()
    term = term[:M]
    same = (got["event"][:M] == term["event"]) & (got["scatter_count"][:M] == term["scatter_count"])
    assert same.mean() >= 0.999
    for i in np.nonzero(same)[0][:M]:
        _check_trace(gv[i], gc[i], gt[i], int(got["event"][i]), got["scatter_count"][i], got["position"][i],
                     got["direction"][i], V, 1.0)
        assert gc[i] == counts[i] and gt[i] == trunc[i]
        a, b = gv[i][:gc[i]], v[i][:counts[i]]
        assert np.array_equal(a["kind"], b["kind"]) and np.array_equal(a["scatter_count"], b["scatter_count"])
        for f in ("x", "y", "z", "ux", "uy", "uz"):
            assert np.allclose(a[f], b[f], atol=1e-9, rtol=0), (i, f)


@pytest.mark.gpu
def test_gpu_trace_is_identical_in_both_forms_and_leaves_histories_unchanged():
    n, M, V = 30_000, 1_000, 32
    p = _params(True)
    plain = capi.run_photon(5, n, p, capi.EXEC_FUSED)
    fused = capi.run_photon(5, n, p, capi.EXEC_FUSED, trace_photons=M, trace_vertices=V)
    flow = capi.run_photon(5, n, p, capi.EXEC_FLOW, chunk_capacity=4096, batch_chunks=4, trace_photons=M,
                           trace_vertices=V)
    for k in ("event", "scatter_count", "position", "direction"):
        assert np.array_equal(plain[k], fused[k]) and np.array_equal(plain[k], flow[k]), k
    for k in ("trace_vertices", "trace_counts", "trace_truncated"):
        assert np.array_equal(fused[k], flow[k]), k


@pytest.mark.gpu
def test_gpu_trace_bounds_and_weighted_model():
    p = _params(True)
    got = capi.run_photon(3, 100, p, capi.EXEC_FUSED, trace_photons=1_000, trace_vertices=0)
    assert got["trace_counts"].shape == (100,) and np.all(got["trace_counts"] == 0)
    assert np.all(got["trace_truncated"] == 1)
    # the weighted FP32 model traces its Henyey-Greenstein scatters the same way
    w = capi.photon_params(model=capi.PHOTON_WEIGHTED, thickness=1.0, sigma_s=10.0, sigma_a=0.1, g=0.9,
                           max_scatters=65535, fp64=False)
    V = 4096
    got = capi.run_photon(9, 2_000, w, capi.EXEC_FUSED, trace_photons=200, trace_vertices=V)
    for i in range(200):
        c, k = int(got["trace_counts"][i]), int(got["scatter_count"][i])
        assert c == min(k + 2, V) and int(got["trace_truncated"][i]) == int(k + 2 > V)
        rows = got["trace_vertices"][i][:c]
        inner = rows[1:min(c, k + 1)]
        assert rows[0]["kind"] == 0 and np.all(inner["kind"] == 1)
        assert np.array_equal(inner["scatter_count"], np.arange(1, len(inner) + 1))
        if c == k + 2:
            assert rows[-1]["kind"] == got["event"][i] + 1
            assert np.array_equal(np.array([rows[-1]["x"], rows[-1]["y"], rows[-1]["z"]]), got["position"][i])


@pytest.mark.gpu
def test_photon_cli_writes_the_path_traces(tmp_path):
    """--trace-photons / --trace-vertices: traces.csv and trace_summary.csv hold the library's
    trace of the same run (17 significant digits round-trip a double), and metadata.csv reports
    the trace settings (PhotonOutput.hpp:131-146, 187-191)."""
    import subprocess
    n, M, V, out = 20_000, 300, 8, tmp_path / "run"
    r = subprocess.run([capi.PHOTON_CLI_PATH, "--backend", "cuda", "--photons", str(n), "--sigma-s", "2",
                        "--sigma-a", "0.5", "--mode", "isotropic", "--seed", "11", "--trace-photons", str(M),
                        "--trace-vertices", str(V), "--output-dir", str(out)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    got = capi.run_photon(11, n, _params(True), capi.EXEC_FUSED, trace_photons=M, trace_vertices=V)
    summary = list(csv.DictReader(open(out / "trace_summary.csv")))
    assert [int(s["id"]) for s in summary] == list(range(M))
    assert [int(s["vertices"]) for s in summary] == got["trace_counts"].tolist()
    assert [int(s["truncated"]) for s in summary] == got["trace_truncated"].tolist()
    rows = list(csv.DictReader(open(out / "traces.csv")))
    assert len(rows) == int(got["trace_counts"].sum())
    at = 0
    for i in range(M):
        for step in range(int(got["trace_counts"][i])):
            row, v = rows[at], got["trace_vertices"][i][step]
            at += 1
            assert int(row["id"]) == i and int(row["step"]) == step
            assert row["kind"] == capi.TRACE_KIND_NAMES[v["kind"]] and int(row["scatter_count"]) == v["scatter_count"]
            assert all(float(row[f]) == v[f] for f in ("x", "y", "z", "ux", "uy", "uz"))
    meta = {row["key"]: row["value"] for row in csv.DictReader(open(out / "metadata.csv"))}
    assert meta["trace_enabled"] == "1" and meta["trace_photons"] == str(M) and meta["trace_vertices"] == str(V)
    assert meta["trace_ids"] == str(M) and meta["trace_truncated_ids"] == str(int(got["trace_truncated"].sum()))
