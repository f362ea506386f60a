"""The command-line drop-in for the reference's example binary graphFlow_particle_feedback
(examples/particle_feedback/main.cpp, Cli.hpp): flags, exit codes and the printed report.

The report format follows main.cpp:22-33 and 48-58: '# ...' lines, '# weight,count', one
'weight,count' row per distinct final weight in ascending order, and '# non-terminating K' when the
visit cap stopped K particles. The GPU tests check the rows against the oracle's scalar model
(tests/reference/ScalarModel.hpp restated) and, at the reference's published configuration, the
SHA-256 the reference published for its rows (docs/benchmarks.md:32-34).
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from graphflow_b200 import capi
from oracle import oracle as O


def _run(*args, timeout=600):
    assert os.path.exists(capi.CLI_PATH), "build the library first (graphflow_b200.capi.build())"
    return subprocess.run([capi.CLI_PATH, *args], capture_output=True, text=True, timeout=timeout)


def _rows(stdout):
    lines = stdout.splitlines()
    start = lines.index("# weight,count") + 1
    rows = [ln for ln in lines[start:] if not ln.startswith("#")]
    capped = [ln for ln in lines[start:] if ln.startswith("# non-terminating ")]
    w = np.array([int(r.split(",")[0]) for r in rows], np.uint64)
    c = np.array([int(r.split(",")[1]) for r in rows], np.uint64)
    ncap = int(capped[0].split()[-1]) if capped else 0
    return w, c, ncap, "".join(r + "\n" for r in rows)


def test_cli_help():
    r = _run("--help")
    assert r.returncode == 0 and r.stdout.startswith("usage: graphflow_b200_particle_feedback")


@pytest.mark.parametrize("args", [
    ["--bogus"],
    ["--particles"],                              # missing value
    ["--particles", "-5"],
    ["--particles", "18446744073709551616"],      # 2^64
    ["--chunk-size", "0"],
    ["--chunk-size", "4294967296"],               # 2^32
    ["--backend", "cpu", "--particles", "10"],    # this build runs on CUDA only
    ["--backend", "cuda", "--workload", "kernel", "--bin-path", "dense", "--bins", "65536"],
    ["--backend", "cuda", "--workload", "kernel", "--bin-path", "hash", "--scatter", "direct"],
    ["--backend", "cuda", "--workload", "kernel", "--bins", "100"],
    ["--backend", "cuda", "--workload", "kernel", "--distribution", "sparse"],  # sparse needs >= 1024 bins
    ["--backend", "cuda", "--bins", "64"],        # a kernel-workload flag without --workload kernel
    ["--backend", "cuda", "--pool-mode", "arena"],
    ["--backend", "cuda", "--workload", "both"],
])
def test_cli_rejects_bad_command_lines(args):
    """Configuration errors exit 2 with the message and the usage text on stderr, before any
    device work (Cli.hpp: parseOptions / resolveOptions throw std::invalid_argument)."""
    r = _run(*args)
    assert r.returncode == 2 and "usage:" in r.stderr and r.stdout == ""


def _distribution_bin(dist, ids, bins):
    """KernelAxes.hpp:29-42 distributionBin."""
    ids = ids.astype(np.uint64)
    if dist == "one-hot":
        return np.zeros(ids.size, np.uint32)
    if dist == "skewed":
        return np.where(ids % 8 == 0, ids % bins, 0).astype(np.uint32)
    return (ids % bins).astype(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("bins,dist,scatter,path", [(64, "balanced", "shared", "dense"),
                                                    (64, "skewed", "direct", "dense"),
                                                    (1024, "sparse", "shared", "dense"),
                                                    (1024, "one-hot", "direct", "dense"),
                                                    (4096, "balanced", "shared", "dense"),
                                                    (1024, "skewed", "shared", "hash"),
                                                    (65536, "balanced", "shared", "hash"),
                                                    (65536, "sparse", "shared", "hash")])
def test_kernel_workload_sends_every_particle_to_its_port(bins, dist, scatter, path):
    """runKernelAxes (KernelAxes.hpp:115-167): each particle's final weight is the port its id
    maps to, in the fused form and in the plain form with the direct (one atomic per particle) or
    the shared-staging scatter, and through the per-tile hash tables (65536 ports always)."""
    n = 300_007
    for fused in ([False] if scatter == "direct" else [True, False]):
        w, st = capi.run_kernel_axes(9, n, bins, dist, scatter, chunk_capacity=1024, live_particles=8192,
                                     batch_chunks=4, fused=fused, bin_path=path)
        assert np.array_equal(w, _distribution_bin(dist, np.arange(n), bins)) and st.sunk == n


@pytest.mark.gpu
def test_cli_kernel_workload_prints_the_port_occupancy():
    n, bins = 100_000, 1024
    r = _run("--backend", "cuda", "--workload", "kernel", "--particles", str(n), "--bins", str(bins),
             "--distribution", "skewed", "--chunk-size", "1024", "--live-particles", "8192", "--batch-chunks", "2")
    assert r.returncode == 0, r.stderr
    w, c, ncap, _ = _rows(r.stdout)
    ev, ec = np.unique(_distribution_bin("skewed", np.arange(n), bins), return_counts=True)
    assert np.array_equal(w, ev.astype(np.uint64)) and np.array_equal(c, ec.astype(np.uint64)) and ncap == 0
    assert "workload=kernel" in r.stdout.splitlines()[0] and f"bins={bins}" in r.stdout.splitlines()[0]
    h = _run("--backend", "cuda", "--workload", "kernel", "--particles", str(n), "--bins", "65536",
             "--bin-path", "hash", "--chunk-size", "1024", "--live-particles", "8192")
    assert h.returncode == 0, h.stderr
    w, c, _, _ = _rows(h.stdout)
    ev, ec = np.unique(_distribution_bin("balanced", np.arange(n), 65536), return_counts=True)
    assert np.array_equal(w, ev.astype(np.uint64)) and np.array_equal(c, ec.astype(np.uint64))


@pytest.mark.gpu
def test_cli_config1_matches_the_scalar_model():
    """Config 1 (N=1e6, seed 42, C=1024, P=4096, Q=1, 64 visits): the printed rows are the
    oracle's histogram, they sum to N, and the non-terminating count is the oracle's."""
    n = 1_000_000
    r = _run("--backend", "cuda", "--particles", str(n), "--chunk-size", "1024", "--live-particles", "4096",
             "--batch-chunks", "1", "--seed", "42", "--max-visits", "64")
    assert r.returncode == 0, r.stderr
    w, c, ncap, _ = _rows(r.stdout)
    ew, _, encap = O.particle_scalar(42, n, 64)
    erw, erc = O.histogram_u32(ew)
    assert np.array_equal(w, erw.astype(np.uint64)) and np.array_equal(c, erc.astype(np.uint64))
    assert int(c.sum()) == n and ncap == encap
    head = r.stdout.splitlines()[0]
    assert head.startswith("# graphFlow_particle_feedback backend=cuda") and f"particles={n}" in head


@pytest.mark.gpu
def test_cli_device_resident_prints_the_same_rows():
    """--device-resident (a B200 extension) runs the Flow device-resident: the rows equal the host
    runner's."""
    args = ["--backend", "cuda", "--particles", "200000", "--chunk-size", "1024", "--live-particles", "4096",
            "--batch-chunks", "1", "--seed", "42", "--max-visits", "64"]
    a, b = _run(*args), _run(*args, "--device-resident")
    assert a.returncode == 0 and b.returncode == 0, b.stderr
    assert _rows(a.stdout)[3] == _rows(b.stdout)[3] and _rows(a.stdout)[2] == _rows(b.stdout)[2]


@pytest.mark.gpu
def test_cli_inert_flags_are_noted_and_change_nothing():
    base = ["--backend", "cuda", "--particles", "20000", "--chunk-size", "1024", "--live-particles", "4096",
            "--seed", "7"]
    a = _run(*base)
    b = _run(*base, "--frame-cap", "4", "--pool-mode", "slotArena", "--tile-size", "256")
    assert a.returncode == 0 and b.returncode == 0
    assert "--frame-cap has no effect" in b.stderr and "--pool-mode has no effect" in b.stderr
    assert _rows(a.stdout)[3] == _rows(b.stdout)[3]


@pytest.mark.gpu
def test_cli_defaults_come_from_the_device_policy():
    """Without --chunk-size / --live-particles the run takes the device policy's C and P (the
    accelerator ratio 8 under the 3 GiB budget cap: C = 4096, P = 32768 on a B200), and the rows are
    the oracle's whatever C and P are."""
    n = 200_000
    r = _run("--backend", "cuda", "--particles", str(n), "--seed", "5")
    assert r.returncode == 0, r.stderr
    pol = capi.device_policy(n, live_per_chunk=8)
    head = r.stdout.splitlines()[0]
    assert f"chunk-size={pol.chunk_capacity} " in head and f"live-particles={pol.live_particles} " in head
    assert f"tile-size={pol.tile_size} " in head
    w, c, ncap, _ = _rows(r.stdout)
    ew, _, encap = O.particle_scalar(5, n, 64)
    erw, erc = O.histogram_u32(ew)
    assert np.array_equal(w, erw.astype(np.uint64)) and np.array_equal(c, erc.astype(np.uint64)) and ncap == encap


@pytest.mark.gpu
def test_cli_rejects_a_live_particle_count_above_the_run():
    r = _run("--backend", "cuda", "--particles", "1000", "--live-particles", "2000")
    assert r.returncode == 2 and "live-particle count" in r.stderr


@pytest.mark.gpu
def test_cli_published_configuration_reproduces_the_published_rows():
    """N=1e8, C=8192, P=16384, Q=8, seed 42 (docs/benchmarks.md:24-34): the rows the binary prints
    hash to the SHA-256 the reference published for its own run."""
    r = _run("--backend", "cuda", "--particles", "100000000", "--chunk-size", "8192", "--live-particles", "16384",
             "--batch-chunks", "8", "--seed", "42")
    assert r.returncode == 0, r.stderr
    w, c, _, text = _rows(r.stdout)
    assert len(w) == 260 and int(c.sum()) == 100_000_000
    assert hashlib.sha256(text.encode()).hexdigest() == (
        "21ab0aeb9ec72d380af2ce6e9631f8fa7b9111d24ff7831f272aa9f6a7be9dab")


# ---- graphflow_b200_photon_scattering (examples/photon_scattering/main.cpp, PhotonCli.hpp) ----

def _prun(*args, timeout=600):
    assert os.path.exists(capi.PHOTON_CLI_PATH), "build the library first (graphflow_b200.capi.build())"
    return subprocess.run([capi.PHOTON_CLI_PATH, *args], capture_output=True, text=True, timeout=timeout)


def _photon_report(stdout):
    """(event counts by name, {(outcome, scatter count): count}, terminal-sum, inconsistent)."""
    lines = stdout.splitlines()
    ev_at, rows_at = lines.index("# event,count"), lines.index("# outcome,scatter-count,count")
    events = {ln.split(",")[0]: int(ln.split(",")[1]) for ln in lines[ev_at + 1:rows_at]}
    rows, term, bad = {}, None, None
    for ln in lines[rows_at + 1:]:
        if ln.startswith("# terminal-sum,"):
            term = int(ln.split(",")[1])
        elif ln.startswith("# inconsistent,"):
            bad = int(ln.split(",")[1])
        elif not ln.startswith("#"):
            o, s, c = ln.split(",")
            rows[(o, int(s))] = int(c)
    return events, rows, term, bad


def test_photon_cli_help():
    r = _prun("--help")
    assert r.returncode == 0 and r.stdout.startswith("usage: graphflow_b200_photon_scattering")


@pytest.mark.parametrize("args", [
    ["--bogus"],
    ["--photons"],
    ["--mode", "sideways"],
    ["--thickness", "abc"],
    ["--backend", "cpu"],
    ["--backend", "cuda", "--thickness", "0"],
    ["--backend", "cuda", "--sigma-s", "-1"],
    ["--backend", "cuda", "--max-scatters", "70000"],            # the scatter counter is 16-bit here
    ["--backend", "cuda", "--output-dir", ""],
    ["--backend", "cuda", "--trace-vertices", "-1"],
    ["--backend", "cuda", "--pool-mode", "arena"],
    ["--backend", "cuda", "--exec", "both"],
    ["--backend", "cuda", "--device-resident"],                   # a Flow option: needs --exec flow
])
def test_photon_cli_rejects_bad_command_lines(args):
    r = _prun(*args)
    assert r.returncode == 2 and "usage:" in r.stderr and r.stdout == ""


@pytest.mark.gpu
def test_photon_cli_vacuum_transmits_every_photon_uncollided():
    """sigma-s = sigma-a = 0 (the defaults): every photon leaves through the far face with no
    scatter (the vacuum closed form of tests/integration/test_photon_scattering.cpp)."""
    n = 10_000
    r = _prun("--backend", "cuda", "--photons", str(n))
    assert r.returncode == 0, r.stderr
    events, rows, term, bad = _photon_report(r.stdout)
    assert events == {"transmitted": n, "reflected": 0, "absorbed": 0, "capped": 0}
    assert rows == {("transmitted", 0): n} and term == n and bad == 0


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["forward", "isotropic"])
def test_photon_cli_report_matches_the_library_and_both_execution_forms(mode):
    """The printed outcome rows are the (event, scatter count) histogram of the same analog FP64
    run through gf_run_photon, and --exec flow prints the same rows as --exec fused."""
    n, seed = 100_000, 42
    args = ["--backend", "cuda", "--photons", str(n), "--thickness", "1", "--sigma-s", "2", "--sigma-a", "0.5",
            "--mode", mode, "--max-scatters", "64", "--seed", str(seed)]
    fused, flow = _prun(*args), _prun(*args, "--exec", "flow", "--chunk-size", "4096", "--batch-chunks", "4")
    dev = _prun(*args, "--exec", "flow", "--chunk-size", "4096", "--device-resident")
    assert fused.returncode == 0 and flow.returncode == 0 and dev.returncode == 0, fused.stderr + flow.stderr
    ev, rows, term, bad = _photon_report(fused.stdout)
    assert _photon_report(flow.stdout) == (ev, rows, term, bad)
    assert _photon_report(dev.stdout) == (ev, rows, term, bad)
    p = capi.photon_params(model=capi.PHOTON_ANALOG, thickness=1.0, sigma_s=2.0, sigma_a=0.5, max_scatters=64,
                           isotropic=(mode == "isotropic"), fp64=True)
    got = capi.run_photon(seed, n, p, exec_mode=capi.EXEC_FUSED)
    names = {1: "transmitted", 2: "reflected", 3: "absorbed", 4: "capped"}
    expect = {}
    for e, s in zip(got["event"].tolist(), got["scatter_count"].tolist()):
        expect[(names[e], s)] = expect.get((names[e], s), 0) + 1
    assert rows == expect and term == n and bad == 0 and sum(ev.values()) == n


@pytest.mark.gpu
def test_photon_cli_writes_the_reference_run_files(tmp_path):
    """--output-dir writes metadata, outcomes, scatter histogram and exits as the reference does
    (PhotonOutput.hpp:91-197): the outcome files equal the printed report, exits.csv has one row
    per transmitted or reflected photon with a unit exit direction, cos_theta = uz, exits on the
    slab faces; without --trace-photons the trace files carry their headers only and metadata.csv
    reports the trace defaults (0 photons, 64 vertices)."""
    import csv
    import math
    n, out = 20_000, tmp_path / "run"
    r = _prun("--backend", "cuda", "--photons", str(n), "--sigma-s", "2", "--sigma-a", "0.5", "--mode", "isotropic",
              "--seed", "3", "--output-dir", str(out))
    assert r.returncode == 0, r.stderr
    ev, rows, term, bad = _photon_report(r.stdout)
    names = sorted(p.name for p in out.iterdir())
    assert names == sorted(["metadata.csv", "outcomes.csv", "scatter_histogram.csv", "exits.csv", "traces.csv",
                            "trace_summary.csv"])
    outcomes = {row["event"]: int(row["count"]) for row in csv.DictReader(open(out / "outcomes.csv"))}
    assert outcomes == ev
    hist = {(row["event"], int(row["scatter_count"])): int(row["count"])
            for row in csv.DictReader(open(out / "scatter_histogram.csv"))}
    assert hist == rows
    exits = list(csv.DictReader(open(out / "exits.csv")))
    assert len(exits) == ev["transmitted"] + ev["reflected"]
    for row in exits[:2000]:
        ux, uy, uz = float(row["ux"]), float(row["uy"]), float(row["uz"])
        assert abs(ux * ux + uy * uy + uz * uz - 1.0) < 1e-9 and float(row["cos_theta"]) == uz
        assert abs(float(row["phi_rad"]) - math.atan2(uy, ux)) < 1e-12
        z = float(row["z"])
        assert (row["event"] == "transmitted" and abs(z - 1.0) < 1e-9 and uz > 0) or \
               (row["event"] == "reflected" and abs(z) < 1e-9 and uz < 0)
    meta = {row["key"]: row["value"] for row in csv.DictReader(open(out / "metadata.csv"))}
    assert meta["photons"] == str(n) and meta["mode"] == "isotropic" and meta["count_terminated"] == str(n)
    assert open(out / "traces.csv").read() == "id,step,kind,scatter_count,x,y,z,ux,uy,uz\n"
    assert open(out / "trace_summary.csv").read() == "id,vertices,truncated\n"
    assert (meta["trace_enabled"], meta["trace_photons"], meta["trace_vertices"], meta["trace_ids"]) == \
        ("0", "0", "64", "0")
    assert "# output-dir=" in r.stdout
