"""ctypes binding of the graphflow_b200 C ABI (include/graphflow_b200.h).

The shared library is built in-tree (graphflow_b200/_build/libgraphflow_b200.so). Importing a
kernel entry point without it raises immediately: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libgraphflow_b200.so")
# command-line drop-in for the reference's graphFlow_particle_feedback binary (built with the library)
CLI_PATH = os.path.join(_HERE, "_build", "graphflow_b200_particle_feedback")
PHOTON_CLI_PATH = os.path.join(_HERE, "_build", "graphflow_b200_photon_scattering")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "graphflow_b200.h")

GF_OK, GF_INVALID, GF_OVERFLOW, GF_ERR_ARGUMENT, GF_ERR_RANGE, GF_ERR_LOGIC, GF_ERR_CUDA, GF_ERR_TIMEOUT, \
    GF_ERR_TABLE_FULL = range(9)
STATUS_NAMES = {0: "ok", 1: "invalid", 2: "overflow", 3: "invalid argument", 4: "range overflow", 5: "logic error",
                6: "cuda error", 7: "timeout", 8: "hash table full"}

CLS_KEY_MOD, CLS_ID_BALANCED, CLS_ID_ONEHOT, CLS_ID_SKEWED, CLS_KEY_UNMIX = range(5)
SCATTER_SHARED, SCATTER_DIRECT = 0, 1
DIST_UNIFORM, DIST_ZIPF, DIST_ONE_PORT, DIST_ROUND_ROBIN = range(4)
DIST_NAMES = {"uniform": DIST_UNIFORM, "zipf": DIST_ZIPF, "one_port": DIST_ONE_PORT, "round_robin": DIST_ROUND_ROBIN}


class GfError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: {STATUS_NAMES.get(code, code)}")
        self.code = code


class Tile(C.Structure):
    _fields_ = [("chunk_index", C.c_uint32), ("tile_offset", C.c_uint32), ("count", C.c_uint32)]


class DeviceProps(C.Structure):
    """gf_device_props: the device fields the C/P/T policy reads."""
    _fields_ = [("sms", C.c_uint32), ("warp_size", C.c_uint32), ("max_threads_per_block", C.c_uint32),
                ("max_blocks_per_grid", C.c_uint32), ("shared_mem_per_block", C.c_uint32),
                ("global_mem_bytes", C.c_uint64)]


class Policy(C.Structure):
    """gf_policy: C, P, T and the payload budget chosen by gf_device_policy."""
    _fields_ = [("chunk_capacity", C.c_uint32), ("live_particles", C.c_uint32), ("tile_size", C.c_uint32),
                ("live_explicit", C.c_uint32), ("budget_bytes", C.c_uint64)]


class OutDesc(C.Structure):
    _fields_ = [("chunk_index", C.c_uint32), ("fill", C.c_uint32), ("bin", C.c_uint32)]


def build(force: bool = False) -> str:
    """Compile the library with its Makefile (nvcc, sm_100a)."""
    cmd = ["make", "-s", "-C", _HERE]
    if force:
        subprocess.run(cmd + ["clean"], check=True)
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None

_VP, _U32, _U64, _I32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
_SIGS = {
    "gf_output_chunk_bound": [_U64, _U64, _U64, C.POINTER(_U64)],
    "gf_checked_output_chunk_bound": [_U64, _U64, _U64, C.POINTER(_U32)],
    "gf_plan_dense": [_VP, _U32, _U32, _VP, _VP, _U32, C.POINTER(_U32)],
    "gf_build_dense_table": [_VP, _U32, _VP, _U32, _VP],
    "gf_tile_count": [_U32, _U32, C.POINTER(_U32)],
    "gf_flatten_tiles": [_VP, _VP, _U32, _U32, _VP, _U32, C.POINTER(_U32)],
    "gf_classify_dense_u32": [_VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _I32, _VP, _VP, _VP],
    "gf_scatter_dense_u32": [_VP, _VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _VP, _VP, _VP, _VP, _I32, _VP],
    "gf_fused_scratch_bytes": [_U32, _U32, C.POINTER(_U64)],
    "gf_partition_fused_u32": [_VP, _VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _I32, _VP, _U32, _VP, _VP, _U32,
                               _VP, _U64, _VP],
    "gf_fused_finish": [_VP, _VP, _VP, _U32, _U32, _U32, _VP, _VP, _VP, _U32, _VP, _VP],
    "gf_partition_fused_full_u32": [_VP, _VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _I32, _VP, _U32, _VP, _VP,
                                    _U32, _VP, _U64, _VP, _VP, _U32, _VP, _VP],
    "gf_zipf_cdf": [C.c_double, _U32, _VP],
    "gf_generate_keys_u32": [_VP, _I32, _U64, _U64, _U64, _U32, _VP, _VP],
    "gf_classify_hash_r16": [_VP, _VP, _I32, _U32, _U64, _VP, _U32, _U32, _U32, _U64, _VP, _VP, _VP],
    "gf_scatter_hash_r16": [_VP, _VP, _VP, _I32, _U32, _U64, _VP, _U32, _U32, _U32, _U64, _VP, _VP, _VP, _VP, _VP],
    "gf_plan_device": [_VP, _VP, _U32, _U32, _VP, _U32, _VP, _VP, _U32, _VP, _VP, _VP],
    "gf_generate_records16": [_VP, _U64, _U64, _U64, _VP, _U32, _U64, _VP, _I32],
    "gf_run_particle_feedback": [_U64, _U64, _U32, _U32, _U32, _U32, _I32, _I32, _VP, _VP, _VP],
    "gf_set_tuning": [C.c_char_p, _I32],
    "gf_run_kernel_axes": [_U64, _U64, _U32, _I32, _I32, _I32, _U32, _U32, _U32, _I32, _VP, _VP],
    "gf_device_policy": [_VP, _U64, _U32, _U32, _U32, _U32, _U64, _U64, _VP],
    "gf_run_particle_feedback_kernel": [_U64, _U64, _U32, _VP, _VP, _VP],
    "gf_run_set_transform": [_U64, _U64, _U32, _U32, _U32, _U32, _VP, _VP, _VP],
    "gf_serve": [_VP, _U32, _I32, _U64, _U32, _VP, _VP],
    "gf_histogram_scratch_bytes": [_U64, _VP],
    "gf_histogram_u32": [_VP, _VP, _U64, _VP, _U64, _VP, _VP, _VP, _VP],
    "gf_run_dense_chain": [_U64, _U64, _U32, _U32, _I32, C.c_double, _U32, _U32, _U32, _I32, _I32, _VP, _VP],
    "gf_run_dense_chain_device": [_U64, _U64, _U32, _U32, _I32, C.c_double, _VP, _VP, _VP, _VP],
    "gf_device_pool_bytes": [_U32, C.POINTER(_U64)],
    "gf_device_pool_init": [_VP, _VP, _U32],
    "gf_device_pool_acquire": [_VP, _VP, _U32, _VP, _VP],
    "gf_device_pool_settle": [_VP, _VP, _VP, _U32, _VP, _U32, _VP, _U32, _VP, _U32, _VP],
    "gf_device_pool_read": [_VP, _VP, _VP],
    "gf_run_photon": [_U64, _U64, _U64, _VP, _I32, _U32, _U32, _U32, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                      _VP],
    "gf_run_photon_traced": [_U64, _U64, _U64, _VP, _I32, _U32, _U32, _U32, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                             _VP, _VP, _VP, _U32, _U32, _VP, _VP, _VP],
    "gf_classify_dense": [_VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _I32, _VP, _VP, _VP, _VP],
    "gf_scatter": [_VP, _VP, _VP, _U32, _U64, _VP, _U32, _U32, _U32, _VP, _VP, _VP, _VP, _I32, _I32, _VP, _VP],
    "gf_transform": [_VP, _VP, _VP, _U32, _U64, _VP, _U32, _VP, _U32, _I32, _VP, _VP],
    "gf_partition_fused": [_VP, _VP, _U32, _U64, _VP, _U32, _U32, _I32, _I32, _VP, _VP, _U32, _VP, _VP, _U32, _VP,
                           _U64, _VP, _VP, _U32, _VP, _VP],
}

# generic ABI (gf_generic.cu): record types, classifiers, updaters, transforms
REC_U32, REC_KEYREC, REC_PARTICLE, REC_R16 = 0, 1, 2, 3
CLS_FEEDBACK_FILTER, CLS_FEEDBACK_SELECT = 16, 17
UPD_NONE, UPD_SET_BIN, UPD_FEEDBACK = 0, 1, 2
XF_IDENTITY, XF_ADD_WEIGHT = 0, 1


class Columns(C.Structure):
    """gf_columns: a registered record type, its layout and device column pointers."""
    _fields_ = [("record", C.c_int32), ("layout", C.c_int32), ("column", C.c_void_p * 4)]


class FunctorParams(C.Structure):
    """gf_functor_params: seed, stream purpose and the registered functors' constants."""
    _fields_ = [("seed", C.c_uint64), ("purpose", C.c_uint32), ("max_visits", C.c_uint32),
                ("increment", C.c_uint32), ("pad", C.c_uint32)]

LAYOUT_SOA, LAYOUT_AOS = 0, 1
LAYOUT_RECORD = 2  # gf_run_particle_feedback only: the graph over a Record payload


class FlowStats(C.Structure):
    """gf_flow_stats (SchedulerStats subset)."""
    _fields_ = [("completed_batches", C.c_uint64), ("partition_batches", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("loop_iterations", C.c_uint64), ("generated", C.c_uint64),
                ("sunk", C.c_uint64), ("pool_chunks", C.c_uint32), ("peak_live_chunks", C.c_uint32),
                ("peak_reserved_chunks", C.c_uint32), ("peak_ready_chunks", C.c_uint32), ("seconds", C.c_double),
                ("setup_seconds", C.c_double), ("loop_seconds", C.c_double), ("partition_launches", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PHOTON_ANALOG, PHOTON_WEIGHTED = 0, 1
EXEC_FLOW, EXEC_FUSED = 0, 1


class PhotonParams(C.Structure):
    """gf_photon_params."""
    _fields_ = [("thickness", C.c_double), ("sigma_s", C.c_double), ("sigma_a", C.c_double), ("g", C.c_double),
                ("roulette_threshold", C.c_double), ("roulette_survival", C.c_double),
                ("max_scatters", C.c_uint32), ("hist_bins", C.c_uint32), ("model", C.c_int), ("isotropic", C.c_int),
                ("fp64", C.c_int)]


def photon_params(model=PHOTON_WEIGHTED, thickness=1.0, sigma_s=10.0, sigma_a=0.1, g=0.9, roulette_threshold=1e-4,
                  roulette_survival=0.1, max_scatters=65535, hist_bins=256, isotropic=True, fp64=False):
    return PhotonParams(thickness, sigma_s, sigma_a, g, roulette_threshold, roulette_survival, max_scatters, hist_bins,
                        model, int(isotropic), int(fp64))


TRACE_VERTEX_DTYPE = [("kind", "<u4"), ("scatter_count", "<u4"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                      ("ux", "<f8"), ("uy", "<f8"), ("uz", "<f8")]  # gf_trace_vertex, 56 bytes
TRACE_KIND_NAMES = ("source", "scatter", "transmitted", "reflected", "absorbed", "capped")


def run_photon(seed, n, params, exec_mode=EXEC_FUSED, first_id=0, chunk_capacity=8192, live_particles=0,
               batch_chunks=8, records=True, trace_photons=0, trace_vertices=64):
    """photon_scattering transform bodies on the GPU. Returns a dict of numpy arrays.

    trace_photons > 0 also records the bounded path trace of ids < min(n, trace_photons)
    (gf_run_photon_traced): out["trace_vertices"] (M, trace_vertices) TRACE_VERTEX_DTYPE,
    out["trace_counts"] (M,) and out["trace_truncated"] (M,)."""
    import numpy as np
    m = max(n, 1)
    out = {}
    if records:
        out["event"] = np.zeros(m, np.uint32)
        out["scatter_count"] = np.zeros(m, np.uint32)
        out["weight"] = np.zeros(m, np.float64)
        out["cos_exit"] = np.zeros(m, np.float64)
        out["position"] = np.zeros(3 * m, np.float64)
        out["direction"] = np.zeros(3 * m, np.float64)
    hb = max(params.hist_bins, 1)
    out["refl"] = np.zeros(hb, np.float64)
    out["trans"] = np.zeros(hb, np.float64)
    out["event_counts"] = np.zeros(5, np.uint64)
    stats = FlowStats()
    ptr = (lambda k: out[k].ctypes.data) if records else (lambda k: None)
    args = (seed, first_id, n, C.byref(params), exec_mode, chunk_capacity, live_particles, batch_chunks, ptr("event"),
            ptr("scatter_count"), ptr("weight"), ptr("cos_exit"), ptr("position"), ptr("direction"),
            out["refl"].ctypes.data, out["trans"].ctypes.data, out["event_counts"].ctypes.data, C.byref(stats))
    if trace_photons:
        ids = min(n, trace_photons)
        out["trace_vertices"] = np.zeros((max(ids, 1), max(trace_vertices, 1)), TRACE_VERTEX_DTYPE)
        out["trace_counts"] = np.zeros(max(ids, 1), np.uint32)
        out["trace_truncated"] = np.zeros(max(ids, 1), np.uint32)
        rc = lib().gf_run_photon_traced(*args, trace_photons, trace_vertices, out["trace_vertices"].ctypes.data,
                                        out["trace_counts"].ctypes.data, out["trace_truncated"].ctypes.data)
        out["trace_vertices"] = out["trace_vertices"][:ids, :trace_vertices]
        out["trace_counts"] = out["trace_counts"][:ids]
        out["trace_truncated"] = out["trace_truncated"][:ids]
    else:
        rc = lib().gf_run_photon(*args)
    if rc != GF_OK:
        raise GfError(rc, "photon: " + last_error())
    if records:
        for k in ("event", "scatter_count", "weight", "cos_exit"):
            out[k] = out[k][:n]
        out["position"] = out["position"][:3 * n].reshape(-1, 3)
        out["direction"] = out["direction"][:3 * n].reshape(-1, 3)
    out["stats"] = stats
    return out


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().gf_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def run_particle_feedback(seed, n, max_visits=64, chunk_capacity=1024, live_particles=4096, batch_chunks=1,
                          fused=True, layout=None):
    """runParticleFeedback through the C++ front end on the GPU. Returns (weights, capped, stats)."""
    import numpy as np
    layout = LAYOUT_SOA if layout is None else layout
    weights = np.zeros(max(n, 1), np.uint32)
    capped = np.zeros(max(n, 1), np.uint32)
    stats = FlowStats()
    rc = lib().gf_run_particle_feedback(seed, n, max_visits, chunk_capacity, live_particles, batch_chunks,
                                        int(bool(fused)), layout, weights.ctypes.data, capped.ctypes.data,
                                        C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "particle feedback: " + last_error())
    return weights[:n], capped[:n], stats


KDIST_NAMES = {"balanced": 0, "one-hot": 1, "skewed": 2, "sparse": 3}


def run_kernel_axes(seed, n, bins, distribution="balanced", scatter="shared", chunk_capacity=1024,
                    live_particles=4096, batch_chunks=1, fused=True, bin_path="dense"):
    """runKernelAxes through the C++ front end: each particle's port (its final weight) and the stats."""
    import numpy as np
    weights = np.zeros(max(n, 1), np.uint32)
    stats = FlowStats()
    rc = lib().gf_run_kernel_axes(seed, n, bins, KDIST_NAMES[distribution],
                                  SCATTER_DIRECT if scatter == "direct" else SCATTER_SHARED, int(bin_path == "hash"),
                                  chunk_capacity,
                                  live_particles, batch_chunks, int(bool(fused)), weights.ctypes.data,
                                  C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "kernel axes: " + last_error())
    return weights[:n], stats


def run_set_transform(seed, n, increment, chunk_capacity=1024, live_particles=4096, batch_chunks=1):
    """Generate -> transform<Set<WeightTag, VisitTag>> -> sink over a Record payload. Returns
    (weights, visits, stats)."""
    import numpy as np
    weights = np.zeros(max(n, 1), np.uint32)
    visits = np.zeros(max(n, 1), np.uint32)
    stats = FlowStats()
    rc = lib().gf_run_set_transform(seed, n, increment, chunk_capacity, live_particles, batch_chunks,
                                    weights.ctypes.data, visits.ctypes.data, C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "set transform: " + last_error())
    return weights[:n], visits[:n], stats


def run_particle_feedback_kernel(seed, n, max_visits=64):
    """The feedback graph as one per-particle kernel. Returns (weights, capped, stats)."""
    import numpy as np
    weights = np.zeros(max(n, 1), np.uint32)
    capped = np.zeros(max(n, 1), np.uint32)
    stats = FlowStats()
    rc = lib().gf_run_particle_feedback_kernel(seed, n, max_visits, weights.ctypes.data, capped.ctypes.data,
                                               C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "particle feedback kernel: " + last_error())
    return weights[:n], capped[:n], stats


def histogram_u32(values, stream=None):
    """Device histogram of a u32 CUDA tensor (int32 storage): sorted (values, counts) numpy arrays."""
    import numpy as np
    import torch
    n = int(values.numel())
    dev = values.device
    need = C.c_uint64()
    check(lib().gf_histogram_scratch_bytes(n, C.byref(need)), "histogram scratch")
    scratch = torch.empty((need.value + 255) // 8 + 32, dtype=torch.int64, device=dev)
    base = (scratch.data_ptr() + 255) & ~255
    rows_v = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    rows_c = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    num = torch.zeros(1, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().gf_histogram_u32(s, values.data_ptr() if n else None, n, base, need.value, rows_v.data_ptr(),
                                 rows_c.data_ptr(), num.data_ptr(), status.data_ptr()), "histogram")
    torch.cuda.synchronize()
    if int(status.item()) != 0:
        raise GfError(int(status.item()), "histogram: device status")
    r = int(num.item())
    return rows_v[:r].cpu().numpy().view(np.uint32), rows_c[:r].cpu().numpy().astype(np.uint64)


# ---- request server ----
REQ_PARTICLE_FEEDBACK, REQ_PHOTON, REQ_DENSE_CHAIN = 0, 1, 2
SERVE_PLAIN, SERVE_BATCHED, SERVE_FLOW_DEVICE = 0, 1, 2
REQUEST_DTYPE = None
RESULT_DTYPE = None


def _serve_dtypes():
    import numpy as np
    global REQUEST_DTYPE, RESULT_DTYPE
    if REQUEST_DTYPE is None:
        REQUEST_DTYPE = np.dtype([("kind", "<u4"), ("bins", "<u4"), ("n", "<u8"), ("seed", "<u8"),
                                  ("arrival_s", "<f8")])
        RESULT_DTYPE = np.dtype([("admit_s", "<f8"), ("done_s", "<f8"), ("digest", "<u8"), ("status", "<u4"),
                                 ("pad", "<u4")])
    return REQUEST_DTYPE, RESULT_DTYPE


class ServeStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("peak_bytes", C.c_uint64), ("peak_inflight", C.c_uint32),
                ("pad", C.c_uint32)]


def make_requests(count, seed=1, n_min=1_000, n_max=10_000_000, rate_per_s=None, photon_scale=100,
                  chain_bins=(2, 8, 32)):
    """A mixed request stream: Poisson arrivals at rate_per_s (all at t=0 if None), N log-uniform in
    [n_min, n_max], topology uniform over particle_feedback / photon (N / photon_scale photons) /
    dense chain (bins uniform over chain_bins), and a seed per request."""
    import numpy as np
    req_t, _ = _serve_dtypes()
    rng = np.random.default_rng(seed)
    r = np.zeros(count, req_t)
    r["kind"] = rng.integers(0, 3, count)
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(np.uint64)
    n = np.where(r["kind"] == REQ_PHOTON, np.maximum(n // photon_scale, 1), n)
    r["n"] = n
    r["bins"] = np.where(r["kind"] == REQ_DENSE_CHAIN, rng.choice(np.asarray(chain_bins), count), 0)
    r["seed"] = rng.integers(1, 2**62, count, dtype=np.uint64)
    r["arrival_s"] = 0.0 if rate_per_s is None else np.cumsum(rng.exponential(1.0 / rate_per_s, count))
    return r


def serve(requests, mode=SERVE_BATCHED, memory_cap_bytes=40 << 30, max_inflight=32):
    """Serves a request array (make_requests' dtype). Returns (results array, ServeStats)."""
    import numpy as np
    req_t, res_t = _serve_dtypes()
    req = np.ascontiguousarray(requests, dtype=req_t)
    res = np.zeros(max(len(req), 1), res_t)
    stats = ServeStats()
    rc = lib().gf_serve(req.ctypes.data if len(req) else None, len(req), mode, memory_cap_bytes, max_inflight,
                        res.ctypes.data, C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "serve: " + last_error())
    return res[:len(req)], stats


def run_dense_chain(seed, n, bins, nodes=1, dist="uniform", zipf_s=1.1, chunk_capacity=8192, live_particles=16384,
                    batch_chunks=8, fused=True, layout=None, want_ports=True):
    """The dense sweep through the C++ Flow (1 to 4 chained partition nodes). Returns
    (port_of, stats): each particle's final port by id (None unless want_ports)."""
    import numpy as np
    layout = LAYOUT_SOA if layout is None else layout
    port_of = np.zeros(max(n, 1), np.uint32) if want_ports else None
    stats = FlowStats()
    rc = lib().gf_run_dense_chain(seed, n, bins, nodes, DIST_NAMES[dist], zipf_s, chunk_capacity, live_particles,
                                  batch_chunks, int(bool(fused)), layout,
                                  port_of.ctypes.data if want_ports else None, C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "dense chain: " + last_error())
    return (port_of[:n] if want_ports else None), stats


class DevicePoolStats(C.Structure):
    """gf_device_pool_stats: counters of a device-resident chunk pool."""
    _fields_ = [("num_chunks", C.c_uint32), ("free_chunks", C.c_uint32), ("peak_live", C.c_uint32),
                ("status", C.c_uint32), ("acquired", C.c_uint64), ("released", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def run_dense_chain_device(seed, n, bins, nodes=1, dist="uniform", zipf_s=1.1, want_ports=True):
    """The dense chain of run_dense_chain run entirely on the device with a device-resident chunk
    pool. Returns (port_of, node_totals[nodes, bins], pool_stats, flow_stats)."""
    import numpy as np
    port_of = np.zeros(max(n, 1), np.uint32) if want_ports else None
    totals = np.zeros((nodes, bins), np.uint32)
    pool, stats = DevicePoolStats(), FlowStats()
    rc = lib().gf_run_dense_chain_device(seed, n, bins, nodes, DIST_NAMES[dist], zipf_s,
                                         port_of.ctypes.data if want_ports else None, totals.ctypes.data,
                                         C.byref(pool), C.byref(stats))
    if rc != GF_OK:
        raise GfError(rc, "device dense chain: " + last_error())
    return (port_of[:n] if want_ports else None), totals, pool, stats


def device_pool_bytes(num_chunks):
    out = C.c_uint64(0)
    check(lib().gf_device_pool_bytes(num_chunks, C.byref(out)), "device pool bytes")
    return out.value


class Rec16Columns(C.Structure):
    """gf_rec16_columns: device pointers of the 16-byte record columns (SoA) or records (AoS)."""
    _fields_ = [("key", C.c_void_p), ("weight", C.c_void_p), ("tag", C.c_void_p), ("records", C.c_void_p)]


def lib():
    """The loaded library. Raises if it has not been built: the product has no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"graphflow_b200: native library missing at {LIB_PATH}; run graphflow_b200.capi.build()")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        for name in ("gf_supported_tile_sizes", "gf_supported_hash_tile_sizes"):
            getattr(L, name).argtypes = [_VP, _U32]
            getattr(L, name).restype = _U32
        L.gf_last_error.argtypes = [_VP, C.c_size_t]
        L.gf_last_error.restype = C.c_size_t
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != GF_OK:
        raise GfError(rc, what)


def declared_symbols(header: str = HEADER):
    """Every function name the public header declares."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:gf_status|uint32_t|size_t)\s+(gf_\w+)\s*\(", text, re.M)))


# ---- host planning ------------------------------------------------------------------------------
def output_chunk_bound(n, capacity, max_bins):
    out = _U64()
    check(lib().gf_output_chunk_bound(n, capacity, max_bins, C.byref(out)), "outputChunkBound")
    return out.value


def checked_output_chunk_bound(n, capacity, max_bins):
    out = _U32()
    check(lib().gf_checked_output_chunk_bound(n, capacity, max_bins, C.byref(out)), "checkedOutputChunkBound")
    return out.value


def plan_dense(totals, capacity):
    import numpy as np
    totals = np.ascontiguousarray(totals, np.uint32)
    base = np.zeros(max(totals.size, 1), np.uint32)
    cap = int(((totals.astype(np.int64) + capacity - 1) // capacity).sum()) if capacity else 0
    fills = np.zeros(max(cap, 1), np.uint32)
    num = _U32()
    check(lib().gf_plan_dense(totals.ctypes.data, totals.size, capacity, base.ctypes.data, fills.ctypes.data, cap,
                              C.byref(num)), "planDenseBins")
    return base[:totals.size], fills[:num.value], num.value


def device_policy(n, props=None, chunk_capacity=0, live_particles=0, tile_size=0, live_per_chunk=0,
                  budget_bytes=0, slot_bytes=0):
    """gf_device_policy: the reference's default C, P, T for n particles on `props` (a DeviceProps,
    or None for the current CUDA device); 0 means "derive". Raises GfError for impossible requests."""
    out = Policy()
    check(lib().gf_device_policy(C.byref(props) if props is not None else None, n, chunk_capacity, live_particles,
                                 tile_size, live_per_chunk, budget_bytes, slot_bytes, C.byref(out)), "device policy")
    return out


def build_dense_table(bin_base, chunk_indices):
    import numpy as np
    bin_base = np.ascontiguousarray(bin_base, np.uint32)
    chunk_indices = np.ascontiguousarray(chunk_indices, np.uint32)
    table = np.zeros(bin_base.size + chunk_indices.size, np.uint32)
    check(lib().gf_build_dense_table(bin_base.ctypes.data, bin_base.size, chunk_indices.ctypes.data,
                                     chunk_indices.size, table.ctypes.data), "buildDenseTable")
    return table


def tile_count(fill, tile_size):
    out = _U32()
    check(lib().gf_tile_count(fill, tile_size, C.byref(out)), "tileCount")
    return out.value


def flatten_tiles(chunk_index, fills, tile_size):
    """Flatten chunks into tile descriptors; returns an (n, 3) uint32 array."""
    import numpy as np
    chunk_index = np.ascontiguousarray(chunk_index, np.uint32)
    fills = np.ascontiguousarray(fills, np.uint32)
    cap = int(((fills.astype(np.int64) + tile_size - 1) // tile_size).sum()) if tile_size else 0
    out = np.zeros((max(cap, 1), 3), np.uint32)
    n = _U32()
    check(lib().gf_flatten_tiles(chunk_index.ctypes.data, fills.ctypes.data, chunk_index.size, tile_size,
                                 out.ctypes.data, cap, C.byref(n)), "flattenTiles")
    return out[:n.value]


def supported_tile_sizes():
    import numpy as np
    buf = np.zeros(16, np.uint32)
    n = lib().gf_supported_tile_sizes(buf.ctypes.data, 16)
    return [int(x) for x in buf[:n]]


def zipf_cdf(s, k):
    import numpy as np
    cdf = np.zeros(k, np.float64)
    check(lib().gf_zipf_cdf(s, k, cdf.ctypes.data), "zipfCdf")
    return cdf


def fused_scratch_bytes(n_tiles, bins):
    out = _U64()
    check(lib().gf_fused_scratch_bytes(n_tiles, bins, C.byref(out)), "fusedScratchBytes")
    return out.value
