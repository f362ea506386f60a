"""ctypes binding of the CPU oracle (oracle/gf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the
CPU-baseline legs of ``bench.py``, always as the checker or as the timed CPU restatement of the
reference. The product package ``graphflow_b200`` never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgforacle.so")

OK, INVALID, OVERFLOW, LOGIC = 0, 1, 2, 3

CLS_KEY_MOD, CLS_ID_BALANCED, CLS_ID_ONEHOT, CLS_ID_SKEWED, CLS_KEY_UNMIX = range(5)
DIST_UNIFORM, DIST_ZIPF, DIST_ONE_PORT, DIST_ROUND_ROBIN = range(4)
DIST_NAMES = {"uniform": DIST_UNIFORM, "zipf": DIST_ZIPF, "one_port": DIST_ONE_PORT,
              "round_robin": DIST_ROUND_ROBIN}


class OracleError(RuntimeError):
    pass


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class Tile(C.Structure):
    _fields_ = [("chunk_index", C.c_uint32), ("tile_offset", C.c_uint32), ("count", C.c_uint32)]


class OutDesc(C.Structure):
    _fields_ = [("chunk_index", C.c_uint32), ("fill", C.c_uint32), ("bin", C.c_uint32)]


class PhotonTerminal(C.Structure):
    _fields_ = [("event", C.c_uint32), ("scatter_count", C.c_uint32), ("x", C.c_double), ("y", C.c_double),
                ("z", C.c_double), ("ux", C.c_double), ("uy", C.c_double), ("uz", C.c_double)]


class HgParams(C.Structure):
    _fields_ = [("thickness", C.c_double), ("mu_a", C.c_double), ("mu_s", C.c_double), ("g", C.c_double),
                ("roulette_threshold", C.c_double), ("roulette_survival", C.c_double),
                ("max_scatters", C.c_uint32), ("hist_bins", C.c_uint32)]


class HgTerminal(C.Structure):
    _fields_ = [("event", C.c_uint32), ("scatter_count", C.c_uint32), ("weight", C.c_double),
                ("cos_exit", C.c_double)]


_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _declare(L):
    u64, u32, i32 = C.c_uint64, C.c_uint32, C.c_int
    L.gfo_mix64.restype = u64
    L.gfo_mix64.argtypes = [u64]
    L.gfo_unmix64.restype = u64
    L.gfo_unmix64.argtypes = [u64]
    L.gfo_stream_key.restype = u64
    L.gfo_stream_key.argtypes = [u64, u64, u64, u32]
    L.gfo_draw.restype = u32
    L.gfo_draw.argtypes = [u64, u64, u64, u32]
    L.gfo_draws.argtypes = [u64, u64, u64, u32, _u32p, u32]
    L.gfo_uniform_f32.restype = C.c_float
    L.gfo_uniform_f32.argtypes = [u32]
    L.gfo_uniform_f64.restype = C.c_double
    L.gfo_uniform_f64.argtypes = [u32]
    L.gfo_output_chunk_bound.restype = i32
    L.gfo_output_chunk_bound.argtypes = [u64, u64, u64, C.POINTER(u64)]
    L.gfo_checked_output_chunk_bound.restype = i32
    L.gfo_checked_output_chunk_bound.argtypes = [u64, u64, u64, C.POINTER(u32)]
    L.gfo_plan_dense.restype = i32
    L.gfo_plan_dense.argtypes = [_u32p, u64, u32, _u32p, _u32p, u64, C.POINTER(u32)]
    L.gfo_tile_count.restype = i32
    L.gfo_tile_count.argtypes = [u32, u32, C.POINTER(u32)]
    L.gfo_flatten_tiles.restype = C.c_int64
    L.gfo_flatten_tiles.argtypes = [_u32p, _u32p, u32, u32, C.POINTER(Tile), u64]
    L.gfo_classify.restype = u32
    L.gfo_classify.argtypes = [i32, u64, u32, u64]
    L.gfo_partition_stable_u32.restype = i32
    L.gfo_partition_stable_u32.argtypes = [_u32p, u64, u32, i32, _u32p, C.c_void_p, i32]
    L.gfo_partition_stable_u64.restype = i32
    L.gfo_partition_stable_u64.argtypes = [_u64p, u64, u32, i32, u64, _u32p, C.c_void_p, i32]
    L.gfo_partition_pool_u32.restype = i32
    L.gfo_partition_pool_u32.argtypes = [_u32p, _u32p, u32, C.POINTER(Tile), u64, u32, i32, _u32p, _u32p,
                                         _u32p, u64, _u32p, C.POINTER(OutDesc), C.POINTER(u32), i32]
    L.gfo_dist_purpose.restype = u32
    L.gfo_dist_purpose.argtypes = [i32]
    L.gfo_zipf_cdf.argtypes = [C.c_double, u32, _f64p]
    L.gfo_zipf_sample.restype = u32
    L.gfo_zipf_sample.argtypes = [_f64p, u32, u32]
    L.gfo_generate_keys_u32.argtypes = [i32, u64, u64, u64, u32, C.c_void_p, _u32p, i32]
    L.gfo_generate_records16.argtypes = [u64, u64, u64, _f64p, u32, u64, _u64p, _f32p, _u32p, i32]
    L.gfo_particle_scalar.restype = i32
    L.gfo_particle_scalar.argtypes = [u64, u64, u32, _u32p, C.c_void_p, C.POINTER(u64), i32]
    L.gfo_histogram_u32.restype = u64
    L.gfo_histogram_u32.argtypes = [_u32p, u64, C.c_void_p, C.c_void_p]
    L.gfo_photon_analog.restype = i32
    L.gfo_photon_analog.argtypes = [u64, u64, C.c_double, C.c_double, C.c_double, i32, u32,
                                    C.POINTER(PhotonTerminal), i32]
    L.gfo_photon_analog_traced.restype = i32
    L.gfo_photon_analog_traced.argtypes = [u64, u64, C.c_double, C.c_double, C.c_double, i32, u32,
                                           C.POINTER(PhotonTerminal), u32, u32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, i32]
    L.gfo_photon_hg.restype = i32
    L.gfo_photon_hg.argtypes = [u64, u64, u64, C.POINTER(HgParams), C.c_void_p, _f64p, _f64p, _u64p, i32]


def _check(rc, what):
    if rc == OK:
        return
    raise OracleError(f"{what}: " + {INVALID: "invalid argument", OVERFLOW: "overflow",
                                     LOGIC: "logic error"}.get(rc, f"error {rc}"))


# ---- RNG ----
def mix64(v): return lib().gfo_mix64(v)
def unmix64(v): return lib().gfo_unmix64(v)
def stream_key(seed, i, event, purpose): return lib().gfo_stream_key(seed, i, event, purpose)
def draw(seed, i, event, purpose): return lib().gfo_draw(seed, i, event, purpose)


def draws(seed, i, event, purpose, n):
    out = np.zeros(n, np.uint32)
    lib().gfo_draws(seed, i, event, purpose, out, n)
    return out


def uniform_f32(x): return lib().gfo_uniform_f32(x)
def uniform_f64(x): return lib().gfo_uniform_f64(x)


# ---- reservation / plan ----
def output_chunk_bound(n, capacity, max_bins):
    out = C.c_uint64()
    _check(lib().gfo_output_chunk_bound(n, capacity, max_bins, C.byref(out)), "outputChunkBound")
    return out.value


def checked_output_chunk_bound(n, capacity, max_bins):
    out = C.c_uint32()
    _check(lib().gfo_checked_output_chunk_bound(n, capacity, max_bins, C.byref(out)), "checkedOutputChunkBound")
    return out.value


def plan_dense(totals, capacity):
    totals = np.ascontiguousarray(totals, np.uint32)
    bins = totals.size
    base = np.zeros(max(bins, 1), np.uint32)
    cap = int(((totals.astype(np.int64) + capacity - 1) // capacity).sum()) if capacity else 0
    fills = np.zeros(max(cap, 1), np.uint32)
    num = C.c_uint32()
    _check(lib().gfo_plan_dense(totals if bins else np.zeros(1, np.uint32), bins, capacity, base, fills, cap,
                                C.byref(num)), "planDenseBins")
    return base[:bins], fills[:num.value], num.value


def build_dense_table(bin_base, chunk_indices, num_out):
    if len(chunk_indices) != num_out:
        raise OracleError("buildDenseTable: chunk index count does not match the plan")
    return np.concatenate([np.asarray(bin_base, np.uint32), np.asarray(chunk_indices, np.uint32)])


def tile_count(fill, tile_size):
    out = C.c_uint32()
    _check(lib().gfo_tile_count(fill, tile_size, C.byref(out)), "tileCount")
    return out.value


def flatten_tiles(chunk_index, fills, tile_size, cap=None):
    chunk_index = np.ascontiguousarray(chunk_index, np.uint32)
    fills = np.ascontiguousarray(fills, np.uint32)
    if cap is None:
        cap = int(sum(-(-int(f) // tile_size) for f in fills)) if tile_size else 0
    arr = (Tile * max(cap, 1))()
    n = lib().gfo_flatten_tiles(chunk_index, fills, chunk_index.size, tile_size, arr, cap)
    if n < 0:
        _check(-n, "flattenTiles")
    return np.array([(arr[i].chunk_index, arr[i].tile_offset, arr[i].count) for i in range(n)],
                    dtype=np.uint32).reshape(-1, 3)


def classify(cls, key, bins, salt=0):
    return lib().gfo_classify(cls, key, bins, salt)


def partition_stable_u32(keys, bins, cls=CLS_KEY_MOD, threads=0, want_order=True):
    keys = np.ascontiguousarray(keys, np.uint32)
    counts = np.zeros(bins, np.uint32)
    order = np.zeros(max(keys.size, 1), np.uint32) if want_order else None
    rc = lib().gfo_partition_stable_u32(keys, keys.size, bins, cls, counts,
                                        order.ctypes.data if order is not None else None, threads)
    _check(rc, "partition")
    return counts, (order[:keys.size] if order is not None else None)


def partition_stable_u64(keys, bins, cls=CLS_KEY_UNMIX, salt=0, threads=0, want_order=True):
    keys = np.ascontiguousarray(keys, np.uint64)
    counts = np.zeros(bins, np.uint32)
    order = np.zeros(max(keys.size, 1), np.uint32) if want_order else None
    rc = lib().gfo_partition_stable_u64(keys, keys.size, bins, cls, salt, counts,
                                        order.ctypes.data if order is not None else None, threads)
    _check(rc, "partition")
    return counts, (order[:keys.size] if order is not None else None)


def partition_pool_u32(pool_in, capacity, tiles, bins, free_chunks, cls=CLS_KEY_MOD, threads=0, pool_out=None,
                       bin_ids=None):
    """Reference-structured classify -> plan -> scatter over a chunk pool (timed CPU baseline)."""
    pool_in = np.ascontiguousarray(pool_in, np.uint32)
    if pool_out is None:
        pool_out = np.zeros_like(pool_in)
    if bin_ids is None:
        bin_ids = np.zeros_like(pool_in)
    tiles = np.ascontiguousarray(tiles, np.uint32).reshape(-1, 3)
    tarr = tiles.ctypes.data_as(C.POINTER(Tile))
    free_chunks = np.ascontiguousarray(free_chunks, np.uint32)
    counts = np.zeros(bins, np.uint32)
    table = np.zeros(bins + free_chunks.size, np.uint32)
    outs = (OutDesc * max(free_chunks.size, 1))()
    n_outs = C.c_uint32()
    rc = lib().gfo_partition_pool_u32(pool_in, pool_out, capacity, tarr, tiles.shape[0], bins, cls, bin_ids, counts,
                                      free_chunks, free_chunks.size, table, outs, C.byref(n_outs), threads)
    _check(rc, "partition pool")
    descs = np.array([(outs[i].chunk_index, outs[i].fill, outs[i].bin) for i in range(n_outs.value)],
                     dtype=np.uint32).reshape(-1, 3)
    return pool_out, counts, table[:bins + n_outs.value], descs


# ---- generators ----
def zipf_cdf(s, k):
    cdf = np.zeros(k, np.float64)
    lib().gfo_zipf_cdf(s, k, cdf)
    return cdf


def generate_keys_u32(dist, seed, n, bins, zipf_s=1.1, first_id=0, threads=0):
    dist = DIST_NAMES.get(dist, dist)
    keys = np.zeros(max(n, 1), np.uint32)
    cdf = zipf_cdf(zipf_s, bins) if dist == DIST_ZIPF else None
    lib().gfo_generate_keys_u32(dist, seed, first_id, n, bins, cdf.ctypes.data if cdf is not None else None, keys,
                                threads)
    return keys[:n]


def generate_records16(seed, n, k, zipf_s, salt, first_id=0, threads=0):
    cdf = zipf_cdf(zipf_s, k)
    keys = np.zeros(max(n, 1), np.uint64)
    weights = np.zeros(max(n, 1), np.float32)
    tags = np.zeros(max(n, 1), np.uint32)
    lib().gfo_generate_records16(seed, first_id, n, cdf, k, salt, keys, weights, tags, threads)
    return keys[:n], weights[:n], tags[:n]


# ---- particle feedback ----
def particle_scalar(seed, n, max_visits, threads=0):
    weights = np.zeros(max(n, 1), np.uint32)
    capped = np.zeros(max(n, 1), np.uint8)
    ncap = C.c_uint64()
    _check(lib().gfo_particle_scalar(seed, n, max_visits, weights, capped.ctypes.data, C.byref(ncap), threads),
           "scalar model")
    return weights[:n], capped[:n], ncap.value


def histogram_u32(values):
    v = np.array(values, np.uint32, copy=True)
    w = np.zeros(max(v.size, 1), np.uint32)
    c = np.zeros(max(v.size, 1), np.uint64)
    rows = lib().gfo_histogram_u32(v, v.size, w.ctypes.data, c.ctypes.data)
    return w[:rows], c[:rows]


# ---- photons ----
def photon_analog(seed, n, thickness, sigma_s, sigma_a, isotropic, max_scatters, threads=0):
    arr = (PhotonTerminal * max(n, 1))()
    _check(lib().gfo_photon_analog(seed, n, thickness, sigma_s, sigma_a, int(isotropic), max_scatters, arr, threads),
           "photon analog")
    out = np.ctypeslib.as_array(arr)[:n]
    return out


TRACE_VERTEX_DTYPE = [("kind", "<u4"), ("scatter_count", "<u4"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                      ("ux", "<f8"), ("uy", "<f8"), ("uz", "<f8")]  # gfo_trace_vertex


def photon_analog_traced(seed, n, thickness, sigma_s, sigma_a, isotropic, max_scatters, trace_photons,
                         trace_vertices, threads=0):
    """photon_analog plus the bounded path trace: (terminals, vertices (M, V), counts (M,), truncated (M,))."""
    ids = min(n, trace_photons)
    arr = (PhotonTerminal * max(n, 1))()
    v = np.zeros((max(ids, 1), max(trace_vertices, 1)), TRACE_VERTEX_DTYPE)
    counts = np.zeros(max(ids, 1), np.uint32)
    truncated = np.zeros(max(ids, 1), np.uint32)
    _check(lib().gfo_photon_analog_traced(seed, n, thickness, sigma_s, sigma_a, int(isotropic), max_scatters, arr,
                                          trace_photons, trace_vertices, v.ctypes.data, counts.ctypes.data,
                                          truncated.ctypes.data, threads), "photon analog traced")
    return np.ctypeslib.as_array(arr)[:n], v[:ids, :trace_vertices], counts[:ids], truncated[:ids]


def hg_params(thickness=1.0, mu_a=0.1, mu_s=10.0, g=0.9, roulette_threshold=1e-4, roulette_survival=0.1,
              max_scatters=65535, hist_bins=256):
    return HgParams(thickness, mu_a, mu_s, g, roulette_threshold, roulette_survival, max_scatters, hist_bins)


def photon_hg(seed, n, params=None, first_id=0, threads=0, want_terminals=False):
    p = params or hg_params()
    refl = np.zeros(p.hist_bins, np.float64)
    trans = np.zeros(p.hist_bins, np.float64)
    ev = np.zeros(5, np.uint64)
    arr = (HgTerminal * max(n, 1))() if want_terminals else None
    _check(lib().gfo_photon_hg(seed, first_id, n, C.byref(p), C.cast(arr, C.c_void_p) if arr is not None else None,
                               refl, trans, ev, threads), "photon hg")
    terms = np.ctypeslib.as_array(arr)[:n] if arr is not None else None
    return refl, trans, ev, terms


def cpu_threads():
    return os.cpu_count() or 1
