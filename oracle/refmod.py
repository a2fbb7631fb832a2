"""Loaders for the oracle: the reference's own compiled modules and the C restatement.

ORACLE INFRASTRUCTURE. Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module, and only as the checker (or the timed CPU baseline). Product code never imports it.

* ``load_ref(name)`` imports a module built by ``oracle/Makefile`` from the reference sources
  (``linear_ann_cpp``, ``ivf_lsh_cpp``, ``ref_linear_shim``, ``ref_ivf_shim``), choosing the
  AVX-512 or the AVX2 build according to what the host CPU supports, as the reference's
  ``-march=native`` build would (competitors/ivf_lsh/src/simd.h:3-11).
* ``restate()`` loads ``oracle/lib/liborestate.so`` (oracle/restate.c) through ctypes.
"""
from __future__ import annotations

import ctypes
import importlib.machinery
import importlib.util
import os
import sysconfig

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(HERE, "lib", "liborestate.so")

_AVX512_FLAGS = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_isa() -> str:
    """'avx512' when the host CPU has the x86-64-v4 AVX-512 subset, else 'avx2'."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return "avx512" if all(x in flags for x in _AVX512_FLAGS) else "avx2"
    except OSError:
        pass
    return "avx2"


def isa_lanes(isa: str) -> int:
    return {"avx512": 16, "avx2": 8, "scalar": 1}[isa]


_loaded: dict = {}


def ref_available(isa: str | None = None) -> bool:
    isa = isa or host_isa()
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    return os.path.exists(os.path.join(REF_DIR, isa, "ref_ivf_shim" + ext))


def load_ref(name: str, isa: str | None = None):
    """Import oracle/_ref/<isa>/<name>.so under its own module name."""
    isa = isa or host_isa()
    key = (name, isa)
    if key in _loaded:
        return _loaded[key]
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    path = os.path.join(REF_DIR, isa, name + ext)
    if not os.path.exists(path):
        raise FileNotFoundError(f"reference module not built: {path} (run `make -C oracle ref`)")
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    _loaded[key] = mod
    return mod


_F = ctypes.POINTER(ctypes.c_float)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)
_lib = None


def restate():
    """The C restatement (oracle/restate.c) as a ctypes library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"restatement not built: {LIB_PATH} (run `make -C oracle restate`)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.orc_l2.restype = ctypes.c_float
    lib.orc_l2.argtypes = [_F, _F, ctypes.c_int, ctypes.c_float, ctypes.c_int]
    lib.orc_l2_sq8.restype = ctypes.c_float
    lib.orc_l2_sq8.argtypes = [_U8, _F, ctypes.c_int, _F, ctypes.c_float, ctypes.c_int]
    lib.orc_linear_values.argtypes = [_F, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, _F, ctypes.c_int,
                                      ctypes.c_int, _F]
    lib.orc_linear_query_batch.restype = ctypes.c_int
    lib.orc_linear_query_batch.argtypes = [_F, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, _F, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, _I64, _F]
    lib.orc_ivf_query.restype = ctypes.c_int64
    lib.orc_ivf_query.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  _F, _U8, _F, _F, _F, _F, _I32, _F, _I64, _I32, _F,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int64, _I64, _F]
    lib.orc_sq8_train.argtypes = [_F, ctypes.c_int64, ctypes.c_int, _F, _F]
    lib.orc_sq8_encode.argtypes = [_F, ctypes.c_int64, ctypes.c_int, _F, _F, _U8]
    lib.orc_kmeans_order.argtypes = [ctypes.c_int64, _I32]
    lib.orc_kmeans.restype = ctypes.c_int
    lib.orc_kmeans.argtypes = [_F, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.c_int, _F, _I32]
    lib.orc_gf_train.argtypes = [_F, ctypes.c_int64, ctypes.c_int, _F, _F]
    lib.orc_gf_encode.argtypes = [_F, ctypes.c_int64, ctypes.c_int, _F, _F, _U8]
    lib.orc_gf_query.restype = ctypes.c_int
    lib.orc_gf_query.argtypes = [_F, _U8, ctypes.c_int64, ctypes.c_int, _F, _F, _F, ctypes.c_int, ctypes.c_int,
                                 _I64, _I64]
    _lib = lib
    return lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def l2(a, b, threshold=np.finfo(np.float32).max, lanes=16) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(restate().orc_l2(_p(a, _F), _p(b, _F), a.size, threshold, lanes))


def l2_sq8(code, q_shifted, scale, threshold=np.finfo(np.float32).max, lanes=16) -> float:
    code = np.ascontiguousarray(code, np.uint8)
    qs = np.ascontiguousarray(q_shifted, np.float32)
    sc = np.ascontiguousarray(scale, np.float32)
    return float(restate().orc_l2_sq8(_p(code, _U8), _p(qs, _F), code.size, _p(sc, _F), threshold, lanes))


def linear_values(data, q, k, lanes=16) -> np.ndarray:
    """Per-point ranking values of the reference linear scan for one query."""
    data = np.ascontiguousarray(data, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    n, d = data.shape
    out = np.empty(n, np.float32)
    restate().orc_linear_values(_p(data, _F), n, d, d, _p(q, _F), k, lanes, _p(out, _F))
    return out


def linear_query(data, queries, k, lanes=16):
    """Reference linear scan (ids int64 [nq, k], ranking values float32 [nq, k])."""
    data = np.ascontiguousarray(data, np.float32)
    queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
    n, d = data.shape
    nq = queries.shape[0]
    kk = min(k, n)
    ids = np.empty((nq, kk), np.int64)
    vals = np.empty((nq, kk), np.float32)
    rc = restate().orc_linear_query_batch(_p(data, _F), n, d, d, _p(queries, _F), nq, kk, lanes,
                                          _p(ids, _I64), _p(vals, _F))
    if rc != 0:
        raise MemoryError("orc_linear_query_batch failed")
    return ids, vals


def ivf_query(state: dict, q, k, n_probes=0, n_probe_clusters=8, refine_r=-1, num_threads=8, lanes=16,
              max_cands=-1):
    """Reference IVF-LSH query over an exported index state. Returns (ids, dists, n_cands)."""
    s = state
    q = np.ascontiguousarray(q, np.float32)
    arr = {key: np.ascontiguousarray(s[key]) for key in
           ("centroids", "quantized_data", "original_data", "scale", "offset", "mean",
            "reordered_to_original", "projections", "table_offsets", "table_ids")}
    if arr["table_ids"].size == 0:
        arr["table_ids"] = np.zeros(1, np.int32)
    if arr["projections"].size == 0:
        arr["projections"] = np.zeros(1, np.float32)
    ids = np.empty(k, np.int64)
    dists = np.empty(k, np.float32)
    nc = restate().orc_ivf_query(
        int(s["npts"]), int(s["dim"]), int(s["n_clusters"]), int(s["n_tables"]), int(s["n_bits"]),
        _p(arr["centroids"], _F), _p(arr["quantized_data"], _U8), _p(arr["original_data"], _F),
        _p(arr["scale"], _F), _p(arr["offset"], _F), _p(arr["mean"], _F),
        _p(arr["reordered_to_original"], _I32), _p(arr["projections"], _F),
        _p(arr["table_offsets"], _I64), _p(arr["table_ids"], _I32), _p(q, _F),
        k, n_probes, n_probe_clusters, refine_r, num_threads, lanes, max_cands,
        _p(ids, _I64), _p(dists, _F))
    if nc < 0:
        raise MemoryError("orc_ivf_query failed")
    return ids, dists, int(nc)


def kmeans_order(n: int) -> np.ndarray:
    """rand_indices of the reference's k-means: std::shuffle(iota(n), std::mt19937(1337))."""
    out = np.empty(n, np.int32)
    restate().orc_kmeans_order(n, _p(out, _I32))
    return out


def kmeans(x, n_clusters: int, num_threads: int, iters: int = 15, lanes: int = 16, workers: int | None = None):
    """The reference's k-means restated (oracle/restate_kmeans.cpp) with a ThreadPool of `num_threads`:
    (centroids float32 [C, dim], last assignment int32 [n]). C = min(n_clusters, n) as the reference's fit."""
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    c = min(int(n_clusters), n)
    cent = np.empty((c, d), np.float32)
    assign = np.empty(n, np.int32)
    rc = restate().orc_kmeans(_p(x, _F), n, d, c, iters, num_threads, lanes, workers or os.cpu_count() or 1,
                              _p(cent, _F), _p(assign, _I32))
    if rc != 0:
        raise ValueError("orc_kmeans: bad arguments")
    return cent, assign


def ref_fit(x, n_tables: int, n_bits: int, n_clusters: int, num_threads: int, isa: str | None = None):
    """The reference's own LSHIndex.fit with its thread count pinned to `num_threads` (the shim's
    set_fit_threads); returns the fitted index, whose query pool has the same size."""
    m = load_ref("ref_ivf_shim", isa)
    ix = m.LSHIndex()
    m.set_fit_threads(num_threads)
    try:
        ix.fit(np.ascontiguousarray(x, np.float32), n_tables, n_bits, n_clusters)
    finally:
        m.set_fit_threads(0)
    return ix


def sq8_train(x):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    scale = np.empty(d, np.float32)
    offset = np.empty(d, np.float32)
    restate().orc_sq8_train(_p(x, _F), n, d, _p(scale, _F), _p(offset, _F))
    return scale, offset


def sq8_encode(x, scale, offset):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    codes = np.empty((n, d), np.uint8)
    scale = np.ascontiguousarray(scale, np.float32)
    offset = np.ascontiguousarray(offset, np.float32)
    restate().orc_sq8_encode(_p(x, _F), n, d, _p(scale, _F), _p(offset, _F), _p(codes, _U8))
    return codes


def exact_topk_f64(data, queries, k, metric="l2", chunk=256):
    """FP64 exact top-k by brute force, ties broken by lower id: (ids, squared distances) for
    "l2", (ids, inner products, best first) for "ip"."""
    data64 = np.asarray(data, np.float64)
    queries = np.atleast_2d(np.asarray(queries, np.float64))
    xn = np.einsum("ij,ij->i", data64, data64)
    n = data64.shape[0]
    kk = min(k, n)
    ids = np.empty((queries.shape[0], kk), np.int64)
    dist = np.empty((queries.shape[0], kk), np.float64)
    for s in range(0, queries.shape[0], chunk):
        qb = queries[s:s + chunk]
        ip = qb @ data64.T
        if metric == "ip":
            key = -ip
        else:
            key = xn[None, :] - 2.0 * ip + np.einsum("ij,ij->i", qb, qb)[:, None]
        part = np.argpartition(key, kk - 1, axis=1)[:, :kk]
        pk = np.take_along_axis(key, part, 1)
        order = np.lexsort((part, pk), axis=1)
        ids[s:s + chunk] = np.take_along_axis(part, order, 1)
        sk = np.take_along_axis(pk, order, 1)
        dist[s:s + chunk] = -sk if metric == "ip" else sk
    return ids, dist


def gf_search(x, queries, k, r):
    """The GPU quantized-filter contestant (competitors/gpu_filter/src/gpu_filter.cu) restated on the CPU:
    its SQ8 state from x, then gf_query per query. Returns (counts int32 [nq], ids int64 [nq, k] padded
    with -1, the distance count after the queries)."""
    lib = restate()
    x = np.ascontiguousarray(x, np.float32)
    queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
    n, d = x.shape
    scale = np.empty(d, np.float32)
    offset = np.empty(d, np.float32)
    codes = np.empty((n, d), np.uint8)
    lib.orc_gf_train(_p(x, _F), n, d, _p(scale, _F), _p(offset, _F))
    lib.orc_gf_encode(_p(x, _F), n, d, _p(scale, _F), _p(offset, _F), _p(codes, _U8))
    got = np.zeros(queries.shape[0], np.int32)
    ids = np.full((queries.shape[0], k), -1, np.int64)
    ndist = np.zeros(1, np.int64)
    for i, q in enumerate(queries):
        o = np.full(max(k, 1), -1, np.int64)
        got[i] = lib.orc_gf_query(_p(x, _F), _p(codes, _U8), n, d, _p(scale, _F), _p(offset, _F), _p(q, _F), k, r,
                                  _p(o, _I64), _p(ndist, _I64))
        ids[i, :got[i]] = o[:got[i]]
    return got, ids, int(ndist[0])

