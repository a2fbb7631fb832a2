"""IVF-SQ8 index on the GPU: the drop-in for ivf_lsh_cpp.LSHIndex (inverted lists, optionally with
LSH bucket tables over them: n_tables >= 1, n_bits in [0, 16]).

Surface of the reference (competitors/ivf_lsh/src/lsh_index_optimized.cpp:658-666):
``fit(data, n_tables, n_bits, n_clusters=256)``, ``query(query, k, n_probes=0, n_probe_clusters=8,
refine_r=-1) -> int64[k]``, ``total_distances_count()``, ``reset_distances_count()``,
``get_profile_results()``, ``reset_profile_results()``.

Two semantics (``mode``):

* ``"reference"``: the reference's ranking bit for bit -- its coarse ranking arithmetic, candidate
  cap, per-ThreadPool-chunk 64-entry early-abandon SQ8 pass (``num_threads`` = the reference host's
  hardware concurrency, default this host's), FP32 re-rank and id mapping;
* ``"exact"``: the same pipeline with full SQ8 distances (no early abandon) and, by default, no
  candidate cap -- the batched GPU form used for throughput.

Extras: ``search(queries, k, ...)`` (batched; numpy in -> numpy out, CUDA tensor in -> CUDA tensor
out on the current stream), ``import_state`` / ``export_state`` (the reference's state layout, used
for parity), and ``fit(..., centroids=, assign=)`` to build lists from a given coarse quantiser.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib


def _host_out(out, shape, dtype, name):
    """The host array a search writes: `out` (a C-contiguous numpy array, or a CPU torch tensor, of this
    shape and type -- page-locked memory makes the device-to-host copy a direct one) or a new array."""
    if out is None:
        return np.empty(shape, dtype)
    if _lib.is_torch(out):
        if out.is_cuda:
            raise RuntimeError(f"{name}: host queries need a host output")
        out = out.numpy()
    if out.shape != shape or out.dtype != dtype or not out.flags.c_contiguous:
        raise RuntimeError(f"{name} must be a C-contiguous {np.dtype(dtype).name} array of shape {shape}")
    return out


class IVFIndex:
    def __init__(self, device: int = 0, mode: str = "reference", num_threads: int | None = None):
        self._lib = _lib.load()
        if mode not in _lib.MODES:
            raise ValueError(f"unknown mode {mode!r}")
        h = ctypes.c_void_p()
        _lib.check(self._lib.ann_ivf_create(ctypes.byref(h), device))
        self._h = h
        self.device = device
        self.mode = mode
        self.num_threads = int(num_threads) if num_threads else (os.cpu_count() or 1)
        if mode == "reference":  # the reference times every query's stages (lsh_index_optimized.cpp:305-515)
            _lib.check(self._lib.ann_ivf_set_profiling(self._h, 1))
        self._n = 0
        self._dim = 0
        self._C = 0

    # ---- build -----------------------------------------------------------------------------------
    def fit(self, data, n_tables: int = 1, n_bits: int = 0, n_clusters: int = 256, kmeans_iters: int = 15,
            centroids=None, assign=None) -> None:
        if int(n_tables) < 1 or not 0 <= int(n_bits) <= 16:
            raise RuntimeError("n_tables must be >= 1 and n_bits in [0, 16]")
        if _lib.is_torch(data):
            x = _lib.as_f32_2d(data, "data")
            mem = _lib.MEM_DEVICE if x.is_cuda else _lib.MEM_HOST
            if not x.is_cuda:
                x = x.numpy()
            ld = x.stride(0) if mem == _lib.MEM_DEVICE else x.shape[1]
        else:
            a = np.asarray(data)
            if a.ndim != 2:
                raise RuntimeError("Input data must be 2D")
            x = np.ascontiguousarray(a, np.float32)
            mem, ld = _lib.MEM_HOST, x.shape[1]
        n, d = x.shape
        if n == 0 or d == 0:
            raise RuntimeError("Input data must be a non-empty 2D array")
        cen = asg = None
        if centroids is not None:
            cen = self._like(centroids, mem, np.float32, x)
            if tuple(cen.shape) != (min(int(n_clusters), n), d):
                raise RuntimeError("centroids must have shape [n_clusters, dim]")
        if assign is not None:
            asg = self._like(assign, mem, np.int32, x)
            if asg.shape[0] != n:
                raise RuntimeError("assign must have one entry per row")
        st = _lib.stream_ptr(x) if mem == _lib.MEM_DEVICE else None
        _lib.check(self._lib.ann_ivf_fit(self._h, _lib.ptr(x), n, d, ld, int(n_clusters), _lib.ptr(cen),
                                         _lib.ptr(asg), int(kmeans_iters), int(self.num_threads), mem, st))
        self._n, self._dim = n, d
        self._C = min(int(n_clusters), n)
        if int(n_tables) != 1 or int(n_bits) != 0:  # LSH bucket tables over the lists
            _lib.check(self._lib.ann_ivf_build_tables(self._h, int(n_tables), int(n_bits), st))

    def build_tables(self, n_tables: int, n_bits: int, stream=None) -> None:
        """(Re)builds the LSH bucket tables over the fitted lists, as fit does for n_bits > 0 or several
        tables (lsh_index_optimized.cpp:207-283): projections from mt19937(42), Gram-Schmidt per table,
        buckets (table, list, signature) of list-order ids. n_tables = 1, n_bits = 0 drops the tables."""
        if self._n == 0:
            raise RuntimeError("index not fitted")
        if int(n_tables) < 1 or not 0 <= int(n_bits) <= 16:
            raise RuntimeError("n_tables must be >= 1 and n_bits in [0, 16]")
        st = _lib.stream_ptr(None, stream)
        _lib.check(self._lib.ann_ivf_build_tables(self._h, int(n_tables), int(n_bits), st))

    @staticmethod
    def _like(v, mem, dtype, x):
        if mem == _lib.MEM_DEVICE:
            import torch
            t = v if _lib.is_torch(v) else torch.from_numpy(np.asarray(v))
            return t.to(device=x.device, dtype=torch.float32 if dtype == np.float32 else torch.int32).contiguous()
        return np.ascontiguousarray(v.cpu().numpy() if _lib.is_torch(v) else v, dtype)

    def import_state(self, state: dict) -> None:
        """Loads a state in the reference's layout: keys npts, dim, n_clusters, n_tables, n_bits,
        centroids, original_data, quantized_data, scale, offset, mean, reordered_to_original,
        projections, table_offsets, table_ids. With n_tables = 1 and n_bits = 0 the table offsets are the
        list offsets; otherwise they index the buckets (t, list, signature) and the list offsets follow from
        table 0."""
        n, d, c = int(state["npts"]), int(state["dim"]), int(state["n_clusters"])
        T, B = int(state.get("n_tables", 1)), int(state.get("n_bits", 0))
        toff = np.ascontiguousarray(state["table_offsets"], np.int64)
        if T == 1 and B == 0:
            list_off = toff
        else:
            list_off = np.ascontiguousarray(toff[: c * (1 << B) + 1: 1 << B], np.int64)
        arrs = [np.ascontiguousarray(state[k], t) for k, t in (
            ("centroids", np.float32), ("original_data", np.float32), ("quantized_data", np.uint8),
            ("scale", np.float32), ("offset", np.float32), ("reordered_to_original", np.int32))]
        _lib.check(self._lib.ann_ivf_import(self._h, n, d, c, *[_lib.ptr(a) for a in arrs], _lib.ptr(list_off)))
        self._n, self._dim, self._C = n, d, c
        if T != 1 or B != 0:
            proj = np.ascontiguousarray(state["projections"], np.float32).reshape(T * B, d) if B else None
            mean = np.ascontiguousarray(state["mean"], np.float32)
            ids = np.ascontiguousarray(state["table_ids"], np.int32)
            _lib.check(self._lib.ann_ivf_import_tables(self._h, T, B, _lib.ptr(proj), _lib.ptr(mean), _lib.ptr(toff),
                                                       _lib.ptr(ids)))

    def export_state(self) -> dict:
        n, d, c = self._n, self._dim, self._C
        tb = (ctypes.c_int32 * 2)()
        _lib.check(self._lib.ann_ivf_export_tables(self._h, tb, None, None, None, None))
        T, B = int(tb[0]), int(tb[1])
        out = {"npts": n, "dim": d, "n_clusters": c, "n_tables": T, "n_bits": B,
               "centroids": np.empty((c, d), np.float32), "original_data": np.empty((n, d), np.float32),
               "quantized_data": np.empty((n, d), np.uint8), "scale": np.empty(d, np.float32),
               "offset": np.empty(d, np.float32), "reordered_to_original": np.empty(n, np.int32),
               "table_offsets": np.empty(c + 1, np.int64)}
        _lib.check(self._lib.ann_ivf_export(self._h, *[_lib.ptr(out[k]) for k in (
            "centroids", "original_data", "quantized_data", "scale", "offset", "reordered_to_original",
            "table_offsets")]))
        if T == 1 and B == 0:
            out["mean"] = np.zeros(d, np.float32)
            out["projections"] = np.zeros((0, d), np.float32)
            out["table_ids"] = np.arange(n, dtype=np.int32)
        else:
            out["projections"] = np.empty((T * B, d), np.float32)
            out["mean"] = np.empty(d, np.float32)
            out["table_offsets"] = np.empty(T * c * (1 << B) + 1, np.int64)
            out["table_ids"] = np.empty(T * n, np.int32)
            _lib.check(self._lib.ann_ivf_export_tables(self._h, None, _lib.ptr(out["projections"]),
                                                       _lib.ptr(out["mean"]), _lib.ptr(out["table_offsets"]),
                                                       _lib.ptr(out["table_ids"])))
        return out

    # ---- reference surface -----------------------------------------------------------------------
    def query(self, query, k: int, n_probes: int = 0, n_probe_clusters: int = 8, refine_r: int = -1,
              max_candidates: int | None = None) -> np.ndarray:
        qa = np.asarray(query.cpu() if _lib.is_torch(query) else query, np.float32)
        if qa.ndim != 1 or qa.shape[0] != self._dim:
            raise RuntimeError("Query dimension mismatch")
        ids, _ = self.search(qa.reshape(1, -1), k, n_probes=n_probes, n_probe_clusters=n_probe_clusters,
                             refine_r=refine_r, max_candidates=max_candidates)
        return ids[0]

    def total_distances_count(self) -> int:
        return int(self._lib.ann_ivf_total_distances(self._h))

    def reset_distances_count(self) -> None:
        _lib.check(self._lib.ann_ivf_reset_distances(self._h))

    def set_profiling(self, enable: bool = True) -> None:
        _lib.check(self._lib.ann_ivf_set_profiling(self._h, int(enable)))

    def get_profile_results(self) -> dict:
        """The reference's keys (lsh_index_optimized.cpp:535-548): with queries answered, the six
        averages per query, else {"query_count": 0}, as the reference returns them. The stage times come
        from CUDA events on the query stream while profiling is on (the default in reference mode; a
        batch's stage time is divided by its queries): centroid search = the coarse ranking, signature
        calc = the LSH signatures and flips, bucket lookup = the candidate plan / bucket walk, distance
        calc = the SQ8 (or BF16) keys plus the exact FP32 re-rank and its top-k, candidate sort = the
        selection of the best R candidates (the reference's partial sort before its re-rank)."""
        out = (ctypes.c_double * 8)()
        _lib.check(self._lib.ann_ivf_profile(self._h, out))
        nq = int(out[7])
        if nq == 0:
            return {"query_count": 0}
        coarse, sig, plan, keys, select, rerank = (float(out[i]) for i in range(6))
        return {"avg_centroid_search_ms": coarse / nq, "avg_signature_calc_ms": sig / nq,
                "avg_bucket_lookup_ms": plan / nq, "avg_distance_calc_ms": (keys + rerank) / nq,
                "avg_candidate_sort_ms": select / nq, "query_count": nq,
                "stage_ms": {"coarse": coarse, "signatures": sig, "plan": plan, "keys": keys, "select": select,
                             "rerank": rerank},
                "profiled_calls": int(out[6])}

    OPTIONS = {"sample_div": 2, "sampled_min_queries": 3}

    def set_option(self, name: str, value: int) -> None:
        """Query options (ann_ivf_set_option): "sample_div" (the sampled bars score the first
        ceil(size / div) rows of each list), "sampled_min_queries" (batch size from which the tensor-core
        forms take the sampled path). Neither changes results."""
        if name not in self.OPTIONS:
            raise RuntimeError(f"unknown option {name!r}")
        _lib.check(self._lib.ann_ivf_set_option(self._h, self.OPTIONS[name], int(value)))

    def get_kernel_times(self) -> dict:
        """Single-kernel CUDA-event times of the profiled calls (totals): {slot: {"ms", "launches"}} for
        the list-keys kernel ("keys"), the sampled bars ("bars"), the best-R selection ("select") and the
        exact re-rank ("rerank")."""
        out = (ctypes.c_double * 8)()
        _lib.check(self._lib.ann_ivf_kernel_profile(self._h, out))
        return {name: {"ms": float(out[i]), "launches": int(out[4 + i])}
                for i, name in enumerate(("keys", "bars", "select", "rerank"))}

    def reset_profile_results(self) -> None:
        _lib.check(self._lib.ann_ivf_reset_profile(self._h))

    # ---- batched API -----------------------------------------------------------------------------
    @property
    def dim(self) -> int:
        return self._dim

    @property
    def ntotal(self) -> int:
        return self._n

    def search(self, queries, k: int, n_probes: int = 0, n_probe_clusters: int = 8, refine_r: int = -1,
               max_candidates: int | None = None, mode: str | None = None, workspace=None, out_ids=None,
               out_dists=None, stream=None, with_dists: bool = True, shard: bool = False):
        """Top-k per query row: (ids int64 [nq, k], squared distances float32 [nq, k]).
        max_candidates: None = the mode's default (reference: the reference's cap; exact: none),
        -1 = the reference's cap, 0 = none, > 0 = that cap. shard: this index holds one rank's share of the
        lists (ShardedIVFIndex); a query short of k candidates returns what it has (-1 padded).
        out_ids / out_dists: where the results go -- device tensors for device queries, or for host queries
        host arrays (numpy or CPU torch, C-contiguous [nq, k]; page-locked ones take a direct copy)."""
        if self._n == 0:
            raise RuntimeError("index not fitted")
        k = int(k)
        if k < 1:
            raise RuntimeError("k must be >= 1")
        mode = mode or self.mode
        if max_candidates is None:
            max_candidates = -1 if mode == "reference" else 0
        ws = workspace.handle if workspace is not None else None
        mode_v = _lib.MODES[mode] | (_lib.QUERY_SHARD if shard else 0)
        args = (int(n_probes), int(n_probe_clusters), int(refine_r), int(max_candidates), mode_v,
                int(self.num_threads))
        if _lib.is_torch(queries) and queries.is_cuda:
            import torch
            x = _lib.as_f32_2d(queries, "queries")
            if x.shape[1] != self._dim:
                raise RuntimeError("Query dimension mismatch")
            nq = x.shape[0]
            if out_ids is None:
                out_ids = torch.empty(nq, k, dtype=torch.int64, device=x.device)
            if out_dists is None and with_dists:
                out_dists = torch.empty(nq, k, dtype=torch.float32, device=x.device)
            _lib.check(self._lib.ann_ivf_query(self._h, ws, _lib.ptr(x), nq, x.stride(0), k, *args, _lib.MEM_DEVICE,
                                               _lib.ptr(out_ids), _lib.ptr(out_dists), _lib.stream_ptr(x, stream)))
            return out_ids, out_dists
        x = _lib.as_f32_2d(queries.numpy() if _lib.is_torch(queries) else queries, "queries")
        if x.shape[1] != self._dim:
            raise RuntimeError("Query dimension mismatch")
        nq = x.shape[0]
        ids = _host_out(out_ids, (nq, k), np.int64, "out_ids")
        dists = _host_out(out_dists, (nq, k), np.float32, "out_dists") if with_dists else None
        _lib.check(self._lib.ann_ivf_query(self._h, ws, _lib.ptr(x), nq, x.shape[1], k, *args, _lib.MEM_HOST,
                                           _lib.ptr(ids), _lib.ptr(dists), None))
        return ids, dists

    @property
    def ntotal(self) -> int:
        return self._n

    @property
    def dim(self) -> int:
        return self._dim

    @property
    def n_lists(self) -> int:
        return self._C

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ann_ivf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# the reference's class name
LSHIndex = IVFIndex
