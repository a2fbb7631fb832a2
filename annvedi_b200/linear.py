"""Linear (brute-force) index on the GPU: the drop-in for linear_ann_cpp.LinearIndex.

``LinearIndex`` keeps the reference's surface (competitors/linear/src/linear_index.cpp:126-131):
``fit(float32[N, d])``, ``query(float32[d], k) -> int64[k]``, ``total_distances_count()``, with
the same errors (RuntimeError for a non-2-D fit, a query before fit, or a query of the wrong
shape; linear_index.cpp:75-76, 91-96) and the same k clipping to N (:110).

Two semantics are available:

* ``"reference"`` (default for the drop-in): the reference's own ranking, including its 64-entry
  early-abandon heap (linear_index.cpp:27-60) -- identical ids to linear_ann_cpp on the same input;
* ``"exact"``: the true top-k by (squared distance, id) -- what ``search`` uses for benchmarks.

``search(queries, k)`` is the batched entry point: numpy inputs run synchronously through host
staging, torch CUDA tensors run asynchronously on the current stream and return device tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class Workspace:
    """Device scratch for one stream of concurrent queries (include/annvedi_b200.h)."""

    def __init__(self, device: int = 0):
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.ann_workspace_create(ctypes.byref(h), device))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def nbytes(self) -> int:
        return int(_lib.load().ann_workspace_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().ann_workspace_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LinearIndex:
    def __init__(self, device: int = 0, metric: str = "l2", mode: str = "reference"):
        self._lib = _lib.load()
        if metric not in _lib.METRICS:
            raise ValueError(f"unknown metric {metric!r}")
        if mode not in _lib.MODES:
            raise ValueError(f"unknown mode {mode!r}")
        h = ctypes.c_void_p()
        _lib.check(self._lib.ann_flat_create(ctypes.byref(h), device))
        self._h = h
        self.device = device
        self.metric = metric
        self.mode = mode
        self._dim = 0
        self._n = 0

    # ---- reference surface -------------------------------------------------------------------
    def fit(self, arr) -> None:
        if _lib.is_torch(arr):
            x = _lib.as_f32_2d(arr, "Input")
            mem = _lib.MEM_DEVICE if x.is_cuda else _lib.MEM_HOST
            ld = x.stride(0)
        else:
            a = np.asarray(arr)
            if a.ndim != 2:
                raise RuntimeError("Input must be a 2-D array")
            x = np.ascontiguousarray(a, dtype=np.float32)
            mem = _lib.MEM_HOST
            ld = x.shape[1]
        n, d = x.shape
        if n == 0 or d == 0:
            raise RuntimeError("Input must be a non-empty 2-D array")
        st = _lib.stream_ptr(x) if mem == _lib.MEM_DEVICE else None
        _lib.check(self._lib.ann_flat_fit(self._h, _lib.ptr(x), n, d, ld, _lib.METRICS[self.metric], mem, st))
        if mem == _lib.MEM_DEVICE:
            import torch
            torch.cuda.current_stream(x.device).synchronize()
        self._n, self._dim = n, d

    def query(self, q, k: int) -> np.ndarray:
        if self._n == 0:
            raise RuntimeError("index not fitted")
        qa = np.asarray(q.cpu() if _lib.is_torch(q) else q)
        if qa.ndim != 1 or qa.shape[0] != self._dim:
            raise RuntimeError(f"query must be a 1-D vector of length {self._dim}")
        ids, _ = self.search(qa.reshape(1, -1), k)
        return ids[0]

    def total_distances_count(self) -> int:
        return int(self._lib.ann_flat_total_distances(self._h))

    # ---- batched API ---------------------------------------------------------------------------
    def search(self, queries, k: int, mode: str | None = None, workspace: Workspace | None = None,
               out_ids=None, out_dists=None, stream=None, with_dists: bool = True):
        """Top-k of each query row. Returns (ids int64 [nq, k'], values float32 [nq, k']) with
        k' = min(k, N); values are squared distances (inner products for metric "ip") in exact
        mode and the reference's ranking values in reference mode."""
        if self._n == 0:
            raise RuntimeError("index not fitted")
        if int(k) < 1:
            raise RuntimeError("k must be >= 1")
        mode = mode or self.mode
        kk = min(int(k), self._n)
        ws = workspace.handle if workspace is not None else None
        if _lib.is_torch(queries) and queries.is_cuda:
            import torch
            x = _lib.as_f32_2d(queries, "queries")
            if x.shape[1] != self._dim:
                raise RuntimeError(f"queries must have {self._dim} columns")
            nq = x.shape[0]
            if out_ids is None:
                out_ids = torch.empty(nq, kk, dtype=torch.int64, device=x.device)
            if out_dists is None and with_dists:
                out_dists = torch.empty(nq, kk, dtype=torch.float32, device=x.device)
            st = _lib.stream_ptr(x, stream)
            _lib.check(self._lib.ann_flat_query(self._h, ws, _lib.ptr(x), nq, x.stride(0), kk,
                                                _lib.MODES[mode], _lib.MEM_DEVICE, _lib.ptr(out_ids),
                                                _lib.ptr(out_dists), st))
            return out_ids, out_dists
        x = _lib.as_f32_2d(queries.numpy() if _lib.is_torch(queries) else queries, "queries")
        if x.shape[1] != self._dim:
            raise RuntimeError(f"queries must have {self._dim} columns")
        nq = x.shape[0]
        ids = np.empty((nq, kk), np.int64)
        dists = np.empty((nq, kk), np.float32) if with_dists else None
        _lib.check(self._lib.ann_flat_query(self._h, ws, _lib.ptr(x), nq, x.shape[1], kk, _lib.MODES[mode],
                                            _lib.MEM_HOST, _lib.ptr(ids), _lib.ptr(dists), None))
        return ids, dists

    def search_tc(self, queries, k: int, refine_r: int = -1, workspace: Workspace | None = None, out_ids=None,
                  out_dists=None, stream=None, with_dists: bool = True):
        """Tensor-core form: BF16 tcgen05 scores for every row, the best R = max(k, refine_r > 0 ?
        refine_r : 4k) per query re-ranked with exact FP32 distances (inner products for metric "ip")."""
        if self._n == 0:
            raise RuntimeError("index not fitted")
        k = int(k)
        if k < 1:
            raise RuntimeError("k must be >= 1")
        kk = min(k, self._n)
        ws = workspace.handle if workspace is not None else None
        if _lib.is_torch(queries) and queries.is_cuda:
            import torch
            x = _lib.as_f32_2d(queries, "queries")
            nq = x.shape[0]
            if out_ids is None:
                out_ids = torch.empty(nq, kk, dtype=torch.int64, device=x.device)
            if out_dists is None and with_dists:
                out_dists = torch.empty(nq, kk, dtype=torch.float32, device=x.device)
            _lib.check(self._lib.ann_flat_query_tc(self._h, ws, _lib.ptr(x), nq, x.stride(0), kk, int(refine_r),
                                                   _lib.MEM_DEVICE, _lib.ptr(out_ids), _lib.ptr(out_dists),
                                                   _lib.stream_ptr(x, stream)))
            return out_ids, out_dists
        x = _lib.as_f32_2d(queries.numpy() if _lib.is_torch(queries) else queries, "queries")
        nq = x.shape[0]
        ids = np.empty((nq, kk), np.int64)
        dists = np.empty((nq, kk), np.float32) if with_dists else None
        _lib.check(self._lib.ann_flat_query_tc(self._h, ws, _lib.ptr(x), nq, x.shape[1], kk, int(refine_r),
                                               _lib.MEM_HOST, _lib.ptr(ids), _lib.ptr(dists), None))
        return ids, dists

    def set_query_tile(self, tile: int = 0) -> None:
        """Queries per CTA of the exact scan's staged form (ANN_FLAT_OPT_QUERY_TILE): 8, 16 or 32, or 0 to pick
        by the batch size. Results are the same for 8, 16 and 32; the tile changes speed only."""
        _lib.check(self._lib.ann_flat_set_option(self._h, 1, int(tile)))

    def set_tc_precision(self, precision: str = "bf16") -> None:
        """Element kind of search_tc / scores_tc: "bf16" (default) or "e4m3" (scaled FP8: twice the tensor
        rate, a coarser key; pair it with a deeper refine_r)."""
        kinds = {"bf16": 0, "e4m3": 1}
        if precision not in kinds:
            raise ValueError(f"unknown precision {precision!r}")
        _lib.check(self._lib.ann_flat_set_tc_precision(self._h, kinds[precision]))

    def scores_tc(self, queries):
        """Diagnostic: the tensor-core key matrix [nq, N] (device tensor in, device tensor out)."""
        import torch
        x = _lib.as_f32_2d(queries, "queries")
        out = torch.empty(x.shape[0], self._n, dtype=torch.float32, device=x.device)
        _lib.check(self._lib.ann_flat_scores_tc(self._h, _lib.ptr(x), x.shape[0], x.stride(0), _lib.ptr(out),
                                                _lib.stream_ptr(x)))
        return out

    # ---- profiling (CUDA events on the query stream) ---------------------------------------
    def set_profiling(self, enable: bool = True) -> None:
        _lib.check(self._lib.ann_flat_set_profiling(self._h, int(enable)))

    def get_profile_results(self) -> dict:
        out = (ctypes.c_double * 4)()
        _lib.check(self._lib.ann_flat_profile(self._h, out))
        return {"scan_ms": out[0], "merge_ms": out[1], "scan_launches": int(out[2]), "query_calls": int(out[3])}

    def get_stage_times(self) -> dict:
        """Every stage total: the exact scan's and the tensor-core search's (sample pass and bars, filter
        pass, selections, exact re-rank), with launch counts."""
        out = (ctypes.c_double * 10)()
        _lib.check(self._lib.ann_flat_profile_stages(self._h, out))
        return {"scan_ms": out[0], "merge_ms": out[1], "tc_sample_ms": out[2], "tc_filter_ms": out[3],
                "tc_select_ms": out[4], "rerank_ms": out[5], "scan_launches": int(out[6]),
                "tc_gemm_launches": int(out[7]), "tc_filter_launches": int(out[8]), "query_calls": int(out[9])}

    def reset_profile_results(self) -> None:
        _lib.check(self._lib.ann_flat_reset_profile(self._h))

    @property
    def ntotal(self) -> int:
        return self._n

    @property
    def dim(self) -> int:
        return self._dim

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ann_flat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
