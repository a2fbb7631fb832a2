"""The reference's GPU quantized-filter contestant (competitors/gpu_filter/algorithm.py:19-59) on this
library's kernels: the same class, methods, parameters (query parameter ``r``, default 500) and errors,
through the same five-function C ABI (include/annvedi_gpu_filter.h), served by libannvedi_b200.so.

fit() quantises the rows to per-dimension SQ8 on the GPU (the reference does it on the host); query()
scans every row's SQ8 key, keeps the r rows with the smallest (key, id), re-ranks them in FP32 and
returns the best k ids -- the reference's ids, with the re-rank on the GPU instead of the host.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class Algorithm:
    """GPU quantized filter with an exact FP32 re-rank of the best r SQ8 candidates."""

    def __init__(self):
        self._lib = _lib.load()
        self._handle = None

    def fit(self, train: np.ndarray, **index_params) -> None:
        x = np.ascontiguousarray(train, dtype=np.float32)
        if x.ndim != 2:
            raise RuntimeError("train must be a 2-D array")
        if self._handle:
            self._lib.gf_free(self._handle)
            self._handle = None
        n, dim = x.shape
        h = self._lib.gf_create(x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, dim)
        if not h:
            raise RuntimeError(self._lib.gf_last_error().decode(errors="replace"))
        self._handle = h

    def query(self, query: np.ndarray, k: int, **query_params) -> np.ndarray:
        if not self._handle:
            raise RuntimeError("index not fitted")
        r = int(query_params.get("r", 500))
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        out = np.empty(k, dtype=np.int64)
        got = self._lib.gf_query(self._handle, q.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), k, r,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        if got < 0:
            raise RuntimeError(self._lib.gf_last_error().decode(errors="replace"))
        return out[:got]

    def get_n_distances(self) -> int:
        return int(self._lib.gf_ndist(self._handle)) if self._handle else 0

    def __del__(self):
        if getattr(self, "_handle", None):
            self._lib.gf_free(self._handle)
            self._handle = None
