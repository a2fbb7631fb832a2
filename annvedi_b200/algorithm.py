"""The competition plugin: ``Algorithm.fit / query / get_n_distances`` with scenarios.yaml routing.

Drop-in for the reference facade (algorithm.py:12-90) and its bundles
(competitors/linear/algorithm.py, competitors/ivf_lsh/algorithm.py): the harness
(orthogonal-competition/harness.py:141-176) constructs ``Algorithm()``, calls
``fit(train, **index_params)``, then ``query(q, k, **query_params)`` once per query, then
``get_n_distances()``.

Routing follows ``index_params['backend']`` (algorithm.py:23):

* ``linear`` (default) -> ``LinearIndex`` with the reference's ranking (identical ids);
* ``gpu_flat``         -> ``LinearIndex`` in exact mode (true top-k);
* ``ivf_lsh`` / ``ivf`` -> ``IVFIndex`` with the reference's query semantics (per-dimension SQ8
  IVF-LSH fork: n_tables, n_bits, n_clusters; n_probes, n_probe_clusters, refine_r);
* ``gpu_ivf_sq8``      -> ``IVFIndex`` in exact-selection mode (no candidate cap, full SQ8
  distances, exact FP32 re-rank).

``ds_size`` truncates the training set (algorithm.py:19-21). Backends outside this package's scope
(``lsh``, ``hnsw``, ``multiprobe``) raise NotImplementedError.
"""
from __future__ import annotations

import numpy as np

_OUT_OF_SCOPE = ("lsh", "hnsw", "multiprobe")


class Algorithm:
    def __init__(self):
        self._backend = "linear"
        self._index = None
        self._query_defaults: dict = {}

    def fit(self, train, **index_params) -> None:
        index_params = dict(index_params)
        ds_size = index_params.pop("ds_size", None)
        if ds_size is not None:
            train = train[: int(ds_size)]
        self._backend = str(index_params.pop("backend", "linear")).lower()
        device = int(index_params.pop("device", 0))
        if self._backend in ("linear", "gpu_flat"):
            from .linear import LinearIndex
            mode = "reference" if self._backend == "linear" else "exact"
            mode = str(index_params.get("mode", mode))
            metric = str(index_params.get("metric", "l2"))
            self._index = LinearIndex(device=device, metric=metric, mode=mode)
            self._index.fit(np.asarray(train, dtype=np.float32) if not hasattr(train, "is_cuda") else train)
        elif self._backend in ("ivf_lsh", "ivf", "gpu_ivf_sq8"):
            from .ivf import IVFIndex
            exact = self._backend == "gpu_ivf_sq8"
            self._index = IVFIndex(device=device, mode="exact" if exact else "reference",
                                   num_threads=int(index_params.get("num_threads", 0)) or None)
            n_tables = int(index_params.get("n_tables", 1 if exact else 10))
            n_bits = int(index_params.get("n_bits", 0 if exact else 8))
            n_clusters = int(index_params.get("n_clusters", 256))
            self._index.fit(train, n_tables=n_tables, n_bits=n_bits, n_clusters=n_clusters,
                            kmeans_iters=int(index_params.get("kmeans_iters", 15)))
            for key in ("n_probes", "n_probe_clusters", "refine_r", "max_candidates"):
                if key in index_params:
                    self._query_defaults[key] = int(index_params[key])
        elif self._backend in _OUT_OF_SCOPE:
            raise NotImplementedError(f"backend {self._backend!r} is not part of the GPU search path")
        else:
            raise ValueError(f"unknown backend {self._backend!r}")

    def query(self, query, k: int, **query_params) -> np.ndarray:
        if self._index is None:
            raise RuntimeError("index not fitted")
        if self._backend in ("linear", "gpu_flat"):
            return self._index.query(query, k)
        p = dict(self._query_defaults)
        p.update({key: int(v) for key, v in query_params.items()})
        return self._index.query(query, k, n_probes=p.get("n_probes", 0),
                                 n_probe_clusters=p.get("n_probe_clusters", 8),
                                 refine_r=p.get("refine_r", -1),
                                 max_candidates=p.get("max_candidates", -1 if self._backend != "gpu_ivf_sq8" else 0))

    def query_batch(self, queries, k: int, **query_params):
        """Batched form (not part of the harness contract): ids [nq, k]."""
        if self._backend in ("linear", "gpu_flat"):
            return self._index.search(queries, k)[0]
        p = dict(self._query_defaults)
        p.update({key: int(v) for key, v in query_params.items()})
        return self._index.search(queries, k, **p)[0]

    def get_n_distances(self) -> int:
        if self._index is None:
            return 0
        return int(self._index.total_distances_count())
