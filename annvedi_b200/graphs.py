"""CUDA graphs for fixed-shape searches: a query batch of a fixed size captured once, replayed per batch.

At one to a few queries per call a search is a handful of short kernels, and launching them costs a
visible share of the call. `GraphedSearch` captures one call of a search that makes no host
synchronisation -- the plain exact scan (`LinearIndex.search`, mode "exact") and the IVF-SQ8 query for
batches of fewer than 32 queries (`IVFIndex.search`, mode "exact"; larger batches group their (query,
list) pairs on the host) -- and replays it for each new batch copied into its input buffer.

The captured launches bake in the addresses of their scratch memory, so a graphed search owns a
workspace of its own: one eager call before the capture sizes it, and nothing else may use it. The
flat index's distance counter is kept on the host and does not advance on replays; the IVF counter is
kept on the device and does.
"""
from __future__ import annotations

from typing import Callable


class GraphedSearch:
    """search(queries_dev, out_ids, out_dists, stream, workspace) captured for `batch` queries of `dim`
    floats; `__call__(queries)` copies them into the captured input and replays the graph on the current
    stream, returning the captured output tensors (overwritten by the next call)."""

    def __init__(self, search: Callable, batch: int, dim: int, k: int, device: int = 0, warmup: int = 2):
        import torch
        from .linear import Workspace
        dev = f"cuda:{device}"
        self.ws = Workspace(device)
        self.x = torch.zeros(batch, dim, dtype=torch.float32, device=dev)
        self.ids = torch.empty(batch, k, dtype=torch.int64, device=dev)
        self.dists = torch.empty(batch, k, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.Stream(device=dev)
        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):  # sizes the workspace and runs one-time set-up outside the capture
                search(self.x, self.ids, self.dists, self.stream, self.ws)
        self.stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            search(self.x, self.ids, self.dists, self.stream, self.ws)
        self.batch = batch

    def __call__(self, queries):
        if queries.shape[0] != self.batch:
            raise RuntimeError(f"graphed search of {self.batch} queries called with {queries.shape[0]}")
        self.x.copy_(queries, non_blocking=True)
        self.graph.replay()
        return self.ids, self.dists


def flat_exact(index, batch: int, k: int, device: int = 0) -> GraphedSearch:
    """The plain exact scan of a LinearIndex for `batch` queries, captured."""
    def search(x, ids, dists, stream, ws):
        index.search(x, k, mode="exact", workspace=ws, out_ids=ids, out_dists=dists, stream=stream)
    return GraphedSearch(search, batch, index.dim, k, device)


def ivf_exact(index, batch: int, k: int, n_probe_clusters: int, refine_r: int, device: int = 0) -> GraphedSearch:
    """The exact-selection IVF-SQ8 query of an IVFIndex (no candidate cap) for `batch` < 32 queries, captured."""
    if batch >= 32:
        raise ValueError("IVF batches of 32 or more queries synchronise with the host (list grouping)")

    def search(x, ids, dists, stream, ws):
        index.search(x, k, 0, n_probe_clusters, refine_r, max_candidates=0, mode="exact", workspace=ws,
                     out_ids=ids, out_dists=dists, stream=stream)
    return GraphedSearch(search, batch, index.dim, k, device)
