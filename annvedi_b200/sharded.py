"""Row sharding of the exact linear scan over the ranks of a process group: an index larger than one GPU.

Each rank holds the contiguous rows [n * r / W, n * (r + 1) / W) of the base (W ranks) and searches a
query batch against them (the exact scan or the tensor-core search with its exact FP32 re-rank); its
ids are offset by its first row. One all-gather exchanges the W lists of (distance, id) -- nq * k * 12
bytes per rank, 12 MB for 10,000 queries at k = 100 -- and `ann_merge_topk` keeps the best k by
(distance, id) on every rank. The result equals the single-index search over all rows: each row's
distance does not depend on the shard holding it, and the merge breaks ties by the lower id as the
single search does. The distance counter is summed over the ranks.

The reference's linear_index keeps its whole base in one process (competitors/linear/src/
linear_index.cpp:73-88); this is the exchange step such an index needs once its rows span several
GPUs. The reference's own ranking (the 64-entry early-abandon heap, mode "reference") depends on the
order the whole base is scanned in and is not sharded.
"""
from __future__ import annotations

from typing import Callable


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[first, last) rows of `rank`'s shard of n rows over `world` ranks."""
    return n * rank // world, n * (rank + 1) // world


def merge_topk(dists, ids, k: int, metric: str = "l2", stream=None):
    """Best k of per-part top-k lists on the GPU: dists / ids [nq, parts, k] CUDA tensors (float32,
    int64; each part sorted, ids < 0 empty, parts in increasing id ranges) -> (ids [nq, k], dists [nq, k])."""
    import torch
    from . import _lib
    lib = _lib.load()
    nq, parts, kk = dists.shape
    if kk != k or tuple(ids.shape) != (nq, parts, k):
        raise RuntimeError("merge_topk: dists and ids must be [nq, parts, k]")
    d = dists.contiguous().to(torch.float32)
    i = ids.contiguous().to(torch.int64)
    out_i = torch.empty(nq, k, dtype=torch.int64, device=d.device)
    out_d = torch.empty(nq, k, dtype=torch.float32, device=d.device)
    _lib.check(lib.ann_merge_topk(_lib.ptr(d), _lib.ptr(i), nq, parts, k, _lib.METRICS[metric], _lib.ptr(out_i),
                                  _lib.ptr(out_d), _lib.stream_ptr(d, stream)))
    return out_i, out_d


class ShardedLinearIndex:
    """The exact linear scan with its rows split over the ranks of `group` (torch.distributed, NCCL for
    CUDA tensors). fit(data) takes the full base (each rank keeps its own rows) or fit_shard(rows, first,
    n) only this rank's rows; search(queries, k) must be called by every rank with the same queries and
    returns the same (ids, distances) on every rank.

    `local` (a factory of the per-rank index) and `merge` exist so that the exchange can be exercised on
    CPU ranks; by default the shard is a LinearIndex in exact mode and the merge is ann_merge_topk."""

    def __init__(self, group=None, device: int = 0, metric: str = "l2", local: Callable | None = None,
                 merge: Callable | None = None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.metric = metric
        if local is None:
            from .linear import LinearIndex
            self.local = LinearIndex(device=device, metric=metric, mode="exact")
        else:
            self.local = local()
        self._merge = merge or (lambda d, i, k: merge_topk(d, i, k, metric))
        self.first = 0
        self.n = 0

    def fit(self, data) -> None:
        n = data.shape[0]
        r0, r1 = shard_range(n, self.rank, self.world)
        self.fit_shard(data[r0:r1], r0, n)

    def fit_shard(self, rows, first: int, n: int) -> None:
        self.local.fit(rows)
        self.first, self.n = int(first), int(n)

    def search(self, queries, k: int, form: str = "exact", **kw):
        """(ids [nq, k] int64, distances [nq, k] float32) over all ranks' rows. form "exact": the exact
        scan; "tc": the tensor-core search with its exact FP32 re-rank (kw: refine_r)."""
        import torch
        import torch.distributed as dist
        if form == "tc":
            ids, d = self.local.search_tc(queries, k, **kw)
        else:
            ids, d = self.local.search(queries, k, mode="exact", **kw)
        ids = torch.as_tensor(ids)
        d = torch.as_tensor(d)
        ids = torch.where(ids >= 0, ids + self.first, ids)
        parts_d = [torch.empty_like(d) for _ in range(self.world)]
        parts_i = [torch.empty_like(ids) for _ in range(self.world)]
        dist.all_gather(parts_d, d.contiguous(), group=self.group)
        dist.all_gather(parts_i, ids.contiguous(), group=self.group)
        # part r of query q is rank r's list: [nq, W, k]
        return self._merge(torch.stack(parts_d, 1), torch.stack(parts_i, 1), k)

    def total_distances_count(self) -> int:
        """Distances computed over all ranks (a collective: every rank calls it)."""
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([int(self.local.total_distances_count())], dtype=torch.int64, device=dev)
        dist.all_reduce(t, group=self.group)
        return int(t.item())
