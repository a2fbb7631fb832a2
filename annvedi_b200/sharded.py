"""Sharding over the ranks of a process group: an index larger than one GPU.

Row sharding of the exact linear scan (ShardedLinearIndex) and list sharding of the IVF index
(ShardedIVFIndex, below).

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


def assign_lists(sizes, world: int):
    """Owner rank of every list: lists by decreasing size (ties by lower id), each to the rank with the
    fewest rows so far (ties by lower rank) -- balanced rows, the same on every rank."""
    import numpy as np
    sizes = np.asarray(sizes, np.int64)
    owner = np.empty(len(sizes), np.int64)
    load = np.zeros(world, np.int64)
    for l in np.lexsort((np.arange(len(sizes)), -sizes)):
        r = int(np.argmin(load))
        owner[l] = r
        load[r] += sizes[l]
    return owner


class ShardedIVFIndex:
    """The IVF index with its inverted lists split over the ranks of `group` (torch.distributed). Every rank
    keeps the whole coarse quantiser (all centroids) and the rows of its own lists (assign_lists), so all
    ranks rank the centroids alike and probe the same lists; each rank scores the probed lists it holds
    (exact SQ8 selection or a tensor-core form, no candidate cap, exact FP32 re-rank), maps its ids to the
    global numbering, and one all-gather + ann_merge_topk keep the best k by (distance, id) on every rank.

    The reference scans every row when a query's probed lists hold fewer than k rows
    (competitors/ivf_lsh/src/lsh_index_optimized.cpp:453-457). A shard cannot decide that alone (its share of
    the lists may hold none of a query's rows), so shards search with ANN_QUERY_SHARD and the rule is applied
    to the merged result: a query with fewer than k ids there had fewer than k candidates over all ranks,
    and every rank searches it again over every list -- which is every row.

    Each rank quantises its own rows (per-dimension SQ8 over its share), so the SQ8 keys, and with them
    the best R candidates of a query, can differ from a single index's; the exact re-rank then orders what
    each rank kept. With R at least a query's candidates the result equals the single index's exact top-k
    over its probed lists. `local` / `merge` exist so the exchange can be exercised on CPU ranks."""

    def __init__(self, group=None, device: int = 0, mode: str = "exact", local=None, merge=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.mode = mode
        if local is None:
            from .ivf import IVFIndex
            self.local = IVFIndex(device=device, mode="exact")
        else:
            self.local = local()
        self._merge = merge or (lambda d, i, k: merge_topk(d, i, k, "l2"))
        self.gids = None
        self.n_lists = 0

    def fit(self, data, centroids, assign) -> None:
        """data [n, dim] (every rank the whole base), the coarse quantiser centroids [C, dim] and each row's
        list assign [n]; this rank keeps the rows of its lists, in ascending global id."""
        import numpy as np
        a = np.asarray(assign.cpu() if hasattr(assign, "cpu") else assign).astype(np.int64)
        C = int(centroids.shape[0])
        owner = assign_lists(np.bincount(a, minlength=C), self.world)
        rows = np.nonzero(owner[a] == self.rank)[0]
        self.fit_shard(data[rows] if not hasattr(data, "cuda") else data[rows], rows, centroids, a[rows])

    def fit_shard(self, rows, gids, centroids, assign) -> None:
        import numpy as np
        self.gids = np.asarray(gids, np.int64)
        self.n_lists = int(centroids.shape[0])
        self.local.fit(rows, 1, 0, self.n_lists, centroids=centroids, assign=np.asarray(assign, np.int32))

    def _search_local(self, queries, k, npc, refine_r):
        import torch
        ids, d = self.local.search(queries, k, 0, npc, refine_r, max_candidates=0, mode=self.mode, shard=True)
        ids, d = torch.as_tensor(ids), torch.as_tensor(d)
        g = torch.as_tensor(self.gids, device=ids.device)
        gid = torch.where(ids >= 0, g[ids.clamp(min=0)], ids)
        return gid, torch.where(ids >= 0, d, torch.full_like(d, float("inf")))

    def _exchange(self, d, ids, k):
        import torch
        import torch.distributed as dist
        parts_d = [torch.empty_like(d) for _ in range(self.world)]
        parts_i = [torch.empty_like(ids) for _ in range(self.world)]
        dist.all_gather(parts_d, d.contiguous(), group=self.group)
        dist.all_gather(parts_i, ids.contiguous(), group=self.group)
        return self._merge(torch.stack(parts_d, 1), torch.stack(parts_i, 1), k)

    def search(self, queries, k: int, n_probe_clusters: int = 8, refine_r: int = 300):
        """(ids [nq, k] int64, squared distances [nq, k] float32) over all ranks' lists; every rank calls it
        with the same queries and gets the same result."""
        import torch
        ids, d = self._search_local(queries, k, n_probe_clusters, refine_r)
        ids, d = self._exchange(d, ids, k)
        short = torch.nonzero((ids >= 0).sum(1) < min(k, self._n_total())).flatten()
        if short.numel() > 0:  # the same set on every rank: the merged results are identical
            q2 = queries[short.to(queries.device)] if hasattr(queries, "device") else queries[short.cpu().numpy()]
            i2, d2 = self._search_local(q2, k, self.n_lists, refine_r)
            i2, d2 = self._exchange(d2, i2, k)
            ids[short] = i2
            d[short] = d2
        return ids, d

    def _n_total(self) -> int:
        import torch
        import torch.distributed as dist
        if not hasattr(self, "_n_all"):
            dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
            t = torch.tensor([len(self.gids)], dtype=torch.int64, device=dev)
            dist.all_reduce(t, group=self.group)
            self._n_all = int(t.item())
        return self._n_all

    def total_distances_count(self) -> int:
        """Distances computed over all ranks (a collective: every rank calls it)."""
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([int(self.local.total_distances_count())], dtype=torch.int64, device=dev)
        dist.all_reduce(t, group=self.group)
        return int(t.item())
