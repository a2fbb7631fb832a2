"""List sharding of the IVF index on two `gloo` ranks (world_size 2): the lists are split over the ranks, each
rank searches the probed lists it holds, the ranks' lists are all-gathered and merged, and every rank ends
with the single index's result -- including queries whose probed lists hold fewer than k rows, which the
reference widens to every row (competitors/ivf_lsh/src/lsh_index_optimized.cpp:453-457). Each rank's index is
a numpy stand-in of the GPU IVF index's exact semantics with the whole base's re-rank (R covering every
candidate), so this checks the list assignment, the id map, the gather layout, the every-row rule over the
merged result and the collective steps."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from annvedi_b200.sharded import assign_lists


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _IVFBrute:
    """Exact top-k by (squared distance, id) over the rows of the npc lists nearest to the query (FP64
    centroid ranking, ties by the lower list); with shard=False a query short of k candidates takes every
    row, as the reference does."""

    def __init__(self):
        self.x = self.assign = self.cent = None
        self.nd = 0

    def fit(self, rows, n_tables, n_bits, n_clusters, centroids=None, assign=None):
        self.x = np.asarray(rows, np.float64)
        self.assign = np.asarray(assign, np.int64)
        self.cent = np.asarray(centroids, np.float64)
        assert self.cent.shape[0] == n_clusters

    def search(self, q, k, n_probes, npc, refine_r, max_candidates=0, mode="exact", shard=False):
        import torch
        q = np.asarray(q, np.float64)
        ids = np.full((q.shape[0], k), -1, np.int64)
        dd = np.full((q.shape[0], k), np.inf, np.float32)
        for i in range(q.shape[0]):
            cd = ((self.cent - q[i]) ** 2).sum(1)
            probes = np.lexsort((np.arange(len(cd)), cd))[:npc]
            cand = np.nonzero(np.isin(self.assign, probes))[0]
            if len(cand) < k and not shard:
                cand = np.arange(self.x.shape[0])
            self.nd += len(cand)
            d = ((self.x[cand] - q[i]) ** 2).sum(1)
            o = np.lexsort((cand, d))[:k]
            ids[i, :len(o)] = cand[o]
            dd[i, :len(o)] = d[o]
        return torch.from_numpy(ids), torch.from_numpy(dd)

    def total_distances_count(self):
        return self.nd


def _merge_np(d, i, k):
    import torch
    d, i = d.numpy(), i.numpy()
    out_i = np.full((d.shape[0], k), -1, np.int64)
    out_d = np.full((d.shape[0], k), np.inf, np.float32)
    for q in range(d.shape[0]):
        dd, ii = d[q].ravel(), i[q].ravel()
        ok = ii >= 0
        o = np.lexsort((ii[ok], dd[ok]))[:k]
        out_i[q, :len(o)] = ii[ok][o]
        out_d[q, :len(o)] = dd[ok][o]
    return torch.from_numpy(out_i), torch.from_numpy(out_d)


def _data():
    rng = np.random.default_rng(3)
    C = 24
    sizes = np.array([60, 45, 30, 30, 20, 12, 9, 7] + [3] * 16)  # a few large lists, many tiny ones
    assign = np.repeat(np.arange(C), sizes)
    rng.shuffle(assign)
    cent = rng.standard_normal((C, 6)).astype(np.float32)
    base = (cent[assign] + 0.3 * rng.standard_normal((len(assign), 6))).astype(np.float32)
    # queries near tiny lists: 2 probes hold fewer than k = 10 rows there (the every-row rule)
    q = (cent[rng.integers(8, C, 9)] + 0.05 * rng.standard_normal((9, 6))).astype(np.float32)
    q = np.concatenate([q, (cent[:3] + 0.05).astype(np.float32)])
    return base, cent, assign, q


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import datetime
    import torch.distributed as dist
    from annvedi_b200.sharded import ShardedIVFIndex
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        base, cent, assign, q = _data()
        ix = ShardedIVFIndex(local=_IVFBrute, merge=_merge_np)
        ix.fit(base, cent, assign)
        ids, d = ix.search(q, 10, n_probe_clusters=2, refine_r=1000)
        ids4, d4 = ix.search(q, 10, n_probe_clusters=4, refine_r=1000)
        out[rank] = (ids.numpy(), d.numpy(), ids4.numpy(), d4.numpy(), ix.gids.copy(), ix.total_distances_count())
    finally:
        dist.destroy_process_group()


def test_list_assignment_balances_rows():
    sizes = np.array([100, 80, 60, 50, 40, 10, 5, 5])
    owner = assign_lists(sizes, 3)
    load = np.bincount(owner, weights=sizes, minlength=3)
    assert load.max() - load.min() <= sizes.max()
    np.testing.assert_array_equal(owner, assign_lists(sizes, 3))
    assert set(owner.tolist()) == {0, 1, 2}


def test_two_ranks_equal_the_single_ivf_index():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    base, cent, assign, q = _data()
    single = _IVFBrute()
    single.fit(base, 1, 0, len(cent), centroids=cent, assign=assign)
    wi, wd = single.search(q, 10, 0, 2, 1000)
    wi4, wd4 = single.search(q, 10, 0, 4, 1000)
    # some queries took the every-row rule in the single index
    probes = [np.lexsort((np.arange(len(cent)), ((cent.astype(np.float64) - qq) ** 2).sum(1)))[:2] for qq in q]
    assert any(np.isin(assign, p).sum() < 10 for p in probes)
    for r in range(world):
        ids, d, ids4, d4, gids, nd = res[r]
        np.testing.assert_array_equal(ids, wi.numpy())
        np.testing.assert_array_equal(d, wd.numpy())
        np.testing.assert_array_equal(ids4, wi4.numpy())
        np.testing.assert_array_equal(d4, wd4.numpy())
    # the ranks' rows partition the base
    allg = np.sort(np.concatenate([res[r][4] for r in range(world)]))
    np.testing.assert_array_equal(allg, np.arange(base.shape[0]))
    assert res[0][5] == res[1][5] > 0
