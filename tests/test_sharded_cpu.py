"""Row sharding's exchange on two `gloo` ranks (world_size 2): each rank searches its rows, the ranks'
lists are all-gathered and merged, and every rank ends with the single-index result over all rows and
the summed distance counter. The per-rank search and the merge are numpy stand-ins for the GPU index
and ann_merge_topk (this checks the offsets, the gather layout and the collective steps)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Brute:
    """Exact top-k by (squared distance, id) over the rows it holds."""

    def __init__(self):
        self.x, self.nd = None, 0

    def fit(self, rows):
        self.x = np.asarray(rows, np.float64)

    def search(self, q, k, mode="exact"):
        import torch
        d = ((self.x[None, :, :] - np.asarray(q, np.float64)[:, None, :]) ** 2).sum(-1)
        self.nd += d.size
        ids = np.full((q.shape[0], k), -1, np.int64)
        dd = np.full((q.shape[0], k), np.inf, np.float32)
        for i in range(q.shape[0]):
            o = np.lexsort((np.arange(d.shape[1]), d[i]))[:k]
            ids[i, :len(o)] = o
            dd[i, :len(o)] = d[i, o]
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


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import datetime
    import torch.distributed as dist
    from annvedi_b200.sharded import ShardedLinearIndex
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(0)
        base = rng.standard_normal((301, 8)).astype(np.float32)
        base[150] = base[3]  # a tie across the shard boundary: the lower id wins
        q = rng.standard_normal((7, 8)).astype(np.float32)
        q[0] = base[3]
        ix = ShardedLinearIndex(local=_Brute, merge=_merge_np)
        ix.fit(base)
        ids, d = ix.search(q, 5)
        out[rank] = (ids.numpy(), d.numpy(), ix.total_distances_count(), ix.first)
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_the_single_index():
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
    rng = np.random.default_rng(0)
    base = rng.standard_normal((301, 8)).astype(np.float32)
    base[150] = base[3]
    q = rng.standard_normal((7, 8)).astype(np.float32)
    q[0] = base[3]
    want_i, want_d = _Brute(), None
    want_i.fit(base)
    wi, wd = want_i.search(q, 5)
    for r in range(world):
        ids, d, nd, first = res[r]
        np.testing.assert_array_equal(ids, wi.numpy())
        np.testing.assert_array_equal(d, wd.numpy())
        assert nd == 301 * 7
    assert res[0][3] == 0 and res[1][3] == 150
    assert res[0][0][0][0] == 3 and res[0][0][0][1] == 150  # the tie kept in id order
