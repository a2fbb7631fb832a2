"""Row sharding on the GPU: the shards' lists merged by ann_merge_topk equal the single index over all
rows (ids and distances), for the exact scan (squared L2 and inner product) and the tensor-core form;
and ShardedLinearIndex over a one-rank NCCL process group (the collective path without ranks that wait
on each other on one GPU)."""
import datetime
import socket

import numpy as np
import pytest

from annvedi_b200 import synth

pytestmark = pytest.mark.gpu


def _shards(base, metric, parts):
    from annvedi_b200.linear import LinearIndex
    from annvedi_b200.sharded import shard_range
    out = []
    for r in range(parts):
        r0, r1 = shard_range(base.shape[0], r, parts)
        ix = LinearIndex(device=0, metric=metric, mode="exact")
        ix.fit(base[r0:r1])
        out.append((r0, ix))
    return out


@pytest.mark.parametrize("metric,form,parts", [("l2", "exact", 2), ("ip", "exact", 3), ("l2", "tc", 2)])
def test_merged_shards_equal_the_full_index(cuda, metric, form, parts):
    import torch
    from annvedi_b200.linear import LinearIndex
    from annvedi_b200.sharded import merge_topk
    w = synth.mixture(60000, 96, 64, c=64, sigma=0.4, seed=9, metric=metric)
    base = torch.from_numpy(w.base).cuda()
    q = torch.from_numpy(w.queries).cuda()
    base[40000] = base[7]  # a duplicate row in another shard: ties resolve to the lower id
    q[0] = base[7]
    k = 50
    full = LinearIndex(device=0, metric=metric, mode="exact")
    full.fit(base)
    run = (lambda ix: ix.search_tc(q, k, refine_r=400)) if form == "tc" else (lambda ix: ix.search(q, k, mode="exact"))
    fi, fd = run(full)
    ds, is_ = [], []
    for r0, ix in _shards(base, metric, parts):
        i, d = run(ix)
        is_.append(torch.where(i >= 0, i + r0, i))
        ds.append(d)
    mi, md = merge_topk(torch.stack(ds, 1), torch.stack(is_, 1), k, metric)
    np.testing.assert_array_equal(mi.cpu().numpy(), fi.cpu().numpy())
    np.testing.assert_array_equal(md.cpu().numpy(), fd.cpu().numpy())
    assert mi[0, 0].item() == 7 and mi[0, 1].item() == 40000


def test_sharded_index_over_nccl_one_rank(cuda):
    import torch
    import torch.distributed as dist
    from annvedi_b200.linear import LinearIndex
    from annvedi_b200.sharded import ShardedLinearIndex
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = synth.mixture(20000, 64, 32, c=32, sigma=0.4, seed=4, metric="l2")
        base = torch.from_numpy(w.base).cuda()
        q = torch.from_numpy(w.queries).cuda()
        ix = ShardedLinearIndex(device=0)
        ix.fit(base)
        ids, d = ix.search(q, 20)
        full = LinearIndex(device=0, metric="l2", mode="exact")
        full.fit(base)
        fi, fd = full.search(q, 20, mode="exact")
        np.testing.assert_array_equal(ids.cpu().numpy(), fi.cpu().numpy())
        np.testing.assert_array_equal(d.cpu().numpy(), fd.cpu().numpy())
        assert ix.total_distances_count() == 20000 * 32
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode,parts", [("exact", 2), ("tc", 3), ("tc_sq8", 2)])
def test_merged_list_shards_equal_the_full_ivf_index(cuda, mode, parts):
    """List sharding: each shard holds its lists' rows (and every centroid), searches with ANN_QUERY_SHARD;
    the merged lists equal the single IVF index when the re-rank covers every candidate."""
    import torch
    from annvedi_b200.ivf import IVFIndex
    from annvedi_b200.sharded import assign_lists, merge_topk
    from tests.helpers import assert_ids_equal_up_to_ties
    w = synth.zipf_mixture(6000, 64, 64, c=48, lo=20, hi=250, seed=17)
    k, npc, R = 50, 4, 1000
    full = IVFIndex(device=0, mode="exact")
    full.fit(w.base, 1, 0, 48, centroids=w.centres, assign=w.assign)
    fi, fd = full.search(w.queries, k, 0, npc, R, max_candidates=0, mode=mode)
    owner = assign_lists(np.bincount(w.assign, minlength=48), parts)
    ds, is_ = [], []
    for r in range(parts):
        rows = np.nonzero(owner[w.assign] == r)[0]
        ix = IVFIndex(device=0, mode="exact")
        ix.fit(w.base[rows], 1, 0, 48, centroids=w.centres, assign=w.assign[rows])
        i, d = ix.search(w.queries, k, 0, npc, R, max_candidates=0, mode=mode, shard=True)
        i = torch.from_numpy(i)
        g = torch.from_numpy(rows)
        is_.append(torch.where(i >= 0, g[i.clamp(min=0)], i).cuda())
        ds.append(torch.from_numpy(np.where(i.numpy() >= 0, d, np.inf).astype(np.float32)).cuda())
    mi, md = merge_topk(torch.stack(ds, 1), torch.stack(is_, 1), k)
    assert_ids_equal_up_to_ties(w.base, w.queries, mi.cpu().numpy(), fi, rtol=1e-6)
    np.testing.assert_allclose(md.cpu().numpy(), fd, rtol=1e-6, atol=1e-7)


def test_sharded_ivf_index_over_nccl_one_rank(cuda):
    """ShardedIVFIndex over a one-rank NCCL group, with queries whose probed list holds fewer than k rows:
    the every-row rule applied to the merged result gives the single index's answer."""
    import torch
    import torch.distributed as dist
    from annvedi_b200.ivf import IVFIndex
    from annvedi_b200.sharded import ShardedIVFIndex
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = synth.zipf_mixture(6000, 64, 40, c=48, lo=20, hi=250, seed=5)
        ix = ShardedIVFIndex(device=0, mode="exact")
        ix.fit(w.base, w.centres, w.assign)
        q = torch.from_numpy(w.queries).cuda()
        ids, d = ix.search(q, 50, n_probe_clusters=1, refine_r=1000)
        full = IVFIndex(device=0, mode="exact")
        full.fit(w.base, 1, 0, 48, centroids=w.centres, assign=w.assign)
        fi, fd = full.search(w.queries, 50, 0, 1, 1000, max_candidates=0)
        sizes = np.bincount(w.assign, minlength=48)
        assert (sizes < 50).any()
        np.testing.assert_array_equal(ids.cpu().numpy(), fi)
        np.testing.assert_allclose(d.cpu().numpy(), fd, rtol=1e-6, atol=1e-7)
        assert ix.total_distances_count() > 0
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
