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
