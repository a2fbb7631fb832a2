"""The multi-rank bench path on CPU: two `gloo` ranks (world_size 2) as torchrun would start them, each
with its own batch and its own step time; the whole-job figure counts every rank's queries over the
slowest rank's time, and every rank takes the same collective steps."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_setup("gloo")
    try:
        ms = 100.0 * (r + 1)  # rank 1 is the slower one
        bench.barrier(w)
        out[r] = (bench.max_over_ranks(ms, w), bench.whole_job_qps(1000, 4, ms, w))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
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
    assert res[0] == res[1]
    slowest, qps = res[0]
    assert slowest == 200.0
    assert qps == pytest.approx(2 * 1000 * 4 / 0.2)
