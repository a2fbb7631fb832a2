"""The serving loop (annvedi_b200.serving): continuous batching over two resident indexes.

1. Each request's result is the same alone (one call of the index for that request only) and in the
   mix (batched with whatever else was queued, on concurrent workers): identical ids and distances for
   the exact tensor-core form and for the IVF lists on the tensor cores; for the IVF-SQ8 form too (its
   batched and per-query kernels share one arithmetic), except that a differing id is allowed where
   both ids' distances tie within 1e-5 relative.
2. Admission by free HBM: with the reserve set so that only a few queries' scratch fits, batches are
   cut down to what fits and every request still completes.
"""
import numpy as np
import pytest

from annvedi_b200 import synth

pytestmark = pytest.mark.gpu


def _traffic(rng, n_req, dims, routes, cap=64, p=0.1, qpool=None, shares=(0.7, 0.3)):
    out = []
    t = 0.0
    cum = np.cumsum(shares)
    for i in range(n_req):
        route = routes[int(np.searchsorted(cum, rng.random() * cum[-1], side="right"))]
        b = int(min(cap, rng.geometric(p)))
        rows = rng.integers(0, qpool[route].shape[0], b)
        t += rng.exponential(1.0 / 20000)
        out.append((t, route, qpool[route][rows]))
    return out


@pytest.fixture(scope="module")
def two_indexes():
    import torch
    from annvedi_b200.ivf import IVFIndex
    from annvedi_b200.linear import LinearIndex
    wa = synth.mixture(300_000, 96, 512, c=256, sigma=0.35, seed=3, metric="l2")
    flat = LinearIndex(device=0, metric="l2", mode="exact")
    flat.fit(torch.from_numpy(wa.base).cuda())
    wb = synth.zipf_mixture(120_000, 64, 512, c=128, sigma=0.3, lo=20, hi=8000, seed=4)
    ivf = IVFIndex(device=0, mode="exact")
    ivf.fit(torch.from_numpy(wb.base).cuda(), 1, 0, 128, centroids=wb.centres)
    return flat, wa, ivf, wb


def test_results_alone_equal_results_in_the_mix(cuda, two_indexes):
    import torch
    from annvedi_b200 import serving
    from tests.helpers import assert_ids_equal_up_to_ties
    flat, wa, ivf, wb = two_indexes
    routes = [serving.tc_route("exact", flat, refine_r=400),
              serving.ivf_route("ivf_tc", ivf, 8, 300, max_list=8000, mode="tc"),
              serving.ivf_route("ivf_sq8", ivf, 8, 300, max_list=8000, mode="exact")]
    rng = np.random.default_rng(0)
    qpool = {"exact": wa.queries, "ivf_tc": wb.queries, "ivf_sq8": wb.queries}
    traffic = _traffic(rng, 180, None, ["exact", "ivf_tc", "ivf_sq8"], qpool=qpool, shares=(0.3, 0.35, 0.35))
    srv = serving.Server(routes, workers=3, max_batch=1024).start()
    try:
        reqs = serving.poisson_run(srv, traffic, k=100)
    finally:
        srv.stop()
    st = srv.stats()
    assert st["requests"] == len(traffic)
    assert max(r.batch_queries - r.queries.shape[0] for r in reqs) > 0, "no request was batched with another"
    seen = set()
    for req in reqs:
        seen.add(req.route)
        x = torch.from_numpy(req.queries).cuda()
        if req.route == "exact":
            ids, d = flat.search_tc(x, 100, refine_r=400)
        else:
            ids, d = ivf.search(x, 100, 0, 8, 300, max_candidates=0, mode="tc" if req.route == "ivf_tc" else "exact")
        ids, d = ids.cpu().numpy(), d.cpu().numpy()
        if req.route == "ivf_sq8":
            assert_ids_equal_up_to_ties(wb.base, req.queries, req.ids, ids, rtol=1e-5, err_msg="ivf_sq8")
            same = req.ids == ids
            np.testing.assert_array_equal(req.dists[same], d[same])
        else:
            np.testing.assert_array_equal(req.ids, ids, err_msg=req.route)
            np.testing.assert_array_equal(req.dists, d, err_msg=req.route)
    assert seen == {"exact", "ivf_tc", "ivf_sq8"}


def test_sq8_keys_do_not_depend_on_the_batch(cuda, two_indexes):
    """The IVF-SQ8 exact form: 300 queries at once (list-major batched kernel) and one at a time
    (per-query kernel) give the same ids and distances."""
    _, _, ivf, wb = two_indexes
    q = wb.queries[:300]
    ids_b, d_b = ivf.search(q, 100, 0, 8, 300, max_candidates=0)
    for i in range(0, 300, 7):
        ids_1, d_1 = ivf.search(q[i:i + 1], 100, 0, 8, 300, max_candidates=0)
        np.testing.assert_array_equal(ids_1[0], ids_b[i], err_msg=f"query {i}")
        np.testing.assert_array_equal(d_1[0], d_b[i], err_msg=f"query {i}")


def test_admission_cuts_batches_to_free_hbm(cuda, two_indexes):
    import torch
    from annvedi_b200 import serving
    flat, wa, _, _ = two_indexes
    base_route = serving.flat_route("exact", flat)
    per_q = 256 << 20  # pretend each query needs 256 MB of fresh scratch
    route = serving.Route("exact", base_route.dim, base_route.search, lambda nq: nq * per_q)
    free, _ = torch.cuda.mem_get_info(0)
    reserve = free - 3 * per_q - (64 << 20)  # room for about three queries' scratch
    srv = serving.Server([route], workers=1, max_batch=64, hbm_reserve=reserve).start()
    try:
        reqs = [srv.submit("exact", wa.queries[i:i + 2], 10) for i in range(0, 40, 2)]
        for r in reqs:
            assert r.wait(60)
    finally:
        srv.stop()
    assert all(r.ids is not None and r.ids.shape == (2, 10) for r in reqs)
    assert max(b[1] for b in srv.batches) <= 3 * 2
    ids, _ = flat.search(wa.queries[:40], 10, mode="exact")
    np.testing.assert_array_equal(np.concatenate([r.ids for r in reqs]), ids)
