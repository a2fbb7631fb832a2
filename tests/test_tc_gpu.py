"""The tensor-core (tcgen05, BF16 in / FP32 accumulate) scan through the C ABI.

1. The raw key matrix equals a torch FP32 computation on the same BF16-rounded operands (the only
   difference is summation order), including partial 128 x 256 tiles and padded dimensions.
2. The full form (BF16 keys -> best R -> exact FP32 re-rank) returns exact FP32 distances for its ids,
   and its ids match the FP64 exact top-k up to ties when the re-rank depth covers the BF16 error.
"""
import numpy as np
import pytest

from annvedi_b200 import synth

pytestmark = pytest.mark.gpu


def _ref_keys(base, queries, metric):
    import torch
    xb = base.to(torch.bfloat16).float()
    qb = queries.to(torch.bfloat16).float()
    dot = qb @ xb.T
    if metric == "ip":
        return -dot
    return (base.float() ** 2).sum(1)[None, :] - 2.0 * dot


@pytest.mark.parametrize("n,dim,nq", [(1000, 100, 200), (300, 64, 130), (5000, 384, 256), (4096, 768, 64)])
@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_tc_key_matrix(cuda, n, dim, nq, metric):
    import torch
    from annvedi_b200.linear import LinearIndex
    w = synth.flat_normal(n, dim, nq, seed=n + dim)
    base = torch.from_numpy(w.base).cuda()
    q = torch.from_numpy(w.queries).cuda()
    ix = LinearIndex(device=0, metric=metric, mode="exact")
    ix.fit(base)
    keys = ix.scores_tc(q)
    torch.cuda.synchronize()
    ref = _ref_keys(base, q, metric)
    err = (keys - ref).abs().max().item()
    assert err < 2e-4, f"max |key - ref| = {err}"


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_tc_search_matches_exact(cuda, metric):
    from oracle.refmod import exact_topk_f64
    from tests.helpers import check_exact_topk
    from annvedi_b200.linear import LinearIndex
    w = synth.mixture(30000, 256, 64, c=64, sigma=0.35, seed=11, metric=metric)
    ix = LinearIndex(device=0, metric=metric, mode="exact")
    ix.fit(w.base)
    ids, d = ix.search_tc(w.queries, 50, refine_r=1000)
    check_exact_topk(w.base, w.queries, ids, d, 50, metric=metric)
    # a shallow re-rank still finds nearly all of the exact top-k on this data
    ids2, _ = ix.search_tc(w.queries, 50, refine_r=100)
    gt, _ = exact_topk_f64(w.base, w.queries, 50, metric)
    assert np.mean([len(set(a) & set(b)) / 50 for a, b in zip(ids2, gt)]) > 0.97
    assert ix.total_distances_count() == 2 * 30000 * 64


def test_tc_device_and_host_agree(cuda):
    import torch
    from annvedi_b200.linear import LinearIndex
    w = synth.flat_normal(20000, 384, 40, seed=2)
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda())
    a, ad = ix.search_tc(torch.from_numpy(w.queries).cuda(), 20)
    torch.cuda.synchronize()
    b, bd = ix.search_tc(w.queries, 20)
    np.testing.assert_array_equal(a.cpu().numpy(), b)
    np.testing.assert_array_equal(ad.cpu().numpy(), bd)


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_tc_sampled_bar_path_is_exact(cuda, metric):
    """Bases of >= 262,144 rows take the sampled-bar path (sample pass, fast bar, filtered full pass,
    re-runs under the safe bar where needed); with R >= the BF16 error margin the result is the exact
    top-k."""
    import torch
    from tests.helpers import check_exact_topk
    from annvedi_b200.linear import LinearIndex
    w = synth.mixture(300_000, 64, 96, c=256, sigma=0.35, seed=21, metric=metric)
    ix = LinearIndex(device=0, metric=metric, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda())
    ids, d = ix.search_tc(torch.from_numpy(w.queries).cuda(), 20, refine_r=400)
    torch.cuda.synchronize()
    check_exact_topk(w.base, w.queries, ids.cpu().numpy(), d.cpu().numpy(), 20, metric=metric)


def _weyl_mult(n):
    """Row order of the BF16 base copy: position p holds row (p * g) mod n."""
    g = max(1, int(0.6180339887498949 * n))
    while np.gcd(g, n) != 1:
        g += 1
    return g


def test_tc_rerun_under_safe_bar_is_exact(cuda):
    """Queries whose nearest rows all sit at sampled positions of the base copy: the sample
    over-represents them, the fast bar (the ~134th best sampled key) lets fewer than R = 400 keys through
    over all rows, and the query is re-run under its safe bar. The result is still the exact top-k."""
    import torch
    from tests.helpers import check_exact_topk
    from annvedi_b200.linear import LinearIndex
    rng = np.random.default_rng(5)
    n, dim, R = 300_032, 64, 400
    g = _weyl_mult(n)
    full_tiles = n // 256
    stride = full_tiles // max(128, -(-16 * R // 256))  # sample: every stride-th 256-row tile
    tiles = np.arange(full_tiles // stride) * stride
    pos = (tiles[:, None] * 256 + np.arange(256)[None, :]).ravel()
    sampled_rows = (pos.astype(object) * g % n).astype(np.int64)
    base = rng.normal(size=(n, dim)).astype(np.float32)
    nclu, size = 8, 300
    centres = 4.0 * rng.normal(size=(nclu, dim)).astype(np.float32)
    rows = rng.choice(sampled_rows, nclu * size, replace=False).reshape(nclu, size)
    for i in range(nclu):
        base[rows[i]] = centres[i] + 0.05 * rng.normal(size=(size, dim))
    plain = rng.normal(size=(24, dim)).astype(np.float32)
    queries = np.concatenate([centres + 0.05 * rng.normal(size=(nclu, dim)), plain]).astype(np.float32)
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(base).cuda())
    ix.set_profiling(True)
    ix.reset_profile_results()
    ids, d = ix.search_tc(queries, 20, refine_r=R)
    st = ix.get_stage_times()
    check_exact_topk(base, queries, ids, d, 20)
    assert st["tc_gemm_launches"] >= 3, st  # sample, filter and at least one re-run


def _ref_keys_e4m3(base, queries, metric):
    """Keys from the same E4M3 operands: each row over its own scale max|x| / 448, rounded to nearest."""
    import torch

    def quant(x):
        s = x.abs().amax(1, keepdim=True) / 448.0
        s = torch.where(s > 0, s, torch.ones_like(s))
        xq = (x / s).clamp(-448.0, 448.0).to(torch.float8_e4m3fn).float()
        return xq, s[:, 0]

    xb, sb = quant(base)
    qb, sq = quant(queries)
    dot = (qb.double() @ xb.double().T) * sq[:, None].double() * sb[None, :].double()
    if metric == "ip":
        return -dot
    return (base.double() ** 2).sum(1)[None, :] - 2.0 * dot


@pytest.mark.parametrize("n,dim,nq", [(1000, 100, 200), (5000, 256, 130), (4096, 768, 64)])
@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_tc_e4m3_key_matrix(cuda, n, dim, nq, metric):
    """E4M3 operands (a scale per vector), FP32 accumulation: the keys equal an FP64 computation on the same
    E4M3-rounded operands up to the accumulation's rounding. The tensor cores' E4M3 accumulation keeps fewer
    bits than FP32 over long K (measured: 2e-5 of the key scale at K = 256, 1.6e-4 at K = 768), far below the
    E4M3 rounding of the operands themselves (2^-4 per element); the bound is 4e-4 of the key scale."""
    import torch
    from annvedi_b200.linear import LinearIndex
    w = synth.scaled_mixture(n, dim, nq, c=64, seed=n + dim)
    base = torch.from_numpy(w.base).cuda()
    q = torch.from_numpy(w.queries).cuda()
    ix = LinearIndex(device=0, metric=metric, mode="exact")
    ix.fit(base)
    ix.set_tc_precision("e4m3")
    keys = ix.scores_tc(q).double()
    torch.cuda.synchronize()
    ref = _ref_keys_e4m3(base, q, metric)
    scale = ref.abs().max().item()
    err = (keys - ref).abs().max().item()
    assert err < 4e-4 * scale + 1e-5, f"max |key - ref| = {err} (key scale {scale})"


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_tc_e4m3_search_recovers_exact(cuda, metric):
    """The scaled-FP8 form with a deep re-rank returns exact FP32 distances for its ids and nearly all of
    the exact top-k (the sampled-bar path: 300,000 rows)."""
    import torch
    from oracle.refmod import exact_topk_f64
    from tests.helpers import fp64_dists
    from annvedi_b200.linear import LinearIndex
    w = synth.scaled_mixture(300_000, 128, 96, c=256, seed=31)
    ix = LinearIndex(device=0, metric=metric, mode="exact")
    ix.fit(torch.from_numpy(w.base).cuda())
    ix.set_tc_precision("e4m3")
    ids, d = ix.search_tc(w.queries, 50, refine_r=1000)
    if metric == "l2":
        np.testing.assert_allclose(d, fp64_dists(w.base, w.queries, ids), rtol=1e-5, atol=1e-5)
    gt, _ = exact_topk_f64(w.base, w.queries, 50, metric)
    assert np.mean([len(set(a) & set(b)) / 50 for a, b in zip(ids, gt)]) > 0.99


def test_bounded_wait_runs_out_and_the_context_stays_usable(cuda):
    """The GEMM's mbarrier waits are bounded: with no copies issued (self-test), the waits give up after
    1 ms, the kernel sets its device flag (2) and returns; afterwards the same process searches normally."""
    import ctypes
    import time
    from annvedi_b200 import _lib
    from annvedi_b200.linear import LinearIndex
    from tests.helpers import check_exact_topk
    lib = _lib.load()
    for _ in range(2):
        flag = ctypes.c_int32(-1)
        t0 = time.perf_counter()
        _lib.check(lib.ann_tc_wait_selftest(0, 1_000_000, ctypes.byref(flag)))
        assert flag.value == 2, f"device flag {flag.value}"
        assert time.perf_counter() - t0 < 5.0
    w = synth.flat_normal(20000, 128, 32, seed=3)
    ix = LinearIndex(device=0, metric="l2", mode="exact")
    ix.fit(w.base)
    ids, d = ix.search_tc(w.queries, 10, refine_r=400)
    check_exact_topk(w.base, w.queries, ids, d, 10)
    assert lib.ann_flat_device_status(ix._h) == _lib.ANN_OK  # the index's own flag was never set
    bad = ctypes.c_int32(0)
    assert lib.ann_tc_wait_selftest(0, 10, ctypes.byref(bad)) == _lib.ANN_ERR_INVALID
