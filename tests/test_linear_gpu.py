"""GPU parity of the linear index (reference semantics and exact semantics) through the C ABI.

Reference mode must return the reference's ids exactly (the GPU replays the reference's AVX-512
arithmetic and 64-entry heap bit for bit), checked against the golden fixtures and the oracle.
Exact mode must return the true top-k: ids may differ from the FP64 top-k only at ties within
1e-5 relative, and distances must match FP64 within 1e-5 relative.
"""
import os

import numpy as np
import pytest

from annvedi_b200 import synth
from oracle import refmod
from tests.golden import make_golden as mg
from tests.helpers import check_exact_topk

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def linear_fx(golden_dir):
    return np.load(os.path.join(golden_dir, "linear_ref.npz"))


def _index(base, mode="reference", metric="l2"):
    from annvedi_b200.linear import LinearIndex
    ix = LinearIndex(device=0, metric=metric, mode=mode)
    ix.fit(base)
    return ix


def test_reference_mode_matches_golden(cuda, linear_fx):
    for name, base, queries, k in mg.linear_cases():
        ix = _index(base)
        ids, vals = ix.search(queries, k)
        np.testing.assert_array_equal(ids, linear_fx[f"{name}/ids"], err_msg=name)
        assert ix.total_distances_count() == int(linear_fx[f"{name}/ndist"])
        # the ranking values equal the oracle's, bit for bit
        oids, ovals = refmod.linear_query(base, queries, k, lanes=16)
        np.testing.assert_array_equal(vals, ovals, err_msg=name)


def test_reference_mode_single_query_drop_in(cuda, linear_fx):
    for name, base, queries, k in mg.linear_cases()[:4]:
        ix = _index(base)
        got = np.stack([ix.query(q, k) for q in queries])
        assert got.dtype == np.int64
        np.testing.assert_array_equal(got, linear_fx[f"{name}/ids"], err_msg=name)


@pytest.mark.parametrize("nq", [1, 2, 3, 4, 8, 17, 64, 200])
@pytest.mark.parametrize("k", [1, 10, 100, 257])
def test_exact_mode_matches_fp64(cuda, nq, k):
    w = synth.flat_normal(20000, 384, nq, seed=nq * 31 + k)
    ix = _index(w.base, mode="exact")
    ids, d = ix.search(w.queries, k)
    check_exact_topk(w.base, w.queries, ids, d, k)


@pytest.mark.parametrize("dim", [8, 20, 100, 256, 768])
def test_exact_mode_dims_and_ip(cuda, dim):
    w = synth.flat_normal(5000, dim, 12, seed=dim)
    for metric in ("l2", "ip"):
        ix = _index(w.base, mode="exact", metric=metric)
        ids, d = ix.search(w.queries, 50)
        check_exact_topk(w.base, w.queries, ids, d, 50, metric=metric)


@pytest.mark.parametrize("nq", [1, 2, 4, 16])
@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_exact_ties_break_by_lower_id(cuda, nq, metric):
    """Rows that are exact copies have equal FP32 distances; the exact top-k orders them by lower id,
    also where the tie straddles the k-th place (every split, the streaming form and the merge)."""
    rng = np.random.default_rng(nq)
    distinct = rng.normal(size=(150, 64)).astype(np.float32)
    group = rng.integers(0, 150, 60000)
    base = distinct[group]
    queries = rng.normal(size=(nq, 64)).astype(np.float32)
    ix = _index(base, mode="exact", metric=metric)
    ids, _ = ix.search(queries, 100)
    for qi in range(nq):
        if metric == "l2":
            score = ((distinct.astype(np.float64) - queries[qi]) ** 2).sum(1)
        else:
            score = -(distinct.astype(np.float64) @ queries[qi])
        order = np.argsort(score, kind="stable")
        want = []
        for g in order:
            want.extend(np.flatnonzero(group == g).tolist())
            if len(want) >= 100:
                break
        np.testing.assert_array_equal(ids[qi], np.array(want[:100]), err_msg=f"query {qi}")


def test_exact_mode_device_tensors_match_host(cuda):
    import torch
    w = synth.flat_normal(30000, 384, 40, seed=7)
    ix = _index(torch.from_numpy(w.base).to(cuda), mode="exact")
    qd = torch.from_numpy(w.queries).to(cuda)
    ids_d, d_d = ix.search(qd, 100)
    torch.cuda.synchronize()
    ids_h, d_h = ix.search(w.queries, 100)
    np.testing.assert_array_equal(ids_d.cpu().numpy(), ids_h)
    np.testing.assert_array_equal(d_d.cpu().numpy(), d_h)


def test_edge_cases(cuda):
    # k > n clips to n; duplicates give ties that resolve by lower id; n not a multiple of tiles
    w = synth.flat_normal(37, 16, 3, seed=1)
    ix = _index(w.base, mode="exact")
    ids, d = ix.search(w.queries, 100)
    assert ids.shape == (3, 37)
    assert sorted(ids[0].tolist()) == list(range(37))
    base = np.repeat(np.eye(4, 32, dtype=np.float32), 50, axis=0)  # 200 rows, 4 distinct
    ix = _index(base, mode="exact")
    ids, d = ix.search(base[:1], 60)
    np.testing.assert_array_equal(ids[0, :50], np.arange(50))  # exact ties -> lower id first
    assert (d[0, :50] == 0).all()


def test_errors(cuda):
    from annvedi_b200.linear import LinearIndex
    ix = LinearIndex(device=0)
    with pytest.raises(RuntimeError):
        ix.query(np.zeros(8, np.float32), 3)
    with pytest.raises(RuntimeError):
        ix.fit(np.zeros(8, np.float32))
    ix.fit(np.zeros((10, 8), np.float32))
    with pytest.raises(RuntimeError):
        ix.query(np.zeros(7, np.float32), 3)
    with pytest.raises(RuntimeError):
        ix.search(np.zeros((2, 8), np.float32), 0)


def test_reference_unit_tests_through_algorithm(cuda):
    """tests/test_logic.py of the reference, against the drop-in Algorithm."""
    from annvedi_b200.algorithm import Algorithm
    rng = np.random.default_rng(0)
    data = rng.random((50, 16), dtype=np.float32)
    a = Algorithm()
    a.fit(data)
    assert len(a.query(data[0], 5)) == 5
    assert a.query(data[10], 1)[0] == 10
    data = rng.random((20, 8), dtype=np.float32)
    a = Algorithm()
    a.fit(data)
    a.query(data[0], 3)
    assert a.get_n_distances() == 20


@pytest.mark.slow
def test_full_size_c1_exact_and_reference(cuda):
    """100k x 384, 1,000 queries: exact mode equals FP64 up to ties; reference mode equals the
    oracle restatement for a sample of queries."""
    w = synth.flat_normal(100_000, 384, 1000, seed=0)
    ix = _index(w.base, mode="exact")
    ids, d = ix.search(w.queries, 100)
    check_exact_topk(w.base, w.queries[:200], ids[:200], d[:200], 100)
    rids, rvals = ix.search(w.queries[:32], 100, mode="reference")
    oids, ovals = refmod.linear_query(w.base, w.queries[:32], 100, lanes=16)
    np.testing.assert_array_equal(rids, oids)
    assert ix.total_distances_count() == 100_000 * 1032


@pytest.mark.parametrize("k", [10, 100])
def test_query_tile_does_not_change_results(cuda, k):
    """The exact scan's query tile (ANN_FLAT_OPT_QUERY_TILE) changes speed only: tiles of 8, 16 and 32 queries
    (the last with its queries in packed pairs) return the same ids and distances as the automatic choice for
    this batch, bit for bit; other tiles are refused."""
    import torch
    from annvedi_b200.linear import LinearIndex
    rng = np.random.default_rng(40)
    base = rng.standard_normal((60000, 96)).astype(np.float32)
    q = torch.from_numpy(rng.standard_normal((301, 96)).astype(np.float32)).cuda()  # odd: a half-empty pair
    ix = LinearIndex(device=0, mode="exact")
    ix.fit(torch.from_numpy(base).cuda())
    want_i, want_d = ix.search(q, k, mode="exact")
    want_i, want_d = want_i.cpu().numpy(), want_d.cpu().numpy()
    for tile in (8, 16, 32):
        ix.set_query_tile(tile)
        got_i, got_d = ix.search(q, k, mode="exact")
        np.testing.assert_array_equal(got_i.cpu().numpy(), want_i, err_msg=f"tile {tile}")
        np.testing.assert_array_equal(got_d.cpu().numpy(), want_d, err_msg=f"tile {tile}")
    for bad in (1, 4, 3):
        with pytest.raises(Exception):
            ix.set_query_tile(bad)
