"""Checks shared by the parity tests."""
from __future__ import annotations

import numpy as np


def fp64_dists(base, queries, ids, metric="l2"):
    """FP64 distance (or inner product) of each returned id; NaN where id == -1."""
    base = np.asarray(base, np.float64)
    q = np.asarray(queries, np.float64)
    ids = np.asarray(ids)
    out = np.full(ids.shape, np.nan)
    for i in range(ids.shape[0]):
        m = ids[i] >= 0
        x = base[ids[i][m]]
        if metric == "ip":
            out[i, m] = x @ q[i]
        else:
            diff = x - q[i]
            out[i, m] = np.einsum("ij,ij->i", diff, diff)
    return out


def check_exact_topk(base, queries, ids, dists, k, metric="l2", rtol=1e-5, atol=1e-6):
    """The returned ids are a true top-k up to ties within tolerance, and the returned values
    match FP64 within rtol. Returns the recall against the FP64 top-k (ties counted as hits)."""
    from oracle.refmod import exact_topk_f64
    ids = np.asarray(ids)
    gt_ids, gt_d = exact_topk_f64(base, queries, k, metric)
    got = fp64_dists(base, queries, ids, metric)
    assert not np.isnan(got).any(), "fewer than k results"
    if dists is not None:
        dd = np.asarray(dists, np.float64)
        np.testing.assert_allclose(dd, got, rtol=rtol, atol=atol)
    sign = -1.0 if metric == "ip" else 1.0
    key_got = sign * got
    key_gt = sign * gt_d
    kth = key_gt[:, -1:]
    tol = rtol * np.abs(kth) + atol
    # every returned id is within tolerance of the true k-th value ...
    assert (key_got <= kth + tol).all(), f"returned ids beyond the k-th distance: {(key_got > kth + tol).sum()}"
    # ... and the sorted returned values match the true sorted values within tolerance
    np.testing.assert_allclose(np.sort(key_got, 1), key_gt, rtol=rtol, atol=atol)
    hits = (key_got <= kth + tol).mean()
    return float(hits)


def recall_at_k(true_d_kth, got_d, k):
    """Evaluator recall: mean(pred_d[:k] <= true_d[k-1]) (orthogonal-competition/evaluator.py:149-157)."""
    return float(np.mean(got_d[:, :k] <= true_d_kth[:, None]))


def assert_ids_equal_up_to_ties(base, queries, got, want, rtol=1e-6, err_msg=""):
    """Per query: the same ids, or -- where they differ -- ids whose FP64 distances, sorted, equal the
    wanted ids' within rtol (the two lists differ only by which of equally distant rows they keep).
    Returns the number of queries that needed the tie rule."""
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, err_msg
    nties = 0
    for i in range(got.shape[0]):
        if np.array_equal(got[i], want[i]):
            continue
        nties += 1
        assert ((got[i] >= 0) == (want[i] >= 0)).all(), f"{err_msg}: query {i} returns a different count"
        dg = np.sort(fp64_dists(base, queries[i:i + 1], got[i:i + 1])[0])
        dw = np.sort(fp64_dists(base, queries[i:i + 1], want[i:i + 1])[0])
        np.testing.assert_allclose(dg, dw, rtol=rtol, atol=1e-12, err_msg=f"{err_msg}: query {i}")
    return nties
