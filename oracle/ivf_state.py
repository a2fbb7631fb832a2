"""Builds an IVF-LSH index state in the reference's layout from (data, centroids, assignment).

ORACLE INFRASTRUCTURE: used by tests/, the golden-fixture script and the smoke check only.

The layout is the one IVFLSHIndex::fit leaves behind (competitors/ivf_lsh/src/
lsh_index_optimized.cpp:154-283), so the state can be imported into the reference (through the
test shim, oracle/ref_ivf_shim.cpp) and into the GPU index alike:

* points reordered cluster by cluster, in ascending original id inside a cluster (:155-173);
* per-dimension SQ8 scale/offset over the reordered data and uint8 codes (:187-214), computed by
  the restatement (oracle/restate.c), which is pinned bit-for-bit against the reference;
* bucket tables [n_tables][n_clusters][2^n_bits] of reordered ids (:261-283); with n_bits = 0
  each cluster's single bucket is its whole inverted list.

For n_bits > 0 the random projections are an input (they come from the reference's
std::mt19937(42) + std::normal_distribution stream, :217-258, exported once from a reference fit)
and the signature of a point is the sign of its mean-centred projection, summed in order.
"""
from __future__ import annotations

import numpy as np

from . import refmod


def build_state(data: np.ndarray, centroids: np.ndarray, assign: np.ndarray, n_tables: int = 1, n_bits: int = 0,
                projections: np.ndarray | None = None) -> dict:
    data = np.ascontiguousarray(data, np.float32)
    centroids = np.ascontiguousarray(centroids, np.float32)
    assign = np.asarray(assign).astype(np.int64)
    n, d = data.shape
    c = centroids.shape[0]
    order = np.argsort(assign, kind="stable")
    original = np.ascontiguousarray(data[order])
    scale, offset = refmod.sq8_train(original)
    codes = refmod.sq8_encode(original, scale, offset)
    mean = np.zeros(d, np.float32)
    for i in range(n):  # the reference's float accumulation order (:176-184)
        mean += original[i]
    # -ffast-math turns the division by npts into a multiplication by its float reciprocal
    mean = (mean * (np.float32(1) / np.float32(n))).astype(np.float32)
    sorted_assign = assign[order]
    nb = 1 << n_bits
    if n_bits > 0:
        if projections is None or projections.shape != (n_tables * n_bits, d):
            raise ValueError("n_bits > 0 needs projections [n_tables * n_bits, dim]")
        proj = np.ascontiguousarray(projections, np.float32)
        centred = original - mean
        sig = np.zeros((n_tables, n), np.int64)
        for t in range(n_tables):
            for b in range(n_bits):
                dots = centred.astype(np.float64) @ proj[t * n_bits + b].astype(np.float64)
                sig[t] |= (dots > 0).astype(np.int64) << b
    else:
        proj = np.zeros((0, d), np.float32)
        sig = np.zeros((n_tables, n), np.int64)
    offsets = np.zeros(n_tables * c * nb + 1, np.int64)
    ids = []
    pos = 0
    for t in range(n_tables):
        key = sorted_assign * nb + sig[t]
        counts = np.bincount(key, minlength=c * nb)
        # reordered ids are already grouped by cluster; a stable sort by bucket keeps id order
        members = np.argsort(key, kind="stable").astype(np.int32)
        ids.append(members)
        offsets[pos + 1: pos + 1 + c * nb] = offsets[pos] + np.cumsum(counts)
        pos += c * nb
    return {
        "npts": n, "dim": d, "n_clusters": c, "n_tables": n_tables, "n_bits": n_bits, "num_threads": 0,
        "centroids": centroids, "original_data": original, "quantized_data": codes, "scale": scale,
        "offset": offset, "mean": mean, "reordered_to_original": order.astype(np.int32),
        "projections": proj, "table_offsets": offsets,
        "table_ids": np.concatenate(ids) if ids else np.zeros(0, np.int32),
    }


def nearest_centroid(data: np.ndarray, centroids: np.ndarray) -> np.ndarray:
    """FP64 nearest-centroid assignment (ties to the lower centroid)."""
    x = np.asarray(data, np.float64)
    c = np.asarray(centroids, np.float64)
    d2 = (x * x).sum(1)[:, None] - 2 * x @ c.T + (c * c).sum(1)[None, :]
    return d2.argmin(1)
