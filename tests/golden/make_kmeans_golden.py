"""Golden outputs of the reference's own k-means fit (IVFLSHIndex::fit with n_tables = 1, n_bits = 0,
competitors/ivf_lsh/src/lsh_index_optimized.cpp:128-173, 551-616), with the fit's thread count pinned.

    python tests/golden/make_kmeans_golden.py     # needs oracle/_ref (make -C oracle ref REF=...)

Writes tests/golden/kmeans_ref.npz: per case the pinned thread count's results -- the reference's
final centroids, its list order (reordered_to_original) and list sizes, and the ids and distance
count of a few queries answered by that fitted index (same thread count). The fit sums per
ThreadPool chunk, so the thread count is part of the case. The cases cover remainder dimensions
(dim % 16 = 0, 4, 5, 8), more threads than rows, a single list, and duplicated rows (equal
distances, empty lists reseeded from rand_indices[(c * 37) % n]).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import refmod  # noqa: E402

ISA = "avx512"


def kmeans_cases():
    """(name, n, dim, n_clusters, threads, duplicate_rows, seed, query params (k, npc, refine_r))."""
    return [
        ("normal_3000x64_c16_t3", 3000, 64, 16, 3, 0, 0, (20, 3, 60)),
        ("normal_5000x100_c37_t8", 5000, 100, 37, 8, 0, 1, (30, 4, 100)),
        ("normal_2000x20_c200_t5", 2000, 20, 200, 5, 0, 2, (10, 8, 40)),
        ("normal_4000x384_c64_t16", 4000, 384, 64, 16, 0, 3, (100, 6, 300)),
        ("normal_1200x24_c30_t7", 1200, 24, 30, 7, 0, 4, (10, 5, 30)),
        ("normal_1500x37_c40_t2", 1500, 37, 40, 2, 0, 5, (10, 5, 30)),
        ("dups_1500x16_c64_t4", 1500, 16, 64, 4, 40, 6, (20, 8, 60)),
        ("tiny_10x8_c4_t16", 10, 8, 4, 16, 0, 7, (3, 2, 5)),
        ("single_list_800x32_c1_t6", 800, 32, 1, 6, 0, 8, (10, 1, 50)),
    ]


def make_rows(n, dim, dup, seed):
    rng = np.random.default_rng(seed)
    if dup:
        distinct = rng.standard_normal((dup, dim)).astype(np.float32)
        x = distinct[rng.integers(0, dup, n)]
    else:
        x = rng.standard_normal((n, dim)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    q = rng.standard_normal((8, dim)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return np.ascontiguousarray(x, np.float32), np.ascontiguousarray(q, np.float32)


def main():
    m = refmod.load_ref("ref_ivf_shim", ISA)
    out = {}
    for name, n, dim, c, t, dup, seed, (k, npc, rr) in kmeans_cases():
        x, q = make_rows(n, dim, dup, seed)
        ix = refmod.ref_fit(x, 1, 0, c, t, ISA)
        st = m.export_state(ix)
        out[f"{name}/centroids"] = st["centroids"]
        out[f"{name}/reordered_to_original"] = st["reordered_to_original"]
        out[f"{name}/list_sizes"] = np.diff(st["table_offsets"]).astype(np.int64)
        assert m.get_num_threads(ix) == t
        ix.reset_distances_count()
        out[f"{name}/ids"] = np.stack([ix.query(qq, k, 0, npc, rr) for qq in q]).astype(np.int64)
        out[f"{name}/ndist"] = np.int64(ix.total_distances_count())
    np.savez_compressed(os.path.join(HERE, "kmeans_ref.npz"), **out)
    print("k-means cases:", len(kmeans_cases()))


if __name__ == "__main__":
    main()
