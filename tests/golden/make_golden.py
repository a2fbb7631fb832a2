"""Generates the golden fixtures in tests/golden/ by running the reference's own compiled code.

    make -C oracle ref restate && python tests/golden/make_golden.py

Needs the reference modules built from the reference sources (oracle/_ref/, AVX-512 build). Inputs
are not stored: every case is regenerated from its seed by annvedi_b200.synth (numpy
default_rng, identical on every machine) and, for IVF cases, by oracle.ivf_state.build_state.
Only the reference's outputs (ids, distance counters) and, for one case, a whole state exported
from a reference fit are committed.

Files:
  linear_ref.npz  LinearIndex (competitors/linear/src/linear_index.cpp) top-k ids per case.
  ivf_ref.npz     LSHIndex (competitors/ivf_lsh/src/lsh_index_optimized.cpp) ids and
                  get_n_distances per query configuration, over imported states.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from annvedi_b200 import synth  # noqa: E402
from oracle import ivf_state, refmod  # noqa: E402

ISA = "avx512"


def linear_cases():
    """(name, base, queries, k) for the linear fixture."""
    cases = []
    w = synth.flat_normal(20000, 384, 48, seed=101)
    cases.append(("c1_shape_20k_384", w.base, w.queries, 100))
    rng = np.random.default_rng(102)
    d = rng.random((50, 16), dtype=np.float32)
    cases.append(("ref_test_50x16_k5", d, d[[0, 10]], 5))
    cases.append(("ref_test_50x16_k1", d, d[[10]], 1))
    rng = np.random.default_rng(103)
    d = rng.random((20, 8), dtype=np.float32)
    cases.append(("ref_test_20x8_k3", d, d[[0, 1]], 3))
    w = synth.flat_normal(3000, 100, 16, seed=104)
    cases.append(("ragged_dim100", w.base, w.queries, 100))
    w = synth.flat_normal(60, 32, 4, seed=105)
    cases.append(("k_above_n", w.base, w.queries, 100))
    rng = np.random.default_rng(106)
    distinct = rng.standard_normal((100, 64), dtype=np.float32)
    base = distinct[rng.integers(0, 100, 1000)]
    cases.append(("duplicates_ties", base, np.concatenate([distinct[:4], base[:4]]), 100))
    w = synth.flat_normal(5000, 256, 8, seed=107)
    cases.append(("k64", w.base, w.queries, 64))
    cases.append(("k65", w.base, w.queries, 65))
    w = synth.flat_normal(2000, 20, 8, seed=108)
    cases.append(("dim20_remainder", w.base, w.queries, 50))
    w = synth.flat_normal(4000, 768, 8, seed=109)
    cases.append(("dim768", w.base, w.queries, 100))
    return cases


def ivf_cases():
    """(name, state builder kwargs, queries, query configs)."""
    w = synth.zipf_mixture(30000, 384, 32, c=64, lo=20, hi=3000, seed=201)
    c1 = dict(workload=("zipf_mixture", dict(n=30000, d=384, q=32, c=64, lo=20, hi=3000, seed=201)),
              n_tables=1, n_bits=0)
    cfg1 = [  # (k, n_probes, n_probe_clusters, refine_r, num_threads)
        (100, 0, 8, 300, 8), (100, 0, 32, -1, 8), (100, 0, 64, 2000, 3), (100, 0, 4, 100, 1),
        (10, 0, 2, -1, 8),
    ]
    w2 = dict(workload=("zipf_mixture", dict(n=8000, d=64, q=16, c=16, lo=20, hi=2000, seed=202)),
              n_tables=3, n_bits=4)
    cfg2 = [(50, 3, 6, 200, 4), (50, 0, 4, -1, 2)]
    w3 = dict(workload=("zipf_mixture", dict(n=3000, d=32, q=8, c=200, lo=2, hi=40, seed=203)),
              n_tables=1, n_bits=0)
    cfg3 = [(100, 0, 1, -1, 8)]  # fewer candidates than k: falls back to all points (:453-457)
    return [("zipf_30k_384_c64", c1, cfg1), ("lsh_8k_64_t3b4", w2, cfg2), ("fallback_all", w3, cfg3)], w


def make_workload(spec):
    kind, kw = spec
    return synth.make(kind, **kw)


def projections_from_reference(n_tables, n_bits, dim):
    """The reference's random projections depend only on (n_tables, n_bits, dim): fit a tiny
    index and export them."""
    ivfm = refmod.load_ref("ref_ivf_shim", ISA)
    ix = ivfm.LSHIndex()
    x = np.random.default_rng(0).standard_normal((64, dim), dtype=np.float32)
    ix.fit(x, n_tables, n_bits, 2)
    return ivfm.export_state(ix)["projections"]


def main():
    linm = refmod.load_ref("ref_linear_shim", ISA)
    ivfm = refmod.load_ref("ref_ivf_shim", ISA)
    out = {}
    for name, base, queries, k in linear_cases():
        ix = linm.LinearIndex()
        ix.fit(np.ascontiguousarray(base, np.float32))
        ids = np.stack([ix.query(np.ascontiguousarray(q, np.float32), k) for q in queries])
        out[f"{name}/ids"] = ids.astype(np.int32)
        out[f"{name}/ndist"] = np.int64(ix.total_distances_count())
    np.savez_compressed(os.path.join(HERE, "linear_ref.npz"), **out)
    print("linear cases:", len(linear_cases()))

    out = {}
    cases, _ = ivf_cases()
    for name, spec, cfgs in cases:
        w = make_workload(spec["workload"])
        proj = projections_from_reference(spec["n_tables"], spec["n_bits"], w.base.shape[1]) if spec["n_bits"] else None
        st = ivf_state.build_state(w.base, w.centres, w.assign, spec["n_tables"], spec["n_bits"], proj)
        if proj is not None:
            out[f"{name}/projections"] = proj
        for ci, (k, n_probes, npc, rr, nt) in enumerate(cfgs):
            ix = ivfm.LSHIndex()
            ivfm.import_state(ix, st, nt)
            ids = np.stack([ix.query(q, k, n_probes, npc, rr) for q in w.queries])
            out[f"{name}/cfg{ci}/ids"] = ids.astype(np.int32)
            out[f"{name}/cfg{ci}/ndist"] = np.int64(ix.total_distances_count())
            out[f"{name}/cfg{ci}/params"] = np.array([k, n_probes, npc, rr, nt], np.int64)

    # one state produced by the reference's own fit (k-means on this host's thread count), stored
    # whole, with its query outputs
    w = synth.zipf_mixture(2000, 32, 8, c=16, lo=20, hi=400, seed=204)
    ix = ivfm.LSHIndex()
    ix.fit(w.base, 1, 0, 16)
    st = ivfm.export_state(ix)
    for key in ("centroids", "original_data", "quantized_data", "scale", "offset", "mean",
                "reordered_to_original", "table_offsets", "table_ids"):
        out[f"reffit/state/{key}"] = st[key]
    out["reffit/queries"] = w.queries
    ivfm.set_num_threads(ix, 4)
    ix.reset_distances_count()
    out["reffit/ids"] = np.stack([ix.query(q, 20, 0, 3, 60) for q in w.queries]).astype(np.int32)
    out["reffit/ndist"] = np.int64(ix.total_distances_count())
    out["reffit/params"] = np.array([20, 0, 3, 60, 4], np.int64)
    np.savez_compressed(os.path.join(HERE, "ivf_ref.npz"), **out)
    print("ivf fixture keys:", len(out))


if __name__ == "__main__":
    main()
