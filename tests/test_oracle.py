"""The oracle (oracle/restate.c, oracle/ivf_state.py) pinned against the reference.

CPU only. Two sources of truth:
* the committed golden fixtures (outputs of the reference's own compiled code, made by
  tests/golden/make_golden.py) -- always checked;
* the compiled reference itself (oracle/_ref/, built from the reference sources by
  oracle/Makefile) -- checked bit-for-bit where it is present and the host runs its AVX-512 build.
"""
import os

import numpy as np
import pytest

from annvedi_b200 import synth
from oracle import ivf_state, refmod
from tests.golden import make_golden as mg

LANES = 16  # the fixtures come from the reference's AVX-512 build


@pytest.fixture(scope="module")
def linear_fx(golden_dir):
    return np.load(os.path.join(golden_dir, "linear_ref.npz"))


@pytest.fixture(scope="module")
def ivf_fx(golden_dir):
    return np.load(os.path.join(golden_dir, "ivf_ref.npz"))


def test_restatement_matches_linear_golden(linear_fx):
    for name, base, queries, k in mg.linear_cases():
        ids, _ = refmod.linear_query(base, queries, k, lanes=LANES)
        np.testing.assert_array_equal(ids, linear_fx[f"{name}/ids"], err_msg=name)
        assert int(linear_fx[f"{name}/ndist"]) == base.shape[0] * queries.shape[0]


def test_restatement_matches_ivf_golden(ivf_fx):
    cases, _ = mg.ivf_cases()
    for name, spec, cfgs in cases:
        w = mg.make_workload(spec["workload"])
        proj = ivf_fx[f"{name}/projections"] if spec["n_bits"] else None
        st = ivf_state.build_state(w.base, w.centres, w.assign, spec["n_tables"], spec["n_bits"], proj)
        for ci, (k, n_probes, npc, rr, nt) in enumerate(cfgs):
            got = []
            nd = 0
            for q in w.queries:
                ids, _, nc = refmod.ivf_query(st, q, k, n_probes, npc, rr, num_threads=nt, lanes=LANES)
                got.append(ids)
                nd += nc
            np.testing.assert_array_equal(np.stack(got), ivf_fx[f"{name}/cfg{ci}/ids"], err_msg=f"{name} cfg{ci}")
            assert nd == int(ivf_fx[f"{name}/cfg{ci}/ndist"])


def test_restatement_matches_reference_fit_state(ivf_fx):
    st = {key.split("/")[-1]: ivf_fx[key] for key in ivf_fx.files if key.startswith("reffit/state/")}
    n, d = st["original_data"].shape
    st.update(npts=n, dim=d, n_clusters=st["centroids"].shape[0], n_tables=1, n_bits=0,
              projections=np.zeros((0, d), np.float32))
    # the stored codes / scales are reproduced by the restatement from the stored reordered data
    sc, of = refmod.sq8_train(st["original_data"])
    np.testing.assert_array_equal(sc, st["scale"])
    np.testing.assert_array_equal(of, st["offset"])
    np.testing.assert_array_equal(refmod.sq8_encode(st["original_data"], sc, of), st["quantized_data"])
    k, n_probes, npc, rr, nt = [int(v) for v in ivf_fx["reffit/params"]]
    got, nd = [], 0
    for q in ivf_fx["reffit/queries"]:
        ids, _, nc = refmod.ivf_query(st, q, k, n_probes, npc, rr, num_threads=nt, lanes=LANES)
        got.append(ids)
        nd += nc
    np.testing.assert_array_equal(np.stack(got), ivf_fx["reffit/ids"])
    assert nd == int(ivf_fx["reffit/ndist"])


def test_restatement_exact_mode_is_true_topk():
    w = synth.flat_normal(3000, 64, 8, seed=5)
    ids, vals = refmod.linear_query(w.base, w.queries, 64, lanes=LANES)
    gt, _ = refmod.exact_topk_f64(w.base, w.queries, 64)
    # with k <= 64 the reference heap never truncates: its ranking is the exact one
    assert (ids == gt).mean() > 0.999


def test_synthetic_generators_deterministic():
    a = synth.zipf_mixture(5000, 32, 10, c=32, lo=20, hi=1000, seed=3)
    b = synth.zipf_mixture(5000, 32, 10, c=32, lo=20, hi=1000, seed=3)
    np.testing.assert_array_equal(a.base, b.base)
    np.testing.assert_array_equal(a.queries, b.queries)
    sizes = synth.zipf_sizes(1_000_000, 2048)
    assert sizes.sum() == 1_000_000 and sizes.min() >= 20 and sizes.max() == 40000
    np.testing.assert_allclose(np.linalg.norm(a.base, axis=1), 1.0, rtol=1e-5)
    s = synth.scaled_mixture(2000, 16, 4, c=8, seed=1)
    nrm = np.linalg.norm(s.base, axis=1)
    assert nrm.min() >= 0.5 - 1e-4 and nrm.max() <= 2.0 + 1e-4


# ---- against the compiled reference (where available) ---------------------------------------

needs_ref = pytest.mark.skipif(not (refmod.ref_available("avx512") and refmod.host_isa() == "avx512"),
                               reason="reference AVX-512 build not available on this host")


@needs_ref
def test_distance_kernels_bit_exact_vs_reference():
    lin = refmod.load_ref("ref_linear_shim", "avx512")
    ivfm = refmod.load_ref("ref_ivf_shim", "avx512")
    rng = np.random.default_rng(0)
    for t in range(600):
        d = int(rng.choice([8, 12, 16, 20, 24, 96, 100, 256, 384, 768]))
        a = rng.standard_normal(d).astype(np.float32)
        b = rng.standard_normal(d).astype(np.float32)
        full = lin.l2_distance(a, b)
        thr = np.float32(full * rng.uniform(0.2, 1.1)) if t % 2 else np.finfo(np.float32).max
        assert np.float32(lin.l2_distance(a, b, thr)) == np.float32(refmod.l2(a, b, thr, LANES))
        c = rng.integers(0, 256, d).astype(np.uint8)
        sc = rng.uniform(0.001, 0.02, d).astype(np.float32)
        qs = rng.uniform(0, 3, d).astype(np.float32)
        assert np.float32(ivfm.l2_distance_sq8(c, qs, sc, thr)) == np.float32(refmod.l2_sq8(c, qs, sc, thr, LANES))


@needs_ref
def test_state_builder_matches_reference_fit():
    ivfm = refmod.load_ref("ref_ivf_shim", "avx512")
    w = synth.zipf_mixture(4000, 48, 4, c=20, lo=20, hi=1500, seed=9)
    for n_tables, n_bits in ((1, 0), (3, 4)):
        ix = ivfm.LSHIndex()
        ix.fit(w.base, n_tables, n_bits, 20)
        st = ivfm.export_state(ix)
        nb = 1 << n_bits
        off, r2o = st["table_offsets"], st["reordered_to_original"]
        assign = np.empty(w.base.shape[0], np.int64)
        for c in range(20):
            for s in range(nb):
                assign[r2o[st["table_ids"][off[c * nb + s]:off[c * nb + s + 1]]]] = c
        mine = ivf_state.build_state(w.base, st["centroids"], assign, n_tables, n_bits,
                                     st["projections"] if n_bits else None)
        for key in ("original_data", "quantized_data", "scale", "offset", "mean", "reordered_to_original",
                    "table_offsets", "table_ids"):
            np.testing.assert_array_equal(mine[key], st[key], err_msg=key)


# ---- k-means (IVFLSHIndex::run_kmeans) --------------------------------------------------------

def test_kmeans_restatement_matches_reference_golden(golden_dir):
    from tests.golden import make_kmeans_golden as mk
    fx = np.load(os.path.join(golden_dir, "kmeans_ref.npz"))
    for name, n, dim, c, t, dup, seed, _ in mk.kmeans_cases():
        x, _ = mk.make_rows(n, dim, dup, seed)
        cent, assign = refmod.kmeans(x, c, t, lanes=LANES)
        np.testing.assert_array_equal(cent, fx[f"{name}/centroids"], err_msg=name)
        np.testing.assert_array_equal(np.argsort(assign, kind="stable"), fx[f"{name}/reordered_to_original"],
                                      err_msg=name)
        np.testing.assert_array_equal(np.bincount(assign, minlength=min(c, n)), fx[f"{name}/list_sizes"],
                                      err_msg=name)


def test_kmeans_restatement_depends_on_thread_count():
    # the reason the thread count is pinned: per-chunk float sums change the centroids' last bits
    from tests.golden import make_kmeans_golden as mk
    x, _ = mk.make_rows(3000, 64, 0, 0)
    a, _ = refmod.kmeans(x, 16, 3, lanes=LANES)
    b, _ = refmod.kmeans(x, 16, 4, lanes=LANES)
    assert not np.array_equal(a, b)
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)


def test_kmeans_order_is_a_permutation():
    o = refmod.kmeans_order(1000)
    np.testing.assert_array_equal(np.sort(o), np.arange(1000))
    np.testing.assert_array_equal(o, refmod.kmeans_order(1000))


@needs_ref
def test_kmeans_restatement_matches_reference_fit_directly():
    ivfm = refmod.load_ref("ref_ivf_shim", "avx512")
    w = synth.zipf_mixture(6000, 48, 4, c=24, lo=20, hi=1500, seed=11)
    for t in (1, 6, 13):
        ix = refmod.ref_fit(w.base, 1, 0, 24, t, "avx512")
        st = ivfm.export_state(ix)
        cent, assign = refmod.kmeans(w.base, 24, t, lanes=LANES)
        np.testing.assert_array_equal(cent, st["centroids"])
        np.testing.assert_array_equal(np.argsort(assign, kind="stable"), st["reordered_to_original"])
