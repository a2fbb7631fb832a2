"""The GPU IVF fit against the reference's own fit (IVFLSHIndex::fit, n_tables = 1, n_bits = 0,
competitors/ivf_lsh/src/lsh_index_optimized.cpp:128-173, 551-616).

With the ThreadPool size pinned on both sides, the GPU k-means must leave the reference's centroids
bit for bit and the same lists, so that fit followed by query returns the reference's ids and
distance counts -- the harness's own sequence (orthogonal-competition/harness.py:141-176). Where
rows are duplicated, distances tie exactly; the reference orders candidates by distance alone
(std::partial_sort on .first, :476-479, :498-501), which leaves the order of equal distances to
the sort's internals, so there ids may differ among exactly equal distances only.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from annvedi_b200 import synth
from annvedi_b200.algorithm import Algorithm
from annvedi_b200.ivf import IVFIndex
from oracle import refmod
from tests.golden import make_kmeans_golden as mk
from tests.helpers import assert_ids_equal_up_to_ties

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not (refmod.ref_available("avx512") and refmod.host_isa() == "avx512"),
                               reason="reference AVX-512 build not available on this host")


def assert_same_up_to_exact_ties(base, queries, got, want, err_msg=""):
    """The same ids per query; where positions differ, the ids there are rows at exactly equal distances
    (the reference's own arithmetic, restated bit for bit): the reference orders its candidates by
    distance alone with std::partial_sort (lsh_index_optimized.cpp:476-479, 498-501), whose order among
    equal distances is its sort's internal one. Returns the number of queries with such swaps."""
    swaps = 0
    for i in range(got.shape[0]):
        if np.array_equal(got[i], want[i]):
            continue
        swaps += 1
        assert sorted(got[i].tolist()) == sorted(want[i].tolist()), f"{err_msg}: query {i} returns other ids"
        for p in np.nonzero(got[i] != want[i])[0]:
            dg = refmod.l2(base[got[i][p]], queries[i]) if got[i][p] >= 0 else None
            dw = refmod.l2(base[want[i][p]], queries[i]) if want[i][p] >= 0 else None
            assert dg == dw, f"{err_msg}: query {i} position {p}: {got[i][p]} ({dg}) vs {want[i][p]} ({dw})"
    return swaps


def test_fit_reproduces_reference_kmeans_goldens(cuda, golden_dir):
    fx = np.load(os.path.join(golden_dir, "kmeans_ref.npz"))
    for name, n, dim, c, t, dup, seed, (k, npc, rr) in mk.kmeans_cases():
        x, q = mk.make_rows(n, dim, dup, seed)
        ix = IVFIndex(device=0, mode="reference", num_threads=t)
        ix.fit(x, 1, 0, c)
        st = ix.export_state()
        np.testing.assert_array_equal(st["centroids"], fx[f"{name}/centroids"], err_msg=name)
        np.testing.assert_array_equal(st["reordered_to_original"], fx[f"{name}/reordered_to_original"], err_msg=name)
        np.testing.assert_array_equal(np.diff(st["table_offsets"]), fx[f"{name}/list_sizes"], err_msg=name)
        ids = np.stack([ix.query(qq, k, 0, npc, rr) for qq in q])
        if dup:
            assert_ids_equal_up_to_ties(x, q, ids, fx[f"{name}/ids"], err_msg=name)
        else:
            np.testing.assert_array_equal(ids, fx[f"{name}/ids"], err_msg=name)
        assert ix.total_distances_count() == int(fx[f"{name}/ndist"]), name


def test_fit_from_device_rows_equals_fit_from_host_rows(cuda):
    import torch
    x, _ = mk.make_rows(3000, 100, 0, 12)
    a = IVFIndex(device=0, num_threads=5)
    a.fit(x, 1, 0, 24)
    b = IVFIndex(device=0, num_threads=5)
    b.fit(torch.from_numpy(x).cuda(), 1, 0, 24)
    torch.cuda.synchronize()
    sa, sb = a.export_state(), b.export_state()
    for key in ("centroids", "reordered_to_original", "table_offsets", "quantized_data"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)


def test_fit_matches_restated_kmeans_on_duplicates_and_ties(cuda):
    # 30 distinct rows repeated: every row is equidistant to duplicated seeds, lists end empty and are
    # reseeded; the near-tie path (reference arithmetic) decides these assignments
    x, _ = mk.make_rows(2500, 48, 30, 13)
    for t in (1, 7):
        cent, assign = refmod.kmeans(x, 50, t)
        ix = IVFIndex(device=0, num_threads=t)
        ix.fit(x, 1, 0, 50)
        st = ix.export_state()
        np.testing.assert_array_equal(st["centroids"], cent)
        np.testing.assert_array_equal(st["reordered_to_original"], np.argsort(assign, kind="stable"))


@needs_ref
def test_algorithm_fit_query_equals_reference_fit_query_50k(cuda):
    """Algorithm().fit(X, backend='ivf_lsh', n_tables=1, n_bits=0, ...) then query, against the
    compiled ivf_lsh_cpp's fit then query, both with a ThreadPool of 16, on seeded 50k x 384 rows."""
    T, C = 16, 256
    w = synth.zipf_mixture(50_000, 384, 200, c=C, lo=20, hi=3000, seed=21)
    ref = refmod.ref_fit(w.base, 1, 0, C, T, "avx512")
    algo = Algorithm()
    algo.fit(w.base, backend="ivf_lsh", n_tables=1, n_bits=0, n_clusters=C, num_threads=T)
    st = algo._index.export_state()
    rst = refmod.load_ref("ref_ivf_shim", "avx512").export_state(ref)
    np.testing.assert_array_equal(st["centroids"], rst["centroids"])
    np.testing.assert_array_equal(st["reordered_to_original"], rst["reordered_to_original"])
    for npc, rr in ((8, 300), (32, 2000), (4, -1)):
        ref.reset_distances_count()
        n0 = algo.get_n_distances()
        want = np.stack([ref.query(q, 100, 0, npc, rr) for q in w.queries])
        got = np.stack([algo.query(q, 100, n_probe_clusters=npc, refine_r=rr) for q in w.queries])
        swaps = assert_same_up_to_exact_ties(w.base, w.queries, got, want, err_msg=f"npc={npc} refine_r={rr}")
        assert swaps <= 3, swaps  # exact FP32 ties among a query's top 100: about one query in a hundred
        assert algo.get_n_distances() - n0 == ref.total_distances_count()


@needs_ref
@pytest.mark.slow
def test_linear_c1_all_queries_equal_compiled_reference(cuda):
    """The linear backend on the full 100k x 384 shape with 1,000 queries: every query's ids equal
    the compiled linear_ann_cpp's, and get_n_distances = 1,000 x 100,000."""
    w = synth.flat_normal(100_000, 384, 1000, seed=0)
    ref = refmod.load_ref("linear_ann_cpp", "avx512").LinearIndex()
    ref.fit(w.base)
    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:  # the reference releases the GIL in query
        want = np.stack(list(ex.map(lambda q: ref.query(q, 100), w.queries)))
    algo = Algorithm()
    algo.fit(w.base, backend="linear")
    got = np.stack([algo.query(q, 100) for q in w.queries])
    np.testing.assert_array_equal(got, want)
    assert algo.get_n_distances() == 1000 * 100_000
    assert ref.total_distances_count() == 1000 * 100_000


@needs_ref
@pytest.mark.slow
def test_ivf_c3_shape_reference_mode_equals_compiled_reference(cuda):
    """1M x 384 with 2,048 Zipf-sized lists: the reference-mode query over the same state returns the
    compiled reference's ids and distance counts on 256 queries (ThreadPool of 16), with its
    candidate cap binding (refine_r 300) and lifted (refine_r 8,000)."""
    from oracle import ivf_state
    z = synth.zipf_mixture(1_000_000, 384, 256, c=2048, lo=20, hi=40_000, sigma=0.3, seed=7)
    st = ivf_state.build_state(z.base, z.centres, z.assign, 1, 0)
    shim = refmod.load_ref("ref_ivf_shim", "avx512")
    ref = shim.LSHIndex()
    shim.import_state(ref, st, 16)
    ix = IVFIndex(device=0, mode="reference", num_threads=16)
    ix.import_state(st)
    for npc, rr in ((8, 300), (16, 8000)):
        ref.reset_distances_count()
        ix.reset_distances_count()
        want = np.stack([ref.query(q, 100, 0, npc, rr) for q in z.queries])
        got, _ = ix.search(z.queries, 100, 0, npc, rr)
        assert_same_up_to_exact_ties(z.base, z.queries, got, want, err_msg=f"npc={npc} refine_r={rr}")
        assert ix.total_distances_count() == ref.total_distances_count()
