"""GPU parity of the IVF-SQ8 index through the C ABI.

* reference mode over an imported state returns the reference's ids and get_n_distances exactly
  (golden fixtures made by the reference's own LSHIndex, and the oracle restatement);
* the GPU build (given centroids and lists) produces the reference's state bit for bit
  (reorder, per-dimension SQ8 scale/offset, codes);
* exact mode returns the exact-selection result: ids may differ from the oracle only at ties
  within 1e-5 relative, distances match FP64 within 1e-5 relative.
"""
import os

import numpy as np
import pytest

from annvedi_b200 import synth
from oracle import ivf_state, refmod
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ivf_fx(golden_dir):
    return np.load(os.path.join(golden_dir, "ivf_ref.npz"))


def _ivf(mode="reference", threads=8):
    from annvedi_b200.ivf import IVFIndex
    return IVFIndex(device=0, mode=mode, num_threads=threads)


def test_reference_mode_matches_golden(cuda, ivf_fx):
    cases, _ = mg.ivf_cases()
    for name, spec, cfgs in cases:
        w = mg.make_workload(spec["workload"])
        proj = mg.projections_from_reference(spec["n_tables"], spec["n_bits"], w.base.shape[1]) if spec["n_bits"] \
            else None
        st = ivf_state.build_state(w.base, w.centres, w.assign, spec["n_tables"], spec["n_bits"], proj)
        for ci, (k, n_probes, npc, rr, nt) in enumerate(cfgs):
            ix = _ivf(threads=nt)
            ix.import_state(st)
            ids, d = ix.search(w.queries, k, n_probes, npc, rr)
            np.testing.assert_array_equal(ids, ivf_fx[f"{name}/cfg{ci}/ids"], err_msg=f"{name} cfg{ci}")
            assert ix.total_distances_count() == int(ivf_fx[f"{name}/cfg{ci}/ndist"])
            # one query at a time through the drop-in surface gives the same ids
            if ci == 0:
                one = np.stack([ix.query(q, k, n_probes, npc, rr) for q in w.queries[:4]])
                np.testing.assert_array_equal(one, ivf_fx[f"{name}/cfg{ci}/ids"][:4])


def test_reference_mode_matches_reference_fit_state(cuda, ivf_fx):
    st = {key.split("/")[-1]: ivf_fx[key] for key in ivf_fx.files if key.startswith("reffit/state/")}
    n, d = st["original_data"].shape
    st.update(npts=n, dim=d, n_clusters=st["centroids"].shape[0], n_tables=1, n_bits=0)
    k, n_probes, npc, rr, nt = [int(v) for v in ivf_fx["reffit/params"]]
    ix = _ivf(threads=nt)
    ix.import_state(st)
    ids, _ = ix.search(ivf_fx["reffit/queries"], k, n_probes, npc, rr)
    np.testing.assert_array_equal(ids, ivf_fx["reffit/ids"])
    assert ix.total_distances_count() == int(ivf_fx["reffit/ndist"])


def test_reference_mode_matches_oracle_random_configs(cuda):
    w = synth.zipf_mixture(20000, 96, 24, c=48, lo=20, hi=2500, seed=77)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    for k, npc, rr, nt, cap in ((100, 6, 300, 16, -1), (20, 12, -1, 5, -1), (50, 48, 500, 16, 0), (1, 3, 10, 2, -1)):
        ix = _ivf(threads=nt)
        ix.import_state(st)
        ids, dd = ix.search(w.queries, k, 0, npc, rr, max_candidates=cap)
        nd = 0
        for i, q in enumerate(w.queries):
            oi, od, nc = refmod.ivf_query(st, q, k, 0, npc, rr, num_threads=nt, lanes=16, max_cands=cap)
            np.testing.assert_array_equal(ids[i], oi, err_msg=f"k={k} npc={npc} rr={rr} T={nt} q={i}")
            np.testing.assert_array_equal(dd[i], od)
            nd += nc
        assert ix.total_distances_count() == nd


def test_gpu_build_matches_reference_state(cuda):
    from annvedi_b200.ivf import IVFIndex
    w = synth.zipf_mixture(12000, 100, 8, c=40, lo=20, hi=2000, seed=31)
    ix = IVFIndex(device=0)
    ix.fit(w.base, 1, 0, 40, centroids=w.centres, assign=w.assign)
    got = ix.export_state()
    want = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    for key in ("original_data", "quantized_data", "scale", "offset", "reordered_to_original", "table_offsets"):
        np.testing.assert_array_equal(got[key], want[key], err_msg=key)
    # lists from the given centroids alone (nearest centroid) match the FP64 assignment
    ix2 = IVFIndex(device=0)
    ix2.fit(w.base, 1, 0, 40, centroids=w.centres)
    st2 = ix2.export_state()
    a64 = ivf_state.nearest_centroid(w.base, w.centres)
    sizes = np.diff(st2["table_offsets"])
    np.testing.assert_array_equal(sizes, np.bincount(a64, minlength=40))


def test_gpu_kmeans_fit_is_consistent(cuda):
    from annvedi_b200.ivf import IVFIndex
    w = synth.zipf_mixture(30000, 64, 16, c=64, lo=20, hi=3000, seed=5)
    ix = IVFIndex(device=0, mode="exact")
    ix.fit(w.base, 1, 0, 64, kmeans_iters=10)
    st = ix.export_state()
    # every row once, in list order; codes are the SQ8 encoding of the reordered rows
    assert sorted(st["reordered_to_original"].tolist()) == list(range(30000))
    np.testing.assert_array_equal(st["original_data"], w.base[st["reordered_to_original"]])
    sc, of = refmod.sq8_train(st["original_data"])
    np.testing.assert_array_equal(sc, st["scale"])
    np.testing.assert_array_equal(refmod.sq8_encode(st["original_data"], sc, of), st["quantized_data"])
    # deterministic: a second fit gives the same state
    ix2 = IVFIndex(device=0, mode="exact")
    ix2.fit(w.base, 1, 0, 64, kmeans_iters=10)
    np.testing.assert_array_equal(ix2.export_state()["centroids"], st["centroids"])
    # and it searches well
    ids, d = ix.search(w.queries, 10, 0, 16, 100)
    gt, gd = refmod.exact_topk_f64(w.base, w.queries, 10)
    assert np.mean([len(set(a) & set(b)) / 10 for a, b in zip(ids, gt)]) > 0.9


def _exact_ivf_oracle(st, queries, k, npc, R):
    """Exact-mode semantics in FP64: lists by centroid distance, full SQ8 distances of every
    candidate, best R, FP64 re-rank, best k. Returns (ids, d) with d the FP64 squared distances."""
    cen = st["centroids"].astype(np.float64)
    off = st["table_offsets"]
    codes = st["quantized_data"].astype(np.float64)
    recon = codes * st["scale"].astype(np.float64)
    orig = st["original_data"].astype(np.float64)
    out_i, out_d = [], []
    for q in queries.astype(np.float64):
        cd = ((cen - q) ** 2).sum(1)
        probes = np.lexsort((np.arange(len(cd)), cd))[:npc]
        rows = np.concatenate([np.arange(off[c], off[c + 1]) for c in probes])
        qs = q - st["offset"].astype(np.float64)
        sd = ((recon[rows] - qs) ** 2).sum(1)
        top = rows[np.lexsort((rows, sd))[:R]]
        ed = ((orig[top] - q) ** 2).sum(1)
        o = np.lexsort((top, ed))[:k]
        out_i.append(st["reordered_to_original"][top[o]])
        out_d.append(ed[o])
    return np.array(out_i), np.array(out_d)


@pytest.mark.parametrize("nq", [1, 7, 64, 300])
def test_exact_mode_matches_fp64_pipeline(cuda, nq):
    w = synth.zipf_mixture(40000, 128, nq, c=96, lo=20, hi=4000, seed=nq)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode="exact")
    ix.import_state(st)
    k, npc, R = 100, 12, 300
    ids, d = ix.search(w.queries, k, 0, npc, R)
    oi, od = _exact_ivf_oracle(st, w.queries, k, npc, R)
    from tests.helpers import fp64_dists
    got = fp64_dists(w.base, w.queries, ids)
    np.testing.assert_allclose(d, got, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(np.sort(got, 1), od, rtol=1e-5, atol=1e-6)
    agree = np.mean([len(set(a) & set(b)) / k for a, b in zip(ids, oi)])
    assert agree > 0.995


def test_exact_mode_device_tensors_and_counter(cuda):
    import torch
    w = synth.zipf_mixture(20000, 64, 50, c=32, lo=20, hi=2000, seed=3)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode="exact")
    ix.import_state(st)
    qd = torch.from_numpy(w.queries).cuda()
    a, ad = ix.search(qd, 50, 0, 8, 200)
    torch.cuda.synchronize()
    b, bd = ix.search(w.queries, 50, 0, 8, 200)
    np.testing.assert_array_equal(a.cpu().numpy(), b)
    np.testing.assert_array_equal(ad.cpu().numpy(), bd)
    # the counter adds the candidates scanned: the probed lists' sizes
    off = st["table_offsets"]
    sizes = np.diff(off)
    cd = ((st["centroids"][None].astype(np.float64) - w.queries[:, None].astype(np.float64)) ** 2).sum(-1)
    probes = np.argsort(cd, axis=1, kind="stable")[:, :8]
    assert ix.total_distances_count() == 2 * int(sizes[probes].sum())
    ix.reset_distances_count()
    assert ix.total_distances_count() == 0


def test_ivf_errors_and_facade(cuda):
    from annvedi_b200.algorithm import Algorithm
    from annvedi_b200.ivf import IVFIndex
    w = synth.zipf_mixture(5000, 32, 6, c=16, lo=20, hi=800, seed=1)
    ix = IVFIndex(device=0)
    with pytest.raises(RuntimeError):
        ix.query(w.queries[0], 5)
    with pytest.raises(RuntimeError):  # the reference's LSHIndex accepts n_bits in [0, 16] only
        ix.fit(w.base, 1, 17, 16)
    with pytest.raises(RuntimeError):
        ix.fit(w.base, 0, 8, 16)
    ix.fit(w.base, 1, 0, 16, centroids=w.centres, assign=w.assign)
    # n_bits = 0 leaves no bit to flip (lsh_index_optimized.cpp:408-426): multi-probe changes nothing
    np.testing.assert_array_equal(ix.query(w.queries[0], 5, n_probes=2), ix.query(w.queries[0], 5))
    with pytest.raises(RuntimeError):
        ix.query(w.queries[0][:5], 5)
    algo = Algorithm()
    algo.fit(w.base, backend="ivf", n_tables=1, n_bits=0, n_clusters=16)
    res = algo.query(w.queries[0], 5, n_probe_clusters=4, refine_r=50)
    assert len(res) == 5 and res.dtype == np.int64
    assert algo.get_n_distances() > 0
    algo2 = Algorithm()
    algo2.fit(w.base, backend="gpu_ivf_sq8", n_clusters=16)
    assert len(algo2.query(w.queries[1], 10, n_probe_clusters=16)) == 10


def test_reference_ivf_unit_test_shape(cuda):
    """tests/test_lsh.py::test_ivf_lsh_fit_query of the reference (with inverted lists)."""
    from annvedi_b200.algorithm import Algorithm
    data = np.random.default_rng(0).random((50, 16), dtype=np.float32)
    a = Algorithm()
    a.fit(data, backend="ivf_lsh", n_tables=1, n_bits=0, n_clusters=4)
    assert len(a.query(data[0], 5)) == 5


@pytest.mark.parametrize("mode", ["tc", "tc_sq8"])
@pytest.mark.parametrize("nq", [1, 7, 64, 300])
def test_tc_mode_ranks_the_same_streams(cuda, nq, mode):
    """The tensor-core forms rank each query's candidate stream (the same probed lists) by tensor-core keys
    -- BF16 rows ("tc"), or the SQ8 codes themselves against int8 query weights ("tc_sq8") -- before the
    exact FP32 re-rank: distances are exact for the ids returned, the result agrees with the
    exact-selection pipeline, and the distance counter counts the same candidates."""
    w = synth.zipf_mixture(40000, 128, nq, c=96, lo=20, hi=4000, seed=nq)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    k, npc, R = 100, 12, 300
    ids, d = ix.search(w.queries, k, 0, npc, R)
    oi, od = _exact_ivf_oracle(st, w.queries, k, npc, R)
    from tests.helpers import fp64_dists
    got = fp64_dists(w.base, w.queries, ids)
    np.testing.assert_allclose(d, got, rtol=1e-5, atol=1e-6)
    agree = np.mean([len(set(a) & set(b)) / k for a, b in zip(ids, oi)])
    assert agree > 0.995
    ex = _ivf(mode="exact")
    ex.import_state(st)
    ex.search(w.queries, k, 0, npc, R)
    assert ix.total_distances_count() == ex.total_distances_count()


@pytest.mark.parametrize("c", [40, 96, 700, 2048, 2050])
def test_tc_coarse_probes_the_exact_lists(cuda, c):
    """The tensor-core coarse ranking (BF16 keys to every centroid, then exact FP32 distances inside the
    keys' certified error window) probes the lists the exact FP32 ranking probes: from the keys' 32-list
    chunk minima (up to 2,048 lists; with 40 or 96 lists there are fewer chunks than probes and every
    chunk is read) and without them (2,050 lists): the same candidates are counted per query and over a
    300-query batch."""
    w = synth.zipf_mixture(20000, 64, 300, c=c, lo=5, hi=2000, seed=c)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    k, R = 20, 60
    for npc in (2, 5):
        counts = {}
        for mode in ("exact", "tc"):
            ix = _ivf(mode=mode)
            ix.import_state(st)
            per = []
            for i in range(24):
                ix.reset_distances_count()
                ix.search(w.queries[i:i + 1], k, 0, npc, R)
                per.append(ix.total_distances_count())
            ix.reset_distances_count()
            ix.search(w.queries, k, 0, npc, R)
            counts[mode] = (per, ix.total_distances_count())
        assert counts["tc"] == counts["exact"], npc


@pytest.mark.parametrize("nq,npc,R,mode", [(1200, 12, 300, "tc"), (600, 40, 100, "tc"), (256, 3, 500, "tc"),
                                           (1200, 12, 300, "tc_sq8"), (300, 20, 200, "tc_sq8")])
def test_tc_sampled_bars_select_what_the_key_stream_selects(cuda, nq, npc, R, mode):
    """Batches of 256+ queries on the tensor cores keep only keys under sampled per-query bars (a pass over
    the heads of the probed lists, re-runs under a safe bar where a query falls short); smaller batches
    select from the whole key stream. Both take each query's exact best R BF16 keys, so the same queries
    return the same ids and distances in one batch and in batches of 200."""
    from tests.helpers import assert_ids_equal_up_to_ties
    w = synth.zipf_mixture(80000, 128, nq, c=128, lo=20, hi=6000, seed=nq + npc)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    ids, d = ix.search(w.queries, 100, 0, npc, R)
    parts = [ix.search(w.queries[s:s + 200], 100, 0, npc, R) for s in range(0, nq, 200)]
    ids2 = np.concatenate([p[0] for p in parts])
    d2 = np.concatenate([p[1] for p in parts])
    assert_ids_equal_up_to_ties(w.base, w.queries, ids, ids2, rtol=1e-6)
    same = ids == ids2
    np.testing.assert_array_equal(d[same], d2[same])
    from tests.helpers import fp64_dists
    np.testing.assert_allclose(d, fp64_dists(w.base, w.queries, ids), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("mode", ["tc", "tc_sq8"])
def test_tc_sampled_bars_rerun_path(cuda, mode):
    """Lists of two rows: a query's sample is half its candidates, so about 2.3 R/3 keys pass the fast bar
    and most queries are redone under their safe bars; the result still equals the key-stream path's."""
    from tests.helpers import assert_ids_equal_up_to_ties
    rng = np.random.default_rng(5)
    base = rng.standard_normal((8192, 64)).astype(np.float32)
    base /= np.linalg.norm(base, axis=1, keepdims=True)
    q = base[rng.integers(0, 8192, 300)] + 0.05 * rng.standard_normal((300, 64)).astype(np.float32)
    q = np.ascontiguousarray(q / np.linalg.norm(q, axis=1, keepdims=True), np.float32)
    st = ivf_state.build_state(base, np.ascontiguousarray(base[::2]), np.arange(8192) // 2, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    ids, d = ix.search(q, 100, 0, 400, 300)
    parts = [ix.search(q[s:s + 150], 100, 0, 400, 300) for s in range(0, 300, 150)]
    ids2 = np.concatenate([p[0] for p in parts])
    assert_ids_equal_up_to_ties(base, q, ids, ids2, rtol=1e-6)
    from tests.helpers import fp64_dists
    np.testing.assert_allclose(d, fp64_dists(base, q, ids), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("mode", ["tc", "tc_sq8"])
def test_tc_mode_over_all_lists_is_exact(cuda, mode):
    """Probing every list makes each candidate stream the whole base: the result is the exact top-k."""
    import torch
    from tests.helpers import check_exact_topk
    w = synth.zipf_mixture(60000, 96, 80, c=64, lo=20, hi=6000, seed=9)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    ids, d = ix.search(torch.from_numpy(w.queries).cuda(), 50, 0, 64, 400)
    torch.cuda.synchronize()
    check_exact_topk(w.base, w.queries, ids.cpu().numpy(), d.cpu().numpy(), 50)


def _lsh_state(seed=3, n=12000, d=64, c=24, T=3, B=4):
    w = synth.zipf_mixture(n, d, 40, c=c, lo=20, hi=2000, seed=seed)
    proj = mg.projections_from_reference(T, B, d)
    return w, ivf_state.build_state(w.base, w.centres, w.assign, T, B, proj)


def test_lsh_reference_mode_matches_oracle(cuda):
    """Bucket tables (3 tables of 4 bits) in the reference's semantics: the candidate streams (exact and
    multiprobe buckets, caps at bucket granularity, fallback to every row), the per-chunk heaps and the
    re-rank give the oracle's ids, distances and counter."""
    w, st = _lsh_state()
    for k, n_probes, npc, rr, nt, cap in ((10, 0, 4, 40, 4, -1), (50, 3, 6, 200, 8, -1), (20, 6, 3, -1, 3, 0),
                                          (100, 2, 2, 300, 16, -1)):
        ix = _ivf(threads=nt)
        ix.import_state(st)
        ids, dd = ix.search(w.queries, k, n_probes, npc, rr, max_candidates=cap)
        nd = 0
        for i, q in enumerate(w.queries):
            oi, od, nc = refmod.ivf_query(st, q, k, n_probes, npc, rr, num_threads=nt, lanes=16, max_cands=cap)
            np.testing.assert_array_equal(ids[i], oi, err_msg=f"k={k} probes={n_probes} npc={npc} q={i}")
            np.testing.assert_array_equal(dd[i], od)
            nd += nc
        assert ix.total_distances_count() == nd


def test_lsh_reference_mode_every_row_fallback(cuda):
    """Sparse buckets (8 bits over ~500-row lists): streams shorter than k become every row
    (lsh_index_optimized.cpp:453-457). Those queries are redone with a full-length scratch; a batch with
    both kinds matches the oracle query by query."""
    w, st = _lsh_state(seed=5, T=1, B=8)
    n = w.base.shape[0]
    for k, n_probes, npc, rr, nt in ((40, 0, 1, 60, 4), (100, 0, 2, -1, 16), (30, 1, 1, 60, 8)):
        ix = _ivf(threads=nt)
        ix.import_state(st)
        ids, dd = ix.search(w.queries, k, n_probes, npc, rr)
        counts = []
        for i, q in enumerate(w.queries):
            oi, od, nc = refmod.ivf_query(st, q, k, n_probes, npc, rr, num_threads=nt, lanes=16)
            np.testing.assert_array_equal(ids[i], oi, err_msg=f"k={k} probes={n_probes} q={i}")
            np.testing.assert_array_equal(dd[i], od)
            counts.append(nc)
        assert ix.total_distances_count() == sum(counts)
        assert any(c == n for c in counts) and any(c < n for c in counts), "not a mixed batch"


def test_lsh_candidate_walks_agree(cuda):
    """A query's candidate stream, and so its result, does not depend on its batch: a batch of 700 and the
    same queries 50 at a time return identical ids, distances and counts (reference semantics: caps, flips,
    per-chunk heaps)."""
    w = synth.zipf_mixture(12000, 64, 700, c=24, lo=20, hi=2000, seed=6)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 3, 6, mg.projections_from_reference(3, 6, 64))
    for n_probes, npc, rr, cap in ((3, 6, 40, -1), (0, 10, -1, -1), (6, 4, 100, 0)):
        big = _ivf(threads=8)
        big.import_state(st)
        ids, d = big.search(w.queries, 20, n_probes, npc, rr, max_candidates=cap)
        small = _ivf(threads=8)
        small.import_state(st)
        for s0 in range(0, 700, 50):
            i2, d2 = small.search(w.queries[s0:s0 + 50], 20, n_probes, npc, rr, max_candidates=cap)
            np.testing.assert_array_equal(ids[s0:s0 + 50], i2, err_msg=f"probes={n_probes} npc={npc} s0={s0}")
            np.testing.assert_array_equal(d[s0:s0 + 50], d2)
        assert big.total_distances_count() == small.total_distances_count()


def test_lsh_exact_mode_every_row_batch_equals_alone(cuda):
    """Exact selection in a large batch redoes its every-row queries apart, split over the whole GPU:
    each query's ids and distances equal those of the query run alone."""
    w = synth.zipf_mixture(12000, 64, 120, c=24, lo=20, hi=2000, seed=5)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 8, mg.projections_from_reference(1, 8, 64))
    ix = _ivf(mode="exact")
    ix.import_state(st)
    k, n_probes, npc, rr = 40, 0, 1, 60
    ids, d = ix.search(w.queries, k, n_probes, npc, rr, max_candidates=-1)
    every = 0
    for i in range(len(w.queries)):
        ix.reset_distances_count()
        oi, od = ix.search(w.queries[i:i + 1], k, n_probes, npc, rr, max_candidates=-1)
        every += ix.total_distances_count() == w.base.shape[0]
        np.testing.assert_array_equal(ids[i], oi[0], err_msg=f"q={i}")
        np.testing.assert_array_equal(d[i], od[0])
    assert 0 < every < len(w.queries), every


def test_lsh_exact_mode_and_state_round_trip(cuda):
    """Exact selection over the bucket streams: exact FP32 distances for the ids returned, and the ids of
    an exact selection over the same candidates; export gives back the imported tables."""
    w, st = _lsh_state(seed=8)
    ix = _ivf(mode="exact")
    ix.import_state(st)
    got = ix.export_state()
    for key in ("projections", "mean", "table_offsets", "table_ids", "original_data"):
        np.testing.assert_array_equal(got[key], st[key], err_msg=key)
    k, n_probes, npc, rr = 20, 3, 6, 200
    ids, d = ix.search(w.queries, k, n_probes, npc, rr, max_candidates=0)
    from tests.helpers import fp64_dists
    np.testing.assert_allclose(d, fp64_dists(w.base, w.queries, ids), rtol=1e-5, atol=1e-6)
    # the reference semantics over the same streams, with the 64-heap, keeps a subset of what exact keeps
    ref = _ivf(mode="reference", threads=1)
    ref.import_state(st)
    rid, _ = ref.search(w.queries, k, n_probes, npc, rr, max_candidates=0)
    assert np.mean([len(set(a) & set(b)) / k for a, b in zip(ids, rid)]) > 0.9


def test_lsh_gpu_build_matches_reference_tables(cuda):
    """The GPU build of 3 tables of 4 bits over given lists: the reference's projections (mt19937(42),
    N(0,1), Gram-Schmidt) and bucket tables, up to rows on a hyperplane within rounding."""
    from annvedi_b200.ivf import IVFIndex
    w = synth.zipf_mixture(12000, 64, 8, c=24, lo=20, hi=2000, seed=3)
    ix = IVFIndex(device=0)
    ix.fit(w.base, 3, 4, 24, centroids=w.centres, assign=w.assign)
    got = ix.export_state()
    want = ivf_state.build_state(w.base, w.centres, w.assign, 3, 4, mg.projections_from_reference(3, 4, 64))
    np.testing.assert_allclose(got["projections"], want["projections"], atol=1e-5)
    np.testing.assert_allclose(got["mean"], want["mean"], atol=1e-6)

    def bucket_of_row(stt):
        off, ids = stt["table_offsets"], stt["table_ids"]
        out = np.empty(ids.shape[0], np.int64)
        out[ids + np.repeat(np.arange(3) * 12000, 12000)] = np.repeat(np.arange(off.shape[0] - 1), np.diff(off))
        return out

    same = np.mean(bucket_of_row(got) == bucket_of_row(want))
    assert same > 0.999, same


@pytest.mark.parametrize("mode", ["tc", "tc_sq8"])
def test_sample_divisor_does_not_change_results(cuda, mode):
    """The sampled bars over 1/4, 1/8 or 1/16 of each probed list (ANN_IVF_OPT_SAMPLE_DIV) only prune: the
    result is the same id for id and bit for bit; out-of-range values are refused."""
    w = synth.zipf_mixture(60000, 128, 3000, c=128, lo=20, hi=5000, seed=31)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    want_i, want_d = ix.search(w.queries, 100, 0, 6, 150)
    for div in (4, 16, 2):
        ix.set_option("sample_div", div)
        got_i, got_d = ix.search(w.queries, 100, 0, 6, 150)
        np.testing.assert_array_equal(got_i, want_i)
        np.testing.assert_array_equal(got_d, want_d)
    with pytest.raises(Exception):
        ix.set_option("sample_div", 1)
    with pytest.raises(Exception):
        ix.set_option("sampled_min_queries", 0)


def test_kernel_timers_count_the_profiled_launches(cuda):
    """ann_ivf_kernel_profile: CUDA-event times of the list-keys, bars, selection and re-rank launches of
    the profiled calls, cleared by reset_profile_results."""
    import torch
    w = synth.zipf_mixture(40000, 128, 600, c=96, lo=20, hi=4000, seed=8)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode="tc")
    ix.import_state(st)
    q = torch.from_numpy(w.queries).cuda()
    ix.search(q, 100, 0, 8, 200)
    ix.reset_profile_results()
    ix.set_profiling(True)
    for _ in range(3):
        ix.search(q, 100, 0, 8, 200)
    ix.set_profiling(False)
    kt = ix.get_kernel_times()
    assert kt["keys"]["launches"] == 3 and kt["select"]["launches"] == 3 and kt["rerank"]["launches"] == 3
    assert kt["bars"]["launches"] == 3
    assert all(v["ms"] > 0 for v in kt.values())
    ix.reset_profile_results()
    assert all(v["launches"] == 0 for v in ix.get_kernel_times().values())


@pytest.mark.parametrize("mode", ["exact", "tc"])
def test_batch_with_every_row_queries_equals_alone(cuda, mode):
    """A batch of 300 queries, some of whose probed lists hold fewer than k rows (those scan every row, as
    the reference does): the batch sets them apart after its own set-up and redoes them over the whole GPU;
    every query's ids and distances equal those of the query run alone."""
    from tests.helpers import assert_ids_equal_up_to_ties
    w = synth.zipf_mixture(30000, 64, 300, c=300, lo=5, hi=1500, seed=12)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode=mode)
    ix.import_state(st)
    k, npc, rr = 40, 1, 100
    ids, d = ix.search(w.queries, k, 0, npc, rr)
    alone_i, alone_d, every = [], [], 0
    for i in range(len(w.queries)):
        ix.reset_distances_count()
        oi, od = ix.search(w.queries[i:i + 1], k, 0, npc, rr)
        every += ix.total_distances_count() == w.base.shape[0]
        alone_i.append(oi[0])
        alone_d.append(od[0])
    assert 0 < every < len(w.queries), every
    assert_ids_equal_up_to_ties(w.base, w.queries, ids, np.stack(alone_i), rtol=1e-6)
    np.testing.assert_allclose(d, np.stack(alone_d), rtol=1e-6, atol=1e-7)


def test_host_search_into_callers_page_locked_arrays(cuda):
    """Host queries may give their own output arrays (page-locked torch CPU tensors or numpy arrays): the
    search writes them and returns them, equal to a search that allocates its own; wrong shapes or types
    are refused."""
    import torch
    w = synth.zipf_mixture(30000, 64, 500, c=64, lo=20, hi=3000, seed=21)
    st = ivf_state.build_state(w.base, w.centres, w.assign, 1, 0)
    ix = _ivf(mode="tc")
    ix.import_state(st)
    want_i, want_d = ix.search(w.queries, 50, 0, 4, 100)
    oi = torch.empty(500, 50, dtype=torch.int64, pin_memory=True)
    od = torch.empty(500, 50, dtype=torch.float32, pin_memory=True)
    got_i, got_d = ix.search(w.queries, 50, 0, 4, 100, out_ids=oi, out_dists=od)
    np.testing.assert_array_equal(got_i, want_i)
    np.testing.assert_array_equal(oi.numpy(), want_i)
    np.testing.assert_array_equal(od.numpy(), want_d)
    with pytest.raises(RuntimeError):
        ix.search(w.queries, 50, 0, 4, 100, out_ids=np.empty((500, 49), np.int64))
    with pytest.raises(RuntimeError):
        ix.search(w.queries, 50, 0, 4, 100, out_ids=np.empty((500, 50), np.int32))
