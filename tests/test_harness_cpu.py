"""The h5py-free runner and scoring (annvedi_b200.harness) on the CPU, with a brute-force stand-in for the
plugin: scenario resolution and its errors (orthogonal-competition/harness.py:73-114), the result-shape
check (:160-166), the results file, and the evaluator's recall (evaluator.py:149-157)."""
import os
import textwrap

import numpy as np
import pytest

from annvedi_b200 import harness

SCEN = textwrap.dedent("""
    scenarios:
      fast:
        default:
          index_params: {n_tables: 15, n_bits: 8, n_clusters: 128}
          query_params: {n_probes: 6, n_probe_clusters: 12, refine_r: 50}
        tiny-64:
          index_params: {n_clusters: 4}
      nodefault:
        other-set:
          index_params: {}
""")


class BruteForce:
    """Exact top-k in numpy; counts N distances per query like the reference linear scan."""

    def __init__(self):
        self.x = None
        self.nd = 0

    def fit(self, train, **params):
        self.x = np.asarray(train, np.float64)
        self.params = params

    def query(self, q, k, **params):
        d = ((self.x - q) ** 2).sum(1)
        self.nd += self.x.shape[0]
        return np.lexsort((np.arange(len(d)), d))[:k]

    def query_batch(self, qs, k, **params):
        return np.stack([self.query(q, k) for q in qs])

    def get_n_distances(self):
        return self.nd


class WrongShape(BruteForce):
    def query(self, q, k, **params):
        return super().query(q, k)[:-1]


def _data(n=600, d=16, q=25, seed=0):
    rng = np.random.default_rng(seed)
    return {"train": rng.standard_normal((n, d)).astype(np.float32),
            "test": rng.standard_normal((q, d)).astype(np.float32)}


def test_scenario_resolution(tmp_path):
    f = tmp_path / "scenarios.yaml"
    f.write_text(SCEN)
    p = harness.load_scenario(str(f), "fast", "tiny-64")
    assert p == {"index_params": {"n_clusters": 4}, "query_params": {}}
    p = harness.load_scenario(str(f), "fast", "sift-128")
    assert p["index_params"] == {"n_tables": 15, "n_bits": 8, "n_clusters": 128}
    assert p["query_params"]["n_probes"] == 6
    with pytest.raises(ValueError, match="not found"):
        harness.load_scenario(str(f), "missing", "x")
    with pytest.raises(ValueError, match="no 'default' fallback"):
        harness.load_scenario(str(f), "nodefault", "x")


def test_run_evaluate_and_results_file(tmp_path):
    data = _data()
    k = 10
    res = harness.run(BruteForce, data, {"index_params": {}, "query_params": {}}, k=k, log=lambda *_: None)
    assert res["neighbors"].dtype == np.int32 and res["neighbors"].shape == (25, k)
    assert res["n_dist_queries"] == 600 * 25
    td, tn = harness.true_distances(data["train"], data["test"], k)
    np.testing.assert_array_equal(res["neighbors"], tn)
    m = harness.evaluate(data, res, k)
    assert m["avg_recall"] == 1.0 and m["qps"] > 0
    path = str(tmp_path / "res" / "results.npz")
    harness.save_results(path, res)
    back = harness.load_results(path)
    np.testing.assert_array_equal(back["neighbors"], res["neighbors"])
    assert back["n_dist_queries"] == res["n_dist_queries"]
    # batched loop: same neighbours, every query charged its batch's share
    rb = harness.run(BruteForce, data, {"index_params": {}, "query_params": {}}, k=k, batch=8, log=lambda *_: None)
    np.testing.assert_array_equal(rb["neighbors"], res["neighbors"])
    # a wrong result shape is the harness's ValueError
    with pytest.raises(ValueError, match="length k=10"):
        harness.run(WrongShape, data, {"index_params": {}, "query_params": {}}, k=k, log=lambda *_: None)


def test_recall_definition():
    td = np.array([[1.0, 2.0, 3.0], [1.0, 1.0, 1.0]])
    pd = np.array([[1.0, 3.0, 3.5], [0.5, 1.0, 2.0]])
    np.testing.assert_allclose(harness.recalls(td, pd, 3), [2 / 3, 2 / 3])
    # evaluator semantics: -1 ids are misses
    data = _data(n=50, q=2)
    res = {"neighbors": np.array([[0, -1], [1, 2]], np.int32), "query_times": np.ones(2), "build_time": 0.0,
           "n_dist_queries": 0, "index_mem_mb": 0.0}
    m = harness.evaluate(data, res, 2)
    assert m["avg_recall"] <= 0.75


def test_cli_and_algorithm_file(tmp_path):
    data = _data(q=8)
    ds = str(tmp_path / "tiny-64.npz")
    harness.save_dataset(ds, data["train"], data["test"])
    (tmp_path / "scenarios.yaml").write_text(SCEN)
    algo = tmp_path / "algorithm.py"
    algo.write_text("import sys\nsys.path.insert(0, %r)\nfrom tests.test_harness_cpu import BruteForce as Algorithm\n"
                    % os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    out = str(tmp_path / "results.npz")
    assert harness.main(["--dataset", ds, "--results", out, "--scenario", "fast", "--scenarios-file",
                         str(tmp_path / "scenarios.yaml"), "--algorithm-file", str(algo), "--k", "5",
                         "--evaluate"]) == 0
    assert harness.load_results(out)["neighbors"].shape == (8, 5)
    bad = tmp_path / "bad.py"
    bad.write_text("class Algorithm:\n    def fit(self, x): pass\n")
    with pytest.raises(ImportError, match="query"):
        harness.load_algorithm_class(str(bad))
