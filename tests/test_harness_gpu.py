"""The plugin through the h5py-free runner, as the competition harness drives it: one query per call, the
scenario's parameters, get_n_distances, then the evaluator's recall; the batched loop gives the same
neighbours and distance count."""
import textwrap

import numpy as np
import pytest

from annvedi_b200 import harness, synth

pytestmark = pytest.mark.gpu

SCEN = textwrap.dedent("""
    scenarios:
      exact:
        default:
          index_params: {backend: linear}
      fast:
        default:
          index_params: {backend: ivf_lsh, n_tables: 15, n_bits: 8, n_clusters: 32}
          query_params: {n_probes: 6, n_probe_clusters: 12, refine_r: 50}
""")


@pytest.fixture(scope="module")
def dataset():
    w = synth.zipf_mixture(20000, 48, 60, c=32, lo=20, hi=3000, seed=11)
    return {"train": w.base, "test": w.queries}


def test_linear_scenario(cuda, dataset, tmp_path):
    f = tmp_path / "scenarios.yaml"
    f.write_text(SCEN)
    params = harness.load_scenario(str(f), "exact", "zipf-48")
    res = harness.run(harness.load_algorithm_class(), dataset, params, k=10, log=lambda *_: None)
    assert res["n_dist_queries"] == 20000 * 60  # the reference's linear counter: N per query
    m = harness.evaluate(dataset, res, 10)
    assert m["avg_recall"] == 1.0  # k <= 64: the reference's ranking is the exact one


def test_ivf_lsh_scenario_per_query_and_batched(cuda, dataset, tmp_path):
    f = tmp_path / "scenarios.yaml"
    f.write_text(SCEN)
    params = harness.load_scenario(str(f), "fast", "zipf-48")
    cls = harness.load_algorithm_class()
    one = harness.run(cls, dataset, params, k=10, log=lambda *_: None)
    many = harness.run(cls, dataset, params, k=10, batch=16, log=lambda *_: None)
    np.testing.assert_array_equal(one["neighbors"], many["neighbors"])
    assert one["n_dist_queries"] == many["n_dist_queries"] > 0
    m = harness.evaluate(dataset, one, 10)
    assert m["avg_recall"] > 0.5, m["avg_recall"]
