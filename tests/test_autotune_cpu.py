"""Host logic of the autotuner (annvedi_b200/autotune.py) on the CPU: a fake index whose recall and cost
follow set rules, timed by a fake timer, so that the tuner's choices can be checked against the rules it
states -- per (mode, refine_r) the probe counts rise until the recall target is met, the fastest passing
point wins, the tensor-core forms then sweep their sample share and keep the fastest on the index, and the
exact scan keeps its fastest query tile."""
import numpy as np
import pytest
import torch

from annvedi_b200 import autotune


def _workload(n=400, d=8, nq=12, k=10, seed=5):
    rng = np.random.default_rng(seed)
    base = rng.standard_normal((n, d))
    queries = rng.standard_normal((nq, d))
    dist = ((queries[:, None, :] - base[None]) ** 2).sum(-1)
    order = np.argsort(dist, axis=1, kind="stable")
    kth = np.take_along_axis(dist, order[:, k - 1:k], 1)[:, 0]
    far = order[:, -k:]  # the k farthest rows: outside every query's k nearest
    return (torch.from_numpy(base), torch.from_numpy(queries), torch.from_numpy(kth), order[:, :k], far)


def recall_rule(mode, npc, rr):
    """the share of the true k nearest a point returns (tenths, so that recall is exact)"""
    return min(10, npc + rr // 100 + (1 if mode == "tc" else 0)) / 10


def cost_rule(mode, npc, rr, div):
    return npc * 1.0 + rr * 0.01 + (0.0 if mode == "tc" else 3.0) + (0.0 if div is None else abs(div - 16) * 0.05)


class FakeIVF:
    def __init__(self, near, far):
        self.near, self.far = near, far
        self.div = 8
        self.last = None
        self.set_calls = []

    def set_option(self, name, value):
        assert name == "sample_div"
        self.div = value
        self.set_calls.append(value)

    def search(self, queries, k, n_probes, npc, rr, max_candidates=0, mode="tc", out_ids=None, out_dists=None):
        good = int(round(recall_rule(mode, npc, rr) * k))
        ids = np.concatenate([self.near[:, :good], self.far[:, :k - good]], axis=1)
        out_ids.copy_(torch.from_numpy(ids))
        out_dists.zero_()
        self.last = (mode, npc, rr, self.div if mode in ("tc", "tc_sq8") else None)


def test_tune_ivf_picks_the_fastest_point_meeting_the_target():
    base, queries, kth, near, far = _workload()
    ix = FakeIVF(near, far)
    calls = []

    def timer(fn, reps):
        fn()
        calls.append(ix.last)
        return cost_rule(*ix.last)

    nprobes, refines, divs = (1, 2, 3, 4, 6, 8), (100, 200, 300), (4, 8, 16)
    out = autotune.tune_ivf(ix, base, queries, kth, k=10, target=0.7, modes=("tc", "exact"), nprobes=nprobes,
                            refines=refines, reps=1, sample_divs=divs, timer=timer)
    # per (mode, refine_r): probe counts tried in order up to the first that meets the target
    want_rows = []
    for mode in ("tc", "exact"):
        for rr in refines:
            for npc in nprobes:
                want_rows.append((mode, npc, rr))
                if recall_rule(mode, npc, rr) >= 0.7:
                    break
    got_rows = [(r["mode"], r["nprobe"], r["refine_r"]) for r in out["table"][:len(want_rows)]]
    assert got_rows == want_rows
    assert all(r.get("sample_div") in (4, 16) for r in out["table"][len(want_rows):])  # then the share sweep
    for r in out["table"]:
        assert r["recall"] == pytest.approx(recall_rule(r["mode"], r["nprobe"], r["refine_r"]))
    # the fastest passing point of each mode, then the tensor-core form's sample share swept at it
    passing = [row for row in want_rows if recall_rule(*row) >= 0.7]
    best_exact = min((r for r in passing if r[0] == "exact"), key=lambda r: cost_rule(*r, None))
    best_tc = min((r for r in passing if r[0] == "tc"), key=lambda r: cost_rule(*r, 8))
    assert (out["best_by_mode"]["exact"]["nprobe"], out["best_by_mode"]["exact"]["refine_r"]) == best_exact[1:]
    tc = out["best_by_mode"]["tc"]
    assert (tc["nprobe"], tc["refine_r"]) == best_tc[1:]
    assert tc["sample_div"] == 16  # the cheapest share under cost_rule
    assert ix.set_calls[-1] == 16  # and it is left set on the index
    assert [c[3] for c in calls if c[0] == "tc" and c[1:3] == best_tc[1:3]][-2:] == [4, 16]
    assert out["best"]["mode"] == "tc"
    assert out["best"]["qps"] == max(r["qps"] for r in out["best_by_mode"].values())


def test_tune_ivf_without_a_passing_point():
    base, queries, kth, near, far = _workload()
    ix = FakeIVF(near, far)
    out = autotune.tune_ivf(ix, base, queries, kth, k=10, target=1.01, modes=("exact",), nprobes=(1, 2),
                            refines=(100,), reps=1, timer=lambda fn, reps: (fn(), 1.0)[1])
    assert out["best"] is None and out["best_by_mode"] == {}
    assert len(out["table"]) == 2


class FakeLinear:
    def __init__(self):
        self.tile = 0

    def set_query_tile(self, t):
        self.tile = t

    def search(self, queries, k, mode="exact", out_ids=None, out_dists=None):
        out_ids.zero_()


def test_tune_flat_tile_keeps_the_fastest_tile():
    ix = FakeLinear()
    q = torch.zeros(40, 8)
    cost = {8: 3.0, 16: 1.5, 32: 2.0}
    out = autotune.tune_flat_tile(ix, q, k=5, tiles=(8, 16, 32), reps=1,
                                  timer=lambda fn, reps: (fn(), cost[ix.tile])[1])
    assert [r["tile"] for r in out["table"]] == [8, 16, 32]
    assert out["best"]["tile"] == 16 and ix.tile == 16
