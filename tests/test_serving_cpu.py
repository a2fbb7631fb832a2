"""Host logic of the serving scheduler (annvedi_b200/serving.py, Server._take) on the CPU: which pending
requests form the next batch, and how admission against free device memory cuts, delays or refuses it.
The server is built without its CUDA streams (only the scheduling state), with fake workspaces."""
import collections
import threading

import numpy as np

from annvedi_b200 import serving


class FakeWorkspace:
    def __init__(self, nbytes):
        self._n = nbytes

    def nbytes(self):
        return self._n


def _route(name, per_query, dim=4):
    return serving.Route(name=name, dim=dim, search=None, scratch_bytes=lambda nq: nq * per_query)


def _server(routes, max_batch=64, free=1000, reserve=100):
    s = serving.Server.__new__(serving.Server)  # the scheduling state only: no streams, no device
    s.routes = {r.name: r for r in routes}
    s.max_batch = max_batch
    s.hbm_reserve = reserve
    s._pending = {r.name: collections.deque() for r in routes}
    s._cv = threading.Condition()
    s._growth_in_flight = 0
    s._free_seen = free
    s.in_flight = 0
    s.admission_waits = 0
    return s


def _req(route, nq, k=100, at=0.0):
    r = serving.Request(route, np.zeros((nq, 4), np.float32), k)
    r.arrival = at
    return r


def test_oldest_route_first_and_same_k_runs_batched_up_to_max_batch():
    s = _server([_route("a", 1), _route("b", 1)], max_batch=20)
    s._pending["b"].extend([_req("b", 5, at=1.0), _req("b", 5, at=2.0)])
    s._pending["a"].extend([_req("a", 8, at=1.5), _req("a", 8, at=1.6), _req("a", 8, at=1.7)])
    name, reqs, growth = s._take({"ws": FakeWorkspace(10 ** 6)})
    assert name == "b" and [r.arrival for r in reqs] == [1.0, 2.0] and growth == 0
    name, reqs, _ = s._take({"ws": FakeWorkspace(10 ** 6)})
    assert name == "a" and len(reqs) == 2  # 8 + 8 <= 20 < 8 + 8 + 8
    name, reqs, _ = s._take({"ws": FakeWorkspace(10 ** 6)})
    assert name == "a" and len(reqs) == 1
    assert s._take({"ws": FakeWorkspace(10 ** 6)}) is None


def test_a_different_k_ends_the_batch():
    s = _server([_route("a", 1)])
    s._pending["a"].extend([_req("a", 2, k=10), _req("a", 2, k=10), _req("a", 2, k=50), _req("a", 2, k=10)])
    _, reqs, _ = s._take({"ws": FakeWorkspace(10 ** 6)})
    assert [r.k for r in reqs] == [10, 10]
    _, reqs, _ = s._take({"ws": FakeWorkspace(10 ** 6)})
    assert [r.k for r in reqs] == [50]


def test_admission_admits_fewer_requests_when_the_workspace_must_grow():
    # 50 bytes of scratch a query, 200 held: 900 bytes above the reserve allow 16 queries, not 24
    s = _server([_route("a", 50)], free=1000, reserve=100)
    s._pending["a"].extend([_req("a", 8, at=i) for i in range(4)])
    name, reqs, growth = s._take({"ws": FakeWorkspace(200)})
    assert len(reqs) == 2 and growth == 16 * 50 - 200
    assert len(s._pending["a"]) == 2


def test_admission_waits_while_batches_in_flight_can_free_memory():
    s = _server([_route("a", 200)], free=1000, reserve=100)
    s._pending["a"].append(_req("a", 8))
    s.in_flight = 1
    assert s._take({"ws": FakeWorkspace(200)}) is None
    assert s.admission_waits == 1 and len(s._pending["a"]) == 1


def test_a_request_that_can_never_fit_is_refused_and_the_next_runs():
    s = _server([_route("a", 200)], free=1000, reserve=100)
    big, small = _req("a", 8, at=0.0), _req("a", 2, at=1.0)
    s._pending["a"].extend([big, small])
    name, reqs, growth = s._take({"ws": FakeWorkspace(200)})
    assert big.error and "bytes of scratch" in big.error and big.wait(0)
    assert reqs == [small] and growth == 2 * 200 - 200
