"""Serving loop: continuous batching of search requests against device-resident indexes.

The reference has no server: its harness calls ``Algorithm.query`` once per query from one thread
(orthogonal-competition/harness.py:141-176). This module is the serving form of the same search
path. Requests (a batch of queries for one resident index) arrive at any time and are queued per
index. A fixed set of GPU workers, each with its own CUDA stream, workspace and pinned host
buffers, takes work as it frees up: a free worker takes every queued request of the index whose
oldest request has waited longest (FIFO within the index), up to ``max_batch`` queries, provided the
scratch the batch needs fits in free device memory (admission by free HBM). Requests that arrive
while others are on the GPU are admitted as soon as a worker and memory free up; batches on
different workers run concurrently on the device (their streams overlap), and a worker's own host
work (splitting results, copying the next batch in) overlaps the others' kernels.

Each query's result does not depend on which requests it was batched with: the exact search forms
are per-query computations (the tensor-core form's bars and survivors are per query; the plain scan
is exact), and the IVF form differs between batch sizes only in the summation order of the SQ8
candidate keys, which can move a candidate across the re-rank depth R only at ties.

Latency of a request = completion time - arrival time (host clock), reported as p50 / p99 beside
the sustained throughput in queries per second.
"""
from __future__ import annotations

import collections
import gc
import threading
import time
from dataclasses import dataclass, field
from typing import Callable

import numpy as np


@dataclass
class Route:
    """A resident index the server routes requests to.

    search(queries_dev, k, stream, workspace, out_ids, out_dists) -> (ids_dev int64 [nq, k], dists_dev
        float32 [nq, k]), written into the given device tensors
    scratch_bytes(nq) -> device scratch (bytes) a call with nq queries needs in its workspace.
    """
    name: str
    dim: int
    search: Callable
    scratch_bytes: Callable[[int], int]


@dataclass
class Request:
    route: str
    queries: np.ndarray  # float32 [b, dim]
    k: int
    arrival: float = field(default_factory=time.perf_counter)
    ids: np.ndarray | None = None
    dists: np.ndarray | None = None
    done_at: float | None = None
    batch_queries: int = 0  # size of the batch the request ran in
    error: str | None = None  # set when the request could not be served
    _event: threading.Event = field(default_factory=threading.Event)

    def wait(self, timeout: float | None = None) -> bool:
        return self._event.wait(timeout)

    @property
    def latency_ms(self) -> float:
        return (self.done_at - self.arrival) * 1e3 if self.done_at is not None else float("nan")


class Server:
    """Continuous-batching request loop over device-resident indexes (see the module docstring).

    workers      concurrent GPU batches (one CUDA stream and workspace each)
    max_batch    queries per batch at most
    hbm_reserve  bytes of device memory left free by admission
    """

    def __init__(self, routes: list[Route], device: int = 0, workers: int = 3, max_batch: int = 4096,
                 hbm_reserve: int = 2 << 30):
        import torch
        from .linear import Workspace
        self.routes = {r.name: r for r in routes}
        self.device = device
        self.max_batch = int(max_batch)
        self.hbm_reserve = int(hbm_reserve)
        self._pending: dict[str, collections.deque] = {r.name: collections.deque() for r in routes}
        self._cv = threading.Condition()
        self._running = False
        self._threads: list[threading.Thread] = []
        self._growth_in_flight = 0  # workspace growth promised to admitted batches not yet allocated
        self._workers = [{"stream": torch.cuda.Stream(device=device), "ws": Workspace(device), "pin": {}}
                         for _ in range(workers)]
        self.completed: list[Request] = []
        self.batches: list[tuple[str, int, int, float, float]] = []  # (route, queries, requests, start, end)
        self.admission_waits = 0
        # Free device memory as admission sees it: read from the driver at start and after a batch that
        # grew its workspace (outside the scheduling lock), lowered by the growth granted meanwhile. A
        # driver query under the lock on every batch stalled every worker whenever it was slow (tens of
        # ms while other threads launch and synchronise).
        self._free_seen = 0
        self._free_read_at = 0.0
        self.free_reads = 0
        self.in_flight = 0
        self.max_in_flight = 0  # most batches on the GPU at once
        self.errors: list[BaseException] = []

    # ---- client side ----------------------------------------------------------------------
    def submit(self, route: str, queries, k: int = 100) -> Request:
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim == 1:
            q = q[None, :]
        r = self.routes.get(route)
        if r is None:
            raise KeyError(f"unknown route {route!r}")
        if q.shape[1] != r.dim:
            raise RuntimeError(f"query length {q.shape[1]} != index dim {r.dim}")
        if q.shape[0] > self.max_batch:
            raise RuntimeError(f"request of {q.shape[0]} queries > max_batch {self.max_batch}")
        req = Request(route, q, int(k))
        with self._cv:
            self._pending[route].append(req)
            self._cv.notify()
        return req

    def start(self, prewarm: bool = True) -> "Server":
        """Starts the workers. The first call of each route runs here on one thread (one-time set-up
        such as the BF16 copy is not raced). With prewarm, every worker then runs a full max_batch
        batch of random unit queries on every route, so its workspace already has the size of the
        largest batch: a workspace that grows mid-stream frees and reallocates device memory, which
        stalls every stream on the device."""
        import torch
        dev = f"cuda:{self.device}"
        for r in self.routes.values():
            w = self._workers[0]
            x = torch.zeros(1, r.dim, dtype=torch.float32, device=dev)
            r.search(x, 1, w["stream"], w["ws"], None, None)
            w["stream"].synchronize()
        if prewarm:
            g = torch.Generator(device=dev).manual_seed(0)
            for w in self._workers:
                for r in self.routes.values():
                    _, _, _, dev_in, dev_ids, dev_d = self._pinned(w, r, 100)
                    dev_in.copy_(torch.nn.functional.normalize(
                        torch.randn(self.max_batch, r.dim, generator=g, device=dev), dim=1))
                    with torch.cuda.stream(w["stream"]):
                        r.search(dev_in, 100, w["stream"], w["ws"], dev_ids, dev_d)
                    w["stream"].synchronize()
        # Objects that live for the whole run (indexes, buffers, queued traffic) leave the collected
        # generations, so a full collection does not pause the workers for milliseconds.
        gc.collect()
        gc.freeze()
        self._refresh_free()
        self._running = True
        for i in range(len(self._workers)):
            t = threading.Thread(target=self._work, args=(i,), daemon=True, name=f"ann-serve-{i}")
            t.start()
            self._threads.append(t)
        return self

    def stop(self):
        with self._cv:
            self._running = False
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        self._threads = []
        if self.errors:
            raise self.errors[0]

    # ---- scheduling ------------------------------------------------------------------------
    def _refresh_free(self) -> None:
        """Reads free device memory from the driver; never called with the scheduling lock held."""
        import torch
        free, _ = torch.cuda.mem_get_info(self.device)
        with self._cv:
            self._free_seen = int(free)
            self._free_read_at = time.perf_counter()
            self.free_reads += 1

    def _free_hbm(self) -> int:
        return self._free_seen

    def _take(self, w) -> tuple[str, list[Request], int] | None:
        """Under the lock: the next batch for worker w, admitted against free device memory."""
        order = sorted((dq[0].arrival, name) for name, dq in self._pending.items() if dq)
        for _, name in order:
            dq = self._pending[name]
            r = self.routes[name]
            k = dq[0].k
            reqs, nq = [], 0
            for req in dq:
                if req.k != k or nq + req.queries.shape[0] > self.max_batch:
                    break
                reqs.append(req)
                nq += req.queries.shape[0]
            have = w["ws"].nbytes()
            avail = None  # the admission figure is consulted only when a batch must grow the workspace
            while reqs:
                growth = max(0, int(r.scratch_bytes(nq)) - have)
                if growth > 0 and avail is None:
                    avail = self._free_hbm() - self.hbm_reserve - self._growth_in_flight
                if growth == 0 or growth <= avail:
                    for _ in reqs:
                        dq.popleft()
                    return name, reqs, growth
                nq -= reqs.pop().queries.shape[0]  # admit fewer
            if avail is None:
                avail = self._free_hbm() - self.hbm_reserve - self._growth_in_flight
            if self.in_flight == 0 and self._growth_in_flight == 0:
                # nothing will free memory: the head request can never be admitted
                req = dq.popleft()
                req.error = (f"needs {int(r.scratch_bytes(req.queries.shape[0]))} bytes of scratch; "
                             f"{max(0, avail)} free above the reserve")
                req.done_at = time.perf_counter()
                req._event.set()
                return self._take(w)
            self.admission_waits += 1
        return None

    def _work(self, wi: int):
        import torch
        w = self._workers[wi]
        dev = f"cuda:{self.device}"
        torch.cuda.set_device(self.device)
        while True:
            with self._cv:
                job = None
                while self._running or any(self._pending.values()):
                    job = self._take(w)
                    if job is not None:
                        break
                    self._cv.wait(timeout=0.002)
                if job is None:
                    return
                name, reqs, growth = job
                self._growth_in_flight += growth
                self.in_flight += 1
                self.max_in_flight = max(self.max_in_flight, self.in_flight)
            before = w["ws"].nbytes()
            try:
                self._run(w, dev, name, reqs)
            except BaseException as e:  # surfaced by stop()
                self.errors.append(e)
                for req in reqs:
                    req.done_at = time.perf_counter()
                    req._event.set()
            finally:
                grew = w["ws"].nbytes() > before
                if grew:
                    self._refresh_free()  # the granted growth is now in the driver's figure
                with self._cv:
                    self._growth_in_flight -= growth
                    self.in_flight -= 1
                    self._cv.notify_all()

    def _pinned(self, w, r: Route, k: int):
        """The worker's staging buffers for route r and k, max_batch rows: pinned host input and
        outputs, and the device input and outputs (allocated once: allocations mid-stream are slow,
        and pinned ones synchronise the device)."""
        import torch
        key = (r.name, k)
        if key not in w["pin"]:
            dev = f"cuda:{self.device}"
            w["pin"][key] = (torch.empty(self.max_batch, r.dim, dtype=torch.float32, pin_memory=True),
                             torch.empty(self.max_batch, k, dtype=torch.int64, pin_memory=True),
                             torch.empty(self.max_batch, k, dtype=torch.float32, pin_memory=True),
                             torch.empty(self.max_batch, r.dim, dtype=torch.float32, device=dev),
                             torch.empty(self.max_batch, k, dtype=torch.int64, device=dev),
                             torch.empty(self.max_batch, k, dtype=torch.float32, device=dev))
        return w["pin"][key]

    def _run(self, w, dev, name, reqs):
        import torch
        t_start = time.perf_counter()
        r = self.routes[name]
        k = reqs[0].k
        nq = sum(q.queries.shape[0] for q in reqs)
        pin_in_all, pin_ids_all, pin_d_all, dev_in, dev_ids, dev_d = self._pinned(w, r, k)
        pin_in = pin_in_all[:nq]
        o = 0
        for req in reqs:
            b = req.queries.shape[0]
            pin_in[o:o + b].numpy()[:] = req.queries
            o += b
        st = w["stream"]
        with torch.cuda.stream(st):
            qdev = dev_in[:nq]
            qdev.copy_(pin_in, non_blocking=True)
            ids, dists = r.search(qdev, k, st, w["ws"], dev_ids[:nq], dev_d[:nq])
            pin_ids_all[:nq].copy_(ids, non_blocking=True)
            pin_d_all[:nq].copy_(dists, non_blocking=True)
        st.synchronize()
        now = time.perf_counter()
        ids_h = pin_ids_all[:nq].numpy()
        d_h = pin_d_all[:nq].numpy()
        o = 0
        for req in reqs:
            b = req.queries.shape[0]
            req.ids = ids_h[o:o + b].copy()
            req.dists = d_h[o:o + b].copy()
            req.done_at = now
            req.batch_queries = nq
            o += b
            req._event.set()
        with self._cv:
            self.completed.extend(reqs)
            self.batches.append((name, nq, len(reqs), t_start, now))

    # ---- reporting -------------------------------------------------------------------------
    def stats(self, since: float | None = None) -> dict:
        done = [r for r in self.completed if since is None or r.arrival >= since]
        if not done:
            return {"requests": 0}
        lat = np.array([r.latency_ms for r in done])
        nq = sum(r.queries.shape[0] for r in done)
        t0 = min(r.arrival for r in done)
        t1 = max(r.done_at for r in done)
        per_route = {}
        for name in self.routes:
            lr = np.array([r.latency_ms for r in done if r.route == name])
            if lr.size:
                per_route[name] = {"requests": int(lr.size), "p50_ms": round(float(np.percentile(lr, 50)), 3),
                                   "p99_ms": round(float(np.percentile(lr, 99)), 3)}
        sizes = [b[1] for b in self.batches]
        bms = np.array([(b[4] - b[3]) * 1e3 for b in self.batches]) if self.batches else np.zeros(1)
        return {"requests": len(done), "queries": int(nq), "qps": round(nq / max(t1 - t0, 1e-9), 1),
                "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "mean_batch_queries": round(float(np.mean(sizes)), 1) if sizes else 0.0,
                "batches": len(sizes), "batch_ms_p50": round(float(np.percentile(bms, 50)), 3),
                "batch_ms_p99": round(float(np.percentile(bms, 99)), 3), "batch_ms_max": round(float(bms.max()), 3),
                "max_batches_in_flight": self.max_in_flight,
                "admission_waits": self.admission_waits, "routes": per_route}


# ---- routes over this package's indexes ------------------------------------------------------
def tc_route(name: str, index, refine_r: int = 400) -> Route:
    """The tensor-core exact search of a LinearIndex (ann_flat_query_tc)."""
    def search(x, k, stream, ws, out_ids=None, out_dists=None):
        return index.search_tc(x, k, refine_r=refine_r, workspace=ws, stream=stream, out_ids=out_ids,
                               out_dists=out_dists)

    def scratch(nq):
        # sampled keys (~32k FP32 per query) + survivor regions + per-query sets + queries
        r = max(refine_r, 100)
        return nq * (4 * 33_000 + 24 * 3 * r + 8 * r + 2 * 4 * index.dim) + (64 << 20)
    return Route(name, index.dim, search, scratch)


def flat_route(name: str, index) -> Route:
    """The plain FP32 exact scan of a LinearIndex (ann_flat_query, exact mode)."""
    def search(x, k, stream, ws, out_ids=None, out_dists=None):
        return index.search(x, k, mode="exact", workspace=ws, stream=stream, out_ids=out_ids, out_dists=out_dists)
    return Route(name, index.dim, search, lambda nq: nq * (200 * 8 * 100 + 8 * index.dim) + (16 << 20))


def ivf_route(name: str, index, n_probe_clusters: int, refine_r: int = 300, max_list: int = 40_000,
              mode: str = "exact") -> Route:
    """An IVFIndex search (ann_ivf_query, no candidate cap): mode "exact" ranks the candidates by SQ8
    distances, "tc" by BF16 tensor-core keys; both re-rank in exact FP32."""
    def search(x, k, stream, ws, out_ids=None, out_dists=None):
        return index.search(x, k, 0, n_probe_clusters, refine_r, max_candidates=0, mode=mode, workspace=ws,
                            stream=stream, out_ids=out_ids, out_dists=out_dists)

    def scratch(nq):
        # candidate keys over the probed lists (bounded by the largest lists) + selections
        return nq * (4 * n_probe_clusters * max_list + 16 * refine_r + 8 * index.dim) + (64 << 20)
    return Route(name, index.dim, search, scratch)


def poisson_run(server: Server, traffic: list[tuple[float, str, np.ndarray]], k: int = 100) -> list[Request]:
    """Submits (arrival offset s, route, queries) in real time and waits for every request."""
    gc.collect()
    gc.freeze()  # the traffic list is long-lived: keep it out of the collected generations
    t0 = time.perf_counter()
    reqs = []
    for at, route, q in traffic:
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(route, q, k))
    for r in reqs:
        r.wait()
    return reqs
