"""Competition runner and scoring without h5py: the reference harness and evaluator over .npz / .npy files.

The reference harness (orthogonal-competition/harness.py:117-196) loads `train` / `test` from an HDF5
dataset, resolves `index_params` / `query_params` for (scenario, dataset) from scenarios.yaml (:73-114),
builds the index with `Algorithm().fit(train, **index_params)` (timed, with the RSS growth as index
memory), calls `query(q, k=k, **query_params)` once per query (each timed), checks that every result
is a length-k int32 array, reads `get_n_distances()`, and writes `neighbors`, `build_time`,
`query_times`, `n_dist_queries` and `index_mem_mb`. The evaluator (orthogonal-competition/evaluator.py:
149-157,437-509) recomputes the Euclidean distance of every returned id and scores recall@k as
mean(pred_dist[:k] <= true_dist[k-1]), QPS as queries / total query time, and latency percentiles.

Here datasets are `.npz` files (or directories of `.npy` files) with the HDF5 datasets' keys `train`,
`test` and optionally `distances` (the true neighbour distances, ascending; computed in FP64 when
absent), results are `.npz` files with the harness's keys, and the same environment variables drive
the command line (DATASET_PATH, RESULTS_PATH, SCENARIO_NAME, DATASET_NAME, QUERY_K; SCENARIOS_FILE
and ALGORITHM_FILE default to this package's plugin). `batch > 0` adds a batched query loop (the
GPU form: `Algorithm.query_batch` per batch, each query charged the batch time / batch size), which
the reference harness does not have; `batch = 0` is the harness's own loop.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import resource
import time

import numpy as np

RESULT_KEYS = ("neighbors", "build_time", "query_times", "n_dist_queries", "index_mem_mb")


# ---- data --------------------------------------------------------------------------------------------
def load_dataset(path: str) -> dict:
    """{"train": float32 [N, d], "test": float32 [Q, d], "distances": [Q, >=k] or absent} from an .npz
    file or a directory holding train.npy, test.npy and optionally distances.npy."""
    if os.path.isdir(path):
        out = {}
        for key in ("train", "test", "distances", "neighbors"):
            f = os.path.join(path, key + ".npy")
            if os.path.exists(f):
                out[key] = np.load(f)
    else:
        with np.load(path) as z:
            out = {key: z[key] for key in z.files}
    for key in ("train", "test"):
        if key not in out:
            raise ValueError(f"dataset {path!r} has no {key!r} array")
        out[key] = np.ascontiguousarray(out[key], dtype=np.float32)
    return out


def save_dataset(path: str, train, test, distances=None, neighbors=None) -> None:
    arrs = {"train": np.asarray(train, np.float32), "test": np.asarray(test, np.float32)}
    if distances is not None:
        arrs["distances"] = np.asarray(distances)
    if neighbors is not None:
        arrs["neighbors"] = np.asarray(neighbors)
    np.savez(path, **arrs)


def true_distances(train, test, k: int, chunk: int = 256):
    """(distances, neighbors): the k nearest Euclidean distances in FP64, ascending (ties by lower id),
    as the datasets' `distances` / `neighbors` hold them."""
    xb = np.asarray(train, np.float64)
    xn = (xb * xb).sum(1)
    dist, nbr = [], []
    for s in range(0, test.shape[0], chunk):
        q = np.asarray(test[s:s + chunk], np.float64)
        d2 = np.maximum(xn[None, :] - 2.0 * q @ xb.T + (q * q).sum(1)[:, None], 0.0)
        kk = min(k, xb.shape[0])
        part = np.argpartition(d2, kk - 1, axis=1)[:, :kk]
        # exact FP64 distances of the chosen ids, then (distance, id) order
        dd = np.sqrt(((xb[part] - q[:, None, :]) ** 2).sum(-1))
        order = np.lexsort((part, dd), axis=1)
        nbr.append(np.take_along_axis(part, order, 1))
        dist.append(np.take_along_axis(dd, order, 1))
    return np.concatenate(dist), np.concatenate(nbr)


# ---- scenarios ---------------------------------------------------------------------------------------
def load_scenario(scenarios_file: str, scenario_name: str, dataset_name: str) -> dict:
    """index_params / query_params of (scenario, dataset): the dataset's own block, else `default`
    (harness.py:73-114); ValueError otherwise."""
    import yaml
    with open(scenarios_file) as f:
        raw = yaml.safe_load(f)
    if not isinstance(raw, dict) or not isinstance(raw.get("scenarios"), dict):
        raise ValueError("scenarios.yaml must contain a top-level 'scenarios' mapping.")
    if scenario_name not in raw["scenarios"]:
        available = ", ".join(raw["scenarios"])
        raise ValueError(f"Scenario {scenario_name!r} not found in scenarios.yaml. Available: {available}")
    cfg = raw["scenarios"][scenario_name] or {}
    if dataset_name in cfg:
        block = cfg[dataset_name]
    elif "default" in cfg:
        block = cfg["default"]
    else:
        raise ValueError(f"Scenario {scenario_name!r} has no entry for dataset {dataset_name!r} and no "
                         "'default' fallback.")
    block = block or {}
    return {"index_params": dict(block.get("index_params") or {}),
            "query_params": dict(block.get("query_params") or {})}


def load_algorithm_class(algorithm_file: str | None = None):
    """The plugin's Algorithm class; it must have callable fit, query and get_n_distances (harness.py:52-70).
    None: this package's plugin."""
    if algorithm_file is None:
        from .algorithm import Algorithm as cls
    else:
        spec = importlib.util.spec_from_file_location("algorithm", algorithm_file)
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        if not hasattr(module, "Algorithm"):
            raise ImportError("algorithm.py must define a class named 'Algorithm'.")
        cls = module.Algorithm
    for method in ("fit", "query", "get_n_distances"):
        if not callable(getattr(cls, method, None)):
            raise ImportError(f"Algorithm is missing a callable method '{method}'.")
    return cls


def _device_used() -> int:
    try:
        import torch
        if torch.cuda.is_available():
            free, total = torch.cuda.mem_get_info()
            return total - free
    except Exception:  # noqa: BLE001 - no device: host memory only
        pass
    return 0


# ---- the run -----------------------------------------------------------------------------------------
def run(algo_cls, data: dict, params: dict, k: int = 10, batch: int = 0, log=print) -> dict:
    """Builds and queries one index as the harness does; returns the result arrays (RESULT_KEYS) plus
    `index_dev_mb`, the device memory the build took (the harness counts host RSS only)."""
    train, queries = data["train"], data["test"]
    nq = queries.shape[0]
    algo = algo_cls()
    rss0 = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss
    dev0 = _device_used()
    t0 = time.perf_counter()
    algo.fit(train, **params["index_params"])
    build_time = time.perf_counter() - t0
    index_mem_mb = (resource.getrusage(resource.RUSAGE_SELF).ru_maxrss - rss0) / 1024
    index_dev_mb = max(0, _device_used() - dev0) / 2 ** 20
    log(f"[harness] fit() done: {build_time:.4f}s memory_mb={index_mem_mb:.4f}Mb device_mb={index_dev_mb:.1f}")
    neighbors = np.empty((nq, k), dtype=np.int32)
    query_times = np.empty(nq, dtype=np.float64)
    qp = params["query_params"]
    if batch <= 0:
        for i in range(nq):
            t0 = time.perf_counter()
            result = algo.query(queries[i], k=k, **qp)
            query_times[i] = time.perf_counter() - t0
            result = np.asarray(result, dtype=np.int32)
            if result.shape != (k,):
                raise ValueError(f"algo.query() must return a 1-D array of length k={k}, got shape "
                                 f"{result.shape} on query index {i}.")
            neighbors[i] = result
    else:
        if not callable(getattr(algo, "query_batch", None)):
            raise ValueError("batched runs need Algorithm.query_batch")
        for s in range(0, nq, batch):
            qb = queries[s:s + batch]
            t0 = time.perf_counter()
            result = algo.query_batch(qb, k, **qp)
            result = np.asarray(result.cpu().numpy() if hasattr(result, "cpu") else result, dtype=np.int32)
            dt = time.perf_counter() - t0
            if result.shape != (qb.shape[0], k):
                raise ValueError(f"algo.query_batch() must return shape ({qb.shape[0]}, {k}), got "
                                 f"{result.shape} at query index {s}.")
            neighbors[s:s + qb.shape[0]] = result
            query_times[s:s + qb.shape[0]] = dt / qb.shape[0]
    n_dist_queries = int(algo.get_n_distances())
    total = query_times.sum()
    log(f"[harness] queries done: total={total:.4f}s  QPS={nq / total:.1f}  "
        f"median={np.median(query_times) * 1e3:.3f}ms  p99={np.percentile(query_times, 99) * 1e3:.3f}ms  "
        f"n_dist_queries={n_dist_queries}")
    return {"neighbors": neighbors, "build_time": float(build_time), "query_times": query_times,
            "n_dist_queries": n_dist_queries, "index_mem_mb": float(index_mem_mb), "index_dev_mb": index_dev_mb}


def save_results(path: str, res: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, **{key: np.asarray(res[key]) for key in RESULT_KEYS})


def load_results(path: str) -> dict:
    with np.load(path) as z:
        missing = [key for key in RESULT_KEYS if key not in z.files]
        if missing:
            raise ValueError(f"results file {path!r} lacks {missing}")
        return {"neighbors": z["neighbors"], "build_time": float(z["build_time"][()]),
                "query_times": z["query_times"], "n_dist_queries": int(z["n_dist_queries"][()]),
                "index_mem_mb": float(z["index_mem_mb"][()])}


# ---- scoring -----------------------------------------------------------------------------------------
def recalls(true_distances: np.ndarray, predicted_distances: np.ndarray, k: int) -> np.ndarray:
    """Per query: mean(pred[:k] <= true[k-1]) (evaluator.py:149-157)."""
    return np.array([np.mean(predicted_distances[i][:k] <= true_distances[i][k - 1])
                     for i in range(true_distances.shape[0])])


def evaluate(data: dict, res: dict, k: int) -> dict:
    """The evaluator's metrics (evaluator.py:437-509): Euclidean distances of the returned ids, recall,
    QPS from the summed query times, latency percentiles. An id of -1 (fewer than k results) counts as a
    miss."""
    train, queries = data["train"], data["test"]
    pred = np.asarray(res["neighbors"])
    n_test = queries.shape[0]
    for name, arr in (("neighbors", pred), ("query_times", res["query_times"])):
        if arr.shape[0] != n_test:
            raise ValueError(f"'{name}' has {arr.shape[0]} rows, expected {n_test}.")
    td = data.get("distances")
    if td is None or td.shape[1] < k:
        td, _ = true_distances(train, queries, k)
    pdist = np.empty(pred.shape, np.float64)
    for i in range(n_test):
        ok = pred[i] >= 0
        pdist[i] = np.inf
        pdist[i, ok] = np.linalg.norm(train[pred[i, ok]].astype(np.float64) - queries[i].astype(np.float64), axis=1)
    rec = recalls(td, pdist, k)
    qt = np.asarray(res["query_times"], np.float64)
    lat = qt * 1e3
    return {"status": "success", "build_time_s": res["build_time"], "total_query_time_s": float(qt.sum()),
            "qps": n_test / float(qt.sum()), "n_dist_queries": res["n_dist_queries"],
            "index_mem_mb": res["index_mem_mb"], "avg_recall": float(rec.mean()),
            "latency_ms": {"mean": float(lat.mean()), "median": float(np.median(lat)),
                           "p95": float(np.percentile(lat, 95)), "p99": float(np.percentile(lat, 99)),
                           "p999": float(np.percentile(lat, 99.9)), "max": float(lat.max())}}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--dataset", default=os.environ.get("DATASET_PATH"))
    ap.add_argument("--results", default=os.environ.get("RESULTS_PATH"))
    ap.add_argument("--scenario", default=os.environ.get("SCENARIO_NAME"))
    ap.add_argument("--dataset-name", default=os.environ.get("DATASET_NAME"))
    ap.add_argument("--scenarios-file", default=os.environ.get("SCENARIOS_FILE"))
    ap.add_argument("--algorithm-file", default=os.environ.get("ALGORITHM_FILE"))
    ap.add_argument("--k", type=int, default=int(os.environ.get("QUERY_K", 10)))
    ap.add_argument("--batch", type=int, default=0, help="0: one query per call (the harness); >0: batched")
    ap.add_argument("--evaluate", action="store_true", help="also score the results as the evaluator does")
    a = ap.parse_args(argv)
    if not a.dataset or not a.scenario or not a.scenarios_file:
        ap.error("--dataset, --scenario and --scenarios-file (or their environment variables) are required")
    name = a.dataset_name or os.path.splitext(os.path.basename(a.dataset.rstrip("/")))[0]
    data = load_dataset(a.dataset)
    params = load_scenario(a.scenarios_file, a.scenario, name)
    print(f"[harness] {data['train'].shape[0]} train | {data['test'].shape[0]} queries | "
          f"dim={data['train'].shape[1]} | k={a.k}; index_params: {params['index_params']}; "
          f"query_params: {params['query_params']}")
    res = run(load_algorithm_class(a.algorithm_file), data, params, a.k, a.batch)
    if a.results:
        save_results(a.results, res)
        print(f"[harness] Results written to {a.results}")
    if a.evaluate:
        m = evaluate(data, res, a.k)
        print(f"[evaluator] QPS={m['qps']:.1f} build={m['build_time_s']:.2f}s avg_recall={m['avg_recall']:.4f} "
              f"dist_query={m['n_dist_queries']} p99={m['latency_ms']['p99']:.3f}ms")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
