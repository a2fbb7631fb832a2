"""Autotuner: the cheapest search configuration that meets a recall target, measured on the device.

The knobs are the IVF probe count (nprobe), the re-rank depth (refine_r, the oversampling of the
exact FP32 re-rank) and the scoring form (the SQ8 candidate keys or the BF16 tensor-core keys); the
flat tensor-core search has only its re-rank depth. For each form and depth the probe counts are tried in
increasing order (recall and cost both grow with nprobe) and the first that meets the target is kept;
every point tried is timed with CUDA events over `reps` calls after a warm-up call. The result is the
fastest point that meets the target, with the whole table.

recall@k is the evaluator's definition (orthogonal-competition/evaluator.py:149-157): the share of the
returned ids whose FP64 distance is within the FP64 k-th nearest distance of their query.
"""
from __future__ import annotations


def recall_at_k(base, queries, ids, kth) -> float:
    """mean(d(q, x_id) <= kth(q)) with FP64 distances; base, queries, ids, kth device tensors."""
    hits = 0.0
    for s in range(0, queries.shape[0], 1000):
        ii = ids[s:s + 1000]
        ok = ii >= 0
        x = base[ii.clamp(min=0)].double()
        d = ((x - queries[s:s + 1000].double()[:, None, :]) ** 2).sum(-1)
        hits += float(((d <= kth[s:s + 1000, None] * (1 + 1e-9) + 1e-12) & ok).double().sum().item())
    return hits / ids.numel()


def _time(fn, reps, stream):
    import torch
    fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _timer(timer):
    """timer(fn, reps) -> ms per call: the given one, else CUDA events on the current stream."""
    if timer is not None:
        return timer
    import torch
    stream = torch.cuda.current_stream()
    return lambda fn, reps: _time(fn, reps, stream)


IVF_NPROBES = (2, 3, 4, 5, 6, 8, 10, 12, 16, 24, 32, 64, 128)
IVF_REFINES = (100, 150, 200, 300)


def tune_ivf(index, base, queries, kth, k: int = 100, target: float = 0.95, modes=("tc", "exact"),
             nprobes=IVF_NPROBES, refines=IVF_REFINES, reps: int = 3, sample_divs=(4, 8, 16), timer=None) -> dict:
    """Fastest (mode, nprobe, refine_r) of an IVFIndex whose recall@k on `queries` is >= target.

    For every mode and re-rank depth the probe counts run in increasing order up to the first that meets
    the target. At each tensor-core mode's best point the sampled bars' list share (sample_divs) is then
    swept and the fastest kept on the index. Returns {"best": {...} or None, "best_by_mode": {mode: {...}},
    "table": [...]}; each entry has mode, nprobe, refine_r, recall, ms_per_batch and qps (queries per second at
    this batch size), and sample_div where swept. The index keeps the last mode's best sample_div. timer(fn,
    reps) -> ms per call replaces the CUDA-event timing (the host-logic tests)."""
    import torch
    time_fn = _timer(timer)
    nq = queries.shape[0]
    ids = torch.empty(nq, k, dtype=torch.int64, device=queries.device)
    dists = torch.empty(nq, k, dtype=torch.float32, device=queries.device)
    table, best = [], None
    for mode in modes:
        for rr in refines:
            for npc in nprobes:
                fn = lambda: index.search(queries, k, 0, npc, rr, max_candidates=0, mode=mode, out_ids=ids,
                                          out_dists=dists)
                ms = time_fn(fn, reps)
                rec = recall_at_k(base, queries, ids, kth)
                row = {"mode": mode, "nprobe": npc, "refine_r": rr, "recall": round(rec, 4),
                       "ms_per_batch": round(ms, 4), "qps": round(nq / (ms / 1e3), 1)}
                table.append(row)
                if rec >= target:
                    if best is None or row["qps"] > best["qps"]:
                        best = row
                    break  # a larger nprobe costs more for this (mode, refine_r)
    by_mode = {}
    for row in table:
        b = by_mode.get(row["mode"])
        if row["recall"] >= target and (b is None or row["qps"] > b["qps"]):
            by_mode[row["mode"]] = row
    # the tensor-core forms' sampling knob at each mode's best point: the share of every probed list the
    # sampled bars score (results do not depend on it; time does)
    for mode, row in list(by_mode.items()):
        if mode not in ("tc", "tc_sq8") or not sample_divs:
            continue
        row["sample_div"] = 8
        for div in sample_divs:
            if div == 8:
                continue
            index.set_option("sample_div", div)
            fn = lambda: index.search(queries, k, 0, row["nprobe"], row["refine_r"], max_candidates=0, mode=mode,
                                      out_ids=ids, out_dists=dists)
            ms = time_fn(fn, reps)
            alt = {**row, "sample_div": div, "ms_per_batch": round(ms, 4), "qps": round(nq / (ms / 1e3), 1)}
            table.append(alt)
            if alt["qps"] > by_mode[mode]["qps"]:
                by_mode[mode] = alt
        index.set_option("sample_div", by_mode[mode].get("sample_div", 8))
    best = max(by_mode.values(), key=lambda r: r["qps"]) if by_mode else best
    return {"best": best, "best_by_mode": by_mode, "table": table, "target": target}


def tune_flat_tc(index, base, queries, kth, k: int = 100, target: float = 0.95, refines=(100, 200, 400),
                 reps: int = 3, timer=None) -> dict:
    """Fastest re-rank depth of a LinearIndex's tensor-core search whose recall@k is >= target."""
    import torch
    time_fn = _timer(timer)
    nq = queries.shape[0]
    ids = torch.empty(nq, k, dtype=torch.int64, device=queries.device)
    dists = torch.empty(nq, k, dtype=torch.float32, device=queries.device)
    table, best = [], None
    for rr in refines:
        fn = lambda: index.search_tc(queries, k, refine_r=rr, out_ids=ids, out_dists=dists)
        ms = time_fn(fn, reps)
        rec = recall_at_k(base, queries, ids, kth)
        row = {"refine_r": rr, "recall": round(rec, 4), "ms_per_batch": round(ms, 4), "qps": round(nq / (ms / 1e3), 1)}
        table.append(row)
        if rec >= target and (best is None or row["qps"] > best["qps"]):
            best = row
    return {"best": best, "table": table, "target": target}


def tune_flat_tile(index, queries, k: int = 100, tiles=(8, 16, 32), reps: int = 2, timer=None) -> dict:
    """Fastest query tile (queries per CTA) of a LinearIndex's exact scan for this batch, timed over `reps`
    calls after a warm-up call; the tile is left set on the index. Results do not depend on the tile, so no
    recall is needed. Returns {"best": {...}, "table": [...]} with tile, ms_per_batch and qps."""
    import torch
    time_fn = _timer(timer)
    nq = queries.shape[0]
    ids = torch.empty(nq, k, dtype=torch.int64, device=queries.device)
    dists = torch.empty(nq, k, dtype=torch.float32, device=queries.device)
    table = []
    for tile in tiles:
        index.set_query_tile(tile)
        ms = time_fn(lambda: index.search(queries, k, mode="exact", out_ids=ids, out_dists=dists), reps)
        table.append({"tile": tile, "ms_per_batch": round(ms, 3), "qps": round(nq / (ms / 1e3), 1)})
    best = min(table, key=lambda r: r["ms_per_batch"])
    index.set_query_tile(best["tile"])
    return {"best": best, "table": table}
