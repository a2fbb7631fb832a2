"""Benchmark: top-100 search QPS on one B200 (or N replicas under torchrun).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form ...]

Workload: the IVF-SQ8 configuration's data set -- 1,000,000 x 384 float32, a 2,048-centre Gaussian
mixture with Zipf(1.1) cluster sizes (20..40,000 points), sigma 0.3, rows L2-normalised, seeded
synthetic data standing in for the reference's embedding sets -- with 10,000 queries drawn from
the same mixture, k = 100, squared L2. One step = one search of a 10,000-query batch.

Forms (--form): "flat" is the plain FP32 exact scan (the correctness oracle of the GPU side and
the metric's denominator); "ivf" is the batched IVF-SQ8 scan with exact FP32 re-rank at the
smallest nprobe whose recall@100 against the FP64 exact top-100 is >= 0.95 (the headline).

Timing: W untimed warm-up steps, then exactly K steps between a barrier + device synchronize on
each side, timed with CUDA events on the search stream; max over ranks. The base (1.5 GB) is
larger than L2, so every step streams it from HBM. `e2e` repeats the steps through the public
API with host buffers (queries copied host->device and ids device->host inside the timed region).
Multi-GPU: every rank holds a replica of the index and searches its own query batch (weak
scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS at recall@100>=0.95 (1M x 384)"
K_NN = 100


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def make_workload(seed_queries: int, device: str, n: int, d: int, q: int):
    from annvedi_b200 import synth
    import torch
    w = synth.zipf_mixture(n, d, q, c=2048, sigma=0.3, seed=1234, backend="torch", device=device)
    if seed_queries:
        # a different query batch per rank, same base
        w2 = synth.zipf_mixture(n, d, q, c=2048, sigma=0.3, seed=1234 + seed_queries, backend="torch",
                                device=device)
        w.queries = w2.queries
        del w2
        torch.cuda.empty_cache()
    return w


def ground_truth(base, queries, k):
    """FP64 exact top-k distances (k-th value per query) on the GPU, chunked."""
    import torch
    xb = base.double()
    xn = (xb * xb).sum(1)
    kth = []
    for s in range(0, queries.shape[0], 256):
        qb = queries[s:s + 256].double()
        d = xn[None, :] - 2.0 * qb @ xb.T + (qb * qb).sum(1)[:, None]
        kth.append(torch.topk(d, k, dim=1, largest=False).values[:, -1])
    return torch.cat(kth)


def recall_evaluator(base, queries, ids, kth):
    """mean(pred_d[:k] <= true_d[k-1]) with FP64 distances (orthogonal-competition/evaluator.py:149-157)."""
    import torch
    ok = ids >= 0
    x = base[ids.clamp(min=0)].double()
    d = ((x - queries.double()[:, None, :]) ** 2).sum(-1)
    hit = (d <= kth[:, None] * (1 + 1e-9) + 1e-12) & ok
    return float(hit.double().mean().item())


def run_ours(args, rank, world, local):
    import torch
    from annvedi_b200 import _lib
    from annvedi_b200.linear import LinearIndex

    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    n, d, q = args.n, args.dim, args.batch
    w = make_workload(rank, dev, n, d, q)
    base, queries = w.base.contiguous(), w.queries.contiguous()
    hbm_peak, bf16_peak, peak_kind = _peaks()

    ix = LinearIndex(device=local, metric="l2", mode="exact")
    ix.fit(base)
    stream = torch.cuda.current_stream()
    out_ids = torch.empty(q, K_NN, dtype=torch.int64, device=dev)
    out_d = torch.empty(q, K_NN, dtype=torch.float32, device=dev)

    def step():
        ix.search(queries, K_NN, mode="exact", out_ids=out_ids, out_dists=out_d)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kth = ground_truth(base, queries[:512], K_NN)
    rec = recall_evaluator(base, queries[:512], out_ids[:512], kth)

    clocks = ClockSampler(local).start()
    ix.reset_profile_results()
    ix.set_profiling(True)
    launches0 = _lib.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    launches = _lib.kernel_launches() - launches0
    ix.set_profiling(False)
    prof = ix.get_profile_results()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    qps = world * q * args.steps / (ms_max / 1e3)

    # end to end through the public API with host buffers
    qh = queries.cpu().numpy()
    qpin = torch.from_numpy(qh).pin_memory().numpy()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ids_h, _ = ix.search(qpin, K_NN, mode="exact", with_dists=False)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0, world)
    e2e_qps = world * q * args.steps / e2e_s

    # roofline of the dominant kernel (the fused scan): per launch, the base once + queries
    scan_ms = prof["scan_ms"] / max(1, prof["scan_launches"])
    flops = 3.0 * n * d * q  # sub, mul, add per element pair
    bytes_alg = 4.0 * n * d + 4.0 * q * d
    fp32_peak = 148 * 128 * 2 * (clk["sm_mhz"] or 1965.0) * 1e6 / 1e12
    line = {
        "metric": METRIC, "value": round(qps, 1), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded zipf mixture)",
        "config": {"workload": "flat_exact_fp32 over 1M x 384 zipf mixture (IVF-SQ8 config data)",
                   "form": "flat", "n": n, "dim": d, "batch": q, "k": K_NN, "metric": "l2",
                   "l2": "inputs larger than L2 (1.5 GB base)", "parallelism": f"replicas x{world}"},
        "recall_at_100": round(rec, 4),
        "e2e": {"value": round(e2e_qps, 1), "unit": "queries/s", "h2d_bytes_per_step": q * d * 4,
                "d2h_bytes_per_step": q * K_NN * 8},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": round(bytes_alg / (scan_ms / 1e3) / 1e9, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(bytes_alg / (scan_ms / 1e3) / 1e9 / hbm_peak, 4),
                     "traffic": None, "peak_kind": peak_kind, "kernel": "flat_scan_kernel",
                     "fp32_tflops": round(flops / (scan_ms / 1e3) / 1e12, 2), "fp32_peak_tflops": round(fp32_peak, 1),
                     "fp32_frac": round(flops / (scan_ms / 1e3) / 1e12 / fp32_peak, 4),
                     "scan_ms_per_launch": round(scan_ms, 3)},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_linear(base, queries, args)
    return line


def cpu_baseline_linear(base, queries, args):
    """The reference's linear_ann_cpp (oracle/_ref) on the host cores: one Python thread per core,
    each calling query() (serial per query, GIL released), over a bounded sample of the queries."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import refmod
    lin = refmod.load_ref("linear_ann_cpp")
    xb = base.cpu().numpy()
    ix = lin.LinearIndex()
    ix.fit(xb)
    cores = os.cpu_count() or 1
    nsample = max(2 * cores, 16)
    qs = queries[:nsample].cpu().numpy()
    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        list(ex.map(lambda qq: ix.query(qq, K_NN), list(qs)))
    dt = time.perf_counter() - t0
    return {"value": round(nsample / dt, 2), "unit": "queries/s", "cores": cores, "kind": "reference",
            "sample": f"{nsample} of the batch's queries, linear_ann_cpp ({refmod.host_isa()} build), "
                      f"{cores} Python threads"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation on this host's cores (the reference arm)."""
    if rank != 0:
        return None
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from oracle import refmod
    from annvedi_b200 import synth
    w = synth.zipf_mixture(args.n, args.dim, args.batch, c=2048, sigma=0.3, seed=1234, backend="torch",
                           device="cpu")
    xb = w.base.numpy()
    lin = refmod.load_ref("linear_ann_cpp")
    ix = lin.LinearIndex()
    ix.fit(xb)
    cores = os.cpu_count() or 1
    nsample = max(cores, 8)
    qs = list(w.queries[:nsample].numpy())
    for _ in range(min(args.warmup, 1)):
        ix.query(qs[0], K_NN)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        with ThreadPoolExecutor(cores) as ex:
            list(ex.map(lambda qq: ix.query(qq, K_NN), qs))
        times.append(time.perf_counter() - t0)
    total = sum(times)
    qps = nsample * args.steps / total
    del torch
    return {"metric": METRIC, "value": round(qps, 2), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded zipf mixture)",
            "config": {"workload": "flat_exact_fp32 over 1M x 384 zipf mixture (IVF-SQ8 config data)",
                       "form": "flat", "n": args.n, "dim": args.dim, "batch": nsample, "k": K_NN},
            "impl": "reference",
            "cpu_baseline": {"value": round(qps, 2), "unit": "queries/s", "cores": cores, "kind": "reference",
                             "sample": f"{nsample} queries per step, linear_ann_cpp ({refmod.host_isa()} build)"},
            "e2e": {"value": round(qps, 2), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["flat"], default="flat")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=384)
    ap.add_argument("--batch", type=int, default=10_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = dist_setup()
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
