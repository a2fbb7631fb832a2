"""Bounded runs of one kernel family each, for profiling with ncu (the commands in profiles/ use these).

    python -m annvedi_b200.profiling <case> [--n N] [--dim D] [--nq Q] [--reps R] [...]

Cases (the headline data set: a seeded zipf mixture of 2,048 L2-normalised centres, sigma 0.3):
  flat_scan    exact linear scan of a Q-query batch (flat_scan_kernel, then the split merge)
  flat_stream  exact linear scan of one query per call (flat_stream_kernel)
  ivf_batched  IVF exact selection over SQ8 keys of a Q-query batch (ivf_batched_kernel)
  ivf_tc       IVF on the tensor cores (--form tc or tc_sq8): the grouped list GEMM, sampled bars, best-R
               selection and exact re-rank of a Q-query batch
  gf_scan      the gf_* drop-in (gpu_filter), one query per call (gf_scan_kernel)

Each case warms up, then runs --reps calls and prints one JSON line with the mean call time (CUDA events
on the calling stream). Nothing here is timed by the bench; it only gives ncu a short, repeatable
launch sequence.
"""
from __future__ import annotations

import argparse
import json


def _data(n, dim, nq):
    import torch
    from . import synth
    w = synth.zipf_mixture(n, dim, nq, c=2048, sigma=0.3, seed=1234)
    dev = "cuda:0"
    return w, torch.from_numpy(w.base).to(dev), torch.from_numpy(w.queries).to(dev)


def _time(fn, reps):
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["flat_scan", "flat_stream", "ivf_batched", "ivf_tc", "gf_scan"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=384)
    ap.add_argument("--nq", type=int, default=0, help="queries (default: the case's own)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--k", type=int, default=100)
    ap.add_argument("--nprobe", type=int, default=2)
    ap.add_argument("--refine", type=int, default=100)
    ap.add_argument("--sample-div", type=int, default=16)
    ap.add_argument("--form", choices=["tc", "tc_sq8"], default="tc")
    ap.add_argument("--gf-r", type=int, default=300, help="gf_scan: the drop-in's re-rank depth r")
    ap.add_argument("--sampled-min", type=int, default=0,
                    help="ivf_tc: batch size from which the sampled path runs (0: the library's default)")
    args = ap.parse_args(argv)
    import torch
    nq = args.nq or {"flat_scan": 1000, "flat_stream": 1, "ivf_batched": 10000, "ivf_tc": 10000, "gf_scan": 16}[args.case]
    w, base, queries = _data(args.n, args.dim, max(nq, 1))
    k = args.k
    out = {"case": args.case, "n": args.n, "dim": args.dim, "nq": nq, "reps": args.reps}
    if args.case in ("flat_scan", "flat_stream"):
        from .linear import LinearIndex
        ix = LinearIndex(device=0, mode="exact")
        ix.fit(base)
        ids = torch.empty(nq, k, dtype=torch.int64, device=base.device)
        d = torch.empty(nq, k, dtype=torch.float32, device=base.device)
        out["ms_per_call"] = _time(lambda: ix.search(queries[:nq], k, mode="exact", out_ids=ids, out_dists=d),
                                   args.reps)
    elif args.case in ("ivf_batched", "ivf_tc"):
        from .ivf import IVFIndex
        ix = IVFIndex(device=0, mode="exact")
        ix.fit(base, 1, 0, 2048, centroids=torch.from_numpy(w.centres).to(base.device),
               assign=torch.from_numpy(w.assign.astype("int32")).to(base.device))
        mode = "exact" if args.case == "ivf_batched" else args.form
        if mode != "exact":
            ix.set_option("sample_div", args.sample_div)
            if args.sampled_min:
                ix.set_option("sampled_min_queries", args.sampled_min)
        ids = torch.empty(nq, k, dtype=torch.int64, device=base.device)
        d = torch.empty(nq, k, dtype=torch.float32, device=base.device)
        out.update({"mode": mode, "nprobe": args.nprobe, "refine_r": args.refine})
        call = lambda: ix.search(queries[:nq], k, 0, args.nprobe, args.refine, max_candidates=0, mode=mode,
                                 out_ids=ids, out_dists=d)
        out["ms_per_call"] = _time(call, args.reps)
        ix.reset_profile_results()  # the kernel timers over --reps more calls
        ix.set_profiling(True)
        for _ in range(args.reps):
            call()
        ix.set_profiling(False)
        out["kernel_ms"] = {k2: round(v["ms"] / max(1, v["launches"]), 4) for k2, v in ix.get_kernel_times().items()}
    else:
        import numpy as np
        from .gpu_filter import Algorithm
        gf = Algorithm()
        gf.fit(np.ascontiguousarray(w.base, dtype=np.float32))
        qs = np.ascontiguousarray(w.queries[:nq], dtype=np.float32)
        r = args.gf_r
        out["r"] = r

        def calls():
            for i in range(nq):
                gf.query(qs[i], k, r=r)

        out["ms_per_call"] = _time(calls, args.reps) / nq
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
