"""Seeded synthetic workloads with the shapes and value distributions of the benchmark configs.

The reference is scored on public HDF5 embedding sets that are not available offline; these
generators stand in for them. All are deterministic functions of ``seed``. ``backend="numpy"``
uses ``numpy.random.default_rng`` (identical on every machine; used for fixtures and tests);
``backend="torch"`` draws on the target device with a seeded ``torch.Generator`` (used by the
benchmark for the 1M-4M row sets, so the base never crosses PCIe).

Workloads (N base rows, d dims, Q queries):

* ``flat_normal``   : N(0,1) entries, rows L2-normalised (plain exact scan, 100k x 384).
* ``mixture``       : Gaussian mixture, centres N(0,1), point = centre + N(0, sigma^2), rows
                      L2-normalised (exact scan at scale, 1M x 768, 1,024 centres, sigma 0.35).
* ``zipf_mixture``  : mixture whose cluster sizes follow a Zipf(s) law
                      size_r = clip(round(C0 * r^-s), lo, hi), C0 solved so sizes sum to N
                      (IVF-SQ8, 1M x 384, 2,048 centres, s = 1.1, sizes 20..40,000, sigma 0.3);
                      queries pick their centre with probability proportional to cluster size.
* ``scaled_mixture``: mixture (sigma 0.4) with rows normalised then scaled by U(0.5, 2.0)
                      (scaled-FP8 scan, 4M x 256, 4,096 centres; norms spread 0.5-2.0).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def zipf_sizes(n: int, c: int, s: float = 1.1, lo: int = 20, hi: int = 40000) -> np.ndarray:
    """Cluster sizes clip(round(C0 * r^-s), lo, hi) for ranks r = 1..c, C0 solved by bisection so
    the sizes sum to n (the last cluster absorbs the rounding remainder)."""
    r = np.arange(1, c + 1, dtype=np.float64)

    def total(c0):
        return np.clip(np.round(c0 * r ** -s), lo, hi).sum()

    a, b = 0.0, float(n) * 4
    for _ in range(200):
        m = 0.5 * (a + b)
        if total(m) < n:
            a = m
        else:
            b = m
    sizes = np.clip(np.round(b * r ** -s), lo, hi).astype(np.int64)
    diff = n - int(sizes.sum())
    # absorb the remainder in the smallest clusters, keeping them within [lo, hi]
    i = c - 1
    while diff != 0 and i >= 0:
        step = max(lo - sizes[i], min(hi - sizes[i], diff))
        sizes[i] += step
        diff -= step
        i -= 1
    if diff != 0:
        raise ValueError(f"cannot split {n} points into {c} clusters within [{lo}, {hi}]")
    return sizes


def _normalise_np(x: np.ndarray) -> np.ndarray:
    nrm = np.linalg.norm(x, axis=1, keepdims=True)
    nrm[nrm == 0] = 1
    return (x / nrm).astype(np.float32)


@dataclass
class Workload:
    base: object          # [N, d] float32 (numpy array or torch tensor)
    queries: object       # [Q, d] float32
    centres: object       # [C, d] float32 or None (generating centres, L2-normalised)
    assign: object        # [N] int64 generating cluster of each base row, or None
    metric: str           # "l2" or "ip"
    name: str


def flat_normal(n: int, d: int, q: int, seed: int = 0, backend: str = "numpy", device: str = "cpu") -> Workload:
    if backend == "numpy":
        rng = np.random.default_rng(seed)
        base = _normalise_np(rng.standard_normal((n, d), dtype=np.float32))
        qs = _normalise_np(rng.standard_normal((q, d), dtype=np.float32))
        return Workload(base, qs, None, None, "l2", f"flat_normal_{n}x{d}")
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    base = torch.nn.functional.normalize(torch.randn(n, d, generator=g, device=device), dim=1)
    qs = torch.nn.functional.normalize(torch.randn(q, d, generator=g, device=device), dim=1)
    return Workload(base, qs, None, None, "l2", f"flat_normal_{n}x{d}")


def _mixture(n, d, q, c, sigma, sizes, seed, backend, device, scale_norms, metric, name, query_seed=None):
    if backend == "numpy":
        rng = np.random.default_rng(seed)
        centres = rng.standard_normal((c, d), dtype=np.float32)
        if sizes is None:
            assign = rng.integers(0, c, n)
            p = None
        else:
            assign = np.repeat(np.arange(c), sizes)
            rng.shuffle(assign)
            p = sizes / sizes.sum()
        base = centres[assign] + sigma * rng.standard_normal((n, d), dtype=np.float32)
        if query_seed is not None:  # the same base, queries from their own stream
            rng = np.random.default_rng(query_seed)
        qc = rng.choice(c, size=q, p=p) if p is not None else rng.integers(0, c, q)
        qs = centres[qc] + sigma * rng.standard_normal((q, d), dtype=np.float32)
        base = _normalise_np(base)
        qs = _normalise_np(qs)
        if scale_norms:
            base = (base * rng.uniform(0.5, 2.0, (n, 1))).astype(np.float32)
            qs = (qs * rng.uniform(0.5, 2.0, (q, 1))).astype(np.float32)
        return Workload(base, qs, _normalise_np(centres), assign.astype(np.int64), metric, name)
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    centres = torch.randn(c, d, generator=g, device=device)
    if sizes is None:
        assign = torch.randint(0, c, (n,), generator=g, device=device)
        qc = torch.randint(0, c, (q,), generator=g, device=device)
    else:
        sz = torch.as_tensor(sizes, device=device)
        assign = torch.repeat_interleave(torch.arange(c, device=device), sz)
        assign = assign[torch.randperm(n, generator=g, device=device)]
        qc = torch.multinomial(sz.double() / sz.sum(), q, replacement=True, generator=g)
    base = torch.empty(n, d, device=device)
    chunk = 1 << 18
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        blk = centres[assign[s:e]] + sigma * torch.randn(e - s, d, generator=g, device=device)
        base[s:e] = torch.nn.functional.normalize(blk, dim=1)
    qs = torch.nn.functional.normalize(centres[qc] + sigma * torch.randn(q, d, generator=g, device=device), dim=1)
    if scale_norms:
        base.mul_(torch.rand(n, 1, generator=g, device=device) * 1.5 + 0.5)
        qs.mul_(torch.rand(q, 1, generator=g, device=device) * 1.5 + 0.5)
    return Workload(base, qs, torch.nn.functional.normalize(centres, dim=1), assign.long(), metric, name)


def mixture(n, d, q, c=1024, sigma=0.35, seed=0, backend="numpy", device="cpu", metric="ip") -> Workload:
    return _mixture(n, d, q, c, sigma, None, seed, backend, device, False, metric, f"mixture_{n}x{d}_c{c}")


def zipf_mixture(n, d, q, c=2048, sigma=0.3, s=1.1, lo=20, hi=40000, seed=0, backend="numpy",
                 device="cpu", query_seed=None) -> Workload:
    """query_seed (numpy backend): draw the queries from their own seeded stream (same base)."""
    sizes = zipf_sizes(n, c, s, lo, hi)
    return _mixture(n, d, q, c, sigma, sizes, seed, backend, device, False, "l2", f"zipf_mixture_{n}x{d}_c{c}",
                    query_seed)


def scaled_mixture(n, d, q, c=4096, sigma=0.4, seed=0, backend="numpy", device="cpu") -> Workload:
    return _mixture(n, d, q, c, sigma, None, seed, backend, device, True, "l2", f"scaled_mixture_{n}x{d}_c{c}")


# Full-size shapes of the five benchmark configurations.
CONFIGS = {
    "c1_flat_100k_384": dict(kind="flat_normal", n=100_000, d=384, q=1_000),
    "c2_mixture_1m_768": dict(kind="mixture", n=1_000_000, d=768, q=10_000, c=1024, sigma=0.35),
    "c3_ivf_1m_384": dict(kind="zipf_mixture", n=1_000_000, d=384, q=10_000, c=2048, sigma=0.3),
    "c4_fp8_4m_256": dict(kind="scaled_mixture", n=4_000_000, d=256, q=20_000, c=4096, sigma=0.4),
}


def make(name_or_kind: str, seed: int = 0, backend: str = "numpy", device: str = "cpu", **over) -> Workload:
    cfg = dict(CONFIGS.get(name_or_kind, {"kind": name_or_kind}))
    cfg.update(over)
    kind = cfg.pop("kind")
    fn = {"flat_normal": flat_normal, "mixture": mixture, "zipf_mixture": zipf_mixture,
          "scaled_mixture": scaled_mixture}[kind]
    return fn(seed=seed, backend=backend, device=device, **cfg)


def poisson_arrivals(rate_qps: float, duration_s: float, p_geom: float = 0.1, cap: int = 256,
                     seed: int = 0) -> list:
    """Request stream: (arrival time s, batch size) with Poisson arrivals of *queries* at
    ``rate_qps`` and request batch sizes ~ geometric(p) capped at ``cap``."""
    rng = np.random.default_rng(seed)
    mean_b = min(cap, 1.0 / p_geom)
    req_rate = rate_qps / mean_b
    t, out = 0.0, []
    while t < duration_s:
        t += rng.exponential(1.0 / req_rate)
        out.append((t, int(min(cap, rng.geometric(p_geom)))))
    return out

