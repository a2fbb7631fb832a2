"""The bench line's roofline arithmetic on the CPU (bench.ivf_roofline): the dominant kernel is the one with
the most CUDA-event time; its algorithmic work per launch over its mean launch time, against the peak of
the bound that applies (the dense BF16 rate for the tensor-core list keys, twice it for the int8 form,
HBM for the rest)."""
import pytest

import bench


def _kern(**ms):
    return {name: {"ms": v, "launches": 4} for name, v in ms.items()}


def test_tensor_core_keys_against_the_bf16_peak():
    kern = _kern(keys=1.2, bars=0.3, select=0.2, rerank=0.8)  # keys dominate: 0.3 ms a launch
    cands, q, d, R = 130e6, 10_000, 384, 100
    r = bench.ivf_roofline("ivf_tc", kern, cands, q, d, R, 6550.0, 1590.0, "measured", 437_080)
    assert r["bound"] == "tensor" and r["kernel_ms"] == pytest.approx(0.3)
    tflops = 2 * cands * d / 0.3e-3 / 1e12
    assert r["achieved"] == pytest.approx(round(tflops, 1))
    assert r["frac"] == pytest.approx(round(tflops / 1590.0, 4))
    r8 = bench.ivf_roofline("ivf_tc_sq8", kern, cands, q, d, R, 6550.0, 1590.0, "measured", 437_080)
    assert r8["peak"] == pytest.approx(2 * 1590.0) and r8["frac"] == pytest.approx(round(tflops / 3180.0, 4))


def test_rerank_against_hbm_on_its_unique_rows():
    kern = _kern(keys=0.4, bars=0.3, select=0.2, rerank=0.9)  # re-rank dominates: 0.225 ms a launch
    q, d, R, unique = 10_000, 384, 100, 437_080
    r = bench.ivf_roofline("ivf_tc", kern, 130e6, q, d, R, 6550.0, 1590.0, "measured", unique)
    assert r["bound"] == "hbm" and r["kernel"] == "ivf_rerank_kernel"
    nbytes = unique * d * 4.0 + q * R * 8.0 + q * bench.K_NN * 12.0
    gbs = nbytes / 0.225e-3 / 1e9
    assert r["bytes_per_launch"] == int(nbytes)
    assert r["achieved"] == pytest.approx(round(gbs, 1)) and r["frac"] == pytest.approx(round(gbs / 6550.0, 4))
