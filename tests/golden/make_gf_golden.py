"""Generates tests/golden/gf_ref.npz by running the reference's own GPU contestant
(competitors/gpu_filter/src/gpu_filter.cu, built from its source into oracle/_ref/gpu/ by
`make -C oracle ref`) on a CUDA device:

    python tests/golden/make_gf_golden.py [--out tests/golden/gf_ref.npz]

Inputs are not stored: cases() regenerates every case from its seed (numpy default_rng, identical on
every machine). Stored per case: the reference's gf_query return value and ids for each query, and
gf_ndist after the case's queries.
"""
from __future__ import annotations

import argparse
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "gpu", "libgpufilter.so")


def cases():
    """(name, rows, queries, k, r) of every case."""
    rng = np.random.default_rng(11)
    yield "random", rng.standard_normal((2000, 24)).astype(np.float32), \
        rng.standard_normal((5, 24)).astype(np.float32), 10, 30
    rng = np.random.default_rng(12)
    distinct = rng.standard_normal((150, 16)).astype(np.float32)
    yield "duplicates", distinct[rng.integers(0, 150, 1500)], \
        distinct[:5] + 0.01 * rng.standard_normal((5, 16)).astype(np.float32), 20, 50
    rng = np.random.default_rng(13)
    x = rng.standard_normal((1003, 37)).astype(np.float32)
    x[:, 3] = 1.5
    yield "ragged_constant", x, rng.standard_normal((4, 37)).astype(np.float32), 15, 40
    rng = np.random.default_rng(14)
    x = rng.standard_normal((300, 8)).astype(np.float32)
    qs = rng.standard_normal((3, 8)).astype(np.float32)
    yield "r_above_n", x, qs, 100, 1000
    yield "k_above_n", x[:50].copy(), qs, 100, 10
    yield "r_below_k", x, qs, 20, 5


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "gf_ref.npz"))
    args = ap.parse_args()
    F, LL = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_longlong)
    lib = ctypes.CDLL(REF_SO)
    lib.gf_create.restype = ctypes.c_void_p
    lib.gf_create.argtypes = [F, ctypes.c_long, ctypes.c_long]
    lib.gf_query.restype = ctypes.c_int
    lib.gf_query.argtypes = [ctypes.c_void_p, F, ctypes.c_int, ctypes.c_int, LL]
    lib.gf_ndist.restype = ctypes.c_longlong
    lib.gf_ndist.argtypes = [ctypes.c_void_p]
    lib.gf_free.argtypes = [ctypes.c_void_p]
    lib.gf_last_error.restype = ctypes.c_char_p
    out = {}
    for name, x, qs, k, r in cases():
        x = np.ascontiguousarray(x, np.float32)
        h = lib.gf_create(x.ctypes.data_as(F), x.shape[0], x.shape[1])
        assert h, lib.gf_last_error().decode()
        gots, ids = [], np.full((qs.shape[0], k), -1, np.int64)
        for i, q in enumerate(qs):
            q = np.ascontiguousarray(q, np.float32)
            o = np.full(k, -1, np.int64)
            got = lib.gf_query(h, q.ctypes.data_as(F), k, r, o.ctypes.data_as(LL))
            assert got >= 0, lib.gf_last_error().decode()
            gots.append(got)
            ids[i, :got] = o[:got]
        out[f"{name}_got"] = np.array(gots, np.int32)
        out[f"{name}_ids"] = ids
        out[f"{name}_ndist"] = np.array(lib.gf_ndist(h), np.int64)
        lib.gf_free(h)
    np.savez_compressed(args.out, **out)
    print("wrote", args.out, sorted(out))


if __name__ == "__main__":
    main()
