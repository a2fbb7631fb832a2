"""Parity of the gf_* drop-in (include/annvedi_gpu_filter.h) with the reference's own GPU contestant,
competitors/gpu_filter/src/gpu_filter.cu, built from its source for sm_100a into oracle/_ref/gpu/ by
oracle/Makefile: both libraries get the same rows and queries through the same calls, and must return
the same count, the same ids in the same order and the same distance count. Cases: random rows, rows
duplicated many times (equal SQ8 keys and equal distances: ties go to the lower row id in both
stages), r above n, k above n, r below k, a dimension count that is not a multiple of 4 with n not a
multiple of 16, a constant column (range 0: scale 1), and an r large enough that the top-k kernel
sorts in several rounds."""
import ctypes
import os

import numpy as np
import pytest

from annvedi_b200 import _lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "gpu", "libgpufilter.so")
_F = ctypes.POINTER(ctypes.c_float)
_LL = ctypes.POINTER(ctypes.c_longlong)


class Gf:
    """The gf_* entry points of one library."""

    def __init__(self, lib):
        lib.gf_create.restype = ctypes.c_void_p
        lib.gf_create.argtypes = [_F, ctypes.c_long, ctypes.c_long]
        lib.gf_query.restype = ctypes.c_int
        lib.gf_query.argtypes = [ctypes.c_void_p, _F, ctypes.c_int, ctypes.c_int, _LL]
        lib.gf_ndist.restype = ctypes.c_longlong
        lib.gf_ndist.argtypes = [ctypes.c_void_p]
        lib.gf_free.argtypes = [ctypes.c_void_p]
        lib.gf_last_error.restype = ctypes.c_char_p
        self.lib = lib
        self.keep = []  # the reference borrows the rows for the handle's lifetime

    def create(self, x):
        x = np.ascontiguousarray(x, np.float32)
        self.keep.append(x)
        h = self.lib.gf_create(x.ctypes.data_as(_F), x.shape[0], x.shape[1])
        assert h, self.lib.gf_last_error().decode()
        return h

    def query(self, h, q, k, r):
        q = np.ascontiguousarray(q, np.float32)
        out = np.full(max(k, 1), -7, np.int64)
        got = self.lib.gf_query(h, q.ctypes.data_as(_F), k, r, out.ctypes.data_as(_LL))
        assert got >= 0, self.lib.gf_last_error().decode()
        return got, out[:got].copy()


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/gpu/libgpufilter.so not built (make -C oracle ref)")
    return Gf(ctypes.CDLL(REF_SO))


@pytest.fixture(scope="module")
def ours(cuda):
    return Gf(_lib.load())


def same_results(ref, ours, x, qs, k, r):
    hr, ho = ref.create(x), ours.create(x)
    try:
        for i, q in enumerate(qs):
            gr, ir = ref.query(hr, q, k, r)
            go, io = ours.query(ho, q, k, r)
            assert go == gr, (i, go, gr)
            np.testing.assert_array_equal(io, ir, err_msg=f"query {i}")
        assert ours.lib.gf_ndist(ho) == ref.lib.gf_ndist(hr)
    finally:
        ref.lib.gf_free(hr)
        ours.lib.gf_free(ho)


def test_random_rows(ref, ours):
    rng = np.random.default_rng(0)
    x = rng.standard_normal((20_000, 96)).astype(np.float32)
    same_results(ref, ours, x, rng.standard_normal((16, 96)).astype(np.float32), 10, 50)


def test_unit_rows_384(ref, ours):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((200_000, 384)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    qs = x[rng.choice(x.shape[0], 8, replace=False)] + 0.05 * rng.standard_normal((8, 384)).astype(np.float32)
    same_results(ref, ours, x, qs, 100, 300)


def test_duplicated_rows_tie_to_the_lower_id(ref, ours):
    rng = np.random.default_rng(2)
    distinct = rng.standard_normal((300, 32)).astype(np.float32)
    x = distinct[rng.integers(0, 300, 3_000)]
    qs = distinct[:12] + 0.01 * rng.standard_normal((12, 32)).astype(np.float32)
    same_results(ref, ours, x, qs, 25, 60)


def test_r_above_n_and_k_above_n(ref, ours):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((300, 16)).astype(np.float32)
    qs = rng.standard_normal((4, 16)).astype(np.float32)
    same_results(ref, ours, x, qs, 100, 1_000)
    same_results(ref, ours, x[:50], qs, 100, 10)


def test_r_below_k(ref, ours):
    rng = np.random.default_rng(4)
    x = rng.standard_normal((5_000, 24)).astype(np.float32)
    same_results(ref, ours, x, rng.standard_normal((6, 24)).astype(np.float32), 20, 5)


def test_ragged_dim_rows_and_a_constant_column(ref, ours):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((1_003, 37)).astype(np.float32)
    x[:, 3] = 1.5
    same_results(ref, ours, x, rng.standard_normal((8, 37)).astype(np.float32), 15, 40)


def test_large_r_sorts_in_rounds(ref, ours):
    rng = np.random.default_rng(6)
    x = rng.standard_normal((20_000, 16)).astype(np.float32)
    same_results(ref, ours, x, rng.standard_normal((2, 16)).astype(np.float32), 4_000, 9_000)


def test_algorithm_class(ours):
    from annvedi_b200.gpu_filter import Algorithm
    rng = np.random.default_rng(7)
    x = rng.standard_normal((10_000, 64)).astype(np.float32)
    a = Algorithm()
    a.fit(x)
    q = x[17] + 0.001
    ids = a.query(q, 10, r=40)
    assert ids.shape == (10,) and ids.dtype == np.int64 and ids[0] == 17
    assert a.get_n_distances() == 40
    h = ours.create(x)
    try:
        assert np.array_equal(ours.query(h, q, 10, 40)[1], ids)
    finally:
        ours.lib.gf_free(h)


def test_golden_outputs_of_the_reference(ours, golden_dir):
    """The drop-in against tests/golden/gf_ref.npz: the reference library's own outputs on six seeded
    cases (tests/golden/make_gf_golden.py), so this check needs no reference build on the machine."""
    from tests.golden.make_gf_golden import cases
    g = np.load(os.path.join(golden_dir, "gf_ref.npz"))
    for name, x, qs, k, r in cases():
        h = ours.create(x)
        try:
            for i, q in enumerate(qs):
                got, ids = ours.query(h, q, k, r)
                assert got == g[f"{name}_got"][i], (name, i)
                np.testing.assert_array_equal(ids, g[f"{name}_ids"][i, :got], err_msg=f"{name} query {i}")
            assert ours.lib.gf_ndist(h) == int(g[f"{name}_ndist"]), name
        finally:
            ours.lib.gf_free(h)


def test_replayed_queries_over_changing_k_and_r(ref, ours):
    """Each (k, r) runs its first query launch by launch and later ones as a replayed graph; a larger r
    reallocates the candidate buffers and drops the graphs. Interleaved (k, r) settings, with r growing
    part-way, return the reference's ids every time."""
    rng = np.random.default_rng(7)
    x = rng.standard_normal((50_000, 64)).astype(np.float32)
    qs = rng.standard_normal((15, 64)).astype(np.float32)
    hr, ho = ref.create(x), ours.create(x)
    try:
        settings = [(10, 50), (20, 400), (10, 50), (5, 2000), (20, 400)]
        for i, q in enumerate(qs):
            k, r = settings[i % len(settings)]
            gr, ir = ref.query(hr, q, k, r)
            go, io = ours.query(ho, q, k, r)
            assert go == gr, (i, k, r)
            np.testing.assert_array_equal(io, ir, err_msg=f"query {i} (k={k}, r={r})")
        assert ours.lib.gf_ndist(ho) == ref.lib.gf_ndist(hr)
    finally:
        ref.lib.gf_free(hr)
        ours.lib.gf_free(ho)
