"""The reference GPU contestant's C ABI (include/annvedi_gpu_filter.h): every declared gf_* function is
exported by the library, and the calls that need no device report their errors the reference's way
(NULL / -1 with a message in gf_last_error). No compute calls here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from annvedi_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "annvedi_gpu_filter.h")


def declared_gf():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(gf_\w+)\s*\(", text)))


def test_header_declares_the_reference_abi():
    # the five entry points of competitors/gpu_filter/src/gpu_filter.cu:77-190
    assert declared_gf() == ["gf_create", "gf_free", "gf_last_error", "gf_ndist", "gf_query"]


def test_library_exports_the_gf_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gf_\w+)", out))
    assert set(declared_gf()) <= exported
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_gf()) <= bound


def test_null_handle_errors_without_a_device():
    lib = _lib.load()
    q = np.zeros(8, np.float32)
    out = np.zeros(4, np.int64)
    got = lib.gf_query(None, q.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 4, 10,
                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    assert got == -1
    assert "gf_query" in lib.gf_last_error().decode()
    assert lib.gf_ndist(None) == 0
    lib.gf_free(None)  # a no-op, as the reference's


def test_create_rejects_what_the_reference_rejects():
    lib = _lib.load()
    x = np.zeros((4, 4097), np.float32)
    h = lib.gf_create(x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 4, 4097)
    assert not h
    assert lib.gf_last_error().decode() == "dim 4097 > 4096 unsupported"


def test_create_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    from annvedi_b200.gpu_filter import Algorithm
    with pytest.raises(RuntimeError, match="no CUDA device"):
        Algorithm().fit(np.ones((16, 8), np.float32))


def test_query_before_fit():
    from annvedi_b200.gpu_filter import Algorithm
    with pytest.raises(RuntimeError, match="not fitted"):
        Algorithm().query(np.zeros(8, np.float32), 5)
    assert Algorithm().get_n_distances() == 0


def test_restatement_matches_the_reference_goldens(golden_dir):
    """oracle/restate.c's gf restatement against the reference library's own outputs
    (tests/golden/gf_ref.npz, made by tests/golden/make_gf_golden.py on a GPU)."""
    from oracle import refmod
    from tests.golden.make_gf_golden import cases
    g = np.load(os.path.join(golden_dir, "gf_ref.npz"))
    for name, x, qs, k, r in cases():
        got, ids, ndist = refmod.gf_search(x, qs, k, r)
        np.testing.assert_array_equal(got, g[f"{name}_got"], err_msg=name)
        np.testing.assert_array_equal(ids, g[f"{name}_ids"], err_msg=name)
        assert ndist == int(g[f"{name}_ndist"]), name
