"""The C-ABI library: builds for sm_100a, loads without a GPU, exports every declared symbol, and
reports a clear error (not a crash) when no device is visible. No compute calls here."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

from annvedi_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(ann_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "ann_flat_query" in names and "ann_last_error" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (ann_\w+)", out))
    assert set(declared_functions()) <= exported


def test_bindings_cover_the_header():
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound, set(declared_functions()) - bound


def test_version_and_error_without_device():
    assert _lib.version().startswith("annvedi_b200")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.ann_flat_create(ctypes.byref(h), 0)
    assert rc == _lib.ANN_ERR_CUDA
    assert "CUDA" in _lib.last_error() or "device" in _lib.last_error()


def test_library_is_built_for_sm100a_only():
    from annvedi_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_loaded_library_runs_sm100a_machine_code(cuda):
    out = (ctypes.c_int32 * 2)()
    _lib.check(_lib.load().ann_kernel_arch(0, out))
    assert out[0] == 100, f"binary version {out[0]}"
