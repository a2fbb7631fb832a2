"""ctypes binding of libannvedi_b200.so (include/annvedi_b200.h).

The library is built in-tree by ``python -m annvedi_b200.build``. There is no fallback: importing
an index class when the library is missing, or creating one without a visible CUDA device,
raises. Every non-zero status becomes a Python exception carrying ``ann_last_error()``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libannvedi_b200.so")

ANN_OK = 0
ANN_ERR_INVALID = -1
ANN_ERR_CUDA = -2
ANN_ERR_STATE = -3
ANN_ERR_NOMEM = -4
ANN_ERR_TIMEOUT = -5
ANN_ERR_UNSUPPORTED = -6

METRIC_L2 = 0
METRIC_IP = 1
MODE_EXACT = 0
MODE_REFERENCE = 1
MEM_HOST = 0
MEM_DEVICE = 1

METRICS = {"l2": METRIC_L2, "sqeuclidean": METRIC_L2, "euclidean": METRIC_L2, "ip": METRIC_IP,
           "inner_product": METRIC_IP, "dot": METRIC_IP}
MODE_TC = 2
MODE_TC_SQ8 = 3
QUERY_SHARD = 0x100
MODES = {"exact": MODE_EXACT, "reference": MODE_REFERENCE, "tc": MODE_TC, "tc_sq8": MODE_TC_SQ8}


class AnnError(RuntimeError):
    """A failing call into the native library."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class AnnMemoryError(AnnError, MemoryError):
    pass


class AnnUnsupported(AnnError, NotImplementedError):
    pass


class AnnTimeout(AnnError, TimeoutError):
    pass


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_lib = None

# (name, restype, argtypes) of every exported function the bindings use.
SIGNATURES = [
    ("ann_version", ctypes.c_char_p, []),
    ("ann_kernel_arch", ctypes.c_int, [_i32, _vp]),
    ("ann_tc_wait_selftest", ctypes.c_int, [_i32, _i64, _vp]),
    ("ann_last_error", ctypes.c_char_p, []),
    ("ann_kernel_launches", _i64, []),
    ("ann_workspace_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    ("ann_workspace_destroy", ctypes.c_int, [_vp]),
    ("ann_workspace_bytes", _i64, [_vp]),
    ("ann_flat_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    ("ann_flat_destroy", ctypes.c_int, [_vp]),
    ("ann_flat_fit", ctypes.c_int, [_vp, _vp, _i64, _i32, _i64, _i32, _i32, _vp]),
    ("ann_flat_query", ctypes.c_int, [_vp, _vp, _vp, _i32, _i64, _i32, _i32, _i32, _vp, _vp, _vp]),
    ("ann_flat_query_noalloc", ctypes.c_int, [_vp, _vp, _i32, _i64, _i32, _vp, _vp, _vp]),
    ("ann_flat_query_tc", ctypes.c_int, [_vp, _vp, _vp, _i32, _i64, _i32, _i32, _i32, _vp, _vp, _vp]),
    ("ann_flat_scores_tc", ctypes.c_int, [_vp, _vp, _i32, _i64, _vp, _vp]),
    ("ann_flat_set_tc_precision", ctypes.c_int, [_vp, _i32]),
    ("ann_flat_set_option", ctypes.c_int, [_vp, _i32, ctypes.c_int64]),
    ("ann_flat_device_status", ctypes.c_int, [_vp]),
    ("ann_merge_topk", ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp]),
    ("ann_select_smallest", ctypes.c_int, [_vp, _i64, _vp, _i32, _i32, _vp, _vp, _vp]),
    ("ann_flat_set_profiling", ctypes.c_int, [_vp, _i32]),
    ("ann_flat_profile", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("ann_flat_reset_profile", ctypes.c_int, [_vp]),
    ("ann_flat_profile_stages", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("ann_flat_total_distances", _i64, [_vp]),
    ("ann_flat_dim", _i32, [_vp]),
    ("ann_flat_size", _i64, [_vp]),
    ("ann_ivf_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    ("ann_ivf_destroy", ctypes.c_int, [_vp]),
    ("ann_ivf_fit", ctypes.c_int, [_vp, _vp, _i64, _i32, _i64, _i32, _vp, _vp, _i32, _i32, _i32, _vp]),
    ("ann_ivf_import", ctypes.c_int, [_vp, _i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("ann_ivf_export", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("ann_ivf_info", ctypes.c_int, [_vp, ctypes.POINTER(_i64)]),
    ("ann_ivf_query", ctypes.c_int, [_vp, _vp, _vp, _i32, _i64, _i32, _i32, _i32, _i32, _i64, _i32, _i32, _i32,
                                     _vp, _vp, _vp]),
    ("ann_ivf_device_status", ctypes.c_int, [_vp]),
    ("ann_ivf_import_tables", ctypes.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp]),
    ("ann_ivf_build_tables", ctypes.c_int, [_vp, _i32, _i32, _vp]),
    ("ann_ivf_export_tables", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("ann_ivf_total_distances", _i64, [_vp]),
    ("ann_ivf_reset_distances", ctypes.c_int, [_vp]),
    ("ann_ivf_set_profiling", ctypes.c_int, [_vp, _i32]),
    ("ann_ivf_profile", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("ann_ivf_kernel_profile", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("ann_ivf_set_option", ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int64]),
    ("ann_ivf_reset_profile", ctypes.c_int, [_vp]),
    # the reference GPU contestant's ABI (include/annvedi_gpu_filter.h)
    ("gf_last_error", ctypes.c_char_p, []),
    ("gf_create", _vp, [ctypes.POINTER(ctypes.c_float), ctypes.c_long, ctypes.c_long]),
    ("gf_query", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_longlong)]),
    ("gf_ndist", ctypes.c_longlong, [_vp]),
    ("gf_free", None, [_vp]),
]


def load():
    """Loads the library (once). Raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m annvedi_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().ann_last_error().decode(errors="replace")


def check(status: int) -> None:
    if status == ANN_OK:
        return
    msg = last_error() or f"status {status}"
    if status == ANN_ERR_NOMEM:
        raise AnnMemoryError(status, msg)
    if status == ANN_ERR_UNSUPPORTED:
        raise AnnUnsupported(status, msg)
    if status == ANN_ERR_TIMEOUT:
        raise AnnTimeout(status, msg)
    if status == ANN_ERR_INVALID:
        raise AnnError(status, msg)
    raise AnnError(status, msg)


def version() -> str:
    return load().ann_version().decode()


def kernel_launches() -> int:
    """Kernels launched by the library in this process so far."""
    return int(load().ann_kernel_launches())


# ---- pointer helpers ------------------------------------------------------------------------

def is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def ptr(x):
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if x is None:
        return None
    if is_torch(x):
        return x.data_ptr()
    return x.ctypes.data


def stream_ptr(x, stream=None):
    """The CUDA stream to run on: an explicit torch stream / int handle, else torch's current
    stream for device tensors, else NULL (legacy default stream)."""
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    if x is not None and is_torch(x) and x.is_cuda:
        import torch
        return torch.cuda.current_stream(x.device).cuda_stream
    return None


def as_f32_2d(x, name="array"):
    """Host float32 C-ordered 2-D view of `x` (numpy), or a device tensor checked for layout."""
    if is_torch(x):
        if x.dtype.__str__() != "torch.float32":
            x = x.float()
        if x.dim() != 2:
            raise RuntimeError(f"{name} must be 2-D, got shape {tuple(x.shape)}")
        if x.stride(1) != 1:
            x = x.contiguous()
        return x
    a = np.asarray(x)
    if a.ndim != 2:
        raise RuntimeError(f"{name} must be 2-D, got shape {a.shape}")
    return np.ascontiguousarray(a, dtype=np.float32)
