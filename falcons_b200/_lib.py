"""ctypes binding of libfalcons_b200.so (the C ABI in include/falcons_b200.h).

The library is built in-tree by falcons_b200/build.py.  Loading fails loudly when it is
missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfalcons_b200.so")

F32, F64 = 0, 1
OK, EINVAL, ELENGTH, ERUNTIME, ECUDA, ENOMEM = range(6)
FLAG_WRITEBACK = 1


class FalconsError(RuntimeError):
    pass


class InterpParams(ctypes.Structure):
    _fields_ = [("eb", ctypes.c_double), ("interp_algo", ctypes.c_int32), ("direction", ctypes.c_int32),
                ("anchor_stride", ctypes.c_int64), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
                ("radius", ctypes.c_int32), ("tuning", ctypes.c_int32), ("max_abs", ctypes.c_double)]


class Config(ctypes.Structure):
    """falcons_config: the Falcons::Config fields the path reads and writes."""
    _fields_ = [("N", ctypes.c_int32), ("dims", ctypes.c_uint64 * 4), ("num", ctypes.c_uint64),
                ("cmprAlgo", ctypes.c_int32), ("errorBoundMode", ctypes.c_int32),
                ("absErrorBound", ctypes.c_double), ("relErrorBound", ctypes.c_double),
                ("psnrErrorBound", ctypes.c_double), ("l2normErrorBound", ctypes.c_double),
                ("lorenzo", ctypes.c_int32), ("lorenzo2", ctypes.c_int32), ("regression", ctypes.c_int32),
                ("regression2", ctypes.c_int32), ("openmp", ctypes.c_int32), ("quantbinCnt", ctypes.c_int32),
                ("blockSize", ctypes.c_int32), ("predDim", ctypes.c_int32), ("dataType", ctypes.c_int32),
                ("interpAlgo", ctypes.c_int32), ("interpDirection", ctypes.c_int32),
                ("interpAnchorStride", ctypes.c_int32), ("interpAlpha", ctypes.c_double),
                ("interpBeta", ctypes.c_double)]


class BatchItem(ctypes.Structure):
    """falcons_batch_item: one field of a batch call."""
    _fields_ = [("dtype", ctypes.c_int32), ("status", ctypes.c_int32), ("conf", Config),
                ("d_data", ctypes.c_void_p), ("d_stream", ctypes.c_void_p), ("cap", ctypes.c_size_t),
                ("len", ctypes.c_size_t)]


_lib = None
_lock = threading.Lock()

EXPORTS = [
    "falcons_ctx_create", "falcons_ctx_destroy", "falcons_last_error", "falcons_version", "falcons_kernel_launches",
    "falcons_compress_size_bound", "falcons_compress", "falcons_read_config", "falcons_decompress",
    "falcons_compress_device", "falcons_decompress_device", "falcons_interp_compress",
    "falcons_interp_decompress", "falcons_device_range", "falcons_encode_codes", "falcons_decode_codes",
    "falcons_interp_decompress_noalloc", "falcons_compress_batch", "falcons_decompress_batch",
    "falcons_batch_workers", "falcons_time_levels", "falcons_level_times",
]


def lib() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FalconsError(f"{LIB_PATH} is missing: build it with `python -m falcons_b200.build` "
                                   "(the CUDA extension is required; there is no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            L.falcons_last_error.restype = ctypes.c_char_p
            L.falcons_version.restype = ctypes.c_char_p
            L.falcons_kernel_launches.restype = ctypes.c_uint64
            L.falcons_compress_size_bound.restype = ctypes.c_size_t
            L.falcons_compress_size_bound.argtypes = [ctypes.c_int, ctypes.POINTER(Config)]
            for name in EXPORTS:
                getattr(L, name)  # fail loudly on a missing symbol
            _lib = L
        return _lib


def check(rc: int, what: str = "falcons"):
    if rc != OK:
        msg = lib().falcons_last_error().decode(errors="replace")
        if rc == EINVAL:
            raise ValueError(f"{what}: {msg}")
        if rc == ELENGTH:
            raise OverflowError(f"{what}: {msg}")
        raise FalconsError(f"{what}: {msg} (status {rc})")


class Context:
    """A library context bound to one CUDA device (owns scratch buffers and a stream)."""

    def __init__(self, device: int = 0):
        self.ptr = ctypes.c_void_p()
        check(lib().falcons_ctx_create(ctypes.byref(self.ptr), int(device)), "ctx_create")
        self.device = device

    def close(self):
        if self.ptr:
            lib().falcons_ctx_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = {}


def default_context(device: int = 0) -> Context:
    with _lock:
        if device not in _default_ctx:
            _default_ctx[device] = None
    if _default_ctx[device] is None:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]
