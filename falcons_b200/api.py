"""pyfalcons-compatible host API on the B200 path (NumPy arrays in host memory).

Mirrors the reference's Python frontend (tools/pyfalcons/src/pyfalcons/falcons.pyx:31-153,
pyConfig.pyx, pyConfigEnums.py): the same class and method names, argument meaning, return
values and error types.  Every call goes through the C ABI of libfalcons_b200.so.

    from falcons_b200.api import falcons, falconsConfig, falconsErrorBoundMode
    conf = falconsConfig(100, 200, 300)
    conf.errorBoundMode = falconsErrorBoundMode.ABS
    conf.absErrorBound = 1e-3
    compressed, ratio = falcons.compress(data, conf)          # data is overwritten (copy=False)
    restored, conf_out = falcons.decompress(compressed, np.float32, data.shape)

Only float32 and float64 fields are supported on the GPU build; int32/int64 raise TypeError.
"""
from __future__ import annotations

import ctypes
import operator
from enum import IntEnum

import numpy as np

from . import _lib

__all__ = ["falcons", "falconsConfig", "falconsErrorBoundMode", "falconsAlgorithm", "falconsInterpAlgorithm",
           "Config", "compress", "decompress", "read_config", "size_bound"]


class falconsErrorBoundMode(IntEnum):
    ABS = 0
    REL = 1
    PSNR = 2
    L2NORM = 3
    ABS_AND_REL = 4
    ABS_OR_REL = 5


class falconsAlgorithm(IntEnum):
    LORENZO_REG = 0
    INTERP_LORENZO = 1
    INTERP = 2
    NOPRED = 3
    LOSSLESS = 4


class falconsInterpAlgorithm(IntEnum):
    LINEAR = 0
    CUBIC = 1


_DT = {np.dtype(np.float32): _lib.F32, np.dtype(np.float64): _lib.F64}
_SUPPORTED = frozenset(_DT)


class falconsConfig:
    """Falcons::Config (utils/Config.hpp:142-512) on the fields the path uses."""

    def __init__(self, *dims, **kwargs):
        self.conf = _lib.Config()
        self.conf.N = 1
        self.conf.dims[0] = 1
        self.conf.cmprAlgo = falconsAlgorithm.INTERP_LORENZO
        self.conf.errorBoundMode = falconsErrorBoundMode.ABS
        self.conf.absErrorBound = 1e-3
        self.conf.lorenzo = 1
        self.conf.regression = 1
        self.conf.quantbinCnt = 65536
        self.conf.interpAlgo = falconsInterpAlgorithm.CUBIC
        self.conf.interpDirection = 0
        self.conf.interpAnchorStride = -1
        self.conf.interpAlpha = 1.25
        self.conf.interpBeta = 2.0
        if len(dims) == 1 and isinstance(dims[0], (tuple, list)):
            dims = tuple(dims[0])
        self.setDims(*(dims or (1,)))
        for k, v in kwargs.items():
            if k in ("errorBoundMode",) and isinstance(v, str):
                v = falconsErrorBoundMode[v]
            if k in ("cmprAlgo",) and isinstance(v, str):
                v = falconsAlgorithm[v]
            setattr(self, k, v)

    def setDims(self, *dims):
        if len(dims) == 1 and isinstance(dims[0], (tuple, list)):
            dims = tuple(dims[0])
        d = [int(x) for x in dims if int(x) > 1] or [1]
        if len(d) > 4:
            raise ValueError("Data dimension higher than 4 is not supported.")
        self.conf.N = len(d)
        for i in range(4):
            self.conf.dims[i] = d[i] if i < len(d) else 0
        n = 1
        for x in d:
            n *= x
        self.conf.num = n
        self.conf.predDim = len(d)
        self.conf.blockSize = 128 if len(d) == 1 else (16 if len(d) == 2 else 6)
        return n

    @property
    def dims(self):
        return tuple(int(self.conf.dims[i]) for i in range(self.conf.N))

    @property
    def N(self):
        return int(self.conf.N)

    @property
    def num_elements(self):
        return int(self.conf.num)

    def loadcfg(self, path):
        """Loads an INI file in the reference's format (Config::loadcfg, Config.hpp:189-276)."""
        with open(path) as f:
            self.load_ini(f.read())

    def load_ini(self, text):
        section = ""
        truth = {"true", "1", "yes", "on"}
        for raw in text.splitlines():
            line = raw.strip()
            if not line or line.startswith("#"):
                continue
            if line.startswith("["):
                section = line[1:line.find("]")].lower()
                continue
            if "=" not in line:
                continue
            k, v = (s.strip() for s in line.split("=", 1))
            k = k.lower()
            if section == "globalsettings":
                if k == "cmpralgo":
                    self.conf.cmprAlgo = falconsAlgorithm[v.upper().replace("ALGO_", "")]
                elif k == "errorboundmode":
                    m = {"abs": 0, "rel": 1, "psnr": 2, "norm": 3, "abs_and_rel": 4, "abs_or_rel": 5}
                    self.conf.errorBoundMode = m[v.lower()]
                elif k == "abserrorbound":
                    self.conf.absErrorBound = float(v)
                elif k == "relerrorbound":
                    self.conf.relErrorBound = float(v)
                elif k == "psnrerrorbound":
                    self.conf.psnrErrorBound = float(v)
                elif k == "l2normerrorbound":
                    self.conf.l2normErrorBound = float(v)
                elif k == "openmp":
                    self.conf.openmp = int(v.lower() in truth)
            elif section == "algosettings":
                if k in ("lorenzo", "lorenzo2ndorder", "regression", "regression2ndorder"):
                    name = {"lorenzo": "lorenzo", "lorenzo2ndorder": "lorenzo2", "regression": "regression",
                            "regression2ndorder": "regression2"}[k]
                    setattr(self.conf, name, int(v.lower() in truth))
                elif k == "interpolationalgo":
                    self.conf.interpAlgo = falconsInterpAlgorithm[v.upper().replace("INTERP_ALGO_", "")]
                elif k == "interpolationdirection":
                    self.conf.interpDirection = int(v)
                elif k == "blocksize":
                    self.conf.blockSize = int(v)
                elif k == "quantizationbintotal":
                    self.conf.quantbinCnt = int(v)
                elif k == "interpolationanchorstride":
                    self.conf.interpAnchorStride = int(v)
                elif k == "interpolationalpha":
                    self.conf.interpAlpha = float(v)
                elif k == "interpolationbeta":
                    self.conf.interpBeta = float(v)


def _prop(name, cast=float):
    def g(self):
        return cast(getattr(self.conf, name))

    def s(self, v):
        if hasattr(v, "value"):
            v = v.value
        setattr(self.conf, name, cast(v))
    return property(g, s)


for _n, _c in [("absErrorBound", float), ("relErrorBound", float), ("psnrErrorBound", float),
               ("l2normErrorBound", float), ("quantbinCnt", int), ("blockSize", int),
               ("interpDirection", int), ("interpAnchorStride", int), ("interpAlpha", float),
               ("interpBeta", float), ("lorenzo", bool), ("lorenzo2", bool), ("regression", bool),
               ("regression2", bool), ("openmp", bool), ("dataType", int)]:
    setattr(falconsConfig, _n, _prop(_n, _c))


def _enum_prop(name, enum):
    def g(self):
        return enum(int(getattr(self.conf, name)))

    def s(self, v):
        if not hasattr(v, "value"):
            raise TypeError(f"Use {enum.__name__} enum, got {type(v).__name__}")
        setattr(self.conf, name, int(v.value))
    return property(g, s)


falconsConfig.errorBoundMode = _enum_prop("errorBoundMode", falconsErrorBoundMode)
falconsConfig.cmprAlgo = _enum_prop("cmprAlgo", falconsAlgorithm)
falconsConfig.interpAlgo = _enum_prop("interpAlgo", falconsInterpAlgorithm)
Config = falconsConfig


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def size_bound(config: falconsConfig, dtype) -> int:
    dt = np.dtype(dtype)
    if dt not in _SUPPORTED:
        raise TypeError(f"Unsupported dtype: {dt}. Supported on the GPU build: float32, float64")
    return int(_lib.lib().falcons_compress_size_bound(_DT[dt], ctypes.byref(config.conf)))


class falcons:
    """Static compress / decompress / verify, as pyfalcons.falcons."""

    @staticmethod
    def compress(data: np.ndarray, config, copy: bool = False, ctx=None):
        if not isinstance(data, np.ndarray):
            raise TypeError("data must be a NumPy array")
        if data.dtype not in _SUPPORTED:
            raise TypeError(f"Unsupported dtype: {data.dtype}. Supported on the GPU build: float32, float64")
        if data.size == 0:
            raise ValueError("Cannot compress an empty array")
        if isinstance(config, str):
            path = config
            config = falconsConfig(*data.shape)
            config.loadcfg(path)
        elif isinstance(config, falconsConfig):
            if config.num_elements != data.size:
                config.setDims(*data.shape)
        else:
            raise TypeError(f"config must be falconsConfig or str, got {type(config)}")
        if copy:
            data = np.array(data, order="C", copy=True)
        else:
            if not data.flags["C_CONTIGUOUS"]:
                raise ValueError("copy=False requires a C-contiguous array; pass copy=True")
            if not data.flags["WRITEABLE"]:
                raise ValueError("copy=False requires a writable array; pass copy=True")
        ctx = ctx or _lib.default_context(0)
        cap = size_bound(config, data.dtype)
        out = np.empty(cap, np.uint8)
        n = ctypes.c_size_t(0)
        conf_out = _lib.Config()
        flags = 0 if copy else _lib.FLAG_WRITEBACK
        _lib.check(_lib.lib().falcons_compress(ctx.ptr, _DT[data.dtype], ctypes.byref(config.conf), _ptr(data),
                                               ctypes.c_uint32(flags), _ptr(out), ctypes.c_size_t(cap),
                                               ctypes.byref(n), ctypes.byref(conf_out)), "compress")
        out = out[:n.value]
        return out, data.nbytes / float(n.value)

    @staticmethod
    def decompress(compressed: np.ndarray, dtype, shape=None, config=None, ctx=None):
        if not isinstance(compressed, np.ndarray) or compressed.dtype != np.uint8:
            raise TypeError("Compressed data must be a uint8 NumPy array")
        dtype = np.dtype(dtype)
        if dtype not in _SUPPORTED:
            raise TypeError(f"Unsupported dtype: {dtype}. Supported on the GPU build: float32, float64")
        compressed = np.ascontiguousarray(compressed)
        hdr = _lib.Config()
        _lib.check(_lib.lib().falcons_read_config(_ptr(compressed), ctypes.c_size_t(compressed.size),
                                                  ctypes.byref(hdr)), "read_config")
        num = int(hdr.num)
        if shape is not None:
            shape = tuple(operator.index(d) for d in shape)
            if not shape or any(d <= 0 for d in shape):
                raise ValueError("Shape dimensions must be positive integers")
            if int(np.prod(shape)) != num:
                raise ValueError("Requested shape does not match the compressed element count")
        else:
            shape = tuple(int(hdr.dims[i]) for i in range(hdr.N))
        ctx = ctx or _lib.default_context(0)
        result = np.empty(num, dtype)
        conf_out = _lib.Config()
        _lib.check(_lib.lib().falcons_decompress(ctx.ptr, _DT[dtype], _ptr(compressed),
                                                 ctypes.c_size_t(compressed.size), _ptr(result),
                                                 ctypes.c_size_t(num), ctypes.byref(conf_out)), "decompress")
        conf = config if isinstance(config, falconsConfig) else falconsConfig(*shape)
        conf.conf = conf_out
        return result.reshape(shape), conf

    @staticmethod
    def verify(src_data: np.ndarray, dec_data: np.ndarray):
        """(max abs error, PSNR dB, NRMSE), as the reference's verify (utils/Statistic.hpp:264-359)."""
        if np.shape(src_data) != np.shape(dec_data):
            raise ValueError("Shape mismatch between src_data and dec_data")
        if src_data.dtype != dec_data.dtype:
            raise ValueError("Dtype mismatch between src_data and dec_data")
        if src_data.size == 0:
            raise ValueError("Cannot verify empty arrays")
        src = src_data.astype(np.float64)
        diff = src - dec_data.astype(np.float64)
        rng = float(src.max() - src.min())
        max_diff = float(np.max(np.abs(diff)))
        mse = float(np.mean(diff ** 2))
        if mse == 0:
            return max_diff, float("inf"), 0.0
        if rng == 0:
            return max_diff, -float("inf"), float("inf")
        nrmse = float(np.sqrt(mse) / rng)
        return max_diff, float(-20 * np.log10(nrmse)), nrmse


def compress(data, config, copy=False, ctx=None):
    return falcons.compress(data, config, copy, ctx)


def decompress(compressed, dtype, shape=None, config=None, ctx=None):
    return falcons.decompress(compressed, dtype, shape, config, ctx)


def read_config(compressed: np.ndarray) -> falconsConfig:
    compressed = np.ascontiguousarray(compressed, np.uint8)
    hdr = _lib.Config()
    _lib.check(_lib.lib().falcons_read_config(_ptr(compressed), ctypes.c_size_t(compressed.size),
                                              ctypes.byref(hdr)), "read_config")
    c = falconsConfig(*[int(hdr.dims[i]) for i in range(hdr.N)])
    c.conf = hdr
    return c
