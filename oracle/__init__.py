"""ORACLE — test infrastructure, never product code.

Python access to the two CPU restatements the tests compare the CUDA path with:

* ``Restatement`` wraps ``oracle/liboracle.so``, the plain-C restatements of the reference's
  interpolation decomposition (oracle/interp_oracle.c) and of its 1-D blockwise Lorenzo +
  Huffman path (oracle/lorenzo_oracle.c).  It is built by ``make -C oracle`` and needs no
  reference sources, so it is available on any machine with gcc.
* ``Reference`` wraps ``oracle/_ref/libfalcons_ref.so`` (scalar, serial) or
  ``libfalcons_ref_omp.so`` (AVX2 + OpenMP), built from the reference's own headers by
  ``make -C oracle ref``.  It exists only where the reference sources were present at
  build time.

Only tests/, __graft_entry__.smoke(), tests/golden/make_golden.py and bench.py's CPU
baseline leg import this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfalcons_ref.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libfalcons_ref_omp.so")

# Config enums (include/Falcons/utils/Config.hpp:55-72)
EB_ABS, EB_REL, EB_PSNR, EB_L2NORM, EB_ABS_AND_REL, EB_ABS_OR_REL = range(6)
ALGO_LORENZO_REG, ALGO_INTERP_LORENZO, ALGO_INTERP, ALGO_NOPRED, ALGO_LOSSLESS = range(5)
INTERP_LINEAR, INTERP_CUBIC = 0, 1
DEFAULT_ANCHOR = {1: 4096, 2: 128, 3: 32, 4: 16}


def ensure_restatement() -> str:
    """Build liboracle.so if missing (gcc only)."""
    src = [os.path.join(HERE, f) for f in ("interp_oracle.c", "interp_oracle_impl.h", "lorenzo_oracle.c",
                                           "lorenzo_oracle_impl.h", "Makefile")]
    if (not os.path.exists(RESTATEMENT_SO)
            or any(os.path.getmtime(s) > os.path.getmtime(RESTATEMENT_SO) for s in src)):
        subprocess.check_call(["make", "-s", "-C", HERE, "restatement"])
    return RESTATEMENT_SO


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _ctype(dtype):
    return ctypes.c_float if np.dtype(dtype) == np.float32 else ctypes.c_double


def _sfx(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def anchor_count(dims, anchor):
    """Number of anchor points the anchor grid stores (0 when no dim exceeds the stride)."""
    if anchor <= 0 or not any(d > anchor for d in dims):
        return 0
    n = 1
    for d in dims:
        n *= (d - 1) // anchor + 1
    return n


@dataclass
class InterpResult:
    codes: np.ndarray      # int16, stream order
    unpred: np.ndarray     # T, anchors first then escapes in stream order
    recon: np.ndarray      # T, C order (the decompressed field)
    mutated: np.ndarray    # T, the input buffer after compression (partial reconstruction)


class Restatement:
    """The C restatements: the interpolation decomposition, and the 1-D Lorenzo + Huffman path."""

    def __init__(self, path: str | None = None):
        self.lib = ctypes.CDLL(path or ensure_restatement())
        for name in ("oracle_lorenzo_payload_f32", "oracle_lorenzo_payload_f64", "oracle_lorenzo_decode_f32",
                     "oracle_lorenzo_decode_f64", "oracle_huffman_encode", "oracle_huffman_decode"):
            getattr(self.lib, name).restype = ctypes.c_longlong

    def lorenzo_payload(self, x: np.ndarray, eb: float, radius: int = 32768, block: int = 5):
        """(payload, reconstruction) of the 1-D blockwise Lorenzo path: the bytes the reference
        hands to its trailing zstd stage (FalconsGenericCompressor.hpp:64-81)."""
        x = np.ascontiguousarray(x).ravel()
        cap = 4096 + x.size * (x.itemsize + 8) + 2 * 65540
        out = np.empty(cap, np.uint8)
        recon = np.empty_like(x)
        ct = _ctype(x.dtype)
        n = getattr(self.lib, f"oracle_lorenzo_payload_{_sfx(x.dtype)}")(
            _ptr(x, ct), ctypes.c_size_t(x.size), ctypes.c_double(eb), ctypes.c_int(radius), ctypes.c_int(block),
            _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap), _ptr(recon, ct))
        if n < 0:
            raise RuntimeError(f"oracle lorenzo payload failed: {n}")
        return out[:n].tobytes(), recon

    def lorenzo_decode(self, payload: bytes, n: int, dtype, block: int = 5) -> np.ndarray:
        buf = np.frombuffer(payload, np.uint8)
        out = np.empty(n, dtype)
        used = getattr(self.lib, f"oracle_lorenzo_decode_{_sfx(dtype)}")(
            _ptr(buf, ctypes.c_uint8), ctypes.c_size_t(len(payload)), ctypes.c_size_t(n), ctypes.c_int(block),
            _ptr(out, _ctype(dtype)))
        if used < 0:
            raise ValueError(f"oracle lorenzo decode failed: {used}")
        if used != len(payload):
            raise ValueError(f"oracle lorenzo decode: {len(payload) - used} trailing bytes")
        return out

    def huffman_encode(self, sym: np.ndarray) -> bytes:
        """One Huffman record (HuffmanEncoder<int>::save + encode) of symbols in [0, 65536)."""
        sym = np.ascontiguousarray(sym, np.int32)
        cap = 64 + 2 * 65540 + sym.size * 5
        out = np.empty(cap, np.uint8)
        n = self.lib.oracle_huffman_encode(_ptr(sym, ctypes.c_int32), ctypes.c_size_t(sym.size),
                                           _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap))
        if n < 0:
            raise RuntimeError(f"oracle huffman encode failed: {n}")
        return out[:n].tobytes()

    def huffman_decode(self, rec: bytes, n: int) -> np.ndarray:
        buf = np.frombuffer(rec, np.uint8)
        out = np.empty(max(n, 1), np.int32)
        used = self.lib.oracle_huffman_decode(_ptr(buf, ctypes.c_uint8), ctypes.c_size_t(len(rec)), ctypes.c_size_t(n),
                                              _ptr(out, ctypes.c_int32))
        if used < 0:
            raise ValueError(f"oracle huffman decode failed: {used}")
        return out[:n]

    def _call(self, name, *args):
        rc = getattr(self.lib, name)(*args)
        if rc != 0:
            raise RuntimeError(f"{name} failed: {rc}")

    def compress(self, x: np.ndarray, eb: float, algo: int = INTERP_CUBIC, direction: int = 0,
                 anchor: int | None = None, alpha: float = 1.25, beta: float = 2.0,
                 tuning: bool = False) -> InterpResult:
        x = np.ascontiguousarray(x)
        dims = (ctypes.c_size_t * x.ndim)(*x.shape)
        anchor = DEFAULT_ANCHOR[x.ndim] if anchor is None else anchor
        work = x.copy()
        codes = np.empty(x.size + 16, np.int16)
        unpred = np.empty(x.size + anchor_count(x.shape, anchor) + 16, x.dtype)
        nq, nu = ctypes.c_size_t(0), ctypes.c_size_t(0)
        ct = _ctype(x.dtype)
        self._call(f"oracle_interp_compress_{_sfx(x.dtype)}", dims, x.ndim, ctypes.c_double(eb), algo, direction,
                   ctypes.c_long(anchor), ctypes.c_double(alpha), ctypes.c_double(beta), int(tuning),
                   _ptr(work, ct), _ptr(codes, ctypes.c_int16), ctypes.byref(nq), _ptr(unpred, ct), ctypes.byref(nu))
        codes = codes[:nq.value].copy()
        unpred = unpred[:nu.value].copy()
        recon = self.decompress(x.shape, x.dtype, codes, unpred, eb, algo, direction, anchor, alpha, beta) \
            if not tuning else None
        return InterpResult(codes, unpred, recon, work)

    def decompress(self, shape, dtype, codes, unpred, eb, algo=INTERP_CUBIC, direction=0, anchor=None,
                   alpha=1.25, beta=2.0) -> np.ndarray:
        dims = (ctypes.c_size_t * len(shape))(*shape)
        anchor = DEFAULT_ANCHOR[len(shape)] if anchor is None else anchor
        out = np.zeros(shape, dtype)
        codes = np.ascontiguousarray(codes, np.int16)
        unpred = np.ascontiguousarray(unpred, dtype)
        ct = _ctype(dtype)
        self._call(f"oracle_interp_decompress_{_sfx(dtype)}", dims, len(shape), ctypes.c_double(eb), algo,
                   direction, ctypes.c_long(anchor), ctypes.c_double(alpha), ctypes.c_double(beta),
                   _ptr(codes, ctypes.c_int16), ctypes.c_size_t(codes.size), _ptr(unpred, ct),
                   ctypes.c_size_t(unpred.size), _ptr(out, ct))
        return out


class RefConf(ctypes.Structure):
    _fields_ = [
        ("cmprAlgo", ctypes.c_int32), ("errorBoundMode", ctypes.c_int32),
        ("absErrorBound", ctypes.c_double), ("relErrorBound", ctypes.c_double),
        ("psnrErrorBound", ctypes.c_double), ("l2normErrorBound", ctypes.c_double),
        ("interpAlgo", ctypes.c_int32), ("interpDirection", ctypes.c_int32),
        ("interpAnchorStride", ctypes.c_int32), ("openmp", ctypes.c_int32),
        ("interpAlpha", ctypes.c_double), ("interpBeta", ctypes.c_double),
        ("quantbinCnt", ctypes.c_int32), ("lorenzo", ctypes.c_int32), ("lorenzo2", ctypes.c_int32),
        ("regression", ctypes.c_int32), ("regression2", ctypes.c_int32), ("blockSize", ctypes.c_int32),
    ]


def ref_conf(algo=ALGO_INTERP, eb_mode=EB_ABS, abs_eb=1e-3, rel_eb=0.0, interp=INTERP_CUBIC, direction=0,
             anchor=-1, alpha=1.25, beta=2.0, openmp=False, psnr=0.0, l2=0.0) -> RefConf:
    """A reference Config with the defaults of include/Falcons/utils/Config.hpp:482-511."""
    return RefConf(algo, eb_mode, abs_eb, rel_eb, psnr, l2, interp, direction, anchor, int(openmp), alpha, beta,
                   65536, 1, 0, 1, 0, 0)


def lorenzo_ref_conf(abs_eb: float, quantbin: int = 65536) -> RefConf:
    """The Config the interpolation tuner hands to the 1-D Lorenzo path
    (api/impl/FalconsAlgoInterp.hpp:479-490): Lorenzo orders 1 and 2, no regression, block 5."""
    c = ref_conf(ALGO_LORENZO_REG, EB_ABS, abs_eb)
    c.lorenzo, c.lorenzo2, c.regression, c.regression2, c.blockSize = 1, 1, 0, 0, 5
    c.quantbinCnt = quantbin
    return c


ZSTD_MAGIC = b"\x28\xb5\x2f\xfd"


def lossless_section(stream: bytes, max_header: int = 4096) -> int:
    """Offset of the Lossless_zstd section ([u64 raw length][zstd frame],
    lossless/Lossless_zstd.hpp:29-45) after a stream's Config header."""
    for h in range(0, min(max_header, len(stream) - 12)):
        if stream[h + 8:h + 12] == ZSTD_MAGIC:
            raw = int.from_bytes(stream[h:h + 8], "little")
            if 0 < raw < (1 << 40):
                return h
    raise ValueError("no zstd section found")


def reference_available(omp: bool = False) -> bool:
    return os.path.exists(REF_OMP_SO if omp else REF_SO)


class Reference:
    """The reference itself, compiled from its sources (scalar serial, or AVX2+OpenMP)."""

    def __init__(self, omp: bool = False):
        path = REF_OMP_SO if omp else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.ref_last_error.restype = ctypes.c_char_p
        for n in ("ref_compress_f32", "ref_compress_f64", "ref_size_bound_f32", "ref_size_bound_f64",
                  "ref_rlefse_encode", "ref_rlefse_decode", "ref_zstd_compress", "ref_zstd_decompress"):
            getattr(self.lib, n).restype = ctypes.c_longlong

    def _err(self, what):
        raise RuntimeError(f"{what}: {self.lib.ref_last_error().decode()}")

    def size_bound(self, shape, dtype, conf: RefConf) -> int:
        dims = (ctypes.c_size_t * len(shape))(*shape)
        return int(getattr(self.lib, f"ref_size_bound_{_sfx(dtype)}")(dims, len(shape), ctypes.byref(conf)))

    def compress(self, x: np.ndarray, conf: RefConf, mutate: bool = False) -> bytes:
        """Falcons_compress; with mutate=True the caller's array is overwritten like the reference does."""
        work = x if mutate else np.ascontiguousarray(x).copy()
        dims = (ctypes.c_size_t * x.ndim)(*x.shape)
        cap = self.size_bound(x.shape, x.dtype, conf)
        out = np.empty(cap, np.uint8)
        n = getattr(self.lib, f"ref_compress_{_sfx(x.dtype)}")(dims, x.ndim, ctypes.byref(conf),
                                                               _ptr(work, _ctype(x.dtype)),
                                                               _ptr(out, ctypes.c_char), ctypes.c_size_t(cap))
        if n < 0:
            self._err("ref compress")
        return out[:n].tobytes()

    def decompress(self, stream: bytes, dtype, num: int):
        buf = np.frombuffer(stream, np.uint8)
        out = np.empty(num, dtype)
        dims = (ctypes.c_size_t * 4)()
        N = ctypes.c_int(0)
        rc = getattr(self.lib, f"ref_decompress_{_sfx(dtype)}")(_ptr(buf, ctypes.c_char), ctypes.c_size_t(len(stream)),
                                                                _ptr(out, _ctype(dtype)), ctypes.c_size_t(num), dims,
                                                                ctypes.byref(N))
        if rc != 0:
            self._err("ref decompress")
        shape = tuple(dims[i] for i in range(N.value))
        return out.reshape(shape)

    def interp_compress(self, x: np.ndarray, eb: float, algo=INTERP_CUBIC, direction=0, anchor=-1, alpha=1.25,
                        beta=2.0, tuning=False) -> InterpResult:
        x = np.ascontiguousarray(x)
        work = x.copy()
        dims = (ctypes.c_size_t * x.ndim)(*x.shape)
        conf = ref_conf(ALGO_INTERP, EB_ABS, eb, 0.0, algo, direction, anchor, alpha, beta)
        a = DEFAULT_ANCHOR[x.ndim] if anchor < 0 else anchor
        codes = np.empty(x.size + 16, np.int16)
        unpred = np.empty(x.size + anchor_count(x.shape, a) + 16, x.dtype)
        nq, nu = ctypes.c_size_t(codes.size), ctypes.c_size_t(unpred.size)
        ct = _ctype(x.dtype)
        rc = getattr(self.lib, f"ref_interp_compress_{_sfx(x.dtype)}")(
            dims, x.ndim, ctypes.byref(conf), int(tuning), _ptr(work, ct), _ptr(codes, ctypes.c_int16),
            ctypes.byref(nq), _ptr(unpred, ct), ctypes.byref(nu))
        if rc != 0:
            self._err("ref interp compress")
        codes = codes[:nq.value].copy()
        unpred = unpred[:nu.value].copy()
        recon = None if tuning else self.interp_decompress(x.shape, x.dtype, codes, unpred, eb, algo, direction,
                                                           anchor, alpha, beta)
        return InterpResult(codes, unpred, recon, work)

    def interp_decompress(self, shape, dtype, codes, unpred, eb, algo=INTERP_CUBIC, direction=0, anchor=-1,
                          alpha=1.25, beta=2.0) -> np.ndarray:
        dims = (ctypes.c_size_t * len(shape))(*shape)
        conf = ref_conf(ALGO_INTERP, EB_ABS, eb, 0.0, algo, direction, anchor, alpha, beta)
        out = np.zeros(shape, dtype)
        codes = np.ascontiguousarray(codes, np.int16)
        unpred = np.ascontiguousarray(unpred, dtype)
        ct = _ctype(dtype)
        rc = getattr(self.lib, f"ref_interp_decompress_{_sfx(dtype)}")(
            dims, len(shape), ctypes.byref(conf), _ptr(codes, ctypes.c_int16), ctypes.c_size_t(codes.size),
            _ptr(unpred, ct), ctypes.c_size_t(unpred.size), _ptr(out, ct))
        if rc != 0:
            self._err("ref interp decompress")
        return out

    def rlefse_encode(self, codes: np.ndarray) -> bytes:
        codes = np.ascontiguousarray(codes, np.int16)
        cap = 4 * codes.size + (1 << 20)
        out = np.empty(cap, np.uint8)
        n = self.lib.ref_rlefse_encode(_ptr(codes, ctypes.c_int16), ctypes.c_size_t(codes.size),
                                       _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap))
        if n < 0:
            self._err("ref rlefse encode")
        return out[:n].tobytes()

    def rlefse_decode(self, payload: bytes, n_codes: int) -> np.ndarray:
        buf = np.frombuffer(payload, np.uint8)
        out = np.empty(n_codes + 16, np.int16)
        n = self.lib.ref_rlefse_decode(_ptr(buf, ctypes.c_uint8), ctypes.c_size_t(len(payload)),
                                       ctypes.c_size_t(n_codes), _ptr(out, ctypes.c_int16))
        if n < 0:
            self._err("ref rlefse decode")
        return out[:n_codes].copy()

    def lorenzo_payload(self, x: np.ndarray, eb: float, quantbin: int = 65536):
        """(payload, buffer after compress) of the reference's 1-D blockwise Lorenzo path, stage by
        stage: the bytes FalconsGenericCompressor hands to zstd, without the dispatcher's lossless
        choice.  The path compresses a padded copy (utils/BlockwiseIterator.hpp:202-221), so the
        buffer comes back unchanged; the reconstruction is lorenzo_decode's."""
        x = np.ascontiguousarray(x).ravel()
        cap = 4096 + x.size * (x.itemsize + 8) + 2 * 65540
        out = np.empty(cap, np.uint8)
        after = np.empty_like(x)
        fn = getattr(self.lib, f"ref_lorenzo_payload_{_sfx(x.dtype)}")
        fn.restype = ctypes.c_longlong
        ct = _ctype(x.dtype)
        n = fn(_ptr(x, ct), ctypes.c_size_t(x.size), ctypes.c_double(eb), ctypes.c_int(quantbin),
               _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap), _ptr(after, ct))
        if n < 0:
            self._err("ref lorenzo payload")
        return out[:n].tobytes(), after

    def lorenzo_decode(self, payload: bytes, n: int, dtype) -> np.ndarray:
        buf = np.frombuffer(payload, np.uint8)
        out = np.empty(n, dtype)
        fn = getattr(self.lib, f"ref_lorenzo_decode_{_sfx(dtype)}")
        fn.restype = ctypes.c_longlong
        used = fn(_ptr(buf, ctypes.c_uint8), ctypes.c_size_t(len(payload)), ctypes.c_size_t(n),
                  _ptr(out, _ctype(dtype)))
        if used < 0:
            self._err("ref lorenzo decode")
        return out

    def lorenzo_trial(self, blocks: np.ndarray, eb: float, quantbin: int = 65536):
        """(buffer before zstd, ratio) of the tuner's Lorenzo trial over sample blocks (rows of
        `blocks`), as lorenzo_compress_test computes them."""
        blocks = np.ascontiguousarray(blocks)
        B, V = blocks.shape
        cap = 4096 + blocks.size * (blocks.itemsize + 8) + 2 * 65540
        out = np.empty(cap, np.uint8)
        n = ctypes.c_longlong(0)
        fn = getattr(self.lib, f"ref_lorenzo_trial_{_sfx(blocks.dtype)}")
        fn.restype = ctypes.c_double
        r = fn(_ptr(blocks, _ctype(blocks.dtype)), ctypes.c_size_t(B), ctypes.c_size_t(V), ctypes.c_double(eb),
               ctypes.c_int(quantbin), _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap), ctypes.byref(n))
        if r < 0:
            self._err("ref lorenzo trial")
        return out[:n.value].tobytes(), r

    def fse_compress(self, raw: bytes) -> bytes:
        """One zfse FSE_compress block: b"" when not compressible (0), b"\\x01" for a single symbol."""
        src = np.frombuffer(raw, np.uint8)
        out = np.empty(len(raw) + 1024, np.uint8)
        fn = self.lib.ref_fse_compress
        fn.restype = ctypes.c_longlong
        n = fn(_ptr(src, ctypes.c_uint8), ctypes.c_size_t(len(raw)), _ptr(out, ctypes.c_uint8),
               ctypes.c_size_t(out.size))
        if n < 0:
            self._err("ref fse compress")
        return b"" if n == 0 else (b"\x01" if n == 1 else out[:n].tobytes())

    def fse_decompress(self, block: bytes, n: int) -> bytes:
        src = np.frombuffer(block, np.uint8)
        out = np.empty(max(n, 1), np.uint8)
        fn = self.lib.ref_fse_decompress
        fn.restype = ctypes.c_longlong
        r = fn(_ptr(src, ctypes.c_uint8), ctypes.c_size_t(len(block)), _ptr(out, ctypes.c_uint8), ctypes.c_size_t(n))
        if r < 0:
            self._err("ref fse decompress")
        return out[:r].tobytes()

    def zstd_compress(self, raw: bytes) -> bytes:
        src = np.frombuffer(raw, np.uint8)
        cap = len(raw) + len(raw) // 128 + 1024
        out = np.empty(cap, np.uint8)
        n = self.lib.ref_zstd_compress(_ptr(src, ctypes.c_uint8), ctypes.c_size_t(len(raw)),
                                       _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap))
        if n < 0:
            self._err("ref zstd compress")
        return out[:n].tobytes()

    def zstd_decompress(self, payload: bytes, cap: int) -> bytes:
        src = np.frombuffer(payload, np.uint8)
        out = np.empty(max(cap, 1), np.uint8)
        n = self.lib.ref_zstd_decompress(_ptr(src, ctypes.c_uint8), ctypes.c_size_t(len(payload)),
                                         _ptr(out, ctypes.c_uint8), ctypes.c_size_t(cap))
        if n < 0:
            self._err("ref zstd decompress")
        return out[:n].tobytes()
