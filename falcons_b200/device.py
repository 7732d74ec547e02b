"""Stage-level entry points on device-resident torch tensors (CUDA), through the C ABI.

These expose the individual stages of the path — value range, interpolation decomposition,
entropy coding — for tests, benchmarks and callers that keep fields in HBM.  PyTorch is used
only to own device memory and streams.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

_DT = {torch.float32: _lib.F32, torch.float64: _lib.F64}


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype not in _DT:
        raise TypeError("unsupported on GPU build: only float32 and float64 fields are supported")
    return _DT[t.dtype]


def _stream_ptr(stream) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def interp_params(eb, interp_algo=1, direction=0, anchor_stride=None, ndim=3, alpha=1.25, beta=2.0,
                  radius=32768, tuning=False, max_abs=-1.0) -> _lib.InterpParams:
    """falcons_interp_params.  max_abs: the field's largest |value| if known (compress measures it
    otherwise)."""
    if anchor_stride is None or anchor_stride < 0:
        anchor_stride = {1: 4096, 2: 128, 3: 32, 4: 16}[ndim]
    return _lib.InterpParams(float(eb), int(interp_algo), int(direction), int(anchor_stride), float(alpha),
                             float(beta), int(radius), int(tuning), float(max_abs))


def value_range(x: torch.Tensor, ctx=None, stream=None) -> float:
    ctx = ctx or _lib.default_context(x.device.index or 0)
    out = ctypes.c_double(0)
    _lib.check(_lib.lib().falcons_device_range(ctx.ptr, _dtype_code(x), ctypes.c_void_p(x.data_ptr()),
                                                ctypes.c_size_t(x.numel()), ctypes.byref(out),
                                                _stream_ptr(stream)), "device_range")
    return out.value


def interp_compress(x: torch.Tensor, params: _lib.InterpParams, ctx=None, stream=None):
    """Predict + quantize `x` in place (it ends as the reference's partial reconstruction).

    Returns (codes int16 [n_codes], unpred [anchors + escapes]) in stream order, on the device.
    """
    assert x.is_cuda and x.is_contiguous()
    ctx = ctx or _lib.default_context(x.device.index or 0)
    dims = (ctypes.c_size_t * x.dim())(*x.shape)
    codes = torch.empty(x.numel() + 16, dtype=torch.int16, device=x.device)
    unpred = torch.empty(x.numel() + 16, dtype=x.dtype, device=x.device)
    nq, nu = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _lib.check(_lib.lib().falcons_interp_compress(ctx.ptr, _dtype_code(x), dims, x.dim(), ctypes.byref(params),
                                                  ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(codes.data_ptr()),
                                                  ctypes.c_void_p(unpred.data_ptr()), ctypes.byref(nq),
                                                  ctypes.byref(nu), _stream_ptr(stream)), "interp_compress")
    return codes[:nq.value], unpred[:nu.value]


def time_levels(on: bool = True, ctx=None, device: int = 0):
    """Turns per-launch device timing of interp_compress on this context on or off (measurement)."""
    ctx = ctx or _lib.default_context(device)
    _lib.check(_lib.lib().falcons_time_levels(ctx.ptr, int(bool(on))), "time_levels")


def level_times(ctx=None, device: int = 0):
    """The last timed interp_compress call's launches: [(level, ms, codes of that level)], levels in
    coding order (the coarsest first, the unit-step level last)."""
    ctx = ctx or _lib.default_context(device)
    cap = 256
    lv = (ctypes.c_int * cap)()
    ms = (ctypes.c_float * cap)()
    cd = (ctypes.c_ulonglong * cap)()
    n = ctypes.c_int(0)
    _lib.check(_lib.lib().falcons_level_times(ctx.ptr, lv, ms, cd, cap, ctypes.byref(n)), "level_times")
    return [(int(lv[i]), float(ms[i]), int(cd[i])) for i in range(min(n.value, cap))]


def interp_decompress(shape, dtype, codes: torch.Tensor, unpred: torch.Tensor, params: _lib.InterpParams,
                      out: torch.Tensor | None = None, ctx=None, stream=None) -> torch.Tensor:
    dev = codes.device
    ctx = ctx or _lib.default_context(dev.index or 0)
    if out is None:
        out = torch.empty(tuple(shape), dtype=dtype, device=dev)
    dims = (ctypes.c_size_t * len(shape))(*shape)
    codes = codes.contiguous()
    unpred = unpred.contiguous()
    _lib.check(_lib.lib().falcons_interp_decompress(ctx.ptr, _dtype_code(out), dims, len(shape),
                                                    ctypes.byref(params), ctypes.c_void_p(codes.data_ptr()),
                                                    ctypes.c_size_t(codes.numel()),
                                                    ctypes.c_void_p(unpred.data_ptr()),
                                                    ctypes.c_size_t(unpred.numel()), ctypes.c_void_p(out.data_ptr()),
                                                    _stream_ptr(stream)), "interp_decompress")
    return out


def encode_codes(codes: torch.Tensor, ctx=None, stream=None) -> torch.Tensor:
    """RleFseEncoder-format entropy coding of int16 codes on the device; returns a uint8 tensor."""
    assert codes.dtype == torch.int16 and codes.is_cuda
    ctx = ctx or _lib.default_context(codes.device.index or 0)
    codes = codes.contiguous()
    cap = 4 * codes.numel() + (1 << 20)
    out = torch.empty(cap, dtype=torch.uint8, device=codes.device)
    n = ctypes.c_size_t(0)
    _lib.check(_lib.lib().falcons_encode_codes(ctx.ptr, ctypes.c_void_p(codes.data_ptr()),
                                               ctypes.c_size_t(codes.numel()), ctypes.c_void_p(out.data_ptr()),
                                               ctypes.c_size_t(cap), ctypes.byref(n), _stream_ptr(stream)),
               "encode_codes")
    return out[:n.value]


def decode_codes(payload: torch.Tensor, n: int, ctx=None, stream=None) -> torch.Tensor:
    assert payload.dtype == torch.uint8 and payload.is_cuda
    ctx = ctx or _lib.default_context(payload.device.index or 0)
    payload = payload.contiguous()
    out = torch.empty(max(n, 1), dtype=torch.int16, device=payload.device)
    _lib.check(_lib.lib().falcons_decode_codes(ctx.ptr, ctypes.c_void_p(payload.data_ptr()),
                                               ctypes.c_size_t(payload.numel()), ctypes.c_size_t(n),
                                               ctypes.c_void_p(out.data_ptr()), _stream_ptr(stream)), "decode_codes")
    return out[:n]


def compress(x: torch.Tensor, config, out: torch.Tensor | None = None, ctx=None, stream=None):
    """Falcons_compress on a device-resident field; returns (uint8 stream tensor on the device, config).

    `x` is overwritten with the reference's partial reconstruction (the in-place compressor).
    `config` is a falcons_b200.api.falconsConfig.
    """
    assert x.is_cuda and x.is_contiguous()
    ctx = ctx or _lib.default_context(x.device.index or 0)
    if config.num_elements != x.numel():
        config.setDims(*x.shape)
    cap = int(_lib.lib().falcons_compress_size_bound(_dtype_code(x), ctypes.byref(config.conf)))
    if out is None or out.numel() < cap:
        out = torch.empty(cap, dtype=torch.uint8, device=x.device)
    n = ctypes.c_size_t(0)
    conf_out = _lib.Config()
    _lib.check(_lib.lib().falcons_compress_device(ctx.ptr, _dtype_code(x), ctypes.byref(config.conf),
                                                  ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                  ctypes.c_size_t(out.numel()), ctypes.byref(n),
                                                  ctypes.byref(conf_out), _stream_ptr(stream)), "compress_device")
    return out[:n.value], conf_out


def decompress(stream_bytes: torch.Tensor, dtype, out: torch.Tensor | None = None, ctx=None, stream=None):
    """Falcons_decompress of a device-resident stream into a device tensor (flat)."""
    assert stream_bytes.is_cuda and stream_bytes.dtype == torch.uint8
    ctx = ctx or _lib.default_context(stream_bytes.device.index or 0)
    if out is None:
        # the field's size from the header (at most 255 bytes, inside the first 256 of the stream):
        # a small device-to-host read, made only when the caller gives no output tensor
        head = stream_bytes[:256].cpu().numpy()
        c = _lib.Config()
        buf = bytearray(head.tobytes())
        _lib.check(_lib.lib().falcons_read_config((ctypes.c_char * len(buf)).from_buffer(buf),
                                                  ctypes.c_size_t(len(buf)), ctypes.byref(c)), "read_config")
        out = torch.empty(int(c.num), dtype=dtype, device=stream_bytes.device)
    conf_out = _lib.Config()
    _lib.check(_lib.lib().falcons_decompress_device(ctx.ptr, _dtype_code(out), ctypes.c_void_p(stream_bytes.data_ptr()),
                                                    ctypes.c_size_t(stream_bytes.numel()),
                                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_size_t(out.numel()),
                                                    ctypes.byref(conf_out), _stream_ptr(stream)), "decompress_device")
    return out, conf_out


def _batch_items(n):
    return (_lib.BatchItem * n)()


def compress_batch(fields, configs, outs=None, workers: int = 0, ctx=None):
    """Falcons_compress of many device-resident fields in one call (falcons_compress_batch).

    `fields` are contiguous CUDA tensors (float32 / float64), each overwritten with its partial
    reconstruction; `configs` are falcons_b200.api.falconsConfig.  Returns a list of (uint8 stream
    tensor on the device, stored config).  workers <= 0: the context's autotuned worker count."""
    n = len(fields)
    if n == 0:
        return []
    dev = fields[0].device
    ctx = ctx or _lib.default_context(dev.index or 0)
    items = _batch_items(n)
    bufs = []
    for i, (x, c) in enumerate(zip(fields, configs)):
        assert x.is_cuda and x.is_contiguous()
        if c.num_elements != x.numel():
            c.setDims(*x.shape)
        cap = int(_lib.lib().falcons_compress_size_bound(_dtype_code(x), ctypes.byref(c.conf)))
        out = outs[i] if outs is not None and outs[i] is not None and outs[i].numel() >= cap else \
            torch.empty(cap, dtype=torch.uint8, device=dev)
        bufs.append(out)
        it = items[i]
        it.dtype = _dtype_code(x)
        it.conf = c.conf
        it.d_data = x.data_ptr()
        it.d_stream = out.data_ptr()
        it.cap = out.numel()
    _lib.check(_lib.lib().falcons_compress_batch(ctx.ptr, items, ctypes.c_size_t(n), int(workers)), "compress_batch")
    return [(bufs[i][:items[i].len], items[i].conf) for i in range(n)]


def decompress_batch(streams, dtypes, outs, workers: int = 0, ctx=None):
    """Falcons_decompress of many device-resident streams in one call (falcons_decompress_batch)
    into the flat device tensors `outs` (one per stream, of the streams' field sizes)."""
    n = len(streams)
    if n == 0:
        return []
    ctx = ctx or _lib.default_context(streams[0].device.index or 0)
    items = _batch_items(n)
    for i, (s, out) in enumerate(zip(streams, outs)):
        assert s.is_cuda and s.dtype == torch.uint8 and out.is_cuda and out.is_contiguous()
        it = items[i]
        it.dtype = _dtype_code(out)
        it.d_data = out.data_ptr()
        it.d_stream = s.data_ptr()
        it.cap = out.numel()
        it.len = s.numel()
    _lib.check(_lib.lib().falcons_decompress_batch(ctx.ptr, items, ctypes.c_size_t(n), int(workers)),
               "decompress_batch")
    return [items[i].conf for i in range(n)]
