"""GPU tests of falcons_interp_decompress_noalloc, the allocation-free decompress entry point.

It must reconstruct exactly what falcons_interp_decompress reconstructs, call after call, allocate
no device memory after its first (set-up) call on a device, and reject fields whose scratch does
not fit its static region.  The file is named to be collected last, so that in a full run the
entry point is exercised after every other test in the same process; it also passes alone.
"""
import ctypes

import numpy as np
import pytest
import torch

from falcons_b200 import _lib
from falcons_b200 import device as D
from falcons_b200.synth import sinusoid_field

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 64 << 20  # FALCONS_NOALLOC_SCRATCH_BYTES


def _noalloc(shape, codes, unpred, params, out, stream=None):
    """One call through the C ABI; returns the status code."""
    dims = (ctypes.c_size_t * len(shape))(*shape)
    s = stream if stream is not None else torch.cuda.current_stream()
    return _lib.lib().falcons_interp_decompress_noalloc(
        D._dtype_code(out), dims, len(shape), ctypes.byref(params), ctypes.c_void_p(codes.data_ptr()),
        ctypes.c_size_t(codes.numel()), ctypes.c_void_p(unpred.data_ptr()), ctypes.c_size_t(unpred.numel()),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream))


def _case(shape, dtype, algo, seed):
    """Compress a field with the context entry point; return (params, codes, unpred, reference recon)."""
    x = sinusoid_field(shape, seed=seed, noise=1e-3, dtype=np.float64)
    x[np.random.default_rng(seed).random(shape) < 0.01] += 40.0  # escapes into the unpredictable list
    x = x.astype(dtype)
    eb = 1e-3 * float(x.max() - x.min())
    p = D.interp_params(eb, algo, 0, None, len(shape))
    xd = torch.from_numpy(x).cuda()
    codes, unpred = D.interp_compress(xd, p)
    ref = D.interp_decompress(shape, xd.dtype, codes, unpred, p)
    torch.cuda.synchronize()
    assert unpred.numel() > 0
    return p, codes, unpred, ref


def _same_bits(a, b):
    it = torch.int32 if a.dtype == torch.float32 else torch.int64
    return torch.equal(a.view(it), b.view(it))


def test_matches_context_entry_point_on_consecutive_calls():
    cases = [((64, 80, 96), np.float32, 1, 11), ((300, 500), np.float64, 0, 12), ((20, 30, 40, 8), np.float32, 1, 13)]
    prepared = [_case(*c) for c in cases]
    outs = [torch.full(tuple(c[0]), float("nan"), dtype=ref.dtype, device="cuda") for c, (_, _, _, ref) in
            zip(cases, prepared)]
    launches0 = _lib.lib().falcons_kernel_launches()
    # first call on this device (set-up, unless an earlier test already made it), then two in a row
    for (shape, *_), (p, codes, unpred, ref), out in zip(cases, prepared, outs):
        _lib.check(_noalloc(shape, codes, unpred, p, out), "interp_decompress_noalloc")
        torch.cuda.synchronize()
        assert _same_bits(out, ref), shape
    assert _lib.lib().falcons_kernel_launches() > launches0

    # Later calls allocate no device memory; repeated calls into stale scratch stay exact.
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        for (shape, *_), (p, codes, unpred, ref), out in zip(cases, prepared, outs):
            out.fill_(float("nan"))
            _lib.check(_noalloc(shape, codes, unpred, p, out), "interp_decompress_noalloc")
            torch.cuda.synchronize()
            assert _same_bits(out, ref), shape
    assert torch.cuda.mem_get_info()[0] == free0


def test_runs_on_a_caller_stream():
    shape = (48, 50, 52)
    p, codes, unpred, ref = _case(shape, np.float32, 1, 21)
    out = torch.empty_like(ref)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        _lib.check(_noalloc(shape, codes, unpred, p, out, stream=s), "interp_decompress_noalloc")
    s.synchronize()
    assert _same_bits(out, ref)


def test_rejects_fields_beyond_the_static_scratch():
    shape = (256, 256, 260)  # about 17 million float codes: more than the 64 MiB region holds
    p, codes, unpred, _ = _case(shape, np.float32, 1, 31)
    assert 4 * codes.numel() > SCRATCH_BYTES
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    launches0 = _lib.lib().falcons_kernel_launches()
    rc = _noalloc(shape, codes, unpred, p, out)
    assert rc == _lib.EINVAL
    msg = _lib.lib().falcons_last_error().decode()
    assert "FALCONS_NOALLOC_SCRATCH_BYTES" in msg and "bytes of scratch" in msg
    assert _lib.lib().falcons_kernel_launches() == launches0


def test_rejects_inconsistent_arguments():
    shape = (33, 34, 35)
    p, codes, unpred, ref = _case(shape, np.float32, 0, 41)
    out = torch.empty_like(ref)
    assert _noalloc(shape, codes[:-1], unpred, p, out) == _lib.EINVAL
    assert "code count" in _lib.lib().falcons_last_error().decode()
    bad = _lib.InterpParams(p.eb, p.interp_algo, p.direction, p.anchor_stride, p.alpha, p.beta, p.radius, p.tuning,
                            p.max_abs)
    dims = (ctypes.c_size_t * 3)(*shape)
    rc = _lib.lib().falcons_interp_decompress_noalloc(7, dims, 3, ctypes.byref(bad), ctypes.c_void_p(codes.data_ptr()),
                                                      ctypes.c_size_t(codes.numel()),
                                                      ctypes.c_void_p(unpred.data_ptr()),
                                                      ctypes.c_size_t(unpred.numel()),
                                                      ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(0))
    assert rc == _lib.EINVAL


def test_rejects_codes_with_more_escapes_than_the_list():
    """A code array naming one escape more than the unpredictable list holds (a mismatched buffer or
    a damaged stream) is refused with FALCONS_EINVAL; the escape beyond the list is not read."""
    shape = (40, 41, 42)
    p, codes, unpred, ref = _case(shape, np.float32, 1, 51)
    bad = codes.clone()
    h = bad.cpu().numpy()
    pos = int(np.flatnonzero(h != -p.radius)[len(h) // 2])
    bad[pos] = -p.radius
    out = torch.empty_like(ref)
    assert _noalloc(shape, bad, unpred, p, out) == _lib.EINVAL
    assert "unpredictable values" in _lib.lib().falcons_last_error().decode()
    # the entry point is still usable and exact after the refusal
    _lib.check(_noalloc(shape, codes, unpred, p, out), "interp_decompress_noalloc")
    torch.cuda.synchronize()
    assert _same_bits(out, ref)
