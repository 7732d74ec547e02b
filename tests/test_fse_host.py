"""The FSE block coder of falcons_b200/csrc/fse.cuh (the device code of the entropy kernels, compiled
for the host by tests/native/fse_host.cu), against the reference's zfse FSE_compress /
FSE_decompress (include/Falcons/encoder/zfse).

* Every block written here decodes with the reference's FSE_decompress; every block the reference
  writes decodes here (including its low-probability -1 counts).
* The normalization is the library's own (nearest shares, then single-cell moves by marginal coded
  size), so the bytes differ from FSE_compress's; the total size stays within 0.5 % of it.
* The NCount header round-trips, and the reader refuses truncated or malformed headers.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "fse_host.cu")
HDR = os.path.join(ROOT, "falcons_b200", "csrc", "fse.cuh")
OUT = os.path.join(ROOT, "tests", "native", "_build", "libfse_host.so")


@pytest.fixture(scope="module")
def fh():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.check_call([nvcc, "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "-x", "cu",
                               "-gencode", "arch=compute_100a,code=sm_100a", SRC, "-o", OUT])
    lib = ctypes.CDLL(OUT)
    for f in ("fseh_compress", "fseh_write_ncount", "fseh_read_ncount"):
        getattr(lib, f).restype = ctypes.c_longlong
    return lib


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def compress(fh, raw):
    src = np.frombuffer(raw, np.uint8)
    out = np.empty(len(raw) + 1024, np.uint8)
    n = fh.fseh_compress(_p(src, ctypes.c_uint8), ctypes.c_size_t(len(raw)), _p(out, ctypes.c_uint8),
                         ctypes.c_size_t(out.size))
    return b"" if n == 0 else (b"\x01" if n == 1 else out[:n].tobytes())


def decompress(fh, block, n):
    src = np.frombuffer(block, np.uint8)
    out = np.empty(max(n, 1), np.uint8)
    rc = fh.fseh_decompress(_p(src, ctypes.c_uint8), ctypes.c_size_t(len(block)), _p(out, ctypes.c_uint8),
                            ctypes.c_size_t(n))
    assert rc == 0
    return out[:n].tobytes()


def _blocks():
    """Class-stream-like blocks: geometric and two-sided laplacian alphabets, skewed ones with rare
    symbols (the low-probability case), near-uniform ones, few-symbol and tiny blocks."""
    rng = np.random.default_rng(7)
    out = []
    for i in range(400):
        n = int(rng.choice([3, 4, 17, 100, 700, 4096, 30000, 65536]))
        kind = i % 6
        if kind == 0:
            b = rng.geometric(rng.uniform(0.05, 0.9), n) - 1
        elif kind == 1:
            b = np.abs(rng.laplace(0, rng.uniform(0.3, 20), n)).astype(int)
        elif kind == 2:
            b = np.where(rng.random(n) < rng.uniform(0.9, 0.9999), rng.integers(0, 3, n), rng.integers(0, 256, n))
        elif kind == 3:
            b = rng.integers(0, int(rng.integers(2, 256)), n)
        elif kind == 4:
            b = rng.integers(0, 2, n) * int(rng.integers(1, 255))
        else:
            b = rng.zipf(rng.uniform(1.1, 3.0), n)
        out.append(np.clip(b, 0, 255).astype(np.uint8).tobytes())
    return out


def test_blocks_decode_both_ways_and_stay_within_size(fh, reference):
    ours_total = ref_total = 0
    for raw in _blocks():
        n = len(raw)
        ours = compress(fh, raw)
        ref = reference.fse_compress(raw)
        if ours == b"\x01":
            assert len(set(raw)) == 1
        elif ours:
            assert reference.fse_decompress(ours, n) == raw      # our header and stream, their decoder
            assert decompress(fh, ours, n) == raw
        if len(ref) > 1:
            assert decompress(fh, ref, n) == raw                  # their header and stream, our decoder
        size = lambda b: n if len(b) == 0 else len(b)            # a raw block costs its symbols
        ours_total += size(ours)
        ref_total += size(ref)
    assert ours_total <= 1.005 * ref_total, (ours_total, ref_total)


def test_normalization_fills_the_table_and_keeps_every_symbol(fh):
    rng = np.random.default_rng(3)
    for _ in range(300):
        m = int(rng.integers(1, 256))
        cnt = (rng.geometric(rng.uniform(0.01, 0.5), m) * (rng.random(m) < 0.8)).astype(np.uint32)
        cnt[int(rng.integers(0, m))] += 1
        if (cnt > 0).sum() < 2:
            cnt[(int(rng.integers(0, m)) + 1) % m] += 1
        if (cnt > 0).sum() < 2:
            continue
        tl = int(rng.integers(5, 14))
        norm = np.zeros(256, np.int16)
        r = fh.fseh_normalize(_p(cnt, ctypes.c_uint32), m - 1, ctypes.c_ulonglong(int(cnt.sum())), tl,
                              _p(norm, ctypes.c_int16))
        if (cnt > 0).sum() > (1 << tl):
            assert r == 0
            continue
        assert r == tl
        assert norm[:m].sum() == 1 << tl
        assert ((norm[:m] > 0) == (cnt > 0)).all()
        # no single cell moved from one symbol to another shortens the coded size by more than the
        # rounding of the integer saving proxy allows (about 0.2 % of it)
        c = cnt[cnt > 0].astype(np.float64)
        k = norm[:m][cnt > 0].astype(np.float64)
        gain = c * np.log2((k + 1) / k)                               # one more cell
        loss = np.where(k > 1, c * np.log2(k / np.maximum(k - 1, 1)), np.inf)  # one cell less
        cost = float((c * np.log2((1 << tl) / k)).sum())
        assert gain.max() - loss.min() <= 2e-3 * cost + 1e-9


def test_single_symbol_and_overfull_cases(fh):
    cnt = np.zeros(8, np.uint32)
    cnt[3] = 50
    norm = np.zeros(256, np.int16)
    assert fh.fseh_normalize(_p(cnt, ctypes.c_uint32), 7, ctypes.c_ulonglong(50), 6, _p(norm, ctypes.c_int16)) == 1
    assert compress(fh, bytes([9]) * 100) == b"\x01"
    assert compress(fh, b"\x01\x02") == b""


def test_ncount_round_trip_and_malformed_headers(fh):
    rng = np.random.default_rng(11)
    for _ in range(200):
        tl = int(rng.integers(5, 14))
        m = int(rng.integers(2, min(256, (1 << tl) // 2)))
        norm = np.zeros(256, np.int16)
        w = rng.dirichlet(np.full(m, 0.3)) * ((1 << tl) - m)
        norm[:m] = np.floor(w).astype(np.int16)
        norm[:m][rng.random(m) < 0.3] = 0
        norm[:m][rng.random(m) < 0.1] = -1                        # low-probability marks
        norm[m - 1] = 0
        rest = (1 << tl) - int(np.abs(norm[:m]).sum())
        if rest <= 0:
            continue
        norm[m - 1] = rest
        hdr = np.zeros(1024, np.uint8)
        size = fh.fseh_write_ncount(_p(norm, ctypes.c_int16), m - 1, tl, _p(hdr, ctypes.c_uint8))
        assert size > 0
        back = np.zeros(256, np.int16)
        mx, tl2 = ctypes.c_uint(255), ctypes.c_uint(0)
        got = fh.fseh_read_ncount(_p(hdr, ctypes.c_uint8), ctypes.c_size_t(size), _p(back, ctypes.c_int16),
                                  ctypes.byref(mx), ctypes.byref(tl2))
        assert got == size and tl2.value == tl and mx.value == m - 1
        np.testing.assert_array_equal(back[:m], norm[:m])
        # a header cut short, or read with a smaller alphabet than it codes, is refused
        if size > 1:
            assert fh.fseh_read_ncount(_p(hdr, ctypes.c_uint8), ctypes.c_size_t(size - 1), _p(back, ctypes.c_int16),
                                       ctypes.byref(ctypes.c_uint(255)), ctypes.byref(tl2)) == 0
        assert fh.fseh_read_ncount(_p(hdr, ctypes.c_uint8), ctypes.c_size_t(size), _p(back, ctypes.c_int16),
                                   ctypes.byref(ctypes.c_uint(m - 2)), ctypes.byref(tl2)) == 0
    # counts that do not fill the table, or below -1, are not written
    norm = np.zeros(256, np.int16)
    norm[:2] = (10, 11)
    assert fh.fseh_write_ncount(_p(norm, ctypes.c_int16), 1, 5, _p(np.zeros(64, np.uint8), ctypes.c_uint8)) == 0
    norm[:3] = (30, -2, 4)
    assert fh.fseh_write_ncount(_p(norm, ctypes.c_int16), 2, 5, _p(np.zeros(64, np.uint8), ctypes.c_uint8)) == 0


def test_table_log_choice(fh):
    assert fh.fseh_choose_table_log(65536, 40) == 11
    assert fh.fseh_choose_table_log(100, 3) == 5
    assert fh.fseh_choose_table_log(4096, 200) == 10
