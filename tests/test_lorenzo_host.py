"""The device code of the 1-D Lorenzo + Huffman decoder (falcons_b200/csrc/lorenzo.cuh: payload
parse, canonical Huffman tables and decode, the sequential reconstruction), compiled for the host
from the same source (tests/native/lorenzo_host.cu) and checked bit for bit against the
reference's decoder and the golden vectors.  The GPU runs these functions in single-thread CTAs
(k_lz_huff_decode, k_lz_reconstruct); tests/test_zzz_lorenzo_gpu.py checks the device build."""
import ctypes
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from test_lorenzo_oracle import CASES, same_bits, series

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "lorenzo_host.cu")
HDR = os.path.join(ROOT, "falcons_b200", "csrc", "lorenzo.cuh")
OUT = os.path.join(ROOT, "tests", "native", "_build", "liblz_host.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def host_decoder():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.check_call([nvcc, "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "-x", "cu",
                               "-gencode", "arch=compute_100a,code=sm_100a", SRC, "-o", OUT])
    lib = ctypes.CDLL(OUT)

    def decode(payload, n, dtype, block=5, l1=1, l2=1):
        buf = np.frombuffer(payload, np.uint8)
        out = np.empty(n, dtype)
        ct = ctypes.c_float if dtype == np.float32 else ctypes.c_double
        fn = lib.lzh_decode_f32 if dtype == np.float32 else lib.lzh_decode_f64
        rc = fn(buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.c_size_t(len(payload)),
                ctypes.c_size_t(n), block, l1, l2, out.ctypes.data_as(ctypes.POINTER(ct)))
        return rc, out

    def encode(x, eb, radius=32768, block=5, l1=1, l2=1):
        x = np.ascontiguousarray(x)
        cap = 4096 + x.size * (x.itemsize + 8) + 2 * 65540
        out = np.empty(cap, np.uint8)
        ct = ctypes.c_float if x.dtype == np.float32 else ctypes.c_double
        fn = lib.lzh_encode_f32 if x.dtype == np.float32 else lib.lzh_encode_f64
        fn.restype = ctypes.c_longlong
        n = fn(x.ctypes.data_as(ctypes.POINTER(ct)), ctypes.c_size_t(x.size), ctypes.c_double(eb), radius, block,
               l1, l2, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.c_size_t(cap))
        assert n >= 0, n
        return out[:n].tobytes()

    def trial(blocks, eb, radius=32768):
        blocks = np.ascontiguousarray(blocks)
        B, V = blocks.shape
        cap = 4096 + blocks.size * (blocks.itemsize + 8) + 2 * 65540
        out = np.empty(cap, np.uint8)
        ct = ctypes.c_float if blocks.dtype == np.float32 else ctypes.c_double
        fn = lib.lzh_trial_f32 if blocks.dtype == np.float32 else lib.lzh_trial_f64
        fn.restype = ctypes.c_longlong
        n = fn(blocks.ctypes.data_as(ctypes.POINTER(ct)), ctypes.c_size_t(B), ctypes.c_size_t(V),
               ctypes.c_double(eb), radius, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.c_size_t(cap))
        assert n >= 0, n
        return out[:n].tobytes()

    decode.encode = encode
    decode.trial = trial
    return decode


@pytest.mark.parametrize("kind,n,dtype,eb,quantbin", CASES,
                         ids=[f"{c[0]}-{c[1]}-{np.dtype(c[2]).name}-{c[3]:g}-{c[4]}" for c in CASES])
def test_decoder_matches_reference(host_decoder, reference, kind, n, dtype, eb, quantbin):
    x = series(kind, n, dtype, seed=n)
    payload, _ = reference.lorenzo_payload(x, eb, quantbin)
    rc, y = host_decoder(payload, n, dtype)
    assert rc == 0
    assert same_bits(y, reference.lorenzo_decode(payload, n, dtype))


@pytest.mark.parametrize("kind,n,dtype,eb,quantbin", CASES,
                         ids=[f"{c[0]}-{c[1]}-{np.dtype(c[2]).name}-{c[3]:g}-{c[4]}" for c in CASES])
def test_encoder_matches_reference(host_decoder, reference, kind, n, dtype, eb, quantbin):
    """The encoder functions (blockwise quantization, Huffman lengths in the reference's heap
    order, canonical codes, the table flag, packing) give the reference's payload bytes."""
    x = series(kind, n, dtype, seed=n)
    payload, _ = reference.lorenzo_payload(x, eb, quantbin)
    assert host_decoder.encode(x, eb, quantbin // 2) == payload


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "lorenzo_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_encoder_matches_golden(host_decoder, path):
    g = np.load(path)
    assert host_decoder.encode(g["x"], float(g["eb"]), int(g["radius"]), int(g["block"])) == g["payload"].tobytes()


@pytest.mark.parametrize("l1,l2", [(1, 0), (0, 1)])
def test_single_predictor_encoder(host_decoder, reference, l1, l2):
    x = series("sine", 20000, np.float32, 11)
    conf = oracle.lorenzo_ref_conf(1e-3)
    conf.lorenzo, conf.lorenzo2 = l1, l2
    stream = reference.compress(x, conf)
    h = oracle.lossless_section(stream)
    payload = reference.zstd_decompress(stream[h:], int.from_bytes(stream[h:h + 8], "little"))
    assert host_decoder.encode(x, 1e-3, 32768, 5, l1, l2) == payload


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "lorenzo_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_decoder_matches_golden(host_decoder, path):
    g = np.load(path)
    rc, y = host_decoder(g["payload"].tobytes(), g["x"].size, g["x"].dtype, int(g["block"]))
    assert rc == 0
    assert same_bits(y, g["recon"])


@pytest.mark.parametrize("l1,l2", [(1, 0), (0, 1)])
def test_single_predictor_streams(host_decoder, reference, l1, l2):
    """A stream of one Lorenzo predictor alone (no ComposedPredictor, so no selection record:
    FalconsAlgoLorenzoReg.hpp:29-43, LorenzoPredictor.hpp:44-48 saves nothing)."""
    x = series("sine", 20000, np.float32, 11)
    conf = oracle.lorenzo_ref_conf(1e-3)
    conf.lorenzo, conf.lorenzo2 = l1, l2
    stream = reference.compress(x, conf)
    h = oracle.lossless_section(stream)
    payload = reference.zstd_decompress(stream[h:], int.from_bytes(stream[h:h + 8], "little"))
    rc, y = host_decoder(payload, x.size, np.float32, 5, l1, l2)
    assert rc == 0
    assert same_bits(y, reference.decompress(stream, np.float32, x.size).ravel())


def test_damaged_payloads_are_rejected(host_decoder, restatement):
    x = series("sine", 3000, np.float64, 4)
    payload, recon = restatement.lorenzo_payload(x, 1e-4)
    rc, y = host_decoder(payload, x.size, np.float64)
    assert rc == 0 and same_bits(y, recon)
    for cut in (1, 9, 40, len(payload) // 2, len(payload) - 1):
        rc, _ = host_decoder(payload[:cut], x.size, np.float64)
        assert rc != 0
    assert host_decoder(payload, x.size + 5, np.float64)[0] != 0
    bad = bytearray(payload)
    bad[12] = 0xFF  # the selection record's state count (big-endian, most significant byte)
    assert host_decoder(bytes(bad), x.size, np.float64)[0] != 0


@pytest.mark.parametrize("kind,B,V,dtype,eb,quantbin", [
    ("walk", 12, 513, np.float32, 1e-2, 65536), ("sine", 7, 1025, np.float64, 1e-6, 65536),
    ("noise", 5, 257, np.float32, 1e-4, 65536), ("spikes", 9, 129, np.float64, 1e-3, 65536),
    ("walk", 4, 4097, np.float32, 1e-3, 16384)])
def test_tuner_trial_layout_and_ratio(host_decoder, reference, kind, B, V, dtype, eb, quantbin):
    """The tuner's Lorenzo trial (lorenzo_compress_test): the buffer laid out as lorenzo.cu's
    lorenzo_trial_ratio writes it is the reference's byte for byte (its quantizer header comes
    before the code count, unlike the stream), and the reference's ratio is the input bytes over
    the zstd size of that buffer plus its length word."""
    blocks = np.stack([series(kind, V, dtype, seed=b) for b in range(B)])
    ref_buf, ref_ratio = reference.lorenzo_trial(blocks, eb, quantbin)
    assert host_decoder.trial(blocks, eb, quantbin // 2) == ref_buf
    zs = len(reference.zstd_compress(ref_buf))
    assert ref_ratio == pytest.approx(blocks.nbytes / zs, rel=0, abs=0)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "tunedlz_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_encoder_matches_tuned_streams(host_decoder, path):
    """The encoder functions at the tuner's final Config (block size 128, the chosen bins) give the
    payload of the reference's own tuned stream."""
    from test_lorenzo_oracle import tuned_fixture
    x, eb, c, payload = tuned_fixture(path)
    assert host_decoder.encode(x, eb, c.quantbinCnt // 2, 128) == payload
    rc, y = host_decoder(payload, x.size, x.dtype, 128)
    assert rc == 0
