"""The C restatement of the 1-D blockwise Lorenzo + Huffman path (oracle/lorenzo_oracle.c), pinned
against the reference build and against the golden vectors written from it.

The path is the one the interpolation tuner switches 1-D fields to (ALGO_LORENZO_REG with Lorenzo
orders 1 and 2, block size 5: api/impl/FalconsAlgoInterp.hpp:479-490, 497-498).  The oracle
produces the payload that the reference hands to its trailing zstd stage
(compressor/FalconsGenericCompressor.hpp:64-81); the tests take the reference's payload out of its
stream (the Lossless_zstd section after the Config header) and require the same bytes, the same
reconstruction, and that each decoder reads the other's payload.
"""
import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def series(kind, n, dtype, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64)
    if kind == "walk":
        x = np.cumsum(rng.normal(size=n))
    elif kind == "sine":
        x = 10 * np.sin(0.01 * t) + 1e-3 * rng.normal(size=n)
    elif kind == "noise":
        x = 100 * rng.normal(size=n)
    elif kind == "const":
        x = np.zeros(n)
    elif kind == "spikes":
        x = np.sin(0.05 * t)
        x[rng.random(n) < 0.02] = 1e20
    elif kind == "nonfinite":
        x = np.sin(0.05 * t)
        x[n // 3] = np.nan
        x[n // 2] = np.inf
        x[(2 * n) // 3] = -np.inf
    else:
        raise ValueError(kind)
    return x.astype(dtype)


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    u = np.uint32 if a.dtype == np.float32 else np.uint64
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(u), b.view(u))


def reference_payload(reference, stream):
    h = oracle.lossless_section(stream)
    raw = int.from_bytes(stream[h:h + 8], "little")
    return reference.zstd_decompress(stream[h:], raw)


CASES = (
    [("walk", n, np.float32, 1e-2, 65536) for n in (1, 2, 3, 4, 5, 6, 7, 10, 11, 1000, 4099, 65537)]
    + [("walk", 5003, np.float64, 1e-3, 65536), ("sine", 20000, np.float32, 1e-4, 65536),
       ("sine", 7777, np.float64, 1e-6, 65536), ("noise", 3000, np.float32, 1e-6, 65536),
       ("noise", 3000, np.float32, 10.0, 65536), ("const", 1, np.float32, 1e-3, 65536),
       ("const", 23, np.float64, 1e-3, 65536), ("spikes", 2500, np.float32, 1e-3, 65536),
       ("spikes", 2500, np.float64, 1e-3, 65536), ("nonfinite", 301, np.float32, 1e-3, 65536),
       ("walk", 9001, np.float32, 1e-3, 16384), ("noise", 4000, np.float64, 1e-2, 16384)]
)


@pytest.mark.parametrize("kind,n,dtype,eb,quantbin", CASES,
                         ids=[f"{c[0]}-{c[1]}-{np.dtype(c[2]).name}-{c[3]:g}-{c[4]}" for c in CASES])
def test_payload_and_reconstruction_match_reference(restatement, reference, kind, n, dtype, eb, quantbin):
    x = series(kind, n, dtype, seed=n)
    ref_payload, after = reference.lorenzo_payload(x, eb, quantbin)
    assert same_bits(after, x)  # this path leaves the caller's buffer as it was
    payload, recon = restatement.lorenzo_payload(x, eb, radius=quantbin // 2)
    assert payload == ref_payload
    ref_recon = reference.lorenzo_decode(ref_payload, n, dtype)
    assert same_bits(recon, ref_recon)
    # the oracle's decoder reads the reference's payload
    assert same_bits(restatement.lorenzo_decode(ref_payload, n, dtype), ref_recon)
    finite = np.isfinite(x)
    assert np.all(np.abs(recon[finite].astype(np.float64) - x[finite]) <= eb)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_stream_carries_the_payload(restatement, reference, dtype):
    """A whole reference stream of the path (a smooth series the dispatcher keeps lossy): its
    zstd section holds exactly the oracle's payload, and the reference decodes it to the
    oracle's reconstruction."""
    x = series("sine", 50000, dtype, seed=5)
    eb = 1e-3
    stream = reference.compress(x, oracle.lorenzo_ref_conf(eb))
    payload, recon = restatement.lorenzo_payload(x, eb)
    assert reference_payload(reference, stream) == payload
    assert same_bits(reference.decompress(stream, dtype, x.size).ravel(), recon)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "lorenzo_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_restatement_matches_golden(restatement, path):
    g = np.load(path)
    x, eb, radius = g["x"], float(g["eb"]), int(g["radius"])
    payload, recon = restatement.lorenzo_payload(x, eb, radius=radius)
    assert payload == g["payload"].tobytes()
    assert same_bits(recon, g["recon"])
    assert same_bits(restatement.lorenzo_decode(g["payload"].tobytes(), x.size, x.dtype), g["recon"])
    if path.endswith("_stream.npz"):
        # the whole reference stream: its zstd section (after the Config header) is the payload
        import pyarrow as pa
        s = g["stream"].tobytes()
        h = oracle.lossless_section(s)
        raw = int.from_bytes(s[h:h + 8], "little")
        assert pa.decompress(s[h + 8:], raw, codec="zstd", asbytes=True) == g["payload"].tobytes()


def test_golden_lorenzo_fixtures_present():
    assert len(glob.glob(os.path.join(GOLDEN, "lorenzo_*.npz"))) >= 4


@pytest.mark.parametrize("case", ["one", "two", "skewed", "wide", "uniform", "codes"])
def test_huffman_round_trip(restatement, case):
    rng = np.random.default_rng(len(case))
    if case == "one":
        sym = np.full(1000, 4242)
    elif case == "two":
        sym = rng.integers(0, 2, 5000)
    elif case == "skewed":
        sym = np.minimum(rng.geometric(0.3, 100000), 200) + 30000
    elif case == "wide":
        sym = rng.integers(0, 65536, 70000)
    elif case == "uniform":
        sym = rng.integers(100, 116, 4096)
    else:
        sym = np.clip(np.round(rng.laplace(32768, 3, 200000)), 0, 65535)
    sym = sym.astype(np.int32)
    rec = restatement.huffman_encode(sym)
    assert np.array_equal(restatement.huffman_decode(rec, sym.size), sym)
    if case == "one":  # one symbol: no code bits at all (HuffmanEncoder.hpp:1071-1082, 615-645)
        assert int.from_bytes(rec[-8:], "little") == 0


def test_decoder_rejects_damaged_payloads(restatement):
    x = series("walk", 500, np.float32, 3)
    payload, _ = restatement.lorenzo_payload(x, 1e-2)
    with pytest.raises(ValueError):
        restatement.lorenzo_decode(payload[:-3], x.size, np.float32)
    with pytest.raises(ValueError):
        restatement.lorenzo_decode(payload, x.size + 7, np.float32)
    bad = bytearray(payload)
    bad[8 + 4] ^= 0xFF  # the selection record's state count
    with pytest.raises(ValueError):
        restatement.lorenzo_decode(bytes(bad), x.size, np.float32)


TUNED = sorted(glob.glob(os.path.join(GOLDEN, "tunedlz_*.npz")))


def tuned_fixture(path):
    """(input, eb, the reference stream's Config, its payload) of a tuner-choice fixture."""
    import pyarrow as pa
    from falcons_b200 import api
    g = np.load(path)
    s = g["stream"].tobytes()
    h = oracle.lossless_section(s)
    payload = pa.decompress(s[h + 8:], int.from_bytes(s[h:h + 8], "little"), codec="zstd", asbytes=True)
    return g["x"], float(g["eb"]), api.read_config(g["stream"]), payload


@pytest.mark.parametrize("path", TUNED, ids=lambda p: os.path.basename(p))
def test_tuned_lorenzo_streams_match_oracle(restatement, path):
    """1-D fields on which the reference's ALGO_INTERP_LORENZO tuner switches to the Lorenzo path
    (FalconsAlgoInterp.hpp:479-537): the stream's Config carries the Lorenzo orders 1 and 2, the
    chosen bins and block size 128 (Config::setDims, utils/Config.hpp:165-181, undoes the trial's
    5), and its payload is the oracle's for that Config."""
    x, eb, c, payload = tuned_fixture(path)
    assert c.cmprAlgo == 0 and c.blockSize == 128 and c.lorenzo and c.lorenzo2 and not c.regression
    ours, recon = restatement.lorenzo_payload(x, eb, radius=c.quantbinCnt // 2, block=128)
    assert ours == payload
    assert same_bits(restatement.lorenzo_decode(payload, x.size, x.dtype, block=128), recon)


def test_tuned_fixtures_cover_both_bin_counts():
    bins = {tuned_fixture(p)[2].quantbinCnt for p in TUNED}
    assert bins == {65536, 16384}
