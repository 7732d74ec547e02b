"""Reference streams of the 1-D blockwise Lorenzo + Huffman path (ALGO_LORENZO_REG, which the
reference's interpolation tuner writes for 1-D fields, FalconsAlgoInterp.hpp:479-537) decoded on
the GPU through the public API, bit for bit against the reference's own decode of the same stream
(golden vectors written by tests/golden/make_golden.py from the reference build).  The decoder's
logic is also checked on the host from the same source (tests/test_lorenzo_host.py)."""
import glob
import os

import numpy as np
import pytest

from test_lorenzo_oracle import same_bits

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "lorenzo_*.npz")))


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_reference_lorenzo_streams_decode_on_gpu(cuda, path):
    import torch
    from falcons_b200 import api
    from falcons_b200 import device as D
    g = np.load(path)
    x, stream = g["x"], g["stream"]
    y, _ = api.falcons.decompress(stream, x.dtype, x.shape)
    assert same_bits(np.asarray(y).ravel(), g["stream_recon"])
    tdt = torch.float32 if x.dtype == np.float32 else torch.float64
    yd, _ = D.decompress(torch.from_numpy(stream.copy()).to(cuda), tdt)
    torch.cuda.synchronize()
    assert same_bits(yd.cpu().numpy().ravel(), g["stream_recon"])


@pytest.mark.gpu
def test_damaged_lorenzo_stream_is_rejected(cuda):
    import oracle
    from falcons_b200 import api
    g = np.load(os.path.join(GOLDEN, "lorenzo_walk_f32.npz"))
    assert api.read_config(g["stream"]).cmprAlgo == 0  # ALGO_LORENZO_REG
    s = g["stream"].tobytes()
    with pytest.raises(ValueError):  # the zstd section cut short
        api.falcons.decompress(np.frombuffer(s[:-7], np.uint8).copy(), np.float32, g["x"].shape)
    # a payload whose code count disagrees with the field: rebuilt with the same zstd section
    # layout ([u64 raw length][frame]) around a damaged payload
    h = oracle.lossless_section(s)
    import pyarrow as pa
    raw = bytearray(pa.decompress(s[h + 8:], int.from_bytes(s[h:h + 8], "little"), codec="zstd", asbytes=True))
    bad = bytearray(raw)
    bad[8 + 4] = 0xFF  # the selection record's state count
    frame = pa.compress(bytes(bad), codec="zstd", asbytes=True)
    damaged = s[:h] + len(bad).to_bytes(8, "little") + frame
    with pytest.raises(ValueError):
        api.falcons.decompress(np.frombuffer(damaged, np.uint8).copy(), np.float32, g["x"].shape)


def lorenzo_config(api, n, eb, l1=1, l2=1):
    """The Config of the 1-D Lorenzo path as the reference's tuner sets it
    (FalconsAlgoInterp.hpp:479-490), requested explicitly."""
    conf = api.falconsConfig(n)
    conf.cmprAlgo = api.falconsAlgorithm.LORENZO_REG
    conf.errorBoundMode = api.falconsErrorBoundMode.ABS
    conf.absErrorBound = eb
    conf.conf.lorenzo, conf.conf.lorenzo2, conf.conf.regression, conf.conf.regression2 = l1, l2, 0, 0
    conf.conf.blockSize = 5
    return conf


def stream_payload(buf):
    """The payload of one of the library's streams ([Config][u64 L][zstd raw-block frame])."""
    import pyarrow as pa
    import oracle
    s = buf.tobytes()
    h = oracle.lossless_section(s)
    return pa.decompress(s[h + 8:], int.from_bytes(s[h:h + 8], "little"), codec="zstd", asbytes=True)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n,dtype,eb,l1,l2", [
    ("walk", 100000, np.float32, 1e-2, 1, 1), ("sine", 60000, np.float64, 1e-6, 1, 1),
    ("walk", 30011, np.float32, 1e-3, 1, 0), ("sine", 20000, np.float32, 1e-4, 0, 1)])
def test_lorenzo_compress_matches_oracle(cuda, restatement, kind, n, dtype, eb, l1, l2):
    """Explicit ALGO_LORENZO_REG compress of 1-D series the dispatcher keeps lossy: the payload is
    the oracle's byte for byte, the field is left as it was, and the stream decodes to the
    oracle's reconstruction (here and, through its format, with the reference)."""
    from falcons_b200 import api
    from test_lorenzo_oracle import series
    x = series(kind, n, dtype, seed=n)
    before = x.copy()
    buf, _ = api.falcons.compress(x, lorenzo_config(api, n, eb, l1, l2))
    assert same_bits(x, before)
    assert api.read_config(buf).cmprAlgo == 0  # kept as ALGO_LORENZO_REG
    y, _ = api.falcons.decompress(buf, dtype, x.shape)
    if l1 and l2:
        payload, recon = restatement.lorenzo_payload(x, eb)
        assert stream_payload(buf) == payload
        assert same_bits(y, recon)
    assert np.all(np.abs(y.astype(np.float64) - x) <= eb)


@pytest.mark.gpu
def test_lorenzo_compress_of_golden_inputs(cuda):
    """The golden inputs compressed here: where the library's stream keeps the Lorenzo path its
    payload is the reference's (golden) one; a stream the dispatcher stores losslessly decodes to
    the input itself."""
    from falcons_b200 import api
    for path in FIXTURES:
        g = np.load(path)
        x = g["x"].copy()
        buf, _ = api.falcons.compress(x, lorenzo_config(api, x.size, float(g["eb"])))
        y, _ = api.falcons.decompress(buf, x.dtype, x.shape)
        if api.read_config(buf).cmprAlgo == 0:
            if int(g["radius"]) == 32768:
                assert stream_payload(buf) == g["payload"].tobytes()
                assert same_bits(y, g["recon"])
        else:
            assert same_bits(y, g["x"])


@pytest.mark.gpu
def test_unsupported_lorenzo_configs_are_rejected(cuda):
    from falcons_b200 import api
    x = np.linspace(0, 1, 1000, dtype=np.float32)
    conf = lorenzo_config(api, x.size, 1e-3)
    conf.conf.regression = 1  # the regression predictor is not built
    with pytest.raises(ValueError):
        api.falcons.compress(x.copy(), conf)
    x2 = np.ones((30, 40), np.float32)
    conf2 = api.falconsConfig(30, 40)
    conf2.cmprAlgo = api.falconsAlgorithm.LORENZO_REG
    conf2.conf.regression = 0
    with pytest.raises(ValueError):  # N > 1
        api.falcons.compress(x2, conf2)


@pytest.mark.gpu
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "tunedlz_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_tuner_picks_lorenzo_like_reference(cuda, restatement, path):
    """ALGO_INTERP_LORENZO on 1-D fields where the reference's tuner switches to the Lorenzo path:
    the same choice (bins, block size 128), the reference's payload byte for byte, and the
    oracle's reconstruction; the reference stream decodes to the same values."""
    from falcons_b200 import api
    from test_lorenzo_oracle import tuned_fixture
    x, eb, ref_conf, payload = tuned_fixture(path)
    conf = api.falconsConfig(x.size)
    conf.cmprAlgo = api.falconsAlgorithm.INTERP_LORENZO
    conf.errorBoundMode = api.falconsErrorBoundMode.ABS
    conf.absErrorBound = eb
    buf, _ = api.falcons.compress(x.copy(), conf, copy=True)
    c = api.read_config(buf)
    assert c.cmprAlgo == api.falconsAlgorithm.LORENZO_REG
    assert c.quantbinCnt == ref_conf.quantbinCnt and c.blockSize == 128
    assert stream_payload(buf) == payload
    y, _ = api.falcons.decompress(buf, x.dtype, x.shape)
    assert same_bits(y, restatement.lorenzo_decode(payload, x.size, x.dtype, block=128))
    yr, _ = api.falcons.decompress(np.load(path)["stream"], x.dtype, x.shape)
    assert same_bits(yr, y)
