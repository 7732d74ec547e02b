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
