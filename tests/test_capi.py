"""The C ABI without a GPU: the library loads, exports every declared entry point, and its host-only
entry points (stream header parsing, size bound) behave like the reference's."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names += re.findall(r"^\s*(?:int|size_t|uint64_t|const char \*)\s*(falcons_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from falcons_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS)


def test_version_string():
    from falcons_b200 import _lib
    assert b"falcons_b200" in _lib.lib().falcons_version()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "stream_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_read_config_of_reference_streams(path):
    from falcons_b200 import api
    g = np.load(path)
    c = api.read_config(g["stream"])
    assert c.dims == tuple(d for d in g["x"].shape if d > 1)
    assert c.num_elements == g["x"].size
    assert c.errorBoundMode == api.falconsErrorBoundMode.ABS
    assert c.cmprAlgo in (api.falconsAlgorithm.INTERP, api.falconsAlgorithm.LOSSLESS)


def test_read_config_rejects_truncated_and_foreign_streams():
    from falcons_b200 import api
    g = np.load(os.path.join(ROOT, "tests", "golden", "stream_interp_abs_f32.npz"))
    s = g["stream"]
    for bad in (s[:0], s[:1], s[:5], s[: s[0]]):
        with pytest.raises(ValueError):
            api.read_config(bad)
    t = s.copy()
    t[1] ^= 0xFF  # magic number
    with pytest.raises(ValueError, match="magic"):
        api.read_config(t)


def test_size_bound_matches_reference_formula():
    from falcons_b200 import api
    for shape, dt in (((100, 200, 300), np.float32), ((10,), np.float64), ((1800, 3600), np.float32)):
        c = api.falconsConfig(*shape)
        n = int(np.prod(shape)) * np.dtype(dt).itemsize
        zb = n + (n >> 8) + (((128 << 10) - n) >> 11 if n < (128 << 10) else 0)
        hdr = api.size_bound(c, dt) - 4096 - zb
        assert 20 <= hdr <= 60


def test_integer_fields_are_rejected():
    from falcons_b200 import api
    with pytest.raises(TypeError, match="GPU build"):
        api.falcons.compress(np.zeros((4, 4), np.int32), api.falconsConfig(4, 4))
