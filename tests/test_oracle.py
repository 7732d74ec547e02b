"""The oracle itself: the C restatement against the golden fixtures made by the reference build,
and (where the reference build exists here) against the reference on fresh random cases."""
import glob
import itertools
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _interp_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "interp_*.npz")))


@pytest.mark.parametrize("path", _interp_cases(), ids=lambda p: os.path.basename(p))
def test_restatement_matches_golden(restatement, path):
    g = np.load(path)
    r = restatement.compress(g["x"], float(g["eb"]), int(g["algo"]), int(g["direction"]), None,
                             float(g["alpha"]), float(g["beta"]))
    np.testing.assert_array_equal(r.codes, g["codes"])
    np.testing.assert_array_equal(r.unpred, g["unpred"])
    np.testing.assert_array_equal(r.mutated, g["mutated"])
    np.testing.assert_array_equal(r.recon, g["recon"])
    assert np.abs(r.recon.astype(np.float64) - g["x"].astype(np.float64)).max() <= float(g["eb"])


def test_interpolator_known_answers(restatement):
    # tools/test/modules/test_interpolators.cpp:67-70: interp_linear(10, 30) = 20 and
    # interp_cubic(0, 20, 40, 60) = 30.  With anchor stride 2 the even points are stored exactly,
    # so on a linear ramp every predictor (linear, linear1, quad1/2, cubic) is exact: all codes 0.
    x = np.array([10, 20, 30, 40], np.float32)
    r = restatement.compress(x, 1e-6, 0, 0, 2)
    np.testing.assert_array_equal(r.codes, [0, 0])
    x = np.arange(0, 90, 10, dtype=np.float32)
    r = restatement.compress(x, 1e-6, 1, 0, 2)
    np.testing.assert_array_equal(r.codes, np.zeros(4, np.int16))
    np.testing.assert_array_equal(r.recon, x)


def _field(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    g = np.meshgrid(*[np.linspace(0, 3, s) for s in shape], indexing="ij")
    x = sum(np.sin((i + 1.3) * gi) for i, gi in enumerate(g)) + 0.01 * rng.standard_normal(shape)
    x[rng.random(shape) < 0.02] += 50
    return x.astype(dtype)


def test_restatement_matches_reference(restatement, reference):
    rng = np.random.default_rng(11)
    n = 0
    for N, sizes in ((1, [2, 3, 5, 8, 9, 100, 4097]), (2, [2, 3, 6, 9, 33]), (3, [2, 3, 5, 8, 9, 17])):
        for shape in itertools.product(sizes, repeat=N):
            if N == 3 and rng.random() > 0.3:
                continue
            for algo in (0, 1):
                for direction in ((0,) if N == 1 else (0, {2: 1, 3: 5}[N])):
                    for tuning in (False, True):
                        x = _field(shape, np.float32, n)
                        eb = 1e-3 * float(x.max() - x.min())
                        a = reference.interp_compress(x, eb, algo, direction, -1, 1.25, 2.0, tuning)
                        b = restatement.compress(x, eb, algo, direction, None, 1.25, 2.0, tuning)
                        np.testing.assert_array_equal(a.codes, b.codes)
                        np.testing.assert_array_equal(a.unpred, b.unpred)
                        np.testing.assert_array_equal(a.mutated, b.mutated)
                        if not tuning:
                            np.testing.assert_array_equal(a.recon, b.recon)
                        n += 1
    assert n > 300


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "stream_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_golden_streams_decode_with_reference(reference, path):
    g = np.load(path)
    y = reference.decompress(g["stream"].tobytes(), g["x"].dtype, g["x"].size).reshape(g["x"].shape)
    np.testing.assert_array_equal(y, g["recon"])
