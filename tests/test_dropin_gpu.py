"""The C++ drop-in API on the GPU: the same C++ caller built against include/falcons_gpu.hpp and
against the reference's falcons.hpp (tests/native/dropin_api.cpp), and the reference's own CLI
source built both ways (tests/native/Makefile), on the plain-method workload: a 100 x 200 x 300
float32 field of 16 seeded sinusoids plus N(0, 1e-4^2) noise, EB_ABS 1e-3, the default
(tuned) algorithm.  Reconstructions are bit-identical and every stream decodes on the other
build.  The binaries are built beforehand (build() or `make -C tests/native`) and travel with the
repository."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "native", "_build")
SHAPE = (100, 200, 300)


@pytest.fixture(scope="module")
def bins(cuda):
    b = {n: os.path.join(BUILD, n) for n in ("dropin_api", "dropin_api_ref", "falcons_cli", "falcons_cli_ref")}
    missing = [n for n, p in b.items() if not os.path.exists(p)]
    if missing:
        pytest.skip(f"drop-in binaries not built: {missing}")
    return b


@pytest.fixture(scope="module")
def field(tmp_path_factory):
    from falcons_b200 import synth
    x = synth.sinusoid_field(SHAPE, seed=0)
    p = tmp_path_factory.mktemp("c1") / "c1.f32"
    x.tofile(p)
    return x, p


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (exe, args, r.stdout, r.stderr)
    return r.stdout


def test_cpp_api_round_trip_matches_reference(bins, field, tmp_path):
    x, path = field
    outs = {}
    for name in ("dropin_api", "dropin_api_ref"):
        s, y = tmp_path / f"{name}.stream", tmp_path / f"{name}.f32"
        conf = run(bins[name], "roundtrip", path, s, y, *SHAPE, 1e-3)
        outs[name] = (s, np.fromfile(y, np.float32), conf)
    (s_gpu, y_gpu, c_gpu), (s_ref, y_ref, c_ref) = outs["dropin_api"], outs["dropin_api_ref"]
    np.testing.assert_array_equal(y_gpu, y_ref)
    assert c_gpu == c_ref                                   # the Config the stream carries
    assert np.abs(y_gpu.astype(np.float64) - x.ravel()).max() <= 1e-3
    for name, stream in (("dropin_api_ref", s_gpu), ("dropin_api", s_ref)):  # each decodes the other's
        yo = tmp_path / f"x_{name}.f32"
        run(bins[name], "decompress", stream, yo)
        np.testing.assert_array_equal(np.fromfile(yo, np.float32), y_ref)


def test_reference_cli_on_the_drop_in(bins, field, tmp_path):
    x, path = field
    dims = ["-3", SHAPE[2], SHAPE[1], SHAPE[0]]                # the CLI takes the fastest dimension first
    rec = {}
    for name in ("falcons_cli", "falcons_cli_ref"):
        z, o = tmp_path / f"{name}.falcons", tmp_path / f"{name}.out"
        out = run(bins[name], "-f", "-i", path, "-z", z, *dims, "-M", "ABS", "1e-3")
        assert "compression ratio" in out
        run(bins[name], "-f", "-z", z, "-o", o, *dims, "-M", "ABS", "1e-3")
        rec[name] = (z, np.fromfile(o, np.float32))
    np.testing.assert_array_equal(rec["falcons_cli"][1], rec["falcons_cli_ref"][1])
    for name, other in (("falcons_cli", "falcons_cli_ref"), ("falcons_cli_ref", "falcons_cli")):
        o = tmp_path / f"cross_{name}.out"
        run(bins[name], "-f", "-z", rec[other][0], "-o", o, *dims, "-M", "ABS", "1e-3")
        np.testing.assert_array_equal(np.fromfile(o, np.float32), rec["falcons_cli_ref"][1])
