"""The C++ drop-in API (include/falcons_gpu.hpp, reached through include/dropin/Falcons/api/falcons.hpp)
compiled against the reference's own Falcons::Config, without a GPU.

tests/native/Makefile builds one caller (tests/native/dropin_api.cpp) twice, against the drop-in
header and against the reference's falcons.hpp, and builds the reference's CLI source
(tools/falcons/falcons.cpp) unchanged against the drop-in.  Here the two builds must agree on
everything that needs no GPU: the Config read from streams, the compressed-size bound, the
exception type of malformed streams; and integral element types are refused.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
BUILD = os.path.join(NATIVE, "_build")
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def bins():
    if not os.path.isdir("/root/reference/include/Falcons") or shutil.which("g++") is None:
        pytest.skip("the reference's headers are needed to build the drop-in checks")
    subprocess.check_call(["make", "-s", "-C", NATIVE])
    return {n: os.path.join(BUILD, n) for n in ("dropin_api", "dropin_api_ref", "falcons_cli", "falcons_cli_ref")}


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=120)
    return r.returncode, r.stdout.strip()


@pytest.mark.parametrize("name", sorted(f for f in os.listdir(GOLDEN) if f.startswith(("stream_", "tunedlz_"))))
def test_read_config_matches_reference(bins, tmp_path, name):
    g = np.load(os.path.join(GOLDEN, name))
    path = tmp_path / "s.bin"
    path.write_bytes(g["stream"].tobytes())
    ours, ref = run(bins["dropin_api"], "config", path), run(bins["dropin_api_ref"], "config", path)
    assert ours[0] == 0 and ours == ref


def test_malformed_streams_raise_invalid_argument_like_reference(bins, tmp_path):
    g = np.load(os.path.join(GOLDEN, "stream_interp_abs_f32.npz"))
    s = g["stream"].tobytes()
    for bad in (s[:6], s[:int(s[0])], b"\x20" + b"\x00" * 40, b"\x05XYZWVUTSRQ" + s[12:]):
        p = tmp_path / "bad.bin"
        p.write_bytes(bad)
        ours, ref = run(bins["dropin_api"], "config", p), run(bins["dropin_api_ref"], "config", p)
        assert ours[0] == ref[0] == 5, (bad[:12], ours, ref)      # std::invalid_argument on both


@pytest.mark.parametrize("dims", [(1000,), (300, 200), (100, 200, 300), (9, 10, 11, 12), (1, 512, 1, 7)])
def test_size_bound_matches_reference(bins, dims):
    ours, ref = run(bins["dropin_api"], "bound", 0, *dims), run(bins["dropin_api_ref"], "bound", 0, *dims)
    assert ours[0] == 0 and ours == ref


def test_integral_types_are_refused(bins):
    rc, out = run(bins["dropin_api"], "integral")
    assert rc == 0 and out == "invalid_argument: unsupported on GPU build"


def test_reference_cli_builds_on_the_drop_in(bins):
    assert run(bins["falcons_cli"], "-v") == run(bins["falcons_cli_ref"], "-v")
    out = subprocess.run(["ldd", bins["falcons_cli"]], capture_output=True, text=True).stdout
    assert "libfalcons_b200.so" in out
