"""Generates the golden fixtures of tests/golden from the reference build (oracle/_ref).

Run from the repository root where the reference sources are available:
    make -C oracle ref && python tests/golden/make_golden.py            (every fixture)
    make -C oracle ref && python tests/golden/make_golden.py lorenzo    (the 1-D Lorenzo ones only)
Each case stores its seeded input, so the fixtures do not depend on the generators.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

R = oracle.Reference()


def field(shape, dtype, seed, spikes=0.01):
    rng = np.random.default_rng(seed)
    g = np.meshgrid(*[np.linspace(0, 3, s) for s in shape], indexing="ij")
    x = sum(np.sin((i + 1.3) * gi) for i, gi in enumerate(g)) + 0.01 * rng.standard_normal(shape)
    x[rng.random(shape) < spikes] += 50
    return x.astype(dtype)


INTERP_CASES = [
    # name, shape, dtype, algo, direction, alpha, beta, eb_rel
    ("f32_3d_cubic_dir0", (17, 20, 23), np.float32, 1, 0, 1.25, 2.0, 1e-3),
    ("f32_3d_linear_dir5", (33, 9, 40), np.float32, 0, 5, 1.25, 2.0, 1e-3),
    ("f64_3d_cubic_dir5", (12, 35, 16), np.float64, 1, 5, 1.25, 2.0, 1e-5),
    ("f32_2d_cubic_dir1", (130, 77), np.float32, 1, 1, 1.0, 1.0, 1e-3),
    ("f64_2d_linear_dir0", (64, 200), np.float64, 0, 0, 1.5, 2.5, 1e-4),
    ("f32_1d_cubic", (5001,), np.float32, 1, 0, 1.0, 1.0, 1e-3),
    ("f32_4d_cubic", (9, 10, 11, 12), np.float32, 1, 0, 1.25, 2.0, 1e-3),
]

STREAM_CASES = [
    # name, shape, dtype, cmprAlgo, eb mode, abs, rel
    ("interp_abs_f32", (20, 30, 40), np.float32, oracle.ALGO_INTERP, oracle.EB_ABS, 1e-3, 0.0),
    ("interp_rel_f64", (16, 40, 41), np.float64, oracle.ALGO_INTERP, oracle.EB_REL, 0.0, 1e-5),
    ("tuned_f32_3d", (40, 50, 60), np.float32, oracle.ALGO_INTERP_LORENZO, oracle.EB_ABS, 1e-3, 0.0),
    ("interp_rel_f32_2d", (300, 400), np.float32, oracle.ALGO_INTERP, oracle.EB_REL, 0.0, 1e-3),
    ("lossless_f32", (10, 10), np.float32, oracle.ALGO_INTERP, oracle.EB_ABS, 0.0, 0.0),
]


LORENZO_CASES = [
    # name, n, dtype, kind, eb (absolute), quantbinCnt
    ("walk_f32", 3001, np.float32, "walk", 1e-2, 65536),
    ("spiky_f64", 1237, np.float64, "spikes", 1e-6, 65536),
    ("const_f32", 17, np.float32, "const", 1e-3, 65536),
    ("sine_f32_q16384", 2003, np.float32, "sine", 1e-4, 16384),
    ("sine_f64_stream", 6000, np.float64, "sine", 1e-4, 65536),
]


def lorenzo_series(kind, n, dtype, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64)
    if kind == "walk":
        x = np.cumsum(rng.normal(size=n))
    elif kind == "spikes":
        x = np.sin(0.05 * t) + 1e-6 * rng.normal(size=n)
        x[rng.random(n) < 0.02] = 1e20
    elif kind == "const":
        x = np.zeros(n)
    else:
        x = 10 * np.sin(0.01 * t) + 1e-3 * rng.normal(size=n)
    return x.astype(dtype)


def lorenzo_fixtures(out):
    """The 1-D blockwise Lorenzo path: input, the payload before zstd, its reconstruction, the
    whole reference stream and the reference's decode of it (the dispatcher may store tiny or
    incompressible series losslessly)."""
    for name, n, dt, kind, eb, qb in LORENZO_CASES:
        x = lorenzo_series(kind, n, dt, len(name))
        payload, _ = R.lorenzo_payload(x, eb, qb)
        recon = R.lorenzo_decode(payload, n, dt)
        stream = R.compress(x, oracle.lorenzo_ref_conf(eb, qb))
        stream_recon = R.decompress(stream, dt, n).ravel()
        np.savez_compressed(os.path.join(HERE, f"lorenzo_{name}.npz"), x=x, eb=eb, radius=qb // 2, block=5,
                            payload=np.frombuffer(payload, np.uint8), recon=recon,
                            stream=np.frombuffer(stream, np.uint8), stream_recon=stream_recon)
        out["lorenzo_" + name] = len(payload)


TUNED_LORENZO_CASES = [
    # name, n, dtype, eb (absolute): 1-D fields on which the reference's ALGO_INTERP_LORENZO tuner
    # switches to the blockwise Lorenzo path (the last one with 16384 quantization bins)
    ("spikes_f32", 20000, np.float32, 0.1),
    ("spikes_f64", 20000, np.float64, 0.01),
    ("spikes_f32_q16384", 50000, np.float32, 0.1),
]


def tuned_lorenzo_fixtures(out):
    """The tuner's choice of the Lorenzo path: input and the reference's whole stream (its payload
    is the stream's zstd section; its Config carries the chosen bins and block size)."""
    for name, n, dt, eb in TUNED_LORENZO_CASES:
        t = np.arange(n, dtype=np.float64)
        rng = np.random.default_rng(n)
        x = np.sin(0.05 * t)
        x[rng.random(n) < 0.02] = 1e20
        x = x.astype(dt)
        stream = R.compress(x, oracle.ref_conf(algo=oracle.ALGO_INTERP_LORENZO, abs_eb=eb))
        np.savez_compressed(os.path.join(HERE, f"tunedlz_{name}.npz"), x=x, eb=eb,
                            stream=np.frombuffer(stream, np.uint8))
        out["tunedlz_" + name] = len(stream)


def main():
    out = {}
    if sys.argv[1:] == ["lorenzo"]:
        lorenzo_fixtures(out)
        tuned_lorenzo_fixtures(out)
        print(out)
        return
    for name, shape, dt, algo, d, a, b, rel in INTERP_CASES:
        x = field(shape, dt, len(name))
        eb = rel * float(x.max() - x.min())
        r = R.interp_compress(x, eb, algo, d, -1, a, b)
        np.savez_compressed(os.path.join(HERE, f"interp_{name}.npz"), x=x, eb=eb, algo=algo, direction=d,
                            alpha=a, beta=b, codes=r.codes, unpred=r.unpred, recon=r.recon, mutated=r.mutated)
        out[name] = len(r.codes)
    for name, shape, dt, algo, mode, ab, rl in STREAM_CASES:
        x = field(shape, dt, len(name), spikes=0.0)
        conf = oracle.ref_conf(algo=algo, eb_mode=mode, abs_eb=ab, rel_eb=rl)
        s = R.compress(x, conf)
        y = R.decompress(s, dt, x.size).reshape(shape)
        np.savez_compressed(os.path.join(HERE, f"stream_{name}.npz"), x=x, stream=np.frombuffer(s, np.uint8),
                            recon=y)
        out[name] = len(s)
    rng = np.random.default_rng(7)
    for name, q in [("sparse", np.where(rng.random(200000) < 0.9, 0, rng.integers(-5, 6, 200000))),
                    ("dense", np.round(rng.laplace(0, 60, 300000)).clip(-32767, 32767)),
                    ("delta", np.repeat(rng.integers(-3, 4, 4000), 50))]:
        q = q.astype(np.int16)
        enc = R.rlefse_encode(q)
        np.savez_compressed(os.path.join(HERE, f"rlefse_{name}.npz"), codes=q, payload=np.frombuffer(enc, np.uint8))
        out["rlefse_" + name] = len(enc)
    lorenzo_fixtures(out)
    tuned_lorenzo_fixtures(out)
    print(out)


if __name__ == "__main__":
    main()
