"""Run one stage of the path on a seeded synthetic field, for profiling a single stage under ncu.

    python -m falcons_b200.stage --stage interp_compress --size 512 --iters 1

Stages: interp_compress, interp_decompress, encode, decode, compress, decompress.  The field is
the spectral k^-11/3 Gaussian random field of ``synth.spectral_field_torch`` (size^3 float32),
the error bound REL --rel with cubic interpolation, direction 0.  Everything the chosen stage
needs is prepared first (untimed); the stage then runs --iters times and its mean CUDA-event
time is printed.  The stream of the last `compress` (or the codes of the last
`interp_compress`) is checked against the error bound so that a profiled run is a correct run.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import _lib, api, synth
from . import device as D


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", required=True,
                    choices=["interp_compress", "interp_decompress", "encode", "decode", "compress", "decompress"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--rel", type=float, default=1e-4)
    ap.add_argument("--iters", type=int, default=1)
    a = ap.parse_args(argv)
    shape = (a.size,) * 3
    x0 = synth.spectral_field_torch(shape, seed=1)
    eb = a.rel * float(x0.max() - x0.min())
    p = D.interp_params(eb, 1, 0, None, 3, max_abs=float(x0.abs().max()))
    ctx = _lib.default_context(0)
    x = x0.clone()
    rec = torch.empty_like(x0)
    codes = unpred = payload = stream = None
    if a.stage != "interp_compress" and a.stage not in ("compress", "decompress"):
        codes, unpred = D.interp_compress(x, p, ctx=ctx)
        if a.stage == "decode":
            payload = D.encode_codes(codes, ctx=ctx)
    conf = api.falconsConfig(*shape)
    conf.cmprAlgo = api.falconsAlgorithm.INTERP
    conf.errorBoundMode = api.falconsErrorBoundMode.REL
    conf.relErrorBound = a.rel
    if a.stage == "decompress":
        stream, _ = D.compress(x0.clone(), conf, ctx=ctx)
    torch.cuda.synchronize()

    times = []
    for _ in range(a.iters):
        if a.stage in ("interp_compress", "compress"):
            x.copy_(x0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if a.stage == "interp_compress":
            codes, unpred = D.interp_compress(x, p, ctx=ctx)
        elif a.stage == "interp_decompress":
            D.interp_decompress(shape, torch.float32, codes, unpred, p, out=rec, ctx=ctx)
        elif a.stage == "encode":
            payload = D.encode_codes(codes, ctx=ctx)
        elif a.stage == "decode":
            D.decode_codes(payload, codes.numel(), ctx=ctx)
        elif a.stage == "compress":
            stream, _ = D.compress(x, conf, ctx=ctx)
        else:
            D.decompress(stream, torch.float32, out=rec.view(-1), ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))

    if a.stage in ("interp_compress", "interp_decompress"):
        if a.stage == "interp_compress":
            D.interp_decompress(shape, torch.float32, codes, unpred, p, out=rec, ctx=ctx)
        err = float((rec.double() - x0.double()).abs().max())
    elif a.stage in ("compress", "decompress"):
        if a.stage == "compress":
            D.decompress(stream, torch.float32, out=rec.view(-1), ctx=ctx)
        err = float((rec.view(shape).double() - x0.double()).abs().max())
    else:
        back = D.decode_codes(payload, codes.numel(), ctx=ctx)
        err = 0.0 if torch.equal(back[:codes.numel()], codes) else float("inf")
    torch.cuda.synchronize()
    if not err <= eb * (1 + 1e-12):
        raise SystemExit(f"stage {a.stage}: check failed (max error {err}, bound {eb})")
    print(f"stage {a.stage} size {a.size}^3 rel {a.rel}: {np.mean(times):.3f} ms mean of {a.iters}, "
          f"max error {err:.3g} <= {eb:.3g}")


if __name__ == "__main__":
    main()
