"""The batched and serving forms on the GPU: every field's stream and reconstruction are the bits
of the single-field device path, whatever runs beside it.

* falcons_compress_batch / falcons_decompress_batch on a mixed batch (cubes, 2-D arrays, 1-D
  series; float32 and float64; per-field relative bounds), against one
  falcons_compress_device / falcons_decompress_device call per field; a failing item fails
  alone and the call names it; the autotuner records a worker count.
* The serving loop (falcons_b200.serve): requests submitted with Poisson arrivals run
  concurrently under a device-memory budget, and each result equals the same request run alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed(n, seed, cuda):
    import torch
    from falcons_b200 import synth
    rng = np.random.default_rng(seed)
    fields = []
    for i in range(n):
        kind = i % 3
        if kind == 0:
            shape = (int(rng.integers(16, 72)),) * 3
        elif kind == 1:
            shape = (int(rng.integers(64, 400)), int(rng.integers(64, 400)))
        else:
            shape = (int(rng.integers(4096, 200000)),)
        dt = torch.float64 if i % 5 == 4 else torch.float32
        x = synth.spectral_field_torch(shape, seed=1000 + i, device=cuda, dtype=dt)
        fields.append((x, float(10 ** rng.uniform(-5, -2))))
    return fields


def _conf(api, shape, rel):
    c = api.falconsConfig(*shape)
    c.cmprAlgo = api.falconsAlgorithm.INTERP
    c.errorBoundMode = api.falconsErrorBoundMode.REL
    c.relErrorBound = rel
    return c


def test_batch_matches_single_field_path(cuda):
    import torch
    from falcons_b200 import _lib, api
    from falcons_b200 import device as D
    fields = _mixed(48, 1, cuda)  # enough for the autotuner's first two candidates (7 x 2 + 7 x 4 fields)
    single, mutated = [], []
    for x, rel in fields:
        w = x.clone()
        s, _ = D.compress(w, _conf(api, x.shape, rel))
        single.append(s.clone())
        mutated.append(w)
    work = [x.clone() for x, _ in fields]
    out = D.compress_batch(work, [_conf(api, x.shape, rel) for x, rel in fields], workers=0)
    torch.cuda.synchronize()
    for (s, conf), s1, w, m in zip(out, single, work, mutated):
        assert torch.equal(s, s1)                      # the same stream bytes
        assert torch.equal(w, m)                       # the same partial reconstruction left behind
    recs = [torch.empty(x.numel(), dtype=x.dtype, device=cuda) for x, _ in fields]
    D.decompress_batch([s for s, _ in out], [x.dtype for x, _ in fields], recs, workers=4)
    torch.cuda.synchronize()
    for (x, rel), (s, _), r in zip(fields, out, recs):
        y, _ = D.decompress(s, x.dtype)
        assert torch.equal(r, y)
        eb = rel * float(x.max() - x.min())
        assert float((r.double() - x.reshape(-1).double()).abs().max()) <= eb
    mean = sum(x.numel() * x.element_size() for x, _ in fields) // len(fields)
    assert _lib.lib().falcons_batch_workers(_lib.default_context(0).ptr, mean) in (2, 4, 8, 16)


def test_batch_item_errors_stay_with_their_item(cuda):
    import ctypes
    import torch
    from falcons_b200 import _lib, api
    fields = _mixed(4, 2, cuda)
    items = (_lib.BatchItem * 4)()
    keep = []
    for i, (x, rel) in enumerate(fields):
        c = _conf(api, x.shape, rel)
        cap = int(_lib.lib().falcons_compress_size_bound(0 if x.dtype == torch.float32 else 1, ctypes.byref(c.conf)))
        out = torch.empty(cap if i != 2 else 16, dtype=torch.uint8, device=cuda)   # item 2: no room
        keep += [out, x]
        items[i].dtype = 0 if x.dtype == torch.float32 else 1
        items[i].conf = c.conf
        items[i].d_data = x.data_ptr()
        items[i].d_stream = out.data_ptr()
        items[i].cap = out.numel()
    rc = _lib.lib().falcons_compress_batch(_lib.default_context(0).ptr, items, ctypes.c_size_t(4), 2)
    assert rc == _lib.EINVAL
    assert "batch item 2" in _lib.lib().falcons_last_error().decode()
    assert [items[i].status for i in range(4)] == [0, 0, _lib.EINVAL, 0]
    assert all(items[i].len > 0 for i in (0, 1, 3))


def test_serving_results_are_the_same_alone_and_in_the_mix(cuda):
    import torch
    from falcons_b200 import api, serve
    from falcons_b200 import device as D
    fields = _mixed(24, 3, cuda)
    confs = [_conf(api, x.shape, rel) for x, rel in fields]
    alone = []
    for (x, _), c in zip(fields, confs):
        s, _ = D.compress(x.clone(), _conf(api, x.shape, c.relErrorBound))
        alone.append(s.clone())
    srv = serve.Server(workers=6, budget_bytes=4 << 30)
    try:
        reqs = [(lambda t, x=x, rel=rel: srv.submit_compress(x.clone(), _conf(api, x.shape, rel), arrival=t))
                for x, rel in fields]
        # decompress requests of streams made alone, mixed in
        reqs += [(lambda t, s=s, x=x: srv.submit_decompress(s, x.dtype, arrival=t))
                 for s, (x, _) in zip(alone[:8], fields[:8])]
        order = np.random.default_rng(0).permutation(len(reqs))
        futs, wall = serve.open_loop(srv, [reqs[i] for i in order], rate=400.0)
        results = [None] * len(reqs)
        for i, f in zip(order, futs):
            results[i] = f.result()
        for i in range(len(fields)):
            assert torch.equal(results[i][0], alone[i])
        for j in range(8):
            y, _ = D.decompress(alone[j], fields[j][0].dtype)
            assert torch.equal(results[len(fields) + j][0], y)
        st = serve.latency_stats(srv.completed)
        assert st["n"] == len(reqs) and st["p50_ms"] <= st["p99_ms"]
        assert srv.in_use == 0
    finally:
        srv.close()


def test_serving_budget_refuses_oversized_requests(cuda):
    import torch
    from falcons_b200 import api, serve
    srv = serve.Server(workers=2, budget_bytes=1 << 20)
    try:
        x = torch.zeros(1 << 20, device=cuda)
        f = srv.submit_compress(x, _conf(api, x.shape, 1e-3))
        with pytest.raises(ValueError, match="budget"):
            f.result(timeout=10)
    finally:
        srv.close()
