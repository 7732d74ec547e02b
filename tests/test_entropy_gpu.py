"""GPU entropy stage (RleFseEncoder format) against the reference encoder/decoder."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _codes(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "sparse":      # p(0) >= 0.8 -> method 0 (RLE + gamma + FSE)
        q = np.where(rng.random(n) < 0.9, 0, rng.integers(-5, 6, n))
    elif kind == "dense":     # method 1 (order-1 tANS), wide codes with escapes
        q = np.round(rng.laplace(0, 60, n)).clip(-32767, 32767)
    elif kind == "smooth":    # delta helps
        q = np.repeat(rng.integers(-3, 4, n // 50 + 1), 50)[:n]
    elif kind == "escapes":
        q = np.round(rng.laplace(0, 400, n)).clip(-32767, 32767)
        q[rng.random(n) < 0.01] = -32768
    else:                     # mixed stream with long zero runs and a trailing zero run
        q = np.zeros(n)
        idx = rng.choice(n, max(1, n // 100), replace=False)
        q[idx] = rng.integers(-100, 100, idx.size)
    return q.astype(np.int16)


CASES = [(k, n) for k in ("sparse", "dense", "smooth", "escapes", "mixed")
         for n in (1, 2, 3, 100, 5000, 76799, 76800, 300001, 1 << 20, 3 << 20)]


@pytest.mark.parametrize("kind,n", CASES)
def test_gpu_stream_decodes_with_reference(cuda, reference, kind, n):
    import torch
    from falcons_b200 import device as D
    q = _codes(kind, n, n)
    enc = D.encode_codes(torch.from_numpy(q).to(cuda)).cpu().numpy().tobytes()
    ref_enc = reference.rlefse_encode(q)
    assert enc[0] == ref_enc[0], "method/delta byte differs from the reference's choice"
    np.testing.assert_array_equal(reference.rlefse_decode(enc, n), q)
    back = D.decode_codes(torch.frombuffer(bytearray(enc), dtype=torch.uint8).to(cuda), n).cpu().numpy()
    np.testing.assert_array_equal(back, q)


@pytest.mark.parametrize("kind,n", CASES)
def test_reference_stream_decodes_on_gpu(cuda, reference, kind, n):
    import torch
    from falcons_b200 import device as D
    q = _codes(kind, n, n + 1)
    ref_enc = reference.rlefse_encode(q)
    back = D.decode_codes(torch.frombuffer(bytearray(ref_enc), dtype=torch.uint8).to(cuda), n).cpu().numpy()
    np.testing.assert_array_equal(back, q)
