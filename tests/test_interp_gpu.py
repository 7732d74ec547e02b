"""GPU parity of the interpolation decomposition against the C restatement (bit-exact)."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _field(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    g = np.meshgrid(*[np.linspace(0, 3, s) for s in shape], indexing="ij")
    x = sum(np.sin((i + 1.3) * gi) for i, gi in enumerate(g)) + 0.01 * rng.standard_normal(shape)
    x[rng.random(shape) < 0.02] += 50
    return x.astype(dtype)


def _run(cuda, restatement, x, algo, direction, anchor=None, alpha=1.25, beta=2.0, tuning=False):
    import torch
    from falcons_b200 import device as D
    eb = 1e-3 * float(x.max() - x.min())
    ref = restatement.compress(x, eb, algo, direction, anchor, alpha, beta, tuning)
    p = D.interp_params(eb, algo, direction, anchor, x.ndim, alpha, beta, tuning=tuning)
    xd = torch.from_numpy(x.copy()).to(cuda)
    codes, unpred = D.interp_compress(xd, p)
    np.testing.assert_array_equal(codes.cpu().numpy(), ref.codes)
    np.testing.assert_array_equal(unpred.cpu().numpy(), ref.unpred)
    np.testing.assert_array_equal(xd.cpu().numpy(), ref.mutated)
    if not tuning:
        rec = D.interp_decompress(x.shape, xd.dtype, codes, unpred, p)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rec.cpu().numpy(), ref.recon)
        assert np.abs(rec.cpu().numpy().astype(np.float64) - x).max() <= eb


SMALL = {1: [(2,), (3,), (5,), (8,), (9,), (100,), (4097,), (5000,)],
         2: [(2, 2), (3, 7), (5, 6), (9, 12), (33, 130), (140, 17), (129, 257)],
         3: [(2, 2, 2), (3, 4, 5), (6, 7, 8), (9, 11, 16), (33, 33, 33), (40, 17, 9), (65, 66, 67)]}


@pytest.mark.parametrize("N", [1, 2, 3])
@pytest.mark.parametrize("algo", [0, 1])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_small_shapes(cuda, restatement, N, algo, dtype):
    for i, shape in enumerate(SMALL[N]):
        for direction in ((0,) if N == 1 else (0, {2: 1, 3: 5}[N])):
            _run(cuda, restatement, _field(shape, dtype, i), algo, direction)


def test_exhaustive_small_3d(cuda, restatement):
    for shape in itertools.product([2, 3, 4, 5, 6, 7, 8, 9], repeat=3):
        if sum(shape) % 3:
            continue
        for algo in (0, 1):
            for direction in (0, 5):
                _run(cuda, restatement, _field(shape, np.float32, sum(shape)), algo, direction)


@pytest.mark.parametrize("shape,dtype", [((4, 700, 90), np.float32), ((5, 330, 75), np.float64),
                                         ((3, 64, 200), np.float32), ((650, 101), np.float32),
                                         ((6, 9, 133), np.float64)])
def test_fused_level_passes(cuda, restatement, shape, dtype):
    # the y and x passes of a level run as one kernel over x chunks (with halos); long rows, long
    # columns (narrower chunks) and ragged last chunks
    for algo in (0, 1):
        for direction in ((0, 1) if len(shape) == 2 else (0, 5)):
            _run(cuda, restatement, _field(shape, dtype, 11), algo, direction)


@pytest.mark.parametrize("shape", [(9, 100, 132), (10, 130, 68), (6, 67, 72), (7, 129, 260), (4, 64, 4),
                                   (131, 196), (64, 4), (70, 8)])
def test_unit_step_level_kernel(cuda, restatement, shape):
    # the finest level of a float field whose rows are 16-byte aligned runs the split-column
    # kernel: tiles cut short in x and in y, odd and even plane counts (the last plane's own z
    # pass), an even row count (the last row's own y pass), rows of 4 and 8 values
    for x in (_field(shape, np.float32, 13), _field(shape, np.float32, 14) * 1e-3):
        _run(cuda, restatement, x, 1, 0)


def test_fused_kernels_only_where_requantization_is_exact(cuda, restatement):
    """A float field far from zero (values near 1e4, range about 53) at an error bound of 1e-4 of
    its range: the bound is below 2^-20 of the largest |value|, where quantizing a reconstruction
    again may not give it back, so compress runs the level passes one kernel each instead of the
    fused kernels (which re-quantize the halo targets that a neighbouring tile may already have
    overwritten).  Codes and reconstruction stay bit-exact, and that compress launches more
    kernels than the same field near zero."""
    import torch
    from falcons_b200 import _lib
    from falcons_b200 import device as D
    x = _field((12, 70, 136), np.float32, 3)
    counts = []
    for field in (x, (x + np.float32(1e4)).astype(np.float32)):
        eb = 1e-4 * float(field.max() - field.min())
        assert (eb < 2.0 ** -20 * float(np.abs(field).max())) == (field is not x)
        _run(cuda, restatement, field, 1, 0)  # 1e-3 of the range: fused for both fields
        ref = restatement.compress(field, eb, 1, 0)
        xd = torch.from_numpy(field.copy()).to(cuda)
        torch.cuda.synchronize()
        l0 = _lib.lib().falcons_kernel_launches()
        codes, unpred = D.interp_compress(xd, D.interp_params(eb, 1, 0, None, 3))
        counts.append(_lib.lib().falcons_kernel_launches() - l0)
        np.testing.assert_array_equal(codes.cpu().numpy(), ref.codes)
        np.testing.assert_array_equal(unpred.cpu().numpy(), ref.unpred)
        np.testing.assert_array_equal(xd.cpu().numpy(), ref.mutated)
    assert counts[1] > counts[0]


@pytest.mark.parametrize("shape", [(33, 40, 17), (20, 21, 22), (5, 6, 7, 8), (17, 3, 9, 4)])
def test_generic_and_tuning_sweeps(cuda, restatement, shape):
    for algo in (0, 1):
        if len(shape) == 3:
            for direction in range(6):
                _run(cuda, restatement, _field(shape, np.float32, 7), algo, direction, tuning=True)
        else:
            for direction in (0, 23):
                _run(cuda, restatement, _field(shape, np.float32, 7), algo, direction)


@pytest.mark.parametrize("ab", [(1.0, 1.0), (1.5, 2.5), (-1.0, -1.0), (0.5, 3.0)])
def test_alpha_beta_and_anchors(cuda, restatement, ab):
    x = _field((40, 41, 42), np.float64, 3)
    _run(cuda, restatement, x, 1, 0, None, *ab)
    for anchor in (0, 8, 64):
        _run(cuda, restatement, _field((30, 31, 32), np.float32, 4), 1, 5, anchor, *ab)


def test_nonfinite(cuda, restatement):
    x = _field((30, 31, 32), np.float32, 5)
    x[3, 4, 5] = np.nan
    x[10, 10, 10] = np.inf
    x[11, 11, 11] = -np.inf
    import torch
    from falcons_b200 import device as D
    ref = restatement.compress(x, 1e-2, 1, 0)
    xd = torch.from_numpy(x.copy()).to(cuda)
    codes, unpred = D.interp_compress(xd, D.interp_params(1e-2, 1, 0, None, 3))
    np.testing.assert_array_equal(codes.cpu().numpy(), ref.codes)
    np.testing.assert_array_equal(unpred.cpu().numpy(), ref.unpred)


def test_value_range(cuda):
    import torch
    from falcons_b200 import device as D
    x = _field((50, 60, 70), np.float32, 9)
    r = D.value_range(torch.from_numpy(x).to(cuda))
    assert r == float(np.float32(x.max()) - np.float32(x.min()))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_decompress_refuses_more_escapes_than_the_list(cuda, restatement, dtype):
    """Codes built on the host with one escape more than the unpredictable list holds: the context
    entry point returns EINVAL (ValueError) and reads nothing past the list."""
    import torch
    from falcons_b200 import device as D
    x = _field((30, 31, 32), dtype, 7)
    eb = 1e-3 * float(x.max() - x.min())
    ref = restatement.compress(x, eb, 1, 0)
    p = D.interp_params(eb, 1, 0, None, 3)
    codes = ref.codes.copy()
    pos = int(np.flatnonzero(codes != -p.radius)[codes.size // 3])
    codes[pos] = -p.radius
    dc = torch.from_numpy(codes).to(cuda)
    du = torch.from_numpy(ref.unpred.copy()).to(cuda)
    with pytest.raises(ValueError, match="unpredictable values"):
        D.interp_decompress(x.shape, du.dtype, dc, du, p)
    # a list of exactly the right length still decodes bit-exact
    rec = D.interp_decompress(x.shape, du.dtype, torch.from_numpy(ref.codes.copy()).to(cuda), du, p)
    np.testing.assert_array_equal(rec.cpu().numpy(), ref.recon)
