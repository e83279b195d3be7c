"""Per-op C-ABI kernels against numpy / the oracle: N-D FFT (BackEnd.ft/ift), norm, pointwise matrix product."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the last six take the register-staged passes on some or all axes (lengths 64 .. 512), alone or mixed with the
# runtime-radix passes, with small and large contiguous tiles
SHAPES = [(5, 10, 20), (64,), (1024,), (128, 96), (16, 24, 20), (12, 7, 13), (30, 64), (256, 256), (3, 11),
          (128, 128), (64, 64, 64), (512, 256), (32, 256), (256, 30), (16, 128, 512)]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or 0)


@pytest.mark.parametrize('shape', SHAPES)
@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_fftn_matches_numpy(shape, dtype):
    import torch
    from macromax_b200 import _native as nat
    rng = np.random.default_rng(3)
    nb = 3
    x = (rng.standard_normal((nb, *shape)) + 1j * rng.standard_normal((nb, *shape))).astype(dtype)
    prec = nat.MMX_C64 if dtype == np.complex64 else nat.MMX_C128
    plan = nat.Plan(shape, 1, 1, prec)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty_like(xt)
    nat.call('mmx_fftn', plan.handle, _ptr(xt), _ptr(yt), nb, 0, _stream())
    axes = tuple(range(1, 1 + len(shape)))
    ref = np.fft.fftn(x.astype(np.complex128), axes=axes)
    tol = 2e-6 if dtype == np.complex64 else 1e-13
    assert np.linalg.norm(yt.cpu().numpy() - ref) <= tol * np.linalg.norm(ref)
    zt = torch.empty_like(xt)
    nat.call('mmx_fftn', plan.handle, _ptr(yt), _ptr(zt), nb, 1, _stream())
    assert np.linalg.norm(zt.cpu().numpy() - x) <= tol * np.linalg.norm(x)
    # in place
    nat.call('mmx_fftn', plan.handle, _ptr(xt), _ptr(xt), nb, 1, _stream())
    ref_i = np.fft.ifftn(x.astype(np.complex128), axes=axes)
    assert np.linalg.norm(xt.cpu().numpy() - ref_i) <= tol * np.linalg.norm(ref_i)
    plan.close()


def test_fft_delta_is_flat():
    """test_backend.py:162-169 known answer: the transform of a unit delta at the origin is all ones."""
    import torch
    from macromax_b200 import _native as nat
    shape = (5, 10, 20)
    x = np.zeros((9, *shape), dtype=np.complex128)
    x[:, 0, 0, 0] = 1
    plan = nat.Plan(shape, 1, 1, nat.MMX_C128)
    xt = torch.from_numpy(x).cuda()
    nat.call('mmx_fftn', plan.handle, _ptr(xt), _ptr(xt), 9, 0, _stream())
    np.testing.assert_array_almost_equal(xt.cpu().numpy(), np.ones((9, *shape)), decimal=14)
    nat.call('mmx_fftn', plan.handle, _ptr(xt), _ptr(xt), 9, 1, _stream())
    np.testing.assert_array_almost_equal(xt.cpu().numpy(), x, decimal=14)


@pytest.mark.parametrize('n', [0, 1, 1000, 1 << 20])
@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_norm(n, dtype):
    import torch
    from macromax_b200 import _native as nat
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(max(n, 1)) + 1j * rng.standard_normal(max(n, 1))).astype(dtype)[:n]
    plan = nat.Plan((8,), 1, 1, nat.MMX_C64)
    xt = torch.from_numpy(x).cuda() if n else torch.zeros(1, dtype=torch.complex64, device='cuda')
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    prec = nat.MMX_C64 if dtype == np.complex64 else nat.MMX_C128
    nat.call('mmx_norm', plan.handle, _ptr(xt), n, prec, _ptr(out), _stream())
    assert np.isclose(out.item(), np.linalg.norm(x.astype(np.complex128)), rtol=1e-12, atol=0)


def test_pointwise_mul_matches_oracle():
    import torch
    from conftest import load_golden
    from macromax_b200 import _native as nat
    z = load_golden('backend_ops')
    chi, x = z['chi'], z['x']
    nvox = int(np.prod(chi.shape[2:]))
    A = torch.from_numpy(np.ascontiguousarray(chi.reshape(3, 3, nvox))).cuda()
    B = torch.from_numpy(np.ascontiguousarray(x.reshape(3, 1, nvox))).cuda()
    out = torch.empty((3, 1, nvox), dtype=torch.complex128, device='cuda')
    nat.call('mmx_pointwise_mul', _ptr(A), 3, 3, _ptr(B), 1, 0, _ptr(out), nvox, nat.MMX_C128, _stream())
    ref = z['mul'].reshape(3, 1, nvox)
    assert np.linalg.norm(out.cpu().numpy() - ref) <= 1e-13 * np.linalg.norm(ref)
