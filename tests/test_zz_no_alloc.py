"""
The allocation-free FFT entry point ``mmx_fftn_noalloc``, called through the C ABI, against the plan-based
``mmx_fftn`` on the same inputs, for two calls in a row.

``mmx_fftn_noalloc`` serves callers that must not let a library allocate or free device memory -- applications
whose buffers all come from their own pool or fixed memory plan, where a side cudaMalloc can fail on a fully
committed GPU and a cudaFree stalls the device.  Its twiddle tables live in a file-scope device array shared by all
calls, so the test also checks that a later call with another shape and precision does not see stale tables, up to
the 4096-sample limit.
This file is collected last (``test_zz``) so that a stop-at-first-failure run has finished every other test first.
"""
import ctypes

import numpy as np
import pytest

from macromax_b200 import _native as nat


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    s = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(s) if s else None


def _shape_arg(shape):
    return (ctypes.c_int64 * len(shape))(*shape)


def _noalloc(shape, x, out, nb, inverse, prec):
    nat.call('mmx_fftn_noalloc', len(shape), _shape_arg(shape), _ptr(x), _ptr(out), nb, inverse, prec, _stream())


def _planned(shape, x, out, nb, inverse, prec):
    plan = nat.Plan(shape, 1, 1, prec)
    nat.call('mmx_fftn', plan.handle, _ptr(x), _ptr(out), nb, inverse, _stream())
    plan.close()


# the FFT tolerance of tests/test_gpu_ops.py: relative L2 2e-6 (complex64), 1e-13 (complex128)
TOL = {np.complex64: 2e-6, np.complex128: 1e-13}


@pytest.mark.gpu
def test_noalloc_fft_matches_planned_fft_on_two_calls():
    import torch
    rng = np.random.default_rng(17)
    # two ordinary calls, then the bound: a 4096-sample axis in the last twiddle slot (complex128, the largest
    # words) and a 1-D 4096-sample transform
    calls = [((128, 96, 20), np.complex64, 0), ((30, 64), np.complex128, 1), ((2, 3, 4096), np.complex128, 0),
             ((4096,), np.complex64, 1)]
    for shape, dtype, inverse in calls:
        nb = 2
        x = (rng.standard_normal((nb, *shape)) + 1j * rng.standard_normal((nb, *shape))).astype(dtype)
        prec = nat.MMX_C64 if dtype == np.complex64 else nat.MMX_C128
        xt = torch.from_numpy(x).cuda()
        ref = torch.empty_like(xt)
        got = torch.empty_like(xt)
        _planned(shape, xt, ref, nb, inverse, prec)
        _noalloc(shape, xt, got, nb, inverse, prec)
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.linalg.norm(g - r) <= TOL[dtype] * np.linalg.norm(r), (shape, dtype)


def test_noalloc_fft_rejects_axes_beyond_its_scratch():
    lib = nat.load()
    buf = ctypes.c_void_p(1)
    rc = lib.mmx_fftn_noalloc(1, _shape_arg((8192,)), buf, buf, 1, 0, nat.MMX_C64, None)
    assert rc == -3
    assert b'4096' in lib.mmx_last_error()
