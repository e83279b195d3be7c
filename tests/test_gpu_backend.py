"""
The per-op backend (BackEndB200, the 'b200' entry of the reference's backend.load) against the reference's own
BackEndNumpy outputs on the reference test suite's grid (tests/golden/backend_ops.npz: a 3-vector field on a
5 x 10 x 20 grid, step 100 nm, k0 = 1e7): ft, ift, the longitudinal and transversal projections, the spectral
curl, the 3x3 matrix multiply and the norm, complex128.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _backend():
    from macromax_b200.backend import BackEndB200
    from macromax_b200.grid import Grid
    # the reference's test takes grid * k0 with step 100 nm and k0 = 1e7: a unit step
    return BackEndB200(3, Grid(shape=(5, 10, 20), step=100e-9 * 10e6), np.complex128)


def test_backend_ops_match_reference_numpy_backend():
    z = load_golden('backend_ops')
    be = _backend()
    x = be.astype(z['x'])
    close = lambda a, b, rtol, atol: np.allclose(be.asnumpy(a), b, rtol=rtol, atol=atol)
    assert close(be.ft(x), z['ft'], 1e-13, 1e-12)
    assert close(be.ift(x), z['ift'], 1e-13, 1e-15)
    assert close(be.longitudinal_projection_ft(x), z['longitudinal'], 1e-13, 1e-14)
    assert close(be.transversal_projection_ft(x), z['transversal'], 1e-13, 1e-14)
    assert close(be.curl_ft(x), z['curl_ft'], 1e-13, 1e-14)  # mmx_curl_ft
    assert close(be.mul(be.astype(z['chi']), x), z['mul'], 1e-13, 1e-14)
    assert np.isclose(be.norm(x), float(z['norm']), rtol=1e-14)


def test_backend_ft_round_trip_and_curl_of_gradient():
    """ift(ft(x)) == x, and the curl of a gradient field i k phi is zero (backend test known answers)."""
    be = _backend()
    rng = np.random.default_rng(4)
    x = be.astype(rng.standard_normal((3, 1, 5, 10, 20)) + 1j * rng.standard_normal((3, 1, 5, 10, 20)))
    assert np.allclose(be.asnumpy(be.ift(be.ft(x))), be.asnumpy(x), rtol=1e-13, atol=1e-14)
    phi = be.astype(rng.standard_normal((5, 10, 20)) + 0j)
    grad = be.astype(np.stack([1j * be.asnumpy(k) * be.asnumpy(phi) for k in be.k])[:, None])
    assert np.abs(be.asnumpy(be.curl_ft(grad))).max() < 1e-12 * np.abs(be.asnumpy(grad)).max()
