"""
Magnetic and bi-(an)isotropic media (macromax_b200/magnetic.py: the reference's magnetic preconditioner and chi_op
with spectral curls, composed of device kernels) against the reference: its iterates on a negative-index plate and a
chiral sphere (tests/golden/magnetic2d_48_c128.npz, chiral3d_16_c128.npz) and the known answer of the reference test
suite's magnetic solve (tests/test_solution.py:360-411).
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _solution(z, dtype):
    from macromax_b200 import Bound, Grid, Solution
    from macromax_b200.magnetic import MagneticSolution
    grid = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    sol = Solution(grid, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'], xi=z['xi'], zeta=z['zeta'],
                   mu=z['mu'], source_distribution=z['source'], bound=Bound(grid, thickness=float(z['bound_thickness'])),
                   dtype=dtype)
    assert isinstance(sol, MagneticSolution) and sol.magnetic
    return sol


@pytest.mark.parametrize('fused', [False, True])
@pytest.mark.parametrize('name', ['magnetic2d_48_c128', 'chiral3d_16_c128'])
def test_magnetic_iterates_match_reference(name, fused, monkeypatch):
    if fused:
        monkeypatch.setenv('MMX_MAG_FUSED', '1')
    z = load_golden(name)
    sol = _solution(z, np.complex128)
    assert abs(sol.alpha - complex(z['alpha0'])) <= 1e-12 * abs(complex(z['alpha0']))
    assert abs(sol.beta - float(z['beta'])) <= 1e-12 * abs(float(z['beta']))
    record = set(int(r) for r in z['record'])
    for s in sol:
        if s.iteration in record:
            assert rel(s.E, z[f'E{s.iteration}']) < 1e-10, s.iteration
        if s.iteration >= max(record):
            break
    assert abs(sol.alpha - complex(z['alpha_final'])) <= 1e-12 * abs(complex(z['alpha_final']))


def test_magnetic_complex64():
    z = load_golden('chiral3d_16_c128')
    sol = _solution(z, np.complex64)
    for s in sol:
        if s.iteration == 5:
            assert rel(s.E, z['E5']) < 1e-4
            break


@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_device_stop_rule_equals_per_iteration_loop(dtype):
    """solve() with a tolerance runs chunks of iterations with the stop rule on the device (the chunks may pass the
    stopping iteration: those iterations leave E and the state unchanged).  It stops at the same iteration as the
    Python callback loop, with the same field, alpha and rejections."""
    z = load_golden('magnetic2d_48_c128')
    a, b = _solution(z, dtype), _solution(z, dtype)
    rtol = 1e-3
    a.solve(None, rtol=rtol, maxiter=1e4)
    b.solve(lambda s: s.iteration < 1e4 and s.residue > rtol)
    assert a.iteration == b.iteration and a.residue <= rtol < 1.0
    assert a.rejections == b.rejections and a.alpha == b.alpha
    assert np.array_equal(a.E, b.E)


def test_reference_negative_index_plate_known_answer():
    """The reference's magnetic solve: a -1.5 index plate, 128^2 grid, complex64, to residue 1e-3 in at most 1000
    iterations, with the field norms in front of and behind the plate that its test asserts to 5 decimals."""
    from macromax_b200 import Grid, LinearBound, solve
    wavelength = 500e-9
    boundary_thickness = 2e-6
    beam_diameter = 5e-6
    plate_thickness = 5e-6
    k0 = 2 * np.pi / wavelength
    grid = Grid(shape=(128, 128), step=wavelength / 4)
    angle = 30 * np.pi / 180

    def rot_z(a):
        return np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])

    incident_k = rot_z(angle) * k0 @ np.array([1, 0, 0])
    polarisation = (rot_z(angle) @ np.array([0, 1, 1j]) / np.sqrt(2))[:, np.newaxis, np.newaxis]
    current = np.exp(1j * (incident_k[0] * grid[0] + incident_k[1] * grid[1]))
    source_pixel = grid.shape[0] - int(boundary_thickness / grid.step[0])
    current[:source_pixel, :] = 0
    current[source_pixel + 1:, :] = 0
    current = current * np.exp(-0.5 * ((grid[1] - grid[1].ravel()[grid.shape[0] // 3]) / (beam_diameter / 2)) ** 2)
    current = current[np.newaxis, ...] * polarisation
    n = 1 + (-1.5 - 1) * np.ones(grid[1].shape) * (np.abs(grid[0]) < plate_thickness / 2)
    bound = LinearBound(grid, thickness=boundary_thickness, max_extinction_coefficient=0.50)
    sol = solve(grid, vacuum_wavelength=wavelength, current_density=current, refractive_index=n, bound=bound,
                callback=lambda s: s.iteration < 1e4 and s.residue > 1e-3, dtype=np.complex64)
    assert sol.residue < 1e-3 and sol.iteration <= 1000
    E = sol.E
    front = E[:, source_pixel + 1:source_pixel + 8, :]
    back = E[:, -source_pixel - 8:-source_pixel - 1, :]
    assert abs(np.linalg.norm(back.ravel()) - 0.0001864) < 1.5e-5  # numpy decimal=5, as in the reference test
    assert abs(np.linalg.norm(front.ravel()) - 0.0002582) < 1.5e-5
    assert E.dtype == np.complex64


def test_magnetic_building_blocks_match_numpy():
    """The per-op entry points behind BackEnd.curl and the magnetic chi_op (mmx_curl_ft, mmx_green_ft, mmx_chi_mix,
    mmx_axpby) against numpy restatements (the oracle's curl_ft and longitudinal projection), complex128."""
    import ctypes
    import torch
    from macromax_b200 import _native as nat
    from oracle import mmoracle as mo
    shape, step, k0 = (6, 10, 8), 0.3, 1.7
    ndim, N = len(shape), int(np.prod(shape))
    rng = np.random.default_rng(9)
    cplx = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    ks = mo.k_vectors(shape, (step,) * ndim, k0)
    plan = nat.Plan(shape, 1, 1, nat.MMX_C128)
    plan.set_kvectors([np.asarray(k, dtype=np.float64).ravel() for k in ks])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).cuda()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    F = cplx(3, *shape)
    Ft, out = dev(F.reshape(3, N)), dev(np.zeros((3, N)))
    nat.call('mmx_curl_ft', plan.handle, nat.device_ptr(Ft), nat.device_ptr(out), s)
    ref = mo.curl_ft(F, ks)
    assert rel(out.cpu().numpy().reshape(ref.shape), ref) < 1e-14
    alpha = 1.3 + 0.4j
    nat.call('mmx_green_ft', plan.handle, nat.device_ptr(Ft), alpha.real, alpha.imag, s)
    pl = mo.longitudinal_projection_ft(F[:, None], ks, ndim)[:, 0]
    g = -1j * alpha.imag / (mo.k2_field(ks) - alpha)
    ref = g * (F - pl) + (1j * alpha.imag / alpha) * pl
    assert rel(Ft.cpu().numpy().reshape(ref.shape), ref) < 1e-13
    x, d = cplx(3, N), cplx(3, N)
    blocks = [cplx(3, 3, N) for _ in range(4)]  # EE, EH, HE, HH
    coef = [0.8 + 0.1j, 0.2 - 0.3j, 1.1 + 0.0j, 0.9 - 0.2j, 0.7 + 0.4j]
    u, w = dev(np.zeros((3, N))), dev(np.zeros((3, N)))
    bt = [dev(bk.reshape(9, N)) for bk in blocks]
    cvals = (ctypes.c_double * 10)(*[v for c in coef for v in (c.real, c.imag)])
    xt, dt = dev(x), dev(d)  # kept alive: a temporary's memory would be reused by the next allocation
    nat.call('mmx_chi_mix', nat.device_ptr(xt), nat.device_ptr(dt), *[nat.device_ptr(t) for t in bt], cvals,
             nat.device_ptr(u), nat.device_ptr(w), N, nat.MMX_C128, s)
    mv = lambda m, v: np.einsum('rsn,sn->rn', m, v)
    ref_u = coef[0] * mv(blocks[0], x) + coef[1] * x + coef[3] * mv(blocks[2], d)
    ref_w = coef[2] * mv(blocks[1], x) + coef[4] * mv(blocks[3], d)
    assert rel(u.cpu().numpy(), ref_u) < 1e-14 and rel(w.cpu().numpy(), ref_w) < 1e-14
    o = dev(np.zeros((3, N)))
    nat.call('mmx_axpby', nat.device_ptr(o), nat.device_ptr(xt), nat.device_ptr(dt), 0.5, -1.0, 2.0, 0.25,
             3 * N, nat.MMX_C128, s)
    assert rel(o.cpu().numpy(), (0.5 - 1j) * x + (2 + 0.25j) * d) < 1e-15
    plan.close()


@pytest.mark.parametrize('name, dtype, tol', [('magnetic2d_48_c128', np.complex128, 1e-12),
                                             ('chiral3d_16_c128', np.complex128, 1e-12),
                                             ('chiral3d_16_c128', np.complex64, 2e-5)])
def test_fused_passes_equal_the_eight_transform_composition(name, dtype, tol, monkeypatch):
    """The fused pass schedule (MMX_MAG_FUSED=1, k_mag_pass: block products, spectral curls and the Green multiply
    inside the FFT passes; 7 passes per 2D iteration, 13 per 3D one) against the default composition of eight batched
    transforms and pointwise kernels: the same iterates, rejections and alpha after 25 iterations."""
    z = load_golden(name)
    monkeypatch.setenv('MMX_MAG_FUSED', '1')
    a = _solution(z, dtype)
    a.solve(None, rtol=0, maxiter=25)
    monkeypatch.delenv('MMX_MAG_FUSED')
    b = _solution(z, dtype)
    b.solve(None, rtol=0, maxiter=25)
    assert a.iteration == b.iteration == 25
    assert a.rejections == b.rejections and a.alpha == pytest.approx(b.alpha, rel=1e-14)
    assert rel(a.E, b.E) < tol
