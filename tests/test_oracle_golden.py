"""
Pin the numpy oracle (oracle/mmoracle.py) against golden vectors produced by the reference package itself
(tests/golden/make_golden.py): preconditioner constants, iterates, divergence-guard rejections, iteration counts
and converged fields.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import mmoracle as mo

C128_CASES = ['disks2d_64_c128', 'spheres3d_20_c128', 'voronoi3d_16_c128', 'design3d_24_c128', 'gain2d_48_c128']
C64_CASES = ['plane1d_scalar_c64', 'plane1d_vector_c64', 'plane1d_aniso_c64']


def _solve(z, dtype):
    sol = mo.OracleSolution(tuple(z['shape']), float(z['step']), float(z['wavelength']), z['epsilon'], z['source'],
                            float(z['bound_thickness']), dtype=dtype)
    rec = sol.solve(rtol=float(z['rtol']), maxiter=int(z['maxiter']), record=tuple(int(i) for i in z['record']))
    return sol, rec


@pytest.mark.parametrize('name', C128_CASES)
def test_oracle_matches_reference_c128(name):
    z = load_golden(name)
    sol, rec = _solve(z, np.complex128)
    assert sol.beta == float(z['beta'])
    assert abs(complex(z['alphas'][-1]) - sol.alpha) <= 1e-12 * abs(sol.alpha)
    for it in z['record']:
        ref = z[f'E_{it}']
        assert np.linalg.norm(rec[int(it)] - ref) <= 1e-12 * np.linalg.norm(ref), it
    assert sol.iteration == int(z['iterations'])
    assert np.linalg.norm(sol.E - z['final']) <= 1e-11 * np.linalg.norm(z['final'])
    assert sol.rejections == int(np.sum(np.diff(z['alphas']) != 0))


def test_oracle_gain_case_rejects_updates():
    z = load_golden('gain2d_48_c128')
    sol, _ = _solve(z, np.complex128)
    assert sol.rejections > 0
    assert sol.rejections == int(np.sum(np.diff(z['alphas']) != 0))


@pytest.mark.parametrize('name', C64_CASES)
def test_oracle_matches_reference_c64(name):
    """The reference ran in complex64 end to end; the oracle sets up in FP64, so parity is at c64 rounding."""
    z = load_golden(name)
    sol, rec = _solve(z, np.complex64)
    assert abs(complex(z['alpha0']) - complex(sol.alpha)) <= 1e-5 * abs(sol.alpha)
    for it in z['record']:
        ref = z[f'E_{it}']
        assert np.linalg.norm(rec[int(it)] - ref) <= 1e-5 * np.linalg.norm(ref), it
    assert sol.iteration == int(z['iterations'])
    assert np.linalg.norm(sol.E - z['final']) <= 1e-5 * np.linalg.norm(z['final'])


def test_backend_ops_restatement():
    z = load_golden('backend_ops')
    shape = (5, 10, 20)
    ks = mo.k_vectors(shape, [100e-9] * 3, 10e6 / (2 * np.pi) * 2 * np.pi)
    # the reference test uses grid * k0 with k0 = 10e6; k_vectors takes a wavenumber that multiplies the step
    for i in range(3):
        assert np.allclose(np.broadcast_to(ks[i], z[f'k{i}'].shape), z[f'k{i}'].real, rtol=1e-14, atol=0)
    x = z['x']
    assert np.allclose(mo.fftn(x, (2, 3, 4)), z['ft'], rtol=1e-13, atol=1e-12)
    assert np.allclose(mo.ifftn(x, (2, 3, 4)), z['ift'], rtol=1e-13, atol=1e-15)
    assert np.allclose(mo.longitudinal_projection_ft(x, ks, 3), z['longitudinal'], rtol=1e-13, atol=1e-14)
    assert np.allclose(x - mo.longitudinal_projection_ft(x, ks, 3), z['transversal'], rtol=1e-13, atol=1e-14)
    assert np.allclose(mo.curl_ft(x, ks), z['curl_ft'], rtol=1e-13, atol=1e-14)
    assert np.allclose(mo.pointwise_mul(z['chi'], x), z['mul'], rtol=1e-13, atol=1e-14)
    assert np.isclose(np.linalg.norm(x.ravel()), float(z['norm']), rtol=1e-14)


def test_full_size_disks_inputs_match_fixture_checksums():
    from macromax_b200 import workloads
    z = load_golden('disks2d_256_c128')
    wl = workloads.disks_2d(n=256, seed=1)
    eps = wl['epsilon']
    chk = np.sum(np.abs(eps) * np.arange(eps.size).reshape(eps.shape) % 1009)
    assert np.isclose(chk, float(z['epsilon_checksum']), rtol=1e-12)
    assert np.isclose(np.sum(np.abs(wl['source'])), float(z['source_checksum']), rtol=1e-12)


def test_full_size_disks_first_iterate():
    from macromax_b200 import workloads
    z = load_golden('disks2d_256_c128')
    sol = mo.from_workload(workloads.disks_2d(n=256, seed=1), np.complex128)
    assert abs(sol.alpha - complex(z['alpha0'])) <= 1e-12 * abs(sol.alpha)
    rec = sol.solve(rtol=0, maxiter=20, record=(1, 20))
    for it in (1, 20):
        ref = z[f'E_{it}']
        assert np.linalg.norm(rec[it] - ref) <= 1e-6 * np.linalg.norm(ref)


@pytest.mark.parametrize('name', ['magnetic2d_48_c128', 'chiral3d_16_c128'])
def test_magnetic_oracle_matches_reference(name):
    """Magnetic / bi-isotropic media: the restated 2-parameter preconditioner gives the reference's alpha and beta
    exactly, and the iterates (chi_op with spectral curls) agree to 1e-13 (fixtures from make_golden.py)."""
    z = load_golden(name)
    ref = mo.MagneticOracleSolution(tuple(int(s) for s in z['shape']), float(z['step']), float(z['wavelength']),
                                    z['epsilon'], z['source'], xi=z['xi'], zeta=z['zeta'], mu=z['mu'],
                                    bound_thickness=float(z['bound_thickness']))
    assert ref.alpha == complex(z['alpha0']) and ref.beta == float(z['beta'])
    record = tuple(int(r) for r in z['record'])
    rec = ref.solve(rtol=0, maxiter=max(record), record=record)
    for it in record:
        g = z[f'E{it}']
        assert np.linalg.norm(rec[it] - g) <= 1e-13 * np.linalg.norm(g), it
    assert ref.alpha == complex(z['alpha_final'])


@pytest.mark.parametrize('case', ['spheres3d', 'disks2d'])
def test_torch_cpu_form_matches_numpy_oracle(case):
    """The torch-CPU restatement timed beside the numpy oracle (bench.py cpu_baseline) takes the same steps."""
    from macromax_b200 import workloads
    from oracle import mmoracle as mo
    from oracle.torch_cpu import TorchCPUIteration
    wl = workloads.spheres_3d(n=16, nb_spheres=6) if case == 'spheres3d' else workloads.disks_2d(n=32)
    ref = mo.from_workload(wl, np.complex128)
    tc = TorchCPUIteration(mo.from_workload(wl, np.complex128))
    for _ in range(8):
        assert ref.advance() and tc.advance()
        assert np.linalg.norm(tc.E.numpy() - ref.field) <= 1e-12 * np.linalg.norm(ref.field)
