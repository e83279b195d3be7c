"""
The reference package's own API on the B200 kernels: ``macromax.backend.config(type='b200')`` followed by the
reference's ``Solution`` / ``macromax.solve`` (solver.py:1049-1123), with the iteration routed to the fused kernels
by ``macromax_b200.backend.register`` (``refhook``).

- The reference Solution's iterates on 'b200' equal the reference NumPy backend's (the golden fixtures made by the
  reference itself) within 1e-10 relative L2 in complex128, with the same iteration count, rejections and final
  alpha; the per-iteration ``__iter__`` path and the device-chunked ``solve`` path both.
- They equal this library's own ``Solution`` mirror on the same inputs.
- The fused path is the one that ran (the engine's iteration counter).
- ``BackEndB200`` passes the reference's backend conformance suite ``BaseTestBackEnd``
  (python/tests/test_backend.py:11-398), as the reference's torch backend does.

The reference package is read from ``baseline/_ref`` (or ``$MACROMAX_REFERENCE``); without it these tests skip.
"""
import unittest

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

from oracle.refimport import (import_reference, load_reference_test_module, reference_available,  # noqa: E402
                              reference_tests_dir)


def _mm():
    if not reference_available():
        pytest.skip('the reference package is not present')
    mm = import_reference()
    from macromax_b200.backend import register
    register(mm)
    mm.backend.config({'type': 'b200'})
    return mm


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _reference_solution(mm, z, dtype):
    grid = mm.Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    bound = mm.bound.Bound(grid, thickness=float(z['bound_thickness']))
    return mm.Solution(grid, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'],
                       source_distribution=z['source'], bound=bound, dtype=dtype)


@pytest.mark.parametrize('name', ['disks2d_64_c128', 'spheres3d_20_c128', 'gain2d_48_c128', 'voronoi3d_16_c128'])
def test_reference_solution_iterates_on_b200(name):
    mm = _mm()
    from macromax_b200 import refhook
    z = load_golden(name)
    sol = _reference_solution(mm, z, np.complex128)
    assert isinstance(sol._Solution__BE, refhook.backend_class(mm))
    assert abs(complex(sol._Solution__alpha) - complex(z['alpha0'])) <= 1e-12 * abs(complex(z['alpha0']))
    record = tuple(int(i) for i in z['record'])
    residues, fields = [], {}
    for s in sol:
        residues.append(s.residue)
        if s.iteration in record:
            fields[s.iteration] = s.E
        if not (s.iteration < int(z['maxiter']) and s.residue > float(z['rtol'])):
            break
    assert sol.iteration == int(z['iterations'])
    for it in record:
        assert rel(fields[it], z[f'E_{it}']) < 1e-10, it
    assert rel(sol.E, z['final']) < 1e-10
    # the set-up ran through the torch backend on the device, the fixture's through numpy: residues to 1e-8
    np.testing.assert_allclose(residues, z['residues'], rtol=1e-8)
    assert complex(sol._Solution__alpha) == pytest.approx(complex(z['alphas'][-1]), rel=1e-12)
    assert sol.__dict__['_b200_runner'].iterations == sol.iteration  # every iteration ran on the fused kernels


@pytest.mark.parametrize('name', ['disks2d_64_c128', 'gain2d_48_c128'])
def test_reference_solve_function_runs_in_device_chunks(name):
    """macromax.solve(..., callback=None, rtol, maxiter): the stop rule runs on the device; the same iteration count
    and field as the reference NumPy backend, and as this library's own Solution."""
    mm = _mm()
    from macromax_b200 import Bound, Grid, Solution
    z = load_golden(name)
    grid = mm.Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    sol = mm.solve(grid, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'],
                   source_distribution=z['source'], bound=mm.bound.Bound(grid, thickness=float(z['bound_thickness'])),
                   dtype=np.complex128, callback=None, rtol=float(z['rtol']), maxiter=int(z['maxiter']))
    assert sol.iteration == int(z['iterations'])
    assert rel(sol.E, z['final']) < 1e-10
    runner = sol.__dict__['_b200_runner']
    assert runner.iterations == sol.iteration
    g = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    own = Solution(g, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'], source_distribution=z['source'],
                   bound=Bound(g, thickness=float(z['bound_thickness'])), dtype=np.complex128)
    own.solve(None, rtol=float(z['rtol']), maxiter=int(z['maxiter']))
    assert own.iteration == sol.iteration
    assert rel(sol.E, own.E) < 1e-12


def test_reference_solution_picks_up_a_new_field_and_the_default_callback():
    """The E setter between solves resets the update norm (solver.py:824-832); the reference's default callback
    (iteration < 1e4 and residue > 1e-4) runs on the device; complex64."""
    mm = _mm()
    z = load_golden('disks2d_64_c128')
    sol = _reference_solution(mm, z, np.complex64)
    sol.solve()
    first, E1 = sol.iteration, sol.E
    assert 0 < first < 1e4 and sol.residue <= 1e-4
    assert rel(E1, z['final']) < 0.1  # the fixture ran to residue 1e-6
    sol.E = np.zeros_like(sol.E)
    assert sol.previous_update_norm == np.inf
    sol.solve()
    assert sol.iteration == first
    assert rel(sol.E, E1) < 1e-6


def _conformance_names():
    if not reference_available() or reference_tests_dir() is None:
        return []
    try:
        mod = load_reference_test_module('test_backend')
    except Exception:  # pragma: no cover - a reference without its test suite
        return []
    return unittest.defaultTestLoader.getTestCaseNames(mod.BaseTestBackEnd)


@pytest.mark.parametrize('method', _conformance_names())
def test_reference_backend_conformance_suite(method):
    import torch
    mm = _mm()
    from macromax_b200 import refhook
    mod = load_reference_test_module('test_backend')
    cls = refhook.backend_class(mm)

    class TestBackEndB200(mod.BaseTestBackEnd):
        def __init__(self, *args, **kwargs):
            super().__init__(*args, dtype=np.complex64, hardware_dtype=torch.complex64, **kwargs)
            self.BE = cls(self.nb_pol_dims, self.grid * self.wavenumber, hardware_dtype=self.hardware_dtype)

    result = unittest.TestResult()
    TestBackEndB200(method).run(result)
    problems = result.failures + result.errors
    assert not problems, problems[0][1]


@pytest.mark.parametrize('name', ['magnetic2d_48_c128', 'chiral3d_16_c128'])
def test_reference_magnetic_solution_iterates_on_b200(name):
    """Magnetic and bi-(an)isotropic media through the reference's own Solution on 'b200': the iteration runs on
    mmx_magnetic_iterate with the reference's stored blocks; iterates within 1e-10 of the reference NumPy backend's
    fixtures, and the final alpha."""
    mm = _mm()
    z = load_golden(name)
    grid = mm.Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    sol = mm.Solution(grid, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'], xi=z['xi'],
                      zeta=z['zeta'], mu=z['mu'], source_distribution=z['source'],
                      bound=mm.bound.Bound(grid, thickness=float(z['bound_thickness'])), dtype=np.complex128)
    assert sol.magnetic
    assert abs(complex(sol._Solution__alpha) - complex(z['alpha0'])) <= 1e-12 * abs(complex(z['alpha0']))
    record = set(int(r) for r in z['record'])
    for s in sol:
        if s.iteration in record:
            assert rel(s.E, z[f'E{s.iteration}']) < 1e-10, s.iteration
        if s.iteration >= max(record):
            break
    assert complex(sol._Solution__alpha) == pytest.approx(complex(z['alpha_final']), rel=1e-12)
    assert sol.__dict__['_b200_runner'].iterations == sol.iteration
