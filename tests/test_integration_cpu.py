"""
Integration with the reference package (CPU, where the reference tree is present): the 'b200' backend type
registers into the reference's ``backend.load`` and, without a GPU, falls through to the next configured backend
exactly like the reference's own types; host-side conventions agree with the reference's classes.
"""
import numpy as np
import pytest



def _reference():
    from oracle.refimport import import_reference, reference_available
    if not reference_available():
        pytest.skip('reference package not present on this machine')
    return import_reference()


def test_b200_type_falls_through_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip('fall-through is observed on a machine without a GPU')
    mm = _reference()
    from macromax_b200.backend import register
    register(mm)
    from macromax.backend.numpy import BackEndNumpy
    grid = mm.Grid([8, 8], 1.0)
    be = mm.backend.load(1, grid, np.complex128, [{'type': 'b200'}, {'type': 'numpy'}])
    assert isinstance(be, BackEndNumpy)


def test_reference_solution_runs_with_registered_load():
    """The patched load keeps the reference solver working end to end (numpy chosen after 'b200' falls through)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('needs a machine without a GPU')
    mm = _reference()
    from macromax_b200.backend import register
    register(mm)
    mm.backend.config({'type': 'b200'}, {'type': 'numpy'})
    try:
        x = np.arange(64) * 0.1
        sol = mm.solve(x, vacuum_wavelength=1.0, source_distribution=np.exp(-((x - 3.2) / 0.3) ** 2)[None],
                       epsilon=1.5 + 0.05j, callback=lambda s: s.iteration < 5)
        assert sol.iteration == 5
    finally:
        mm.backend.config({'type': 'numpy'})


def test_grid_and_bound_conventions_match_reference():
    mm = _reference()
    from macromax.bound import LinearBound as RefLinearBound
    from macromax_b200 import Grid, LinearBound
    g_ref = mm.Grid([12, 20], [0.25, 0.5])
    g = Grid(shape=(12, 20), step=(0.25, 0.5))
    for a, b in zip(g.k, g_ref.k):
        assert np.allclose(np.broadcast_to(a, np.broadcast_shapes(a.shape, b.shape)),
                           np.broadcast_to(b, np.broadcast_shapes(a.shape, b.shape)), rtol=1e-14, atol=1e-14)
    for a, b in zip(g, g_ref):
        assert np.allclose(a, b)
    kb = LinearBound(g, thickness=1.0, max_extinction_coefficient=0.3).electric_susceptibility
    kr = RefLinearBound(g_ref, thickness=1.0, max_extinction_coefficient=0.3).electric_susceptibility
    assert np.allclose(np.broadcast_to(kb, g.shape), np.broadcast_to(kr, g.shape), rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize('thickness, kmax, bg', [
    (1.0, 0.3, 1.0),
    ([[0.5, 1.25], [0.0, 2.0], [1.0, 0.0]], [[0.1, 0.2], [0.3, 0.4], [0.5, 0.6]], 2.25),
    ([[0.0], [1.5], [0.0]], 0.25, 1.0 + 0.1j),
    (0.0, 0.25, 1.0),
])
def test_bounds_match_reference_3d(thickness, kmax, bg):
    """Extinction, susceptibility, between/beyond and thickness of the bounds equal the reference classes'
    (bound.py:55-215) on a 3D grid with per-(axis, side) thicknesses and peaks, including axes without layers."""
    mm = _reference()
    from macromax import bound as rb
    from macromax_b200 import AbsorbingBound, Bound, Grid, LinearBound
    g_ref = mm.Grid([10, 16, 12], [0.25, 0.5, 0.125])
    g = Grid(shape=(10, 16, 12), step=(0.25, 0.5, 0.125))
    ours, ref = LinearBound(g, thickness, kmax, bg), rb.LinearBound(g_ref, thickness, kmax, bg)
    assert np.array_equal(ours.thickness, ref.thickness)
    k_o, k_r = np.asarray(ours.extinction), np.asarray(ref.extinction)
    assert k_o.shape == k_r.shape
    assert np.allclose(k_o, k_r, rtol=1e-14, atol=1e-15)
    assert np.allclose(ours.electric_susceptibility, ref.electric_susceptibility, rtol=1e-14, atol=1e-15)
    assert np.array_equal(np.broadcast_to(ours.between, g.shape), np.broadcast_to(ref.between, g.shape))
    assert np.array_equal(np.broadcast_to(ours.beyond, g.shape), np.broadcast_to(ref.beyond, g.shape))
    fn = (lambda r: r ** 2)
    a_o, a_r = AbsorbingBound(g, thickness, fn, bg), rb.AbsorbingBound(g_ref, thickness, fn, bg)
    assert np.allclose(a_o.extinction, a_r.extinction, rtol=1e-14, atol=1e-15)
    assert np.array_equal(Bound(g, thickness).thickness, rb.Bound(g_ref, thickness).thickness)


def test_solver_accepts_reference_bound_objects():
    """The reference's own bound objects count as electric bounds here (duck typing on the mixin)."""
    mm = _reference()
    from macromax import bound as rb
    from macromax_b200.bound import is_electric, is_magnetic
    g_ref = mm.Grid([8, 8], 0.25)
    assert is_electric(rb.LinearBound(g_ref, 0.5)) and not is_electric(rb.Bound(g_ref, 0.5))
    assert not is_magnetic(rb.LinearBound(g_ref, 0.5))


def test_hooked_reference_solution_is_unchanged_on_other_backends():
    """With the fused-iteration hook installed, a reference Solution on the NumPy backend runs the reference's own
    iteration: its residues equal the fixture the reference made (to rounding: 1e-13)."""
    from conftest import load_golden
    mm = _reference()
    from macromax_b200.backend import register
    register(mm)
    assert getattr(mm.solver.Solution, '_b200_hooked', False)
    mm.backend.config({'type': 'numpy'})
    z = load_golden('disks2d_64_c128')
    grid = mm.Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    sol = mm.Solution(grid, vacuum_wavelength=float(z['wavelength']), epsilon=z['epsilon'],
                      source_distribution=z['source'], bound=mm.bound.Bound(grid, thickness=float(z['bound_thickness'])),
                      dtype=np.complex128)
    residues = []
    for s in sol:
        residues.append(s.residue)
        if s.iteration >= 30:
            break
    np.testing.assert_allclose(residues, z["residues"][:30], rtol=1e-13)
    sol.solve(None, rtol=0, maxiter=7)
    assert sol.iteration == 7  # the reference resets the count on every solve (solver.py:1063)


def test_stop_rule_recognition():
    """The hook runs on the device only the stop rules of the form iteration < maxiter and residue > rtol: the
    reference's default callbacks and the closure macromax.solve(callback=None) builds; other callbacks run per
    iteration on the host."""
    mm = _reference()
    from macromax_b200 import refhook
    defaults = (mm.solver.Solution.solve.__defaults__[0] if not getattr(mm.solver.Solution, '_b200_hooked', False)
                else mm.solver.Solution._b200_reference_solve.__defaults__[0],)
    assert refhook._stop_rule(None, mm, defaults) is None
    assert refhook._stop_rule(defaults[0], mm, defaults) == (1e-4, 1e4)
    assert refhook._stop_rule(lambda s: s.iteration < 3, mm, defaults) is False
    captured = {}

    class Stop(Exception):
        pass

    def fake_solve(self, callback):
        captured['cb'] = callback
        raise Stop

    orig = mm.solver.Solution.solve
    try:
        mm.solver.Solution.solve = fake_solve
        with pytest.raises(Stop):
            mm.solve(np.arange(8) * 0.1, vacuum_wavelength=1.0, source_distribution=np.ones((1, 8)), epsilon=1.0,
                     callback=None, rtol=1e-7, maxiter=123)
    finally:
        mm.solver.Solution.solve = orig
    assert refhook._stop_rule(captured['cb'], mm, defaults) == (1e-7, 123.0)
