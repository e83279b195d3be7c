"""
Integration with the reference package (CPU, where the reference tree is present): the 'b200' backend type
registers into the reference's ``backend.load`` and, without a GPU, falls through to the next configured backend
exactly like the reference's own types; host-side conventions agree with the reference's classes.
"""
import numpy as np
import pytest



def _reference():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from refimport import import_reference, reference_available
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
