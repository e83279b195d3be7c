"""
Parity of the kernels that carry the benchmarked workloads with the complex128 numpy oracle, at the sizes that
select them.

- 3D vector 128^3 (the bench's default workload, 200 spheres, isotropic chi): the plain pass schedule (variant 0:
  k_regc_pass prologue / epilogue on 128-sample rows, k_reg_pass on the two strided axes, the axis-0 pass with the
  Green function) and the fused epilogue (variant 16: k_regc_epro, the epilogue fused with the next prologue).
- 3D anisotropic (symmetric 3x3 chi, six stored entries) with 192-sample axes: the register-staged strided passes
  (k_reg_pass on 192-sample vector pencils, radix order 8 x 8 x 3, axis-0 Green stage 3 x 8 x 8) and the
  register-staged 3x3-chi prologue / epilogue on 192-sample rows (k_regc_aniso_pass).

Tolerance: 1e-5 relative L2 against the complex128 oracle after 1, 5 and 20 iterations (the specification's bound
for complex64 iterates).  The oracle follows the reference NumPy backend (solver.py:1049-1098).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RECORD = (1, 5, 20)


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _oracle_fields(wl, record=RECORD):
    from oracle import mmoracle as mo
    mo.set_fft_workers(os.cpu_count() or 1)
    ref = mo.from_workload(wl, np.complex128)
    return ref.alpha, ref.solve(rtol=0, maxiter=max(record), record=record)


def _device_fields(wl, variant, record=RECORD):
    from macromax_b200 import Bound, Grid, Solution, autotune
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    if variant is not None:
        autotune.set_variant(sol._engine, variant)
        assert autotune.get_variant(sol._engine) == variant
    fields = {}
    for s in sol:
        if s.iteration in record:
            fields[s.iteration] = s.E
        if s.iteration >= max(record):
            break
    alpha = sol.alpha
    st = sol._engine.read_state()
    assert int(st['status'][0]) == 0
    sol._engine.close()
    return alpha, fields


@pytest.fixture(scope='module')
def spheres128():
    from macromax_b200 import workloads
    wl = workloads.spheres_3d(n=128)
    return wl, _oracle_fields(wl)


@pytest.mark.parametrize('variant', [0, 16])
def test_spheres3d_128_vector_matches_oracle(spheres128, variant):
    """The bench's default workload on the kernel variants the autotuner chooses between (0 and 16)."""
    wl, (alpha_ref, ref) = spheres128
    alpha, fields = _device_fields(wl, variant)
    assert abs(alpha - alpha_ref) <= 1e-9 * abs(alpha_ref)
    for it in RECORD:
        assert rel(fields[it], ref[it]) < 1e-5, (variant, it, rel(fields[it], ref[it]))


def _stacked_voronoi(axis):
    """The 64^3 Voronoi medium repeated three times along one grid axis (192 samples there)."""
    from macromax_b200 import workloads as w
    wl = w.voronoi_3d(n=64, nb_grains=12, boundary_px=48)
    eps = np.concatenate([wl['epsilon']] * 3, axis=2 + axis)
    src = np.concatenate([wl['source']] + [np.zeros_like(wl['source'])] * 2, axis=1 + axis)
    shape = list(wl['shape'])
    shape[axis] *= 3
    return {**wl, 'shape': tuple(shape), 'epsilon': eps, 'source': src}


@pytest.mark.parametrize('axis', [0, 2])
def test_anisotropic_192_axis_matches_oracle(axis):
    """192 samples on axis 0 (strided passes and the axis-0 Green stage) or axis 2 (the 3x3-chi prologue and
    epilogue on 192-sample rows)."""
    wl = _stacked_voronoi(axis)
    alpha_ref, ref = _oracle_fields(wl)
    alpha, fields = _device_fields(wl, None)
    assert abs(alpha - alpha_ref) <= 1e-9 * abs(alpha_ref)
    for it in RECORD:
        assert rel(fields[it], ref[it]) < 1e-5, (axis, it, rel(fields[it], ref[it]))

