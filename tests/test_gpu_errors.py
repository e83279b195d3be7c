"""
Error behaviour of the device path, as the reference behaves or as the C ABI documents it:
- a zero source gives a zero first update, a residue of 0 (solver.py:1037-1039), so a solve stops after it; an
  iteration after that divides a zero update norm by a zero one, which the reference's Solution.__iter__ turns into
  ZeroDivisionError (solver.py:1079): on the electric and the magnetic path alike;
- an axis length with a prime factor above 13 is refused when the plan is made (MMX_ERR_UNSUPPORTED);
- NULL buffers and out-of-range arguments are refused with MMX_ERR_ARG and a message, before any launch.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _disks(n=32):
    from macromax_b200 import workloads
    return workloads.disks_2d(n=n)


def test_zero_source_raises_zero_division_like_the_reference():
    from macromax_b200 import Bound, Grid, Solution
    wl = _disks()
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=np.zeros_like(wl['source']), bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    sol.solve(None, rtol=0, maxiter=5)
    assert sol.iteration == 1 and sol.residue == 0.0
    with pytest.raises(ZeroDivisionError):
        for n, s in enumerate(sol):  # bounded: the second iteration raises
            if n >= 5:
                break


def test_magnetic_zero_source_raises_zero_division():
    from macromax_b200 import Grid, Solution
    grid = Grid(shape=(32, 32), step=125e-9)
    sol = Solution(grid, vacuum_wavelength=500e-9, current_density=np.zeros((3, 32, 32), np.complex64), mu=2.0,
                   dtype=np.complex64)
    sol.solve(None, rtol=0, maxiter=5)
    assert sol.iteration == 1 and sol.residue == 0.0
    with pytest.raises(ZeroDivisionError):
        for n, s in enumerate(sol):  # bounded: the second iteration raises
            if n >= 5:
                break


def test_unsupported_axis_length_is_refused():
    from macromax_b200 import _native as nat
    with pytest.raises(nat.NativeError):
        nat.Plan((17, 32), 1, 1, nat.MMX_C64)


def test_null_and_out_of_range_arguments_are_refused():
    from macromax_b200 import _native as nat
    lib = nat.load()
    plan = nat.Plan((32, 32), 1, 1, nat.MMX_C64)
    null = ctypes.c_void_p(None)
    rc = lib.mmx_iterate(plan.handle, null, null, null, nat.MMX_CHI_SCALAR, null, null, 1, null)
    assert rc == nat.MMX_ERR_ARG and b'NULL' in lib.mmx_last_error()
    rc = lib.mmx_plan_set_variant(plan.handle, 1 << 10)
    assert rc == nat.MMX_ERR_ARG and b'variant' in lib.mmx_last_error()
    rc = lib.mmx_chi_from_eps(null, 9, 10, 1.0, 0.0, 0.0, 0.0, null, nat.MMX_C64, null)
    assert rc == nat.MMX_ERR_ARG
    plan.close()
