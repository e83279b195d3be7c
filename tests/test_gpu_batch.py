"""
Batched right-hand sides (one material, B sources, one launch per pass) against B sequential single-source solves
and against the oracle; per-RHS stop rule, alpha and divergence-guard rejections.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _sources(base, B, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(B):
        shift = rng.integers(-6, 7, size=base.ndim - 1)
        s = np.roll(base, tuple(shift), axis=tuple(range(1, base.ndim)))
        out.append(s * np.exp(1j * rng.uniform(0, 2 * np.pi)) * rng.uniform(0.5, 2.0))
    return np.asarray(out)


@pytest.mark.parametrize('dtype,tol', [(np.complex128, 1e-10), (np.complex64, 1e-5)])
def test_batch_matches_sequential_solves(dtype, tol):
    from macromax_b200 import Bound, Grid, Solution
    from macromax_b200.batch import BatchSolution
    z = load_golden('disks2d_64_c128')
    grid = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    bound = Bound(grid, thickness=float(z['bound_thickness']))
    srcs = _sources(z['source'], 4)
    wl = float(z['wavelength'])
    bs = BatchSolution(grid, srcs, z['epsilon'], bound=bound, vacuum_wavelength=wl, dtype=dtype)
    bs.solve(rtol=1e-5, maxiter=300)
    for b in range(4):
        sol = Solution(grid, vacuum_wavelength=wl, epsilon=z['epsilon'], source_distribution=srcs[b], bound=bound,
                       dtype=dtype)
        sol.solve(None, rtol=1e-5, maxiter=300)
        if dtype == np.complex128:
            assert bs.iterations[b] == sol.iteration
        else:
            assert abs(int(bs.iterations[b]) - sol.iteration) <= 2
        assert rel(bs.E[b], sol.E) < tol


def test_batch_matches_oracle_vector():
    from macromax_b200 import Bound, Grid
    from macromax_b200.batch import BatchSolution
    from oracle import mmoracle as mo
    z = load_golden('spheres3d_20_c128')
    grid = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    srcs = _sources(z['source'], 3, seed=1)
    bs = BatchSolution(grid, srcs, z['epsilon'], bound=Bound(grid, thickness=float(z['bound_thickness'])),
                       vacuum_wavelength=float(z['wavelength']), dtype=np.complex128)
    bs.solve(rtol=0, maxiter=25)
    for b in range(3):
        ref = mo.OracleSolution(tuple(z['shape']), float(z['step']), float(z['wavelength']), z['epsilon'], srcs[b],
                                float(z['bound_thickness']), dtype=np.complex128)
        ref.solve(rtol=0, maxiter=25)
        assert rel(bs.E[b], ref.E) < 1e-10


def test_batch_per_rhs_rejections_and_alpha():
    """Sources of the gain medium: every right-hand side bumps alpha on its own schedule, like its own solve."""
    from macromax_b200 import Bound, Grid
    from macromax_b200.batch import BatchSolution
    from oracle import mmoracle as mo
    z = load_golden('gain2d_48_c128')
    grid = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    srcs = _sources(z['source'], 3, seed=2)
    bs = BatchSolution(grid, srcs, z['epsilon'], bound=Bound(grid, thickness=float(z['bound_thickness'])),
                       vacuum_wavelength=float(z['wavelength']), dtype=np.complex128)
    bs.solve(rtol=1e-5, maxiter=200)
    for b in range(3):
        ref = mo.OracleSolution(tuple(z['shape']), float(z['step']), float(z['wavelength']), z['epsilon'], srcs[b],
                                float(z['bound_thickness']), dtype=np.complex128)
        ref.solve(rtol=1e-5, maxiter=200)
        assert int(bs.rejections[b]) == ref.rejections
        assert int(bs.iterations[b]) == ref.iteration
        assert abs(bs.alphas[b] - ref.alpha) <= 1e-12 * abs(ref.alpha)
        assert rel(bs.E[b], ref.E) < 1e-9


def test_batch_fast_path_vector_128():
    """B = 2 vector sources on a 64^3 grid use the specialised kernels; compare with the single-source solves."""
    from macromax_b200 import Bound, Grid, Solution, workloads
    from macromax_b200.batch import BatchSolution
    wl = workloads.spheres_3d(n=64, nb_spheres=30)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    srcs = _sources(wl['source'], 2, seed=3)
    bs = BatchSolution(grid, srcs, wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'])
    bs.solve(rtol=0, maxiter=12)
    for b in range(2):
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'], source_distribution=srcs[b],
                       bound=bound, dtype=np.complex64)
        sol.solve(None, rtol=0, maxiter=12)
        assert rel(bs.E[b], sol.E) < 1e-6


def test_solve_sharded_on_one_rank_is_the_batch_solve():
    """batch.solve_sharded without a process group: one BatchSolution over all sources, the same fields and counts."""
    from macromax_b200 import Bound, Grid
    from macromax_b200.batch import BatchSolution, solve_sharded
    z = load_golden('disks2d_64_c128')
    grid = Grid(shape=tuple(int(s) for s in z['shape']), step=float(z['step']))
    bound = Bound(grid, thickness=float(z['bound_thickness']))
    srcs = _sources(z['source'], 3, seed=4)
    kw = dict(bound=bound, vacuum_wavelength=float(z['wavelength']), dtype=np.complex128)
    out = solve_sharded(grid, srcs, z['epsilon'], rtol=1e-6, maxiter=400, **kw)
    bs = BatchSolution(grid, srcs, z['epsilon'], **kw)
    bs.solve(rtol=1e-6, maxiter=400)
    assert out['iterations'].tolist() == bs.iterations.tolist()
    assert np.array_equal(out['E'], bs.E)
    assert np.allclose(out['residues'], bs.residues, rtol=0, atol=0)
    bs.close()
