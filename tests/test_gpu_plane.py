"""
Plane passes (k_plane_pass: both inner axes of a 3D grid with 128 x 128 planes in one kernel, one plane per 2-CTA
cluster) against the 5-pass schedule of the same plan and against the numpy oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _slab(kind):
    """A 64 x 128 x 128 slice of a 128^3 workload (axis 0 shortened; the plane axes keep their 128 samples)."""
    from macromax_b200 import workloads
    wl = workloads.spheres_3d(n=128, nb_spheres=120) if kind == 'vector' else workloads.design_3d(n=128)
    wl = dict(wl)
    wl['epsilon'] = np.ascontiguousarray(wl['epsilon'][32:96])
    src = np.asarray(wl['source'])
    wl['source'] = np.ascontiguousarray(src[:, 32:96])
    wl['shape'] = (64, 128, 128)
    return wl


def _solution(wl, plane, batch_sources=None):
    from macromax_b200 import Bound, Grid, Solution, autotune
    from macromax_b200 import _native as nat
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    if batch_sources is not None:
        from macromax_b200.batch import BatchSolution
        sol = BatchSolution(grid, batch_sources, wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'],
                            dtype=np.complex64)
        eng = sol.engine if hasattr(sol, 'engine') else sol._engine
    else:
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'], bound=bound, dtype=np.complex64)
        eng = sol._engine
    autotune.set_variant(eng, nat.MMX_VARIANT_PLANE if plane else 0)
    assert autotune.get_variant(eng) == (nat.MMX_VARIANT_PLANE if plane else 0)
    return sol


@pytest.mark.parametrize('kind', ['vector', 'scalar'])
def test_plane_matches_five_pass_schedule(kind):
    wl = _slab(kind)
    a = _solution(wl, plane=True)
    b = _solution(wl, plane=False)
    a.solve(None, rtol=0, maxiter=15)
    b.solve(None, rtol=0, maxiter=15)
    assert a.iteration == b.iteration == 15
    assert rel(a.E, b.E) < 2e-6
    assert abs(a.residue - b.residue) <= 1e-5 * b.residue


def test_plane_matches_oracle_vector():
    from oracle import mmoracle as mo
    wl = _slab('vector')
    sol = _solution(wl, plane=True)
    ref = mo.from_workload(wl, np.complex128)
    rec = ref.solve(rtol=0, maxiter=20, record=(1, 5, 20))
    fields = {}
    for s in sol:
        if s.iteration in (1, 5, 20):
            fields[s.iteration] = s.E
        if s.iteration >= 20:
            break
    for it in (1, 5, 20):
        assert rel(fields[it], rec[it]) < 1e-5, (it, rel(fields[it], rec[it]))


def test_plane_batched_sources_match_five_pass():
    wl = _slab('scalar')
    base = np.asarray(wl['source'])
    srcs = np.stack([base, np.roll(base, 9, axis=2) * (0.5 - 0.7j), np.roll(base, -5, axis=1) * 1.3])
    a = _solution(wl, plane=True, batch_sources=srcs)
    b = _solution(wl, plane=False, batch_sources=srcs)
    a.solve(rtol=0, maxiter=12)
    b.solve(rtol=0, maxiter=12)
    assert np.array_equal(a.iterations, b.iterations)
    for k in range(3):
        assert rel(a.E[k], b.E[k]) < 2e-6
