"""The autotuner picks one of the plan's kernel variants, caches it, and leaves the solve unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_picks_variant_and_preserves_solution(tmp_path, monkeypatch):
    from macromax_b200 import Bound, Grid, Solution, autotune, workloads
    monkeypatch.setenv('MACROMAX_B200_TUNE_CACHE', str(tmp_path / 'tune.json'))
    wl = workloads.spheres_3d(n=64, nb_spheres=20)
    grid = Grid(shape=wl['shape'], step=wl['step'])

    def make():
        return Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                        source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                        dtype=np.complex64)

    tuned, plain = make(), make()
    tuned.solve(None, rtol=0, maxiter=5)
    plain.solve(None, rtol=0, maxiter=5)
    res = autotune.tune(tuned._engine, iters=5)
    assert set(res['trials']) >= {'0', '2'}
    assert autotune.get_variant(tuned._engine) == res['variant']
    # the trial iterations did not change the solution state
    assert tuned.iteration == 5
    tuned.solve(None, rtol=0, maxiter=10)
    plain.solve(None, rtol=0, maxiter=10)
    assert np.linalg.norm(tuned.E - plain.E) <= 2e-6 * np.linalg.norm(plain.E)
    # cached: a second problem of the same class reuses the choice without timing
    again = make()
    assert autotune.tune(again._engine)['variant'] == res['variant']
    assert (tmp_path / 'tune.json').exists()


def test_autotune_refuses_an_engine_that_does_not_iterate():
    """Zero sources and fields give a 0 / 0 residue and every trial stops at once: no empty-launch timing is taken
    for a variant choice."""
    import torch
    from macromax_b200 import Bound, Grid, autotune, workloads
    from macromax_b200.batch import BatchSolution
    wl = workloads.spheres_3d(n=32, nb_spheres=8)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bs = BatchSolution(grid, torch.zeros((1, *np.shape(wl['source'])), dtype=torch.complex64, device='cuda'),
                       wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       vacuum_wavelength=wl['wavelength'], dtype=np.complex64)
    with pytest.raises(RuntimeError):
        autotune.tune(bs.engine, iters=4, use_cache=False, candidates=(0, 16))
    bs.close()


def test_mixed_solution_tunes_on_its_own_sources():
    """MixedSolution.tune times the inner variants on the problem's sources, restores the inner sources (zero) and
    state, and the tuned solve reaches the same residue as an untuned one."""
    from macromax_b200 import Bound, Grid, workloads
    from macromax_b200 import _native as nat
    from macromax_b200.mixed import MixedSolution
    wl = workloads.voronoi_3d(n=32, nb_grains=8)
    grid = Grid(shape=wl['shape'], step=wl['step'])

    def make():
        return MixedSolution(grid, wl['source'], wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                             vacuum_wavelength=wl['wavelength'])

    tuned, plain = make(), make()
    st0 = tuned.inner.engine.read_state()
    res = tuned.tune(iters=4, candidates=(0, nat.MMX_VARIANT_FUSED_EPILOGUE))
    assert set(res['trials']) == {'0', '16'} and all(t > 0 for t in res['trials'].values())
    assert not tuned.inner.engine.sources.any()
    st1 = tuned.inner.engine.read_state()
    assert st0.tobytes() == st1.tobytes()
    tuned.solve(rtol=1e-8)
    plain.solve(rtol=1e-8)
    assert tuned.converged.all() and tuned.residues.max() < 1e-8
    assert np.linalg.norm(tuned.E - plain.E) <= 1e-7 * np.linalg.norm(plain.E)
    tuned.close()
    plain.close()
