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
