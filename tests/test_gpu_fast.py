"""
The compile-time specialised pass kernels (complex64, axis lengths 64..512) against the runtime-length kernels and
against the numpy oracle at sizes where the specialised path is taken.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solution(wl, dtype=np.complex64, generic=False):
    from macromax_b200 import Bound, Grid, Solution
    old = os.environ.get('MMX_FORCE_GENERIC')
    os.environ['MMX_FORCE_GENERIC'] = '1' if generic else '0'
    try:
        grid = Grid(shape=wl['shape'], step=wl['step'])
        return Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                        source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                        dtype=dtype)
    finally:
        if old is None:
            os.environ.pop('MMX_FORCE_GENERIC', None)
        else:
            os.environ['MMX_FORCE_GENERIC'] = old


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _stacked_voronoi(axis):
    """The 64^3 Voronoi medium repeated three times along one grid axis (192 samples there)."""
    from macromax_b200 import workloads as w
    wl = w.voronoi_3d(n=64, nb_grains=12, boundary_px=48)
    eps = np.concatenate([wl['epsilon']] * 3, axis=2 + axis)
    src = np.concatenate([wl['source']] + [np.zeros_like(wl['source'])] * 2, axis=1 + axis)
    shape = list(wl['shape'])
    shape[axis] *= 3
    return {**wl, 'shape': tuple(shape), 'epsilon': eps, 'source': src}


def _cases():
    from macromax_b200 import workloads as w
    return {
        'spheres3d_64': lambda: w.spheres_3d(n=64, nb_spheres=40),
        'design3d_64': lambda: w.design_3d(n=64),
        'disks2d_128': lambda: w.disks_2d(n=128),
        'disks2d_256': lambda: w.disks_2d(n=256),
        'voronoi3d_64': lambda: w.voronoi_3d(n=64, nb_grains=12, boundary_px=48),
        # anisotropic 3x3 eps with 192-sample strided axes (register-staged 8 x 8 x 3 pencils)
        'voronoi_192x64x64': lambda: _stacked_voronoi(0),
        'voronoi_64x192x64': lambda: _stacked_voronoi(1),
        'voronoi_64x64x192': lambda: _stacked_voronoi(2),  # 192-sample rows: the 3x3-chi contiguous passes
        'mixed_3d': lambda: {**w.design_3d(n=64), 'shape': (64, 40, 64),
                             'epsilon': w.design_3d(n=64)['epsilon'][:, :40, :],
                             'source': w.design_3d(n=64)['source'][:, :, :40, :]},
    }


@pytest.mark.parametrize('name', ['spheres3d_64', 'design3d_64', 'disks2d_128', 'disks2d_256', 'voronoi3d_64',
                                  'mixed_3d'])
def test_specialised_matches_generic(name):
    wl = _cases()[name]()
    fast = _solution(wl)
    gen = _solution(wl, generic=True)
    fast.solve(None, rtol=0, maxiter=15)
    gen.solve(None, rtol=0, maxiter=15)
    assert fast.iteration == gen.iteration == 15
    assert rel(fast.E, gen.E) < 2e-6


@pytest.mark.parametrize('name', ['spheres3d_64', 'disks2d_256'])
def test_specialised_matches_oracle(name):
    from oracle import mmoracle as mo
    wl = _cases()[name]()
    sol = _solution(wl)
    ref = mo.from_workload(wl, np.complex128)
    assert abs(sol.alpha - ref.alpha) <= 1e-9 * abs(ref.alpha)
    rec_ref = ref.solve(rtol=0, maxiter=20, record=(1, 5, 20))
    fields = {}
    for s in sol:
        if s.iteration in (1, 5, 20):
            fields[s.iteration] = s.E
        if s.iteration >= 20:
            break
    for it in (1, 5, 20):
        assert rel(fields[it], rec_ref[it]) < 1e-5, (it, rel(fields[it], rec_ref[it]))


def _solution_env(wl, env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return _solution(wl)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize('name', ['spheres3d_64', 'design3d_64', 'disks2d_256', 'mixed_3d', 'voronoi_192x64x64',
                                  'voronoi_64x192x64', 'voronoi_64x64x192'])
def test_register_staged_matches_shared_staged(name):
    """k_reg_pass (strided passes, 16-pencil tiles, global<->register first/last stages) vs k_fast_pass."""
    wl = _cases()[name]()
    reg = _solution_env(wl, {'MMX_NO_REG': '0'})
    shm = _solution_env(wl, {'MMX_NO_REG': '1'})
    reg.solve(None, rtol=0, maxiter=15)
    shm.solve(None, rtol=0, maxiter=15)
    assert rel(reg.E, shm.E) < 2e-6


def test_register_staged_512_matches_oracle():
    from macromax_b200 import workloads
    from oracle import mmoracle as mo
    wl = workloads.correlated_slab_2d(n=512, nb_modes=1)
    wl['source'] = wl['source'][0]
    sol = _solution(wl)
    ref = mo.from_workload(wl, np.complex128)
    rec = ref.solve(rtol=0, maxiter=10, record=(10,))
    sol.solve(None, rtol=0, maxiter=10)
    assert rel(sol.E, rec[10]) < 1e-5


@pytest.mark.parametrize('name', ['spheres3d_64', 'design3d_64', 'disks2d_256', 'disks2d_128'])
def test_persistent_pipeline_matches_single_tile_passes(name):
    """k_pipe_pass (persistent, double-buffered bulk copies) vs k_regc_pass, bit for bit."""
    wl = _cases()[name]()
    pipe = _solution_env(wl, {'MMX_PIPE': '1'})
    single = _solution_env(wl, {'MMX_PIPE': '0'})
    pipe.solve(None, rtol=0, maxiter=12)
    single.solve(None, rtol=0, maxiter=12)
    assert np.array_equal(pipe.E, single.E)
    st = pipe._engine.read_state()
    assert int(st['status'][0]) == 0


@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_symmetric_chi_six_entries_equals_nine(dtype):
    """A symmetric 3x3 chi is stored as its six distinct entries (MMX_CHI_SYM6); the iteration equals the one on all
    nine entries (MMX_CHI_MAT3) of the same tensor."""
    import torch
    from macromax_b200 import _native as nat
    wl = _cases()['voronoi3d_64']()
    eps = wl['epsilon']
    wl['epsilon'] = (eps + eps.transpose(1, 0, *range(2, eps.ndim))) / 2  # exactly symmetric in FP64 as well
    a, b = _solution(wl, dtype), _solution(wl, dtype)
    ea, eb = a._engine, b._engine
    assert ea.chi_kind == nat.MMX_CHI_SYM6 and ea.chi.shape[0] == 6
    full = torch.empty((9, eb.N), dtype=eb.chi.dtype, device=eb.chi.device)
    for k, row in enumerate((0, 1, 2, 1, 3, 4, 2, 4, 5)):
        full[k] = eb.chi[row]
    eb.chi, eb.chi_kind = full, nat.MMX_CHI_MAT3
    a.solve(None, rtol=0, maxiter=20)
    b.solve(None, rtol=0, maxiter=20)
    assert rel(a.E, b.E) < (1e-6 if dtype == np.complex64 else 1e-13)


def test_persistent_pipeline_wait_limit_raises_timeout_and_keeps_fields_exact():
    """k_pipe_pass's staged-input wait gives up after MMX_PIPE_POLL_LIMIT polls (here 0, so every wait runs out): the
    pass raises MMX_STATUS_TIMEOUT in the right-hand side's state, computes the tile from global memory instead and
    drains its copies before re-arming the stage; the fields equal the single-tile passes' bit for bit."""
    from macromax_b200 import _native as nat
    wl = _cases()['spheres3d_64']()
    pipe = _solution_env(wl, {'MMX_PIPE': '1', 'MMX_PIPE_POLL_LIMIT': '0'})
    single = _solution_env(wl, {'MMX_PIPE': '0', 'MMX_PIPE_POLL_LIMIT': ''})
    pipe.solve(None, rtol=0, maxiter=6)
    single.solve(None, rtol=0, maxiter=6)
    st = pipe._engine.read_state()
    assert int(st['status'][0]) & nat.MMX_STATUS_TIMEOUT
    assert int(single._engine.read_state()['status'][0]) == 0
    assert pipe.iteration == single.iteration == 6
    assert np.array_equal(pipe.E, single.E)


@pytest.mark.parametrize('shape', [(128, 64, 48), (128, 32, 128), (128, 48)])
def test_axis0_green_pass_8_and_16_pencil_tiles_agree_exactly(shape):
    """The vector axis-0 pass (forward FFT, dyadic Green multiply, inverse FFT along 128-sample pencils) runs in
    8-pencil tiles by default and in 16-pencil tiles with MMX_WIDE_GREEN=1.  Every pencil goes through the same
    arithmetic in both, so the fields agree bit for bit (the DC pencil's tile included, on 3D and 2D grids)."""
    from macromax_b200 import workloads as w
    base = w.spheres_3d(n=48, nb_spheres=20)
    rng = np.random.default_rng(3)
    eps = 1.0 + 0.8 * rng.uniform(size=shape) + 0.02j
    src = np.zeros((3, *shape), dtype=np.complex128)
    src[0][(slice(None),) * (len(shape) - 1) + (shape[-1] // 3,)] = 1.0
    src[2][(shape[0] // 2,) + (slice(None),) * (len(shape) - 1)] = 0.5j
    wl = {**base, 'shape': shape, 'epsilon': eps, 'source': src, 'bound_thickness': 4 * base['step']}
    eight = _solution_env(wl, {'MMX_WIDE_GREEN': '0'})
    sixteen = _solution_env(wl, {'MMX_WIDE_GREEN': '1'})
    eight.solve(None, rtol=0, maxiter=12)
    sixteen.solve(None, rtol=0, maxiter=12)
    assert eight.iteration == sixteen.iteration == 12
    assert np.array_equal(eight.E, sixteen.E)
