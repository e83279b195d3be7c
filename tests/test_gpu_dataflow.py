"""
Dataflow schedule of the 3D passes (MMX_VARIANT_DATAFLOW): the axis-0, inverse axis-1 and epilogue passes wait for
the tiles that wrote their inputs (per-chunk / per-plane counters) instead of for the whole previous pass.  Only
the order in which tiles run changes, not what any tile computes, so fields, norms, iteration counts, rejections
and alpha must equal those of the whole-pass schedule bit for bit: with and without the fused epilogue, for scalar
and vector fields, for batches whose members stop at different iterations, and in a gain medium that rejects
updates.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solution(wl, flags):
    from macromax_b200 import Bound, Grid, Solution
    from macromax_b200 import autotune
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    autotune.set_variant(sol._engine, flags)
    assert autotune.get_variant(sol._engine) == flags
    return sol


def _gain_3d(n=64):
    """spheres3d with a gain cube in the centre: the divergence guard rejects updates (the complex64 oracle counts
    11 rejections in the first 40 iterations at n = 64)."""
    from macromax_b200 import workloads
    wl = workloads.spheres_3d(n=n, nb_spheres=30)
    eps = wl['epsilon'].copy()
    lo, hi = int(n * 0.4), int(n * 0.6)
    eps[lo:hi, lo:hi, lo:hi] = 2.0 - 0.8j
    wl['epsilon'] = eps
    return wl


def _cases():
    from macromax_b200 import workloads as w
    return {
        'spheres3d_64': lambda: w.spheres_3d(n=64, nb_spheres=40),
        'design3d_64': lambda: w.design_3d(n=64),
        'design3d_128': lambda: w.design_3d(n=128),
        'spheres3d_128': lambda: w.spheres_3d(n=128),
        'gain3d_64': lambda: _gain_3d(64),
    }


def _same_state(sa, sb):
    for key in ('iteration', 'rejections', 'cur', 'active', 'status', 'alpha_im', 'prev_norm', 'last_norm',
                'field_norm', 'residue'):
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize('name,fused', [('spheres3d_64', False), ('spheres3d_64', True), ('design3d_64', False),
                                        ('design3d_64', True), ('design3d_128', True), ('spheres3d_128', True),
                                        ('gain3d_64', False), ('gain3d_64', True)])
def test_dataflow_equals_whole_pass_schedule(name, fused):
    from macromax_b200 import _native as nat
    wl = _cases()[name]()
    base = nat.MMX_VARIANT_FUSED_EPILOGUE if fused else 0
    a, b = _solution(wl, base | nat.MMX_VARIANT_DATAFLOW), _solution(wl, base)
    a.solve(None, rtol=0, maxiter=40)
    b.solve(None, rtol=0, maxiter=40)
    sa, sb = a._engine.read_state(), b._engine.read_state()
    assert int(sa['iteration'][0]) == 40
    _same_state(sa, sb)
    assert np.array_equal(a.E, b.E)
    if name.startswith('gain'):
        assert int(sa['rejections'][0]) > 0  # the case exercises the rejection path


def test_dataflow_batch_members_stopping_at_different_iterations():
    """Members that stop early skip every pass (no tile of theirs signals or waits) while the others go on."""
    from macromax_b200 import Bound, Grid
    from macromax_b200 import _native as nat
    from macromax_b200 import autotune, workloads
    from macromax_b200.batch import BatchSolution
    wl = workloads.design_3d(n=64, nb_sources=4)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    runs = []
    for flags in (nat.MMX_VARIANT_DATAFLOW, 0, nat.MMX_VARIANT_DATAFLOW | nat.MMX_VARIANT_FUSED_EPILOGUE,
                  nat.MMX_VARIANT_FUSED_EPILOGUE):
        bs = BatchSolution(grid, wl['source'], wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                           vacuum_wavelength=wl['wavelength'])
        autotune.set_variant(bs.engine, flags)
        assert autotune.get_variant(bs.engine) == flags
        st = bs.engine.read_state()
        st['iteration'] = 0
        st['rtol'] = 0.0
        st['maxiter'] = np.array([5, 31, 13, 24], dtype=np.float64)
        st['active'] = 1
        st['status'] = 0
        bs.engine.write_state(st)
        bs.engine.iterate(8)
        bs.engine.iterate(24)
        runs.append((bs.engine.read_state(), bs.E))
    for (sa, ea), (sb, eb) in (runs[0:2], runs[2:4]):
        assert list(sa['iteration']) == [5, 31, 13, 24]
        _same_state(sa, sb)
        assert np.array_equal(ea, eb)


def test_dataflow_only_where_eligible():
    """2D grids keep the whole-pass waits (the flag is not taken)."""
    from macromax_b200 import Bound, Grid, Solution
    from macromax_b200 import _native as nat
    from macromax_b200 import autotune, workloads
    wl = workloads.disks_2d(n=128)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    autotune.set_variant(sol._engine, nat.MMX_VARIANT_DATAFLOW)
    assert autotune.get_variant(sol._engine) == 0
