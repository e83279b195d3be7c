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



def _solve_variant(wl, variant, iters):
    from macromax_b200 import Bound, Grid, Solution, autotune
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    autotune.set_variant(sol._engine, variant)
    assert autotune.get_variant(sol._engine) == variant
    sol.solve(None, rtol=0, maxiter=iters)
    E, st = sol.E, sol._engine.read_state()
    sol._engine.close()
    return E, st


@pytest.mark.parametrize('variant', [32, 48])
def test_tensor_staged_passes_equal_register_staged_passes(spheres128, variant):
    """The strided passes staged by bulk tensor copies (variant 32: k_tma_pass, alone and with the fused epilogue)
    run the same arithmetic as k_reg_pass: identical fields, bit for bit, on the 128^3 vector workload; and the
    oracle's iterates within 1e-5."""
    wl, (alpha_ref, ref) = spheres128
    a, st_a = _solve_variant(wl, variant, 20)
    b, st_b = _solve_variant(wl, variant & ~32, 20)
    assert int(st_a['status'][0]) == 0 and int(st_a['iteration'][0]) == 20
    assert np.array_equal(a, b)
    assert rel(a, ref[20]) < 1e-5


def test_tensor_staged_scalar_passes_equal_register_staged_passes():
    """The scalar (one-component) tensor-staged passes on the 128^3 design problem."""
    from macromax_b200 import workloads
    wl = workloads.design_3d(n=128)
    a, st = _solve_variant(wl, 32, 12)
    b, _ = _solve_variant(wl, 0, 12)
    assert int(st['status'][0]) == 0
    assert np.array_equal(a, b)


def test_tensor_staged_passes_in_a_batch_with_finished_members():
    """A batch whose members stop at different iterations: tiles of inactive right-hand sides are skipped without a
    copy, and every member equals its solve with the register-staged passes."""
    import torch
    from macromax_b200 import Bound, Grid, autotune, workloads
    from macromax_b200.batch import BatchSolution
    wl = workloads.spheres_3d(n=128, nb_spheres=60)
    src = np.stack([wl['source'], 0.3 * np.roll(wl['source'], 7, axis=2), np.roll(wl['source'], -5, axis=1)])
    grid = Grid(shape=wl['shape'], step=wl['step'])
    out = {}
    for variant in (0, 32):
        bs = BatchSolution(grid, src, wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                           vacuum_wavelength=wl['wavelength'], dtype=np.complex64)
        eng = bs.engine
        autotune.set_variant(eng, variant)
        st = eng.read_state()
        st['iteration'], st['rtol'], st['active'], st['status'] = 0, -1.0, 1, 0
        st['maxiter'] = [15, 30, 45]  # the members stop one after the other
        eng.write_state(st)
        for _ in range(6):
            eng.iterate(8)
        out[variant] = (bs.E.copy(), bs.iterations.copy())
        bs.close()
        torch.cuda.empty_cache()
    assert list(out[32][1]) == [15, 30, 45]
    assert np.array_equal(out[0][1], out[32][1])
    assert np.array_equal(out[0][0], out[32][0])


@pytest.mark.parametrize('variant', [0, 16])
def test_zero_source_components_are_skipped_without_changing_the_iterates(spheres128, variant):
    """The headline source is x-polarised, so components 1 and 2 of s' are identically zero: set_sources marks them
    (bit c of the state's reserved[1]) and the prologue kernels skip reading them.  The iterates equal those of the
    same solve with the marks cleared (every component read)."""
    from macromax_b200 import Bound, Grid, Solution, autotune
    wl = spheres128[0]
    fields = []
    for keep in (True, False):
        grid = Grid(shape=wl['shape'], step=wl['step'])
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       dtype=np.complex64)
        eng = sol._engine
        autotune.set_variant(eng, variant)
        st = eng.read_state()
        assert int(st['reserved'][0, 1]) == 0b110
        if not keep:
            st['reserved'][:, 1] = 0
            eng.write_state(st)
        sol.solve(None, rtol=0, maxiter=12)
        fields.append(sol.E)
        eng.close()
    assert np.array_equal(fields[0], fields[1])


def test_anisotropic_192_fused_epilogue_matches_oracle_and_plain_schedule():
    """The 3x3-chi epilogue fused with the next prologue on 192-sample rows (variant 16: k_regc_aniso_epro, with
    k_regc_aniso_repair after a rejection) against the oracle's iterates at 1, 5 and 20 iterations, and against the
    plain schedule (k_regc_aniso_pass) of the same plan."""
    wl = _stacked_voronoi(2)
    alpha_ref, ref = _oracle_fields(wl)
    alpha, fields = _device_fields(wl, 16)
    _, plain = _device_fields(wl, 0)
    assert abs(alpha - alpha_ref) <= 1e-9 * abs(alpha_ref)
    for it in RECORD:
        assert rel(fields[it], ref[it]) < 1e-5, (it, rel(fields[it], ref[it]))
        assert rel(fields[it], plain[it]) < 2e-6, (it, rel(fields[it], plain[it]))


def _anisotropic_gain():
    """The stacked Voronoi medium (192 samples on the contiguous axis) with a gain block (-0.5i on the diagonal of
    chi): the oracle rejects 10 of the first 40 updates and raises alpha."""
    wl = _stacked_voronoi(2)
    eps = wl['epsilon'].copy()
    for c in range(3):
        eps[c, c, 24:40, 24:40, 88:104] -= 0.5j
    return {**wl, 'epsilon': eps}


def test_anisotropic_192_fused_epilogue_with_rejections():
    """Rejected updates on the 3x3-chi path: the repair pass recomputes the prologue from the kept field at the
    raised alpha.  Same rejections and alpha as the oracle and the plain schedule, and no further from the complex128
    oracle than the plain schedule (the gain amplifies the rounding of either complex64 schedule)."""
    from oracle import mmoracle as mo
    wl = _anisotropic_gain()
    mo.set_fft_workers(os.cpu_count() or 1)
    ref = mo.from_workload(wl, np.complex128)
    rec = ref.solve(rtol=0, maxiter=40, record=(40,))
    a, st_a = _solve_variant(wl, 16, 40)
    b, st_b = _solve_variant(wl, 0, 40)
    assert int(st_a['status'][0]) == 0 and int(st_a['iteration'][0]) == 40
    assert int(st_a['rejections'][0]) == int(st_b['rejections'][0]) == ref.rejections > 0
    assert abs(st_a['alpha_im'][0] - ref.alpha.imag) <= 1e-9 * abs(ref.alpha.imag)
    ea, eb = rel(a, rec[40]), rel(b, rec[40])
    assert ea <= 2.0 * eb + 1e-6, (ea, eb)
