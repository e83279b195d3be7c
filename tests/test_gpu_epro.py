"""
Epilogue fused with the next iteration's speculative prologue (k_regc_epro + k_regc_repair) against the plain
schedule of the same plan: fields, iteration counts, divergence-guard rejections and alpha, including a gain medium
whose updates are rejected (the repair pass recomputes the prologue from the kept field).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _gain_2d(n=64, seed=7, gain=1.0):
    """A 2D scalar medium with a gain inclusion: the divergence guard rejects updates and raises alpha (the
    oracle counts 8 rejections in the first 40 iterations at n = 64, gain 1.0, and 4 at n = 128, gain 0.4)."""
    from macromax_b200 import workloads
    rng = np.random.default_rng(seed)
    wl = workloads.disks_2d(n=n, seed=seed)
    eps = wl['epsilon'].copy()
    lo, hi = int(round(n * 20 / 48)), int(round(n * 28 / 48))
    eps[lo:hi, lo:hi] = 2.0 - 1j * gain
    eps += 0.02j * rng.uniform(size=eps.shape)
    wl['epsilon'] = eps
    return wl


def _set(eng, fused):
    from macromax_b200 import _native as nat
    from macromax_b200 import autotune
    flags = nat.MMX_VARIANT_FUSED_EPILOGUE if fused else 0
    autotune.set_variant(eng, flags)
    assert autotune.get_variant(eng) == flags


def _solution(wl, fused):
    from macromax_b200 import Bound, Grid, Solution
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                   source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                   dtype=np.complex64)
    _set(sol._engine, fused)
    return sol


def _cases():
    from macromax_b200 import workloads as w
    return {
        'spheres3d_64': lambda: w.spheres_3d(n=64, nb_spheres=40),
        'design3d_64': lambda: w.design_3d(n=64),
        'disks2d_256': lambda: w.disks_2d(n=256),
        'design3d_128': lambda: w.design_3d(n=128),
        'slab2d_512': lambda: {**w.correlated_slab_2d(n=512, nb_modes=1),
                               'source': w.correlated_slab_2d(n=512, nb_modes=1)['source'][0]},
        'gain2d_64': lambda: _gain_2d(64),
        'gain2d_128': lambda: _gain_2d(128, seed=3, gain=0.4),
    }


@pytest.mark.parametrize('name', ['spheres3d_64', 'design3d_64', 'disks2d_256', 'design3d_128', 'slab2d_512'])
def test_fused_epilogue_matches_plain_schedule(name):
    """The fused epilogue against the plain schedule, including the scalar 128- and 512-sample rows that the
    autotuner times for the adjoint design problem and the batched slab."""
    wl = _cases()[name]()
    a, b = _solution(wl, True), _solution(wl, False)
    a.solve(None, rtol=0, maxiter=40)
    b.solve(None, rtol=0, maxiter=40)
    sa, sb = a._engine.read_state(), b._engine.read_state()
    assert int(sa['iteration'][0]) == int(sb['iteration'][0]) == 40
    assert int(sa['rejections'][0]) == int(sb['rejections'][0])
    assert rel(a.E, b.E) < 2e-6


@pytest.mark.parametrize('name', ['gain2d_64', 'gain2d_128'])
def test_fused_epilogue_with_rejections_matches_oracle(name):
    """A gain medium: rejected updates make the repair pass recompute the prologue from the kept field at the
    raised alpha.  The same rejections as the plain schedule, and no further from the complex128 oracle (the
    gain amplifies the rounding of either complex64 schedule, so the two are compared through the oracle)."""
    from oracle import mmoracle as mo
    wl = _cases()[name]()
    a, b = _solution(wl, True), _solution(wl, False)
    a.solve(None, rtol=0, maxiter=40)
    b.solve(None, rtol=0, maxiter=40)
    sa, sb = a._engine.read_state(), b._engine.read_state()
    ref = mo.from_workload(wl, np.complex128)
    rec = ref.solve(rtol=0, maxiter=40, record=(40,))
    assert int(sa['rejections'][0]) == int(sb['rejections'][0]) == ref.rejections > 0
    assert abs(sa['alpha_im'][0] - ref.alpha.imag) <= 1e-9 * abs(ref.alpha.imag)
    ea, eb = rel(a.E, rec[40]), rel(b.E, rec[40])
    assert ea <= 2.0 * eb + 1e-6, (ea, eb)


def test_fused_epilogue_stop_rule_and_oracle():
    """Solve to a residue with the fused schedule: same iteration count as the plain one, oracle within 1e-5."""
    from macromax_b200 import workloads
    from oracle import mmoracle as mo
    wl = workloads.disks_2d(n=64)
    a, b = _solution(wl, True), _solution(wl, False)
    a.solve(None, rtol=1e-4, maxiter=2000)
    b.solve(None, rtol=1e-4, maxiter=2000)
    assert a.iteration == b.iteration
    ref = mo.from_workload(wl, np.complex128)
    rec = ref.solve(rtol=0, maxiter=20, record=(20,))
    c = _solution(wl, True)
    c.solve(None, rtol=0, maxiter=20)
    assert rel(c.E, rec[20]) < 1e-5


def test_fused_epilogue_batched_rejections():
    """Per-right-hand-side rejections in one batch: the repair pass redoes exactly the rejected right-hand sides,
    so every member of the batch follows its own single-source solve on the same (fused) kernels."""
    from macromax_b200 import Bound, Grid
    from macromax_b200.batch import BatchSolution
    wl = _gain_2d(64)
    base = np.asarray(wl['source'])
    rng = np.random.default_rng(2)
    srcs = np.stack([np.roll(base, int(rng.integers(-9, 9)), axis=1) * (0.5 + rng.uniform()) for _ in range(5)])
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])

    def run(s):
        bs = BatchSolution(grid, s, wl['epsilon'], bound=bound, vacuum_wavelength=wl['wavelength'],
                           dtype=np.complex64)
        _set(bs.engine, True)
        bs.solve(rtol=0, maxiter=60)
        out = (bs.iterations, bs.rejections, bs.alphas, bs.E)
        bs.close()
        return out

    ib, rb, ab, eb = run(srcs)
    assert np.any(rb > 0) and len(set(rb.tolist())) > 1  # the members reject on their own schedules
    for k in range(len(srcs)):
        i1, r1, a1, e1 = run(srcs[k:k + 1])
        assert ib[k] == i1[0] and rb[k] == r1[0] and ab[k] == a1[0]
        assert rel(eb[k], e1[0]) < 1e-6


def test_fused_epilogue_dense_vector_source_matches_plain_schedule():
    """A source with all three components nonzero (no source component is skipped): the fused epilogue follows the
    plain schedule."""
    from macromax_b200 import workloads as w
    wl = w.spheres_3d(n=64, nb_spheres=40)
    rng = np.random.default_rng(11)
    src = np.asarray(wl['source']).copy()
    src[1] = 0.3 * np.roll(src[0], 5, axis=0)
    src[2] = (rng.standard_normal(src[2].shape) + 1j * rng.standard_normal(src[2].shape)) * 1e-2
    wl['source'] = src
    a, b = _solution(wl, True), _solution(wl, False)
    a.solve(None, rtol=0, maxiter=30)
    b.solve(None, rtol=0, maxiter=30)
    assert a.iteration == b.iteration == 30
    assert rel(a.E, b.E) < 2e-6


def _chunks(wl, seq):
    """Run chunks of iterations on one fused-epilogue solution: (niter, cont) items, or 'variant' (set the variant
    again, which clears the plan's record of the previous call); returns the state and the current field."""
    import torch
    sol = _solution(wl, True)
    eng = sol._engine
    st = eng.read_state()
    st['rtol'] = -1.0
    st['maxiter'] = np.inf
    st['active'] = 1
    eng.write_state(st)
    for op in seq:
        if op == 'variant':
            _set(eng, True)
        else:
            eng.iterate(op[0], cont=op[1])
    torch.cuda.synchronize()
    out = eng.read_state(), eng.current()[0].cpu().numpy()
    eng.close()
    return out


def test_continued_chunks_equal_one_longer_chunk():
    """mmx_iterate_graph_continue: the chunks of a solve after the first start from the first pass that the previous
    chunk's fused epilogue left in the work buffer, so three continued chunks of 10 iterations give one 30-iteration
    graph's fields bit for bit.  A variant change in between clears the plan's record: the next chunk then starts
    with its own first pass, exactly like a self-contained call, and agrees with the continuation to complex64
    rounding."""
    wl = _cases()['spheres3d_64']()
    sa, ea = _chunks(wl, [(10, False), (10, True), (10, True)])
    sb, eb = _chunks(wl, [(30, False)])
    assert int(sa['iteration'][0]) == int(sb['iteration'][0]) == 30
    assert np.array_equal(ea, eb)
    sc, ec = _chunks(wl, [(10, False), 'variant', (10, True)])
    sd, ed = _chunks(wl, [(10, False), (10, False)])
    assert int(sc['iteration'][0]) == int(sd['iteration'][0]) == 20
    assert np.array_equal(ec, ed)
    se, ee = _chunks(wl, [(10, False), (10, True)])
    assert rel(ee, ed) < 1e-6


def test_continued_chunks_with_rejections_follow_the_oracle():
    """A gain medium whose updates are rejected: the chunk boundaries fall between rejected and accepted updates,
    and the continued solve keeps the rejection count and the iterates of one longer call."""
    wl = _cases()['gain2d_64']()
    sa, ea = _chunks(wl, [(8, False)] + [(8, True)] * 4)
    sb, eb = _chunks(wl, [(40, False)])
    assert int(sa['rejections'][0]) == int(sb['rejections'][0]) > 0
    assert np.array_equal(ea, eb)
