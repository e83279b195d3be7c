"""
Adjoint gradient (torch.autograd.Function) against central finite differences and against a two-solve gradient
built from the numpy oracle (forward solve + adjoint solve with the transposed material).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(n=24):
    """Small version of the design workload: 4-voxel absorbing ramp, sheet at z = n/4, detector at z = 3n/4."""
    from macromax_b200 import Bound, Grid, workloads
    s = 128.0 / n
    wl = workloads.design_3d(n=n, design_px=int(8 * s), boundary_px=int(4 * s), sheet_index=int(n / 4 * s),
                             detector_index=int(3 * n / 4 * s), patch_px=9)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    return wl, grid, Bound(grid, thickness=wl['bound_thickness'])


def _loss(E, patch):
    return -(E[0, 0][patch].abs() ** 2).sum()


def test_adjoint_matches_finite_differences():
    import torch
    from macromax_b200 import adjoint
    wl, grid, bound = _problem()
    k0 = 2 * np.pi / wl['wavelength']
    eps = torch.tensor(wl['epsilon'].real, dtype=torch.float64, device='cuda', requires_grad=True)
    eps_imag = torch.tensor(wl['epsilon'].imag, dtype=torch.float64, device='cuda')
    src = torch.tensor(wl['source'], dtype=torch.complex128, device='cuda')

    def run(e, grad=False):
        epsc = torch.complex(e, eps_imag)
        E = adjoint.solve(epsc, src, grid, k0, bound=bound, dtype=np.complex128, rtol=1e-12, maxiter=20000)
        return _loss(E, wl['patch'])

    L = run(eps)
    L.backward()
    g = eps.grad.detach().cpu().numpy()
    rng = np.random.default_rng(5)
    design = np.argwhere(np.ones(grid.shape, dtype=bool)[wl['design']])
    lo = np.array([s.start for s in wl['design']])
    picks = design[rng.choice(len(design), size=8, replace=False)] + lo
    h = 1e-3
    for idx in picks:
        idx = tuple(int(i) for i in idx)
        with torch.no_grad():
            e1 = eps.detach().clone(); e1[idx] += h
            e2 = eps.detach().clone(); e2[idx] -= h
            fd = (run(e1).item() - run(e2).item()) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-4 * max(abs(fd), 1e-30) + 1e-4 * np.abs(g).max() * 1e-3, (idx, fd, g[idx])


def test_adjoint_matches_two_solve_oracle_gradient():
    import torch
    from macromax_b200 import adjoint
    from oracle import mmoracle as mo
    wl, grid, bound = _problem()
    k0 = 2 * np.pi / wl['wavelength']
    eps = torch.tensor(wl['epsilon'], dtype=torch.complex128, device='cuda', requires_grad=True)
    src = torch.tensor(wl['source'], dtype=torch.complex128, device='cuda')
    E = adjoint.solve(eps, src, grid, k0, bound=bound, dtype=np.complex128, rtol=1e-12, maxiter=20000)
    L = _loss(E, wl['patch'])
    L.backward()
    g_dev = eps.grad.detach().cpu().numpy()
    # two oracle solves: forward field and adjoint field for source conj(dL/dE) = conj(-2 E) on the patch
    fwd = mo.OracleSolution(wl['shape'], wl['step'], wl['wavelength'], wl['epsilon'], wl['source'],
                            wl['bound_thickness'], dtype=np.complex128)
    fwd.solve(rtol=1e-12, maxiter=20000)
    Ef = fwd.E[0]
    gE = np.zeros_like(Ef)
    gE[wl['patch']] = -2 * Ef[wl['patch']]
    adj = mo.OracleSolution(wl['shape'], wl['step'], wl['wavelength'], wl['epsilon'], np.conj(gE)[None],
                            wl['bound_thickness'], dtype=np.complex128)
    adj.solve(rtol=1e-12, maxiter=20000)
    nu = adj.field[0, 0]          # k0^2-scaled adjoint field
    F = fwd.field[0, 0]           # k0^2-scaled forward field
    g_ref = np.conj(nu * F) / k0 ** 2
    assert np.linalg.norm(g_dev - g_ref) <= 1e-6 * np.linalg.norm(g_ref)


def test_adjoint_source_gradient_complex64_batch():
    """Batched sources in complex64: the gradient w.r.t. the sources equals the complex128 adjoint gradient of the same
    problem within 1e-4 relative L2 (complex64 solves to residue 1e-7)."""
    import torch
    from macromax_b200 import adjoint
    wl, grid, bound = _problem(n=16)
    assert wl['source'].any()
    k0 = 2 * np.pi / wl['wavelength']
    grads = {}
    for dt, tdt, rtol in ((np.complex64, torch.complex64, 1e-7), (np.complex128, torch.complex128, 1e-12)):
        eps = torch.tensor(wl['epsilon'], dtype=tdt, device='cuda')
        base = torch.tensor(wl['source'], dtype=tdt, device='cuda')
        src = torch.stack([base, 0.5 * torch.roll(base, 2, dims=2)]).requires_grad_(True)
        E = adjoint.solve(eps, src, grid, k0, bound=bound, dtype=dt, rtol=rtol, maxiter=20000)
        L = sum(_loss(E[b:b + 1], wl['patch']) for b in range(2))
        L.backward()
        grads[dt] = src.grad.detach().cpu().numpy().astype(np.complex128)
    g32, g64 = grads[np.complex64], grads[np.complex128]
    assert np.abs(g64).max() > 0
    assert np.linalg.norm(g32 - g64) <= 1e-4 * np.linalg.norm(g64)


def test_adjoint_complex64_permittivity_gradient_matches_finite_differences_128():
    """The design problem at its full size (128^3 scalar, 64^3 design region, 9 x 9 detector patch), the loss summed
    over a batch of two sources.  The complex64 adjoint gradient dL/d eps (forward and adjoint solves in complex64)
    against central finite differences (h = 1e-3) on 64 seeded design voxels; every finite-difference loss comes
    from an FP64 solve (complex64 inner iterations with FP64 defect correction to residue 1e-12, started from the
    unperturbed FP64 solution).  Tolerance: 1e-4 relative L2 over the 64 voxels."""
    import torch
    from macromax_b200 import Bound, Grid, adjoint, workloads
    from macromax_b200.mixed import MixedSolution
    wl = workloads.design_3d(n=128)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    k0 = 2 * np.pi / wl['wavelength']
    base = np.asarray(wl['source'])
    sources = np.stack([base, 0.5 * np.roll(base, 9, axis=2)])
    patch = wl['patch']
    eps_re = torch.tensor(wl['epsilon'].real, dtype=torch.float32, device='cuda', requires_grad=True)
    eps_im = torch.tensor(wl['epsilon'].imag, dtype=torch.float32, device='cuda')
    src = torch.tensor(sources, dtype=torch.complex64, device='cuda')
    E = adjoint.solve(torch.complex(eps_re, eps_im), src, grid, k0, bound=bound, dtype=np.complex64, rtol=3e-7,
                      maxiter=20000)
    L = -sum((E[b, 0][patch].abs() ** 2).sum() for b in range(2))
    L.backward()
    g = eps_re.grad.detach().cpu().numpy().astype(np.float64)

    def loss64(eps, x0):
        ms = MixedSolution(grid, sources, eps, bound=bound, vacuum_wavelength=wl['wavelength'], initial_field=x0)
        ms.solve(rtol=1e-12)
        assert float(ms.residues.max()) < 1e-12
        Ex = ms.E
        ms.close()
        return -sum(float(np.sum(np.abs(Ex[b, 0][patch]) ** 2)) for b in range(2)), Ex

    _, E0 = loss64(wl['epsilon'], None)
    rng = np.random.default_rng(5)
    lo = np.array([s.start for s in wl['design']])
    hi = np.array([s.stop for s in wl['design']])
    picks = [tuple(int(v) for v in rng.integers(lo, hi)) for _ in range(64)]
    h = 1e-3
    fd = np.empty(64)
    for n, idx in enumerate(picks):
        e1 = wl['epsilon'].copy()
        e1[idx] += h
        e2 = wl['epsilon'].copy()
        e2[idx] -= h
        fd[n] = (loss64(e1, E0)[0] - loss64(e2, E0)[0]) / (2 * h)
    ga = np.array([g[idx] for idx in picks])
    err = np.linalg.norm(ga - fd) / np.linalg.norm(fd)
    assert err <= 1e-4, (err, np.max(np.abs(ga - fd) / np.abs(fd)))


def test_mixed_precision_adjoint_matches_complex128_adjoint():
    """precision='mixed' (complex64 inner iterations, FP64 defect correction for both solves) gives the complex128
    adjoint gradient of the same problem within 1e-7 relative, for the permittivity and the sources, in a batch."""
    import torch
    from macromax_b200 import adjoint
    wl, grid, bound = _problem()
    k0 = 2 * np.pi / wl['wavelength']
    grads = {}
    # the same complex128 inputs for both (the mixed solve's own arithmetic is complex64 inside, FP64 outside)
    for name, dt, tdt, kw in (('c128', np.complex128, torch.complex128, dict(rtol=1e-12)),
                              ('mixed', np.complex128, torch.complex128, dict(rtol=1e-12, precision='mixed'))):
        eps = torch.tensor(wl['epsilon'], dtype=tdt, device='cuda', requires_grad=True)
        base = torch.tensor(wl['source'], dtype=tdt, device='cuda')
        src = torch.stack([base, 0.5 * torch.roll(base, 3, dims=2)]).requires_grad_(True)
        E = adjoint.solve(eps, src, grid, k0, bound=bound, dtype=dt, maxiter=20000, **kw)
        L = sum(_loss(E[b:b + 1], wl['patch']) for b in range(2))
        L.backward()
        assert eps.grad.dtype == tdt and src.grad.dtype == tdt
        grads[name] = (eps.grad.detach().cpu().numpy().astype(np.complex128),
                       src.grad.detach().cpu().numpy().astype(np.complex128))
    for k in range(2):
        a, b = grads['mixed'][k], grads['c128'][k]
        assert np.linalg.norm(a - b) <= 1e-7 * np.linalg.norm(b)
