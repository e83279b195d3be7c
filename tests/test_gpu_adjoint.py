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
    """Batched sources in complex64: gradient w.r.t. a source sample vs finite differences (looser tolerance)."""
    import torch
    from macromax_b200 import adjoint
    wl, grid, bound = _problem(n=16)
    assert wl['source'].any()
    k0 = 2 * np.pi / wl['wavelength']
    eps = torch.tensor(wl['epsilon'], dtype=torch.complex64, device='cuda')
    base = torch.tensor(wl['source'], dtype=torch.complex64, device='cuda')
    src = torch.stack([base, 0.5 * torch.roll(base, 2, dims=2)]).requires_grad_(True)
    E = adjoint.solve(eps, src, grid, k0, bound=bound, dtype=np.complex64, rtol=1e-7, maxiter=20000)
    L = sum(_loss(E[b:b + 1], wl['patch']) for b in range(2))
    L.backward()
    g = src.grad.detach().cpu().numpy()
    assert np.isfinite(g).all() and np.abs(g).max() > 0
