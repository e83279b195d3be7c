"""
Generate the golden fixtures under ``tests/golden/`` by running the REFERENCE MacroMax package (NumPy backend).

Run from the repository root, where the reference tree is present:

    python tests/golden/make_golden.py                     # every fixture
    python tests/golden/make_golden.py --only-scattering   # the scattering-matrix fixtures only
    python tests/golden/make_golden.py --only-magnetic     # the magnetic-media fixtures only

Every case builds a reference ``macromax.Solution`` on seeded synthetic inputs (``macromax_b200.workloads``) and
records the preconditioner constants (alpha, beta), the field E after selected iterations, the residue and
update-norm history, the iteration count at which the workload's stopping rule fires, and the converged field.
Inputs are stored in the fixture too, so the fixtures do not depend on the generators staying bit-identical.
The fixtures pin both the numpy oracle (``oracle/mmoracle.py``) and, through it and directly, the CUDA path.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle.refimport import import_reference  # noqa: E402
from macromax_b200 import workloads  # noqa: E402

RECORD = (1, 2, 3, 5, 10, 20)


def run_reference(mm, wl, dtype, record=RECORD, rtol=None, maxiter=None, source=None, store_dtype=None):
    from macromax.bound import Bound
    from macromax.utils.ft import Grid
    grid = Grid(shape=wl['shape'], step=wl['step'])
    bound = Bound(grid, thickness=wl['bound_thickness'])
    src = wl['source'] if source is None else source
    sol = mm.Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'], source_distribution=src,
                      bound=bound, dtype=dtype)
    alpha0 = complex(sol._Solution__alpha)
    beta = float(sol._Solution__beta)
    rtol = wl['rtol'] if rtol is None else rtol
    maxiter = wl['maxiter'] if maxiter is None else maxiter
    fields, residues, update_norms, alphas = {}, [], [], []
    t0 = time.perf_counter()
    for s in sol:
        residues.append(s.residue)
        update_norms.append(s.previous_update_norm)
        alphas.append(complex(s._Solution__alpha))
        if s.iteration in record:
            fields[s.iteration] = s.E.copy()
        if not (s.iteration < maxiter and s.residue > rtol):
            break
    elapsed = time.perf_counter() - t0
    sd = store_dtype or dtype
    out = dict(alpha0=np.complex128(alpha0), beta=np.float64(beta), iterations=np.int64(sol.iteration),
               residues=np.asarray(residues), update_norms=np.asarray(update_norms), alphas=np.asarray(alphas),
               final=sol.E.astype(sd), rtol=np.float64(rtol), maxiter=np.int64(maxiter),
               record=np.asarray(sorted(fields)), seconds=np.float64(elapsed))
    for it, f in fields.items():
        out[f'E_{it}'] = f.astype(sd)
    return out


def save_case(name, wl, result, store_inputs=True, input_dtype=np.complex128):
    payload = dict(result)
    payload['shape'] = np.asarray(wl['shape'])
    payload['step'] = np.float64(wl['step'])
    payload['wavelength'] = np.float64(wl['wavelength'])
    payload['bound_thickness'] = np.float64(wl['bound_thickness'])
    if store_inputs:
        payload['epsilon'] = np.asarray(wl['epsilon'], dtype=input_dtype)
        payload['source'] = np.asarray(wl['source'], dtype=input_dtype)
    path = os.path.join(HERE, f'{name}.npz')
    np.savez_compressed(path, **payload)
    print(f'{name}: iterations={int(result["iterations"])} alpha={complex(result["alpha0"]):.10g} '
          f'residue={result["residues"][-1]:.3e} ({float(result["seconds"]):.1f}s) -> {os.path.getsize(path)} B')


def plane_wave_1d(vectorial: bool, anisotropic: bool = False):
    """The 1D plane-wave problem of the reference's test_solution.py:91-358, as source_distribution."""
    import scipy.constants as const
    wavelength = 500e-9
    k0 = 2 * np.pi / wavelength
    nb = 1024
    pitch = wavelength / 16
    bt = 10e-6
    x = pitch * np.arange(nb) - bt
    frac = np.maximum((x[0] + bt) - x, x - (x[-1] - bt)) / bt
    frac = np.maximum(0, frac)
    n = 1 + 1j * 0.1 * frac
    eps = n ** 2
    if anisotropic:
        eps = eps * np.eye(3)[..., None]
        eps[:, :, frac <= 0] = np.array([[1.1, 0.0, 0.3], [0.0, 1.0, 0.0], [0.3, 0.0, 1.1]])[..., None]
    j = np.zeros(x.shape)
    j[np.argmin(np.abs(x))] = 1.0
    if vectorial:
        j = np.array([0, 1, 0])[:, None] * j[None, :]
    else:
        j = j[None, :]
    j = j.astype(np.complex64)
    omega = k0 * const.c
    src = j * (-1j * omega * const.mu_0)
    return dict(shape=(nb,), step=pitch, wavelength=wavelength, epsilon=eps, source=src.astype(np.complex64),
                bound_thickness=0.0, rtol=1e-6, maxiter=10000)


def gain_case():
    """A 2D scalar medium with a small gain inclusion: the divergence guard rejects updates and bumps alpha."""
    rng = np.random.default_rng(7)
    wl = workloads.disks_2d(n=48, seed=7)
    eps = wl['epsilon'].copy()
    eps[20:28, 20:28] = 2.0 - 0.4j
    eps += 0.02j * rng.uniform(size=eps.shape)
    wl['epsilon'] = eps
    wl['rtol'] = 1e-5
    wl['maxiter'] = 200
    return wl


def backend_ops(mm):
    """Known outputs of the reference NumPy backend's per-op methods on seeded random inputs."""
    from macromax.backend.numpy import BackEndNumpy
    from macromax.utils.ft import Grid
    rng = np.random.default_rng(11)
    grid = Grid([5, 10, 20], 100e-9)
    k0 = 10e6
    be = BackEndNumpy(3, grid * k0, hardware_dtype=np.complex128)
    x = (rng.standard_normal((3, 1, 5, 10, 20)) + 1j * rng.standard_normal((3, 1, 5, 10, 20)))
    out = dict(x=x)
    out['ft'] = be.ft(x.copy()).copy()
    out['ift'] = be.ift(x.copy()).copy()
    out['longitudinal'] = be.longitudinal_projection_ft(x.copy()).copy()
    out['transversal'] = be.transversal_projection_ft(x.copy()).copy()
    out['curl_ft'] = be.curl_ft(x.copy()).copy()
    out['k2'] = np.asarray(be.k2).copy()
    for i in range(3):
        out[f'k{i}'] = np.asarray(be.k[i]).copy()
    chi = rng.standard_normal((3, 3, 5, 10, 20)) + 1j * rng.standard_normal((3, 3, 5, 10, 20))
    out['chi'] = chi
    out['mul'] = be.mul(chi, x.copy()).copy()
    out['norm'] = np.float64(be.norm(x))
    path = os.path.join(HERE, 'backend_ops.npz')
    np.savez_compressed(path, **out)
    print(f'backend_ops -> {os.path.getsize(path)} B')


def scattering_media():
    """Seeded slab media for the scattering-matrix fixtures: (name, grid shape, step, vectorial, refractive index)."""
    wavelength = 500e-9
    rng = np.random.default_rng(13)
    cases = []
    for name, shape, vectorial in (('smatrix_1d_scalar', (256,), False),
                                   ('smatrix_2d_scalar', (256, 7), False),
                                   ('smatrix_2d_vector', (256, 7), True),
                                   ('smatrix_3d_scalar', (256, 5, 3), False)):
        n = np.ones(shape)
        lo, hi = shape[0] // 2 - 8, shape[0] // 2 + 8
        ripple = 0.15 * rng.uniform(-1, 1, size=(hi - lo, *shape[1:]))
        n[lo:hi] = 1.5 + ripple
        cases.append((name, shape, wavelength / 4, vectorial, n))
    return wavelength, cases


def scattering_cases(mm):
    """Full scattering matrices of the reference ``ScatteringMatrix`` (complex128, default callback) on small slab
    media, with the reference test suite's boundary (a 20-wavelength linear absorber on both sides of axis 0), plus
    outputs of its host-side vector conversions for seeded vectors and fields."""
    from macromax import matrix
    from macromax.bound import LinearBound
    from macromax.utils.ft import Grid
    wavelength, cases = scattering_media()
    rng = np.random.default_rng(17)
    for name, shape, step, vectorial, n in cases:
        grid = Grid(list(shape), step)
        thickness = np.zeros((grid.ndim, 1))
        thickness[0, 0] = 20 * wavelength
        bound = LinearBound(grid, thickness=thickness, max_extinction_coefficient=0.25)
        t0 = time.perf_counter()
        m = matrix.ScatteringMatrix(grid, vectorial=vectorial, vacuum_wavelength=wavelength, refractive_index=n,
                                    bound=bound, dtype=np.complex128)
        side = m.shape[0]
        vec = rng.standard_normal(side) + 1j * rng.standard_normal(side)
        fld = rng.standard_normal((1 + 2 * vectorial, *shape)) + 1j * rng.standard_normal((1 + 2 * vectorial, *shape))
        out = dict(shape=np.asarray(shape), step=np.float64(step), wavelength=np.float64(wavelength),
                   vectorial=np.bool_(vectorial), refractive_index=n, bound_thickness=np.float64(20 * wavelength),
                   vec=vec, field=fld,
                   freespace=m.srcvec2freespace(vec), source=m.srcvec2source(vec), detvec=m.detfield2detvec(fld),
                   S=np.asarray(m).copy())
        out['seconds'] = np.float64(time.perf_counter() - t0)
        path = os.path.join(HERE, f'{name}.npz')
        np.savez_compressed(path, **out)
        print(f'{name}: side {side}, {out["seconds"]:.1f} s -> {os.path.getsize(path)} B', flush=True)


def magnetic_media():
    """Seeded magnetic media for the magnetic-iteration fixtures: (name, shape, epsilon, xi, zeta, mu, source)."""
    wavelength, step = 500e-9, 500e-9 / 4
    cases = []
    # a negative-index plate (epsilon = mu = -|n|, the conversion of solver.py:227-236 for n = -1.5) in 2D
    n = 48
    x0 = (np.arange(n) - n // 2)[:, None] * step
    plate = np.abs(x0) < 8 * step
    ramp = workloads.ramp_extinction((n, n), 8, 0.5)
    eps = np.where(plate, -2.25, 1.0) + 0.01j + 1j * ramp
    mu = np.where(plate, -1.0, 1.0) + 0.01j + np.zeros((n, n))
    src = np.zeros((3, n, n), dtype=np.complex128)
    g = np.exp(-0.5 * ((np.arange(n) - n / 3) / 6.0) ** 2)
    src[1, n - 10, :] = g
    src[2, n - 10, :] = 1j * g
    cases.append(('magnetic2d_48_c128', (n, n), eps, 0.0, 0.0, mu, src))
    # a lossy chiral sphere (bi-isotropic: xi = -i kappa, zeta = i kappa) in 3D
    n = 16
    grid = np.ogrid[0:n, 0:n, 0:n]
    r2 = sum((gg - n / 2 + 0.5) ** 2 for gg in grid)
    sphere = r2 <= 4.5 ** 2
    ramp = workloads.ramp_extinction((n, n, n), 3, 0.5)
    eps = np.where(sphere, 2.0 + 0.1j, 1.0) + 1j * ramp
    mu = np.where(sphere, 1.2 + 0.05j, 1.0) + np.zeros((n, n, n))
    kappa = np.where(sphere, 0.1, 0.0)
    xi, zeta = -1j * kappa, 1j * kappa
    src = np.zeros((3, n, n, n), dtype=np.complex128)
    src[0, :, :, 4] = np.outer(np.exp(-0.5 * ((np.arange(n) - n / 2) / 4.0) ** 2),
                               np.exp(-0.5 * ((np.arange(n) - n / 2) / 4.0) ** 2))
    cases.append(('chiral3d_16_c128', (n, n, n), eps, xi, zeta, mu, src))
    return wavelength, step, cases


def magnetic_cases(mm):
    """Iterates of the reference Solution on magnetic media (complex128, NumPy backend): alpha, beta, fields after
    selected iterations and the update-norm history."""
    from macromax.bound import Bound
    from macromax.utils.ft import Grid
    wavelength, step, cases = magnetic_media()
    for name, shape, eps, xi, zeta, mu, src in cases:
        grid = Grid(list(shape), step)
        bound = Bound(grid, thickness=2 * step)
        t0 = time.perf_counter()
        sol = mm.Solution(grid, vacuum_wavelength=wavelength, epsilon=eps, xi=xi, zeta=zeta, mu=mu,
                          source_distribution=src, bound=bound, dtype=np.complex128)
        out = dict(shape=np.asarray(shape), step=np.float64(step), wavelength=np.float64(wavelength), epsilon=eps,
                   xi=np.asarray(xi), zeta=np.asarray(zeta), mu=np.asarray(mu), source=src,
                   bound_thickness=np.float64(2 * step), alpha0=np.complex128(sol._Solution__alpha),
                   beta=np.float64(np.real(sol._Solution__beta)))
        norms, fields = [], {}
        for s in sol:
            norms.append(s.previous_update_norm)
            if s.iteration in (1, 5, 60):
                fields[s.iteration] = s.E.copy()
            if s.iteration >= 60:
                break
        out['update_norms'] = np.asarray(norms)
        out['record'] = np.asarray(sorted(fields))
        for it, f in fields.items():
            out[f'E{it}'] = f
        out['alpha_final'] = np.complex128(sol._Solution__alpha)
        out['seconds'] = np.float64(time.perf_counter() - t0)
        path = os.path.join(HERE, f'{name}.npz')
        np.savez_compressed(path, **out)
        print(f'{name}: alpha {out["alpha0"]:.6g} beta {out["beta"]:.6g}, {out["seconds"]:.1f} s -> '
              f'{os.path.getsize(path)} B', flush=True)


def main():
    mm = import_reference()
    if '--only-magnetic' in sys.argv:
        magnetic_cases(mm)
        return
    if '--only-scattering' in sys.argv:
        scattering_cases(mm)
        return
    backend_ops(mm)

    wl = workloads.disks_2d(n=64, seed=1)
    save_case('disks2d_64_c128', wl, run_reference(mm, wl, np.complex128))
    rec3 = (1, 2, 5, 20)
    wl = workloads.spheres_3d(n=20, seed=2, nb_spheres=30, boundary_px=32)  # 5-voxel ramp
    save_case('spheres3d_20_c128', wl, run_reference(mm, wl, np.complex128, record=rec3, maxiter=600))
    wl = workloads.voronoi_3d(n=16, seed=3, nb_grains=8, boundary_px=48)  # 4-voxel ramp
    save_case('voronoi3d_16_c128', wl, run_reference(mm, wl, np.complex128, record=rec3, rtol=1e-8, maxiter=600))
    wl = workloads.design_3d(n=24, seed=5)
    save_case('design3d_24_c128', wl, run_reference(mm, wl, np.complex128, record=rec3))
    wl = gain_case()
    save_case('gain2d_48_c128', wl, run_reference(mm, wl, np.complex128))
    for vec, aniso, name in ((False, False, 'plane1d_scalar_c64'), (True, False, 'plane1d_vector_c64'),
                             (True, True, 'plane1d_aniso_c64')):
        wl = plane_wave_1d(vec, aniso)
        save_case(name, wl, run_reference(mm, wl, np.complex64, record=(1, 2, 5, 20)), input_dtype=np.complex128)
    # full-size 256^2 disks (the complex128 configuration): inputs come from the seeded generator (checksummed)
    wl = workloads.disks_2d(n=256, seed=1)
    res = run_reference(mm, wl, np.complex128, record=(1, 20), store_dtype=np.complex64)
    res['epsilon_checksum'] = np.float64(np.sum(np.abs(wl['epsilon']) * np.arange(wl['epsilon'].size).reshape(
        wl['epsilon'].shape) % 1009))
    res['source_checksum'] = np.float64(np.sum(np.abs(wl['source'])))
    save_case('disks2d_256_c128', wl, res, store_inputs=False)
    scattering_cases(mm)
    magnetic_cases(mm)


if __name__ == '__main__':
    main()
