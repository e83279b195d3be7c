"""
Seeded synthetic inputs for the five benchmark workloads of the split-Richardson solver.

The reference publishes no dataset for this path, so every workload is generated here from
``numpy.random.default_rng(seed)`` with the shapes, sizes and value distributions of the benchmark
configurations.  Units: vacuum wavelength 500 nm, sample pitch wavelength / 4.  Array axis i is the
Cartesian axis (x, y, z)[i] and, for vector fields, component index == axis index (the convention of
``backend/__init__.py:500-507, 633-644`` in the reference).

Every generator returns a plain ``dict`` with numpy arrays, so the same inputs can be fed to the
reference NumPy backend, to the numpy oracle, and to the B200 backend:

- ``shape``: grid shape; ``step``: sample pitch [m]; ``wavelength``: vacuum wavelength [m]
- ``epsilon``: permittivity, shape ``shape`` (isotropic) or ``(3, 3, *shape)`` (anisotropic),
  boundary ramp already included
- ``source``: ``source_distribution`` ([1|3, *shape], or ``(B, 1|3, *shape)`` for batches)
- ``bound_thickness``: thickness [m] of the absorbing layer, to build a plain ``Bound`` whose only
  role is to bias alpha (reference ``solver.py:591-627``)
- ``rtol``: stopping residue of the workload
"""
from __future__ import annotations

import numpy as np

WAVELENGTH = 500e-9
STEP = WAVELENGTH / 4


def ramp_extinction(shape, thickness_px: int, max_value: float) -> np.ndarray:
    """
    Linear ramp 0 -> max_value over the outer ``thickness_px`` samples of every axis; at corners the maximum over
    axes is kept, as ``AbsorbingBound.extinction`` does (reference ``bound.py:158-183``).
    """
    result = np.zeros(shape)
    if thickness_px <= 0:
        return result
    for axis, n in enumerate(shape):
        idx = np.arange(n, dtype=np.float64)
        depth = np.maximum((thickness_px - idx) / thickness_px, (idx - (n - 1 - thickness_px)) / thickness_px)
        depth = np.clip(depth, 0.0, 1.0)
        view = [1] * len(shape)
        view[axis] = n
        result = np.maximum(result, max_value * depth.reshape(view))
    return result


def _gaussian(n: int, centre: float, waist: float) -> np.ndarray:
    x = np.arange(n, dtype=np.float64)
    return np.exp(-((x - centre) / waist) ** 2)


def disks_2d(n: int = 256, seed: int = 1, nb_disks: int = 20, boundary_px: int = 16,
             source_index: int = 24, waist_px: float = 40.0) -> dict:
    """2D scalar Helmholtz: 20 disks of radius U(5, 20) px, eps = n^2 + 0.01i, n ~ U(1.3, 1.6), 16-px ramp."""
    rng = np.random.default_rng(seed)
    shape = (n, n)
    eps = np.ones(shape, dtype=np.complex128)
    xx, yy = np.meshgrid(np.arange(n), np.arange(n), indexing='ij')
    scale = n / 256.0
    for _ in range(nb_disks):
        cx, cy = rng.uniform(0, n, size=2)
        radius = rng.uniform(5, 20) * scale
        ri = rng.uniform(1.3, 1.6)
        inside = (xx - cx) ** 2 + (yy - cy) ** 2 <= radius ** 2
        eps[inside] = ri ** 2 + 0.01j
    bpx = max(1, int(round(boundary_px * scale))) if boundary_px > 0 else 0
    eps = eps + 1j * ramp_extinction(shape, bpx, 0.5)
    src = np.zeros((1, *shape), dtype=np.complex128)
    sidx = min(int(round(source_index * scale)), n - 1)
    src[0, :, sidx] = _gaussian(n, n / 2, waist_px * scale)
    return dict(name=f'disks2d_{n}', shape=shape, step=STEP, wavelength=WAVELENGTH, epsilon=eps, source=src,
                bound_thickness=bpx * STEP, rtol=1e-6, maxiter=500)


def spheres_3d(n: int = 128, seed: int = 2, nb_spheres: int = 200, boundary_px: int = 12,
               sheet_index: int = 16, waist_px: float = 30.0) -> dict:
    """3D vector Maxwell, isotropic: 200 spheres of radius U(2, 8) voxels, eps = n^2, n ~ U(1.33, 1.6)."""
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    scale = n / 128.0
    eps = np.ones(shape, dtype=np.complex128)
    grid = np.ogrid[0:n, 0:n, 0:n]
    for _ in range(nb_spheres):
        c = rng.uniform(0, n, size=3)
        radius = rng.uniform(2, 8) * scale
        ri = rng.uniform(1.33, 1.6)
        lo = np.maximum(np.floor(c - radius).astype(int), 0)
        hi = np.minimum(np.ceil(c + radius).astype(int) + 1, n)
        sub = ((grid[0][lo[0]:hi[0]] - c[0]) ** 2 + (grid[1][:, lo[1]:hi[1]] - c[1]) ** 2
               + (grid[2][:, :, lo[2]:hi[2]] - c[2]) ** 2) <= radius ** 2
        block = eps[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        block[sub] = ri ** 2
    bpx = max(1, int(round(boundary_px * scale)))
    eps = eps + 1j * ramp_extinction(shape, bpx, 0.5)
    src = np.zeros((3, *shape), dtype=np.complex128)
    prof = _gaussian(n, n / 2, waist_px * scale)
    zi = min(int(round(sheet_index * scale)), n - 1)
    src[0, :, :, zi] = prof[:, None] * prof[None, :]
    return dict(name=f'spheres3d_{n}', shape=shape, step=STEP, wavelength=WAVELENGTH, epsilon=eps, source=src,
                bound_thickness=bpx * STEP, rtol=1e-5, maxiter=10000)


def haar_rotation(rng) -> np.ndarray:
    """Uniformly random rotation (Haar measure): QR of a Gaussian matrix with the sign fix, det = +1."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def voronoi_3d(n: int = 192, seed: int = 3, nb_grains: int = 64, boundary_px: int = 16,
               sheet_index: int = 24, waist_px: float = 40.0) -> dict:
    """3D anisotropic: 64 Voronoi grains of a uniaxial crystal (n_o 1.50, n_e 1.65, extinction 1e-3)."""
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    scale = n / 192.0
    seeds = rng.uniform(0, n, size=(nb_grains, 3))
    tensors = []
    for _ in range(nb_grains):
        rot = haar_rotation(rng)
        d = np.array([1.50 + 1e-3j, 1.50 + 1e-3j, 1.65 + 1e-3j]) ** 2
        tensors.append(rot @ np.diag(d) @ rot.T)
    tensors = np.asarray(tensors)  # [G, 3, 3], complex symmetric
    idx = np.arange(n, dtype=np.float64)
    label = np.empty(shape, dtype=np.int32)
    for i0 in range(n):
        d2 = ((i0 - seeds[:, 0])[:, None, None] ** 2
              + (idx[None, :, None] - seeds[:, 1][:, None, None]) ** 2
              + (idx[None, None, :] - seeds[:, 2][:, None, None]) ** 2)
        label[i0] = np.argmin(d2, axis=0)
    eps = np.moveaxis(tensors[label], (-2, -1), (0, 1)).astype(np.complex128)  # [3, 3, *shape]
    bpx = max(1, int(round(boundary_px * scale)))
    ramp = ramp_extinction(shape, bpx, 0.5)
    for i in range(3):
        eps[i, i] += 1j * ramp
    src = np.zeros((3, *shape), dtype=np.complex128)
    prof = _gaussian(n, n / 2, waist_px * scale)
    zi = min(int(round(sheet_index * scale)), n - 1)
    src[0, :, :, zi] = prof[:, None] * prof[None, :]
    return dict(name=f'voronoi3d_{n}', shape=shape, step=STEP, wavelength=WAVELENGTH, epsilon=eps, source=src,
                bound_thickness=bpx * STEP, rtol=1e-8, maxiter=10000)


def correlated_slab_2d(n: int = 512, seed: int = 4, slab_px: int = 128, sigma_px: float = 4.0,
                       nb_modes: int = 256, boundary_px: int = 16, source_index: int = 24) -> dict:
    """
    2D scalar batch: a slab ``slab_px`` thick (along axis 1) of Gaussian-correlated permittivity (white noise filtered
    by a Gaussian of width sigma, mapped through its CDF to Re eps ~ U(1.0, 2.25), Im eps = 1e-3), illuminated by
    ``nb_modes`` plane waves at angles U(-60, 60) deg: line sources along x with phase exp(i k0 sin(theta) x).
    """
    from math import erf, sqrt
    rng = np.random.default_rng(seed)
    shape = (n, n)
    slab_px = min(slab_px, n // 2)
    noise = rng.standard_normal((n, slab_px))
    f0 = np.fft.fftfreq(n)[:, None]
    f1 = np.fft.fftfreq(slab_px)[None, :]
    filt = np.exp(-2 * (np.pi * sigma_px) ** 2 * (f0 ** 2 + f1 ** 2))
    field = np.fft.ifft2(np.fft.fft2(noise) * filt).real
    field = (field - field.mean()) / field.std()
    cdf = 0.5 * (1 + np.vectorize(erf)(field / sqrt(2)))
    eps = np.ones(shape, dtype=np.complex128)
    start = (n - slab_px) // 2
    eps[:, start:start + slab_px] = 1.0 + 1.25 * cdf + 1e-3j
    bpx = boundary_px
    eps = eps + 1j * ramp_extinction(shape, bpx, 0.5)
    theta = rng.uniform(-np.pi / 3, np.pi / 3, size=nb_modes)
    k0 = 2 * np.pi / WAVELENGTH
    x = np.arange(n) * STEP
    src = np.zeros((nb_modes, 1, *shape), dtype=np.complex128)
    sidx = min(source_index, n - 1)
    src[:, 0, :, sidx] = np.exp(1j * k0 * np.sin(theta)[:, None] * x[None, :])
    return dict(name=f'slab2d_{n}x{nb_modes}', shape=shape, step=STEP, wavelength=WAVELENGTH, epsilon=eps,
                source=src, bound_thickness=bpx * STEP, rtol=1e-8, maxiter=10000, theta=theta)


def design_3d(n: int = 128, seed: int = 5, design_px: int = 64, boundary_px: int = 16, sheet_index: int = 16,
              detector_index: int = 112, patch_px: int = 9, waist_px: float = 30.0, nb_sources: int = 1) -> dict:
    """
    3D scalar adjoint workload: eps ~ U(1.0, 2.25) in the central design cube, 1 elsewhere, a Gaussian beam sheet at
    z = ``sheet_index`` and a detector patch at z = ``detector_index``.  An absorbing 16-px ramp is added so that the
    problem is not periodic.  With ``nb_sources > 1`` the sheet is laterally shifted per source.
    """
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    scale = n / 128.0
    dpx = max(2, int(round(design_px * scale)))
    lo = (n - dpx) // 2
    eps = np.ones(shape, dtype=np.complex128)
    eps[lo:lo + dpx, lo:lo + dpx, lo:lo + dpx] = rng.uniform(1.0, 2.25, size=(dpx, dpx, dpx))
    bpx = max(1, int(round(boundary_px * scale)))
    eps = eps + 1j * ramp_extinction(shape, bpx, 0.5)
    zi = min(int(round(sheet_index * scale)), n - 1)
    src = np.zeros((nb_sources, 1, *shape), dtype=np.complex128)
    shifts = rng.uniform(-0.15 * n, 0.15 * n, size=(nb_sources, 2)) if nb_sources > 1 else np.zeros((1, 2))
    for b in range(nb_sources):
        px = _gaussian(n, n / 2 + shifts[b, 0], waist_px * scale)
        py = _gaussian(n, n / 2 + shifts[b, 1], waist_px * scale)
        src[b, 0, :, :, zi] = px[:, None] * py[None, :]
    det = min(int(round(detector_index * scale)), n - 1)
    p = max(1, int(round(patch_px * scale)) if scale < 1 else patch_px)
    c = n // 2
    patch = (slice(c - p // 2, c - p // 2 + p), slice(c - p // 2, c - p // 2 + p), det)
    design = (slice(lo, lo + dpx),) * 3
    if nb_sources == 1:
        src = src[0]
    return dict(name=f'design3d_{n}', shape=shape, step=STEP, wavelength=WAVELENGTH, epsilon=eps, source=src,
                bound_thickness=bpx * STEP, rtol=1e-6, maxiter=10000, patch=patch, design=design)


WORKLOADS = {
    'disks2d': disks_2d,
    'spheres3d': spheres_3d,
    'voronoi3d': voronoi_3d,
    'slab2d': correlated_slab_2d,
    'design3d': design_3d,
}
