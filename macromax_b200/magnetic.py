"""
The split-Richardson iteration for magnetic and bi-(an)isotropic media on the device.

Set-up: the magnetic branch of ``Solution.__prepare_preconditioner`` (solver.py:270-493) in host FP64: with
mu_inv = mu^-1, chi_EH beta = -i xi mu_inv, chi_HE beta = i mu_inv zeta and E_xz = epsilon - xi mu_inv zeta, alpha_r
and beta minimise (by the reference's 2-parameter Nelder-Mead) beta times the sum of the largest singular values
sigma_D^2 sigma_HH(beta) + sigma_D (sigma_EH + sigma_HE) / beta + sigma_EE(alpha_r, beta) (sigma_D = the largest
spatial frequency over k0), and alpha_i is that sum; then the kernel-width bias (solver.py:591-627).

Iteration (solver.py:1064-1098 with chi_op of solver.py:531-552):
    d = chi[G(chi E + s') - E],   chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x),   D = i k x
composed of device kernels: batched FFTs (mmx_fftn), the spectral curl (mmx_curl_ft), the dyadic Green multiply
(mmx_green_ft), the 3x3 block products (mmx_chi_mix) and linear combinations (mmx_axpby); FP64 norms (mmx_norm).
The four blocks and s' stay at their set-up alpha0: a divergence-guard rejection (alpha_i x 1.5) only changes the
complex scale factors passed to mmx_chi_mix (solver.py:514-528).  The accept / reject decision is taken on the host
after each iteration, as in the reference loop.
"""
from __future__ import annotations

from math import inf

import numpy as np
import scipy.constants as const
import scipy.optimize
import torch

from . import _native as nat
from .bound import Electric, Magnetic, PeriodicBound
from .grid import Grid
from .preconditioner import has_gain, increase_bias


def _is_scalar(a) -> bool:
    a = np.asarray(a)
    return a.ndim == 0 or (a.shape[0] == 1 and (a.ndim == 1 or a.shape[1] == 1))


def _matrix_field(a, ndim):
    a = np.asarray(a, dtype=np.complex128)
    while a.ndim < ndim + 2:
        a = a[np.newaxis]
    if a.shape[0] == 1 and a.shape[1] > 1:
        a = a.swapaxes(0, 1)
    return a


def _adj(m):
    return np.conj(np.swapaxes(m, 0, 1))


def _mul(a, b):
    if _is_scalar(a) or _is_scalar(b):
        return a * b
    return np.einsum('ij...,jk...->ik...', a, b)


def _largest_eigenvalue(h) -> float:
    """Largest |eigenvalue| of a Hermitian matrix field (a scalar field: its largest |value|)."""
    if _is_scalar(h):
        return float(np.amax(np.abs(h)))
    return float(np.amax(np.abs(np.linalg.eigvalsh(np.moveaxis(h, (0, 1), (-2, -1))))))


def is_magnetic(xi, zeta, mu) -> bool:
    """solver.py:305-307: xi or zeta non-zero, or mu not constant."""
    mu = np.asarray(mu)
    return not (np.allclose(xi, 0.0) and np.allclose(zeta, 0.0) and np.allclose(mu, mu.ravel()[0]))


def needs_magnetic_solver(grid, epsilon=None, xi=0.0, zeta=0.0, mu=1.0, refractive_index=None, bound=None) -> bool:
    """True for the media the reference iterates with its magnetic chi_op: xi or zeta non-zero, mu not constant
    (including a magnetic boundary), or, when epsilon is derived from it, a negative (scalar) refractive index."""
    def func2arr(f):
        return f(*grid) if callable(f) else np.asarray(f)

    mu_arr = func2arr(mu)
    if isinstance(bound, Magnetic) and np.any(np.asarray(bound.magnetic_susceptibility) != 0):
        return True
    if epsilon is None and refractive_index is not None:
        n = _matrix_field(func2arr(refractive_index), grid.ndim)
        if _is_scalar(n) and np.any(n.real < 0):
            return True
    return is_magnetic(func2arr(xi), func2arr(zeta), mu_arr)


class MagneticPreconditioner:
    def __init__(self, epsilon, xi, zeta, mu, step, wavenumber: float, thickness, eps_dtype: float):
        ndim = len(np.atleast_1d(step))
        eye = np.eye(3).reshape(3, 3, *([1] * ndim))

        def subtract(left, right):  # backend/__init__.py:397-413
            if not _is_scalar(left) or not _is_scalar(right):
                if _is_scalar(left):
                    left = eye * _matrix_field(left, ndim)
                if _is_scalar(right):
                    right = eye * _matrix_field(right, ndim)
            return left - right

        eps = _matrix_field(epsilon, ndim)
        xi = _matrix_field(xi, ndim)
        zeta = _matrix_field(zeta, ndim)
        mu = _matrix_field(mu, ndim)
        if _is_scalar(mu):
            mu_inv = _matrix_field(1.0, ndim) / mu
        else:
            mu_inv = np.moveaxis(np.linalg.inv(np.moveaxis(mu, (0, 1), (-2, -1))), (-2, -1), (0, 1))
        mu_inv_t = _adj(mu_inv)
        mu_inv2 = _mul(mu_inv_t, mu_inv)

        def chi_hh(beta_):
            return subtract(1.0, mu_inv / beta_)

        def sigma_hh(beta_):
            h = mu_inv2 + subtract(np.abs(beta_) ** 2, mu_inv_t * beta_ + mu_inv * np.conj(beta_))
            return _largest_eigenvalue(h) ** 0.5 / abs(beta_)

        chi_eh_b = -1.0j * _mul(xi, mu_inv)
        chi_he_b = 1.0j * _mul(mu_inv, zeta)
        e_xz = subtract(eps, _mul(xi, -1.0j * chi_he_b))

        def sigma_ee(alpha_, beta_):
            ab = np.asarray(np.real(alpha_) * beta_, dtype=np.complex128)
            res = _adj(e_xz) * ab
            res = res + e_xz * np.conj(ab)
            res = subtract(np.abs(ab) ** 2, res)
            res = res + _mul(_adj(e_xz), e_xz)
            return float(_largest_eigenvalue(res)) ** 0.5 / abs(float(beta_))

        sigma_d = float(np.linalg.norm(2.0 * np.pi / (2.0 * np.asarray(step, dtype=float)))) / wavenumber
        sigma_he = _largest_eigenvalue(_mul(_adj(chi_he_b), chi_he_b)) ** 0.5
        sigma_eh = _largest_eigenvalue(_mul(_adj(chi_eh_b), chi_eh_b)) ** 0.5

        def total(eta_, beta_):
            return sigma_d ** 2 * sigma_hh(beta_) + sigma_d * (sigma_eh + sigma_he) / np.abs(beta_) \
                + sigma_ee(eta_, beta_)

        def target(vec):
            beta_ = vec[1] ** 2
            return total(vec[0], beta_) * beta_ + np.maximum(0.0, beta_ - 1e-3) ** 2

        vec = scipy.optimize.fmin(target, [0, 1], initial_simplex=[[0, 1], [1, 1], [0, 0.9]], disp=False,
                                  full_output=False, ftol=0.01, xtol=0.01, maxiter=100, maxfun=200)
        self.beta = float(vec[1] ** 2)
        alpha = complex(vec[0] + 1.0j * total(vec[0], self.beta))
        self.alpha = increase_bias(alpha, thickness, wavenumber)
        self.gain = any(has_gain(a, eps_dtype) for a in (eps, xi, zeta, mu))
        s = 1.0j / self.alpha.imag / self.beta
        self.chi_eh = chi_eh_b * s
        self.chi_he = chi_he_b * s
        self.chi_hh = chi_hh(self.beta) * (1.0j / self.alpha.imag)
        chi_ee = e_xz * s
        self.chi_ee = subtract(chi_ee, self.alpha * 1.0j / self.alpha.imag) if not _is_scalar(chi_ee) else \
            chi_ee - self.alpha * 1.0j / self.alpha.imag
        self.source_scale = s


class MagneticSolution:
    """
    ``Solution`` for magnetic and bi-(an)isotropic media (the reference's magnetic code path), with the same
    constructor arguments and the same properties (E, iteration, residue, previous_update_norm, alpha, beta, ...).
    """

    def __init__(self, grid, vectorial=None, wavenumber=1.0, angular_frequency=None, vacuum_wavelength=None,
                 current_density=None, source_distribution=None, epsilon=None, xi=0.0, zeta=0.0, mu=1.0,
                 refractive_index=None, bound=None, initial_field=0.0, dtype=None, device=None):
        if not isinstance(grid, Grid):
            if np.isscalar(grid[0]):
                grid = [grid]
            grid = Grid.from_ranges(*grid)
        self._grid = grid
        if angular_frequency is not None:
            self._wavenumber = angular_frequency / const.c
        elif vacuum_wavelength is not None:
            self._wavenumber = 2 * const.pi / vacuum_wavelength
        else:
            self._wavenumber = wavenumber
        ndim = grid.ndim

        def func2arr(f):
            return f(*grid) if callable(f) else np.asarray(f)

        if source_distribution is None:
            if current_density is None:
                current_density = np.zeros((3, *grid.shape), dtype=dtype if dtype is not None else np.complex128)
            source_distribution = np.asarray(func2arr(current_density)) * (-1j * self.angular_frequency * const.mu_0)
        source_distribution = np.asarray(func2arr(source_distribution))
        if vectorial is False:
            raise ValueError('magnetic media need vector fields')
        if dtype is None:
            dtype = source_distribution.dtype
        if not np.issubdtype(dtype, np.complexfloating):
            dtype = np.complex64 if dtype in (np.float16, np.float32) else np.complex128
        self._dtype = np.dtype(dtype)
        self._precision = nat.MMX_C128 if self._dtype == np.complex128 else nat.MMX_C64
        self._tdtype = torch.complex128 if self._dtype == np.complex128 else torch.complex64
        self._bound = bound if bound is not None else PeriodicBound(grid)
        mu = func2arr(mu)
        # solver.py:227-236: a negative refractive index flips the signs of both epsilon and mu
        if epsilon is None:
            n = _matrix_field(func2arr(refractive_index) if refractive_index is not None else 1.0, ndim)
            epsilon = _mul(n, n)
            if _is_scalar(n) and np.any(n.real < 0):
                sign = 1 - 2 * (n.real < 0)
                mu = mu * sign
                epsilon = epsilon * sign
        epsilon = _matrix_field(func2arr(epsilon), ndim)
        mu = _matrix_field(mu, ndim)
        eye = np.eye(3).reshape(3, 3, *([1] * ndim))
        if isinstance(self._bound, Electric):
            chi_b = np.asarray(self._bound.electric_susceptibility)
            epsilon = epsilon + (eye * chi_b if not _is_scalar(epsilon) else chi_b)
        if isinstance(self._bound, Magnetic):
            chi_b = np.asarray(self._bound.magnetic_susceptibility)
            mu = mu + (eye * chi_b if not _is_scalar(mu) else chi_b)
        self._pre = MagneticPreconditioner(epsilon, func2arr(xi), func2arr(zeta), mu, grid.step, self._wavenumber,
                                           self._bound.thickness, float(np.finfo(self._dtype).eps))
        self._alpha0 = self._pre.alpha
        self._alpha = self._pre.alpha
        self._device = torch.device(device if device is not None else 'cuda')
        N = grid.size
        self._N = N
        with torch.cuda.device(self._device):
            self._plan = nat.Plan(grid.shape, 1, 1, self._precision)
            self._plan.set_kvectors([np.asarray(k, dtype=np.float64).ravel() for k in (grid * self._wavenumber).k])

            def blocks(b):
                b = np.asarray(b)
                full = eye * b if _is_scalar(b) else b
                full = np.broadcast_to(full, (3, 3, *grid.shape)).reshape(9, N)
                return torch.from_numpy(np.array(full, dtype=self._dtype, order='C')).to(self._device)

            self._ee, self._eh = blocks(self._pre.chi_ee), blocks(self._pre.chi_eh)
            self._he, self._hh = blocks(self._pre.chi_he), blocks(self._pre.chi_hh)

            def field():
                return torch.zeros((3, N), dtype=self._tdtype, device=self._device)

            self._E, self._t, self._u, self._w, self._dx, self._d = (field() for _ in range(6))
            self._F, self._G, self._src = field(), field(), field()
            self._norm_dev = torch.zeros(1, dtype=torch.float64, device=self._device)
        self.source_distribution = source_distribution
        self.E = initial_field
        self._iteration = 0
        self._rejections = 0

    # -- properties of the reference Solution ------------------------------------------------------------------------
    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def vectorial(self) -> bool:
        return True

    @property
    def magnetic(self) -> bool:
        return True

    @property
    def dtype(self):
        return self._dtype

    @property
    def wavenumber(self) -> float:
        return self._wavenumber

    @property
    def angular_frequency(self) -> float:
        return self._wavenumber * const.c

    @property
    def wavelength(self) -> float:
        return 2 * const.pi / self._wavenumber

    @property
    def bound(self):
        return self._bound

    @property
    def alpha(self) -> complex:
        return self._alpha

    @property
    def beta(self) -> float:
        return self._pre.beta

    @property
    def iteration(self) -> int:
        return self._iteration

    @iteration.setter
    def iteration(self, it: int = 0):
        self._iteration = int(it)

    @property
    def previous_update_norm(self) -> float:
        """solver.py:1018-1024: in field units (the stored field is E k0^2)."""
        return float(self._prev / self._wavenumber ** 2)

    @property
    def rejections(self) -> int:
        return self._rejections

    @property
    def residue(self) -> float:
        """solver.py:1026-1042: the last accepted update norm over the field norm."""
        e = self._norm(self._E)
        return self._prev / e if e > 0 and np.isfinite(self._prev) else (0.0 if self._prev == 0 else inf)

    @property
    def source_distribution(self) -> np.ndarray:
        s = self._src.cpu().numpy().reshape(3, *self._grid.shape) / (self._pre.source_scale)
        return s.astype(self._dtype)

    @source_distribution.setter
    def source_distribution(self, s):
        """solver.py:702-720: stored normalised, i s / (alpha_i beta), at the set-up alpha."""
        s = np.broadcast_to(_matrix_field(s, self._grid.ndim)[:, 0], (3, *self._grid.shape))
        self._src.copy_(torch.from_numpy(np.ascontiguousarray(s * self._pre.source_scale, dtype=self._dtype))
                        .reshape(3, -1).to(self._device))
        self._prev = inf

    @property
    def E(self) -> np.ndarray:
        f = self._E * (1.0 / self._wavenumber ** 2)
        return f.cpu().numpy().reshape(3, *self._grid.shape).astype(self._dtype, copy=False)

    @E.setter
    def E(self, E):
        E = np.broadcast_to(np.asarray(E), (3, *self._grid.shape)) * self._wavenumber ** 2
        self._E.copy_(torch.from_numpy(np.ascontiguousarray(E, dtype=self._dtype)).reshape(3, -1).to(self._device))
        self._prev = inf

    # -- device operators --------------------------------------------------------------------------------------------
    def _stream(self):
        import ctypes
        s = torch.cuda.current_stream(self._device).cuda_stream
        return ctypes.c_void_p(s) if s else None

    def _norm(self, t) -> float:
        nat.call('mmx_norm', self._plan.handle, nat.device_ptr(t), t.numel(), self._precision,
                 nat.device_ptr(self._norm_dev), self._stream())
        return float(self._norm_dev.item())

    def _axpby(self, out, x, y, a, b):
        a, b = complex(a), complex(b)
        nat.call('mmx_axpby', nat.device_ptr(out), nat.device_ptr(x), nat.device_ptr(y), a.real, a.imag, b.real,
                 b.imag, out.numel(), self._precision, self._stream())

    def _curl(self, x, out):
        """out = D x = IFFT(i k x FFT(x))."""
        p, s = self._plan.handle, self._stream()
        nat.call('mmx_fftn', p, nat.device_ptr(x), nat.device_ptr(self._F), 3, 0, s)
        nat.call('mmx_curl_ft', p, nat.device_ptr(self._F), nat.device_ptr(self._G), s)
        nat.call('mmx_fftn', p, nat.device_ptr(self._G), nat.device_ptr(out), 3, 1, s)

    def _coef(self):
        """chi(alpha) from the blocks at alpha0 (solver.py:514-528): EE = f EE0 + i (alpha0 - alpha) / alpha_i I,
        the other blocks and s' scaled by f = alpha0_i / alpha_i."""
        import ctypes
        a0, a = self._alpha0, self._alpha
        f = a0.imag / a.imag
        ee_b = 1.0j * (a0 - a) / a.imag
        vals = [f, 0.0, ee_b.real, ee_b.imag, f, 0.0, f, 0.0, f, 0.0]
        return (ctypes.c_double * 10)(*vals)

    def _chi_op(self, x, out):
        self._curl(x, self._dx)
        nat.call('mmx_chi_mix', nat.device_ptr(x), nat.device_ptr(self._dx), nat.device_ptr(self._ee),
                 nat.device_ptr(self._eh), nat.device_ptr(self._he), nat.device_ptr(self._hh), self._coef(),
                 nat.device_ptr(self._u), nat.device_ptr(self._w), self._N, self._precision, self._stream())
        self._curl(self._w, self._dx)
        self._axpby(out, self._u, self._dx, 1.0, 1.0)

    def _update(self):
        """d = chi [G (chi E + s') - E] into self._d."""
        p, s = self._plan.handle, self._stream()
        self._chi_op(self._E, self._t)
        self._axpby(self._t, self._t, self._src, 1.0, self._alpha0.imag / self._alpha.imag)
        nat.call('mmx_fftn', p, nat.device_ptr(self._t), nat.device_ptr(self._F), 3, 0, s)
        nat.call('mmx_green_ft', p, nat.device_ptr(self._F), self._alpha.real, self._alpha.imag, s)
        nat.call('mmx_fftn', p, nat.device_ptr(self._F), nat.device_ptr(self._t), 3, 1, s)
        self._axpby(self._t, self._t, self._E, 1.0, -1.0)
        self._chi_op(self._t, self._d)

    # -- iteration ---------------------------------------------------------------------------------------------------
    def __iter__(self):
        while True:
            self._iteration += 1
            self._update()
            nu = self._norm(self._d)
            if self._prev == 0.0:
                raise ZeroDivisionError('float division by zero')
            if nu / self._prev < 1.0:
                self._axpby(self._E, self._E, self._d, 1.0, 1.0)
                self._prev = nu
            else:  # solver.py:1090-1094
                self._alpha = complex(self._alpha.real, 1.5 * self._alpha.imag)
                self._rejections += 1
            yield self

    def solve(self, callback=None, rtol: float = 0, maxiter=inf):
        if callback is None:
            def callback(sol):
                return sol.iteration < maxiter and sol.residue > rtol
        for sol in self:
            if not callback(sol):
                break
        return self

    def close(self):
        self._plan.close()
