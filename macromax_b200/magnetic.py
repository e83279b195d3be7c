"""
The split-Richardson iteration for magnetic and bi-(an)isotropic media on the device.

Set-up: the magnetic branch of ``Solution.__prepare_preconditioner`` (solver.py:270-493) in host FP64: with
mu_inv = mu^-1, chi_EH beta = -i xi mu_inv, chi_HE beta = i mu_inv zeta and E_xz = epsilon - xi mu_inv zeta, alpha_r
and beta minimise (by the reference's 2-parameter Nelder-Mead) beta times the sum of the largest singular values
sigma_D^2 sigma_HH(beta) + sigma_D (sigma_EH + sigma_HE) / beta + sigma_EE(alpha_r, beta) (sigma_D = the largest
spatial frequency over k0), and alpha_i is that sum; then the kernel-width bias (solver.py:591-627).

Iteration (solver.py:1064-1098 with chi_op of solver.py:531-552):
    d = chi[G(chi E + s') - E],   chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x),   D = i k x
run by mmx_magnetic_iterate: batched FFTs, the spectral curl, the dyadic Green multiply, the 3x3 block products and
a fused update that also accumulates the FP64 norms.  The four blocks and s' stay at their set-up alpha0: a
divergence-guard rejection (alpha_i x 1.5) only changes the scale factors the kernels derive from the right-hand
side's device state (solver.py:514-528).  The accept / reject decision and the stop rule are taken on the device, so
a chunk of iterations replays from one CUDA graph without a host round trip.
"""
from __future__ import annotations

from math import inf

import numpy as np
import scipy.constants as const
import scipy.optimize
import torch

from . import _native as nat
from .bound import PeriodicBound, is_electric
from .bound import is_magnetic as has_magnetic_bound
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
    if has_magnetic_bound(bound) and np.any(np.asarray(bound.magnetic_susceptibility) != 0):
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
        if is_electric(self._bound):
            chi_b = np.asarray(self._bound.electric_susceptibility)
            epsilon = epsilon + (eye * chi_b if not _is_scalar(epsilon) else chi_b)
        if has_magnetic_bound(self._bound):
            chi_b = np.asarray(self._bound.magnetic_susceptibility)
            mu = mu + (eye * chi_b if not _is_scalar(mu) else chi_b)
        self._pre = MagneticPreconditioner(epsilon, func2arr(xi), func2arr(zeta), mu, grid.step, self._wavenumber,
                                           self._bound.thickness, float(np.finfo(self._dtype).eps))
        self._alpha0 = self._pre.alpha
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

            self._E, self._src = field(), field()
            self._work = [field() for _ in range(7)]
            self._state = torch.zeros(nat.STATE_DTYPE.itemsize, dtype=torch.uint8, device=self._device)
        self._buffers = nat.MagneticBuffers(
            E=nat.device_ptr(self._E), src=nat.device_ptr(self._src), chi_ee=nat.device_ptr(self._ee),
            chi_eh=nat.device_ptr(self._eh), chi_he=nat.device_ptr(self._he), chi_hh=nat.device_ptr(self._hh),
            work=(nat.ctypes.c_void_p * 7)(*[t.data_ptr() for t in self._work]))
        st = np.zeros(1, dtype=nat.STATE_DTYPE)
        st['alpha_re'] = st['alpha0_re'] = self._alpha0.real
        st['alpha_im'] = st['alpha0_im'] = self._alpha0.imag
        st['prev_norm'] = inf
        st['rtol'] = -1.0
        st['maxiter'] = inf
        st['active'] = 1
        self._write_state(st)
        self.source_distribution = source_distribution
        self.E = initial_field

    # -- device state (mmx_rhs_state) --------------------------------------------------------------------------------
    def _read_state(self) -> np.ndarray:
        return self._state.cpu().numpy().view(nat.STATE_DTYPE).copy()

    def _write_state(self, st: np.ndarray):
        raw = np.ascontiguousarray(st, dtype=nat.STATE_DTYPE).view(np.uint8)
        self._state.copy_(torch.from_numpy(raw.copy()).to(self._device))

    def _set_state(self, **values):
        st = self._read_state()
        for k, v in values.items():
            st[k] = v
        self._write_state(st)

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
        st = self._read_state()[0]
        return complex(st['alpha_re'], st['alpha_im'])

    @property
    def beta(self) -> float:
        return self._pre.beta

    @property
    def iteration(self) -> int:
        return int(self._read_state()[0]['iteration'])

    @iteration.setter
    def iteration(self, it: int = 0):
        self._set_state(iteration=int(it))

    @property
    def previous_update_norm(self) -> float:
        """solver.py:1018-1024: in field units (the stored field is E k0^2)."""
        return float(self._read_state()[0]['prev_norm'] / self._wavenumber ** 2)

    @property
    def rejections(self) -> int:
        return int(self._read_state()[0]['rejections'])

    @property
    def residue(self) -> float:
        """solver.py:1026-1042: the last accepted update norm over the field norm (as of the last iteration)."""
        st = self._read_state()[0]
        prev = float(st['prev_norm'])
        if not np.isfinite(prev):
            return inf
        return float(st['residue'])

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
        self._set_state(prev_norm=inf)

    @property
    def E(self) -> np.ndarray:
        f = self._E * (1.0 / self._wavenumber ** 2)
        return f.cpu().numpy().reshape(3, *self._grid.shape).astype(self._dtype, copy=False)

    @E.setter
    def E(self, E):
        E = np.broadcast_to(np.asarray(E), (3, *self._grid.shape)) * self._wavenumber ** 2
        self._E.copy_(torch.from_numpy(np.ascontiguousarray(E, dtype=self._dtype)).reshape(3, -1).to(self._device))
        self._set_state(prev_norm=inf)

    # -- iteration ---------------------------------------------------------------------------------------------------
    def _run(self, niter: int):
        import ctypes
        stream = torch.cuda.current_stream(self._device).cuda_stream
        nat.call('mmx_magnetic_iterate', self._plan.handle, ctypes.byref(self._buffers),
                 nat.device_ptr(self._state), int(niter), 1, ctypes.c_void_p(stream) if stream else None)

    def _check(self, st):
        if int(st['status']) == nat.MMX_STATUS_ZERODIV:
            raise ZeroDivisionError('float division by zero')

    def __iter__(self):
        """solver.py:1049-1098: every next() runs one iteration on the device; obtaining the iterator resets the
        iteration count (solver.py:1063)."""
        self._set_state(rtol=-1.0, maxiter=inf, active=1, status=0, iteration=0)
        while True:
            self._run(1)
            self._check(self._read_state()[0])
            yield self

    def solve(self, callback=None, rtol: float = 0, maxiter=inf, chunk: int = 8, max_chunk: int = 64):
        """solver.py:1100-1123.  With no callback (or the reference's default one) the stop rule runs on the device
        in chunks of iterations; any other callback is called after every iteration."""
        from .solver import _default_callback
        if callback is _default_callback:
            callback, rtol, maxiter = None, 1e-4, 1e4
        if callback is not None:
            for sol in self:
                if not callback(sol):
                    break
            return self
        self._set_state(rtol=float(rtol), maxiter=float(maxiter), active=1, status=0, iteration=0)
        while True:
            self._run(chunk)
            st = self._read_state()[0]
            self._check(st)
            if not st['active']:
                break
            chunk = min(2 * chunk, max_chunk)
        return self

    def close(self):
        self._plan.close()
