"""
Host-side (FP64) preconditioner set-up of the split-Richardson iteration for non-magnetic media.

Follows ``Solution.__prepare_preconditioner`` (solver.py:270-493, non-magnetic branch 444-467) and
``__increase_bias_to_limit_kernel_width`` (solver.py:591-627): beta = 1 / mu, alpha_r minimises the largest
singular value of (alpha_r beta - eps) by Nelder-Mead (scipy ``fmin`` with the reference's simplex and
tolerances), alpha_i = that minimum, conjugated for pure-gain media, then raised so that the Green kernel decays
to 1e-3 across the thinnest absorbing boundary.  chi = i (eps - alpha) / alpha_i, s' = i s / (alpha_i beta).
This runs once per material, not per iteration.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.optimize


def _adjoint(m):
    return np.conj(np.swapaxes(m, 0, 1))


def _is_scalar_field(m) -> bool:
    return m.shape[0] == 1 and m.shape[1] == 1


def largest_sigma(alpha_real: float, beta: float, eps) -> float:
    """
    sqrt(largest eigenvalue of Delta) / |beta| with Delta = |ab|^2 - (eps^H ab + eps conj(ab)) + eps^H eps, the
    expanded form of (ab - eps)^H (ab - eps) evaluated term by term as in solver.py:392-401.
    """
    ab = complex(float(np.ravel(np.real(alpha_real))[0]) * beta)
    res = _adjoint(eps) * ab
    res = res + eps * np.conj(ab)
    if _is_scalar_field(eps):
        res = abs(ab) ** 2 - res
        res = res + _adjoint(eps) * eps
        return float(np.amax(np.abs(res[0, 0]))) ** 0.5 / abs(beta)
    ndim = eps.ndim - 2
    res = abs(ab) ** 2 * np.eye(3).reshape(3, 3, *([1] * ndim)) - res
    res = res + np.einsum('ij...,jk...->ik...', _adjoint(eps), eps)
    lam = np.linalg.eigvalsh(np.moveaxis(res, (0, 1), (-2, -1)))
    return float(np.amax(np.abs(lam))) ** 0.5 / abs(beta)


def has_gain(a, eps_dtype: float) -> bool:
    """solver.py:322-329."""
    h = -0.5j * (a - _adjoint(a))
    if _is_scalar_field(h):
        vals = h[0, 0].real
    else:
        vals = np.linalg.eigvalsh(np.moveaxis(h, (0, 1), (-2, -1)))
    return bool(np.any(vals < -math.sqrt(eps_dtype)))


def increase_bias(alpha: complex, thickness: np.ndarray, wavenumber: float, max_kernel_field_residue=0.001):
    """solver.py:591-627."""
    offset = alpha.imag + 0.05
    t = np.asarray(thickness)
    t = t[t != 0]
    if t.size > 0:
        bt = float(np.amin(t))
        min_kappa = np.log(max_kernel_field_residue) / (-wavenumber * bt)
        n_real = max(0.0, float(alpha.real) + min_kappa ** 2) ** 0.5
        min_offset = 2 * n_real * min_kappa
        if offset < min_offset:
            offset = min_offset
    return complex(alpha.real, offset)


class Preconditioner:
    """
    alpha, beta and the susceptibility chi = eps i / (alpha_i beta) - i alpha / alpha_i I at alpha (solver.py:480-484).
    chi is held either as a host matrix field [1|3, 1|3, *shape] or, for a 3x3 permittivity whose set-up ran on the
    device, as a device tensor [m, nvox] complex128 (``chi_device``); ``chi`` copies the latter to the host on first use.
    """

    def __init__(self, alpha: complex, beta: float, transpose: bool, chi=None, eps_field=None, chi_device=None):
        self.alpha, self.beta, self.transpose = alpha, beta, transpose
        self.eps_field = eps_field
        self._chi = chi
        self.chi_device = chi_device

    @property
    def chi_rows(self) -> int:
        if self.chi_device is not None:
            return 3 if self.chi_device.shape[0] == 9 else 1
        return int(self._chi.shape[0])

    @property
    def chi(self) -> np.ndarray:
        if self._chi is None:
            r = self.chi_rows
            self._chi = self.chi_device.cpu().numpy().reshape(r, r, *self.eps_field.shape[2:])
        return self._chi

    def chi_for_engine(self):
        """The device tensor when there is one (no host round trip), else the host matrix field."""
        return self.chi_device if self.chi_device is not None else self._chi


class DeviceSetup:
    """
    The set-up reductions of an anisotropic (3x3) permittivity on the GPU (``mmx_mat3_extremes``): the alpha
    objective and the gain / loss test, in FP64 with closed-form 3x3 eigenvalues.  On a 192^3 grid a host
    ``eigvalsh`` pass takes seconds and Nelder-Mead needs ~30 of them.
    """

    def __init__(self, eps_field: np.ndarray, device=None):
        import ctypes
        import torch
        from . import _native as nat
        self._nat, self._ctypes, self._torch = nat, ctypes, torch
        ndim = eps_field.ndim - 2
        shape = eps_field.shape[2:]
        self.nvox = int(np.prod(shape))
        dev = torch.device(device if device is not None else 'cuda')
        m = np.ascontiguousarray(np.broadcast_to(eps_field, (3, 3, *shape)).reshape(9, self.nvox), np.complex128)
        self.M = torch.from_numpy(np.require(m, requirements='W')).to(dev)  # a read-only view is copied first
        self.out = torch.zeros(2, dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            self.plan = nat.Plan((8,) * max(1, min(ndim, 1)), 1, 1, nat.MMX_C128)

    def _run(self, mode: int, ab: float):
        c = self._ctypes
        s = self._torch.cuda.current_stream().cuda_stream
        self._nat.call('mmx_mat3_extremes', self.plan.handle, c.c_void_p(self.M.data_ptr()), self.nvox, mode,
                       float(ab), c.c_void_p(self.out.data_ptr()), c.c_void_p(s) if s else None)
        return self.out.cpu().numpy()

    def sigma(self, alpha_real, beta: float) -> float:
        ab = float(np.ravel(np.real(alpha_real))[0]) * beta
        lam = float(self._run(0, ab)[1])
        return abs(lam) ** 0.5 / abs(beta)

    def gain_loss(self, eps_dtype: float):
        lo, hi = self._run(1, 0.0)
        thr = math.sqrt(eps_dtype)
        return bool(lo < -thr), bool(hi > thr)

    def chi(self, alpha: complex, beta: float):
        """chi = eps i / (alpha_i beta) - i alpha / alpha_i I (solver.py:480-484) from the permittivity already on the
        device (``mmx_chi_from_eps``), as a complex128 device tensor [9, nvox]."""
        c = self._ctypes
        s = self._torch.cuda.current_stream().cuda_stream
        sc = 1.0j / alpha.imag / beta
        d = alpha * 1.0j / alpha.imag
        out = self._torch.empty_like(self.M)
        self._nat.call('mmx_chi_from_eps', c.c_void_p(self.M.data_ptr()), 9, self.nvox, sc.real, sc.imag, d.real,
                       d.imag, c.c_void_p(out.data_ptr()), self._nat.MMX_C128, c.c_void_p(s) if s else None)
        return out


class ScalarDeviceObjective:
    """
    The alpha objective of a scalar permittivity on the GPU (``mmx_scalar_sigma``).  largest_sigma evaluates
    |ab|^2 - (conj(eps) ab + eps conj(ab)) + conj(eps) eps over the whole grid for every Nelder-Mead step; for real ab
    its imaginary part is exactly zero and its real part is (ab^2 - 2 round(Re(eps) ab)) + Re(conj(eps) eps).  The last
    term is taken from numpy once, and the device evaluates the rest with explicitly rounded FP64 operations, so every
    objective value -- and hence the simplex path and alpha -- is the host's bit for bit.
    """

    def __init__(self, eps_field: np.ndarray, device=None):
        import ctypes
        import torch
        from . import _native as nat
        self._nat, self._ctypes, self._torch = nat, ctypes, torch
        e = np.ravel(eps_field[0, 0])
        self.nvox = e.size
        xp = np.empty((self.nvox, 2), dtype=np.float64)
        xp[:, 0] = e.real
        xp[:, 1] = (np.conj(e) * e).real
        dev = torch.device(device if device is not None else 'cuda')
        self.xp = torch.from_numpy(xp).to(dev)
        self.out = torch.zeros(2, dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            self.plan = nat.Plan((8,), 1, 1, nat.MMX_C128)

    def __call__(self, alpha_real, beta: float) -> float:
        ab = float(np.ravel(np.real(alpha_real))[0]) * beta
        c = self._ctypes
        s = self._torch.cuda.current_stream().cuda_stream
        self._nat.call('mmx_scalar_sigma', self.plan.handle, c.c_void_p(self.xp.data_ptr()), self.nvox, float(ab),
                       c.c_void_p(self.out.data_ptr()), c.c_void_p(s) if s else None)
        lo, hi = self.out.cpu().numpy()
        return max(abs(float(lo)), abs(float(hi))) ** 0.5 / abs(beta)


def prepare(eps_field: np.ndarray, thickness: np.ndarray, wavenumber: float, eps_dtype: float,
            mu: complex = 1.0, objective=None, device_setup: bool = False, device=None) -> Preconditioner:
    """
    eps_field: permittivity as a matrix field [1|3, 1|3, *grid] (boundary susceptibility included).
    objective: optional callable alpha_r -> sigma replacing ``largest_sigma``.
    device_setup: evaluate the objective on the GPU: the anisotropic objective and gain/loss test (DeviceSetup), and
    the scalar objective for grids of 65536 voxels or more (ScalarDeviceObjective, the same values as the host's).
    """
    beta = float(np.real(1.0 / mu))  # solver.py:446
    dev = None
    if device_setup and not _is_scalar_field(eps_field):
        dev = DeviceSetup(eps_field, device)
        gain, loss = dev.gain_loss(eps_dtype)
    elif _is_scalar_field(eps_field):
        # for a scalar permittivity -0.5i (eps - conj(eps)) is Im(eps) exactly, so has_gain's test is on Im(eps)
        im = np.asarray(eps_field[0, 0]).imag
        thr = math.sqrt(eps_dtype)
        gain, loss = bool(np.any(im < -thr)), bool(np.any(im > thr))
    else:
        gain = has_gain(eps_field, eps_dtype)
        loss = has_gain(-eps_field, eps_dtype)
    transpose = gain and not loss
    if objective is None and dev is not None:
        def objective(ar):
            return dev.sigma(ar, beta)
    if objective is None and device_setup and _is_scalar_field(eps_field) and eps_field[0, 0].size >= (1 << 16):
        scalar_dev = ScalarDeviceObjective(eps_field, device)

        def objective(ar):
            return scalar_dev(ar, beta)
    if objective is None:
        def objective(ar):
            return largest_sigma(ar, beta, eps_field)
    alpha_real, min_value = scipy.optimize.fmin(objective, 0.0, initial_simplex=[[0.0], [1.0]], disp=False,
                                                full_output=True, ftol=0.01, xtol=0.01, maxiter=100,
                                                maxfun=100)[:2]
    alpha = complex(alpha_real[0], float(min_value))
    if transpose:
        alpha = alpha.conjugate()
    alpha = increase_bias(alpha, thickness, wavenumber)
    # solver.py:480-484 (beta == 1 / mu)
    if dev is not None and dev.nvox == int(np.prod(eps_field.shape[2:])):
        return Preconditioner(alpha=alpha, beta=beta, transpose=transpose, eps_field=eps_field,
                              chi_device=dev.chi(alpha, beta))
    chi = eps_field * (1.0j / alpha.imag / beta)
    if _is_scalar_field(chi):
        chi = chi - alpha * 1.0j / alpha.imag
    else:
        chi = chi - np.eye(3).reshape(3, 3, *([1] * (chi.ndim - 2))) * (alpha * 1.0j / alpha.imag)
    return Preconditioner(alpha=alpha, beta=beta, transpose=transpose, chi=chi, eps_field=eps_field)
