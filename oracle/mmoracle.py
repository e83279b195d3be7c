"""
CPU ORACLE for the MacroMax split-Richardson iteration -- TEST INFRASTRUCTURE ONLY.

This module restates, in plain numpy, the algorithm of the reference NumPy backend for the hot path:
the preconditioner set-up (alpha, beta, chi, normalised source) and the iteration
``E <- E + chi [G (chi E + s) - E]`` with its divergence guard.  It is the checker for the CUDA path and the timed
CPU baseline; nothing in the ``macromax_b200`` package imports it, and only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py`` (its ``cpu_baseline`` leg and its ``--impl reference`` arm) may call it.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference package itself on seeded inputs and
``tests/test_oracle_golden.py`` checks this restatement against those committed vectors (alpha, beta, the first
iterates, iteration counts and converged fields).

Scope: non-magnetic media (mu = 1, xi = zeta = 0), isotropic (scalar) or 3x3 anisotropic permittivity,
scalar (1-component) or vector (3-component) fields on 1D/2D/3D periodic grids, a ``Bound`` that contributes its
thickness to the alpha bias.  Each function cites the reference file:line it follows (paths relative to the
reference's ``python/macromax`` package).
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.optimize

try:  # multi-threaded pocketfft (the same algorithm as numpy.fft) for the timed baseline
    import scipy.fft as _sfft
except ImportError:  # pragma: no cover
    _sfft = None

_FFT_WORKERS = None  # None: numpy.fft (the reference's own choice, utils/ft/ft_implementation.py:43-57)


def set_fft_workers(workers: int | None):
    """Use scipy.fft's threaded pocketfft with ``workers`` threads (None: single-threaded numpy.fft)."""
    global _FFT_WORKERS
    _FFT_WORKERS = workers


def fftn(a, axes):
    """BackEndNumpy.ft (backend/numpy.py:112-121, 93)."""
    if _FFT_WORKERS is not None and _sfft is not None:
        return _sfft.fftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.fftn(a, axes=axes)


def ifftn(a, axes):
    """BackEndNumpy.ift (backend/numpy.py:123-133, 94): scaled by 1/N, so ift(ft(x)) == x."""
    if _FFT_WORKERS is not None and _sfft is not None:
        return _sfft.ifftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.ifftn(a, axes=axes)


def k_vectors(shape, step, wavenumber):
    """
    Open-grid k-vectors of the k0-scaled grid (utils/ft/grid.py:426-439; backend/__init__.py:651-656):
    k_a[j] = 2 pi fftfreq(n_a, step_a k0)[j], origin at index 0, broadcastable along axis a.
    """
    ndim = len(shape)
    ks = []
    for axis, (n, d) in enumerate(zip(shape, step)):
        k = 2 * np.pi * np.fft.fftfreq(n, d * wavenumber)
        view = [1] * ndim
        view[axis] = n
        ks.append(k.reshape(view))
    return ks


def k2_field(ks):
    """backend/__init__.py:658-668: |k|^2 as the sum of the squared open grids."""
    return sum(k.astype(np.complex128) ** 2 for k in ks)


def to_matrix_field(arr, ndim):
    """backend/__init__.py:355-385: prepend singleton axes until ndim + 2 axes; 1xN becomes Nx1."""
    arr = np.asarray(arr)
    while arr.ndim < ndim + 2:
        arr = arr[np.newaxis]
    if arr.shape[0] == 1 and arr.shape[1] > 1:
        arr = arr.swapaxes(0, 1)
    return arr


def adjoint(mat):
    """backend/__init__.py:387-395."""
    return np.conj(mat.swapaxes(0, 1))


def pointwise_mul(left, right):
    """backend/__init__.py:415-444: scalar fields multiply elementwise, matrix fields contract their first axes."""
    if (left.shape[0] == 1 and left.shape[1] == 1) or (right.shape[0] == 1 and right.shape[1] == 1):
        return left * right
    return np.einsum('ij...,jk...->ik...', left, right)


def largest_hermitian_eigenvalue(a, ndim):
    """amax(abs(mat3_eigh(a))) (solver.py:313-314; backend/__init__.py:670-723) for Hermitian fields."""
    if a.shape[0] == 1 and a.shape[1] == 1:
        return float(np.amax(np.abs(a[0, 0])))
    m = np.moveaxis(a, (0, 1), (-2, -1))
    return float(np.amax(np.abs(np.linalg.eigvalsh(m))))


def has_gain(a, ndim, eps):
    """solver.py:322-329: any eigenvalue of the anti-Hermitian part -(a - a^H)/2i below -sqrt(eps)."""
    h = -0.5j * (a - adjoint(a))
    if h.shape[0] == 1 and h.shape[1] == 1:
        vals = h[0, 0].real
    else:
        vals = np.linalg.eigvalsh(np.moveaxis(h, (0, 1), (-2, -1)))
    return bool(np.any(vals < -math.sqrt(eps)))


def longitudinal_projection_ft(F, ks, ndim):
    """
    backend/__init__.py:606-649: P_L F = k (k . F) / |k|^2 for the first ``ndim`` components, with the DC sample of
    those components passed through unchanged, and zeros for components >= ndim.
    """
    F = np.asarray(F)
    proj = F[0, 0] * ks[0]
    for a in range(1, ndim):
        proj = proj + ks[a] * F[a, 0]
    k2 = k2_field(ks)
    proj = np.array(proj, dtype=F.dtype)
    flat = proj.reshape(-1)
    flat[1:] /= np.broadcast_to(k2, proj.shape).reshape(-1)[1:]
    result = np.zeros_like(F)
    zero = (0,) * ndim
    for a in range(ndim):
        result[a, 0] = ks[a] * proj
        result[a, 0][zero] = F[a, 0][zero]
    return result


def curl_ft(F, ks):
    """backend/__init__.py:483-509: i k x F for 3-vector fields, with missing k components taken as zero."""
    n = 3
    out = np.zeros((n, *F.shape[1:]), dtype=np.result_type(F.dtype, np.complex64))
    for d in range(n):
        o = (d + np.array([-1, 1])) % n
        if o[0] < F.shape[0] and o[1] < len(ks):
            out[d] = ks[o[1]] * F[o[0]]
        if o[1] < F.shape[0] and o[0] < len(ks):
            out[d] -= ks[o[0]] * F[o[1]]
    return 1j * out


class OracleSolution:
    """
    Restatement of ``Solution`` (solver.py:92-268) for non-magnetic media, with the iteration of
    ``Solution.__iter__`` (solver.py:1049-1098).  All arrays are numpy; ``field`` is stored times k0^2 like the
    reference (solver.py:811-832).
    """

    def __init__(self, shape, step, wavelength, epsilon, source, bound_thickness=0.0, dtype=np.complex128,
                 initial_field=0.0):
        self.shape = tuple(int(s) for s in shape)
        self.ndim = len(self.shape)
        self.step = np.broadcast_to(np.asarray(step, dtype=np.float64), (self.ndim,)).copy()
        self.wavenumber = 2 * np.pi / wavelength
        self.dtype = np.dtype(dtype)
        self.eps_dtype = float(np.finfo(self.dtype).eps)
        source = np.asarray(source)
        self.vectorial = source.ndim > self.ndim and source.shape[0] == 3
        self.nb_pol = 3 if self.vectorial else 1
        self.ft_axes = tuple(range(2, 2 + self.ndim))
        self.ks = k_vectors(self.shape, self.step, self.wavenumber)
        self.thickness = np.broadcast_to(np.asarray(bound_thickness, dtype=np.float64), (self.ndim, 2))
        # solver.py:214-219, 831
        self.field = np.zeros((self.nb_pol, 1, *self.shape), dtype=self.dtype)
        self.field[...] = np.asarray(initial_field) * self.wavenumber ** 2
        self.previous_update_norm = np.inf
        self.iteration = 0
        self.rejections = 0
        self._prepare(epsilon, source)

    # -- set-up ---------------------------------------------------------------------------------------------------
    def _sigma_ee(self, alpha_real, beta, eps_field):
        """solver.py:392-401: sqrt(largest eigenvalue of (ab - eps)^H (ab - eps)) / |beta|."""
        ab = np.asarray(np.real(alpha_real) * beta, dtype=np.complex128)
        res = adjoint(eps_field) * ab
        res = res + eps_field * np.conj(ab)
        if res.shape[0] == 1 and res.shape[1] == 1:
            res = np.abs(ab) ** 2 - res
        else:
            res = np.abs(ab) ** 2 * np.eye(3).reshape(3, 3, *([1] * self.ndim)) - res
        res = res + pointwise_mul(adjoint(eps_field), eps_field)
        return float(largest_hermitian_eigenvalue(res, self.ndim)) ** 0.5 / abs(float(beta))

    def _increase_bias(self, alpha, max_kernel_field_residue=0.001):
        """solver.py:591-627."""
        offset = alpha.imag + 0.05
        thicknesses = self.thickness[self.thickness != 0]
        if thicknesses.size > 0:
            bound_thickness = np.amin(thicknesses)
            min_kappa = np.log(max_kernel_field_residue) / (-self.wavenumber * bound_thickness)
            n_real = np.maximum(0, float(alpha.real) + min_kappa ** 2) ** 0.5
            min_offset = 2 * n_real * min_kappa
            if offset < min_offset:
                offset = min_offset
        return alpha.real + 1j * offset

    def _prepare(self, epsilon, source):
        """solver.py:270-493 for mu = 1, xi = zeta = 0 (non-magnetic branch 444-467)."""
        eps_field = to_matrix_field(np.asarray(epsilon, dtype=np.complex128), self.ndim)
        if not (eps_field.shape[0] == 1 and eps_field.shape[1] == 1) and not self.vectorial:
            raise ValueError('an anisotropic permittivity needs a vector field')
        gain = has_gain(eps_field, self.ndim, self.eps_dtype)
        loss = has_gain(-eps_field, self.ndim, self.eps_dtype)
        self.transpose = gain and not loss  # solver.py:334-336
        self.beta = 1.0  # solver.py:446: real(first(inv(mu))) with mu = 1

        def target(alpha_):
            return self._sigma_ee(alpha_, self.beta, eps_field)

        alpha_real, min_value = scipy.optimize.fmin(target, 0.0, initial_simplex=[[0.0], [1.0]], disp=False,
                                                    full_output=True, ftol=0.01, xtol=0.01, maxiter=100,
                                                    maxfun=100)[:2]  # solver.py:452-456
        alpha = alpha_real[0] + 1.0j * min_value
        if self.transpose:
            alpha = alpha.conj()
        alpha = self._increase_bias(alpha)  # solver.py:470
        self.alpha = alpha
        # solver.py:480-484
        chi = eps_field.astype(self.dtype) * (1.0j / self.alpha.imag / self.beta)
        if chi.shape[0] == 1:
            chi = chi - self.alpha * 1.0j / self.alpha.imag
        else:
            chi = chi - np.eye(3).reshape(3, 3, *([1] * self.ndim)) * (self.alpha * 1.0j / self.alpha.imag)
        self.chi = np.asarray(chi, dtype=self.dtype)
        self.epsilon_field = eps_field
        # solver.py:702-720 (source setter) then 492 (__update_operators with the same alpha)
        src = to_matrix_field(np.asarray(source, dtype=self.dtype), self.ndim)
        if src.shape[0] != self.nb_pol:
            src = np.broadcast_to(src, (self.nb_pol, *src.shape[1:]))
        self.source_normalized = np.asarray(src * (1.0j / self.alpha.imag / self.beta), dtype=self.dtype)
        self.previous_update_norm = np.inf
        self._update_operators(alpha)

    def _update_operators(self, alpha):
        """solver.py:496-589 (non-magnetic): rescale s', shift chi to the new alpha, rebuild g."""
        old = self.alpha
        self.source_normalized *= old.imag / alpha.imag
        chi = self.chi / (1.0j / old.imag)
        if chi.shape[0] == 1:
            chi = chi + (old - alpha)
        else:
            chi = chi + np.eye(3).reshape(3, 3, *([1] * self.ndim)) * (old - alpha)
        self.chi = np.asarray(chi * (1.0j / alpha.imag), dtype=self.dtype)
        self.alpha = alpha
        k2 = k2_field(self.ks).astype(self.dtype)
        self.g_scalar_ft = (np.asarray(-1.0j, self.dtype) * np.asarray(self.alpha.imag, self.dtype)
                            / (k2 - np.asarray(self.alpha, self.dtype)))

    # -- operators --------------------------------------------------------------------------------------------------
    def chi_op(self, x):
        """solver.py:554-562."""
        return np.asarray(pointwise_mul(self.chi, x), dtype=self.dtype)

    def g_ft_op(self, F):
        """solver.py:570-581."""
        if self.vectorial:
            pil = longitudinal_projection_ft(F, self.ks, self.ndim).astype(self.dtype)
            F = F - pil
            F = F * self.g_scalar_ft
            pil = pil * np.asarray(1.0j * self.alpha.imag / self.alpha, dtype=self.dtype)
            return np.asarray(F + pil, dtype=self.dtype)
        return np.asarray(F * self.g_scalar_ft, dtype=self.dtype)

    def green_op(self, x):
        """solver.py:583-584 via backend/__init__.py:306-319."""
        return np.asarray(ifftn(self.g_ft_op(np.asarray(fftn(x, self.ft_axes), dtype=self.dtype)), self.ft_axes),
                          dtype=self.dtype)

    def update(self):
        """d = chi [G (chi E + s') - E] (solver.py:1070-1075)."""
        d = self.chi_op(self.field)
        d = d + self.source_normalized
        d = self.green_op(d)
        d = d - self.field
        return self.chi_op(d)

    # -- iteration --------------------------------------------------------------------------------------------------
    def advance(self):
        """One pass of ``Solution.__iter__`` (solver.py:1064-1098)."""
        self.iteration += 1
        d = self.update()
        nu = float(np.linalg.norm(d.ravel()))
        rel = nu / self.previous_update_norm
        if rel < 1:
            self.field += d
            self.previous_update_norm = nu
            return True
        alpha_new = self.alpha.real + 1.50j * self.alpha.imag
        self._update_operators(alpha_new)
        self.rejections += 1
        return False

    @property
    def residue(self):
        """solver.py:1026-1042."""
        if self.previous_update_norm > 0:
            return float(self.previous_update_norm / np.linalg.norm(self.field.ravel()))
        return 0.0

    @property
    def E(self):
        """solver.py:811-821."""
        return self.field[:, 0] / self.wavenumber ** 2

    def solve(self, rtol=1e-6, maxiter=10000, record=(), callback=None):
        """solver.py:1100-1123 with the callback ``iteration < maxiter and residue > rtol``; stores E at ``record``."""
        recorded = {}
        self.iteration = 0  # solver.py:1063
        while True:
            self.advance()
            if self.iteration in record:
                recorded[self.iteration] = self.E.copy()
            keep_going = callback(self) if callback is not None else (self.iteration < maxiter
                                                                      and self.residue > rtol)
            if not keep_going:
                break
        return recorded


def from_workload(wl: dict, dtype=np.complex128, batch_index: int | None = None) -> OracleSolution:
    """Build an ``OracleSolution`` from a ``macromax_b200.workloads`` dictionary."""
    src = wl['source']
    if batch_index is not None:
        src = src[batch_index]
    return OracleSolution(wl['shape'], wl['step'], wl['wavelength'], wl['epsilon'], src,
                          bound_thickness=wl.get('bound_thickness', 0.0), dtype=dtype)


def inverse_green_op(sol: OracleSolution, x):
    """
    G^{-1} x for the preconditioned Green operator of ``sol``: scalar 1/g, vector P_T/g + P_L/(i a_i / a).
    Used to check the defect s + chi x - G^{-1} x of the mixed-precision refinement.
    """
    F = np.asarray(fftn(x, sol.ft_axes), dtype=np.complex128)
    g = sol.g_scalar_ft.astype(np.complex128)
    if sol.vectorial:
        pil = longitudinal_projection_ft(F, sol.ks, sol.ndim)
        h = 1.0j * sol.alpha.imag / sol.alpha
        F = (F - pil) / g + pil / h
    else:
        F = F / g
    return ifftn(F, sol.ft_axes)


def num_threads() -> int:
    return os.cpu_count() or 1


class MagneticOracleSolution(OracleSolution):
    """
    Restatement of ``Solution`` for magnetic and bi-(an)isotropic media: the magnetic branch of
    ``__prepare_preconditioner`` (solver.py:270-493: alpha and beta by a 2-parameter Nelder-Mead search over the sum of
    the largest singular values of the E-E, E-H, H-E and H-H blocks), the magnetic ``chi_op`` (solver.py:531-552:
    chi_EE E + chi_HE D E + D(chi_EH E + chi_HH D E), D the spectral curl of backend/__init__.py:472-509) and the
    rescaling of all four blocks in ``__update_operators`` (solver.py:514-528).  Fields are vectorial.
    """

    def __init__(self, shape, step, wavelength, epsilon, source, xi=0.0, zeta=0.0, mu=1.0, bound_thickness=0.0,
                 dtype=np.complex128, initial_field=0.0):
        self._material = (xi, zeta, mu)
        super().__init__(shape, step, wavelength, epsilon, source, bound_thickness=bound_thickness, dtype=dtype,
                         initial_field=initial_field)

    # backend-like helpers for matrix fields with scalar fields as multiples of the 3x3 identity
    def _eye(self):
        return np.eye(3).reshape(3, 3, *([1] * self.ndim)).astype(self.dtype)

    @staticmethod
    def _is_scalar(a):
        a = np.asarray(a)
        return a.ndim == 0 or (a.shape[0] == 1 and (a.ndim == 1 or a.shape[1] == 1))

    def _field(self, a):
        return to_matrix_field(np.asarray(a, dtype=self.dtype), self.ndim)

    def _subtract(self, left, right):
        """backend/__init__.py:397-413: a scalar term becomes a multiple of the identity next to a matrix."""
        if not self._is_scalar(left) or not self._is_scalar(right):
            if self._is_scalar(left):
                left = self._eye() * self._field(left)
            if self._is_scalar(right):
                right = self._eye() * self._field(right)
        return left - right

    def _inv(self, m):
        """backend/numpy.py:135-170 (ldivide with numerator 1)."""
        m = self._field(m)
        if self._is_scalar(m):
            return np.asarray(self._field(1.0), dtype=self.dtype) / m
        moved = np.moveaxis(m, (0, 1), (-2, -1))
        return np.moveaxis(np.linalg.inv(moved), (-2, -1), (0, 1))

    def _largest_eigenvalue(self, a):
        return largest_hermitian_eigenvalue(a, self.ndim)

    def _prepare(self, epsilon, source):
        if not self.vectorial:
            raise ValueError('magnetic media need a vector field')
        xi, zeta, mu = self._material
        eps = self._field(epsilon)
        xi = self._field(xi)
        zeta = self._field(zeta)
        mu = self._field(mu)
        gain = any(has_gain(a, self.ndim, self.eps_dtype) for a in (eps, xi, zeta, mu))
        loss = any(has_gain(-a, self.ndim, self.eps_dtype) for a in (eps, xi, zeta, mu))
        self.transpose = gain and not loss  # not applied to alpha in the magnetic branch (solver.py:421-442)
        mu_inv = self._inv(mu)
        mu_inv_t = adjoint(mu_inv)
        mu_inv2 = pointwise_mul(mu_inv_t, mu_inv)

        def chi_hh(beta_):
            return self._subtract(1.0, mu_inv / beta_)

        def chi_hh_beta2(beta_):
            return mu_inv2 + self._subtract(np.abs(beta_) ** 2, mu_inv_t * beta_ + mu_inv * np.conj(beta_))

        def sigma_hh(beta_):
            return self._largest_eigenvalue(chi_hh_beta2(beta_)) ** 0.5 / abs(beta_)

        chi_eh_beta = -1.0j * pointwise_mul(xi, mu_inv)
        chi_he_beta = 1.0j * pointwise_mul(mu_inv, zeta)
        e_xz = self._subtract(eps, pointwise_mul(xi, -1.0j * chi_he_beta))

        def delta_ee_beta2(alpha_, beta_):
            ab = np.asarray(np.real(alpha_) * beta_, dtype=self.dtype)
            res = adjoint(e_xz) * ab
            res = res + e_xz * np.conj(ab)
            res = self._subtract(np.abs(ab) ** 2, res)
            return res + pointwise_mul(adjoint(e_xz), e_xz)

        def sigma_ee(alpha_, beta_):
            return float(self._largest_eigenvalue(delta_ee_beta2(alpha_, beta_))) ** 0.5 / abs(float(beta_))

        sigma_d = float(np.linalg.norm(2.0 * np.pi / (2.0 * self.step))) / self.wavenumber
        sigma_he = self._largest_eigenvalue(pointwise_mul(adjoint(chi_he_beta), chi_he_beta)) ** 0.5
        sigma_eh = self._largest_eigenvalue(pointwise_mul(adjoint(chi_eh_beta), chi_eh_beta)) ** 0.5

        def singular_value_sum(eta_, beta_):
            return sigma_d ** 2 * sigma_hh(beta_) + sigma_d * (sigma_eh + sigma_he) / np.abs(beta_) \
                + sigma_ee(eta_, beta_)

        def target(vec):
            beta_ = vec[1] ** 2  # positive
            return singular_value_sum(vec[0], beta_) * beta_ + np.maximum(0.0, beta_ - 1e-3) ** 2

        vec = scipy.optimize.fmin(target, [0, 1], initial_simplex=[[0, 1], [1, 1], [0, 0.9]], disp=False,
                                  full_output=False, ftol=0.01, xtol=0.01, maxiter=100, maxfun=200)
        self.beta = float(vec[1] ** 2)
        alpha = vec[0] + 1.0j * singular_value_sum(vec[0], self.beta)
        alpha = self._increase_bias(complex(alpha))
        self.alpha = alpha
        s = 1.0j / alpha.imag / self.beta
        self.chi_eh = np.asarray(chi_eh_beta * s, dtype=self.dtype)
        self.chi_he = np.asarray(chi_he_beta * s, dtype=self.dtype)
        self.chi_hh = np.asarray(chi_hh(self.beta) * (1.0j / alpha.imag), dtype=self.dtype)
        chi = e_xz * s
        if chi.shape[0] == 1:
            chi = chi - alpha * 1.0j / alpha.imag
        else:
            chi = chi - self._eye() * (alpha * 1.0j / alpha.imag)
        self.chi = np.asarray(chi, dtype=self.dtype)
        self.epsilon_field = eps
        src = to_matrix_field(np.asarray(source, dtype=self.dtype), self.ndim)
        if src.shape[0] != self.nb_pol:
            src = np.broadcast_to(src, (self.nb_pol, *src.shape[1:]))
        self.source_normalized = np.asarray(src * s, dtype=self.dtype)
        self.previous_update_norm = np.inf
        self._update_operators(alpha)

    def _update_operators(self, alpha):
        old = getattr(self, 'alpha', alpha)
        if hasattr(self, 'chi_eh'):
            f = old.imag / alpha.imag
            self.chi_eh = np.asarray(self.chi_eh * f, dtype=self.dtype)
            self.chi_he = np.asarray(self.chi_he * f, dtype=self.dtype)
            self.chi_hh = np.asarray(self.chi_hh * f, dtype=self.dtype)
        super()._update_operators(alpha)

    def curl(self, F):
        """D: the spectral curl i k x F of the k0-scaled grid (backend/__init__.py:472-509)."""
        return np.asarray(ifftn(curl_ft(np.asarray(fftn(F, self.ft_axes)), self.ks), self.ft_axes), dtype=self.dtype)

    def chi_op(self, x):
        """solver.py:531-552: chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x)."""
        chi_e = pointwise_mul(self.chi, x)
        chi_h = pointwise_mul(self.chi_eh, x)
        dx = self.curl(x)
        chi_e = chi_e + pointwise_mul(self.chi_he, dx)
        chi_h = chi_h + pointwise_mul(self.chi_hh, dx)
        return np.asarray(chi_e + self.curl(chi_h), dtype=self.dtype)
