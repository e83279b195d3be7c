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
from dataclasses import dataclass

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


@dataclass
class Preconditioner:
    alpha: complex
    beta: float
    transpose: bool
    chi: np.ndarray        # [1|3, 1|3, *shape] complex128, i (eps - alpha) / alpha_i (beta = 1)
    eps_field: np.ndarray  # [1|3, 1|3, *shape] complex128


def prepare(eps_field: np.ndarray, thickness: np.ndarray, wavenumber: float, eps_dtype: float,
            mu: complex = 1.0, objective=None) -> Preconditioner:
    """
    eps_field: permittivity as a matrix field [1|3, 1|3, *grid] (boundary susceptibility included).
    objective: optional callable alpha_r -> sigma replacing ``largest_sigma`` (e.g. a device implementation).
    """
    beta = float(np.real(1.0 / mu))  # solver.py:446
    gain = has_gain(eps_field, eps_dtype)
    loss = has_gain(-eps_field, eps_dtype)
    transpose = gain and not loss
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
    chi = eps_field * (1.0j / alpha.imag / beta)
    if _is_scalar_field(chi):
        chi = chi - alpha * 1.0j / alpha.imag
    else:
        chi = chi - np.eye(3).reshape(3, 3, *([1] * (chi.ndim - 2))) * (alpha * 1.0j / alpha.imag)
    return Preconditioner(alpha=alpha, beta=beta, transpose=transpose, chi=chi, eps_field=eps_field)
