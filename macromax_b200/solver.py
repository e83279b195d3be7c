"""
``solve`` and ``Solution`` with the public API of the reference (solver.py:25-1123), running the iteration on the
B200 through the native fused kernels.

Set-up (alpha, beta, chi, normalised source) is computed on the host in FP64 exactly as the reference's
non-magnetic ``__prepare_preconditioner`` does (see ``preconditioner.py``); every iteration then runs on the device:
``Solution.__iter__`` launches one fused iteration per ``next()``, and ``solve`` with an ``rtol``/``maxiter`` stop rule
(or the default callback) iterates on the device in chunks, evaluating the reference's stop rule after every
iteration on the device, so the iteration count is the reference's.  An arbitrary Python callback is honoured
iteration by iteration.
"""
from __future__ import annotations

import logging
from math import inf
from typing import Callable

import numpy as np
import scipy.constants as const

from . import _native as nat
from . import preconditioner as pc
from .bound import Bound, PeriodicBound, is_electric, is_magnetic
from .engine import IterationEngine
from .grid import Grid

log = logging.getLogger(__name__)


def _default_callback(s: 'Solution') -> bool:
    return s.iteration < 1e4 and s.residue > 1e-4


def solve(grid, vectorial=None, wavenumber=1.0, angular_frequency=None, vacuum_wavelength=None,
          current_density=None, source_distribution=None, epsilon=None, xi=0.0, zeta=0.0, mu=1.0,
          refractive_index=None, bound=None, initial_field=0.0, dtype=None, callback=_default_callback,
          rtol: float = 0, maxiter=inf, device=None) -> 'Solution':
    """macromax.solve (solver.py:25-89): build a Solution and iterate it to convergence."""
    return Solution(grid=grid, vectorial=vectorial, wavenumber=wavenumber, angular_frequency=angular_frequency,
                    vacuum_wavelength=vacuum_wavelength, current_density=current_density,
                    source_distribution=source_distribution, epsilon=epsilon, xi=xi, zeta=zeta, mu=mu,
                    refractive_index=refractive_index, bound=bound, initial_field=initial_field, dtype=dtype,
                    device=device).solve(callback, rtol=rtol, maxiter=maxiter)


class Solution:
    def __new__(cls, grid, vectorial=None, wavenumber=1.0, angular_frequency=None, vacuum_wavelength=None,
                current_density=None, source_distribution=None, epsilon=None, xi=0.0, zeta=0.0, mu=1.0,
                refractive_index=None, bound=None, initial_field=0.0, dtype=None, device=None):
        """Magnetic and bi-(an)isotropic media take the reference's magnetic code path: a MagneticSolution, with
        the same constructor arguments and properties."""
        from .magnetic import MagneticSolution, needs_magnetic_solver
        g = grid
        if not isinstance(g, Grid):
            g = Grid.from_ranges(*([g] if np.isscalar(g[0]) else g))
        if needs_magnetic_solver(g, epsilon, xi, zeta, mu, refractive_index, bound):
            return MagneticSolution(g, vectorial=vectorial, wavenumber=wavenumber,
                                    angular_frequency=angular_frequency, vacuum_wavelength=vacuum_wavelength,
                                    current_density=current_density, source_distribution=source_distribution,
                                    epsilon=epsilon, xi=xi, zeta=zeta, mu=mu, refractive_index=refractive_index,
                                    bound=bound, initial_field=initial_field, dtype=dtype, device=device)
        return super().__new__(cls)

    def __init__(self, grid, vectorial=None, wavenumber=1.0, angular_frequency=None, vacuum_wavelength=None,
                 current_density=None, source_distribution=None, epsilon=None, xi=0.0, zeta=0.0, mu=1.0,
                 refractive_index=None, bound=None, initial_field=0.0, dtype=None, device=None):
        if not isinstance(grid, Grid):
            if np.isscalar(grid[0]):
                grid = [grid]
            grid = Grid.from_ranges(*grid)
        self._grid = grid.immutable
        if angular_frequency is not None:
            self._wavenumber = angular_frequency / const.c
        elif vacuum_wavelength is not None:
            self._wavenumber = 2 * const.pi / vacuum_wavelength
        else:
            self._wavenumber = wavenumber

        def func2arr(f):
            return f(*self._grid) if callable(f) else np.asarray(f)

        # solver.py:173-195
        if source_distribution is None:
            if current_density is None:
                if vectorial is None:
                    vectorial = True
                current_density = np.zeros((1 + 2 * vectorial, *self._grid.shape),
                                           dtype=dtype if dtype is not None else np.complex128)
            current_density = np.asarray(func2arr(current_density))
            source_distribution = current_density * (-1j * self.angular_frequency * const.mu_0)
        else:
            source_distribution = np.asarray(func2arr(source_distribution))
        if vectorial is None:
            vectorial = source_distribution.ndim > self._grid.ndim and source_distribution.shape[0] == 3
        self._vectorial = bool(vectorial)
        self._bound = bound if bound is not None else PeriodicBound(self._grid)
        if dtype is None:
            dtype = np.asarray(source_distribution).dtype
        if not np.issubdtype(dtype, np.complexfloating):
            dtype = np.complex64 if dtype in (np.float16, np.float32) else np.complex128
        self._dtype = np.dtype(dtype)
        self._nb_pol = 3 if self._vectorial else 1
        self._k_grid = self._grid * self._wavenumber

        # material (solver.py:224-254), non-magnetic only
        mu_arr = func2arr(mu)
        if not (np.allclose(func2arr(xi), 0) and np.allclose(func2arr(zeta), 0)
                and np.allclose(mu_arr, np.ravel(mu_arr)[0]) and np.asarray(mu_arr).ndim <= self._grid.ndim):
            raise NotImplementedError('magnetic or bi-anisotropic media are not supported by the B200 backend')
        if is_magnetic(self._bound) and np.any(self._bound.magnetic_susceptibility != 0):
            raise NotImplementedError('magnetic boundaries are not supported by the B200 backend')
        self._mu = complex(np.ravel(mu_arr)[0])
        if epsilon is None:
            n = func2arr(refractive_index) if refractive_index is not None else 1.0
            n = self._to_matrix_field(np.asarray(n, dtype=np.complex128))
            epsilon = self._mul(n, n)
            if n.shape[0] == 1 and np.any(n.real < 0):
                raise NotImplementedError('negative refractive index (magnetic) media are not supported')
        epsilon = self._to_matrix_field(np.asarray(func2arr(epsilon), dtype=np.complex128))
        if is_electric(self._bound):
            chi_b = np.asarray(self._bound.electric_susceptibility)
            if epsilon.shape[0] > 1:
                chi_b = np.eye(3).reshape(3, 3, *([1] * self._grid.ndim)) * chi_b
            epsilon = epsilon + chi_b
        self._engine = None
        self._device = device
        self._prepare(epsilon, source_distribution, initial_field)

    # -- helpers ----------------------------------------------------------------------------------------------------
    def _to_matrix_field(self, arr):
        arr = np.asarray(arr)
        while arr.ndim < self._grid.ndim + 2:
            arr = arr[np.newaxis]
        if arr.shape[0] == 1 and arr.shape[1] > 1:
            arr = arr.swapaxes(0, 1)
        return arr

    @staticmethod
    def _mul(a, b):
        if (a.shape[0] == 1 and a.shape[1] == 1) or (b.shape[0] == 1 and b.shape[1] == 1):
            return a * b
        return np.einsum('ij...,jk...->ik...', a, b)

    def _prepare(self, eps_field, source_distribution, initial_field):
        if eps_field.shape[0] > 1 and not self._vectorial:
            raise ValueError('an anisotropic permittivity needs a vector source')
        eps_dtype = float(np.finfo(self._dtype).eps)
        self._pre = pc.prepare(eps_field, self._bound.thickness, self._wavenumber, eps_dtype, mu=self._mu,
                               device_setup=True, device=self._device)
        self._eps_field = eps_field
        alpha = self._pre.alpha
        if self._engine is None:
            self._engine = IterationEngine(self._grid.shape, self._nb_pol, 1, self._dtype, self._k_grid.k,
                                           self._pre.chi_for_engine(), alpha, device=self._device)
            self.E = initial_field
        else:
            self._engine.rebase_alpha(self._pre.chi_for_engine(), alpha)
        self.source_distribution = source_distribution

    @property
    def _state(self):
        return self._engine.read_state()[0]

    # -- properties of the reference API ----------------------------------------------------------------------------
    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def vectorial(self) -> bool:
        return self._vectorial

    @property
    def dtype(self):
        return self._dtype.type

    @property
    def wavenumber(self) -> float:
        return self._wavenumber

    @property
    def angular_frequency(self) -> float:
        return self._wavenumber * const.c

    @property
    def wavelength(self) -> float:
        return 2.0 * const.pi / self._wavenumber

    @property
    def magnetic(self) -> bool:
        return False

    @property
    def bound(self) -> Bound:
        return self._bound

    @property
    def alpha(self) -> complex:
        st = self._state
        return complex(st['alpha_re'], st['alpha_im'])

    @property
    def beta(self) -> float:
        return self._pre.beta

    @property
    def source_distribution(self) -> np.ndarray:
        """solver.py:690-700: s' beta alpha_i / i at the current alpha == s'0 beta alpha0_i / i."""
        s0 = self._engine.sources[0].cpu().numpy().reshape(self._nb_pol, *self._grid.shape)
        return s0 * (self._pre.beta / 1.0j * self._engine.alpha0.imag)

    @source_distribution.setter
    def source_distribution(self, new_source):
        """solver.py:702-720, stored at alpha0: s'0 = s i / (alpha0_i beta); resets previous_update_norm."""
        src = self._to_matrix_field(np.asarray(new_source))
        src = np.broadcast_to(src, (self._nb_pol, 1, *self._grid.shape))[:, 0]
        self._engine.set_sources(src * (1.0j / self._engine.alpha0.imag / self._pre.beta))
        self._engine.reset_update_norm()

    @property
    def j(self) -> np.ndarray:
        return self.source_distribution / (-1.0j * self.angular_frequency * const.mu_0)

    @j.setter
    def j(self, new_j):
        self.source_distribution = np.asarray(new_j) * (-1.0j * self.angular_frequency * const.mu_0)

    @property
    def epsilon(self) -> np.ndarray:
        eps = self._eps_field
        if is_electric(self._bound):
            chi_b = np.asarray(self._bound.electric_susceptibility)
            if eps.shape[0] > 1:
                chi_b = np.eye(3).reshape(3, 3, *([1] * self._grid.ndim)) * chi_b
            eps = eps - chi_b
        return eps.astype(self._dtype)

    @epsilon.setter
    def epsilon(self, new_value):
        """solver.py:755-787: new material, same source and field; the preconditioner is rebuilt."""
        eps = self._to_matrix_field(np.asarray(new_value, dtype=np.complex128))
        if is_electric(self._bound):
            chi_b = np.asarray(self._bound.electric_susceptibility)
            if eps.shape[0] > 1:
                chi_b = np.eye(3).reshape(3, 3, *([1] * self._grid.ndim)) * chi_b
            eps = eps + chi_b
        src = self.source_distribution
        self._prepare(eps, src, None)

    @property
    def refractive_index(self) -> np.ndarray:
        return self.epsilon ** 0.5

    @refractive_index.setter
    def refractive_index(self, new_value):
        self.epsilon = np.asarray(new_value) ** 2

    @property
    def E(self) -> np.ndarray:
        """solver.py:811-821: the current field divided by k0^2, as a host array."""
        f = self._engine.current()[0] * (1.0 / self._wavenumber ** 2)  # unit conversion on the device
        return self._engine.to_host(f).reshape(self._nb_pol, *self._grid.shape).astype(self._dtype, copy=False)

    @E.setter
    def E(self, E):
        """solver.py:823-832."""
        if E is None:
            return
        E = np.asarray(E)
        if E.ndim == 0:  # a constant field is filled on the device
            import torch
            eng = self._engine
            self._engine.set_fields(torch.full((1, eng.ncomp, eng.N), complex(E) * self._wavenumber ** 2,
                                               dtype=eng.torch_dtype, device=eng.device))
            return
        full = np.broadcast_to(self._to_matrix_field(E), (self._nb_pol, 1, *self._grid.shape))[:, 0]
        self._engine.set_fields(full * (self._wavenumber ** 2))

    @property
    def E_device(self):
        """The current field (times k0^2) as a device tensor [ncomp, *grid] (no host copy)."""
        return self._engine.current()[0].reshape(self._nb_pol, *self._grid.shape)

    @property
    def iteration(self) -> int:
        return int(self._state['iteration'])

    @iteration.setter
    def iteration(self, it: int = 0):
        st = self._engine.read_state()
        st['iteration'] = it
        self._engine.write_state(st)

    @property
    def previous_update_norm(self) -> float:
        return float(self._state['prev_norm'] / (self._wavenumber ** 2))

    @property
    def relative_residue(self) -> float:
        """solver.py:1026-1042: previous_update_norm / ||E|| (0 when the previous update norm is 0)."""
        st = self._state
        prev = float(st['prev_norm'])
        if not prev > 0:
            return 0.0
        if st['iteration'] > 0 and np.isfinite(prev):
            return float(st['residue'])
        import torch
        return prev / float(torch.linalg.vector_norm(self._engine.current()[0]).item())

    @property
    def residue(self) -> float:
        return self.relative_residue

    @property
    def rejections(self) -> int:
        return int(self._state['rejections'])

    def _check_status(self, st):
        if int(st['status']) == nat.MMX_STATUS_ZERODIV:
            raise ZeroDivisionError('float division by zero (update norm after a zero update norm)')

    # -- iteration --------------------------------------------------------------------------------------------------
    def __iter__(self):
        """solver.py:1049-1098: every next() runs one fused iteration on the device; obtaining the iterator resets the
        iteration count (solver.py:1063), and a zero update norm after a zero one raises ZeroDivisionError
        (solver.py:1079)."""
        st = self._engine.read_state()
        st['iteration'] = 0
        st['rtol'] = -1.0
        st['maxiter'] = np.inf
        st['active'] = 1
        st['status'] = 0
        self._engine.write_state(st)
        while True:
            self._engine.iterate(1)
            self._check_status(self._state)
            yield self

    def solve(self, callback: Callable[['Solution'], bool] | None = _default_callback, rtol: float = 0,
              maxiter=inf) -> 'Solution':
        """solver.py:1100-1123."""
        if callback is None or callback is _default_callback:
            if callback is _default_callback:
                rtol, maxiter = 1e-4, 1e4
            st = self._engine.run(float(rtol), float(maxiter), reset_iteration=True)
            self._check_status(st[0])
            return self
        for sol in self:
            if not callback(sol):
                break
        return self

    def __str__(self):
        return f'Solution(grid={self._grid}, vectorial={self._vectorial}, dtype={self._dtype})'
