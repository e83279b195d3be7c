"""
Calculation-volume boundaries, with the interface of the reference's ``macromax.bound`` (bound.py:19-215).

What the iteration needs from a bound is small: its thickness per (axis, side), whose smallest non-zero value biases
alpha (solver.py:591-627), and, for an absorbing bound, the susceptibility that is added to the permittivity before
the preconditioner is built (solver.py:242-247).  Any object with ``thickness`` (and, for absorbing bounds,
``electric_susceptibility``) is accepted by the solvers here, the reference's own bound objects included
(``is_electric`` below).

Absorbing layers are built separably.  Along one axis, a layer of thickness t on the front side reaches depth
``t - d`` at a sample whose distance from the first sample is d (the back side: from the last sample); the relative
depth ``(t - d) / t`` in (0, 1] is mapped through that side's extinction profile.  The axis's profile is the larger
of its two sides, and the N-D extinction is the maximum over the axes' 1-D profiles, broadcast against each other
(so corners take the largest of the overlapping layers, as in bound.py:158-183).  Axes without a layer contribute
nothing, so the result keeps singleton dimensions there.
"""
from __future__ import annotations

from numbers import Complex, Real
from typing import Callable, Sequence, Union

import numpy as np

from .grid import Grid


def is_electric(bound) -> bool:
    """Whether ``bound`` carries an electric susceptibility: the ``Electric`` mixin here or in the reference
    package (matched by class name, so the reference need not be importable)."""
    return any(c.__name__ == 'Electric' for c in type(bound).__mro__)


def is_magnetic(bound) -> bool:
    """Whether ``bound`` carries a magnetic susceptibility (the ``Magnetic`` mixin, here or in the reference)."""
    return any(c.__name__ == 'Magnetic' for c in type(bound).__mro__)


class Electric:
    """Mixin: the bound has a non-zero electric susceptibility."""

    @property
    def background_permittivity(self) -> Complex:
        return 0.0

    @property
    def electric_susceptibility(self) -> np.ndarray:
        return NotImplemented

    @property
    def permittivity(self) -> np.ndarray:
        """Background permittivity plus the bound's susceptibility (may hold singleton dimensions)."""
        return self.background_permittivity + self.electric_susceptibility


class Magnetic:
    """Mixin: the bound has a non-zero magnetic susceptibility."""

    @property
    def magnetic_susceptibility(self) -> np.ndarray:
        return NotImplemented

    @property
    def permeability(self) -> np.ndarray:
        return 1.0 + self.magnetic_susceptibility


class Bound:
    """A boundary of the calculation volume: thickness[axis, side] in the grid's length unit, side 0 at the first
    sample of the axis and side 1 at the last."""

    def __init__(self, grid: Union[Grid, Sequence, np.ndarray, None] = None,
                 thickness: Union[Real, Sequence, np.ndarray] = 0.0, background_permittivity: Complex = 1.0):
        self._grid = grid if isinstance(grid, Grid) else Grid.from_ranges(grid)
        self._thickness = np.array(np.broadcast_to(thickness, (self._grid.ndim, 2)), dtype=float)
        self._background_permittivity = background_permittivity

    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def thickness(self) -> np.ndarray:
        return self._thickness.copy()

    @property
    def background_permittivity(self) -> Complex:
        return self._background_permittivity

    @property
    def electric_susceptibility(self) -> np.ndarray:
        return np.zeros(self.grid.shape)

    @property
    def magnetic_susceptibility(self) -> np.ndarray:
        return np.zeros(self.grid.shape)

    def _distances(self, axis: int) -> tuple[np.ndarray, np.ndarray]:
        """Distance of every sample of ``axis`` from the first and from the last sample (both >= 0)."""
        n = self.grid.shape[axis]
        spacing = abs(float(np.asarray(self.grid.step)[axis]))
        idx = np.arange(n, dtype=float)
        return idx * spacing, (n - 1 - idx) * spacing

    def _plaid(self, axis: int, profile: np.ndarray) -> np.ndarray:
        shape = [1] * self.grid.ndim
        shape[axis] = profile.size
        return profile.reshape(shape)

    @property
    def between(self) -> np.ndarray:
        """True where a sample lies inside the calculation volume proper (the inner edge of a layer included)."""
        inside = np.asarray(True)
        for axis in range(self.grid.ndim):
            d_front, d_back = self._distances(axis)
            keep = (d_front >= self._thickness[axis, 0]) & (d_back >= self._thickness[axis, 1])
            inside = inside & self._plaid(axis, keep)
        return inside

    @property
    def beyond(self) -> np.ndarray:
        return ~self.between


class PeriodicBound(Bound):
    def __init__(self, grid):
        super().__init__(grid=grid, thickness=0.0)


class AbsorbingBound(Bound, Electric):
    """Layers whose extinction coefficient kappa follows a profile of the relative depth (0 at the layer's inner edge,
    1 at the edge of the volume); one profile per (axis, side), or one for all."""

    def __init__(self, grid, thickness=0.0,
                 extinction_coefficient_function: Union[Callable, Sequence, np.ndarray] = lambda rel_depth: rel_depth,
                 background_permittivity: Complex = 1.0):
        super().__init__(grid=grid, thickness=thickness, background_permittivity=background_permittivity)
        profiles = np.empty((self.grid.ndim, 2), dtype=object)
        profiles[...] = np.broadcast_to(np.asarray(extinction_coefficient_function, dtype=object),
                                        (self.grid.ndim, 2))
        self._profiles = profiles

    @property
    def is_electric(self) -> bool:
        return True

    def _axis_extinction(self, axis: int) -> np.ndarray | None:
        """The larger of the axis's two layer profiles at every sample, or None where the axis has no layer."""
        result = None
        for side, dist in enumerate(self._distances(axis)):
            t = self._thickness[axis, side]
            depth = t - dist
            inside = depth > 0
            if not inside.any():
                continue
            rel_depth = np.where(inside, depth / t if t != 0 else 0.0, 0.0)
            kappa = np.where(inside, np.asarray(self._profiles[axis, side](rel_depth), dtype=float), 0.0)
            result = np.maximum(0.0 if result is None else result, kappa)
        return result

    @property
    def extinction(self) -> np.ndarray:
        kappa = 0.0
        for axis in range(self.grid.ndim):
            prof = self._axis_extinction(axis)
            if prof is not None:
                kappa = np.maximum(kappa, self._plaid(axis, prof))
        return kappa

    @property
    def electric_susceptibility(self) -> np.ndarray:
        """chi = (n + i kappa)^2 - eps_background with n the background's (principal) refractive index."""
        n = np.lib.scimath.sqrt(self.background_permittivity)
        return (n + 1j * self.extinction) ** 2 - self.background_permittivity


class LinearBound(AbsorbingBound):
    """Extinction rising linearly with depth to ``max_extinction_coefficient`` (per axis and side, broadcast) at the
    edge of the volume."""

    def __init__(self, grid, thickness=0.0, max_extinction_coefficient=0.25, background_permittivity: Complex = 1.0):
        self._max_extinction_coefficient = max_extinction_coefficient
        grid_ = grid if isinstance(grid, Grid) else Grid.from_ranges(grid)
        peaks = np.broadcast_to(np.asarray(max_extinction_coefficient, dtype=float), (grid_.ndim, 2))
        profiles = np.empty((grid_.ndim, 2), dtype=object)
        for axis in range(grid_.ndim):
            for side in range(2):
                profiles[axis, side] = _Linear(float(peaks[axis, side]))
        super().__init__(grid=grid_, thickness=thickness, extinction_coefficient_function=profiles,
                         background_permittivity=background_permittivity)


class _Linear:
    """kappa(rel_depth) = peak * rel_depth."""

    def __init__(self, peak: float):
        self.peak = peak

    def __call__(self, rel_depth):
        return self.peak * rel_depth
