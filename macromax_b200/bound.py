"""
Calculation-volume boundaries with the semantics of the reference ``macromax.bound`` (bound.py:19-215): a ``Bound``
carries a thickness per axis and side (its smallest non-zero value biases alpha, solver.py:591-627); an ``Electric``
bound adds its susceptibility to the permittivity before the preconditioner is built (solver.py:242-247).
"""
from __future__ import annotations

from numbers import Complex, Real
from typing import Callable, Sequence, Union

import numpy as np

from .grid import Grid


class Electric:
    """Marks a bound with a non-zero electric susceptibility."""

    @property
    def background_permittivity(self) -> Complex:
        return 0.0

    @property
    def electric_susceptibility(self) -> np.ndarray:
        return NotImplemented

    @property
    def permittivity(self) -> np.ndarray:
        return self.background_permittivity + self.electric_susceptibility


class Magnetic:
    """Marks a bound with a non-zero magnetic susceptibility (magnetic media are not supported by this solver)."""

    @property
    def magnetic_susceptibility(self) -> np.ndarray:
        return NotImplemented


class Bound:
    def __init__(self, grid: Union[Grid, Sequence, np.ndarray, None] = None,
                 thickness: Union[Real, Sequence, np.ndarray] = 0.0, background_permittivity: Complex = 1.0):
        if not isinstance(grid, Grid):
            grid = Grid.from_ranges(grid)
        self._grid = grid
        self._thickness = np.broadcast_to(thickness, (grid.ndim, 2)).astype(float)
        self._background_permittivity = background_permittivity

    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def thickness(self) -> np.ndarray:
        """Thickness [axis, front/back] in the grid's length unit."""
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


class PeriodicBound(Bound):
    def __init__(self, grid):
        super().__init__(grid=grid, thickness=0.0)


class AbsorbingBound(Bound, Electric):
    def __init__(self, grid, thickness=0.0,
                 extinction_coefficient_function: Union[Callable, Sequence, np.ndarray] = lambda rel_depth: rel_depth,
                 background_permittivity: Complex = 1.0):
        super().__init__(grid=grid, thickness=thickness, background_permittivity=background_permittivity)
        self._kappa_functions = np.broadcast_to(np.asarray(extinction_coefficient_function, dtype=object),
                                                (self.grid.ndim, 2))

    @property
    def extinction(self) -> np.ndarray:
        """Extinction kappa on the plaid grid; maximum over overlapping axes at corners (bound.py:158-183)."""
        kappa = 0.0
        for axis, rng in enumerate(self.grid):
            for back in range(2):
                t = self._thickness[axis, back] * np.sign(self.grid.step[axis])
                if not back:
                    depth = (rng.ravel()[0] + t) - rng
                else:
                    depth = rng - (rng.ravel()[-1] - t)
                depth = depth * np.sign(self.grid.step[axis])
                inside = depth > 0
                if np.any(inside):
                    rel = inside * depth / t
                    kappa = np.maximum(kappa, self._kappa_functions[axis, back](rel) * inside)
        return kappa

    @property
    def electric_susceptibility(self) -> np.ndarray:
        n = np.lib.scimath.sqrt(self.background_permittivity)
        eps = (n + 1j * self.extinction) ** 2
        return eps - self.background_permittivity


class LinearBound(AbsorbingBound):
    def __init__(self, grid, thickness=0.0, max_extinction_coefficient=0.25, background_permittivity: Complex = 1.0):
        self._max_extinction_coefficient = max_extinction_coefficient
        funcs = np.vectorize(lambda kmax: (lambda rel: kmax * rel), otypes=[object])(max_extinction_coefficient)
        super().__init__(grid=grid, thickness=thickness, extinction_coefficient_function=funcs,
                         background_permittivity=background_permittivity)
