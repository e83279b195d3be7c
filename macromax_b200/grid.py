"""
Uniform plaid sampling grid and its k-space, with the conventions of the reference ``Grid``
(utils/ft/grid.py:10-650): ``grid[axis]`` is an open-grid coordinate vector centred so that index ``n // 2`` sits at
``center``; ``grid.k`` is the k-space grid with the origin at index 0 (ifftshifted), ``k_a[j] = 2 pi f_j`` with
``f = fftfreq(n_a, step_a)``; multiplying a grid by a scalar scales its coordinates (the solver uses ``grid * k0``,
solver.py:212).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


class Grid:
    def __init__(self, shape=None, step=None, *, center=None, first=None, extent=None):
        if shape is None and extent is not None and step is not None:
            shape = np.round(np.asarray(extent, dtype=float) / np.asarray(step, dtype=float)).astype(int)
        shape = np.atleast_1d(np.asarray(shape, dtype=int)).copy()
        ndim = shape.size
        if step is None:
            step = np.asarray(extent, dtype=float) / shape if extent is not None else np.ones(ndim)
        step = np.broadcast_to(np.asarray(step, dtype=float), (ndim,)).copy()
        if center is None:
            if first is not None:
                center = np.asarray(first, dtype=float) + step * (shape // 2)
            else:
                center = np.zeros(ndim)
        self._shape = shape
        self._step = step
        self._center = np.broadcast_to(np.asarray(center, dtype=float), (ndim,)).copy()

    @classmethod
    def from_ranges(cls, *ranges) -> 'Grid':
        """Grid through the given uniformly increasing coordinate vectors (utils/ft/grid.py from_ranges)."""
        shape, step, first = [], [], []
        for r in ranges:
            r = np.asarray(r, dtype=float).ravel()
            shape.append(r.size)
            step.append(r[1] - r[0] if r.size > 1 else 1.0)
            first.append(r[0])
        return cls(shape=shape, step=step, first=first)

    @property
    def immutable(self) -> 'Grid':
        return self

    @property
    def shape(self) -> np.ndarray:
        return self._shape.copy()

    @property
    def step(self) -> np.ndarray:
        return self._step.copy()

    @property
    def center(self) -> np.ndarray:
        return self._center.copy()

    @property
    def ndim(self) -> int:
        return int(self._shape.size)

    @property
    def size(self) -> int:
        return int(np.prod(self._shape))

    @property
    def first(self) -> np.ndarray:
        return self._center - self._step * (self._shape // 2)

    @property
    def extent(self) -> np.ndarray:
        return self._shape * self._step

    def __len__(self) -> int:
        return self.ndim

    def __getitem__(self, axis: int) -> np.ndarray:
        n = int(self._shape[axis])
        rng = self.first[axis] + self._step[axis] * np.arange(n)
        view = [1] * self.ndim
        view[axis] = n
        return rng.reshape(view)

    def __iter__(self):
        for axis in range(self.ndim):
            yield self[axis]

    def __mul__(self, factor) -> 'Grid':
        factor = np.asarray(factor, dtype=float)
        return Grid(shape=self._shape, step=self._step * factor, center=self._center * factor)

    __rmul__ = __mul__

    def __eq__(self, other) -> bool:
        return (isinstance(other, Grid) and np.array_equal(self._shape, other._shape)
                and np.allclose(self._step, other._step) and np.allclose(self._center, other._center))

    @property
    def k(self) -> Sequence[np.ndarray]:
        """Open-grid k-vectors, origin at index 0 (utils/ft/grid.py:426-439)."""
        ks = []
        for axis in range(self.ndim):
            n = int(self._shape[axis])
            k = 2 * np.pi * np.fft.fftfreq(n, self._step[axis])
            view = [1] * self.ndim
            view[axis] = n
            ks.append(k.reshape(view))
        return ks

    def __repr__(self) -> str:
        return f'Grid(shape={self._shape.tolist()}, step={self._step.tolist()}, center={self._center.tolist()})'
