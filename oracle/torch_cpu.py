"""
The split-Richardson iteration restated with torch CPU tensors -- TEST / BASELINE INFRASTRUCTURE ONLY.

The reference's second backend is torch (backend/torch.py): the same ``Solution.__iter__`` (solver.py:1064-1098)
with its operators evaluated by torch, ``ft`` / ``ift`` by torch.fft (backend/torch.py:183-205), the matrix
multiply by ``BackEnd.mul`` (backend/torch.py:220-249) and norms by torch (backend/torch.py:316-317).  This module
evaluates the same steps, for isotropic media, on torch CPU tensors, starting from a prepared numpy oracle
(``oracle.mmoracle.OracleSolution``: alpha, chi, the normalised source and the Green function), so that ``bench.py``
can time the torch-CPU form on the host cores beside the numpy form.  Only ``bench.py``'s ``cpu_baseline`` leg and
``tests/`` use it; it is checked against the numpy oracle in ``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import numpy as np
import torch


class TorchCPUIteration:
    def __init__(self, sol):
        """sol: an isotropic ``OracleSolution`` (chi [1, 1, *grid]), complex64 or complex128."""
        if sol.chi.shape[0] != 1:
            raise ValueError('the torch-CPU form covers isotropic media')
        self.ndim = sol.ndim
        self.axes = tuple(range(2, 2 + sol.ndim))
        self.vectorial = sol.vectorial
        t = lambda a: torch.from_numpy(np.array(a, order='C'))  # a writable copy
        self.chi = t(sol.chi[0, 0])
        self.src = t(sol.source_normalized)
        self.E = t(sol.field).clone()
        self.g = t(np.broadcast_to(sol.g_scalar_ft, sol.field.shape[2:]))
        self.ks = [t(np.asarray(k, dtype=sol.field.real.dtype)) for k in sol.ks]
        k2 = sum(k ** 2 for k in self.ks)
        self.inv_k2 = torch.where(k2 > 0, 1.0 / torch.where(k2 > 0, k2, torch.ones_like(k2)), torch.zeros_like(k2))
        self.h = complex(1.0j * sol.alpha.imag / sol.alpha)
        self.prev = float(sol.previous_update_norm)
        self.iteration = 0

    def _green(self, x):
        F = torch.fft.fftn(x, dim=self.axes)
        if self.vectorial:  # backend/__init__.py:606-649 with the DC sample kept, solver.py:571-577
            proj = sum(self.ks[a] * F[a, 0] for a in range(self.ndim)) * self.inv_k2
            PL = torch.zeros_like(F)
            zero = (0,) * self.ndim
            for a in range(self.ndim):
                PL[a, 0] = self.ks[a] * proj
                PL[a, 0][zero] = F[a, 0][zero]
            F = (F - PL) * self.g + PL * self.h
        else:
            F = F * self.g
        return torch.fft.ifftn(F, dim=self.axes)

    def advance(self) -> bool:
        """One ``Solution.__iter__`` step; a rejection is not handled here (the timed workloads have none)."""
        self.iteration += 1
        d = self.chi * self.E + self.src
        d = self._green(d) - self.E
        d = self.chi * d
        nu = float(torch.linalg.vector_norm(d))
        if nu < self.prev:
            self.E += d
            self.prev = nu
            return True
        return False
