"""
Many right-hand sides sharing one material, solved together on the device.

The reference solves one source at a time: ``ScatteringMatrix`` (matrix.py:770-844) loops over its columns and
re-runs ``Solution.solve`` (matrix.py:650-669) with a new ``source_distribution`` on one shared ``Solution``, so every
column has the same alpha and chi.  ``BatchSolution`` keeps that contract -- one preconditioner built from the
material, B sources -- and iterates all B sources in the same kernel launches: the field layout is
[B][components][grid], chi is stored once, and every right-hand side carries its own state (alpha after
divergence-guard rejections, previous update norm, iteration count, residue).  The stop rule
``iteration < maxiter and residue > rtol`` is evaluated per right-hand side after every iteration on the device; a
finished right-hand side is masked out of later launches (its tiles return immediately), so each one stops at
exactly the iteration where its own sequential solve would stop.
"""
from __future__ import annotations

from math import inf

import numpy as np
import torch

from . import _native as nat
from . import preconditioner as pc
from .bound import Bound, PeriodicBound, is_electric
from .engine import IterationEngine
from .grid import Grid


def _to_matrix_field(arr, ndim):
    arr = np.asarray(arr)
    while arr.ndim < ndim + 2:
        arr = arr[np.newaxis]
    if arr.shape[0] == 1 and arr.shape[1] > 1:
        arr = arr.swapaxes(0, 1)
    return arr


def prepare_material(grid: Grid, epsilon, bound: Bound | None, wavenumber: float, dtype, device=None):
    """Permittivity (plus an Electric bound's susceptibility) as a matrix field, and its preconditioner."""
    bound = bound if bound is not None else PeriodicBound(grid)
    eps = _to_matrix_field(np.asarray(epsilon, dtype=np.complex128), grid.ndim)
    if is_electric(bound):
        chi_b = np.asarray(bound.electric_susceptibility)
        if eps.shape[0] > 1:
            chi_b = np.eye(3).reshape(3, 3, *([1] * grid.ndim)) * chi_b
        eps = eps + chi_b
    pre = pc.prepare(eps, bound.thickness, wavenumber, float(np.finfo(np.dtype(dtype)).eps), device_setup=True,
                     device=device)
    return pre, bound


class BatchSolution:
    """
    B sources [B, 1|3, *grid] (``source_distribution`` units, i.e. i omega mu0 J) in one material.
    ``E`` is [B, 1|3, *grid]; ``iterations``, ``residues``, ``rejections`` and ``alphas`` are per source.
    """

    def __init__(self, grid: Grid, sources, epsilon, bound: Bound | None = None, vacuum_wavelength=None,
                 wavenumber=None, dtype=np.complex64, device=None, preconditioner=None):
        if not isinstance(grid, Grid):
            grid = Grid.from_ranges(*grid)
        self.grid = grid
        self.wavenumber = 2 * np.pi / vacuum_wavelength if vacuum_wavelength is not None else float(wavenumber)
        self.dtype = np.dtype(dtype)
        # a torch tensor (e.g. already on the device) is used as it is; anything else goes through numpy
        src = sources if isinstance(sources, torch.Tensor) else np.asarray(sources)
        if src.ndim == grid.ndim + 1:
            src = src[None]
        if src.ndim != grid.ndim + 2:
            raise ValueError('sources must be [B, 1|3, *grid]')
        self.batch = int(src.shape[0])
        self.ncomp = int(src.shape[1])
        if self.ncomp not in (1, 3):
            raise ValueError('sources need 1 or 3 components')
        if preconditioner is None:
            self.pre, self.bound = prepare_material(grid, epsilon, bound, self.wavenumber, self.dtype, device=device)
        else:
            self.pre, self.bound = preconditioner, bound
        if self.pre.chi_rows > 1 and self.ncomp != 3:
            raise ValueError('an anisotropic permittivity needs vector sources')
        self.engine = IterationEngine(grid.shape, self.ncomp, self.batch, self.dtype, (grid * self.wavenumber).k,
                                      self.pre.chi_for_engine(), self.pre.alpha, device=device)
        self.set_sources(src)

    @property
    def alpha0(self) -> complex:
        return self.pre.alpha

    def set_sources(self, src):
        """s'0 = i s / (alpha0_i beta) (solver.py:702-720); resets every previous_update_norm."""
        scale = 1.0j / self.pre.alpha.imag / self.pre.beta
        if isinstance(src, torch.Tensor):
            self.engine.set_sources(src.to(self.engine.device, self.engine.torch_dtype) * scale)
        else:
            self.engine.set_sources(np.asarray(src) * scale)
        self.engine.reset_update_norm()

    def set_fields(self, E=0.0):
        if np.isscalar(E):  # a constant field is filled on the device (no host array of the batch's size)
            E = torch.full((1, self.ncomp, self.engine.N), complex(E) * self.wavenumber ** 2,
                           dtype=self.engine.torch_dtype, device=self.engine.device)
            self.engine.set_fields(E)
            return
        if isinstance(E, torch.Tensor):
            self.engine.set_fields(E.reshape(-1, self.ncomp, self.engine.N) * self.wavenumber ** 2)
            return
        E = np.broadcast_to(np.asarray(E), (self.batch, self.ncomp, *self.grid.shape))
        self.engine.set_fields(E * self.wavenumber ** 2)

    def solve(self, rtol: float = 1e-6, maxiter=1e4) -> 'BatchSolution':
        """Iterate every source until its residue is below rtol or it has made maxiter iterations (by default the
        reference's default cap, solver.py:81-83: complex64 alone may never reach a small rtol)."""
        st = self.engine.run(float(rtol), float(maxiter))
        if np.any(st['status'] == nat.MMX_STATUS_ZERODIV):
            raise ZeroDivisionError('float division by zero (update norm after a zero update norm)')
        self._state = st
        return self

    def iterate(self, n: int):
        st = self.engine.read_state()
        st['rtol'] = -1.0
        st['maxiter'] = np.inf
        st['active'] = 1
        self.engine.write_state(st)
        self.engine.iterate(n)

    @property
    def state(self) -> np.ndarray:
        return self.engine.read_state()

    @property
    def iterations(self) -> np.ndarray:
        return self.state['iteration'].copy()

    @property
    def residues(self) -> np.ndarray:
        return self.state['residue'].copy()

    @property
    def rejections(self) -> np.ndarray:
        return self.state['rejections'].copy()

    @property
    def alphas(self) -> np.ndarray:
        st = self.state
        return st['alpha_re'] + 1j * st['alpha_im']

    @property
    def E_device(self):
        """Current fields (times k0^2) [B, C, N] on the device."""
        return self.engine.current()

    @property
    def E(self) -> np.ndarray:
        f = self.engine.current() * (1.0 / self.wavenumber ** 2)  # unit conversion on the device
        return self.engine.to_host(f).reshape(self.batch, self.ncomp, *self.grid.shape).astype(self.dtype, copy=False)

    def close(self):
        self.engine.close()


def solve_sharded(grid: Grid, sources, epsilon, rtol: float = 1e-6, maxiter=1e4, **kwargs) -> dict:
    """
    Right-hand sides of one material split over the ranks of the default process group (``torchrun``, one GPU per
    rank, the device chosen by the caller): every rank solves its ``shard_range`` slice of ``sources``
    [B, 1|3, *grid] in one BatchSolution on its own GPU, then the fields ``E`` [B, 1|3, *grid] and the per-source
    ``iterations`` and ``residues`` are gathered in source order on every rank.  The solves exchange nothing (replicas);
    the gather is the only collective.  Without a process group, or with one rank, this is one BatchSolution over all
    sources.  ``kwargs`` go to BatchSolution (bound, vacuum_wavelength, dtype, ...).
    """
    from .distributed import gather_rows, shard_range, world
    rank, size = world()
    src = np.asarray(sources)
    if src.ndim == grid.ndim + 1:
        src = src[None]
    n = int(src.shape[0])
    a, b = shard_range(n, rank, size)
    dtype = np.dtype(kwargs.get('dtype', np.complex64))
    if b > a:
        bs = BatchSolution(grid, src[a:b], epsilon, **kwargs)
        try:
            bs.solve(rtol, maxiter)
            E, its, res = bs.E, bs.iterations, bs.residues
        finally:
            bs.close()
    else:  # more ranks than sources: this rank contributes no rows
        E = np.zeros((0, *src.shape[1:]), dtype=dtype)
        its = np.zeros(0, dtype=np.int32)
        res = np.zeros(0, dtype=np.float64)
    return {'E': gather_rows(E, n), 'iterations': gather_rows(its, n), 'residues': gather_rows(res, n)}


class UnevenBatch:
    """
    Several batches on grids of different sizes (e.g. 64 x 128^2, 32 x 256^2 and 8 x 384^2 sources) iterated by
    ONE captured CUDA graph per chunk of iterations (``mmx_iterate_multi``): each member's pass kernels form an
    independent branch of the graph, so the small grids run concurrently instead of one after another.
    """

    def __init__(self, members):
        import ctypes
        self.members = list(members)
        n = len(self.members)
        engines = [m.engine for m in self.members]
        vp = ctypes.c_void_p
        self._args = (
            n,
            (vp * n)(*[e.plan.handle.value for e in engines]),
            (vp * n)(*[e.fields[0].data_ptr() for e in engines]),
            (vp * n)(*[e.fields[1].data_ptr() for e in engines]),
            (vp * n)(*[e.chi.data_ptr() for e in engines]),
            (ctypes.c_int * n)(*[e.chi_kind for e in engines]),
            (vp * n)(*[e.sources.data_ptr() for e in engines]),
            (vp * n)(*[e.state.data_ptr() for e in engines]),
        )

    def iterate(self, niter: int):
        import ctypes
        s = torch.cuda.current_stream().cuda_stream
        nat.call('mmx_iterate_multi', *self._args, int(niter), ctypes.c_void_p(s) if s else None)

    def solve(self, rtol: float = 1e-6, maxiter=1e4, chunk: int = 8, max_chunk: int = 64) -> 'UnevenBatch':
        for m in self.members:
            st = m.engine.read_state()
            st['iteration'] = 0
            st['rtol'] = rtol
            st['maxiter'] = maxiter
            st['active'] = 1
            st['status'] = 0
            m.engine.write_state(st)
        while True:
            self.iterate(chunk)
            if not any(np.any(m.engine.read_state()['active']) for m in self.members):
                break
            chunk = min(2 * chunk, max_chunk)
        return self
