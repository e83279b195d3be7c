"""
Mixed-precision solve: complex64 inner iterations inside an FP64 defect-correction loop.

The plain iteration's fixed point solves (G^{-1} - chi) E = s' (all at the current alpha; reference
solver.py:1070-1075 with E = G (chi E + s')).  For an FP64 iterate x the defect

    r(x) = s' + chi x - G^{-1} x                                  (FP64 on the device: one FFT pair, mmx_defect)

is a source for which the plain iteration converges to the correction delta = x* - x.  So each outer step casts
r(x) to complex64, runs the unchanged fused complex64 iteration from delta = 0 until its own residue falls below
``inner_rtol``, and accumulates x += delta in FP64 (mmx_accumulate).  The first inner update from delta = 0 is
d(x) = chi G r(x), the update the plain iteration would make at x, so ||d(x)|| / ||x|| is the relative residue of
the outer iterate (the reference's residue, solver.py:1026-1042, evaluated at x).  Divergence-guard rejections in
an inner solve raise alpha for that right-hand side; the defect of the next outer step is taken at that alpha, so
both levels stay consistent.  FP64 is used only for the defect, the norms and the accumulated solution.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as nat
from .batch import BatchSolution, prepare_material
from .engine import pack_symmetric
from .grid import Grid


def _ptr(t):
    return nat.device_ptr(t)


def _stream():
    s = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(s) if s else None


class MixedSolution:
    def __init__(self, grid: Grid, sources, epsilon, bound=None, vacuum_wavelength=None, wavenumber=None,
                 device=None, initial_field=None):
        """``initial_field`` (optional, [B, C, *grid] or [C, *grid], in the units of ``E``): the FP64 iterate to start
        from instead of zero, e.g. the solution of a nearby problem."""
        if not isinstance(grid, Grid):
            grid = Grid.from_ranges(*grid)
        self.grid = grid
        self.wavenumber = 2 * np.pi / vacuum_wavelength if vacuum_wavelength is not None else float(wavenumber)
        pre, bound = prepare_material(grid, epsilon, bound, self.wavenumber, np.complex128)
        src = np.asarray(sources)
        if src.ndim == grid.ndim + 1:
            src = src[np.newaxis]
        # the inner iteration's sources are the defects, written on the device: start them at zero there
        dev0 = torch.device(device if device is not None else 'cuda')
        self.inner = BatchSolution(grid, torch.zeros(src.shape, dtype=torch.complex64, device=dev0), None,
                                   bound=bound, wavenumber=self.wavenumber, dtype=np.complex64, device=device,
                                   preconditioner=pre)
        self.pre = pre
        self.batch, self.ncomp = self.inner.batch, self.inner.ncomp
        eng = self.inner.engine
        self.device = eng.device
        N = eng.N
        with torch.cuda.device(self.device):
            self.plan64 = nat.Plan(grid.shape, self.ncomp, self.batch, nat.MMX_C128)
            self.plan64.set_kvectors([np.asarray(k, dtype=np.float64).ravel() for k in (grid * self.wavenumber).k])
            if pre.chi_device is not None and int(pre.chi_device.shape[1]) == N:
                self.chi64 = pre.chi_device.to(self.device, torch.complex128).contiguous()
            else:
                m = pre.chi.shape[0] * pre.chi.shape[1]
                chi = np.broadcast_to(pre.chi, (pre.chi.shape[0], pre.chi.shape[1], *grid.shape)).reshape(m, N)
                # C order explicitly: a permittivity built as a strided view reshapes to a strided view too
                self.chi64 = torch.from_numpy(np.require(np.ascontiguousarray(chi, dtype=np.complex128),
                                                         requirements='W')).to(self.device)
            # a 3x3 chi equal to its transpose in FP64 is kept as its six distinct entries, as the inner
            # iteration keeps its complex64 copy
            self.chi64, self.chi64_kind = pack_symmetric(self.chi64)
            # s'0 = i s / (alpha_i beta) in FP64, scaled on the device (one upload of the sources, no host copy when
            # they are already contiguous complex128)
            s_host = np.require(np.ascontiguousarray(src, dtype=np.complex128), requirements='W')
            self.src64 = torch.from_numpy(s_host).to(self.device).reshape(self.batch, self.ncomp, N)
            self.src64 *= 1.0j / pre.alpha.imag / pre.beta
            self.x = torch.zeros((self.batch, self.ncomp, N), dtype=torch.complex128, device=self.device)
            if initial_field is not None:
                x0 = torch.as_tensor(initial_field, dtype=torch.complex128, device=self.device)
                self.x.copy_(torch.broadcast_to(x0.reshape(-1, self.ncomp, N), self.x.shape) * self.wavenumber ** 2)
            self._norms = torch.zeros(self.batch, dtype=torch.float64, device=self.device)
        self.outer_residues = []
        self.inner_iterations = []

    def tune(self, iters: int = 10, candidates=None) -> dict:
        """Choose the inner iteration's kernel variant with the autotuner.  The inner solves start from zero sources
        (the defects are written later), so the trials run on this problem's own sources s'0 cast to complex64;
        the inner sources and state are restored afterwards."""
        from . import autotune
        eng = self.inner.engine
        saved_src = eng.sources.clone()
        saved_state = eng.state.clone()
        try:
            eng.sources.copy_(self.src64.to(eng.sources.dtype))
            eng._mark_zero_sources()
            kw = {} if candidates is None else {'candidates': tuple(candidates)}
            return autotune.tune(eng, iters=iters, use_cache=False, **kw)
        finally:
            eng.sources.copy_(saved_src)
            eng.state.copy_(saved_state)

    def _xnorms(self) -> np.ndarray:
        """FP64 norms of every right-hand side's x, read back once (the launches queue on one stream and share the
        plan's scratch in order)."""
        n = self.ncomp * self.inner.engine.N
        for b in range(self.batch):
            nat.call('mmx_norm', self.plan64.handle, _ptr(self.x[b]), n, nat.MMX_C128, _ptr(self._norms[b:b + 1]),
                     _stream())
        return self._norms.cpu().numpy()

    # -- one outer step in phases (MixedUnevenSolution runs the inner solves of several grids together) ---------
    def _outer_begin(self, rtol: float) -> bool:
        """Defect and first correction step of every unconverged right-hand side; True when all have converged."""
        eng = self.inner.engine
        done = self._done
        # every unconverged right-hand side is active for the defect and for one first correction step
        eng.fields.zero_()  # both buffers, in place (no batch-sized allocation)
        st = eng.read_state()
        st['prev_norm'] = np.inf
        st['iteration'] = 0
        st['rtol'] = -1.0
        st['maxiter'] = 1
        st['active'] = (~done).astype(np.int32)
        st['status'] = 0
        st['reserved'][:, 1] = 0  # the defect overwrites the inner sources: no component is known to be zero
        eng.write_state(st)
        nat.call('mmx_defect', self.plan64.handle, _ptr(self.x), _ptr(self.chi64), self.chi64_kind, _ptr(self.src64),
                 _ptr(eng.state), _ptr(eng.sources), _stream())
        eng.iterate(1)  # first correction step: its update norm is ||d(x)||
        st = eng.read_state()
        res = np.full(self.batch, np.inf)
        xn = self._xnorms()
        pos = xn > 0
        res[pos] = st['last_norm'][pos] / xn[pos]
        res[done] = 0.0
        self.outer_residues.append(res.copy())
        done |= (res < rtol) & ~done
        if np.all(done):
            return True
        # the inner solves of the unconverged right-hand sides go on from here
        st['iteration'] = 1
        st['rtol'] = self._inner_rtol
        st['maxiter'] = self._inner_maxiter
        st['active'] = (~done).astype(np.int32)
        eng.write_state(st)
        return False

    def _outer_end(self):
        """x += delta for every right-hand side that was still correcting."""
        eng = self.inner.engine
        st = eng.read_state()
        self.inner_iterations.append(st['iteration'].copy())
        for b in range(self.batch):  # x += delta from the current buffer of each right-hand side (no gather)
            if not self._done[b]:
                nat.call('mmx_accumulate', _ptr(self.x[b]), _ptr(eng.fields[int(st['cur'][b]), b]),
                         self.ncomp * eng.N, _stream())

    def _start(self, inner_rtol: float, inner_maxiter: int):
        self._done = np.zeros(self.batch, dtype=bool)
        self._inner_rtol, self._inner_maxiter = inner_rtol, inner_maxiter

    def solve(self, rtol: float = 1e-8, inner_rtol: float = 1e-4, inner_maxiter: int = 100000, max_outer: int = 30):
        eng = self.inner.engine
        self._start(inner_rtol, inner_maxiter)
        for _ in range(max_outer):
            if self._outer_begin(rtol):
                break
            chunk = 8
            cont = False  # the inner solve's later chunks continue its first (the loop only reads the state)
            while True:
                eng.iterate(chunk, cont=cont)
                cont = True
                if not np.any(eng.read_state()['active']):
                    break
                chunk = min(2 * chunk, 64)
            self._outer_end()
        self.converged = self._done
        return self

    @property
    def residues(self) -> np.ndarray:
        return self.outer_residues[-1] if self.outer_residues else np.full(self.batch, np.inf)

    @property
    def alphas(self) -> np.ndarray:
        return self.inner.alphas

    @property
    def E(self) -> np.ndarray:
        """FP64 solution [B, C, *grid] (divided by k0^2)."""
        return (self.x.cpu().numpy() / self.wavenumber ** 2).reshape(self.batch, self.ncomp, *self.grid.shape)

    @property
    def total_inner_iterations(self) -> int:
        return int(sum(int(np.max(i)) for i in self.inner_iterations)) + len(self.outer_residues)

    def close(self):
        self.plan64.close()
        self.inner.close()


class MixedUnevenSolution:
    """
    The mixed-precision solve for several batches on grids of different sizes (e.g. 64 x 128^2, 32 x 256^2 and
    8 x 384^2 sources of one material class): each member keeps its own FP64 iterate, defect and complex64 inner
    iteration (a MixedSolution), and in every outer step the inner solves of all members run together, one captured
    CUDA graph per chunk of iterations with each member's passes as an independent branch (UnevenBatch).
    """

    def __init__(self, members):
        from .batch import UnevenBatch
        self.members = list(members)
        self._uneven = UnevenBatch([m.inner for m in self.members])

    def solve(self, rtol: float = 1e-8, inner_rtol: float = 1e-4, inner_maxiter: int = 100000, max_outer: int = 30):
        for m in self.members:
            m._start(inner_rtol, inner_maxiter)
        for _ in range(max_outer):
            finished = [m._outer_begin(rtol) if not np.all(m._done) else True for m in self.members]
            if all(finished):
                break
            chunk = 8
            while True:
                self._uneven.iterate(chunk)
                if not any(np.any(m.inner.engine.read_state()['active']) for m in self.members):
                    break
                chunk = min(2 * chunk, 64)
            for m, f in zip(self.members, finished):
                if not f:
                    m._outer_end()
        for m in self.members:
            m.converged = m._done
        return self

    @property
    def residues(self):
        return [m.residues for m in self.members]

    @property
    def total_inner_iterations(self) -> int:
        return max(m.total_inner_iterations for m in self.members)

    def close(self):
        for m in self.members:
            m.close()
