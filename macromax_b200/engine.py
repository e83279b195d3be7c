"""
Device engine of the split-Richardson iteration: one material on one grid, ``batch`` right-hand sides.

Owns (as torch tensors on the plan's device) the susceptibility chi0 stored at alpha0, the normalised sources
s'0, the two field buffers of the ping-pong update and the per-RHS ``mmx_rhs_state`` array, plus the native plan
(twiddles, k tables, work buffer).  All iteration work is done by ``mmx_iterate`` of the native library; the host
only edits the small state array between calls (reset of the update norm, stop rule) and reads it back.
"""
from __future__ import annotations


import numpy as np
import torch

from . import _native as nat


def _complex_dtype(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.complex64:
        return torch.complex64, nat.MMX_C64
    if dtype == np.complex128:
        return torch.complex128, nat.MMX_C128
    raise TypeError(f'unsupported dtype {dtype}: use complex64 or complex128')


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes_void(s.cuda_stream)


def ctypes_void(v):
    import ctypes
    return ctypes.c_void_p(int(v)) if v else None


def _ptr(t: torch.Tensor):
    return nat.device_ptr(t)


def pack_symmetric(chi: torch.Tensor) -> tuple[torch.Tensor, int]:
    """chi: [1 | 9, N] (a scalar or a row-major 3x3 per voxel).  Returns (chi, kind): a 3x3 that equals its transpose
    exactly (every reciprocal medium: a symmetric permittivity, as in uniaxial grains) as its six distinct entries
    xx, xy, xz, yy, yz, zz (MMX_CHI_SYM6), so the prologue and epilogue passes read 6 words per voxel instead of 9;
    any other 3x3 as it is (MMX_CHI_MAT3); a scalar as it is (MMX_CHI_SCALAR)."""
    m = int(chi.shape[0])
    if m == 1:
        return chi, nat.MMX_CHI_SCALAR
    if m != 9:
        raise ValueError('chi must hold 1 or 9 entries per voxel')
    if torch.equal(chi[1], chi[3]) and torch.equal(chi[2], chi[6]) and torch.equal(chi[5], chi[7]):
        return chi[list(nat.SYM6_ROWS)].contiguous(), nat.MMX_CHI_SYM6
    return chi, nat.MMX_CHI_MAT3


class IterationEngine:
    def __init__(self, shape, ncomp: int, batch: int, dtype, ks, chi0: np.ndarray, alpha0: complex,
                 device=None):
        if not torch.cuda.is_available():
            raise ImportError('macromax_b200 needs a CUDA device')
        nat.load()
        self.device = torch.device(device if device is not None else 'cuda')
        self.shape = tuple(int(s) for s in shape)
        self.ndim = len(self.shape)
        self.N = int(np.prod(self.shape))
        self.ncomp = int(ncomp)
        self.batch = int(batch)
        self.np_dtype = np.dtype(dtype)
        self.torch_dtype, self.precision = _complex_dtype(dtype)
        with torch.cuda.device(self.device):
            self.plan = nat.Plan(self.shape, self.ncomp, self.batch, self.precision)
            self.plan.set_kvectors([np.asarray(k, dtype=np.float64).ravel() for k in ks])
            self.fields = torch.zeros((2, self.batch, self.ncomp, self.N), dtype=self.torch_dtype, device=self.device)
            self.sources = torch.zeros((self.batch, self.ncomp, self.N), dtype=self.torch_dtype, device=self.device)
            self.state = torch.zeros((self.batch, nat.STATE_DTYPE.itemsize), dtype=torch.uint8, device=self.device)
        self.set_chi(chi0, alpha0)
        st = np.zeros(self.batch, dtype=nat.STATE_DTYPE)
        st['alpha_re'] = st['alpha0_re'] = alpha0.real
        st['alpha_im'] = st['alpha0_im'] = alpha0.imag
        st['prev_norm'] = np.inf
        st['rtol'] = -1.0
        st['maxiter'] = np.inf
        st['active'] = 1
        self.write_state(st)

    # -- material ---------------------------------------------------------------------------------------------------
    def set_chi(self, chi0, alpha0: complex):
        """chi0: matrix field [1|3, 1|3, *grid-broadcastable] at alpha0 (expanded to the full grid here), or a device
        tensor [m, N] (m = 1 or 9), used without a host round trip."""
        if isinstance(chi0, torch.Tensor):
            m = int(chi0.shape[0])
            if m not in (1, 9) or chi0.dim() != 2 or int(chi0.shape[1]) != self.N:
                raise ValueError('a device chi must be [1 or 9, N]')
            if m == 9 and self.ncomp != 3:
                raise ValueError('an anisotropic susceptibility needs a vector field')
            self.chi_kind = nat.MMX_CHI_SCALAR if m == 1 else nat.MMX_CHI_MAT3
            self.chi = chi0.to(self.device, self.torch_dtype).contiguous()
            self.alpha0 = complex(alpha0)
            self._pack_symmetric()
            return
        chi0 = np.asarray(chi0)
        m = chi0.shape[0] * chi0.shape[1]
        if m not in (1, 9):
            raise ValueError('chi must be 1x1 or 3x3')
        if m == 9 and self.ncomp != 3:
            raise ValueError('an anisotropic susceptibility needs a vector field')
        full = np.broadcast_to(chi0, (chi0.shape[0], chi0.shape[1], *self.shape)).reshape(m, self.N)
        self.chi_kind = nat.MMX_CHI_SCALAR if m == 1 else nat.MMX_CHI_MAT3
        self.chi = torch.from_numpy(np.array(full, dtype=self.np_dtype, order='C')).to(self.device)
        self.alpha0 = complex(alpha0)
        self._pack_symmetric()

    def _pack_symmetric(self):
        self.chi, self.chi_kind = pack_symmetric(self.chi)

    def rebase_alpha(self, chi0: np.ndarray, alpha0: complex, sources0: np.ndarray | None = None):
        """Install a new material (chi at alpha0) and reset every RHS's alpha to alpha0."""
        self.set_chi(chi0, alpha0)
        st = self.read_state()
        st['alpha_re'] = st['alpha0_re'] = alpha0.real
        st['alpha_im'] = st['alpha0_im'] = alpha0.imag
        self.write_state(st)
        if sources0 is not None:
            self.set_sources(sources0)

    def set_sources(self, src0, index=None):
        """Normalised sources s'0 at alpha0: array broadcastable to [batch, ncomp, *grid] (or [ncomp, *grid])."""
        if isinstance(src0, torch.Tensor):
            t = src0.to(self.device, self.torch_dtype)
        else:
            t = torch.from_numpy(np.ascontiguousarray(src0, dtype=self.np_dtype)).to(self.device)
        if index is None:
            self.sources.copy_(t.reshape(-1, self.ncomp, self.N).expand(self.batch, self.ncomp, self.N))
        else:
            self.sources[index].copy_(t.reshape(self.ncomp, self.N))
        self._mark_zero_sources()

    def _mark_zero_sources(self):
        """Record in every right-hand side's state which source components are identically zero (bit c of
        reserved[1]); the prologue kernels then skip reading those components.  Whoever writes the sources by other
        means clears the bits (the mixed-precision defect does)."""
        zero = ~(self.sources != 0).any(dim=2)  # [B, C]
        weights = torch.tensor([1 << c for c in range(self.ncomp)], dtype=torch.int32, device=self.device)
        bits = (zero.to(torch.int32) * weights).sum(dim=1).cpu().numpy()
        st = self.read_state()
        st['reserved'][:, 1] = bits
        self.write_state(st)

    # -- state ------------------------------------------------------------------------------------------------------
    def read_state(self) -> np.ndarray:
        raw = self.state.cpu().numpy()
        return raw.view(nat.STATE_DTYPE).reshape(self.batch).copy()

    def write_state(self, st: np.ndarray):
        raw = np.ascontiguousarray(st, dtype=nat.STATE_DTYPE).view(np.uint8).reshape(self.batch, -1)
        self.state.copy_(torch.from_numpy(raw.copy()).to(self.device))

    def reset_alpha(self, index=None):
        """Return alpha to alpha0 (the stored chi and sources), e.g. before solving a new, unrelated problem."""
        st = self.read_state()
        sel = slice(None) if index is None else index
        st['alpha_re'][sel] = st['alpha0_re'][sel]
        st['alpha_im'][sel] = st['alpha0_im'][sel]
        self.write_state(st)

    def reset_update_norm(self, index=None):
        st = self.read_state()
        sel = slice(None) if index is None else index
        st['prev_norm'][sel] = np.inf
        self.write_state(st)

    # -- fields -----------------------------------------------------------------------------------------------------
    def current(self, st: np.ndarray | None = None) -> torch.Tensor:
        """[batch, ncomp, N] view-gather of the current field buffers."""
        st = self.read_state() if st is None else st
        cur = torch.from_numpy(st['cur'].astype(np.int64)).to(self.device)
        return self.fields[cur, torch.arange(self.batch, device=self.device)]

    def set_fields(self, E, index=None):
        """Set the current field (already scaled by k0^2); resets previous_update_norm like the E setter."""
        st = self.read_state()
        if isinstance(E, torch.Tensor):
            t = E.to(self.device, self.torch_dtype)
        else:
            t = torch.from_numpy(np.ascontiguousarray(E, dtype=self.np_dtype)).to(self.device)
        idx = range(self.batch) if index is None else [index]
        t = t.reshape(-1, self.ncomp, self.N)
        for i, b in enumerate(idx):
            self.fields[int(st['cur'][b]), b].copy_(t[i if t.shape[0] > 1 else 0])
            st['prev_norm'][b] = np.inf
        self.write_state(st)

    # -- iteration --------------------------------------------------------------------------------------------------
    use_graphs = True  # replay captured CUDA graphs for multi-iteration chunks

    def iterate(self, niter: int, stream=None, cont: bool = False):
        """``niter`` iterations on the stream.  cont: the next chunk of the same solve -- nothing has written the
        fields, chi, sources or states since the previous call -- so the chunk may start from the first pass that
        the previous chunk's fused epilogue left in the work buffer (mmx_iterate_graph_continue)."""
        if niter <= 0:
            return
        if self.use_graphs and niter > 1:
            fn = 'mmx_iterate_graph_continue' if cont else 'mmx_iterate_graph'
        else:
            fn = 'mmx_iterate'
        nat.call(fn, self.plan.handle, _ptr(self.fields[0]), _ptr(self.fields[1]), _ptr(self.chi),
                 self.chi_kind, _ptr(self.sources), _ptr(self.state), int(niter), _stream_ptr(stream))

    def prepare_graph(self, niter: int):
        """Capture the graph of an ``niter``-iteration chunk now (so that a later timed chunk does not)."""
        nat.call('mmx_iterate_graph_prepare', self.plan.handle, _ptr(self.fields[0]), _ptr(self.fields[1]),
                 _ptr(self.chi), self.chi_kind, _ptr(self.sources), _ptr(self.state), int(niter))

    def run(self, rtol: float, maxiter: float, chunk: int = 8, max_chunk: int = 64,
            reset_iteration: bool = True) -> np.ndarray:
        """Iterate every active RHS until its stop rule (iteration < maxiter and residue > rtol) fails; the iteration
        count starts from 0 (as every Solution.solve, solver.py:1063), or goes on from its current value
        (reset_iteration=False)."""
        st = self.read_state()
        if reset_iteration:
            st['iteration'] = 0
        st['rtol'] = rtol
        st['maxiter'] = maxiter
        st['active'] = 1
        st['status'] = 0
        self.write_state(st)
        cont = False  # the chunks after the first continue the same solve (the loop only reads the state)
        while True:
            self.iterate(chunk, cont=cont)
            cont = True
            st = self.read_state()
            if not np.any(st['active']):
                break
            chunk = min(chunk * 2, max_chunk)
        return st

    def to_host(self, t: torch.Tensor) -> np.ndarray:
        """Copy a device tensor to a new host array through a pinned staging buffer (kept for the next call), which
        runs at full link speed instead of the pageable-copy rate."""
        nbytes = t.numel() * t.element_size()
        buf = getattr(self, '_pinned', None)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            self._pinned = buf
        view = buf[:nbytes].view(t.dtype).view(t.shape)
        view.copy_(t.contiguous())
        torch.cuda.current_stream(t.device).synchronize()
        return view.numpy().copy()

    def close(self):
        if getattr(self, 'plan', None) is not None:
            self.plan.close()
            self.plan = None
