"""
``BackEndB200``: the reference's ``BackEnd`` interface (backend/__init__.py:37-880) on device tensors, with the
transform and norm served by the native sm_100a kernels, plus ``register()`` which adds the ``'b200'`` type to the
reference's ``macromax.backend.load`` when that package is importable.

The reference's ``Solution`` calls these methods for its set-up and post-processing; its iteration calls ``mul``,
``convolve`` (``ft`` / ``ift``), ``longitudinal_projection_ft`` and ``norm`` per step.  The fused step that replaces
the whole iteration body (solver.py:1070-1096) is ``mmx_iterate``, used by ``macromax_b200.Solution``.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import _native as nat
from .grid import Grid


def _ptr(t):
    return nat.device_ptr(t)


def _stream():
    s = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(s) if s else None


class BackEndB200:
    """Parallel operations on [rows, cols, *grid] matrix fields held on a B200 (backend/__init__.py:37-67)."""

    def __init__(self, nb_dims: int, grid: Grid, hardware_dtype=np.complex128, device: str | None = None):
        if not torch.cuda.is_available():
            raise ImportError('BackEndB200 needs a CUDA device')
        nat.load()  # ImportError when the native library is missing: backend.load falls through
        dt = np.dtype(hardware_dtype)
        if dt == np.complex64:
            self._tdtype, self._prec = torch.complex64, nat.MMX_C64
        elif dt == np.complex128:
            self._tdtype, self._prec = torch.complex128, nat.MMX_C128
        else:
            raise TypeError(f'unsupported dtype {hardware_dtype}')
        self._np_dtype = dt
        self._device = torch.device(device if device else 'cuda')
        self._nb_rows = int(nb_dims)
        self._grid = grid
        self._plan = nat.Plan(tuple(int(s) for s in grid.shape), 1, 1, self._prec)
        self._plan.set_kvectors([np.asarray(k, dtype=np.float64).ravel() for k in grid.k])
        self._k = None
        self._k2 = None
        self._eye = None
        self._ft_in = None
        self._ft_out = None
        self._norm_out = torch.zeros(1, dtype=torch.float64, device=self._device)

    # -- properties (backend/__init__.py:69-128) ----------------------------------------------------------------------
    @property
    def vector_length(self) -> int:
        return self._nb_rows

    @property
    def ft_axes(self) -> tuple:
        return tuple(range(2, 2 + self._grid.ndim))

    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def vectorial(self) -> bool:
        return self._nb_rows > 1

    @property
    def hardware_dtype(self):
        return self._tdtype

    @property
    def numpy_dtype(self):
        return self._np_dtype.type

    @property
    def eps(self) -> float:
        return float(np.finfo(self._np_dtype).eps)

    @property
    def device(self):
        return self._device

    # -- array handling ----------------------------------------------------------------------------------------------
    def astype(self, arr, dtype=None) -> torch.Tensor:
        if dtype is None:
            tdt = self._tdtype
        elif dtype in (np.complex64, torch.complex64):
            tdt = torch.complex64
        elif dtype in (np.complex128, complex, torch.complex128):
            tdt = torch.complex128
        elif dtype in (np.float32, torch.float32):
            tdt = torch.float32
        elif dtype in (np.float64, float, torch.float64):
            tdt = torch.float64
        elif dtype in (bool, np.bool_, torch.bool):
            tdt = torch.bool
        elif dtype in (int, np.int64, torch.int64):
            tdt = torch.int64
        else:
            tdt = dtype
        if isinstance(arr, torch.Tensor):
            return arr.to(dtype=tdt, device=self._device)
        return torch.as_tensor(np.asarray(arr), device=self._device).to(tdt)

    def asnumpy(self, arr) -> np.ndarray:
        if isinstance(arr, torch.Tensor):
            return arr.detach().resolve_conj().cpu().numpy()
        return np.asarray(arr)

    def allocate_array(self, shape=None, dtype=None, fill_value=None) -> torch.Tensor:
        shape = tuple(int(s) for s in (shape if shape is not None else (self._nb_rows, 1, *self._grid.shape)))
        arr = torch.empty(shape, dtype=self.astype(np.zeros(1), dtype).dtype if dtype is not None else self._tdtype,
                          device=self._device)
        if fill_value is not None:
            arr.fill_(fill_value)
        return arr

    @property
    def array_ft_input(self) -> torch.Tensor:
        if self._ft_in is None:
            self._ft_in = self.allocate_array()
        return self._ft_in

    @property
    def array_ft_output(self) -> torch.Tensor:
        if self._ft_out is None:
            self._ft_out = self.allocate_array()
        return self._ft_out

    def assign_exact(self, arr, out):
        out[...] = self.astype(arr)
        return out

    def assign(self, arr, out):
        arr = self.to_matrix_field(arr)
        out[...] = torch.broadcast_to(arr, out.shape)
        return out

    def copy(self, arr):
        return arr.detach().clone() if isinstance(arr, torch.Tensor) else self.astype(arr)

    def ravel(self, arr):
        return arr.reshape(-1) if isinstance(arr, torch.Tensor) else np.ravel(arr)

    def first(self, arr):
        return self.ravel(arr)[0]

    def to_matrix_field(self, arr) -> torch.Tensor:
        """backend/__init__.py:355-385."""
        arr = self.astype(0 if arr is None else arr)
        while arr.dim() < self._grid.ndim + 2:
            arr = arr.unsqueeze(0)
        if arr.shape[0] == 1 and arr.shape[1] > 1:
            arr = arr.transpose(0, 1)
        return arr

    @property
    def eye(self) -> torch.Tensor:
        if self._eye is None:
            n = self._nb_rows
            self._eye = self.astype(np.eye(n).reshape(n, n, *([1] * self._grid.ndim)))
        return self._eye

    def is_scalar(self, arr) -> bool:
        if not isinstance(arr, torch.Tensor):
            arr = np.asarray(arr)
        return arr.ndim == 0 or (arr.shape[0] == 1 and (arr.ndim == 1 or arr.shape[1] == 1))

    def adjoint(self, mat):
        return torch.conj(self.astype(mat).transpose(0, 1))

    def conj(self, arr):
        return torch.conj(self.astype(arr))

    def real(self, arr):
        return arr.real

    def abs(self, arr):
        return self.astype(arr).abs()

    def any(self, arr) -> bool:
        return bool(torch.any(torch.as_tensor(arr, device=self._device).to(torch.bool)))

    def allclose(self, arr, other=0.0) -> bool:
        a = self.astype(arr)
        return bool(torch.allclose(a, torch.broadcast_to(self.astype(other), a.shape)))

    def amax(self, arr) -> float:
        return float(torch.amax(torch.as_tensor(arr, device=self._device).real))

    def sign(self, arr):
        return torch.sign(arr)

    def swapaxes(self, arr, a, b):
        return arr.transpose(a, b)

    @staticmethod
    def expand_dims(arr, axis):
        return arr.unsqueeze(axis)

    def sort(self, arr):
        return torch.sort(arr.real if torch.is_complex(arr) else arr, dim=0).values

    def subtract(self, left, right):
        """backend/__init__.py:397-413."""
        if not self.is_scalar(left) or not self.is_scalar(right):
            if self.is_scalar(left):
                left = self.eye * self.to_matrix_field(left)
            if self.is_scalar(right):
                right = self.eye * self.to_matrix_field(right)
        return self.astype(left) - self.astype(right)

    def mul(self, left, right, out=None):
        """
        Pointwise matrix product (backend/__init__.py:415-444); matrix x matrix-field products run in the native
        kernel ``mmx_pointwise_mul``.
        """
        if self.is_scalar(left) or self.is_scalar(right):
            if out is not None:
                out *= self.astype(left)
                return out
            return self.astype(left) * self.astype(right)
        a = self.to_matrix_field(left)
        b = self.to_matrix_field(right)
        shape = torch.broadcast_shapes(a.shape[2:], b.shape[2:])
        nvox = int(np.prod(shape))
        ra, ca, cb = a.shape[0], a.shape[1], b.shape[1]
        a_full = torch.broadcast_to(a, (ra, ca, *shape)).contiguous().to(self._tdtype)
        b_bcast = b.shape[2:] != shape and all(s == 1 for s in b.shape[2:])
        b_full = (b.contiguous() if b_bcast else torch.broadcast_to(b, (b.shape[0], cb, *shape)).contiguous())
        b_full = b_full.to(self._tdtype)
        res = torch.empty((ra, cb, *shape), dtype=self._tdtype, device=self._device)
        nat.call('mmx_pointwise_mul', _ptr(a_full), ra, ca, _ptr(b_full), cb, int(b_bcast), _ptr(res), nvox,
                 self._prec, _stream())
        if out is not None and out.shape == res.shape:
            out.copy_(res)
            return out
        return res

    def ldivide(self, denominator, numerator=1.0):
        """backend/__init__.py:446-460 (3x3 inverses on the device via torch.linalg)."""
        d = self.to_matrix_field(denominator)
        n = self.to_matrix_field(numerator)
        if self.is_scalar(d):
            return n / d
        dm = d.movedim(0, -1).movedim(0, -1)
        if self.is_scalar(n):
            res = torch.linalg.inv(dm) * n.reshape(())
        else:
            res = torch.linalg.solve(dm, n.movedim(0, -1).movedim(0, -1))
        return res.movedim(-1, 0).movedim(-1, 0)

    def inv(self, mat):
        return self.ldivide(mat, 1.0)

    # -- Fourier space ------------------------------------------------------------------------------------------------
    def _fft(self, arr, inverse: int):
        x = self.astype(arr).contiguous()
        nb = int(np.prod(x.shape[:-self._grid.ndim])) if x.dim() > self._grid.ndim else 1
        out = torch.empty_like(x)
        nat.call('mmx_fftn', self._plan.handle, _ptr(x), _ptr(out), nb, int(inverse), _stream())
        return out

    def ft(self, arr):
        """backend/__init__.py:234-244 on the native FFT (mmx_fftn, forward, unscaled)."""
        return self._fft(arr, 0)

    def ift(self, arr):
        """backend/__init__.py:246-257 on the native FFT (scaled by 1/N)."""
        return self._fft(arr, 1)

    def convolve(self, operation_ft, arr):
        return self.ift(operation_ft(self.ft(arr)))

    @property
    def k(self) -> Sequence[torch.Tensor]:
        if self._k is None:
            self._k = [self.astype(k) for k in self._grid.k]
        return self._k

    @property
    def k2(self) -> torch.Tensor:
        if self._k2 is None:
            self._k2 = sum(k ** 2 for k in self.k)
        return self._k2

    def longitudinal_projection_ft(self, F):
        """backend/__init__.py:606-649 (DC passed through, components >= ndim zero); a per-op tensor expression (the
        fused iteration applies the projection inside its axis-0 pass)."""
        F = self.astype(F)
        nd = self._grid.ndim
        proj = F[0, 0] * self.k[0]
        for a in range(1, nd):
            proj = proj + self.k[a] * F[a, 0]
        k2 = torch.broadcast_to(self.k2, proj.shape).reshape(-1)
        flat = proj.reshape(-1).clone()
        flat[1:] = flat[1:] / k2[1:]
        proj = flat.reshape(proj.shape)
        res = torch.zeros((max(nd, F.shape[0]), *F.shape[1:]), dtype=F.dtype, device=self._device)
        zero = (0,) * nd
        for a in range(nd):
            res[a, 0] = self.k[a] * proj
            res[a, 0][zero] = F[a, 0][zero]
        return res

    def transversal_projection_ft(self, F):
        F = self.astype(F)
        return F - self.longitudinal_projection_ft(F)

    def curl_ft(self, F):
        """backend/__init__.py:483-509: i k x F.  A 3-component field of this grid goes through mmx_curl_ft."""
        F = self.astype(F)
        n = self._nb_rows
        if n == 3 and F.shape[0] == 3 and F.numel() == 3 * self._grid.size:
            Fc = F.contiguous()
            out = torch.empty_like(Fc)
            nat.call('mmx_curl_ft', self._plan.handle, _ptr(Fc), _ptr(out), _stream())
            return out
        out = torch.zeros((n, *F.shape[1:]), dtype=self._tdtype, device=self._device)
        for d in range(n):
            o = (d + np.array([-1, 1])) % n
            if o[0] < F.shape[0] and o[1] < len(self.k):
                out[d] = self.k[o[1]] * F[o[0]]
            if o[1] < F.shape[0] and o[0] < len(self.k):
                out[d] = out[d] - self.k[o[0]] * F[o[1]]
        return 1j * out

    def curl(self, F):
        return self.convolve(self.curl_ft, F)

    def norm(self, arr) -> float:
        """backend/__init__.py:872-874 on the native FP64-accumulated reduction (mmx_norm)."""
        x = self.astype(arr).contiguous()
        nat.call('mmx_norm', self._plan.handle, _ptr(x), x.numel(), self._prec, _ptr(self._norm_out), _stream())
        return float(self._norm_out.item())

    def mat3_eigh(self, arr):
        """Eigenvalues of Hermitian 3x3 fields (backend/__init__.py:670-723), as a [3, *grid] array."""
        a = self.astype(arr)
        if a.shape[0] == 3 and a.shape[1] == 3:
            return torch.linalg.eigvalsh(a.movedim(0, -1).movedim(0, -1)).movedim(-1, 0).to(self._tdtype)
        return a[0] if a.shape[0] == 1 else a[:, 0]

    @staticmethod
    def clear_cache():
        pass

    def __str__(self):
        return f'BackEndB200(vectorial={self.vectorial}, {self._grid}, dtype={self._np_dtype})'


def register(macromax_module=None):
    """
    Add the ``'b200'`` type to the reference's ``macromax.backend.load`` (backend/__init__.py:922-1012) and route the
    reference's ``Solution`` iteration to the fused kernels for it (``refhook.install``).  A config
    ``{'type': 'b200', 'device': 'cuda:0'}`` builds the reference-facing ``BackEndB200`` (a subclass of the
    reference's torch backend, ``refhook.backend_class``); when the GPU or the native library is missing the
    constructor raises ``ImportError`` and ``load`` moves on to the next configured backend, as it does for its own
    types.  Returns the wrapped ``load``.
    """
    if macromax_module is None:
        import macromax as macromax_module  # the reference package
    from . import refhook
    be = macromax_module.backend
    original = getattr(be.load, '_b200_original', be.load)

    def load(nb_pol_dims, grid, dtype, config_list=None):
        configs = list(config_list) if config_list is not None else None
        if configs is None:
            stored = getattr(be, '__config_list', None)  # set by backend.config (backend/__init__.py:914-919)
            configs = list(stored) if stored else []
        # backend.config([...]) stores the list itself as one element (backend/__init__.py:916): flatten it
        configs = [d for item in configs for d in (item if isinstance(item, (list, tuple)) else [item])]
        for i, c in enumerate(configs):
            if str(c.get('type', '')).lower() == 'b200':
                try:
                    return refhook.backend_class(macromax_module)(nb_pol_dims, grid, dtype, device=c.get('device'))
                except ImportError as ie:
                    be.log.info(f'Backend type "b200" did not load as expected: {ie}.')
                    continue
            return original(nb_pol_dims, grid, dtype, [c for c in configs[i:]
                                                       if str(c.get('type', '')).lower() != 'b200'])
        return original(nb_pol_dims, grid, dtype, [])

    load._b200_original = original
    be.load = load
    refhook.install(macromax_module)
    return load
