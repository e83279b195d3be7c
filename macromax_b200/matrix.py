"""
Scattering matrices on the batched B200 solve.

``ScatteringMatrix`` mirrors the reference class of the same name (matrix.py:356-848): the same constructor
arguments, mode ordering, source and detection planes, vector conversions and quarter matrices.  What changes is how
columns are computed.  The reference solves one column at a time with a single ``Solution`` (``_matvec``,
matrix.py:770-820; ``__array__``, matrix.py:831-844).  Here every column that is not cached is solved in one batched
launch of the fused iteration (``BatchSolution``: all right-hand sides share the material, its preconditioner and one
CUDA graph), in chunks that fit the device memory budget.  For the batched columns the mode synthesis and detection
run on the device (transverse plane transforms by mmx_fftn, spectra scattered and gathered at the mode positions by
mmx_mode_scatter / mmx_mode_gather); only the two source planes and the two detection planes of each column are
computed, instead of whole-grid free-space fields.  The single-vector conversions (srcvec2freespace, ...) keep the
host restatement.

Vectors are laid out as in the reference: ``[side (front, back), mode (raster order of the propagating transverse
k-vectors), polarisation (1 scalar, 2 vector)]``, flattened.

One difference from the reference's column loop, only visible in ill-conditioned runs: a divergence-guard rejection
raises alpha for that column only (the reference keeps the raised alpha for the columns after it).
"""
from __future__ import annotations

from typing import Callable, Optional

import ctypes
import time

import numpy as np
import scipy.constants as const
import torch

from .batch import BatchSolution
from .bound import Bound, PeriodicBound
from .grid import Grid
from .solver import Solution

_DEFAULT_RTOL = 1e-6
_DEFAULT_MAXITER = 10000


def _default_callback(s) -> bool:
    return s.iteration < _DEFAULT_MAXITER and s.residue > _DEFAULT_RTOL


def _stream():
    s = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(s) if s else None


def _synced_time() -> float:
    """Host time after the device has finished the queued work (phase timing of the batched columns)."""
    torch.cuda.synchronize()
    return time.perf_counter()


def _unit(v: np.ndarray, axis: int = 0) -> np.ndarray:
    """v / |v| along ``axis`` (zero vectors stay zero)."""
    n = np.linalg.norm(v, axis=axis, keepdims=True)
    return v / (n + (n == 0))


def _dot0(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Sum of products over the first axis."""
    return np.einsum('i...,i...->...', a, b)


class ScatteringMatrix:
    def __init__(self, grid, vectorial: Optional[bool] = True, wavenumber=None, angular_frequency=None,
                 vacuum_wavelength=None, epsilon=None, xi=0.0, zeta=0.0, mu=1.0, refractive_index=None,
                 bound: Bound = None, dtype=None, callback: Callable = None, caching: bool = True, array=None,
                 device=None, max_batch: int = 256, max_batch_bytes: float = 2e9):
        if not isinstance(grid, Grid):  # a coordinate range, or a sequence of them
            grid = Grid.from_ranges(*([grid] if np.isscalar(grid[0]) else grid))
        self._grid = grid
        self._vectorial = bool(vectorial)
        self._callback = callback
        self._device = device
        self._max_batch = int(max_batch)
        self._max_batch_bytes = float(max_batch_bytes)
        if angular_frequency is not None:
            k0 = angular_frequency / const.c
        elif vacuum_wavelength is not None:
            k0 = 2 * np.pi / vacuum_wavelength
        else:
            k0 = 1.0 if wavenumber is None else wavenumber
        self._k0 = float(k0)
        self._dtype = np.dtype(dtype if dtype is not None else np.complex128)
        # the solver of single columns (source2detfield) and source of the shared preconditioner, created on the
        # first solve (the vector conversions below need no device)
        self._material = dict(epsilon=epsilon, xi=xi, zeta=zeta, mu=mu, refractive_index=refractive_index,
                              bound=bound)
        self._solution_obj = None
        # propagating transverse modes (matrix.py:426-446): |k_t| below k0 minus a tolerance, in raster order of the
        # origin-centred transverse k-grid, stored as indices into the (origin-first) FFT layout
        k_centered = [np.fft.fftshift(np.ravel(k)) for k in grid.k]
        tol = np.sqrt(np.finfo(np.float64 if dtype is None else np.dtype(dtype)).eps)
        shape_t = tuple(int(n) for n in grid.shape[1:])
        propagating = np.ones(shape_t if shape_t else (1,), dtype=bool)
        k_rest = np.full(propagating.shape, k0, dtype=float)
        for axis in range(1, grid.ndim):
            view = [1] * len(shape_t)
            view[axis - 1] = shape_t[axis - 1]
            k = k_centered[axis].reshape(view)
            propagating = propagating & (np.abs(k) < k_rest - tol)
            k_rest = np.sqrt(np.maximum(k_rest ** 2 - k ** 2, 0.0))
        centred = np.flatnonzero(propagating.ravel())
        if grid.ndim > 1:
            subs = (np.asarray(np.unravel_index(centred, shape_t)) - (np.asarray(shape_t)[:, None] // 2)) \
                % np.asarray(shape_t)[:, None]
            self._modes = np.ravel_multi_index(subs, shape_t)
        else:
            self._modes = centred
        # source and detection planes along axis 0 (matrix.py:448-460); detection volumes listed back, front
        bnd = bound if bound is not None else PeriodicBound(grid)
        th = np.asarray(bnd.thickness, dtype=float)
        step0 = float(grid.step[0])
        n0 = int(grid.shape[0])
        self._source_planes = (int(th[0, 0] / step0) + 1, n0 - int(th[0, -1] / step0) - 1)
        wl = 2 * np.pi / k0
        self._detector_planes = (n0 - int((th[0, -1] + wl) / step0) - 1, int((th[0, 0] + wl) / step0) + 1)
        self._caching = bool(caching)
        self._columns = {}
        nb_modes = self._modes.size
        self._side = 2 * (1 + self._vectorial) * nb_modes
        if array is not None:
            array = np.asarray(array() if callable(array) else array)
            if np.any(np.array(array.shape) != self._side):
                raise ValueError(f'Number of modes {self._side} is different from the number of rows or columns of '
                                 f'the specified matrix {array.shape}!')
            for j, column in enumerate(array.transpose()):
                self._columns[j] = column
        # unit k-vectors of the propagating modes (rows: axis 0, 1, 2)
        kdir = np.zeros((3, nb_modes))
        for axis in range(1, grid.ndim):
            view = [1] * len(shape_t)
            view[axis - 1] = shape_t[axis - 1]
            kt = np.broadcast_to((np.ravel(grid.k[axis]) / k0).reshape(view), shape_t).ravel()
            kdir[axis] = kt[self._modes]
        kdir[0] = np.sqrt(np.maximum(1.0 - np.sum(kdir[1:] ** 2, axis=0), 0.0))
        self._kdir = kdir

    # -- properties -------------------------------------------------------------------------------------------------
    @property
    def _solution(self) -> Solution:
        if self._solution_obj is None:
            nb_pol = 1 + 2 * self._vectorial
            self._solution_obj = Solution(self._grid, vectorial=self._vectorial, wavenumber=self._k0,
                                          source_distribution=np.zeros((nb_pol, *self._grid.shape), dtype=self._dtype),
                                          dtype=self._dtype, device=self._device, **self._material)
        return self._solution_obj

    @property
    def wavenumber(self) -> float:
        return self._k0

    @property
    def angular_frequency(self) -> float:
        return self._k0 * const.c

    @property
    def grid(self) -> Grid:
        return self._grid

    @property
    def vectorial(self) -> bool:
        return self._vectorial

    @property
    def dtype(self):
        return self._dtype

    @property
    def shape(self):
        return (self._side, self._side)

    @property
    def side(self) -> int:
        return self._side

    @property
    def caching(self) -> bool:
        return self._caching

    @caching.setter
    def caching(self, value: bool):
        self._caching = bool(value)
        if not self._caching:
            self._columns = {}

    # -- vector <-> field conversions (host) -------------------------------------------------------------------------
    def _as_modes(self, vector) -> np.ndarray:
        """[2, P, M] from a flat vector [side, mode, polarisation]."""
        v = np.array(vector, dtype=self._dtype).reshape(2, self._modes.size, 1 + self._vectorial)
        return np.moveaxis(v, -1, 1)

    def _plane_coefficients(self, vectors: np.ndarray, planes):
        """
        Spectral coefficients of the mode vectors ``vectors`` [B, 2, P, M] on the axis-0 planes ``planes``: for each
        side (forward, backward) an array [B, C, len(planes), M] that goes to the transverse spectrum positions of the
        modes, or None for a side without input.  The backward side's coefficients are conjugated here; its field is
        the conjugate of their transform (srcvec2freespace, matrix.py:528-610).
        """
        grid = self._grid
        k0 = self._k0
        kdir = self._kdir
        x0 = np.ravel(grid[0])[list(planes)]
        first_t = np.asarray(grid.first[1:], dtype=float)
        vectors = vectors / np.sqrt(kdir[0])  # entrance-aperture compensation
        if self._vectorial:
            axial = np.array([1.0, 0.0, 0.0])[:, None]
            radial_dir = _unit(_dot0(kdir, axial) * kdir - axial)  # [3, M]
            radial_mode_dir = _unit(kdir[1:])                       # [2, M]
        origin_phase = np.exp(1j * k0 * _dot0(kdir[1:grid.ndim], first_t[:, None])) if grid.ndim > 1 else 1.0
        prop = np.exp(1j * k0 * kdir[0][None, :] * x0[:, None])     # [planes, M]
        out = []
        for side, direction in ((0, 1), (1, -1)):
            vs = vectors[:, side]  # [B, P, M]
            if not np.any(vs != 0):
                out.append(None)
                continue
            if direction < 0:
                vs = vs.conj()
            if self._vectorial:
                rmn = np.einsum('bpm,pm->bm', vs, radial_mode_dir)
                per_mode = rmn[:, None, :] * radial_dir[None]                    # [B, 3, M]
                per_mode[:, 1:] += vs - rmn[:, None, :] * radial_mode_dir[None]
            else:
                per_mode = vs                                                    # [B, 1, M]
            per_mode = per_mode * origin_phase
            out.append((per_mode[:, :, None, :] * prop[None, None]).astype(self._dtype))
        return out

    def _freespace_planes(self, vectors: np.ndarray, planes) -> np.ndarray:
        """
        Free-space fields of the mode vectors ``vectors`` [B, 2, P, M] on the axis-0 planes ``planes``, as
        [B, C, len(planes), *transverse] -- the planes of srcvec2freespace (matrix.py:528-610), on the host.
        """
        shape_t = tuple(int(n) for n in self._grid.shape[1:])
        nt = int(np.prod(shape_t)) if shape_t else 1
        B, nb_pol = vectors.shape[0], 1 + 2 * self._vectorial
        out = np.zeros((B, nb_pol, len(planes), *shape_t), dtype=self._dtype)
        for side, coef in enumerate(self._plane_coefficients(vectors, planes)):
            if coef is None:
                continue
            spec = np.zeros((B, nb_pol, len(planes), nt), dtype=self._dtype)
            spec[..., self._modes[::-1]] = coef
            spec = spec.reshape(B, nb_pol, len(planes), *shape_t)
            field = np.fft.fftn(spec, axes=tuple(range(3, 3 + len(shape_t)))) if shape_t else spec
            out += field.conj() if side == 1 else field
        return out

    # -- the same on the device: spectra scattered / gathered by mmx_mode_scatter / mmx_mode_gather, transverse
    # transforms by mmx_fftn (used by the batched columns of grids with transverse axes) ----------------------------
    def _transverse(self) -> dict:
        if getattr(self, '_transverse_state', None) is None:
            from . import _native as nat
            device = torch.device(self._device if self._device is not None else 'cuda')
            shape_t = tuple(int(n) for n in self._grid.shape[1:])
            prec = nat.MMX_C64 if self._dtype == np.complex64 else nat.MMX_C128
            with torch.cuda.device(device):
                plan = nat.Plan(shape_t, 1, 1, prec)
            idx = torch.from_numpy(np.ascontiguousarray(self._modes[::-1], dtype=np.int64)).to(device)
            self._transverse_state = dict(nat=nat, device=device, plan=plan, idx=idx, prec=prec, shape_t=shape_t,
                                          nt=int(np.prod(shape_t)))
        return self._transverse_state

    def _freespace_planes_device(self, vectors: np.ndarray, planes) -> torch.Tensor:
        """_freespace_planes on the device: [B, C, len(planes), *transverse] (only the mode coefficients cross the
        host link)."""
        ts = self._transverse()
        nat, idx, nt = ts['nat'], ts['idx'], ts['nt']
        B, nb_pol, npl = vectors.shape[0], 1 + 2 * self._vectorial, len(planes)
        rows = B * nb_pol * npl
        tdtype = torch.complex64 if self._dtype == np.complex64 else torch.complex128
        out = torch.zeros((rows, nt), dtype=tdtype, device=ts['device'])
        stream = _stream()
        for side, coef in enumerate(self._plane_coefficients(vectors, planes)):
            if coef is None:
                continue
            c_dev = torch.from_numpy(np.ascontiguousarray(coef)).to(ts['device'])
            spec = torch.zeros((rows, nt), dtype=tdtype, device=ts['device'])
            nat.call('mmx_mode_scatter', nat.device_ptr(c_dev), nat.device_ptr(idx), int(idx.numel()), rows, nt, 0,
                     nat.device_ptr(spec), ts['prec'], stream)
            field = torch.empty_like(spec)
            nat.call('mmx_fftn', ts['plan'].handle, nat.device_ptr(spec), nat.device_ptr(field), rows, 0, stream)
            out += field.conj() if side == 1 else field
        return out.reshape(B, nb_pol, npl, *ts['shape_t'])

    def srcvec2freespace(self, input_vector) -> np.ndarray:
        """Superposition of the vector's free-space plane waves on the whole grid (matrix.py:528-610)."""
        planes = range(int(self._grid.shape[0]))
        f = self._freespace_planes(self._as_modes(input_vector)[None], planes)[0]
        return f.reshape(f.shape[0], *self._grid.shape)

    def _source_scale(self) -> np.ndarray:
        """Per-mode factor from mode amplitude to source_distribution (matrix.py:627-636)."""
        current_density = 1.0 / (const.c * const.mu_0 * float(self._grid.step[0]) / 2)
        amplitude = (-1.0j * self.angular_frequency * const.mu_0) * current_density
        return self._kdir[0] * amplitude  # [M]: cosine of the mode with the transverse plane

    def _sources(self, vectors: np.ndarray) -> np.ndarray:
        """source_distribution [B, C, *grid] of the mode vectors [B, 2, P, M] (srcvec2source, matrix.py:612-648)."""
        B = vectors.shape[0]
        nb_pol = 1 + 2 * self._vectorial
        scaled = vectors * self._source_scale()
        out = np.zeros((B, nb_pol, *self._grid.shape), dtype=self._dtype)
        for side in range(2):
            masked = np.zeros_like(scaled)
            masked[:, side] = scaled[:, side]
            plane = self._source_planes[side]
            out[:, :, plane] = self._freespace_planes(masked, [plane])[:, :, 0]
        return out

    def _source_plane_fields(self, vectors: np.ndarray) -> np.ndarray:
        """The nonzero part of _sources: the fields on the back and front source planes, [B, C, 2, *transverse]."""
        scaled = vectors * self._source_scale()
        out = []
        for side in range(2):
            masked = np.zeros_like(scaled)
            masked[:, side] = scaled[:, side]
            out.append(self._freespace_planes(masked, [self._source_planes[side]])[:, :, 0])
        return np.stack(out, axis=2)

    def _device_sources(self, vectors: np.ndarray) -> torch.Tensor:
        """_sources built on the device: each source plane synthesised there (mmx_mode_scatter + mmx_fftn), so only
        the mode coefficients cross the host link and no dense host array of the batch's size is made."""
        scaled = vectors * self._source_scale()
        if self._grid.ndim > 1:
            planes = []
            for side in range(2):
                masked = np.zeros_like(scaled)
                masked[:, side] = scaled[:, side]
                planes.append(self._freespace_planes_device(masked, [self._source_planes[side]])[:, :, 0])
            planes = torch.stack(planes, dim=2)
        else:
            device = torch.device(self._device if self._device is not None else 'cuda')
            planes = torch.from_numpy(np.ascontiguousarray(self._source_plane_fields(vectors))).to(device)
        B, C = planes.shape[:2]
        src = torch.zeros((B, C, *(int(n) for n in self._grid.shape)), dtype=planes.dtype, device=planes.device)
        for side in range(2):  # in _sources' order: a shared plane keeps the front side's field
            src[:, :, self._source_planes[side]] = planes[:, :, side]
        return src

    def srcvec2source(self, input_vector, out: np.ndarray = None) -> np.ndarray:
        """The source field at the front and back source planes for the vector (matrix.py:612-648)."""
        src = self._sources(self._as_modes(input_vector)[None])[0]
        if out is None:
            return src
        out[...] = src
        return out

    def source2detfield(self, source, out: np.ndarray = None) -> np.ndarray:
        """The field in the whole volume for a source distribution (one solve, matrix.py:650-669)."""
        sol = self._solution
        sol.source_distribution = source
        sol.E = 0
        sol.solve(self._callback if self._callback is not None else _default_callback)
        if out is None:
            return sol.E
        out[...] = sol.E
        return out

    def srcvec2detfield(self, input_vector, out: np.ndarray = None) -> np.ndarray:
        return self.source2detfield(self.srcvec2source(input_vector), out=out)

    def _detect(self, det_fields: np.ndarray) -> np.ndarray:
        """
        Detection vectors [B, side x mode x polarisation] from the outward fields on the detection planes,
        det_fields [B, C, 2 (back plane, front plane), *transverse] (detfield2detvec, matrix.py:685-755), on the host.
        """
        B, nb_pol = det_fields.shape[:2]
        shape_t = tuple(int(n) for n in self._grid.shape[1:])
        f = det_fields.astype(self._dtype, copy=True)
        f[:, :, 1] = f[:, :, 1].conj()  # the backward-propagating side
        if shape_t:
            f = np.fft.ifftn(f, axes=tuple(range(3, 3 + len(shape_t))))
        return self._mode_vectors(f.reshape(B, nb_pol, 2, -1)[..., self._modes[::-1]])

    def _detect_device(self, det_fields: torch.Tensor) -> np.ndarray:
        """_detect for device fields [B, C, 2, *transverse]: the conjugation, the inverse transverse transform and the
        gather at the mode positions on the device (mmx_fftn, mmx_mode_gather); the mode amplitudes go to the host."""
        ts = self._transverse()
        nat, idx, nt = ts['nat'], ts['idx'], ts['nt']
        B, nb_pol = det_fields.shape[:2]
        rows = B * nb_pol * 2
        f = det_fields.reshape(B, nb_pol, 2, nt).clone()
        f[:, :, 1] = f[:, :, 1].conj()  # the backward-propagating side
        f = f.reshape(rows, nt)
        spec = torch.empty_like(f)
        stream = _stream()
        nat.call('mmx_fftn', ts['plan'].handle, nat.device_ptr(f), nat.device_ptr(spec), rows, 1, stream)
        at = torch.empty((rows, int(idx.numel())), dtype=f.dtype, device=f.device)
        nat.call('mmx_mode_gather', nat.device_ptr(spec), nat.device_ptr(idx), int(idx.numel()), rows, nt, 0,
                 nat.device_ptr(at), ts['prec'], stream)
        return self._mode_vectors(at.cpu().numpy().reshape(B, nb_pol, 2, -1))

    def _mode_vectors(self, at_modes: np.ndarray) -> np.ndarray:
        """Detection vectors from the complex amplitudes of the modes on the two detection planes, [B, C, 2, M]: the
        polarisation basis, the phases to the grid origin and to the detection planes, and the aperture weight."""
        grid = self._grid
        k0 = self._k0
        kdir = self._kdir[:, None, :]  # [3, 1, M]
        B = at_modes.shape[0]
        if self._vectorial:
            k3 = kdir[:, 0, :]                                                          # [3, M]
            at_modes = at_modes - np.einsum('bism,im->bsm', at_modes, k3)[:, None] * k3[None, :, None, :]
            axial = np.array([1.0, 0.0, 0.0])[:, None]
            radial_dir = _unit(k3[0][None] * k3 - axial)                                # [3, M]
            radial_mode_dir = _unit(k3[1:])                                             # [2, M]
            rmn = np.einsum('bism,im->bsm', at_modes, radial_dir)                       # [B, 2, M]
            vec = (at_modes[:, 1:] - rmn[:, None] * radial_dir[None, 1:, None, :]
                   + rmn[:, None] * radial_mode_dir[None, :, None, :])                  # [B, 2, 2, M]
        else:
            vec = at_modes                                                              # [B, 1, 2, M]
        first_t = np.asarray(grid.first[1:], dtype=float)
        if grid.ndim > 1:
            vec = vec * np.exp(-1j * k0 * _dot0(kdir[1:grid.ndim], first_t[:, None, None]))
        dist = np.ravel(grid[0])[list(self._detector_planes)]
        vec = vec * np.exp(-1j * k0 * kdir[0] * dist[:, None])
        vec = vec * np.sqrt(kdir[0])
        vec = np.moveaxis(vec, 1, -1)  # [B, 2, M, P]
        vec[:, 1] = vec[:, 1].conj()
        return vec.reshape(B, -1).astype(self._dtype, copy=False)

    def detfield2detvec(self, field) -> np.ndarray:
        """Detection vector of an outward field given on the whole grid (matrix.py:685-755)."""
        field = np.asarray(field)
        det = np.stack([field[:, p] for p in self._detector_planes], axis=1)  # [C, 2, *transverse]
        return self._detect(det[None])[0]

    def detvec2srcvec(self, vec) -> np.ndarray:
        """Time-reversed source vector of a detection vector (matrix.py:757-768)."""
        return np.fft.fftshift(np.asarray(vec).conj())

    # -- columns: batched solves on the device ----------------------------------------------------------------------
    def _batched_outward(self, vectors: np.ndarray) -> np.ndarray:
        """Detection vectors of the mode vectors [B, 2, P, M].  Under ``torchrun`` (a default process group of more
        than one rank) every rank solves its ``shard_range`` slice of the columns on its own GPU and the detection
        vectors are gathered (replicas: no collective inside the solves)."""
        from .distributed import gather_rows, shard_range, world
        rank, size = world()
        if size == 1:
            return self._outward_local(vectors)
        a, b = shard_range(vectors.shape[0], rank, size)
        return gather_rows(self._outward_local(vectors[a:b]), vectors.shape[0])

    def _outward_local(self, vectors: np.ndarray) -> np.ndarray:
        """Detection vectors of the mode vectors [B, 2, P, M], all solved in batched launches on this process's GPU.
        With transverse axes the mode synthesis (sources, incident fields) and the detection run on the device;
        ``self.timing`` keeps the seconds spent in them and in the solves."""
        nb_pol = 1 + 2 * self._vectorial
        B = vectors.shape[0]
        out = np.empty((B, self._side), dtype=self._dtype)
        if B == 0:
            return out
        word = np.dtype(self._dtype).itemsize
        per_rhs = 5.0 * nb_pol * self._grid.size * word  # two field buffers, work buffer, sources, staging
        chunk = int(max(1, min(self._max_batch, self._max_batch_bytes // per_rhs)))
        on_device = self._grid.ndim > 1
        timing = self.__dict__.setdefault('timing', {'modes_s': 0.0, 'solve_s': 0.0})

        def incident_fields(vec):
            """Incident fields on the detection planes: the back detector sees the back input, the front detector
            the front input (matrix.py:795-800)."""
            planes = []
            for plane_idx, side in ((0, 1), (1, 0)):
                masked = np.zeros_like(vec)
                masked[:, side] = vec[:, side]
                plane = [self._detector_planes[plane_idx]]
                planes.append(self._freespace_planes_device(masked, plane)[:, :, 0] if on_device
                              else self._freespace_planes(masked, plane)[:, :, 0])
            return torch.stack(planes, dim=2) if on_device else np.stack(planes, axis=2)

        pre = self._solution._pre
        bound = self._solution.bound
        k0 = self._k0
        rtol, maxiter = _DEFAULT_RTOL, _DEFAULT_MAXITER
        for b0 in range(0, B, chunk):
            sl = slice(b0, min(B, b0 + chunk))
            t0 = _synced_time()
            src = self._device_sources(vectors[sl])
            incident = incident_fields(vectors[sl])
            t1 = _synced_time()
            bs = BatchSolution(self._grid, src, None, bound=bound, wavenumber=k0, dtype=self._dtype,
                               device=self._device, preconditioner=pre)
            del src
            bs.solve(rtol=rtol, maxiter=maxiter)
            E = bs.E_device.reshape(bs.batch, nb_pol, *(int(n) for n in self._grid.shape))
            det = torch.stack([E[:, :, p] for p in self._detector_planes], dim=2) * (1.0 / k0 ** 2)
            bs.close()
            t2 = _synced_time()
            if on_device:
                out[sl] = self._detect_device((det.to(incident.dtype) - incident).contiguous())
            else:
                out[sl] = self._detect(det.cpu().numpy().astype(self._dtype) - incident)
            t3 = _synced_time()
            timing['modes_s'] += (t1 - t0) + (t3 - t2)
            timing['solve_s'] += t2 - t1
        return out

    def _matvec_columns(self, right: np.ndarray) -> np.ndarray:
        result = np.empty((self._side, right.shape[1]), dtype=self._dtype)
        todo = []
        for j in range(right.shape[1]):
            rhs = right[:, j]
            nz = np.flatnonzero(rhs != 0)
            if nz.size == 0:
                result[:, j] = 0.0
            elif self._caching and nz.size == 1 and int(nz[0]) in self._columns:
                result[:, j] = self._columns[int(nz[0])] * rhs[nz[0]]
            else:
                todo.append(j)
        if todo:
            if self._callback is None or self._callback is _default_callback:
                vecs = np.stack([self._as_modes(right[:, j]) for j in todo])
                det = self._batched_outward(vecs)
            else:  # a user callback decides per solve: sequential columns through the Solution mirror
                det = np.stack([self._sequential_column(right[:, j]) for j in todo])
            for k, j in enumerate(todo):
                result[:, j] = det[k]
                nz = np.flatnonzero(right[:, j] != 0)
                if self._caching and nz.size == 1:
                    self._columns[int(nz[0])] = det[k] / right[nz[0], j]
        return result

    def _sequential_column(self, rhs: np.ndarray) -> np.ndarray:
        vec = self._as_modes(rhs)[None]
        incident = np.zeros((1, 1 + 2 * self._vectorial, 2, *self._grid.shape[1:]), dtype=self._dtype)
        for plane_idx, side in ((0, 1), (1, 0)):
            masked = np.zeros_like(vec)
            masked[:, side] = vec[:, side]
            incident[:, :, plane_idx] = self._freespace_planes(masked, [self._detector_planes[plane_idx]])[:, :, 0]
        field = self.srcvec2detfield(rhs)
        det = np.stack([field[:, p] for p in self._detector_planes], axis=1)[None]
        return self._detect(det - incident)[0]

    def _matvec(self, right) -> np.ndarray:
        right = np.asarray(right)
        input_shape = right.shape
        right = right.reshape(-1, right.shape[-1] if right.ndim > 1 else 1)
        if right.shape[0] != self._side:
            raise TypeError(f'Incorrect number of modes specified for this {self.shape} scattering matrix.')
        return self._matvec_columns(right).reshape(input_shape)

    def matvec(self, right) -> np.ndarray:
        return self._matvec(right)

    def __matmul__(self, right) -> np.ndarray:
        return self._matvec(right)

    def __array__(self, dtype=None, copy=None) -> np.ndarray:
        """All columns, solved together (the reference's column loop, matrix.py:831-844)."""
        out = self._matvec_columns(np.eye(self._side, dtype=self._dtype))
        return out if dtype is None else out.astype(dtype)

    def __setitem__(self, key, value):
        raise KeyError('The values of this ScatteringMatrix are calculated from the scattering and cannot be changed '
                       'directly. Use a Matrix object instead.')

    # -- quarters and conversions (matrix.py:271-354, 850-918) -------------------------------------------------------
    def _quarter(self, backwards_output: bool, backwards_input: bool) -> 'QuarterMatrix':
        return QuarterMatrix(self, backwards_output, backwards_input)

    @property
    def forward_transmission(self) -> 'QuarterMatrix':
        return self._quarter(False, False)

    @property
    def front_reflection(self) -> 'QuarterMatrix':
        return self._quarter(True, False)

    @property
    def back_reflection(self) -> 'QuarterMatrix':
        return self._quarter(False, True)

    @property
    def backward_transmission(self) -> 'QuarterMatrix':
        return self._quarter(True, True)

    def transfer(self, noise_level: float = 0.0) -> np.ndarray:
        """The transfer matrix (front-to-back instead of in-to-out, matrix.py:271-314)."""
        return convert(np.asarray(self), noise_level=noise_level)

    def inv(self, noise_level: float = 0.0) -> np.ndarray:
        """The (Tikhonov-regularised) inverse of the matrix (matrix.py:218-227)."""
        return inv(np.asarray(self), noise_level=noise_level)


class QuarterMatrix:
    """One quadrant of a scattering matrix: outputs of one side for inputs from one side (matrix.py:850-882)."""

    def __init__(self, matrix: ScatteringMatrix, backwards_output: bool, backwards_input: bool):
        if matrix.side % 2:
            raise TypeError(f'A QuarterMatrix object can only be constructed using a Matrix with an even number of '
                            f'rows and columns. The specified matrix has dimensions {matrix.shape}.')
        half = matrix.side // 2
        self.full_matrix = matrix
        self._out = slice(half, None) if backwards_output else slice(None, half)
        self._in = slice(half, None) if backwards_input else slice(None, half)
        self.shape = (half, half)

    def __matmul__(self, vec) -> np.ndarray:
        vec = np.asarray(vec)
        cols = vec.reshape(self.shape[1], -1)
        full = np.zeros((self.shape[1] * 2, cols.shape[1]), dtype=np.result_type(vec.dtype, self.full_matrix.dtype))
        full[self._in] = cols
        out = self.full_matrix._matvec_columns(full)[self._out]
        return out.reshape(vec.shape)

    def __array__(self, dtype=None, copy=None) -> np.ndarray:
        out = np.asarray(self.full_matrix)[self._out, self._in]
        return out if dtype is None else out.astype(dtype)


def inv(mat, noise_level: float = 0.0) -> np.ndarray:
    """(Tikhonov-regularised) inverse (matrix.py:996-1006)."""
    mat = np.asarray(mat)
    if noise_level == 0.0:
        return np.linalg.inv(mat)
    u, s, vh = np.linalg.svd(mat)
    s_inv = s / (s ** 2 + noise_level ** 2)
    return (vh.conj().T * s_inv) @ u.conj().T


def convert(s, noise_level: float = 0.0) -> np.ndarray:
    """
    Scattering matrix <-> transfer matrix (matrix.py:1008-1055); the map is its own inverse.  With the blocks
    S = [[A, B], [C, D]] (forward / backward halves of outputs and inputs), T = [[A - B D^-1 C, B D^-1],
    [-D^-1 C, D^-1]].  ``s`` is [N, N] or split as [2, N/2, 2, N/2]; the result has the same shape.
    """
    s = np.asarray(s)
    shape = s.shape
    if s.ndim == 4:
        s = s.reshape(shape[0] * shape[1], shape[2] * shape[3])
    n = s.shape[0] // 2
    A, B, C, D = s[:n, :n], s[:n, n:], s[n:, :n], s[n:, n:]
    D_inv = inv(D, noise_level=noise_level)
    t = np.vstack([np.hstack([A - B @ D_inv @ C, B @ D_inv]), np.hstack([-D_inv @ C, D_inv])])
    return t.reshape(shape)
