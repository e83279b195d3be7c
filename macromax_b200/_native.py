"""
ctypes binding of the native library ``libmacromax_b200.so`` (C ABI in ``include/macromax_b200.h``).

The library is built in-tree (``python -m macromax_b200.build``).  Loading fails loudly with ``ImportError`` when
it is missing, which is also how ``backend.load`` of the reference learns that a backend is unavailable
(backend/__init__.py:1010-1011): there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB_PATH

MMX_C64 = 0
MMX_C128 = 1
MMX_CHI_SCALAR = 1
MMX_CHI_MAT3 = 9
MMX_CHI_SYM6 = 6
SYM6_ROWS = (0, 1, 2, 4, 5, 8)  # xx, xy, xz, yy, yz, zz of a row-major 3x3
MMX_OK = 0
MMX_ERR_ARG = -1
MMX_ERR_CUDA = -2
MMX_ERR_UNSUPPORTED = -3
MMX_STATUS_OK = 0
MMX_STATUS_ZERODIV = 1
MMX_STATUS_TIMEOUT = 2
MMX_VARIANT_GENERIC = 1
MMX_VARIANT_SHARED_STAGED = 2
MMX_VARIANT_PERSISTENT = 4
MMX_VARIANT_PLANE = 8
MMX_VARIANT_FUSED_EPILOGUE = 16
MMX_VARIANT_TMA = 32

# numpy mirror of struct mmx_rhs_state (include/macromax_b200.h)
STATE_DTYPE = np.dtype([
    ('alpha_re', '<f8'), ('alpha_im', '<f8'), ('alpha0_re', '<f8'), ('alpha0_im', '<f8'),
    ('prev_norm', '<f8'), ('last_norm', '<f8'), ('field_norm', '<f8'), ('residue', '<f8'),
    ('rtol', '<f8'), ('maxiter', '<f8'),
    ('iteration', '<i4'), ('cur', '<i4'), ('active', '<i4'), ('accepted', '<i4'), ('rejections', '<i4'),
    ('status', '<i4'), ('reserved', '<i4', (2,)),
])
assert STATE_DTYPE.itemsize == 112

EXPORTED = ['mmx_last_error', 'mmx_version', 'mmx_plan_create', 'mmx_plan_destroy', 'mmx_plan_set_kvectors',
            'mmx_fftn', 'mmx_norm', 'mmx_iterate', 'mmx_defect', 'mmx_accumulate', 'mmx_adjoint_grad',
            'mmx_pointwise_mul', 'mmx_fftn_noalloc', 'mmx_mat3_extremes', 'mmx_iterate_graph',
            'mmx_iterate_multi', 'mmx_iterate_graph_prepare', 'mmx_iterate_graph_continue', 'mmx_plan_set_variant',
            'mmx_plan_get_variant', 'mmx_scalar_sigma', 'mmx_curl_ft', 'mmx_green_ft', 'mmx_chi_mix', 'mmx_axpby', 'mmx_chi_from_eps',
            'mmx_magnetic_iterate', 'mmx_mode_scatter', 'mmx_mode_gather']

_lib = None


class NativeError(RuntimeError):
    pass


def device_ptr(t) -> ctypes.c_void_p:
    """Device address of a tensor for the C ABI, whose buffers are dense and row-major: a strided view would be read
    in the wrong order, so it is refused."""
    if not t.is_contiguous():
        raise ValueError(f'the C ABI needs contiguous tensors (shape {tuple(t.shape)}, strides {t.stride()})')
    return ctypes.c_void_p(t.data_ptr())


class MagneticBuffers(ctypes.Structure):
    """mmx_magnetic_buffers: the field, source and susceptibility blocks and seven scratch fields (device)."""
    _fields_ = [('E', ctypes.c_void_p), ('src', ctypes.c_void_p), ('chi_ee', ctypes.c_void_p),
                ('chi_eh', ctypes.c_void_p), ('chi_he', ctypes.c_void_p), ('chi_hh', ctypes.c_void_p),
                ('work', ctypes.c_void_p * 7)]


def load(path: str | None = None):
    """Load (once) and return the ctypes library handle; ImportError if the library cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f'native library {path} not built (run: python -m macromax_b200.build)')
    try:
        lib = ctypes.CDLL(path)
    except OSError as e:
        raise ImportError(f'cannot load {path}: {e}') from e
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    sig = {
        'mmx_last_error': (ctypes.c_char_p, []),
        'mmx_version': (i32, []),
        'mmx_plan_create': (i32, [i32, ctypes.POINTER(i64), i32, i32, i32, ctypes.POINTER(vp)]),
        'mmx_plan_destroy': (i32, [vp]),
        'mmx_plan_set_kvectors': (i32, [vp, ctypes.POINTER(dbl)]),
        'mmx_fftn': (i32, [vp, vp, vp, i64, i32, vp]),
        'mmx_norm': (i32, [vp, vp, i64, i32, vp, vp]),
        'mmx_iterate': (i32, [vp, vp, vp, vp, i32, vp, vp, i32, vp]),
        'mmx_defect': (i32, [vp, vp, vp, i32, vp, vp, vp, vp]),
        'mmx_accumulate': (i32, [vp, vp, i64, vp]),
        'mmx_adjoint_grad': (i32, [vp, vp, vp, i64, i32, i64, i32, dbl, vp]),
        'mmx_pointwise_mul': (i32, [vp, i32, i32, vp, i32, i32, vp, i64, i32, vp]),
        'mmx_fftn_noalloc': (i32, [i32, ctypes.POINTER(i64), vp, vp, i64, i32, i32, vp]),
        'mmx_scalar_sigma': (i32, [vp, vp, i64, dbl, vp, vp]),
        'mmx_chi_from_eps': (i32, [vp, i32, i64, dbl, dbl, dbl, dbl, vp, i32, vp]),
        'mmx_magnetic_iterate': (i32, [vp, ctypes.POINTER(MagneticBuffers), vp, i32, i32, vp]),
        'mmx_curl_ft': (i32, [vp, vp, vp, vp]),
        'mmx_green_ft': (i32, [vp, vp, dbl, dbl, vp]),
        'mmx_chi_mix': (i32, [vp, vp, vp, vp, vp, vp, ctypes.POINTER(dbl), vp, vp, i64, i32, vp]),
        'mmx_axpby': (i32, [vp, vp, vp, dbl, dbl, dbl, dbl, i64, i32, vp]),
        'mmx_mat3_extremes': (i32, [vp, vp, i64, i32, dbl, vp, vp]),
        'mmx_iterate_graph': (i32, [vp, vp, vp, vp, i32, vp, vp, i32, vp]),
        'mmx_iterate_graph_prepare': (i32, [vp, vp, vp, vp, i32, vp, vp, i32]),
        'mmx_iterate_graph_continue': (i32, [vp, vp, vp, vp, i32, vp, vp, i32, vp]),
        'mmx_mode_scatter': (i32, [vp, vp, i64, i64, i64, i32, vp, i32, vp]),
        'mmx_mode_gather': (i32, [vp, vp, i64, i64, i64, i32, vp, i32, vp]),
        'mmx_plan_set_variant': (i32, [vp, ctypes.c_uint]),
        'mmx_plan_get_variant': (ctypes.c_uint, [vp]),
        'mmx_iterate_multi': (i32, [i32, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                    ctypes.POINTER(vp), ctypes.POINTER(i32), ctypes.POINTER(vp),
                                    ctypes.POINTER(vp), i32, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != MMX_OK:
        msg = _lib.mmx_last_error().decode(errors='replace') if _lib is not None else 'unknown'
        raise NativeError(f'macromax_b200 native call failed ({rc}): {msg}')


def call(name: str, *args):
    lib = load()
    check(getattr(lib, name)(*args))


class Plan:
    """Owning wrapper of an ``mmx_plan``."""

    def __init__(self, shape, ncomp: int, batch: int, precision: int):
        lib = load()
        shape = [int(s) for s in shape]
        arr = (ctypes.c_int64 * len(shape))(*shape)
        handle = ctypes.c_void_p()
        check(lib.mmx_plan_create(len(shape), arr, int(ncomp), int(batch), int(precision), ctypes.byref(handle)))
        self.handle = handle
        self.shape = tuple(shape)
        self.ncomp = int(ncomp)
        self.batch = int(batch)
        self.precision = int(precision)

    def set_kvectors(self, ks):
        k = np.ascontiguousarray(np.concatenate([np.asarray(kk, dtype=np.float64).ravel() for kk in ks]))
        check(load().mmx_plan_set_kvectors(self.handle, k.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def close(self):
        if getattr(self, 'handle', None) is not None and self.handle.value is not None and _lib is not None:
            _lib.mmx_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
