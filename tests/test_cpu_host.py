"""CPU tests of the host side: C ABI exports, state layout, grid/bound/preconditioner conventions, workloads."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADER = os.path.join(ROOT, 'include', 'macromax_b200.h')


def _header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r'^\s*(?:const\s+)?\w+\*?\s+\*?(mmx_\w+)\(', text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from macromax_b200 import _native as nat
    lib = nat.load()
    names = _header_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    assert set(nat.EXPORTED) <= set(names)
    assert lib.mmx_version() == 1
    # every exported entry point has its argument types declared (64-bit counts must not pass as C ints)
    for name in nat.EXPORTED:
        assert getattr(lib, name).argtypes is not None, name


def test_error_reporting_without_gpu():
    """Argument errors are caught before any CUDA call, with a message."""
    from macromax_b200 import _native as nat
    lib = nat.load()
    handle = ctypes.c_void_p()
    shape = (ctypes.c_int64 * 4)(2, 2, 2, 2)
    assert lib.mmx_plan_create(4, shape, 1, 1, 0, ctypes.byref(handle)) == -3
    assert b'1 to 3 axes' in lib.mmx_last_error()
    assert lib.mmx_plan_create(1, shape, 2, 1, 0, ctypes.byref(handle)) == -1
    assert b'ncomp' in lib.mmx_last_error()
    assert lib.mmx_iterate(None, None, None, None, 1, None, None, 1, None) == -1


def test_state_struct_matches_header():
    from macromax_b200 import _native as nat
    text = open(HEADER).read()
    body = text[text.index('typedef struct mmx_rhs_state {'):text.index('} mmx_rhs_state;')]
    fields = re.findall(r'(double|int32_t)\s+([\w\s,\[\]0-9]+);', body)
    names = []
    for _, decl in fields:
        for n in decl.split(','):
            names.append(n.strip().split('[')[0])
    assert names == list(nat.STATE_DTYPE.names)
    assert nat.STATE_DTYPE.itemsize == 112


def test_grid_k_vectors_match_reference_backend():
    from macromax_b200 import Grid
    z = load_golden('backend_ops')
    g = Grid(shape=(5, 10, 20), step=100e-9) * 10e6
    for i, k in enumerate(g.k):
        assert np.allclose(np.broadcast_to(k, z[f'k{i}'].shape), z[f'k{i}'].real, rtol=1e-14, atol=0)


@pytest.mark.parametrize('name', ['disks2d_64_c128', 'spheres3d_20_c128', 'voronoi3d_16_c128', 'design3d_24_c128',
                                  'gain2d_48_c128'])
def test_host_preconditioner_matches_reference_alpha(name):
    from macromax_b200 import preconditioner as pc
    z = load_golden(name)
    ndim = len(z['shape'])
    eps = np.asarray(z['epsilon'])
    while eps.ndim < ndim + 2:
        eps = eps[np.newaxis]
    thickness = np.broadcast_to(float(z['bound_thickness']), (ndim, 2))
    pre = pc.prepare(eps, thickness, 2 * np.pi / float(z['wavelength']), float(np.finfo(np.complex128).eps))
    assert abs(pre.alpha - complex(z['alpha0'])) <= 1e-12 * abs(pre.alpha)
    assert pre.beta == float(z['beta'])


def test_linear_bound_matches_reference_formula():
    from macromax_b200 import Grid, LinearBound
    grid = Grid(shape=(40, 30), step=0.25)
    b = LinearBound(grid, thickness=2.0, max_extinction_coefficient=0.5)
    kappa = np.broadcast_to(b.extinction, grid.shape)
    assert kappa.max() <= 0.5 + 1e-12 and kappa[20, 15] == 0.0
    assert np.isclose(kappa[0, 15], 0.5, rtol=0, atol=1e-12)  # outermost sample: relative depth 1
    chi = b.electric_susceptibility
    assert np.allclose(chi, (1 + 1j * b.extinction) ** 2 - 1)


def test_workloads_are_seeded():
    from macromax_b200 import workloads
    a = workloads.spheres_3d(n=16, nb_spheres=5)
    b = workloads.spheres_3d(n=16, nb_spheres=5)
    assert np.array_equal(a['epsilon'], b['epsilon']) and np.array_equal(a['source'], b['source'])
    c = workloads.correlated_slab_2d(n=64, nb_modes=4)
    re_eps = c['epsilon'].real[:, 32 - 16:32 + 16]
    assert 1.0 <= re_eps.min() and re_eps.max() <= 2.25 + 1e-12
    assert c['source'].shape == (4, 1, 64, 64)


def test_solution_fails_loudly_without_gpu():
    """No CPU fallback: the product path raises instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('needs a machine without a GPU')
    from macromax_b200 import Grid, Solution
    grid = Grid(shape=(16,), step=0.1)
    with pytest.raises(ImportError):
        Solution(grid, vacuum_wavelength=1.0, source_distribution=np.ones((1, 16)), epsilon=np.ones(16))


def test_device_ptr_refuses_strided_tensors():
    import torch
    from macromax_b200 import _native as nat
    t = torch.zeros((4, 6), dtype=torch.complex64)
    assert nat.device_ptr(t).value == t.data_ptr()
    with pytest.raises(ValueError):
        nat.device_ptr(t.t())


def test_symmetric_chi_is_packed_to_six_entries():
    """A 3x3 chi equal to its transpose is stored as xx, xy, xz, yy, yz, zz (MMX_CHI_SYM6); any other 3x3 and a
    scalar are kept as they are.  The rows of the packed form expand back to the full matrix."""
    import torch
    from macromax_b200 import _native as nat
    from macromax_b200.engine import pack_symmetric
    rng = np.random.default_rng(9)
    n = 50
    a = rng.standard_normal((3, 3, n)) + 1j * rng.standard_normal((3, 3, n))
    sym = torch.from_numpy((a + a.transpose(1, 0, 2)).reshape(9, n).astype(np.complex64))
    packed, kind = pack_symmetric(sym)
    assert kind == nat.MMX_CHI_SYM6 and tuple(packed.shape) == (6, n) and packed.is_contiguous()
    full = torch.empty_like(sym)
    for r, (i, j) in zip(range(6), ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        full[3 * i + j] = packed[r]
        full[3 * j + i] = packed[r]
    assert torch.equal(full, sym)
    asym = torch.from_numpy(a.reshape(9, n).astype(np.complex64))
    out, kind = pack_symmetric(asym)
    assert kind == nat.MMX_CHI_MAT3 and out is asym
    almost = sym.clone()
    almost[5, 7] += 1e-6  # symmetric except one voxel of the yz / zy pair: not packed
    assert pack_symmetric(almost)[1] == nat.MMX_CHI_MAT3
    scalar = torch.ones((1, n), dtype=torch.complex64)
    out, kind = pack_symmetric(scalar)
    assert kind == nat.MMX_CHI_SCALAR and out is scalar
    with pytest.raises(ValueError):
        pack_symmetric(torch.ones((4, n), dtype=torch.complex64))


def test_python_constants_match_header_defines():
    """Every MMX_* value of the header's #define lines has the same value in the ctypes mirror."""
    from macromax_b200 import _native as nat
    defines = re.findall(r'^#define\s+(MMX_\w+)\s+\(?(-?\d+)u?\)?', open(HEADER).read(), flags=re.M)
    assert len(defines) >= 15
    for name, value in defines:
        assert getattr(nat, name) == int(value), name
