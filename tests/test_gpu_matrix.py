"""
Scattering matrices with all columns in batched device solves (macromax_b200/matrix.py) against the reference
ScatteringMatrix computed column by column with its NumPy backend (tests/golden/smatrix_*.npz).
"""
import numpy as np
import pytest

from conftest import load_golden
from test_matrix_cpu import CASES, make, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name', CASES)
def test_scattering_matrix_matches_reference(name):
    z = load_golden(name)
    m = make(z)
    S = np.asarray(m)
    assert S.shape == z['S'].shape
    assert rel(S, z['S']) < 1e-8, rel(S, z['S'])
    # quarters are views of the same columns (the cache serves them)
    h = m.side // 2
    assert np.array_equal(np.asarray(m.forward_transmission), S[:h, :h])
    assert np.array_equal(np.asarray(m.front_reflection), S[h:, :h])
    assert np.array_equal(np.asarray(m.back_reflection), S[:h, h:])
    assert np.array_equal(np.asarray(m.backward_transmission), S[h:, h:])
    # a superposition is one more solve (to the same 1e-6 residue), so it agrees with S @ v to that accuracy
    v = np.random.default_rng(1).standard_normal(m.side) + 0j
    assert rel(m @ v, S @ v) < 1e-4


def test_scattering_matrix_complex64():
    z = load_golden('smatrix_2d_vector')
    m = make(z, dtype=np.complex64)
    assert rel(np.asarray(m), z['S']) < 1e-3


def test_batched_columns_equal_sequential_columns():
    """The batched column solves equal the column-by-column path (a user callback forces the latter)."""
    z = load_golden('smatrix_2d_scalar')
    a = make(z)
    b = make(z)
    b._callback = lambda s: s.iteration < 10000 and s.residue > 1e-6
    Sa, Sb = np.asarray(a), np.asarray(b)
    assert rel(Sa, Sb) < 1e-10


def test_lossless_slab_is_nearly_unitary():
    """Reference test_matrix.py test_unitarity: singular values of a lossless scatterer's matrix are close to 1."""
    z = load_golden('smatrix_2d_vector')
    S = np.asarray(make(z))
    sv = np.linalg.svd(S, compute_uv=False)
    assert np.allclose(sv, 1.0, atol=2e-2)


@pytest.mark.parametrize('vectorial, dtype, tol', [(False, np.complex128, 1e-12), (True, np.complex128, 1e-12),
                                                   (True, np.complex64, 2e-6)])
def test_device_mode_synthesis_and_detection_equal_host(vectorial, dtype, tol):
    """The batched columns synthesise their sources and incident fields and detect the outward fields on the device
    (mmx_mode_scatter / mmx_mode_gather around mmx_fftn over the transverse planes); both equal the host
    restatements of srcvec2freespace (matrix.py:528-610) and detfield2detvec (matrix.py:685-755) on random mode
    vectors and fields of a 3D grid (2-D transverse planes)."""
    import torch
    from macromax_b200 import Grid
    from macromax_b200.matrix import ScatteringMatrix
    wavelength = 500e-9
    grid = Grid(shape=(24, 20, 16), step=wavelength / 4)
    sm = ScatteringMatrix(grid, vectorial=vectorial, vacuum_wavelength=wavelength, epsilon=1.0, dtype=dtype)
    rng = np.random.default_rng(3)
    B, P, M = 5, 1 + vectorial, sm._modes.size
    assert M > 10
    vectors = (rng.standard_normal((B, 2, P, M)) + 1j * rng.standard_normal((B, 2, P, M))).astype(dtype)
    vectors[1, 1] = 0  # a side without input
    planes = [3, 11, 20]
    host = sm._freespace_planes(vectors, planes)
    dev = sm._freespace_planes_device(vectors, planes).cpu().numpy()
    assert rel(dev, host) < tol
    C = 1 + 2 * vectorial
    det = (rng.standard_normal((B, C, 2, 20, 16)) + 1j * rng.standard_normal((B, C, 2, 20, 16))).astype(dtype)
    a = sm._detect(det)
    b = sm._detect_device(torch.from_numpy(det).cuda())
    assert rel(b, a) < tol
