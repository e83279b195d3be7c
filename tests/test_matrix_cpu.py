"""
Host side of the scattering matrix (mode synthesis and detection, macromax_b200/matrix.py) against outputs of the
reference ScatteringMatrix (matrix.py:528-755) stored in tests/golden/smatrix_*.npz by make_golden.py; and the
scattering <-> transfer conversion (matrix.py:996-1055).  No device is needed: the solver is created on first use.
"""
import numpy as np
import pytest

from conftest import load_golden

CASES = ['smatrix_1d_scalar', 'smatrix_2d_scalar', 'smatrix_2d_vector', 'smatrix_3d_scalar']


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def make(z, dtype=np.complex128):
    from macromax_b200.bound import LinearBound
    from macromax_b200.grid import Grid
    from macromax_b200.matrix import ScatteringMatrix
    shape = tuple(int(n) for n in z['shape'])
    grid = Grid(shape=shape, step=float(z['step']))
    thickness = np.zeros((grid.ndim, 1))
    thickness[0, 0] = float(z['bound_thickness'])
    bound = LinearBound(grid, thickness=thickness, max_extinction_coefficient=0.25)
    return ScatteringMatrix(grid, vectorial=bool(z['vectorial']), vacuum_wavelength=float(z['wavelength']),
                            refractive_index=z['refractive_index'], bound=bound, dtype=dtype)


@pytest.mark.parametrize('name', CASES)
def test_mode_conversions_match_reference(name):
    z = load_golden(name)
    m = make(z)
    assert m.shape == z['S'].shape
    assert rel(m.srcvec2freespace(z['vec']), z['freespace']) < 1e-12
    assert rel(m.srcvec2source(z['vec']), z['source']) < 1e-12
    assert rel(m.detfield2detvec(z['field']), z['detvec']) < 1e-12


def test_vacuum_detection_inverts_synthesis():
    """In free space, detecting the outward half of each side's plane waves gives back the mode vector (reference
    test_matrix.py test_detfield2detvec): front inputs leave through the back half of the grid, back inputs through
    the front half."""
    for name in ('smatrix_2d_scalar', 'smatrix_2d_vector', 'smatrix_3d_scalar'):
        z = load_golden(name)
        m = make(z)
        n0 = int(z['shape'][0])
        half = m.side // 2
        rng = np.random.default_rng(3)
        v = rng.standard_normal(m.side) + 1j * rng.standard_normal(m.side)
        outward = 0.0
        for side in range(2):
            part = np.zeros_like(v)
            part[side * half:(side + 1) * half] = v[side * half:(side + 1) * half]
            fld = m.srcvec2freespace(part)
            keep = np.zeros(n0)
            if side == 0:
                keep[n0 // 2:] = 1
            else:
                keep[:n0 // 2] = 1
            outward = outward + fld * keep.reshape((1, n0) + (1,) * (fld.ndim - 2))
        assert rel(m.detfield2detvec(outward), v) < 1e-10, name


def test_transfer_conversion_round_trip():
    from macromax_b200.matrix import convert, inv
    z = load_golden('smatrix_2d_vector')
    s = z['S']
    t = convert(s)
    assert rel(convert(t), s) < 1e-10
    split = s.reshape(2, s.shape[0] // 2, 2, s.shape[1] // 2)
    assert np.allclose(convert(split).reshape(s.shape), t)
    assert np.allclose(inv(s) @ s, np.eye(s.shape[0]), atol=1e-10)
    assert np.allclose(inv(s, noise_level=1e-12) @ s, np.eye(s.shape[0]), atol=1e-8)


@pytest.mark.parametrize('name', CASES)
def test_source_planes_rebuild_the_dense_sources(name):
    """The batched columns build their sources on the device from the two source-plane fields alone; scattered
    into zeros, those planes give exactly the dense srcvec2source of every column (the fields are zero elsewhere)."""
    z = load_golden(name)
    m = make(z)
    rng = np.random.default_rng(5)
    v = rng.standard_normal((3, m.side)) + 1j * rng.standard_normal((3, m.side))
    vecs = np.stack([m._as_modes(x) for x in v])
    dense = m._sources(vecs)
    planes = m._source_plane_fields(vecs)
    rebuilt = np.zeros_like(dense)
    for side in range(2):
        rebuilt[:, :, m._source_planes[side]] = planes[:, :, side]
    assert np.array_equal(rebuilt, dense)
