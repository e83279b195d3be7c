"""
CUDA-graph replay of iteration chunks, the uneven batch packed into one graph launch, and the device set-up
reductions for anisotropic media.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _batch(n, B, seed, dtype=np.complex64):
    from macromax_b200 import Bound, Grid, workloads
    from macromax_b200.batch import BatchSolution
    wl = workloads.correlated_slab_2d(n=n, nb_modes=B, seed=seed)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    return BatchSolution(grid, wl['source'], wl['epsilon'], bound=Bound(grid, thickness=wl['bound_thickness']),
                         vacuum_wavelength=wl['wavelength'], dtype=dtype)


def test_graph_replay_is_bitwise_identical_to_launches():
    from macromax_b200 import workloads, Bound, Grid, Solution
    wl = workloads.spheres_3d(n=64, nb_spheres=20)
    grid = Grid(shape=wl['shape'], step=wl['step'])
    sols = []
    for graphs in (True, False):
        sol = Solution(grid, vacuum_wavelength=wl['wavelength'], epsilon=wl['epsilon'],
                       source_distribution=wl['source'], bound=Bound(grid, thickness=wl['bound_thickness']),
                       dtype=np.complex64)
        sol._engine.use_graphs = graphs
        sol.solve(None, rtol=0, maxiter=40)
        assert sol.iteration == 40
        sols.append(sol.E)
    assert np.array_equal(sols[0], sols[1])


def test_uneven_batch_one_graph_matches_separate_solves():
    from macromax_b200.batch import UnevenBatch
    members = [_batch(128, 6, 11), _batch(256, 3, 12), _batch(384, 2, 13)]
    UnevenBatch(members).solve(rtol=1e-5, maxiter=3000)
    for m, (n, B, seed) in zip(members, [(128, 6, 11), (256, 3, 12), (384, 2, 13)]):
        ref = _batch(n, B, seed)
        ref.solve(rtol=1e-5, maxiter=3000)
        assert np.array_equal(m.iterations, ref.iterations)
        assert np.array_equal(m.E, ref.E)
        assert m.residues.max() <= 1e-5


def test_device_setup_reductions_match_host():
    from macromax_b200 import preconditioner as pc
    z = load_golden('voronoi3d_16_c128')
    eps = np.asarray(z['epsilon'])
    dev = pc.DeviceSetup(eps)
    # closed-form cubic roots lose accuracy (~sqrt(eps)) at the (nearly) double eigenvalues of uniaxial media
    for ar in (0.0, 0.5, 1.3, 2.484375, 3.7):
        host = pc.largest_sigma(ar, 1.0, eps)
        assert abs(dev.sigma(ar, 1.0) - host) <= 1e-7 * host
    e = float(np.finfo(np.complex128).eps)
    assert dev.gain_loss(e) == (pc.has_gain(eps, e), pc.has_gain(-eps, e))
    thickness = np.broadcast_to(float(z['bound_thickness']), (3, 2))
    pre = pc.prepare(eps, thickness, 2 * np.pi / float(z['wavelength']), e, device_setup=True)
    assert abs(pre.alpha - complex(z['alpha0'])) <= 1e-12 * abs(pre.alpha)


def test_device_chi_matches_host_expression():
    """A 3x3 permittivity's chi is built on the device from the permittivity the set-up already uploaded; it equals
    the host expression eps i / (alpha_i beta) - i alpha / alpha_i I (solver.py:480-484) to rounding, and the solve
    that uses it equals the reference's iterates."""
    from macromax_b200 import preconditioner as pc
    z = load_golden('voronoi3d_16_c128')
    eps = np.asarray(z['epsilon'])
    e = float(np.finfo(np.complex128).eps)
    thickness = np.broadcast_to(float(z['bound_thickness']), (3, 2))
    pre = pc.prepare(eps, thickness, 2 * np.pi / float(z['wavelength']), e, device_setup=True)
    assert pre.chi_device is not None and pre.chi_rows == 3
    host = eps * (1.0j / pre.alpha.imag / pre.beta) - np.eye(3).reshape(3, 3, 1, 1, 1) * (pre.alpha * 1.0j /
                                                                                         pre.alpha.imag)
    dev = pre.chi_device.cpu().numpy().reshape(host.shape)
    assert rel(dev, host) < 1e-15
    assert np.array_equal(pre.chi, dev)


def test_device_gain_loss_flags_on_lossy_and_gain_media():
    from macromax_b200 import preconditioner as pc
    e = float(np.finfo(np.complex128).eps)
    base = np.zeros((3, 3, 4, 4), dtype=np.complex128)
    for i in range(3):
        base[i, i] = 2.0
    lossy = base.copy()
    lossy[0, 0, 1, 1] += 0.1j
    gain = base.copy()
    gain[1, 1, 2, 2] -= 0.1j
    both = lossy.copy()
    both[2, 2, 3, 3] -= 0.05j
    for m in (base, lossy, gain, both):
        assert pc.DeviceSetup(m).gain_loss(e) == (pc.has_gain(m, e), pc.has_gain(-m, e))


@pytest.mark.parametrize('name', ['disks2d_256', 'spheres3d_64', 'gain2d'])
def test_scalar_device_objective_is_bitwise_host(name):
    """The scalar alpha objective on the device equals the host expression bit for bit, so the Nelder-Mead path and
    alpha are unchanged (solver.py:392-401, 425-461)."""
    from macromax_b200 import preconditioner as pc
    from macromax_b200 import workloads
    if name == 'disks2d_256':
        eps = workloads.disks_2d(n=256)['epsilon']
    elif name == 'spheres3d_64':
        eps = workloads.spheres_3d(n=64, nb_spheres=40)['epsilon']
    else:
        eps = workloads.disks_2d(n=256, seed=7)['epsilon'].copy()
        eps[100:140, 100:140] = 2.0 - 0.4j  # gain: the alpha search is conjugated afterwards
    eps = np.asarray(eps, dtype=np.complex128)[None, None]
    obj = pc.ScalarDeviceObjective(eps)
    for ar in (0.0, 1.0, 0.37, 1.9999, -3.25, 12.5):
        for beta in (1.0, 0.5):
            assert obj(ar, beta) == pc.largest_sigma(ar, beta, eps)
    thickness = np.full((eps.ndim - 2, 2), 2e-6)
    host = pc.prepare(eps, thickness, 2 * np.pi / 500e-9, float(np.finfo(np.float32).eps), device_setup=False)
    devp = pc.prepare(eps, thickness, 2 * np.pi / 500e-9, float(np.finfo(np.float32).eps), device_setup=True)
    assert devp.alpha == host.alpha and devp.transpose == host.transpose
