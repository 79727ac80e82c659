"""The device field solve against the oracle's sparse LU and the analytic known answers."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.constants import epsilon_0

from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from oracle import poisson as oracle
from tests.test_mesh import CASES, build_mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.poisson import IonOpticsPoisson

    return IonOpticsPoisson


def _plates(shape=(21, 11), h=1e-3, geometry="planar"):
    faces = {"x_min": FaceCondition("dirichlet", 0.0),
             "x_max": FaceCondition("dirichlet", 100.0)}  # fmt: skip
    return IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h, geometry=geometry, faces=faces)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_plates(solver, geometry):
    mesh = _plates(geometry=geometry)
    phi = solver(mesh).solve()
    x = mesh.x[:, None]
    assert np.allclose(phi, 100.0 * x / x[-1], atol=1e-9)


def test_uniform_charge_in_a_grounded_tube(solver):
    h = 0.2e-3
    big_r, rho = 8e-3, 1e-6
    mesh = IonOpticsMesh(shape=(5, round(big_r / h) + 1), origin=(0.0, 0.0), h=h,
                         faces={"y_max": FaceCondition("dirichlet", 0.0)})  # fmt: skip
    phi = solver(mesh).solve(np.full(mesh.shape, rho))
    exact = rho * (big_r**2 - mesh.y**2) / (4 * epsilon_0)
    assert np.allclose(phi[2], exact, rtol=1e-9, atol=1e-9 * exact.max())


def test_coaxial_electrode(solver):
    h = 0.25e-3
    a, big_r, v0 = 1.13e-3, 10e-3, 1000.0
    mesh = IonOpticsMesh(shape=(9, round(big_r / h) + 1), origin=(0.0, 0.0), h=h,
                         electrodes=[Electrode(lambda x, r: r <= a, v0)],
                         faces={"y_max": FaceCondition("dirichlet", 0.0)})  # fmt: skip
    phi = solver(mesh).solve()
    expected = oracle.solve(oracle.operator_of_mesh(mesh))
    np.testing.assert_allclose(phi, expected, rtol=0, atol=1e-9 * v0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_meshes_match_the_oracle(solver, name):
    mesh = build_mesh(name)
    rng = np.random.default_rng(3)
    rho = rng.uniform(0.0, 1e-5, mesh.shape)
    phi = solver(mesh).solve(rho)
    expected = oracle.solve(oracle.operator_of_mesh(mesh), rho)
    span = max(np.ptp(expected), 1.0)
    np.testing.assert_allclose(phi, expected, rtol=0, atol=1e-9 * span)


def test_newton_matches_the_oracle(solver):
    from beamtracer_b200.poisson import BoltzmannElectrons

    mesh = build_mesh("planar_plates")
    plasma = BoltzmannElectrons(1e-6, 5.0, 50.0)
    p = solver(mesh)
    phi = p.solve(plasma=plasma, tolerance=1e-12)
    expected, _ = oracle.solve_newton(oracle.operator_of_mesh(mesh), None,
                                      1e-6 / epsilon_0, 5.0, 50.0, -1, tol=1e-12)  # fmt: skip
    assert p.newton_iterations >= 2
    np.testing.assert_allclose(phi, expected, rtol=0, atol=1e-8)


def test_boltzmann_ions_mirror_the_electrons(solver):
    """Ions about -U_p between mirrored plates give the electrons' potential, negated."""
    from beamtracer_b200.poisson import BoltzmannElectrons, BoltzmannIons

    def plates(voltage):
        faces = {"x_min": FaceCondition("dirichlet", 0.0),
                 "x_max": FaceCondition("dirichlet", voltage)}  # fmt: skip
        return IonOpticsMesh(shape=(41, 21), origin=(0.0, 0.0), h=0.5e-3, geometry="planar",
                             faces=faces)  # fmt: skip

    electrons = solver(plates(100.0)).solve(plasma=BoltzmannElectrons(2e-7, 5.0, 60.0),
                                            tolerance=1e-12)  # fmt: skip
    ions = solver(plates(-100.0)).solve(plasma=BoltzmannIons(2e-7, 5.0, -60.0), tolerance=1e-12)
    np.testing.assert_allclose(ions, -electrons, rtol=0, atol=1e-9)
    expected, _ = oracle.solve_newton(oracle.operator_of_mesh(plates(-100.0)), None,
                                      2e-7 / epsilon_0, 5.0, -60.0, 1, tol=1e-12)  # fmt: skip
    np.testing.assert_allclose(ions, expected, rtol=0, atol=1e-8)


def test_region_is_held(solver):
    mesh = _plates()
    p = solver(mesh)
    x, _ = mesh.nodes()
    region = x < 5.5e-3
    phi = p.solve(fixed_region=region, fixed_potential=7.0)
    op = oracle.operator_of_mesh(mesh, region, 7.0)
    np.testing.assert_allclose(phi, oracle.solve(op), rtol=0, atol=1e-9)
    assert np.all(phi[(x < 5.5e-3) & ~mesh.fixed] == 7.0)
    # and released again
    np.testing.assert_allclose(p.solve(), 100.0 * x / x[-1, 0], rtol=0, atol=1e-9)


def test_large_mesh_converges(solver):
    """The bench's einzel-lens mesh size (801 x 201, cylindrical) with three plates."""
    h = 0.1e-3

    def plate(xc):
        return lambda x, r: (np.abs(x - xc) <= 1e-3) & (r >= 5e-3)

    mesh = IonOpticsMesh(shape=(801, 201), origin=(0.0, 0.0), h=h,
                         electrodes=[Electrode(plate(20e-3), 0.0), Electrode(plate(40e-3), 7e3),
                                     Electrode(plate(60e-3), 0.0)])  # fmt: skip
    rho = np.zeros(mesh.shape)
    rho[:, :30] = 1e-5
    p = solver(mesh)
    phi = p.solve(rho)
    expected = oracle.solve(oracle.operator_of_mesh(mesh), rho)
    print("V-cycles", p.krylov_steps)
    np.testing.assert_allclose(phi, expected, rtol=0, atol=1e-9 * 7e3)
    assert p.krylov_steps < 200


def _three_plates(shape, h):
    def plate(xc):
        return lambda x, r: (np.abs(x - xc) <= 4 * h) & (r >= shape[1] * h / 3)

    n = shape[0] * h
    return IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h,
                         electrodes=[Electrode(plate(n / 4), 0.0), Electrode(plate(n / 2), 5e3),
                                     Electrode(plate(3 * n / 4), 0.0)])  # fmt: skip


@pytest.mark.parametrize("sweeps", [(2, 2), (1, 1), (3, 3), (4, 2)])
def test_staged_smoothing_is_exact(solver, sweeps):
    """Smoothing staged through shared memory (several phases per launch, two x buffers)
    gives the values of one launch per colour, and so the same solve."""
    mesh = _three_plates((331, 97), 0.2e-3)
    rho = np.zeros(mesh.shape)
    rho[:, :20] = 2e-5
    out = []
    for staged in (False, True):
        p = solver(mesh)
        p.set_options(fine_sweeps=sweeps[0], coarse_sweeps=sweeps[1], staged=staged)
        out.append((p.solve(rho), p.krylov_steps))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("tail_nodes", [1, 64, 300, 1 << 20])
def test_tail_split_converges(solver, tail_nodes):
    """Any split between launched levels and the one-block tail gives the oracle's field."""
    mesh = _three_plates((257, 65), 0.2e-3)
    rho = np.zeros(mesh.shape)
    rho[:, :10] = 1e-5
    p = solver(mesh)
    p.set_options(tail_nodes=tail_nodes)
    phi = p.solve(rho)
    expected = oracle.solve(oracle.operator_of_mesh(mesh), rho)
    np.testing.assert_allclose(phi, expected, rtol=0, atol=1e-9 * 5e3)


def test_options_are_checked(solver):
    p = solver(_plates())
    with pytest.raises(ValueError):
        p.set_options(fine_sweeps=0)
    with pytest.raises(ValueError):
        p.set_options(coarse_sweeps=5)
    with pytest.raises(ValueError):
        p.set_options(tail_nodes=0)
