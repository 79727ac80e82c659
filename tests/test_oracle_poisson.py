"""The oracle's field solve against the reference's analytic known answers.

The cases and tolerances of the reference's ``tests/unit/test_ion_optics.py:60-125`` and
the manufactured cylindrical solution of ``solver/poisson.py:491-513`` (second order).
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy.constants import epsilon_0

from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from oracle import poisson


def _plates(shape=(21, 11), h=1e-3, geometry="planar", **faces):
    faces = {"x_min": FaceCondition("dirichlet", 0.0),
             "x_max": FaceCondition("dirichlet", 100.0), **faces}  # fmt: skip
    return IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h, geometry=geometry, faces=faces)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_potential_between_plates_is_linear(geometry):
    mesh = _plates(geometry=geometry)
    phi = poisson.solve(poisson.operator_of_mesh(mesh))
    x = mesh.x[:, None]
    assert np.allclose(phi, 100.0 * x / x[-1], atol=1e-9)


def test_coaxial_electrode_off_the_nodes():
    h = 0.25e-3
    a, big_r, v0 = 1.13e-3, 10e-3, 1000.0
    mesh = IonOpticsMesh(
        shape=(9, round(big_r / h) + 1), origin=(0.0, 0.0), h=h,
        electrodes=[Electrode(lambda x, r: r <= a, v0)],
        faces={"y_max": FaceCondition("dirichlet", 0.0)},
    )  # fmt: skip
    phi = poisson.solve(poisson.operator_of_mesh(mesh))
    r = mesh.y
    free = r > a
    exact = v0 * np.log(big_r / r[free]) / np.log(big_r / a)
    assert np.max(np.abs(phi[4, free] - exact)) < 2e-3 * v0


def test_uniform_charge_in_a_grounded_tube():
    h = 0.2e-3
    big_r, rho = 8e-3, 1e-6
    mesh = IonOpticsMesh(
        shape=(5, round(big_r / h) + 1), origin=(0.0, 0.0), h=h,
        faces={"y_max": FaceCondition("dirichlet", 0.0)},
    )  # fmt: skip
    phi = poisson.solve(poisson.operator_of_mesh(mesh), np.full(mesh.shape, rho))
    exact = rho * (big_r**2 - mesh.y**2) / (4 * epsilon_0)
    assert np.allclose(phi[2], exact, rtol=1e-9, atol=1e-9 * exact.max())


def test_boltzmann_electrons_satisfy_the_nonlinear_equation():
    mesh = _plates()
    op = poisson.operator_of_mesh(mesh)
    phi, steps = poisson.solve_newton(op, None, 1e-6 / epsilon_0, 5.0, 50.0, -1)
    assert 1 < steps < 30
    lap = (phi[2:, 1:-1] + phi[:-2, 1:-1] + phi[1:-1, 2:] + phi[1:-1, :-2]
           - 4 * phi[1:-1, 1:-1]) / mesh.h**2  # fmt: skip
    source = 1e-6 * np.exp((phi[1:-1, 1:-1] - 50.0) / 5.0) / epsilon_0
    assert np.allclose(lap, source, rtol=1e-6, atol=1e-6 * source.max())


def test_manufactured_cylindrical_solution_is_second_order():
    errors = []
    for n in (8, 16, 32, 64):
        h = 1.0 / n
        zero = FaceCondition("dirichlet", 0.0)
        mesh = IonOpticsMesh(shape=(2 * n + 1, n + 1), origin=(-1.0, 0.0), h=h,
                             faces={"x_min": zero, "x_max": zero, "y_max": zero})  # fmt: skip
        x, r = mesh.nodes()
        cx, cr = np.cos(0.5 * np.pi * x), np.cos(0.5 * np.pi * r)
        sinc = 0.5 * np.pi * np.sinc(0.5 * r)
        laplacian = -0.5 * np.pi**2 * cx * cr - 0.5 * np.pi * cx * sinc
        phi = poisson.solve(poisson.operator_of_mesh(mesh), -epsilon_0 * laplacian)
        errors.append(np.max(np.abs(phi - cx * cr)))
    orders = np.log2(np.array(errors[:-1]) / np.array(errors[1:]))
    assert np.all(orders > 1.8), orders


def test_neumann_faces_mirror():
    """A uniform charge between grounded x faces, Neumann y faces: a 1D parabola."""
    mesh = IonOpticsMesh(shape=(21, 7), origin=(0.0, 0.0), h=1e-3, geometry="planar",
                         faces={"x_min": FaceCondition("dirichlet", 0.0),
                                "x_max": FaceCondition("dirichlet", 0.0)})  # fmt: skip
    rho = 1e-6
    phi = poisson.solve(poisson.operator_of_mesh(mesh), np.full(mesh.shape, rho))
    x = mesh.x
    exact = rho * x * (x[-1] - x) / (2 * epsilon_0)
    assert np.allclose(phi, exact[:, None], rtol=1e-9, atol=1e-12)
