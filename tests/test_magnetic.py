"""The trace in a magnetic field: the reference's NumPy tracer's step (``tracer.py:851-1054``)
with an axisymmetric field from its on-axis profile (``fields.py:192-279``).

The oracle's magnetic step is pinned by the reference's own known answers for it, ported
as cases: Boris's rotation keeps the speed to 1e-12 in a pure magnetic field and follows
RK4 to 2e-5 m (``test_compiled_tracer.py:371-396``), and Busch's theorem holds through a
solenoid to 1e-3 of its scale (``test_ion_optics.py:221-256``).  On the GPU the kernel
must equal the oracle bit for bit on every per-trajectory output (the same expressions in
the same order, FP64 without fused multiply-adds), its charges to rounding.
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy import constants

from beamtracer_b200.fields import AxisymmetricMagneticField, PlanarSolenoidField, solenoid_on_axis
from beamtracer_b200.mesh import IonOpticsMesh
from beamtracer_b200.tracer import BeamParticles
from oracle import kernels as oracle
from oracle import vlasov as oracle_vlasov
from tests.golden.cases import TRACE_CHARGE, TRACE_OUTPUTS, copy_args, trace_case
from tests.vlasov_cases import mesh_problem


def _beam(position, velocity, charge=1.602e-19, mass=1.67e-27, current=1e-3):
    n = position.shape[1]
    return BeamParticles(position, velocity, np.full(n, charge), np.full(n, mass),
                         np.full(n, current), np.zeros(n, dtype=np.int32))  # fmt: skip


def _oracle_hits(mesh, magnet, particles, *, integrator, plane, step_fraction):
    p = mesh_problem(mesh, planes=(plane,), integrator=integrator, step_fraction=step_fraction,
                     magnetic=magnet)  # fmt: skip
    nx, ny = mesh.shape
    fx, fy = np.zeros((nx + 1, ny)), np.zeros((nx, ny + 1))
    t = oracle_vlasov.trace(p, fx, fy, particles)
    return oracle_vlasov.plane_hits(p, t, particles.current, particles.species)[0]


def _solenoid_lens():
    mesh = IonOpticsMesh(shape=(201, 21), origin=(0.0, 0.0), h=1e-3)
    bz = 0.3 * np.exp(-((((np.arange(201) * 1e-3) - 0.1) / 0.03) ** 2))
    n = 20
    position = np.stack([np.zeros(n), np.linspace(1e-3, 8e-3, n), np.zeros(n)])
    velocity = np.stack([np.full(n, 1e6), np.zeros(n), np.zeros(n)])
    return mesh, AxisymmetricMagneticField(0.0, 1e-3, bz), _beam(position, velocity)


def test_oracle_boris_keeps_the_speed_and_follows_rk4():
    mesh, magnet, particles = _solenoid_lens()
    ends = {}
    for integrator in (0, 1):
        ends[integrator] = _oracle_hits(mesh, magnet, particles, integrator=integrator,
                                        plane=0.19, step_fraction=0.25)  # fmt: skip
    point_rk4, point_boris, velocity_boris = ends[0][0], ends[1][0], ends[1][1]
    assert point_boris.shape[1] == 20
    np.testing.assert_allclose(np.linalg.norm(velocity_boris, axis=0), 1e6, rtol=1e-12)
    np.testing.assert_allclose(point_boris[1], point_rk4[1], rtol=0, atol=2e-5)
    assert np.abs(point_boris[1] - particles.position[1]).max() > 1e-4  # it focuses


def _busch_setup():
    h = 1e-3
    mesh = IonOpticsMesh(shape=(601, 41), origin=(0.0, 0.0), h=h)
    z = np.arange(-0.1, 0.7, 0.5e-3)
    magnet = AxisymmetricMagneticField(z[0], 0.5e-3, solenoid_on_axis(z, 0.3, 0.2, 0.05, 0.1))
    m = constants.m_p
    v = np.sqrt(2 * 1e4 * constants.e / m)
    particles = _beam(np.array([[0.0], [5e-3], [0.0]]), np.array([[v], [0.0], [0.0]]),
                      charge=constants.e, mass=m, current=1e-9)  # fmt: skip
    return mesh, magnet, particles


def _busch_check(magnet, point, velocity):
    m = constants.m_p
    r = np.hypot(point[1], point[2])
    omega = (point[1] * velocity[2] - point[2] * velocity[1]) / r**2
    b_here = magnet(np.array([0.29]), np.array([r]))[0][0]
    canonical = r**2 * (omega + constants.e * b_here / (2 * m))
    b_start = magnet(np.array([0.0]), np.array([5e-3]))[0][0]
    canonical_start = 25e-6 * constants.e * b_start / (2 * m)
    scale = constants.e * b_here / (2 * m) * r**2
    assert canonical == pytest.approx(canonical_start, abs=1e-3 * scale)


def test_oracle_follows_busch_theorem():
    mesh, magnet, particles = _busch_setup()
    point, velocity = _oracle_hits(mesh, magnet, particles, integrator=0, plane=0.29,
                                   step_fraction=0.25)[:2]  # fmt: skip
    assert point.shape[1] == 1
    _busch_check(magnet, point[:, 0], velocity[:, 0])


def test_planar_solenoid_field_mirrors_the_radial_component():
    _, magnet, _ = _solenoid_lens()
    planar = PlanarSolenoidField(magnet, axis_y=2e-3)
    x = np.full(3, 0.09)
    bx, by, bz = planar(x, np.array([1e-3, 2e-3, 3e-3]))
    axial, radial = magnet(x, np.array([1e-3, 0.0, 1e-3]))
    np.testing.assert_array_equal(bx, axial)
    np.testing.assert_array_equal(by, [-radial[0], radial[1], radial[2]])
    np.testing.assert_array_equal(bz, 0.0)


# -- the device kernel ------------------------------------------------------------------------


def _case_field(cylindrical):
    z = np.arange(-5e-3, 40e-3, 0.5e-3)
    magnet = AxisymmetricMagneticField(z[0], 0.5e-3, 0.3 * np.exp(-(((z - 0.015) / 0.008) ** 2)),
                                       order=5)  # fmt: skip
    return magnet if cylindrical == 1 else PlanarSolenoidField(magnet, axis_y=5e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("graded", [False, True])
@pytest.mark.parametrize("integrator", [0, 1])
@pytest.mark.parametrize("cylindrical", [0, 1])
def test_device_magnetic_trace_matches_the_oracle(cylindrical, integrator, graded):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.kernels import trace_trajectories_2d
    from tests.gpu_util import to_device, to_host

    args = trace_case(cylindrical, integrator, graded=graded, seed=31, max_steps=400)
    field = _case_field(cylindrical)
    profile = field.profile()
    expected = copy_args(args)
    oracle.trace_trajectories_2d(*expected, magnetic=profile.oracle_tuple())
    device = to_device(args)
    device[TRACE_CHARGE] = device[TRACE_CHARGE][:1].clone()
    trace_trajectories_2d(*device, window=16, magnetic=profile)
    result = to_host(device)
    status = expected[TRACE_OUTPUTS["status"]]
    assert (status == -2).any() and (status >= 0).any()  # pauses at electrodes, and ends
    for key, i in TRACE_OUTPUTS.items():
        np.testing.assert_array_equal(result[i], expected[i], err_msg=key)
    total = expected[TRACE_CHARGE].sum(0)
    np.testing.assert_allclose(result[TRACE_CHARGE][0], total, rtol=0,
                               atol=1e-12 * np.abs(total).max())  # fmt: skip


@pytest.mark.gpu
def test_device_boris_keeps_the_speed_and_follows_rk4():
    from beamtracer_b200.fields import StaggeredElectricField
    from beamtracer_b200.tracer import BeamTracer

    mesh, magnet, particles = _solenoid_lens()
    zero = StaggeredElectricField(mesh, np.zeros(mesh.shape))
    ends = {}
    for integrator in ("rk4", "boris"):
        tracer = BeamTracer(mesh, zero, magnet, integrator=integrator, planes=[0.19],
                            step_fraction=0.25)  # fmt: skip
        ends[integrator] = tracer.trace(particles).planes[0]
    np.testing.assert_allclose(np.linalg.norm(ends["boris"].velocity, axis=0), 1e6, rtol=1e-12)
    np.testing.assert_allclose(ends["boris"].point[1], ends["rk4"].point[1], rtol=0, atol=2e-5)
    assert np.abs(ends["boris"].point[1] - particles.position[1]).max() > 1e-4
    oracle_points = _oracle_hits(mesh, magnet, particles, integrator=1, plane=0.19,
                                 step_fraction=0.25)[0]  # fmt: skip
    np.testing.assert_array_equal(ends["boris"].point, oracle_points)


@pytest.mark.gpu
def test_device_follows_busch_theorem():
    from beamtracer_b200.fields import StaggeredElectricField
    from beamtracer_b200.tracer import BeamTracer

    mesh, magnet, particles = _busch_setup()
    zero = StaggeredElectricField(mesh, np.zeros(mesh.shape))
    tracer = BeamTracer(mesh, zero, magnet, planes=[0.29], step_fraction=0.25)
    hits = tracer.trace(particles).planes[0]
    _busch_check(magnet, hits.point[:, 0], hits.velocity[:, 0])
