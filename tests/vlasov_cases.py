"""Configurations of the end-to-end cases and the oracle problem of a model."""

from __future__ import annotations

import numpy as np
from scipy import constants

from beamtracer_b200.config import (
    BeamOpticsConfig,
    BeamSpecies,
    ExtractionPlasma,
    FieldBCs,
    FieldBoundaryCondition,
    GridParams,
    ObjectParams,
)
from oracle import vlasov as oracle_vlasov


def diode(*, current_density: float, num_gridpoints=(41, 21), **settings) -> BeamOpticsConfig:
    """A planar diode: ions from x = 0 (0 V) to x = 10 mm (-1 kV); Neumann y walls.  The
    case of the reference's ``tests/unit/test_beam_optics.py:27-58``."""
    neumann = FieldBoundaryCondition.neumann(0.0)
    return BeamOpticsConfig(
        grid=GridParams(ndim=2, num_gridpoints=num_gridpoints, lower_bound=(0.0, 0.0),
                        upper_bound=(10e-3, 5e-3), coordinates="cartesian"),
        bcs_field=FieldBCs(FieldBoundaryCondition.dirichlet(0.0),
                           FieldBoundaryCondition.dirichlet(-1000.0), neumann, neumann),
        beams=[BeamSpecies("H+", current_density, (0.0, 0.0), (0.0, 5e-3), energy=0.01,
                           transverse_temperature=0.0, num_particles=40)],
        diagnostic_planes=[9.9e-3],
        **settings,
    )  # fmt: skip


def child_langmuir_density(d=10e-3, voltage=1000.0) -> float:
    mass = 1.007276 * constants.atomic_mass
    return 4 * constants.epsilon_0 / 9 * np.sqrt(2 * constants.e / mass) * voltage**1.5 / d**2


def plate(x0, x1, r0, r1, voltage) -> ObjectParams:
    """A plate around the axis from radius r0 outwards between x0 and x1."""
    return ObjectParams(type="aperture2d", axis=0, position=0.0,
                        vertices=((x0, r0), (x0, r1), (x1, r1), (x1, r0)),
                        bc_type="dirichlet", bc_value=voltage)  # fmt: skip


def extraction(sign: float = 1.0, **settings) -> BeamOpticsConfig:
    """Ions extracted through a round aperture from a plasma (the reference's
    ``tests/unit/test_beam_optics.py:211-261``), cylindrical 81 x 31."""
    plasma_potential, voltage = 5.0 * sign, -2000.0 * sign
    neumann = FieldBoundaryCondition.neumann(0.0)
    return BeamOpticsConfig(
        grid=GridParams(ndim=2, num_gridpoints=(81, 31), lower_bound=(0.0, 0.0),
                        upper_bound=(8e-3, 3e-3), coordinates="cylindrical"),
        bcs_field=FieldBCs(FieldBoundaryCondition.dirichlet(plasma_potential),
                           FieldBoundaryCondition.dirichlet(voltage), neumann, neumann),
        objects={"pg": plate(0.5e-3, 1.0e-3, 1.0e-3, 3.1e-3, 0.0),
                 "eg": plate(3.0e-3, 4.0e-3, 1.2e-3, 3.1e-3, voltage)},
        beams=[BeamSpecies("ion", 50.0, (0.0, 0.0), (0.0, 0.9e-3), charge=sign, mass=1.0,
                           energy=5.0, transverse_temperature=0.5, num_particles=100)],
        plasma=ExtractionPlasma(5.0, plasma_potential, 0.6e-3),
        **{"iterations": 30, "tolerance": 1e-4, "relaxation": 0.8,
           "diagnostic_planes": [7.5e-3], **settings},
    )  # fmt: skip


def host_twin(mesh):
    """The same mesh classified again on the host alone (no library load): the oracle's
    view of a mesh the product may have classified on the device."""
    from beamtracer_b200.mesh import IonOpticsMesh

    return IonOpticsMesh(
        shape=mesh.shape, origin=mesh.origin, h=mesh.h, geometry=mesh.geometry,
        electrodes=mesh.electrodes, faces=dict(mesh.faces), patch=mesh.patch,
        symmetry_plane=mesh.symmetry_plane, x_nodes=mesh.x_nodes, logical_x0=mesh.logical_x0,
        classify_on_device=False,
    )  # fmt: skip


def mesh_problem(mesh, *, planes=(), integrator: int = 0, step_fraction: float = 0.5,
                 max_steps: int = 100_000, magnetic=None) -> oracle_vlasov.Problem:
    """The oracle's description of a mesh (classified again on the host), its electrodes
    and a trace; ``magnetic`` an `AxisymmetricMagneticField` (cylindrical mesh) or
    `PlanarSolenoidField` (planar)."""
    from beamtracer_b200.fields import PlanarSolenoidField
    from beamtracer_b200.mesh import FACES
    from beamtracer_b200.tracer import electrode_lookup, geometry_code

    if getattr(mesh, "classify_on_device", None) is not False:
        mesh = host_twin(mesh)
    cells, subcells = electrode_lookup(mesh)
    neumann = tuple(0.0 if mesh.faces[f].kind != "neumann" else float(mesh.faces[f].value)
                    for f in FACES)  # fmt: skip
    mag = None
    if isinstance(magnetic, PlanarSolenoidField):
        f = magnetic.field
        mag = (2, f.order, f.z0, f.hz, magnetic.axis_y, f.samples)
    elif magnetic is not None:
        mag = (1, magnetic.order, magnetic.z0, magnetic.hz, 0.0, magnetic.samples)
    return oracle_vlasov.Problem(
        shape=mesh.shape, x=np.asarray(mesh.x, float), h=mesh.h, origin=mesh.origin,
        logical_origin=mesh.logical_origin, logical_upper=mesh.logical_upper,
        geometry=geometry_code(mesh), graded=mesh.graded, fixed=mesh.fixed,
        fixed_value=mesh.fixed_value, solid=mesh.solid, near_solid=mesh.near_solid,
        distance=mesh.distance, neumann=neumann, cells=cells, subcells=subcells,
        inside_solid=mesh.inside_solid, planes=tuple(planes), integrator=integrator,
        step_fraction=step_fraction, max_steps=max_steps, magnetic=mag,
    )  # fmt: skip


def config_problem(config) -> tuple[oracle_vlasov.Problem, object, float]:
    """The oracle's problem, beam and ``sum J / v`` of a `BeamOpticsConfig`, built on the
    host alone: no device classification, no library load."""
    from beamtracer_b200.model import config_magnetic_field, config_mesh, config_particles
    from beamtracer_b200.tracer import INTEGRATORS

    mesh = config_mesh(config, classify_on_device=False)
    problem = mesh_problem(mesh, planes=config.diagnostic_planes,
                           integrator=INTEGRATORS.index(config.integrator),
                           step_fraction=config.step_fraction, max_steps=config.max_steps,
                           magnetic=config_magnetic_field(config, mesh))  # fmt: skip
    particles, j_over_v = config_particles(config)
    return problem, particles, j_over_v


def oracle_problem(model) -> oracle_vlasov.Problem:
    """The oracle's description of a `BeamOptics` model's mesh, electrodes and trace."""
    from beamtracer_b200.tracer import INTEGRATORS

    config = model.config
    return mesh_problem(model.mesh, planes=config.diagnostic_planes,
                        integrator=INTEGRATORS.index(config.integrator),
                        step_fraction=config.step_fraction, max_steps=config.max_steps,
                        magnetic=model.tracer.magnetic)  # fmt: skip


def slit_lens(**settings) -> BeamOpticsConfig:
    """IBSimu's vlasov2d, coarse: protons from a slit through three planar electrodes (the
    reference's ``tests/unit/test_compiled_tracer.py:40-94``), 121 x 51 on 120 x 50 mm."""
    neumann = FieldBoundaryCondition.neumann(0.0)
    objects = {
        "plasma": ObjectParams("rectangle", "dirichlet", -3000.0, midpoint=(0.01, 0.034),
                               side_lengths=(0.02, 0.032)),
        "puller": ObjectParams("rectangle", "dirichlet", -14000.0, midpoint=(0.035, 0.035),
                               side_lengths=(0.01, 0.03)),
        "ground": ObjectParams("polygon", "dirichlet", -1000.0,
                               vertices=((0.06, 0.04), (0.08, 0.03), (0.12, 0.03), (0.12, 0.05),
                                         (0.06, 0.05))),
    }  # fmt: skip
    return BeamOpticsConfig(
        grid=GridParams(num_gridpoints=(121, 51), upper_bound=(0.12, 0.05)),
        objects=objects,
        bcs_field=FieldBCs(x_lower=FieldBoundaryCondition.dirichlet(-3000.0),
                           x_upper=FieldBoundaryCondition.dirichlet(-1000.0),
                           y_lower=neumann, y_upper=neumann),
        beams=[BeamSpecies("H+", 50.0, (0.0, 0.0), (0.0, 0.012), mass=1.0, energy=3000.0,
                           transverse_temperature=0.0, num_particles=300)],
        **{"iterations": 3, "tolerance": 0.0, "diagnostic_planes": [0.05, 0.115], **settings},
    )  # fmt: skip


def refined_problem(config):
    """`config_problem` of a configuration with refined boxes, and the boxes' layout (built
    on the host alone)."""
    from beamtracer_b200.model import config_mesh
    from beamtracer_b200.refinement import Refinement, layout_of_mesh

    problem, particles, j_over_v = config_problem(config)
    mesh = config_mesh(config, classify_on_device=False)
    boxes = [Refinement(b.level, b.lower, b.upper) for b in config.refinement]
    return problem, particles, j_over_v, layout_of_mesh(mesh, boxes)
