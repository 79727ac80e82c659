"""Ion extraction from a plasma into a solenoid: the planar plasma + magnetic workload.

A planar mesh of 1025 x 513 nodes on 40 x 10 mm (x graded with uniform nodes every
39.0625 um over y's 19.53125 um), a Boltzmann-electron plasma (T_e = 5 eV, U_p = 10 V,
n_e = 1e17 m^-3) held at U_p up to x = 0.5 mm in the first iteration, a plasma electrode
(0 V) and an extraction electrode (-10 kV) with 4 mm wide slits centred on y = 5 mm, and a
0.2 T, 40 mm long solenoid of 10 mm winding radius centred at x = 20 mm whose axis is the
line y = 5 mm (its field to first order off the axis, sampled at half the y spacing).  An
H+ beam of 300 A/m^2 leaves the line x = 0, y in [3.5, 6.5] mm at 5 eV with a 1 eV
transverse temperature drawn from ``numpy.random.default_rng(seed)``; Boris's step; the
Newton solve with the multigrid-preconditioned Krylov solver.  The reference enters this
case at ``vlasov_iterate`` with ``BeamTracer(mesh, None, magnetic=f)`` (a planar mesh
takes a magnetic callable, ``tracer.py:401-404``).
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Any

import numpy as np
from scipy import constants

from beamtracer_b200.fields import AxisymmetricMagneticField, PlanarSolenoidField, solenoid_on_axis
from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from beamtracer_b200.tracer import BeamTracer, beam_with_energy
from beamtracer_b200.vlasov import PlasmaModel, VlasovState, vlasov_iterate

PROTON_MASS_U = 1.007276


@dataclass(frozen=True)
class SolenoidExtractionDesign:
    """The case's settings; lengths in m, potentials in V, fields in T."""

    shape: tuple[int, int] = (1025, 513)
    length: float = 40e-3
    height: float = 10e-3
    axis_y: float = 5e-3
    electron_temperature: float = 5.0
    plasma_potential: float = 10.0
    electron_density: float = 1e17  # m^-3
    plasma_x: float = 0.5e-3
    slit: float = 4e-3  # full width
    plasma_electrode: tuple[float, float] = (1.0e-3, 1.5e-3)
    extraction_electrode: tuple[float, float] = (5.0e-3, 6.0e-3)
    extraction_voltage: float = -10e3
    solenoid_centre: float = 20e-3
    solenoid_length: float = 40e-3
    solenoid_radius: float = 10e-3
    solenoid_peak: float = 0.2
    field_order: int = 1
    current_density: float = 300.0
    energy: float = 5.0
    transverse_temperature: float = 1.0
    beam_half_width: float = 1.5e-3
    trajectories: int = 100_000
    iterations: int = 20
    tolerance: float = 1e-3
    relaxation: float = 0.5
    seed: int = 3

    def small(self, shape=(129, 65), trajectories: int = 400) -> SolenoidExtractionDesign:
        """The same case on a coarser mesh with fewer trajectories."""
        return replace(self, shape=shape, trajectories=trajectories)


@dataclass
class SolenoidExtraction:
    """The case built: mesh, beam, plasma, tracer (with its magnetic field)."""

    design: SolenoidExtractionDesign
    mesh: IonOpticsMesh
    particles: Any
    j_over_v: float
    plasma: PlasmaModel
    magnetic: PlanarSolenoidField
    tracer: BeamTracer

    def make_particles(self):
        return self.particles, self.j_over_v

    def run(self, callback=None, poisson=None, iterations: int | None = None,
            tolerance: float | None = None) -> VlasovState:  # fmt: skip
        d = self.design
        return vlasov_iterate(
            self.mesh, self.make_particles, self.tracer,
            iterations=d.iterations if iterations is None else iterations,
            plasma=self.plasma, tolerance=d.tolerance if tolerance is None else tolerance,
            relaxation=d.relaxation, callback=callback, poisson=poisson,
        )  # fmt: skip


def _slit_electrode(x0: float, x1: float, axis_y: float, half: float, voltage: float):
    def inside(x, y):
        x, y = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
        return (x >= x0) & (x <= x1) & (np.abs(y - axis_y) >= half)

    return Electrode(inside, float(voltage))


def solenoid_extraction(design: SolenoidExtractionDesign = SolenoidExtractionDesign(),
                        *, window: int = 64) -> SolenoidExtraction:  # fmt: skip
    nx, ny = design.shape
    h = design.height / (ny - 1)
    x_nodes = np.linspace(0.0, design.length, nx)
    half = 0.5 * design.slit
    mesh = IonOpticsMesh(
        shape=design.shape, origin=(0.0, 0.0), h=h, geometry="planar", x_nodes=x_nodes,
        electrodes=[
            _slit_electrode(*design.plasma_electrode, design.axis_y, half, 0.0),
            _slit_electrode(*design.extraction_electrode, design.axis_y, half,
                            design.extraction_voltage),
        ],
        faces={"x_min": FaceCondition("dirichlet", design.plasma_potential),
               "x_max": FaceCondition("dirichlet", design.extraction_voltage),
               "y_min": FaceCondition("neumann", 0.0), "y_max": FaceCondition("neumann", 0.0)},
    )  # fmt: skip
    dz = 0.5 * h
    z = np.arange(-8 * dz, design.length + 8.5 * dz, dz)
    bz = solenoid_on_axis(z, design.solenoid_centre, design.solenoid_length,
                          design.solenoid_radius, design.solenoid_peak)  # fmt: skip
    field = AxisymmetricMagneticField(float(z[0]), dz, bz, order=design.field_order)
    magnetic = PlanarSolenoidField(field, design.axis_y)
    particles, j_over_v = beam_with_energy(
        design.trajectories, design.current_density, 1.0, PROTON_MASS_U, design.energy, 0.0,
        design.transverse_temperature, (0.0, design.axis_y - design.beam_half_width),
        (0.0, design.axis_y + design.beam_half_width), cylindrical=False,
        sampling=np.random.default_rng(design.seed),
    )  # fmt: skip
    plasma = PlasmaModel(design.electron_temperature, design.plasma_potential, design.plasma_x,
                         constants.e * design.electron_density)  # fmt: skip
    tracer = BeamTracer(mesh, None, magnetic, integrator="boris", window=window)
    return SolenoidExtraction(design, mesh, particles, j_over_v, plasma, magnetic, tracer)
