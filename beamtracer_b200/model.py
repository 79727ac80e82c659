"""Steady ion beams in a self-consistent field: ``BeamOptics(config).run()``.

The interface of the reference's ``model.py`` (``BeamOptics``; ``model.py:129-791``): the
mesh, the tracer and the beams built from a `BeamOpticsConfig`, the Vlasov iteration run
once on the device, and the results -- the potential, the charge density, the plane
crossings and their moments, the statistics and the convergence history.
"""

from __future__ import annotations

import pickle
from collections.abc import Callable
from pathlib import Path
from typing import Any

import numpy as np
from scipy import constants

from beamtracer_b200.config import (
    BeamOpticsConfig,
    BeamSpecies,
    NegativeExtractionPlasma,
    ObjectParams,
)
from beamtracer_b200.diagnostics import BeamMoments, plane_moments
from beamtracer_b200.fields import AxisymmetricMagneticField, solenoid_on_axis
from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from beamtracer_b200.tracer import (
    STATUS_NAMES,
    BeamParticles,
    BeamTracer,
    PlaneHits,
    beam_with_energy,
)
from beamtracer_b200.vlasov import (
    Compensation,
    NegativeIonPlasmaModel,
    PlasmaModel,
    VlasovState,
    vlasov_iterate,
)

_FACES = {"x_min": ("x", "min"), "x_max": ("x", "max"), "y_min": ("y", "min"),
          "y_max": ("y", "max")}  # fmt: skip


def _electrode(name: str, params: ObjectParams) -> Electrode:
    if params.bc_type != "dirichlet" or params.bc_value is None:
        raise ValueError("BeamOptics electrodes need a Dirichlet potential")
    return Electrode(params.inside, float(params.bc_value), name)


class BeamOptics:
    """Steady ion beams in planar or cylindrical geometry (``model.py:129-791``)."""

    name = "BeamOptics"
    Config = BeamOpticsConfig

    def __init__(self, config: BeamOpticsConfig | None = None, /, *, comm: Any = None,
                 verbose: bool = False, **settings: object) -> None:  # fmt: skip
        if config is None:
            config = BeamOpticsConfig(**settings)  # type: ignore[arg-type]
        else:
            if type(config) is not BeamOpticsConfig:
                raise TypeError(f"BeamOptics needs a BeamOpticsConfig, got {type(config).__name__}")
            if settings:
                config = config.replace(**settings)
        self.config = config
        self.comm = comm
        self.rank = comm.Get_rank() if comm is not None else 0
        self.size = comm.Get_size() if comm is not None else 1
        self.verbose = verbose
        grid = config.grid
        self.species_names = [beam.name for beam in config.beams]
        self.species_mass = np.array([beam.mass * constants.atomic_mass for beam in config.beams])
        self._state: VlasovState | None = None
        self._is_finished = False
        self._beam: tuple[BeamParticles, float] | None = None
        self.mesh = IonOpticsMesh(
            shape=grid.num_gridpoints,
            origin=grid.lower_bound,
            h=grid.deltas[0],
            geometry="cylindrical" if grid.coordinates == "cylindrical" else "planar",
            electrodes=[_electrode(name, obj) for name, obj in config.objects.items()],
            faces=self._faces(),
            symmetry_plane=config.symmetry_plane,
        )
        self.axial_magnetic_field = self._magnetic_field()
        self.field_map = None
        self.tracer = BeamTracer(
            self.mesh, None, self.axial_magnetic_field, step_fraction=config.step_fraction,
            integrator=config.integrator,
            relativistic=config.relativistic, max_steps=config.max_steps,
            planes=config.diagnostic_planes, save_trajectories=config.save_trajectories,
        )  # fmt: skip

    def _magnetic_field(self) -> AxisymmetricMagneticField | None:
        """The axisymmetric field of the solenoids and the measured axial field
        (``model.py:169-188``): the solenoids sampled at ``h / 2`` from ``x_min - 8 dz`` to
        ``x_max + 8 dz``, or added to the axial field's samples."""
        config = self.config
        if not config.solenoids and config.axial_field is None:
            return None
        if config.axial_field is not None:
            z0, dz = config.axial_field.z0, config.axial_field.dz
            bz = np.asarray(config.axial_field.bz, dtype=float)
            z = z0 + dz * np.arange(bz.size)
        else:
            dz = 0.5 * self.mesh.h
            lo, hi = self.mesh.origin[0], self.mesh.upper[0]
            z = np.arange(lo - 8 * dz, hi + 8.5 * dz, dz)
            z0 = float(z[0])
            bz = np.zeros(z.size)
        for solenoid in config.solenoids:
            bz = bz + solenoid_on_axis(z, solenoid.centre, solenoid.length, solenoid.radius,
                                       solenoid.peak)  # fmt: skip
        return AxisymmetricMagneticField(z0, dz, bz, order=config.field_order)

    def _faces(self) -> dict[str, FaceCondition]:
        faces = {}
        cylindrical = self.config.grid.coordinates == "cylindrical"
        walls = self.config.bcs_field
        for face, (direction, side) in _FACES.items():
            if cylindrical and face == "y_min":
                continue
            bc = walls.get_bc(dir=direction, side=side)
            if self.config.symmetry_plane and face == "y_min":
                if bc.bc_type != "neumann" or (not callable(bc.value) and float(bc.value) != 0.0):
                    raise ValueError(
                        "with symmetry_plane the y lower face needs a zero normal derivative"
                    )
                continue
            faces[face] = FaceCondition(bc.bc_type, bc.value)
        return faces

    def _particles(self) -> tuple[BeamParticles, float]:
        """The beams and their ``sum J / v`` (``model.py:387-448``); made once, since every
        iteration starts from the same beam."""
        if self._beam is not None:
            return self._beam
        parts = []
        j_over_v = 0.0
        cylindrical = self.mesh.cylindrical
        for number, beam in enumerate(self.config.beams):
            if isinstance(beam, BeamSpecies):
                particles, jv = beam_with_energy(
                    beam.num_particles, beam.current_density, beam.charge, beam.mass,
                    beam.energy, beam.parallel_temperature, beam.transverse_temperature,
                    beam.start, beam.end, cylindrical=cylindrical, species=number,
                    relativistic=self.config.relativistic,
                )  # fmt: skip
                j_over_v += jv
            else:
                n = len(beam)
                position, velocity, current = beam.arrays()
                particles = BeamParticles(
                    position=np.ascontiguousarray(position.T),
                    velocity=np.ascontiguousarray(velocity.T),
                    charge=np.full(n, beam.charge * constants.e),
                    mass=np.full(n, beam.mass * constants.atomic_mass),
                    current=np.array(current, dtype=float),
                    species=np.full(n, number, dtype=np.int32),
                )
            parts.append(particles)
        if not parts:
            raise ValueError("BeamOptics needs at least one beam")
        particles = BeamParticles.concatenate(parts)
        if self.size > 1:
            # every rank traces its share; the node charges are summed over the ranks
            from beamtracer_b200.distributed import share

            particles = particles.subset(share(len(particles), self.rank, self.size))
        self._beam = (particles, j_over_v)
        return self._beam

    def run(self, callback: Callable[[int, VlasovState], None] | None = None, *,
            density_tolerance: float | None = None) -> BeamOptics:  # fmt: skip
        """Run the Vlasov iteration to convergence (once); return the model.

        ``density_tolerance`` also stops the iteration when the largest change of the charge
        density, relative to its largest value, is below it.
        """
        if self._is_finished:
            return self
        config = self.config
        plasma = None
        if isinstance(config.plasma, NegativeExtractionPlasma):
            plasma = NegativeIonPlasmaModel(config.plasma.ion_temperature, config.plasma.plasma_potential,
                                            config.plasma.initial_plasma_x, config.plasma.rho_p)  # fmt: skip
        elif config.plasma is not None:
            plasma = PlasmaModel(config.plasma.electron_temperature, config.plasma.plasma_potential,
                                 config.plasma.initial_plasma_x, config.plasma.rho_e)  # fmt: skip
        compensation = [Compensation(c.x_min, c.x_max, c.fraction) for c in config.compensation]
        if self.size > 1:
            self.tracer.reduce = self.comm.allreduce_tensor
        self._state = vlasov_iterate(
            self.mesh, self._particles, self.tracer, iterations=config.iterations,
            plasma=plasma, compensation=compensation, tolerance=config.tolerance,
            relaxation=config.relaxation, mixing=config.mixing,
            anderson_depth=config.anderson_depth, coarse_particles=config.coarse_particles,
            coarse_tolerance=config.coarse_tolerance, field_backend=config.field_backend,
            callback=callback, density_tolerance=density_tolerance,
        )  # fmt: skip
        if self.size > 1:
            from beamtracer_b200.distributed import gather_trace

            gather_trace(self.comm, self._state.trace)
        self._is_finished = True
        return self

    # -- results ----------------------------------------------------------------------------

    @property
    def state(self) -> VlasovState:
        if self._state is None:
            raise RuntimeError("BeamOptics has not run yet")
        return self._state

    @property
    def potential(self) -> np.ndarray:
        """The potential [V] at the nodes (nx, ny)."""
        return self.state.potential

    @property
    def charge_density(self) -> np.ndarray:
        """The beam's (compensated, mixed) charge density [C/m^3] at the nodes."""
        if self._state is None:
            return np.zeros(self.mesh.shape)
        return self.state.charge_density

    def electric_field_at(self, x, y):
        return self.state.electric(x, y)

    @property
    def trajectories(self) -> list[np.ndarray]:
        return self.state.trace.trajectories

    @property
    def trajectory_species(self) -> np.ndarray:
        return self.state.trace.trajectory_species

    @property
    def convergence_history(self) -> list[dict[str, float]]:
        return self.state.history

    @property
    def stats(self) -> dict[str, int]:
        status = self.state.trace.status
        stats = {name: int(np.sum(status == k)) for k, name in enumerate(STATUS_NAMES)}
        stats["launched"] = int(status.size)
        stats["iterations"] = len(self.state.history)
        stats["converged"] = int(
            self.state.history[-1]["max_potential_change"] < self.config.tolerance
        )
        return stats

    def plane(self, x: float) -> PlaneHits:
        """The crossings of the diagnostic plane at ``x``."""
        for hits in self.state.trace.planes:
            if np.isclose(hits.position_x, x):
                return hits
        raise KeyError(f"no diagnostic plane at x = {x}")

    def beam_moments(self, x: float, species: str | None = None, axis: str = "y") -> BeamMoments:
        """The current, emittance and Twiss parameters at the plane ``x``."""
        index = None if species is None else self.species_names.index(species)
        return plane_moments(self.plane(x), cylindrical=self.mesh.cylindrical,
                             mass=self.species_mass, species=index, axis=axis)  # fmt: skip

    def write_files(self, path: Path) -> None:
        """The fields, trajectories and plane crossings as a pickle (``model.py:754-776``)."""
        with open(Path(path) / "beam_optics.pkl", "wb") as file:
            pickle.dump({"x": self.mesh.x, "y": self.mesh.y, "potential": self.potential,
                         "charge_density": self.state.charge_density,
                         "trajectories": self.trajectories,
                         "trajectory_species": self.trajectory_species,
                         "planes": self.state.trace.planes, "species": self.species_names,
                         "stats": self.stats, "convergence_history": self.convergence_history},
                        file)  # fmt: skip

    @property
    def is_finished(self) -> bool:
        return self._is_finished

    @property
    def time(self) -> float:
        return 0.0

    @property
    def iteration(self) -> int:
        return int(self._is_finished)
