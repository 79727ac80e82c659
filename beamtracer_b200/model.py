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
from beamtracer_b200.refinement import Refinement
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

#: The faces of a mesh and the (direction, side) the configuration names them by.
_FACES = {"x_min": ("x", "min"), "x_max": ("x", "max"), "y_min": ("y", "min"),
          "y_max": ("y", "max")}  # fmt: skip

#: Magnetic profile samples kept beyond each end of the mesh (the series' stencils need 3).
_PROFILE_MARGIN = 8


def _electrode(name: str, params: ObjectParams) -> Electrode:
    if params.bc_type != "dirichlet" or params.bc_value is None:
        raise ValueError("BeamOptics electrodes need a Dirichlet potential")
    return Electrode(params.inside, float(params.bc_value), name)


def config_faces(config: BeamOpticsConfig) -> dict[str, FaceCondition]:
    """The mesh's face conditions of a configuration (the axis and a symmetry plane are
    the mesh's own ``y_min``)."""
    cylindrical = config.grid.coordinates == "cylindrical"
    faces = {}
    for face, (direction, side) in _FACES.items():
        if face == "y_min" and cylindrical:
            continue
        bc = config.bcs_field.get_bc(dir=direction, side=side)
        if face == "y_min" and config.symmetry_plane:
            zero = not callable(bc.value) and float(bc.value) == 0.0
            if bc.bc_type != "neumann" or not zero:
                raise ValueError(
                    "with symmetry_plane the y lower face needs a zero normal derivative"
                )
            continue
        faces[face] = FaceCondition(bc.bc_type, bc.value)
    return faces


def config_mesh(config: BeamOpticsConfig, *, classify_on_device: bool | None = None
                ) -> IonOpticsMesh:  # fmt: skip
    """The `IonOpticsMesh` of a configuration (``classify_on_device=False``: classified on
    the host alone)."""
    grid = config.grid
    return IonOpticsMesh(
        shape=grid.num_gridpoints, origin=grid.lower_bound, h=grid.deltas[0],
        geometry="cylindrical" if grid.coordinates == "cylindrical" else "planar",
        electrodes=[_electrode(name, obj) for name, obj in config.objects.items()],
        faces=config_faces(config), symmetry_plane=config.symmetry_plane,
        classify_on_device=classify_on_device,
    )  # fmt: skip


def config_magnetic_field(config: BeamOpticsConfig, mesh: IonOpticsMesh
                          ) -> AxisymmetricMagneticField | None:  # fmt: skip
    """The axisymmetric field of the solenoids and the measured axial field (the sampling
    of ``model.py:169-188``).  Without an axial field the profile is sampled every half
    node spacing over the mesh and `_PROFILE_MARGIN` samples past each end; the solenoids
    are added to the axial field's samples or to that zero profile."""
    if not config.solenoids and config.axial_field is None:
        return None
    axial = config.axial_field
    if axial is not None:
        z0, dz = float(axial.z0), float(axial.dz)
        bz = np.array(axial.bz, dtype=float)
    else:
        dz = 0.5 * mesh.h
        z0 = mesh.origin[0] - _PROFILE_MARGIN * dz
        span = mesh.upper[0] - mesh.origin[0]
        bz = np.zeros(int(np.ceil(span / dz + 2 * _PROFILE_MARGIN + 0.5)))
    z = z0 + dz * np.arange(bz.size)
    for solenoid in config.solenoids:
        bz += solenoid_on_axis(z, solenoid.centre, solenoid.length, solenoid.radius,
                               solenoid.peak)  # fmt: skip
    return AxisymmetricMagneticField(z0, dz, bz, order=config.field_order)


def _explicit_particles(beam, number: int) -> BeamParticles:
    """A `ParticleBeam`'s given positions, velocities and currents."""
    position, velocity, current = beam.arrays()
    n = len(beam)
    return BeamParticles(
        position=np.ascontiguousarray(np.asarray(position).T),
        velocity=np.ascontiguousarray(np.asarray(velocity).T),
        charge=np.full(n, beam.charge * constants.e),
        mass=np.full(n, beam.mass * constants.atomic_mass),
        current=np.array(current, dtype=float),
        species=np.full(n, number, dtype=np.int32),
    )  # fmt: skip


def config_particles(config: BeamOpticsConfig) -> tuple[BeamParticles, float]:
    """Every beam of a configuration as one `BeamParticles` (species = the beam's place in
    the list) and the ``sum J / v`` of the emitted beams (``model.py:387-448``)."""
    if not config.beams:
        raise ValueError("BeamOptics needs at least one beam")
    cylindrical = config.grid.coordinates == "cylindrical"
    parts, j_over_v = [], 0.0
    for number, beam in enumerate(config.beams):
        if not isinstance(beam, BeamSpecies):
            parts.append(_explicit_particles(beam, number))
            continue
        particles, jv = beam_with_energy(
            beam.num_particles, beam.current_density, beam.charge, beam.mass, beam.energy,
            beam.parallel_temperature, beam.transverse_temperature, beam.start, beam.end,
            cylindrical=cylindrical, species=number, relativistic=config.relativistic,
        )  # fmt: skip
        parts.append(particles)
        j_over_v += jv
    return BeamParticles.concatenate(parts), j_over_v


class BeamOptics:
    """Steady ion beams in planar or cylindrical geometry (``model.py:129-791``)."""

    name = "BeamOptics"
    Config = BeamOpticsConfig

    def __init__(self, config: BeamOpticsConfig | None = None, /, *, comm: Any = None,
                 verbose: bool = False, contracted_trace: bool = False,
                 **settings: object) -> None:  # fmt: skip
        """``contracted_trace``: trace with the build whose multiply-adds are fused (results
        agree with the default build to rounding instead of bit for bit)."""
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
        self.species_names = [beam.name for beam in config.beams]
        self.species_mass = np.array([beam.mass * constants.atomic_mass for beam in config.beams])
        self._state: VlasovState | None = None
        self._is_finished = False
        self._beam: tuple[BeamParticles, float] | None = None
        self.mesh = config_mesh(config)
        self.axial_magnetic_field = config_magnetic_field(config, self.mesh)
        self.field_map = None
        self.tracer = BeamTracer(
            self.mesh, None, self.axial_magnetic_field, step_fraction=config.step_fraction,
            integrator=config.integrator,
            relativistic=config.relativistic, max_steps=config.max_steps,
            planes=config.diagnostic_planes, save_trajectories=config.save_trajectories,
            contracted=contracted_trace,
        )  # fmt: skip

    def _particles(self) -> tuple[BeamParticles, float]:
        """The beams and their ``sum J / v``, made once (every iteration starts from the
        same beam); in a distributed run this rank's share of the trajectories."""
        if self._beam is None:
            particles, j_over_v = config_particles(self.config)
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
            refinement=[Refinement(b.level, b.lower, b.upper) for b in config.refinement],
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

    def surface_fields(self) -> dict[str, float]:
        """The largest |E| [V/m] on the surface of every electrode, by name (the interface
        of ``model.py:591-606``): from the solved potential at the free nodes next to each
        electrode (`surface_field`), 0 for an electrode with no free neighbour."""
        from beamtracer_b200.fields import surface_field_device

        electric = self.state.electric
        # with refined boxes, the base mesh's field (the patches' own fields cover their
        # boxes only)
        base = electric.fields[0] if hasattr(electric, "fields") else electric
        _, _, largest = surface_field_device(self.mesh, base)
        values = largest.cpu().numpy()
        return {name: float(values[k]) for k, name in enumerate(self.config.objects)}

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
        """Trajectories per final status, the launched count, the iterations and whether
        the last iteration met the tolerance."""
        status = np.asarray(self.state.trace.status)
        counts = np.bincount(status[status >= 0].astype(np.int64), minlength=len(STATUS_NAMES))
        stats = dict(zip(STATUS_NAMES, (int(c) for c in counts[: len(STATUS_NAMES)])))
        history = self.state.history
        last_change = history[-1]["max_potential_change"]
        stats.update(launched=int(status.size), iterations=len(history),
                     converged=int(last_change < self.config.tolerance))  # fmt: skip
        return stats

    def plane(self, x: float) -> PlaneHits:
        """The crossings of the diagnostic plane at ``x``."""
        planes = self.state.trace.planes
        match = [hits for hits in planes if np.isclose(hits.position_x, x)]
        if not match:
            raise KeyError(f"no diagnostic plane at x = {x}")
        return match[0]

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
