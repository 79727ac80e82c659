"""The Vlasov iteration: solve the field, trace the beam, deposit its space charge, repeat.

The interface and the loop of the reference's ``solver/vlasov.py`` (``vlasov_iterate``,
``PlasmaModel``, ``NegativeIonPlasmaModel``, ``Compensation``, ``AndersonMixer``,
``VlasovState``, ``thin_particles``; ``vlasov.py:37-429``), with the potential, the edge
fields, the beam and the charge density resident on the device from iteration to
iteration: an iteration is the field solve (``IonOpticsPoisson.solve_device``), the edge
field, the trace of the beam loaded once, and one kernel that turns the node charges into
the mixed density and reports the largest changes.  Only scalars cross to the host inside
the loop; the state's arrays are copied back when they are read.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from beamtracer_b200 import _lib
from beamtracer_b200.fields import MeshArrays, StaggeredElectricField
from beamtracer_b200.mesh import IonOpticsMesh
from beamtracer_b200.poisson import BoltzmannElectrons, BoltzmannIons, IonOpticsPoisson
from beamtracer_b200.tracer import BeamParticles, BeamTracer, TraceResult


@dataclass(frozen=True)
class PlasmaModel:
    """Boltzmann plasma electrons for positive-ion extraction (``vlasov.py:37-64``)."""

    electron_temperature: float
    plasma_potential: float
    initial_plasma_x: float
    rho_e: float | None = None

    @property
    def density(self) -> float | None:
        return self.rho_e

    def boltzmann(self, density: float) -> BoltzmannElectrons:
        return BoltzmannElectrons(density, self.electron_temperature, self.plasma_potential)


@dataclass(frozen=True)
class NegativeIonPlasmaModel:
    """Boltzmann plasma ions for negative-ion extraction (``vlasov.py:67-93``)."""

    ion_temperature: float
    plasma_potential: float
    initial_plasma_x: float
    rho_p: float | None = None

    @property
    def density(self) -> float | None:
        return self.rho_p

    def boltzmann(self, density: float) -> BoltzmannIons:
        return BoltzmannIons(density, self.ion_temperature, self.plasma_potential)


@dataclass(frozen=True)
class Compensation:
    """The beam's charge density times ``1 - fraction`` for ``x_min <= x <= x_max``."""

    x_min: float
    x_max: float
    fraction: float


def compensation_factors(x: np.ndarray, compensation: Sequence[Compensation]) -> np.ndarray | None:
    """The factor of every node column (``vlasov.py:176-184``), or None for no regions."""
    if not compensation:
        return None
    factor = np.ones(len(x))
    for region in compensation:
        inside = (x >= region.x_min) & (x <= region.x_max)
        factor[inside] *= 1.0 - region.fraction
    return factor


class AndersonMixer:
    """Anderson acceleration of ``rho = G(rho)`` (the interface of ``vlasov.py:127-173``),
    on the device (``bt_anderson_mix``).

    Type II: from the last ``depth + 1`` iterates x and residuals f = G(x) - x, the
    differences dX, dF of consecutive ones, ``gamma = argmin |f - dF gamma|`` (singular
    values below 1e-10 of the largest cut off, as NumPy's ``lstsq(rcond=1e-10)``) and
    ``x + w f - (dX + w dF) gamma``; with no history ``x + w f``.  The iterates stay in
    ring buffers on the device; the least-squares problem is solved there too.
    """

    def __init__(self, depth: int = 5, relaxation: float = 1.0) -> None:
        if depth < 1:
            raise ValueError(f"depth must be at least 1, got {depth}")
        if depth > 16:
            raise ValueError(f"depth must be at most 16 on the device, got {depth}")
        self.depth = int(depth)
        self.relaxation = float(relaxation)
        self._rings = None
        self._count = 0
        self._head = -1

    def reset(self) -> None:
        """Forget the stored iterates."""
        self._count = 0
        self._head = -1

    def _buffers(self, n: int):
        import torch

        if self._rings is None or self._rings[0].shape[1] != n:
            rows = self.depth + 1
            make = lambda k: torch.empty((k, n), dtype=torch.float64, device="cuda")  # noqa: E731
            self._rings = (make(rows), make(rows), make(self.depth))
            self.reset()
        return self._rings

    def mix(self, rho, charge, volumes=None, column=None, stats=None) -> None:
        """``rho`` (device, (nx, ny)) <- the mixed density, from the deposit
        ``charge / volumes`` times the column factors ``column`` (device arrays or None);
        ``stats`` (device, 2) gets max |new - old| and max |new|."""
        import torch

        nx, ny = rho.shape
        xs, fs, q = self._buffers(nx * ny)
        self._head = (self._head + 1) % (self.depth + 1)
        self._count = min(self._count + 1, self.depth + 1)
        if stats is None:
            stats = torch.empty(2, dtype=torch.float64, device=rho.device)
        ctx = _lib.context()
        d = _lib.dptr
        _lib.check(_lib.lib().bt_anderson_mix(
            ctx.handle, d(charge), d(volumes), d(column), nx, ny, self.depth, self._count,
            self._head, self.relaxation, d(xs), d(fs), d(q), d(rho), d(stats)))  # fmt: skip

    def update(self, rho, deposit):
        """The next density from ``rho`` and its deposit ``G(rho)`` (device arrays), as
        the reference's ``AndersonMixer.update``."""
        new = rho.reshape(rho.shape[0], -1).clone() if rho.dim() == 2 else rho.reshape(1, -1).clone()
        self.mix(new, deposit.reshape(new.shape).contiguous())
        return new.reshape(rho.shape)


def thin_particles(particles: BeamParticles, stride: int) -> BeamParticles:
    """The coarse phase's beam (the interface of ``vlasov.py:202-215``): of each species
    the trajectories at positions 0, stride, 2 stride, ... of its own list, their currents
    scaled by one factor so that the species keeps its total |current|."""
    species = np.asarray(particles.species)
    order = np.argsort(species, kind="stable")  # each species' trajectories, in list order
    groups = np.split(order, np.flatnonzero(np.diff(species[order])) + 1)
    magnitude = np.abs(particles.current)
    factor = np.zeros(len(particles))
    for members in groups:
        kept = members[::stride]
        kept_total = magnitude[kept].sum()
        factor[kept] = magnitude[members].sum() / kept_total if kept_total > 0.0 else 1.0
    keep = factor > 0.0
    thinned = particles.subset(keep)
    thinned.current = thinned.current * factor[keep]
    return thinned


class VlasovState:
    """The last iteration: fields, charge density, trace and history (``vlasov.py:103-124``).

    ``potential`` and ``charge_density`` are host arrays, copied from the device when first
    read; ``potential_device``, ``charge_density_device`` are the device arrays.
    """

    def __init__(self, potential, rho, electric, trace, history, plasma) -> None:
        self.potential_device = potential
        self.charge_density_device = rho
        self.electric = electric
        self._trace = trace
        self.history = history
        self.plasma = plasma
        self.layout = None
        self._host: dict[str, np.ndarray] = {}

    def _host_copy(self, name: str, array) -> np.ndarray:
        if name not in self._host:
            self._host[name] = array.cpu().numpy()
        return self._host[name]

    @property
    def potential(self) -> np.ndarray:
        return self._host_copy("potential", self.potential_device)

    @property
    def charge_density(self) -> np.ndarray:
        return self._host_copy("charge_density", self.charge_density_device)

    composite_potential = potential
    composite_charge_density = charge_density

    @property
    def trace(self) -> TraceResult:
        if callable(self._trace):
            self._trace = self._trace()
        return self._trace


@dataclass
class _Scalars:
    """Device scalars read back once per iteration."""

    values: Any = field(default=None)


def vlasov_iterate(
    mesh: IonOpticsMesh,
    make_particles: Callable[[], tuple[BeamParticles, float]],
    tracer: BeamTracer,
    *,
    iterations: int,
    plasma: PlasmaModel | NegativeIonPlasmaModel | None = None,
    compensation: Sequence[Compensation] = (),
    tolerance: float = 0.0,
    relaxation: float = 1.0,
    mixing: str = "linear",
    anderson_depth: int = 5,
    coarse_particles: float = 1.0,
    coarse_tolerance: float = 0.0,
    field_backend: str = "multigrid",
    comm: Any = None,
    refinement: Sequence = (),
    adaptive: Any = None,
    self_magnetic: bool = False,
    callback: Callable[[int, VlasovState], None] | None = None,
    density_tolerance: float | None = None,
    poisson: IonOpticsPoisson | None = None,
) -> VlasovState:
    """Run at most ``iterations`` Vlasov iterations (``vlasov.py:246-429``).

    Stop when the largest potential change is below ``tolerance`` [V] or, with
    ``density_tolerance``, when the largest change of the charge density relative to its
    largest value is below it.  ``mixing`` is ``"linear"`` (``relaxation``) or
    ``"anderson"``; ``coarse_particles < 1`` traces that share of the trajectories until the
    potential changes by less than ``coarse_tolerance``.  ``make_particles`` returns the beam
    and its ``sum J / v``; a beam identical to the last one is not copied to the device
    again.  ``poisson`` reuses a field solver of this mesh.
    """
    import torch

    if mixing not in ("linear", "anderson"):
        raise ValueError(f"mixing must be 'linear' or 'anderson', got {mixing!r}")
    if not 0.0 < coarse_particles <= 1.0:
        raise ValueError(f"coarse_particles must be in (0, 1], got {coarse_particles}")
    if adaptive is not None or self_magnetic:
        raise NotImplementedError(
            "adaptive refinement and the self magnetic field are not part of this build"
        )
    if tuple(refinement):
        if tuple(compensation) or coarse_particles < 1.0 or tracer.magnetic is not None:
            raise NotImplementedError(
                "refined boxes take no compensation, no coarse phase and no magnetic field "
                "in this build"
            )
        return _iterate_refined(
            mesh, make_particles, tracer, iterations=iterations, plasma=plasma,
            tolerance=tolerance, relaxation=relaxation, mixing=mixing,
            anderson_depth=anderson_depth, refinement=tuple(refinement), callback=callback,
            density_tolerance=density_tolerance, poisson=poisson,
        )  # fmt: skip
    stride = int(np.ceil(1.0 / coarse_particles - 1e-9))
    coarse = stride > 1
    if coarse and not coarse_tolerance > 0.0:
        raise ValueError("coarse_particles < 1 needs a positive coarse_tolerance")
    mixer = AndersonMixer(anderson_depth, relaxation) if mixing == "anderson" else None
    if poisson is None:
        poisson = IonOpticsPoisson(mesh, backend=field_backend, comm=comm)
    ctx = _lib.context()
    arrays = MeshArrays(mesh)
    nx, ny = mesh.shape
    dev = "cuda"
    rho = torch.zeros((nx, ny), dtype=torch.float64, device=dev)
    phi = torch.zeros((nx, ny), dtype=torch.float64, device=dev)
    previous = torch.zeros_like(phi)
    fx = torch.empty((nx + 1, ny), dtype=torch.float64, device=dev)
    fy = torch.empty((nx, ny + 1), dtype=torch.float64, device=dev)
    factors = compensation_factors(mesh.x, compensation)
    column = None if factors is None else torch.from_numpy(factors).to(dev)
    scalars = torch.zeros(5, dtype=torch.float64, device=dev)
    region_x = None if plasma is None else plasma.initial_plasma_x
    engine = tracer.engine()
    loaded: BeamParticles | None = None
    history: list[dict[str, float]] = []
    boltzmann = None
    j_over_v: float | None = None
    state: VlasovState | None = None
    have_potential = False
    for iteration in range(iterations):
        previous.copy_(phi)
        if plasma is not None and iteration == 0:
            region = lambda x, y: x < region_x  # noqa: E731
            poisson.solve_device(phi, rho, fixed_region=region,
                                 fixed_potential=plasma.plasma_potential)  # fmt: skip
        else:
            if plasma is not None and boltzmann is None:
                density = plasma.density if plasma.density is not None else j_over_v
                boltzmann = plasma.boltzmann(density)
            if not have_potential:
                poisson.solve_device(phi, rho)
            if boltzmann is not None:
                poisson.solve_device(phi, rho, plasma=boltzmann)
            else:
                if have_potential:
                    poisson.solve_device(phi, rho)
        _lib.check(_lib.lib().bt_max_abs_diff(ctx.handle, _lib.dptr(phi), _lib.dptr(previous),
                                              nx * ny, _lib.dptr(scalars)))  # fmt: skip
        efield = StaggeredElectricField(mesh, phi, arrays=arrays, out=(fx, fy))
        tracer.electric = efield
        particles, j_over_v = make_particles()
        if coarse:
            potential_change = float(scalars[0]) if have_potential else float("inf")
            if potential_change < coarse_tolerance:
                coarse = False
                if mixer is not None:
                    mixer.reset()
        if coarse:
            particles = thin_particles(particles, stride)
        if particles is not loaded and particles is not engine.particles:
            engine.load(particles)
        loaded = particles
        engine.run(fx, fy)
        if tracer.reduce is not None:
            tracer.reduce(engine.charge)  # the node charges of every rank's share, summed
        tracer._capacity = engine.capacity
        if mixer is not None and iteration > 0:
            mixer.mix(rho, engine.charge.reshape(nx, ny), engine.volumes, column,
                      scalars[1:3])  # fmt: skip
        else:
            _lib.check(
                _lib.lib().bt_vlasov_mix(
                    ctx.handle, _lib.dptr(engine.charge), _lib.dptr(engine.volumes),
                    _lib.dptr(column), nx, ny, float(relaxation), int(iteration == 0),
                    _lib.dptr(rho), _lib.dptr(scalars) + 8,
                )
            )  # fmt: skip
        if engine.n:
            scalars[3] = engine.steps.max().to(torch.float64)
            scalars[4] = engine.steps.sum().to(torch.float64)  # exact below 2^53 steps
        host = scalars.cpu().numpy()
        total_steps = int(host[4]) if engine.n else 0
        change = float(host[0]) if have_potential else float("inf")
        have_potential = True
        density_change = float(host[1] / host[2]) if host[2] > 0 else 0.0
        history.append({
            "iteration": iteration,
            "max_potential_change": change,
            "relative_density_change": density_change if iteration > 0 else float("inf"),
            "newton_iterations": poisson.newton_iterations,
            "krylov_steps": poisson.krylov_steps,
            "steps": int(host[3]) if engine.n else 0,
            "total_steps": total_steps,
            "trajectories": len(particles),
            "boxes": 1,
            "max_self_magnetic": 0.0,
        })  # fmt: skip
        density_now = engine.density()
        state = VlasovState(phi, rho, efield, lambda d=density_now: engine.result(d), history,
                            boltzmann)  # fmt: skip
        if callback is not None:
            _ = state.trace  # the buffers are reused by the next trace
            callback(iteration, state)
        if not coarse:
            if change < tolerance:
                break
            if density_tolerance is not None and iteration > 0 and density_change < density_tolerance:
                break
    assert state is not None
    return state


class RefinedVlasovState(VlasovState):
    """The last iteration on refined boxes: ``composite_potential`` and
    ``composite_charge_density`` on the layout's composite nodes, ``potential`` and
    ``charge_density`` their values at the base mesh's nodes (``Layout.on_base``)."""

    def __init__(self, layout, potential, rho, electric, trace, history) -> None:
        super().__init__(potential, rho, electric, trace, history, None)
        self.layout = layout

    @property
    def composite_potential(self) -> np.ndarray:
        return self._host_copy("potential", self.potential_device)

    @property
    def composite_charge_density(self) -> np.ndarray:
        return self._host_copy("charge_density", self.charge_density_device)

    @property
    def potential(self) -> np.ndarray:
        return self.layout.on_base(self.composite_potential)

    @property
    def charge_density(self) -> np.ndarray:
        return self.layout.on_base(self.composite_charge_density)


def _iterate_refined(mesh, make_particles, tracer, *, iterations, plasma, tolerance,
                     relaxation, mixing, anderson_depth, refinement, callback,
                     density_tolerance, poisson) -> RefinedVlasovState:  # fmt: skip
    """`vlasov_iterate` on refined boxes (``vlasov.py:304-427`` with a `Layout`): the
    composite field solve, the patches' edge fields, one trace through every patch, the
    patches' deposits summed on the composite nodes and divided by their volumes, mixing.
    """
    import torch

    from beamtracer_b200.composite import PatchedElectricField, PatchedFieldMaps

    if poisson is None or tuple(poisson.refinement) != tuple(refinement):
        poisson = IonOpticsPoisson(mesh, refinement=refinement)
    layout = poisson.layout
    maps = PatchedFieldMaps(layout)
    mixer = AndersonMixer(anderson_depth, relaxation) if mixing == "anderson" else None
    ctx = _lib.context()
    n = layout.size
    dev = "cuda"
    rho = torch.zeros(n, dtype=torch.float64, device=dev)
    phi = torch.zeros(n, dtype=torch.float64, device=dev)
    previous = torch.zeros_like(phi)
    charge = torch.zeros(n, dtype=torch.float64, device=dev)
    scalars = torch.zeros(5, dtype=torch.float64, device=dev)
    engine = tracer.engine()
    engine.set_patches(maps.patch_int, maps.patch_real, maps.n_field_nodes)
    loaded = None
    history: list[dict[str, float]] = []
    state = None
    region_x = None if plasma is None else plasma.initial_plasma_x
    boltzmann = None
    j_over_v = None
    for iteration in range(iterations):
        previous.copy_(phi)
        if plasma is not None and iteration == 0:
            poisson.solve_device(phi, rho, fixed_region=lambda x, y: x < region_x,
                                 fixed_potential=plasma.plasma_potential)  # fmt: skip
        elif plasma is not None:
            if boltzmann is None:
                density = plasma.density if plasma.density is not None else j_over_v
                boltzmann = plasma.boltzmann(density)
            poisson.solve_device(phi, rho, plasma=boltzmann)
        else:
            poisson.solve_device(phi, rho)
        _lib.check(_lib.lib().bt_max_abs_diff(ctx.handle, _lib.dptr(phi), _lib.dptr(previous),
                                              n, _lib.dptr(scalars)))  # fmt: skip
        efield = PatchedElectricField(layout, phi, maps=maps)
        tracer.electric = efield
        particles, j_over_v = make_particles()
        if particles is not loaded and particles is not engine.particles:
            engine.load(particles)
        loaded = particles
        engine.run(maps.fx, maps.fy)
        if tracer.reduce is not None:
            tracer.reduce(engine.charge)
        tracer._capacity = engine.capacity
        maps.charge_map.apply(engine.charge.reshape(-1), charge)
        if mixer is not None and iteration > 0:
            mixer.mix(rho.view(n, 1), charge.view(n, 1), maps.volumes, None, scalars[1:3])
        else:
            _lib.check(_lib.lib().bt_vlasov_mix(
                ctx.handle, _lib.dptr(charge), _lib.dptr(maps.volumes), None, n, 1,
                float(relaxation), int(iteration == 0), _lib.dptr(rho), _lib.dptr(scalars) + 8,
            ))  # fmt: skip
        if engine.n:
            scalars[3] = engine.steps.max().to(torch.float64)
            scalars[4] = engine.steps.sum().to(torch.float64)
        host = scalars.cpu().numpy()
        change = float(host[0]) if iteration > 0 else float("inf")
        density_change = float(host[1] / host[2]) if host[2] > 0 else 0.0
        history.append({
            "iteration": iteration,
            "max_potential_change": change,
            "relative_density_change": density_change if iteration > 0 else float("inf"),
            "newton_iterations": poisson.newton_iterations,
            "krylov_steps": poisson.krylov_steps,
            "steps": int(host[3]) if engine.n else 0,
            "total_steps": int(host[4]) if engine.n else 0,
            "trajectories": len(particles),
            "boxes": len(layout.patches),
            "max_self_magnetic": 0.0,
        })  # fmt: skip
        density_now = charge / maps.volumes
        state = RefinedVlasovState(layout, phi, rho, efield,
                                   lambda d=density_now: engine.result(d), history)  # fmt: skip
        state.plasma = boltzmann
        if callback is not None:
            _ = state.trace
            callback(iteration, state)
        if change < tolerance:
            break
        if density_tolerance is not None and iteration > 0 and density_change < density_tolerance:
            break
    assert state is not None
    return state
