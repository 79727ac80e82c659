"""Beams, the trajectory trace and its results, on the B200.

The interface of the reference's ``solver/tracer.py``: ``BeamParticles``,
``beam_with_energy``, ``PlaneHits``, ``TraceResult`` and ``BeamTracer``
(``tracer.py:87-327, 384-1366``).  The trace is the device kernel of
``trace_trajectories_2d`` (``libbt200.so``); around it, as the reference's
``_trace_compiled`` (``tracer.py:1186-1304``) does on the host:

- trajectories starting inside an electrode end at once (status 3);
- trajectories stopped in a sub-cell that an electrode surface cuts (status -2) are
  decided by the electrodes' own ``inside`` tests and the others resumed;
- a trace that records more plane crossings or path points than its buffers hold is
  repeated with larger buffers, which the tracer keeps;
- the node charges are divided by the node volumes (``tracer.py:678-705``).

`TraceEngine` keeps everything of a trace on the device, so the Vlasov iteration can
trace the same beam again and again without copying it back and forth.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np
from scipy import constants

from beamtracer_b200.mesh import IonOpticsMesh
from beamtracer_b200.shapes import shape_table

#: Status of a finished trajectory.
TRANSMITTED, BACKWARD, WALL, ELECTRODE, MAX_STEPS = 0, 1, 2, 3, 4
STATUS_NAMES = ("transmitted", "backward", "wall", "electrode", "max_steps")
_ALIVE, _PAUSED = -1, -2
#: Sub-cells per cell side of the electrode lookup.
SUBCELLS = 8
INTEGRATORS = ("rk4", "boris")


def lorentz_factor(u: np.ndarray, c: float) -> np.ndarray:
    """``sqrt(1 + |u|^2 / c^2)`` of proper velocities ``u`` (3, N)."""
    return np.sqrt(1.0 + np.einsum("ij,ij->j", u, u) / (c * c))


def proper_velocity(v: np.ndarray, c: float) -> np.ndarray:
    """``v / sqrt(1 - |v|^2 / c^2)`` of velocities ``v`` (3, N)."""
    return v / np.sqrt(1.0 - np.einsum("ij,ij->j", v, v) / (c * c))


#: The per-particle arrays of `BeamParticles` and the axis along which particles run.
_PARTICLE_AXES = {"position": 1, "velocity": 1, "charge": 0, "mass": 0, "current": 0,
                  "species": 0}  # fmt: skip


@dataclass
class BeamParticles:
    """Particle starting states (``tracer.py:87-126``): positions and velocities (3, N),
    charge [C], mass [kg], current [A] and species index per particle."""

    position: np.ndarray
    velocity: np.ndarray
    charge: np.ndarray
    mass: np.ndarray
    current: np.ndarray
    species: np.ndarray

    @staticmethod
    def concatenate(parts: Sequence[BeamParticles]) -> BeamParticles:
        """The particles of every part, in order."""
        return BeamParticles(**{
            name: np.concatenate([getattr(p, name) for p in parts], axis=axis)
            for name, axis in _PARTICLE_AXES.items()
        })  # fmt: skip

    def subset(self, index) -> BeamParticles:
        """The particles selected by ``index`` (a mask, indices or a slice)."""
        return BeamParticles(**{
            name: getattr(self, name)[(slice(None),) * axis + (index,)]
            for name, axis in _PARTICLE_AXES.items()
        })  # fmt: skip

    def __len__(self) -> int:
        return int(np.shape(self.position)[1])


def _gaussian_samples(num: int, sampling) -> np.ndarray:
    """(num, 3) standard normal samples.  ``"sobol"``: the points 1..num of the unscrambled
    3D Sobol sequence (its origin left out: its inverse normal is infinite) through the
    inverse normal distribution, so every call draws the same beam; a NumPy generator:
    its ``standard_normal`` draws."""
    if isinstance(sampling, np.random.Generator):
        return sampling.standard_normal((num, 3))
    if sampling != "sobol":
        raise ValueError(f"sampling must be 'sobol' or a numpy Generator, got {sampling!r}")
    from scipy.stats import norm, qmc

    engine = qmc.Sobol(d=3, scramble=False)
    engine.fast_forward(1)
    return norm.ppf(engine.random(num))


@dataclass(frozen=True)
class _EmissionLine:
    """The line a beam leaves: its start, unit direction ``t``, its right-hand normal ``n``
    (the direction of motion) and its length."""

    start: np.ndarray
    t: np.ndarray
    n: np.ndarray
    length: float

    @staticmethod
    def between(start, end) -> _EmissionLine:
        a, b = np.asarray(start, dtype=float), np.asarray(end, dtype=float)
        length = float(np.hypot(*(b - a)))
        if length == 0.0:
            raise ValueError("the beam start line has zero length")
        t = (b - a) / length
        return _EmissionLine(a, t, np.array([t[1], -t[0]]), length)

    def midpoints(self, count: int) -> np.ndarray:
        """(2, count) points at the centres of ``count`` equal pieces of the line."""
        s = (np.arange(count) + 0.5) / count
        return self.start[:, None] + (self.length * self.t)[:, None] * s[None, :]


def beam_with_energy(
    num_particles: int,
    current_density: float,
    charge: float,
    mass: float,
    energy: float,
    parallel_temperature: float,
    transverse_temperature: float,
    start: tuple[float, float],
    end: tuple[float, float],
    *,
    cylindrical: bool,
    species: int = 0,
    sampling="sobol",
    relativistic: bool = False,
) -> tuple[BeamParticles, float]:
    """A beam emitted from the line ``start``-``end`` with ``energy`` [eV]; and ``J / v``.

    The interface and the draw of ``tracer.py:221-291``: one trajectory at the centre of
    each of ``num_particles`` equal pieces of the line, moving along its right-hand normal
    at the beam speed ``v0`` plus Gaussian spreads ``sqrt(T e / m)`` of the temperatures
    [eV] -- the transverse one along the line (and, cylindrical, around the axis), the
    parallel one along the normal; a ring current ``2 pi J s r / N`` (cylindrical) or
    ``J s / N`` per unit depth.  Relativistic: ``v0`` and the spreads are proper speeds
    (``v0 = c sqrt(g^2 - 1)``, ``g = 1 + E e / (m c^2)``) turned into velocities at the
    end.  ``charge`` [e], ``mass`` [u], ``current_density`` [A/m^2].
    """
    q = charge * constants.e
    m = mass * constants.atomic_mass
    line = _EmissionLine.between(start, end)
    c = constants.c
    if relativistic:
        g = 1.0 + energy * constants.e / (m * c * c)
        v0 = float(c * np.sqrt(g * g - 1.0))
    else:
        v0 = float(np.sqrt(2.0 * energy * constants.e / m))
    spread_t, spread_p = (float(np.sqrt(t * constants.e / m))
                          for t in (transverse_temperature, parallel_temperature))  # fmt: skip
    g3 = _gaussian_samples(num_particles, sampling)
    along_normal = v0 + spread_p * g3[:, 1]
    along_line = spread_t * g3[:, 0]
    velocity = np.zeros((3, num_particles))
    velocity[:2] = line.n[:, None] * along_normal[None, :] + line.t[:, None] * along_line[None, :]
    if cylindrical:
        velocity[2] = spread_t * g3[:, 2]
    position = np.zeros((3, num_particles))
    position[:2] = line.midpoints(num_particles)
    if cylindrical:
        current = (2.0 * np.pi * current_density * line.length / num_particles) * position[1]
    else:
        current = np.full(num_particles, current_density * line.length / num_particles)
    if relativistic:
        velocity = velocity / lorentz_factor(velocity, c)
        v0 = v0 / float(np.sqrt(1.0 + (v0 / c) ** 2))
    particles = BeamParticles(
        position=position, velocity=velocity, charge=np.full(num_particles, q),
        mass=np.full(num_particles, m), current=current,
        species=np.full(num_particles, species, dtype=np.int32),
    )  # fmt: skip
    return particles, current_density / v0


#: The per-crossing arrays of `PlaneHits`, their empty values and the axis crossings run along.
_HIT_FIELDS = {
    "point": (lambda: np.zeros((3, 0)), 1), "velocity": (lambda: np.zeros((3, 0)), 1),
    "current": (lambda: np.zeros(0), 0), "species": (lambda: np.zeros(0, dtype=np.int32), 0),
    "direction": (lambda: np.zeros(0, dtype=np.int8), 0),
}  # fmt: skip


@dataclass
class PlaneHits:
    """Crossings of the plane ``x = position_x`` (``tracer.py:295-325``): point and
    velocity (3, m), current, species and direction (+1 / -1) of each."""

    position_x: float
    point: np.ndarray = field(default_factory=_HIT_FIELDS["point"][0])
    velocity: np.ndarray = field(default_factory=_HIT_FIELDS["velocity"][0])
    current: np.ndarray = field(default_factory=_HIT_FIELDS["current"][0])
    species: np.ndarray = field(default_factory=_HIT_FIELDS["species"][0])
    direction: np.ndarray = field(default_factory=_HIT_FIELDS["direction"][0])
    fractions: np.ndarray | None = None

    def append(self, point, velocity, current, species, direction, fractions=None) -> None:
        """Add crossings after the ones held."""
        new = {"point": point, "velocity": velocity, "current": current,
               "species": np.asarray(species).astype(np.int32),
               "direction": np.asarray(direction).astype(np.int8)}  # fmt: skip
        for name, (_, axis) in _HIT_FIELDS.items():
            setattr(self, name, np.concatenate([getattr(self, name), new[name]], axis=axis))
        if fractions is not None:
            self.fractions = (fractions if self.fractions is None
                              else np.concatenate([self.fractions, fractions], axis=1))  # fmt: skip


@dataclass
class TraceResult:
    """The outcome of a trace (``tracer.py:327-347``)."""

    charge_density: Any
    status: np.ndarray
    electrode: np.ndarray
    planes: list[PlaneHits]
    trajectories: list[np.ndarray]
    trajectory_species: np.ndarray
    steps: int
    fractions: np.ndarray | None = None
    tallies: Any = None
    current_density: np.ndarray | None = None


def node_volumes(mesh: IonOpticsMesh) -> np.ndarray:
    """The node volumes the deposit divides by: a quarter of every adjacent cell, a cell
    ``dx h`` (planar, per unit depth) or ``2 pi r_c dx h`` (cylindrical, ``r_c`` its centre's
    radius) -- the volumes the area-weighted deposit is consistent with
    (``solver/refinement.py:274-296`` on an unrefined mesh)."""
    nx, ny = mesh.shape
    cell = mesh.dx[:, None] * np.full(ny - 1, mesh.h)[None, :]
    if mesh.cylindrical:
        centres = mesh.origin[1] + mesh.h * (np.arange(ny - 1) + 0.5)
        cell = 2.0 * np.pi * centres[None, :] * cell
    volumes = np.zeros((nx, ny))
    quarter = 0.25 * cell
    volumes[:-1, :-1] += quarter
    volumes[1:, :-1] += quarter
    volumes[:-1, 1:] += quarter
    volumes[1:, 1:] += quarter
    return volumes


def electrode_cells(mesh: IonOpticsMesh) -> np.ndarray:
    """Cells with an electrode node or a node next to one (``tracer.py:488-493``)."""
    touch = (mesh.solid >= 0) | mesh.near_solid
    return touch[:-1, :-1] | touch[1:, :-1] | touch[:-1, 1:] | touch[1:, 1:]


def subcell_table(mesh: IonOpticsMesh, ci: np.ndarray, cj: np.ndarray) -> np.ndarray:
    """The electrode of every sub-cell (len(ci), 8, 8) of cells (ci, cj): the electrode
    containing its four corners and its centre, -1 for none, -2 where they disagree
    (``tracer.py:1095-1114``)."""

    def sample(fraction: np.ndarray) -> np.ndarray:
        px = mesh.position_x(ci[:, None, None] + fraction[None, :, None])
        py = mesh.origin[1] + mesh.h * (cj[:, None, None] + fraction[None, None, :])
        px, py = np.broadcast_arrays(px, py)
        return mesh.inside_solid(px.ravel(), py.ravel()).reshape(px.shape)

    corner = sample(np.arange(SUBCELLS + 1) / SUBCELLS)
    centre = sample((np.arange(SUBCELLS) + 0.5) / SUBCELLS)
    same = ((corner[:, :-1, :-1] == centre) & (corner[:, 1:, :-1] == centre)
            & (corner[:, :-1, 1:] == centre) & (corner[:, 1:, 1:] == centre))  # fmt: skip
    return np.where(same, centre, -2).astype(np.int64)


def electrode_lookup(mesh: IonOpticsMesh) -> tuple[np.ndarray, np.ndarray]:
    """``cells`` (nx - 1, ny - 1): the number of every cell touching an electrode (-1 for
    the others); ``subcells``: their sub-cell tables, flattened (``tracer.py:1116-1139``)."""
    touching = electrode_cells(mesh)
    cells = np.full(touching.shape, -1, dtype=np.int64)
    ci, cj = np.nonzero(touching)
    if not mesh.electrodes or not ci.size:
        return cells, np.full(1, -1, dtype=np.int64)
    cells[ci, cj] = np.arange(ci.size, dtype=np.int64)
    return cells, subcell_table(mesh, ci, cj).ravel()


def electrode_lookup_device(mesh: IonOpticsMesh):
    """`electrode_lookup` as device tensors, its sub-cell table sampled on the device when
    every electrode is a configuration shape (else on the host)."""
    import torch

    from beamtracer_b200 import _lib

    table = shape_table(mesh) if mesh.electrodes else None
    touching = electrode_cells(mesh)
    if table is None or not touching.any():
        cells, subcells = electrode_lookup(mesh)
        return torch.from_numpy(cells).cuda(), torch.from_numpy(subcells).cuda()
    cells = np.full(touching.shape, -1, dtype=np.int64)
    ci, cj = np.nonzero(touching)
    cells[ci, cj] = np.arange(ci.size, dtype=np.int64)
    kinds, offsets, params = (torch.from_numpy(a).cuda() for a in table)
    ci_d = torch.from_numpy(ci.astype(np.int64)).cuda()
    cj_d = torch.from_numpy(cj.astype(np.int64)).cuda()
    nodes = torch.from_numpy(np.array(mesh.x, dtype=np.float64)).cuda() if mesh.graded else None
    out = torch.empty(ci.size * SUBCELLS * SUBCELLS, dtype=torch.int64, device="cuda")
    shapes = _lib.ShapesDesc(len(kinds), _lib.dptr(kinds), _lib.dptr(offsets), _lib.dptr(params))
    ctx = _lib.context()
    _lib.check(_lib.lib().bt_subcell_table(
        ctx.handle, ctypes.byref(shapes), _lib.dptr(ci_d), _lib.dptr(cj_d), ci.size,
        float(mesh.origin[0]), float(mesh.origin[1]), float(mesh.h),
        _lib.dptr(nodes) if nodes is not None else None, mesh.shape[0] if nodes is not None else 0,
        SUBCELLS, _lib.dptr(out)))  # fmt: skip
    return torch.from_numpy(cells).cuda(), out


def _project(mesh: IonOpticsMesh, x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The mesh coordinates (x, y) or (x, r) of Cartesian points (3, N)."""
    if mesh.cylindrical:
        return x[0], np.hypot(x[1], x[2])
    if mesh.symmetry_plane:
        y0 = mesh.origin[1]
        return x[0], y0 + np.abs(x[1] - y0)
    return x[0], x[1]


def geometry_code(mesh: IonOpticsMesh) -> int:
    """0 planar, 1 cylindrical, 2 planar with a symmetry plane."""
    if mesh.symmetry_plane:
        return 2
    return int(mesh.cylindrical)


class TraceEngine:
    """A trace setup held on the device: the mesh's tables, a beam, the result buffers.

    ``load`` copies a beam to the device once; every ``run`` traces it from its start
    through edge fields ``fx``, ``fy`` (device arrays) and leaves the node charges in
    ``charge`` and the trajectories' ends in the state arrays.
    """

    def __init__(
        self,
        mesh: IonOpticsMesh,
        *,
        planes: Sequence[float] = (),
        integrator: str = "rk4",
        step_fraction: float = 0.5,
        max_steps: int = 100_000,
        inv_c2: float = 0.0,
        save_trajectories: int = 0,
        capacity: tuple[int, int] = (4, 1024),
        window: int = 64,
        magnetic: Any = None,
        contracted: bool = False,
    ) -> None:
        import torch

        from beamtracer_b200 import _lib

        self.torch = torch
        #: trace with the build whose multiply-adds are fused (rounding-level agreement
        #: with the exact build instead of bit-exact)
        self.contracted = bool(contracted)
        self.mesh = mesh
        self.planes = tuple(float(p) for p in planes)
        self.integrator = integrator
        self.step_fraction = float(step_fraction)
        self.max_steps = int(max_steps)
        self.inv_c2 = float(inv_c2)
        self.save_trajectories = int(save_trajectories)
        self.capacity = tuple(capacity)
        self.window = int(window)
        #: a `MagneticProfile` on the device: the NumPy tracer's step in that field
        self.magnetic = magnetic
        self.ctx = _lib.context()
        dev = "cuda"
        nx, ny = mesh.shape
        self.cells, self.subcells = electrode_lookup_device(mesh)
        lo_x, lo_y = mesh.logical_origin
        up_x, up_y = mesh.logical_upper
        self.patch_int = torch.tensor([[nx, ny, 0, 0, nx * ny, 0]], dtype=torch.int64, device=dev)
        self.patch_real = torch.tensor([[lo_x, lo_y, mesh.h, lo_x, lo_y, up_x, up_y]],
                                       dtype=torch.float64, device=dev)  # fmt: skip
        self.x_nodes = torch.from_numpy(
            np.array(mesh.x if mesh.graded else np.zeros(2), dtype=np.float64, order="C")
        ).to(dev)
        self.planes_dev = torch.tensor(self.planes or (np.nan,), dtype=torch.float64, device=dev)
        self.volumes = torch.from_numpy(node_volumes(mesh)).to(dev)
        self.n_nodes = nx * ny
        self._charge = None
        self.particles: BeamParticles | None = None

    def set_patches(self, patch_int, patch_real, n_nodes: int) -> None:
        """Trace through the patches of refined boxes (device tables of the kernel's
        ``patch_int`` (P, 6) and ``patch_real`` (P, 7), finest first and the base mesh last,
        ``tracer.py:1141-1183``): the edge fields given to `run` are the patches' flattened
        one after the other, and the node charges fill ``n_nodes`` (every patch's field
        mesh nodes, in the same order)."""
        self.patch_int = patch_int
        self.patch_real = patch_real
        if int(n_nodes) != self.n_nodes:
            self.n_nodes = int(n_nodes)
            self._charge = None

    @property
    def charge(self):
        """The node charges of the last run (device (1, nodes))."""
        if self._charge is None:
            self._charge = self.torch.zeros((1, self.n_nodes), dtype=self.torch.float64,
                                            device="cuda")  # fmt: skip
        return self._charge

    # -- the beam -------------------------------------------------------------------------

    def load(self, particles: BeamParticles, buffers: bool = True) -> None:
        """Copy a beam to the device (its start states are kept for every run);
        ``buffers=False`` leaves the trace's state and result buffers to the first `run`
        (a caller that traces the start states elsewhere, as a batch, needs none)."""
        torch = self.torch
        mesh = self.mesh
        n = len(particles)
        dev = "cuda"
        self.particles = particles
        self.n = n
        x = np.ascontiguousarray(particles.position, dtype=np.float64)
        v = np.array(particles.velocity, dtype=np.float64, order="C")
        if self.inv_c2 > 0.0:
            v = np.ascontiguousarray(proper_velocity(v, 1.0 / np.sqrt(self.inv_c2)))
        status = np.full(n, _ALIVE, dtype=np.int64)
        electrode = np.full(n, -1, dtype=np.int64)
        if mesh.electrodes and n:
            hit = mesh.inside_solid(*_project(mesh, x))
            dead = hit >= 0
            status[dead] = ELECTRODE
            electrode[dead] = hit[dead]
        self.start_active = torch.from_numpy(np.flatnonzero(status == _ALIVE).astype(np.int64)).to(dev)
        self.x0 = torch.from_numpy(x).to(dev)
        self.v0 = torch.from_numpy(v).to(dev)
        self.status0 = torch.from_numpy(status).to(dev)
        self.electrode0 = torch.from_numpy(electrode).to(dev)
        self.qm = torch.from_numpy(np.ascontiguousarray(particles.charge / particles.mass,
                                                        dtype=np.float64)).to(dev)  # fmt: skip
        current = particles.current.astype(np.float64)
        self.dq = torch.from_numpy(
            np.ascontiguousarray(np.sign(particles.charge) * np.abs(current))
        ).to(dev)
        save = self.save_trajectories
        self.saved_ids = np.arange(0, n, save) if save else np.zeros(0, int)
        slot = np.full(n, -1, dtype=np.int64)
        slot[self.saved_ids] = np.arange(self.saved_ids.size)
        self.path_slot = torch.from_numpy(slot).to(dev)
        px, py = _project(mesh, x[:, self.saved_ids])
        self.first_points = torch.from_numpy(np.stack([px, py], axis=1).copy()).to(dev)
        self._have_buffers = False
        if buffers:
            self._state_buffers()

    def _state_buffers(self) -> None:
        torch = self.torch
        self.x = torch.empty_like(self.x0)
        self.v = torch.empty_like(self.v0)
        self.steps = torch.zeros(self.n, dtype=torch.int64, device="cuda")
        self.status = torch.empty_like(self.status0)
        self.electrode = torch.empty_like(self.electrode0)
        self._allocate_buffers()
        self._have_buffers = True

    def _allocate_buffers(self) -> None:
        torch = self.torch
        capacity, path_capacity = self.capacity
        slots = max(self.saved_ids.size, 1)
        P = len(self.planes_dev)
        self.hits = torch.zeros((self.n, P, capacity, 8), dtype=torch.float64, device="cuda")
        self.counts = torch.zeros((self.n, P), dtype=torch.int64, device="cuda")
        self.paths = torch.zeros((slots, path_capacity, 2), dtype=torch.float64, device="cuda")
        self.path_count = torch.ones(slots, dtype=torch.int64, device="cuda")

    # -- one trace ------------------------------------------------------------------------

    def _reset(self) -> None:
        self.x.copy_(self.x0)
        self.v.copy_(self.v0)
        self.status.copy_(self.status0)
        self.electrode.copy_(self.electrode0)
        self.steps.zero_()
        self.charge.zero_()
        self.counts.zero_()
        self.path_count.fill_(1)
        k = self.saved_ids.size
        if k:
            self.paths[:k, 0] = self.first_points

    def _kernel(self, active, fx, fy) -> None:
        """One call of the trace entry point: its arguments built straight from the
        engine's device tensors (the plugin's staging and checks are for outside callers)."""
        from beamtracer_b200 import _lib

        mesh = self.mesh
        lo_x, lo_y = mesh.logical_origin
        up_x, up_y = mesh.logical_upper
        d = _lib.dptr
        a = _lib.TraceArgs(
            d(active), int(active.numel()), d(self.x), d(self.v), self.n, d(self.qm),
            d(self.dq), d(self.steps), d(self.status), d(self.electrode), d(fx), d(fy),
            d(self.patch_int), d(self.patch_real), int(self.patch_int.shape[0]), float(lo_x),
            float(lo_y), float(mesh.h),
            float(up_x), float(up_y), geometry_code(mesh), INTEGRATORS.index(self.integrator),
            self.step_fraction, self.max_steps, d(self.cells), d(self.subcells), SUBCELLS,
            d(self.planes_dev), int(self.planes_dev.numel()), d(self.hits),
            int(self.hits.shape[2]), d(self.counts), d(self.path_slot), d(self.paths),
            int(self.paths.shape[1]), d(self.path_count), 1, d(self.charge), self.n_nodes,
            int(mesh.graded), d(self.x_nodes), int(self.x_nodes.numel()), self.inv_c2,
        )  # fmt: skip
        lib, ctx = _lib.lib(), _lib.context()
        fast = self.contracted
        if self.magnetic is None:
            entry = lib.bt_trace_trajectories_2d_fast if fast else lib.bt_trace_trajectories_2d
            _lib.check(entry(ctx.handle, ctypes.byref(a), self.window))
        else:
            m = self.magnetic.descriptor()
            entry = (lib.bt_trace_trajectories_2d_magnetic_fast if fast
                     else lib.bt_trace_trajectories_2d_magnetic)  # fmt: skip
            _lib.check(entry(ctx.handle, ctypes.byref(a), ctypes.byref(m), self.window))

    def run(self, fx, fy) -> None:
        """Trace the loaded beam through the edge fields (device arrays)."""
        torch = self.torch
        mesh = self.mesh
        fx, fy = fx.reshape(-1), fy.reshape(-1)
        if not self._have_buffers:
            self._state_buffers()
        zero = torch.zeros(1, dtype=torch.int64, device="cuda")
        while True:
            self._reset()
            active = self.start_active
            while active.numel():
                self._kernel(active, fx, fy)
                # one read-back: the paused trajectories, the fullest hit and path buffers
                paused_mask = self.status[active] == _PAUSED
                flags = torch.stack([paused_mask.sum(),
                                     self.counts.max() if self.counts.numel() else zero[0],
                                     self.path_count.max()]).cpu().tolist()  # fmt: skip
                most, longest = flags[1], flags[2]
                if flags[0] == 0:
                    break
                paused = active[paused_mask]
                points = self.x[:, paused].cpu().numpy()
                hit = mesh.inside_solid(*_project(mesh, points))
                inside = torch.from_numpy(hit >= 0).to("cuda")
                hit_dev = torch.from_numpy(hit.astype(np.int64)).to("cuda")
                stopped = paused[inside]
                self.status[stopped] = ELECTRODE
                self.electrode[stopped] = hit_dev[inside]
                active = paused[~inside]
                self.status[active] = _ALIVE
            else:
                most = int(self.counts.max()) if self.counts.numel() else 0
                longest = int(self.path_count.max())
            capacity, path_capacity = self.capacity
            if most <= capacity and longest <= path_capacity:
                return
            self.capacity = (max(capacity, most), max(path_capacity, longest))
            self._allocate_buffers()

    # -- results --------------------------------------------------------------------------

    def density(self):
        """The charge density on the nodes (device (nx, ny)): charges over volumes."""
        if int(self.patch_int.shape[0]) > 1:
            raise RuntimeError("a trace through refined boxes has composite densities")
        return (self.charge[0] / self.volumes.reshape(-1)).reshape(self.mesh.shape)

    def result(self, density=None) -> TraceResult:
        """The trace as the reference returns it (host arrays; ``tracer.py:1265-1304``).

        The crossings are picked from the hit buffers and ordered (by step, then trajectory,
        as ``tracer.py:1279-1290``) on the device, so only the crossings that exist come to
        the host, in one copy with the trajectory of each.
        """
        import torch

        particles = self.particles
        current = particles.current.astype(float)
        species = particles.species
        n_planes = len(self.planes)
        slots = torch.arange(self.hits.shape[2], device=self.hits.device)
        pieces, sizes = [], []
        #: per plane, the (trajectory, buffer slot) of every returned crossing, in order
        self.hit_slots = []
        for p in range(n_planes):
            k, c = (slots[None, :] < self.counts[:, p, None]).nonzero(as_tuple=True)
            record = self.hits[k, p, c]
            order = torch.sort(record[:, 7], stable=True).indices
            pieces.append(torch.cat([record[order], k[order, None].to(torch.float64)], dim=1))
            self.hit_slots.append((k[order], c[order]))
            sizes.append(int(k.numel()))
        crossings = (torch.cat(pieces).cpu().numpy() if pieces else np.zeros((0, 9)))
        ints = torch.stack([self.status, self.electrode, self.steps]).cpu().numpy()
        status, electrode, steps = ints
        planes, start = [], 0
        for position, size in zip(self.planes, sizes):
            record = crossings[start : start + size]
            start += size
            k = record[:, 8].astype(np.int64)
            plane = PlaneHits(position)
            plane.append(record[:, 0:3].T.copy(), record[:, 3:6].T.copy(), current[k],
                         species[k], record[:, 6].astype(np.int8))  # fmt: skip
            planes.append(plane)
        if self.saved_ids.size:
            paths = self.paths.cpu().numpy()
            path_count = self.path_count.cpu().numpy()
            trajectories = [paths[i, : path_count[i]].copy() for i in range(self.saved_ids.size)]
        else:
            trajectories = []
        if density is None:
            density = self.density()
        return TraceResult(
            charge_density=density.cpu().numpy() if hasattr(density, "cpu") else density,
            status=status.astype(np.int8),
            electrode=electrode.astype(np.int32),
            planes=planes,
            trajectories=trajectories,
            trajectory_species=species[self.saved_ids],
            steps=int(steps.max()) if steps.size else 0,
        )


class BeamTracer:
    """Trace particles through a static electric field (``tracer.py:384-1366``).

    ``electric`` is a `StaggeredElectricField` of the mesh.  The trace runs on the device.
    ``magnetic`` -- an `AxisymmetricMagneticField` on a cylindrical mesh, or a
    `PlanarSolenoidField` on a planar one -- selects the reference's NumPy tracer's step
    in that field (``tracer.py:851-1054``; non-relativistic, no symmetry plane).  An
    imposed electric field and charge changes are not part of this build.
    """

    def __init__(
        self,
        mesh: IonOpticsMesh,
        electric: Any,
        magnetic: Any = None,
        *,
        imposed_electric: Any = None,
        step_fraction: float = 0.5,
        max_steps: int = 100_000,
        planes: Sequence[float] = (),
        save_trajectories: int = 0,
        charge_changing: Any = None,
        compiled: bool | None = None,
        integrator: str = "rk4",
        relativistic: bool = False,
        speed_of_light: float = constants.c,
        window: int = 64,
        contracted: bool = False,
    ) -> None:
        if not 0.0 < step_fraction <= 1.0:
            raise ValueError(f"step_fraction must be in (0, 1], got {step_fraction}")
        if integrator not in INTEGRATORS:
            raise ValueError(f"integrator must be one of {INTEGRATORS}, got {integrator!r}")
        unsupported = {
            "an imposed electric field": imposed_electric, "charge changes": charge_changing,
        }  # fmt: skip
        given = [name for name, value in unsupported.items() if value is not None]
        if given:
            raise NotImplementedError("this build's tracer takes no " + ", ".join(given))
        self.mesh = mesh
        self.electric = electric
        if magnetic is not None:
            from beamtracer_b200.fields import AxisymmetricMagneticField, PlanarSolenoidField

            if mesh.cylindrical and not isinstance(magnetic, AxisymmetricMagneticField):
                raise NotImplementedError("a cylindrical mesh takes an AxisymmetricMagneticField")
            if not mesh.cylindrical and not isinstance(magnetic, PlanarSolenoidField):
                raise NotImplementedError("a planar mesh takes a PlanarSolenoidField")
            if mesh.symmetry_plane:
                raise NotImplementedError("a magnetic field with a symmetry plane")
            if relativistic:
                raise NotImplementedError("a relativistic trace in a magnetic field")
        self.magnetic = magnetic
        self.step_fraction = float(step_fraction)
        self.max_steps = int(max_steps)
        self.planes = tuple(float(p) for p in planes)
        self.save_trajectories = int(save_trajectories)
        self.integrator = integrator
        self.relativistic = bool(relativistic)
        self.speed_of_light = float(speed_of_light)
        self.compiled = compiled
        self.window = int(window)
        #: the build of the trace with fused multiply-adds (`TraceEngine`)
        self.contracted = bool(contracted)
        self._capacity = (4, 1024)
        #: Sums the node charges over ranks (set by a distributed run), or None.
        self.reduce = None
        self._engine: TraceEngine | None = None

    def _inv_c2(self) -> float:
        return 1.0 / self.speed_of_light**2 if self.relativistic else 0.0

    def engine(self) -> TraceEngine:
        if self._engine is None:
            self._engine = TraceEngine(
                self.mesh, planes=self.planes, integrator=self.integrator,
                step_fraction=self.step_fraction, max_steps=self.max_steps,
                inv_c2=self._inv_c2(), save_trajectories=self.save_trajectories,
                capacity=self._capacity, window=self.window,
                magnetic=None if self.magnetic is None else self.magnetic.profile(),
                contracted=self.contracted,
            )  # fmt: skip
        self._engine.contracted = self.contracted
        return self._engine

    def trace(self, particles: BeamParticles) -> TraceResult:
        """Trace ``particles`` until they leave the mesh or hit an electrode."""
        if self.electric is None:
            raise RuntimeError("the tracer has no electric field yet")
        engine = self.engine()
        engine.load(particles)
        engine.run(self.electric.fx_device, self.electric.fy_device)
        self._capacity = engine.capacity
        density = engine.density()
        if self.reduce is not None:
            density = self.reduce(density)
        return engine.result(density)
