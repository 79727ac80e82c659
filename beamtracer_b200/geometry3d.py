"""The 3D mesh, its edge fields and the 3D beam tracer (the interfaces of the reference's
``solver/mesh3d.py`` (``IonOpticsMesh3D``), ``solver/fields3d.py``
(``StaggeredElectricField3D``) and ``solver/tracer3d.py`` (``BeamTracer3D``)).

The classification of the nodes runs on the host (the electrodes are arbitrary inside
functions); the edge fields (``bt_edge_field_3d``) and the trace
(``bt_trace_trajectories_3d``) on the device.  One mesh, no refined boxes; the beam is
given as `BeamParticles`.
"""

from __future__ import annotations

import ctypes
from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np
from scipy import constants

from beamtracer_b200 import _lib
from beamtracer_b200.mesh import FaceCondition
from beamtracer_b200.tracer import (
    _ALIVE,
    _PAUSED,
    ELECTRODE,
    INTEGRATORS,
    BeamParticles,
    PlaneHits,
    TraceResult,
    proper_velocity,
)

#: The six faces, in the order of the directions -x, +x, -y, +y, -z, +z.
FACES_3D = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")
#: The faces that can be symmetry planes.
SYMMETRY_PLANES = ("y_min", "z_min")
#: Sub-cells per cell edge of the 3D electrode lookup.
SUBCELLS_3D = 4


@dataclass(frozen=True)
class Electrode3D:
    """A solid electrode in 3D: a vectorised ``inside(x, y, z)`` test and its potential [V]."""

    inside: Callable[[np.ndarray, np.ndarray, np.ndarray], np.ndarray]
    potential: float
    name: str = ""


def _neighbour(array: np.ndarray, axis: int, step: int, fill) -> np.ndarray:
    """``out[i] = array[i + step]`` along ``axis``, ``fill`` past the ends."""
    out = np.full_like(array, fill)
    n = array.shape[axis]
    dst = [slice(None)] * array.ndim
    src = [slice(None)] * array.ndim
    dst[axis] = slice(max(-step, 0), n - max(step, 0))
    src[axis] = slice(max(step, 0), n + min(step, 0))
    out[tuple(dst)] = array[tuple(src)]
    return out


@dataclass
class IonOpticsMesh3D:
    """A uniform node mesh of ``shape`` (nx, ny, nz) from ``origin`` with spacing ``h`` and
    electrodes (``mesh3d.py:73-241``).  A node is solid in the first electrode containing it,
    fixed on a Dirichlet face, near solid when free with a solid neighbour along an axis (the
    surface's place on that edge bracketed by 8 bisections of the electrode's own test, in
    units of h / 255, never 0).  ``symmetry_planes``: the lower y and z faces that mirror the
    geometry (with a zero normal derivative)."""

    shape: tuple[int, int, int]
    origin: tuple[float, float, float]
    h: float
    electrodes: Sequence[Electrode3D] = ()
    faces: dict[str, FaceCondition] = field(default_factory=dict)
    symmetry_planes: tuple[str, ...] = ()
    cylindrical = False
    ndim = 3

    def __post_init__(self) -> None:
        self.shape = tuple(int(n) for n in self.shape)  # type: ignore[assignment]
        if len(self.shape) != 3 or min(self.shape) < 3:
            raise ValueError(f"the mesh needs 3 axes of at least 3 nodes, got {self.shape}")
        self.origin = tuple(float(o) for o in self.origin)  # type: ignore[assignment]
        self.h = float(self.h)
        if not self.h > 0.0:
            raise ValueError(f"h must be positive, got {self.h}")
        self.electrodes = tuple(self.electrodes)
        unknown = set(self.faces) - set(FACES_3D)
        if unknown:
            raise ValueError(f"unknown faces {sorted(unknown)}")
        self.faces = {face: self.faces.get(face, FaceCondition()) for face in FACES_3D}
        self.symmetry_planes = tuple(self.symmetry_planes)
        for plane in self.symmetry_planes:
            if plane not in SYMMETRY_PLANES:
                raise ValueError(f"a symmetry plane is one of {SYMMETRY_PLANES}, got {plane!r}")
            if self.faces[plane] != FaceCondition("neumann", 0.0):
                raise ValueError(f"the symmetry plane {plane} needs a zero normal derivative")
        self._classify()

    # -- geometry -----------------------------------------------------------------------

    def axis(self, a: int) -> np.ndarray:
        return self.origin[a] + self.h * np.arange(self.shape[a])

    @property
    def x(self) -> np.ndarray:
        return self.axis(0)

    @property
    def y(self) -> np.ndarray:
        return self.axis(1)

    @property
    def z(self) -> np.ndarray:
        return self.axis(2)

    @property
    def upper(self) -> tuple[float, float, float]:
        return tuple(self.origin[a] + self.h * (self.shape[a] - 1) for a in range(3))

    def nodes(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        return np.meshgrid(self.x, self.y, self.z, indexing="ij")

    def inside_solid(self, x: np.ndarray, y: np.ndarray, z: np.ndarray) -> np.ndarray:
        """The first electrode containing each point, -1 for none."""
        x, y, z = np.broadcast_arrays(*(np.asarray(a, dtype=float) for a in (x, y, z)))
        out = np.full(np.shape(x), -1, dtype=np.int64)
        for number in range(len(self.electrodes) - 1, -1, -1):
            inside = np.asarray(self.electrodes[number].inside(x, y, z), dtype=bool)
            out = np.where(inside, number, out)
        return out

    # -- classification -----------------------------------------------------------------

    def _surface(self, where, owner: np.ndarray, axis: int, step: int) -> np.ndarray:
        """The bracketed distance along (axis, step) from the nodes ``where`` to the
        surface of their neighbours' electrodes ``owner``: a bisection of [0, 255] on the
        electrode's own test, from 128, 8 steps (the result in h, never 0)."""
        start = [self.origin[a] + self.h * where[a] for a in range(3)]
        mark = np.full(where[0].shape, 128, dtype=np.int64)
        half = 128
        for _ in range(8):
            point = list(start)
            point[axis] = start[axis] + step * self.h * mark / 255.0
            hit = np.zeros(mark.shape, dtype=bool)
            for number, electrode in enumerate(self.electrodes):
                mine = owner == number
                if mine.any():
                    hit[mine] = np.asarray(electrode.inside(*(p[mine] for p in point)), bool)
            mark = np.where(hit, mark - half, mark)
            half >>= 1
            mark = mark + half
        return np.where(mark == 0, 1, mark) / 255.0

    def _classify(self) -> None:
        points = self.nodes()
        #: the first electrode of every node (-1 for none)
        self.solid = self.inside_solid(*points)
        is_solid = self.solid >= 0
        potentials = np.array([e.potential for e in self.electrodes] + [0.0])
        fixed = is_solid.copy()
        value = np.where(is_solid, potentials[self.solid], 0.0)
        for number, face in enumerate(FACES_3D):
            condition = self.faces[face]
            if condition.kind != "dirichlet":
                continue
            axis, upper = divmod(number, 2)
            index = [slice(None)] * 3
            index[axis] = slice(-1, None) if upper else slice(0, 1)
            at = tuple(index)
            free = ~is_solid[at]
            value[at] = np.where(free, condition.evaluate(*(p[at] for p in points)), value[at])
            fixed[at] |= free
        self.fixed = fixed
        self.fixed_value = value
        self.distance = np.ones((6, *self.shape))
        self.near_solid = np.zeros(self.shape, dtype=bool)
        for d in range(6):
            axis, step = divmod(d, 2)[0], (-1, 1)[d % 2]
            neighbour = _neighbour(self.solid, axis, step, -1)
            near = ~is_solid & (neighbour >= 0)
            self.near_solid |= near
            where = np.nonzero(near)
            self.distance[(d, *where)] = self._surface(where, neighbour[where], axis, step)


class StaggeredElectricField3D:
    """The electric field of a potential on the edges of a 3D mesh (``fields3d.py:66-122``):
    ``E_x`` on the (nx + 1, ny, nz) edges along x, ``E_y`` (nx, ny + 1, nz), ``E_z``
    (nx, ny, nz + 1), by the 2D edge rule along every line of nodes (built on the device,
    ``bt_edge_field_3d``); ``extrapolation`` per face (`FACES_3D`), ``"symmetric"`` or
    ``"extrapolate"`` (default: symmetric on the symmetry planes).  ``fx_device`` etc. are
    the device arrays, ``fx`` etc. host copies."""

    def __init__(self, mesh: IonOpticsMesh3D, potential,
                 extrapolation: Sequence[str] | None = None) -> None:  # fmt: skip
        import torch

        if extrapolation is None:
            extrapolation = ["extrapolate"] * 6
            for plane in mesh.symmetry_planes:
                extrapolation[FACES_3D.index(plane)] = "symmetric"
        for face in extrapolation:
            if face not in ("extrapolate", "symmetric"):
                raise ValueError(f"unknown face extrapolation {face!r}")
        self.mesh = mesh
        self.extrapolation = tuple(extrapolation)
        nx, ny, nz = mesh.shape
        dev = "cuda"
        if _lib.is_device_array(potential):
            phi = potential
        else:
            phi = torch.from_numpy(np.ascontiguousarray(potential, dtype=np.float64)).to(dev)
        if tuple(phi.shape) != (nx, ny, nz):
            raise ValueError("the potential needs the mesh's shape")
        solid = torch.from_numpy(np.ascontiguousarray(mesh.solid, dtype=np.int32)).to(dev)
        near = torch.from_numpy(np.ascontiguousarray(mesh.near_solid, dtype=np.uint8)).to(dev)
        distance = torch.from_numpy(np.ascontiguousarray(mesh.distance)).to(dev)
        f64 = dict(dtype=torch.float64, device=dev)
        self.fx_device = torch.empty((nx + 1, ny, nz), **f64)
        self.fy_device = torch.empty((nx, ny + 1, nz), **f64)
        self.fz_device = torch.empty((nx, ny, nz + 1), **f64)
        faces = (ctypes.c_int32 * 6)(*[int(f == "symmetric") for f in self.extrapolation])
        d = _lib.dptr
        _lib.check(_lib.lib().bt_edge_field_3d(
            _lib.context().handle, d(phi), d(solid), d(near), d(distance), nx, ny, nz,
            float(mesh.h), faces, d(self.fx_device), d(self.fy_device), d(self.fz_device)))  # fmt: skip

    @property
    def fx(self) -> np.ndarray:
        return self.fx_device.cpu().numpy()

    @property
    def fy(self) -> np.ndarray:
        return self.fy_device.cpu().numpy()

    @property
    def fz(self) -> np.ndarray:
        return self.fz_device.cpu().numpy()

    def __call__(self, x, y, z) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """``(E_x, E_y, E_z)`` [V/m] at the points, trilinear with the cell clamped."""
        mesh = self.mesh
        s = (np.asarray(x, dtype=float) - mesh.origin[0]) / mesh.h
        t = (np.asarray(y, dtype=float) - mesh.origin[1]) / mesh.h
        u = (np.asarray(z, dtype=float) - mesh.origin[2]) / mesh.h
        return (_trilinear(self.fx, s + 0.5, t, u), _trilinear(self.fy, s, t + 0.5, u),
                _trilinear(self.fz, s, t, u + 0.5))  # fmt: skip


def _trilinear(values: np.ndarray, s, t, u) -> np.ndarray:
    """``values`` at fractional indices (s, t, u), the cell clamped to the array."""
    n = values.shape
    i = np.clip(np.floor(s).astype(np.int64), 0, n[0] - 2)
    j = np.clip(np.floor(t).astype(np.int64), 0, n[1] - 2)
    k = np.clip(np.floor(u).astype(np.int64), 0, n[2] - 2)
    a, b, c = s - i, t - j, u - k
    out = np.zeros(np.shape(s))
    for di, wi in ((0, 1.0 - a), (1, a)):
        for dj, wj in ((0, 1.0 - b), (1, b)):
            for dk, wk in ((0, 1.0 - c), (1, c)):
                out += wi * wj * wk * values[i + di, j + dj, k + dk]
    return out


class BeamTracer3D:
    """Trace particles through the fields of a 3D mesh (``tracer3d.py:140-484``):
    ``electric`` a `StaggeredElectricField3D`, ``magnetic`` an optional (3, nx, ny, nz) B [T]
    on the nodes; ``planes`` the diagnostic planes x = const; ``save_trajectories`` keeps
    every n-th path; ``integrator`` "rk4" or "boris"; ``relativistic`` advances proper
    velocities; ``deposit_current`` also deposits the current density.  The trace runs on
    the device (``bt_trace_trajectories_3d``); trajectories stopped in a sub-cell an
    electrode surface cuts are tested here with the electrodes' own test and resumed."""

    def __init__(self, mesh: IonOpticsMesh3D, electric: StaggeredElectricField3D | None = None,
                 magnetic: np.ndarray | None = None, *, step_fraction: float = 0.5,
                 max_steps: int = 100_000, planes: Sequence[float] = (),
                 save_trajectories: int = 0, integrator: str = "rk4",
                 relativistic: bool = False, speed_of_light: float = constants.c,
                 deposit_current: bool = False, window: int = 0) -> None:  # fmt: skip
        if not 0.0 < step_fraction <= 1.0:
            raise ValueError(f"step_fraction must be in (0, 1], got {step_fraction}")
        if integrator not in INTEGRATORS:
            raise ValueError(f"integrator must be one of {INTEGRATORS}, got {integrator!r}")
        if magnetic is not None and np.shape(magnetic) != (3, *mesh.shape):
            raise ValueError(f"magnetic must be (3, *mesh.shape) = {(3, *mesh.shape)}, "
                             f"got {np.shape(magnetic)}")  # fmt: skip
        self.mesh = mesh
        self.electric = electric
        self.magnetic = None if magnetic is None else np.ascontiguousarray(magnetic, dtype=float)
        self.step_fraction = float(step_fraction)
        self.max_steps = int(max_steps)
        self.planes = tuple(float(p) for p in planes)
        self.save_trajectories = int(save_trajectories)
        self.integrator = integrator
        self.relativistic = bool(relativistic)
        self.speed_of_light = float(speed_of_light)
        self.deposit_current = bool(deposit_current)
        self.window = int(window)
        self._capacity = (4, 1024)
        self._lookup: tuple[np.ndarray, np.ndarray] | None = None
        #: the kernel (the device's; a test may put the oracle's here)
        self.kernel: Callable[..., None] | None = None

    # -- geometry -------------------------------------------------------------------------

    def mesh_points(self, x: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """The mesh coordinates of Cartesian points (3, N): mirrored to a symmetry plane's
        side."""
        mesh = self.mesh
        px, py, pz = (np.asarray(x[a], dtype=float) for a in range(3))
        if "y_min" in mesh.symmetry_planes:
            py = mesh.origin[1] + np.abs(py - mesh.origin[1])
        if "z_min" in mesh.symmetry_planes:
            pz = mesh.origin[2] + np.abs(pz - mesh.origin[2])
        return px, py, pz

    def electrode_lookup(self) -> tuple[np.ndarray, np.ndarray]:
        """``cells`` (nx - 1, ny - 1, nz - 1): the number of every cell with an electrode
        node or a node next to one (-1 for the others); ``subcells``: for each, the
        electrode holding all eight corners and the centre of every one of its
        ``SUBCELLS_3D**3`` sub-cells, -1 for none, -2 where they disagree
        (``tracer3d.py:211-286``)."""
        if self._lookup is not None:
            return self._lookup
        mesh, n = self.mesh, SUBCELLS_3D
        touch = (mesh.solid >= 0) | mesh.near_solid
        shape = tuple(s - 1 for s in mesh.shape)
        near = np.zeros(shape, dtype=bool)
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    near |= touch[di : di + shape[0], dj : dj + shape[1], dk : dk + shape[2]]
        cells = np.full(shape, -1, dtype=np.int64)
        ci, cj, ck = np.nonzero(near)
        if not mesh.electrodes or not ci.size:
            self._lookup = (cells, np.full(1, -1, dtype=np.int64))
            return self._lookup
        cells[ci, cj, ck] = np.arange(ci.size, dtype=np.int64)

        def sample(fraction: np.ndarray) -> np.ndarray:
            m = fraction.size
            px = mesh.origin[0] + mesh.h * (ci[:, None, None, None] + fraction[None, :, None, None])
            py = mesh.origin[1] + mesh.h * (cj[:, None, None, None] + fraction[None, None, :, None])
            pz = mesh.origin[2] + mesh.h * (ck[:, None, None, None] + fraction[None, None, None, :])
            px, py, pz = np.broadcast_arrays(px, py, pz)
            return mesh.inside_solid(px.ravel(), py.ravel(), pz.ravel()).reshape((ci.size, m, m, m))

        corner = sample(np.arange(n + 1) / n)
        centre = sample((np.arange(n) + 0.5) / n)
        same = np.ones(centre.shape, dtype=bool)
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    same &= corner[:, di : di + n, dj : dj + n, dk : dk + n] == centre
        self._lookup = (cells, np.where(same, centre, -2).astype(np.int64).ravel())
        return self._lookup

    def _finalize(self, charge: np.ndarray) -> np.ndarray:
        """Node charges over node volumes: h^3, halved on each face."""
        density = charge / self.mesh.h**3
        for axis in range(3):
            index: list[Any] = [slice(None)] * 3
            for end in (0, -1):
                index[axis] = end
                density[tuple(index)] *= 2.0
        return density

    # -- tracing ----------------------------------------------------------------------------

    def trace(self, particles: BeamParticles) -> TraceResult:
        """Trace ``particles`` until they leave the mesh or hit an electrode
        (``tracer3d.py:336-484``); a trace whose crossings or kept paths overflow their
        buffers runs again with larger ones."""
        field = self.electric
        if field is None:
            raise RuntimeError("the tracer has no electric field yet")
        mesh = self.mesh
        n = len(particles)
        x = np.array(particles.position, dtype=float, order="C")
        v = np.array(particles.velocity, dtype=float, order="C")
        inv_c2 = 0.0
        if self.relativistic:
            v = np.ascontiguousarray(proper_velocity(v, self.speed_of_light))
            inv_c2 = 1.0 / self.speed_of_light**2
        qm = np.ascontiguousarray(particles.charge / particles.mass, dtype=float)
        current = particles.current.astype(float)
        dq = np.ascontiguousarray(np.sign(particles.charge) * np.abs(current))
        species = particles.species
        status = np.full(n, _ALIVE, dtype=np.int64)
        electrode = np.full(n, -1, dtype=np.int64)
        steps = np.zeros(n, dtype=np.int64)
        if mesh.electrodes and n:
            hit = mesh.inside_solid(*self.mesh_points(x))
            dead = hit >= 0
            status[dead] = ELECTRODE
            electrode[dead] = hit[dead]
        start = np.flatnonzero(status == _ALIVE).astype(np.int64)
        save = self.save_trajectories
        saved = np.arange(0, n, save) if save else np.zeros(0, int)
        path_slot = np.full(n, -1, dtype=np.int64)
        path_slot[saved] = np.arange(saved.size)
        first = np.stack(self.mesh_points(x[:, saved]))
        cells, subcells = self.electrode_lookup()
        nx, ny, nz = mesh.shape
        nodes = nx * ny * nz
        patch_int = np.array([[nx, ny, nz, 0, 0, 0, nodes, 0]], dtype=np.int64)
        patch_real = np.array([[*mesh.origin, mesh.h, *mesh.origin, *mesh.upper]])
        if self.kernel is None:
            from beamtracer_b200.kernels import KERNELS

            kernel = lambda *a: KERNELS["trace_trajectories_3d"](*a, window=self.window)  # noqa: E731
            fields = [f.reshape(-1) for f in (field.fx_device, field.fy_device, field.fz_device)]
        else:
            kernel = self.kernel
            fields = [np.ascontiguousarray(f).ravel() for f in (field.fx, field.fy, field.fz)]
        has_b = int(self.magnetic is not None)
        magnetic = self.magnetic if has_b else np.zeros((3, 2, 2, 2))
        has_j = int(self.deposit_current)
        planes = np.array(self.planes or (np.nan,), dtype=float)
        mirror_y = int("y_min" in mesh.symmetry_planes)
        mirror_z = int("z_min" in mesh.symmetry_planes)
        # the device path keeps every array on the device across the pause rounds (the
        # oracle's kernel takes host arrays)
        on_device = self.kernel is None
        if on_device:
            import torch

            put = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
            get = lambda a: a.cpu().numpy()  # noqa: E731
        else:
            put = get = lambda a: a  # noqa: E731
        x, v, qm, dq, steps, status, electrode = map(put, (x, v, qm, dq, steps, status, electrode))
        start, path_slot, cells, subcells, planes, magnetic = map(
            put, (start, path_slot, cells, subcells, planes, magnetic))  # fmt: skip
        patch_int, patch_real = put(patch_int), put(patch_real)
        initial = [a.clone() if on_device else a.copy() for a in (x, v, status, electrode)]
        while True:
            capacity, path_capacity = self._capacity
            charge = put(np.zeros((1, nodes)))
            current_nodes = put(np.zeros((1, 3 * nodes) if has_j else (1, 1)))
            hits = put(np.zeros((n, len(planes), capacity, 8)))
            counts = put(np.zeros((n, len(planes)), dtype=np.int64))
            first_paths = np.zeros((max(saved.size, 1), path_capacity, 3))
            first_paths[: saved.size, 0] = first.T
            paths = put(first_paths)
            path_count = put(np.ones(max(saved.size, 1), dtype=np.int64))
            active = start
            while len(active):
                kernel(active, x, v, qm, dq, steps, status, electrode, *fields, patch_int,
                       patch_real, magnetic, has_b, *mesh.origin, mesh.h, *mesh.upper, mirror_y,
                       mirror_z, INTEGRATORS.index(self.integrator), self.step_fraction,
                       self.max_steps, cells, subcells, SUBCELLS_3D, planes, hits, counts,
                       path_slot, paths, path_count, 1, charge, has_j, current_nodes, inv_c2)  # fmt: skip
                paused = active[status[active] == _PAUSED]
                if not len(paused):
                    break
                hit = mesh.inside_solid(*self.mesh_points(get(x[:, paused])))
                inside = put(hit >= 0)
                status[paused[inside]] = ELECTRODE
                electrode[paused[inside]] = put(hit)[inside]
                active = paused[~inside]
                status[active] = _ALIVE
            most = int(counts.max()) if len(counts) else 0
            longest = int(path_count.max())
            if most <= capacity and longest <= path_capacity:
                break
            self._capacity = (max(capacity, most), max(path_capacity, longest))
            x, v, status, electrode = (a.clone() if on_device else a.copy() for a in initial)
            steps[:] = 0
        x, v, steps, status, electrode = map(get, (x, v, steps, status, electrode))
        charge, current_nodes, hits, counts, paths, path_count = map(
            get, (charge, current_nodes, hits, counts, paths, path_count))  # fmt: skip
        #: the steps each trajectory took in the last trace
        self.steps = steps
        current_density = None
        if has_j:
            current_density = np.stack([self._finalize(c) for c in
                                        current_nodes[0].reshape(3, *mesh.shape)])  # fmt: skip
        hit_planes = []
        slots = np.arange(capacity)
        for p, position in enumerate(self.planes):
            k, c = np.nonzero(slots[None, :] < counts[:, p, None])
            record = hits[k, p, c]
            order = np.lexsort((k, record[:, 7]))  # by step, then trajectory
            k, record = k[order], record[order]
            plane = PlaneHits(position)
            plane.append(record[:, 0:3].T.copy(), record[:, 3:6].T.copy(), current[k],
                         species[k], record[:, 6].astype(np.int8))  # fmt: skip
            hit_planes.append(plane)
        return TraceResult(
            charge_density=self._finalize(charge[0].reshape(mesh.shape)),
            status=status.astype(np.int8), electrode=electrode.astype(np.int32),
            planes=hit_planes,
            trajectories=[paths[i, : path_count[i]].copy() for i in range(saved.size)],
            trajectory_species=species[saved], steps=int(steps.max()) if n else 0,
            current_density=current_density,
        )  # fmt: skip
