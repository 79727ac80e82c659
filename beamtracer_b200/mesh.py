"""The ion-optics mesh: node classes, electrode potentials and surface distances.

The interface of the reference's ``solver/mesh.py`` (``IonOpticsMesh``, ``Electrode``,
``FaceCondition``; ``mesh.py:35-377``): a uniform node grid of spacing ``h`` in ``(x, y)``
or, for a cylindrical geometry, ``(x, r)`` with the axis at ``r = 0``, optionally with a
graded ``x`` axis.  A node is solid (inside an electrode, held at its potential), fixed on a
Dirichlet face, near-solid (free with a solid neighbour along ``x`` or ``y``, its distance to
the surface bracketed in eight bisection steps in units of 1/255 of the edge,
``mesh.py:127-156``) or free.  The classification runs once per mesh on the host -- the
electrodes' ``inside`` tests are Python callables -- and the arrays it makes are the inputs
of the device field solve, edge field and tracer.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np

InsideFunction = Callable[[np.ndarray, np.ndarray], np.ndarray]

#: The four faces: x min, x max, y (or r) min, y (or r) max.
FACES = ("x_min", "x_max", "y_min", "y_max")

#: The neighbour directions, (axis, step) for -x, +x, -y, +y.
DIRECTIONS = ((0, -1), (0, 1), (1, -1), (1, 1))


@dataclass(frozen=True)
class Electrode:
    """A solid electrode: a vectorised ``inside(x, y)`` test and its potential [V]."""

    inside: InsideFunction
    potential: float
    name: str = ""


@dataclass(frozen=True)
class FaceCondition:
    """One face's condition: ``"dirichlet"`` (``value`` the potential [V], a number or a
    function of ``(x, y)``) or ``"neumann"`` (``value`` the outward normal derivative [V/m])."""

    kind: str = "neumann"
    value: float | Callable[..., np.ndarray] = 0.0

    def __post_init__(self) -> None:
        if self.kind not in ("dirichlet", "neumann"):
            raise ValueError(f"unknown face condition {self.kind!r}")

    def evaluate(self, x: np.ndarray, *rest: np.ndarray) -> np.ndarray:
        """The face value at the points."""
        if callable(self.value):
            return np.broadcast_to(np.asarray(self.value(x, *rest), dtype=float), x.shape)
        return np.full(x.shape, float(self.value))


@dataclass
class IonOpticsMesh:
    """A 2D node mesh with electrodes, planar or cylindrical (``mesh.py:90-377``).

    ``shape`` ``(nx, ny)`` nodes, ``origin`` the node ``(0, 0)``, ``h`` the spacing (along
    ``y`` only when ``x_nodes`` grades the ``x`` axis), ``faces`` a `FaceCondition` per face
    (Neumann by default).  In cylindrical geometry the ``y_min`` face is the axis at
    ``r = 0``; a planar mesh with ``symmetry_plane`` mirrors the geometry at ``y_min``.
    """

    shape: tuple[int, int]
    origin: tuple[float, float]
    h: float
    geometry: str = "cylindrical"
    electrodes: Sequence[Electrode] = ()
    faces: dict[str, FaceCondition] = field(default_factory=dict)
    patch: bool = False
    symmetry_plane: bool = False
    x_nodes: Any = None
    logical_x0: float | None = None

    def __post_init__(self) -> None:
        if self.geometry not in ("planar", "cylindrical"):
            raise ValueError(
                f"geometry must be 'planar' or 'cylindrical', got {self.geometry!r}"
            )
        self.shape = (int(self.shape[0]), int(self.shape[1]))
        if min(self.shape) < 3:
            raise ValueError(f"the mesh needs at least 3 nodes per axis, got {self.shape}")
        self.origin = (float(self.origin[0]), float(self.origin[1]))
        self.h = float(self.h)
        if not self.h > 0.0:
            raise ValueError(f"h must be positive, got {self.h}")
        if self.x_nodes is not None:
            nodes = np.array(self.x_nodes, dtype=float)
            if nodes.shape != (self.shape[0],):
                raise ValueError(
                    f"x_nodes needs the {self.shape[0]} positions of the nodes along x, "
                    f"got shape {nodes.shape}"
                )
            if not np.all(np.diff(nodes) > 0.0):
                raise ValueError("x_nodes must increase strictly")
            if abs(nodes[0] - self.origin[0]) > 1e-12 * max(1.0, abs(nodes[0])):
                raise ValueError(
                    f"the first of x_nodes ({nodes[0]}) must be the origin's x "
                    f"({self.origin[0]})"
                )
            nodes.setflags(write=False)
            self.x_nodes = nodes
        self.logical_x0 = float(self.origin[0] if self.logical_x0 is None else self.logical_x0)
        self.electrodes = tuple(self.electrodes)
        unknown = set(self.faces) - set(FACES)
        if unknown:
            raise ValueError(f"unknown faces {sorted(unknown)}")
        self.faces = {face: self.faces.get(face, FaceCondition()) for face in FACES}
        if self.cylindrical and not self.patch:
            if abs(self.origin[1]) > 1e-12 * max(1.0, self.h):
                raise ValueError("a cylindrical mesh must start on the axis (r = 0)")
            if self.faces["y_min"] != FaceCondition("neumann", 0.0):
                raise ValueError("the y_min face of a cylindrical mesh is the symmetry axis")
        if self.symmetry_plane:
            if self.cylindrical:
                raise ValueError("a symmetry plane needs planar geometry")
            if self.faces["y_min"] != FaceCondition("neumann", 0.0):
                raise ValueError(
                    "the y_min face of a mesh with a symmetry plane must have a zero "
                    "normal derivative"
                )
        self._classify()

    # -- geometry -------------------------------------------------------------------------

    @property
    def cylindrical(self) -> bool:
        return self.geometry == "cylindrical"

    @property
    def graded(self) -> bool:
        return self.x_nodes is not None

    @property
    def x(self) -> np.ndarray:
        """The node coordinates along ``x``."""
        if self.x_nodes is not None:
            return self.x_nodes
        return self.origin[0] + self.h * np.arange(self.shape[0])

    @property
    def y(self) -> np.ndarray:
        """The node coordinates along ``y`` (the radius in cylindrical geometry)."""
        return self.origin[1] + self.h * np.arange(self.shape[1])

    @property
    def dx(self) -> np.ndarray:
        """The ``nx - 1`` edge lengths along ``x``."""
        if self.x_nodes is not None:
            return np.diff(self.x_nodes)
        return np.full(self.shape[0] - 1, self.h)

    @property
    def upper(self) -> tuple[float, float]:
        return (float(self.x[-1]), self.origin[1] + self.h * (self.shape[1] - 1))

    @property
    def logical_origin(self) -> tuple[float, float]:
        """The uniform coordinates of node ``(0, 0)`` (the kernels locate points by them)."""
        return (float(self.logical_x0), self.origin[1])

    @property
    def logical_upper(self) -> tuple[float, float]:
        if self.x_nodes is None:
            return self.upper
        return (float(self.logical_x0) + self.h * (self.shape[0] - 1), self.upper[1])

    def index_x(self, x: Any) -> np.ndarray:
        """The fractional node index of positions ``x`` (linear between graded nodes)."""
        x = np.asarray(x, dtype=float)
        if self.x_nodes is None:
            return (x - self.origin[0]) / self.h
        nodes = self.x_nodes
        i = np.clip(np.searchsorted(nodes, x, side="right") - 1, 0, nodes.size - 2)
        return i + (x - nodes[i]) / (nodes[i + 1] - nodes[i])

    def position_x(self, index: Any) -> np.ndarray:
        """The position along ``x`` of a fractional node index."""
        index = np.asarray(index, dtype=float)
        if self.x_nodes is None:
            return self.origin[0] + self.h * index
        nodes = self.x_nodes
        i = np.clip(np.floor(index).astype(np.int64), 0, nodes.size - 2)
        return nodes[i] + (index - i) * (nodes[i + 1] - nodes[i])

    def logical_x(self, x: Any) -> np.ndarray:
        """The uniform coordinate ``logical_x0 + h * index_x(x)`` (``x`` itself if uniform)."""
        if self.x_nodes is None:
            return np.asarray(x, dtype=float)
        return float(self.logical_x0) + self.h * self.index_x(x)

    def spacing_at(self, x: Any) -> Any:
        """The smaller edge of the cells at ``x``: ``h``, or less along a graded ``x``."""
        if self.x_nodes is None:
            return self.h
        i = np.clip(np.floor(self.index_x(x)).astype(np.int64), 0, self.shape[0] - 2)
        return np.minimum(self.dx[i], self.h)

    def nodes(self) -> tuple[np.ndarray, np.ndarray]:
        """The node coordinates as two ``(nx, ny)`` arrays."""
        return np.meshgrid(self.x, self.y, indexing="ij")

    def inside_solid(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        """The index of the electrode containing each point (the first listed wins), or -1."""
        x = np.asarray(x, dtype=float)
        y = np.asarray(y, dtype=float)
        shape = np.broadcast(x, y).shape
        xb, yb = np.broadcast_to(x, shape), np.broadcast_to(y, shape)
        out = np.full(shape, -1, dtype=np.int32)
        for number, electrode in enumerate(self.electrodes):
            open_ = out < 0
            if not open_.any():
                break
            hit = np.zeros(shape, dtype=bool)
            hit[open_] = np.asarray(electrode.inside(xb[open_], yb[open_]), dtype=bool)
            out[hit] = number
        return out

    # -- classification -----------------------------------------------------------------

    def _neighbour_solid(self, axis: int, step: int) -> np.ndarray:
        """The electrode index of every node's neighbour in one direction (-1: none)."""
        out = np.full(self.shape, -1, dtype=np.int32)
        src = self.solid
        if axis == 0:
            if step > 0:
                out[:-1] = src[1:]
            else:
                out[1:] = src[:-1]
        elif step > 0:
            out[:, :-1] = src[:, 1:]
        else:
            out[:, 1:] = src[:, :-1]
        return out

    def _bracket(self, i, j, owner, axis: int, step: int) -> np.ndarray:
        """The fraction of the edge from nodes ``(i, j)`` towards their solid neighbours
        where the surface lies: eight bisections of the owner electrode's inside test, on a
        scale of 255 steps (never zero)."""
        x0 = self.x[i]
        y0 = self.origin[1] + self.h * j
        length = self.h if axis == 1 else self.dx[i if step > 0 else i - 1]
        code = np.full(i.shape, 128, dtype=np.int64)
        bit = 128
        for _ in range(8):
            offset = step * length * code / 255.0
            px = x0 + offset if axis == 0 else x0
            py = y0 + offset if axis == 1 else y0
            inside = np.zeros(i.shape, dtype=bool)
            for number, electrode in enumerate(self.electrodes):
                mine = owner == number
                if mine.any():
                    inside[mine] = np.asarray(electrode.inside(px[mine], py[mine]), dtype=bool)
            code = np.where(inside, code - bit, code)
            bit >>= 1
            code = code + bit
        code = np.where(code == 0, 1, code)
        return code / 255.0

    def _classify_on_device(self):
        """``(solid, near, distance)`` sampled on the device (``bt_classify_mesh``) when a
        CUDA device is present and every electrode is a configuration shape; else None."""
        if not self.electrodes:
            return None
        try:
            import torch
        except ImportError:  # pragma: no cover
            return None
        if not torch.cuda.is_available():
            return None
        from beamtracer_b200.shapes import shape_table

        table = shape_table(self)
        if table is None:
            return None
        import ctypes

        from beamtracer_b200 import _lib

        nx, ny = self.shape
        kinds, offsets, params = (torch.from_numpy(a).cuda() for a in table)
        x = torch.from_numpy(np.array(self.x, dtype=np.float64)).cuda()
        dx = torch.from_numpy(np.array(self.dx, dtype=np.float64)).cuda()
        solid = torch.empty((nx, ny), dtype=torch.int32, device="cuda")
        near = torch.empty((nx, ny), dtype=torch.uint8, device="cuda")
        distance = torch.empty((4, nx, ny), dtype=torch.float64, device="cuda")
        shapes = _lib.ShapesDesc(len(table[0]), _lib.dptr(kinds), _lib.dptr(offsets),
                                 _lib.dptr(params))  # fmt: skip
        ctx = _lib.context()
        _lib.check(_lib.lib().bt_classify_mesh(
            ctx.handle, ctypes.byref(shapes), nx, ny, _lib.dptr(x), _lib.dptr(dx),
            float(self.origin[1]), float(self.h), _lib.dptr(solid), _lib.dptr(near),
            _lib.dptr(distance)))  # fmt: skip
        return solid.cpu().numpy(), near.cpu().numpy().astype(bool), distance.cpu().numpy()

    def _classify(self) -> None:
        nx, ny = self.shape
        xn, yn = self.nodes()
        device = self._classify_on_device()
        #: The electrode index of every node (-1: none).
        self.solid = self.inside_solid(xn, yn) if device is None else device[0]
        solid = self.solid >= 0
        potentials = np.array([e.potential for e in self.electrodes] + [0.0])
        fixed = solid.copy()
        value = np.where(solid, potentials[self.solid], 0.0)
        face_nodes = {
            "x_min": (slice(0, 1), slice(None)),
            "x_max": (slice(nx - 1, nx), slice(None)),
            "y_min": (slice(None), slice(0, 1)),
            "y_max": (slice(None), slice(ny - 1, ny)),
        }
        for face in FACES:
            condition = self.faces[face]
            if condition.kind != "dirichlet":
                continue
            index = face_nodes[face]
            open_ = ~solid[index]
            value[index] = np.where(open_, condition.evaluate(xn[index], yn[index]), value[index])
            fixed[index] |= open_
        #: Nodes with a prescribed potential (electrodes and Dirichlet faces).
        self.fixed = fixed
        #: Their potential (0 elsewhere).
        self.fixed_value = value
        if device is not None:
            self.near_solid, self.distance = device[1], device[2]
            return
        #: The fraction of the edge to the surface along -x, +x, -y, +y (1: no surface).
        self.distance = np.ones((4, nx, ny))
        #: Free nodes with an electrode neighbour.
        self.near_solid = np.zeros((nx, ny), dtype=bool)
        for d, (axis, step) in enumerate(DIRECTIONS):
            neighbour = self._neighbour_solid(axis, step)
            near = ~solid & (neighbour >= 0)
            if not near.any():
                continue
            self.near_solid |= near
            i, j = np.nonzero(near)
            self.distance[d, i, j] = self._bracket(i, j, neighbour[i, j], axis, step)
