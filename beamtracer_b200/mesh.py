"""The ion-optics mesh: node classes, electrode potentials and surface distances.

The interface of the reference's ``solver/mesh.py`` (``IonOpticsMesh``, ``Electrode``,
``FaceCondition``; ``mesh.py:35-377``) over a design of its own: a `NodeAxis` holds the
node positions along ``x`` (uniform, or graded by given positions) and answers the
coordinate questions the field solve, the edge field and the tracer ask of it; the node
classes are set once per mesh.

A node is solid (inside an electrode, held at its potential; the first listed electrode
owns a node inside several), fixed on a Dirichlet face, near-solid (free with a solid
neighbour along ``x`` or ``y``) or free.  The surface between a near-solid node and its
solid neighbour is located along their edge as an 8-bit fraction ``s / 255`` (never 0):
the bits decided from the most significant down, each by whether the owner electrode
contains the trial point (``mesh.py:127-156`` states the same bracket).  Configuration
shapes are classified on the device (``bt_classify_mesh``) when a GPU is present; any other
``inside`` callable, or ``classify_on_device=False``, classifies on the host.
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

#: Bits of the surface fraction along an edge (in units of 1 / (2^bits - 1)).
DISTANCE_BITS = 8


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


class NodeAxis:
    """Node positions along one axis: ``start + step * k`` for ``k < count``, or the given
    strictly increasing ``positions`` (a graded axis, ``step`` then only its nominal
    spacing).  Fractional indices are linear within an edge and continue the first or last
    edge beyond the nodes."""

    def __init__(self, start: float, step: float, count: int,
                 positions: np.ndarray | None = None) -> None:  # fmt: skip
        self.start, self.step, self.count = float(start), float(step), int(count)
        self.positions = positions

    @property
    def graded(self) -> bool:
        return self.positions is not None

    def nodes(self) -> np.ndarray:
        if self.positions is not None:
            return self.positions
        return self.start + self.step * np.arange(self.count)

    def edges(self) -> np.ndarray:
        if self.positions is not None:
            return np.diff(self.positions)
        return np.full(self.count - 1, self.step)

    def last(self) -> float:
        if self.positions is not None:
            return float(self.positions[-1])
        return self.start + self.step * (self.count - 1)

    def _edge_of(self, k: np.ndarray) -> np.ndarray:
        return np.clip(k, 0, self.count - 2)

    def fraction(self, x: Any) -> np.ndarray:
        """The fractional index of positions ``x``."""
        x = np.asarray(x, dtype=float)
        if self.positions is None:
            return (x - self.start) / self.step
        p = self.positions
        k = self._edge_of(np.searchsorted(p, x, side="right") - 1)
        return k + (x - p[k]) / (p[k + 1] - p[k])

    def position(self, index: Any) -> np.ndarray:
        """The position of fractional indices (`fraction` inverted)."""
        index = np.asarray(index, dtype=float)
        if self.positions is None:
            return self.start + self.step * index
        p = self.positions
        k = self._edge_of(np.floor(index).astype(np.int64))
        return p[k] + (index - k) * (p[k + 1] - p[k])


def _graded_positions(x_nodes: Any, nx: int, x0: float) -> np.ndarray:
    """The validated, read-only node positions of a graded ``x`` axis."""
    nodes = np.array(x_nodes, dtype=float)
    problems = (
        (nodes.shape != (nx,),
         f"x_nodes needs the {nx} positions of the nodes along x, got shape {nodes.shape}"),
        (nodes.shape == (nx,) and not np.all(np.diff(nodes) > 0.0),
         "x_nodes must increase strictly"),
        (nodes.shape == (nx,) and abs(nodes[0] - x0) > 1e-12 * max(1.0, abs(nodes[0])),
         f"the first of x_nodes ({nodes[0] if nodes.size else None}) must be the origin's "
         f"x ({x0})"),
    )  # fmt: skip
    for failed, message in problems:
        if failed:
            raise ValueError(message)
    nodes.setflags(write=False)
    return nodes


@dataclass
class IonOpticsMesh:
    """A 2D node mesh with electrodes, planar or cylindrical (``mesh.py:90-377``).

    ``shape`` ``(nx, ny)`` nodes, ``origin`` the node ``(0, 0)``, ``h`` the spacing (along
    ``y`` only when ``x_nodes`` grades the ``x`` axis), ``faces`` a `FaceCondition` per face
    (Neumann by default).  In cylindrical geometry the ``y_min`` face is the axis at
    ``r = 0``; a planar mesh with ``symmetry_plane`` mirrors the geometry at ``y_min``.
    ``classify_on_device``: None classifies configuration shapes on a present GPU, False
    always on the host.
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
    classify_on_device: bool | None = None

    def __post_init__(self) -> None:
        self._validate()
        self._axis = NodeAxis(self.origin[0], self.h, self.shape[0], self.x_nodes)
        self._classify()

    def _validate(self) -> None:
        if self.geometry not in ("planar", "cylindrical"):
            raise ValueError(f"geometry must be 'planar' or 'cylindrical', got {self.geometry!r}")
        nx, ny = self.shape = (int(self.shape[0]), int(self.shape[1]))
        if min(nx, ny) < 3:
            raise ValueError(f"the mesh needs at least 3 nodes per axis, got {self.shape}")
        self.origin = (float(self.origin[0]), float(self.origin[1]))
        self.h = float(self.h)
        if not self.h > 0.0:
            raise ValueError(f"h must be positive, got {self.h}")
        if self.x_nodes is not None:
            self.x_nodes = _graded_positions(self.x_nodes, nx, self.origin[0])
        if self.logical_x0 is None:
            self.logical_x0 = self.origin[0]
        self.logical_x0 = float(self.logical_x0)
        self.electrodes = tuple(self.electrodes)
        unknown = sorted(set(self.faces) - set(FACES))
        if unknown:
            raise ValueError(f"unknown faces {unknown}")
        self.faces = {face: self.faces.get(face, FaceCondition()) for face in FACES}
        mirror = FaceCondition("neumann", 0.0)
        if self.cylindrical and not self.patch:
            if abs(self.origin[1]) > 1e-12 * max(1.0, self.h):
                raise ValueError("a cylindrical mesh must start on the axis (r = 0)")
            if self.faces["y_min"] != mirror:
                raise ValueError("the y_min face of a cylindrical mesh is the symmetry axis")
        if self.symmetry_plane:
            if self.cylindrical:
                raise ValueError("a symmetry plane needs planar geometry")
            if self.faces["y_min"] != mirror:
                raise ValueError("the y_min face of a mesh with a symmetry plane must have a "
                                 "zero normal derivative")  # fmt: skip

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
        return self._axis.nodes()

    @property
    def y(self) -> np.ndarray:
        """The node coordinates along ``y`` (the radius in cylindrical geometry)."""
        return NodeAxis(self.origin[1], self.h, self.shape[1]).nodes()

    @property
    def dx(self) -> np.ndarray:
        """The ``nx - 1`` edge lengths along ``x``."""
        return self._axis.edges()

    @property
    def upper(self) -> tuple[float, float]:
        return (self._axis.last(), NodeAxis(self.origin[1], self.h, self.shape[1]).last())

    @property
    def logical_origin(self) -> tuple[float, float]:
        """The uniform coordinates of node ``(0, 0)`` (the kernels locate points by them)."""
        return (float(self.logical_x0), self.origin[1])

    @property
    def logical_upper(self) -> tuple[float, float]:
        """The uniform coordinates of the last node."""
        if not self.graded:
            return self.upper
        return (float(self.logical_x0) + self.h * (self.shape[0] - 1), self.upper[1])

    def index_x(self, x: Any) -> np.ndarray:
        """The fractional node index of positions ``x`` (linear between graded nodes)."""
        return self._axis.fraction(x)

    def position_x(self, index: Any) -> np.ndarray:
        """The position along ``x`` of a fractional node index."""
        return self._axis.position(index)

    def logical_x(self, x: Any) -> np.ndarray:
        """The uniform coordinate ``logical_x0 + h * index_x(x)`` (``x`` itself if uniform)."""
        if not self.graded:
            return np.asarray(x, dtype=float)
        return float(self.logical_x0) + self.h * self._axis.fraction(x)

    def spacing_at(self, x: Any) -> Any:
        """The smaller edge of the cells at ``x``: ``h``, or less along a graded ``x``."""
        if not self.graded:
            return self.h
        k = np.clip(np.floor(self._axis.fraction(x)).astype(np.int64), 0, self.shape[0] - 2)
        return np.minimum(self.dx[k], self.h)

    def nodes(self) -> tuple[np.ndarray, np.ndarray]:
        """The node coordinates as two ``(nx, ny)`` arrays."""
        return np.meshgrid(self.x, self.y, indexing="ij")

    def inside_solid(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        """The index of the electrode containing each point (the first listed wins), or -1."""
        xb, yb = np.broadcast_arrays(np.asarray(x, dtype=float), np.asarray(y, dtype=float))
        owner = np.full(xb.shape, -1, dtype=np.int32)
        for number, electrode in enumerate(self.electrodes):
            pending = np.flatnonzero(owner.ravel() < 0)
            if not pending.size:
                break
            hit = np.asarray(electrode.inside(xb.ravel()[pending], yb.ravel()[pending]), bool)
            owner.ravel()[pending[hit]] = number
        return owner

    # -- classification -------------------------------------------------------------------

    def _owner_contains(self, owner: np.ndarray, px: np.ndarray, py: np.ndarray) -> np.ndarray:
        """Whether each point lies inside the electrode ``owner`` names for it."""
        inside = np.zeros(owner.shape, dtype=bool)
        for number in np.unique(owner):
            sel = owner == number
            inside[sel] = np.asarray(self.electrodes[number].inside(px[sel], py[sel]), bool)
        return inside

    def _surface_fraction(self, i, j, owner, axis: int, step: int) -> np.ndarray:
        """The surface's place on the edges from nodes ``(i, j)`` towards their solid
        neighbours (electrodes ``owner``), as ``s / 255``: the largest 8-bit ``s`` whose
        trial points along the way the electrode does not contain, at least 1."""
        px = self.x[i]
        py = self.origin[1] + self.h * j
        length = self.h if axis == 1 else self.dx[i + min(step, 0)]
        full = (1 << DISTANCE_BITS) - 1
        code = np.zeros(i.shape, dtype=np.int64)
        for bit in reversed(range(DISTANCE_BITS)):
            trial = code | (1 << bit)
            offset = step * length * trial / float(full)
            qx, qy = (px + offset, py) if axis == 0 else (px, py + offset)
            code = np.where(self._owner_contains(owner, qx, qy), code, trial)
        return np.maximum(code, 1) / float(full)

    def _classify_on_device(self):
        """``(solid, near, distance)`` sampled on the device (``bt_classify_mesh``) when
        allowed, a CUDA device is present and every electrode is a configuration shape;
        else None."""
        if not self.electrodes or self.classify_on_device is False:
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

    def _fixed_nodes(self, xn: np.ndarray, yn: np.ndarray) -> None:
        """``fixed`` and ``fixed_value``: the electrodes' nodes at their potentials, then the
        Dirichlet faces' remaining nodes at the faces' values."""
        nx, ny = self.shape
        solid = self.solid >= 0
        potential = np.append([float(e.potential) for e in self.electrodes], 0.0)
        self.fixed = solid.copy()
        self.fixed_value = np.where(solid, potential[self.solid], 0.0)
        rows = {"x_min": np.s_[0, :], "x_max": np.s_[nx - 1, :], "y_min": np.s_[:, 0],
                "y_max": np.s_[:, ny - 1]}  # fmt: skip
        for face, where in rows.items():
            condition = self.faces[face]
            if condition.kind == "dirichlet":
                open_ = ~solid[where]
                values = condition.evaluate(xn[where], yn[where])
                self.fixed_value[where] = np.where(open_, values, self.fixed_value[where])
                self.fixed[where] |= open_

    def _classify(self) -> None:
        xn, yn = self.nodes()
        device = self._classify_on_device()
        #: The electrode index of every node (-1: none).
        self.solid = self.inside_solid(xn, yn) if device is None else device[0]
        self._fixed_nodes(xn, yn)
        if device is not None:
            self.near_solid, self.distance = device[1], device[2]
            return
        nx, ny = self.shape
        #: The fraction of the edge to the surface along -x, +x, -y, +y (1: no surface).
        self.distance = np.ones((4, nx, ny))
        #: Free nodes with an electrode neighbour.
        self.near_solid = np.zeros((nx, ny), dtype=bool)
        padded = np.pad(self.solid, 1, constant_values=-1)
        for d, (axis, step) in enumerate(DIRECTIONS):
            shift = (step, 0) if axis == 0 else (0, step)
            neighbour = padded[1 + shift[0] : 1 + shift[0] + nx, 1 + shift[1] : 1 + shift[1] + ny]
            i, j = np.nonzero((self.solid < 0) & (neighbour >= 0))
            if i.size:
                self.near_solid[i, j] = True
                self.distance[d, i, j] = self._surface_fraction(i, j, neighbour[i, j], axis,
                                                                step)  # fmt: skip
