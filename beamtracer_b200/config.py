"""The configuration of a beam: `BeamOpticsConfig` and its sections.

The settings of the reference's ``config.py`` and ``sections.py`` (``BeamOpticsConfig``,
``GridParams``, ``FieldBCs``, ``FieldBoundaryCondition``, ``ObjectParams``, ``BeamSpecies``,
``ParticleBeam``, ``ExtractionPlasma``, ``NegativeExtractionPlasma``, ``Solenoid``,
``SpaceChargeCompensation``; ``config.py:38-832``, ``sections.py:84-784``), with their
checks and the dictionary form ``to_dict`` / ``from_dict``.  Values are SI numbers (charges
in e, masses in u, energies and temperatures in eV); the reference also parses unit
strings through astropy, which this image does not have.

Electrodes (`ObjectParams`) are rectangles, circles, polygons (triangles), lines and
``aperture2d`` plates (a polygon and its mirror image across the axis), each a closed set:
a point on the boundary is inside.
"""

from __future__ import annotations

from collections.abc import Mapping, Sequence
from dataclasses import asdict, dataclass, field, fields, replace
from typing import Any, ClassVar

import numpy as np

# -- the grid and the walls ----------------------------------------------------------------


def _per_axis(value: Any, ndim: int = 2) -> tuple:
    if isinstance(value, (int, float, bool, np.floating, np.integer)):
        return (value,) * ndim
    values = tuple(np.asarray(value).ravel().tolist())
    if len(values) != ndim:
        raise ValueError(f"need one value per axis ({ndim}), got {value!r}")
    return values


@dataclass
class GridParams:
    """Nodes per axis and the extent [m] of a 2D grid (``sections.py:84-207``)."""

    ndim: int = 2
    num_gridpoints: Any = 64
    lower_bound: Any = 0.0
    upper_bound: Any = 32.0e-3
    coordinates: str = "cartesian"
    x_spacing: Any = None
    x_through: Any = ()

    def __post_init__(self) -> None:
        if int(self.ndim) != 2:
            raise ValueError(f"this build traces 2D grids, got ndim={self.ndim}")
        self.ndim = 2
        self.num_gridpoints = tuple(int(k) for k in _per_axis(self.num_gridpoints))
        self.lower_bound = tuple(float(v) for v in _per_axis(self.lower_bound))
        self.upper_bound = tuple(float(v) for v in _per_axis(self.upper_bound))
        if any(hi <= lo for lo, hi in zip(self.lower_bound, self.upper_bound, strict=True)):
            raise ValueError(
                f"upper_bound {self.upper_bound} must exceed lower_bound {self.lower_bound} "
                "on every axis"
            )
        if self.x_spacing is not None:
            raise NotImplementedError("graded grids from x_spacing are not part of this build")

    @property
    def graded(self) -> bool:
        return False

    @property
    def x_nodes(self) -> None:
        return None

    @property
    def deltas(self) -> list[float]:
        return [(b1 - b0) / (n - 1) for b0, b1, n in
                zip(self.lower_bound, self.upper_bound, self.num_gridpoints, strict=True)]  # fmt: skip

    def to_dict(self) -> dict:
        return {"ndim": 2, "num_gridpoints": list(self.num_gridpoints),
                "lower_bound": list(self.lower_bound), "upper_bound": list(self.upper_bound),
                "coordinates": self.coordinates}  # fmt: skip

    @classmethod
    def from_dict(cls, params: Mapping[str, Any]) -> GridParams:
        keys = ("ndim", "num_gridpoints", "lower_bound", "upper_bound", "coordinates",
                "x_spacing", "x_through")  # fmt: skip
        unknown = set(params) - set(keys) - {"nvel", "domain_decomposition"}
        if unknown:
            raise KeyError(f"unknown grid entries {sorted(unknown)}")
        return cls(**{key: params[key] for key in keys if key in params})


class FieldBoundaryCondition:
    """A Dirichlet (potential [V]) or Neumann (normal derivative [V/m]) face condition
    (``sections.py:385-446``); ``value`` a number or a function of ``(x, y)``."""

    def __init__(self, bc_type: str, value: Any = 0.0) -> None:
        if bc_type not in ("dirichlet", "neumann"):
            raise ValueError(f"the beam tracer's faces are dirichlet or neumann, got {bc_type!r}")
        self._bc_type = bc_type
        self._value = value

    @staticmethod
    def dirichlet(value: Any = 0.0) -> FieldBoundaryCondition:
        return FieldBoundaryCondition("dirichlet", value)

    @staticmethod
    def neumann(normal_derivative: Any = 0.0) -> FieldBoundaryCondition:
        return FieldBoundaryCondition("neumann", normal_derivative)

    @property
    def bc_type(self) -> str:
        return self._bc_type

    @property
    def value(self) -> Any:
        return self._value

    def evaluate(self, x=None, y=None, z=None, t=None):
        if callable(self._value):
            return self._value(x, y)
        return np.full(np.shape(x), float(self._value)) if x is not None else float(self._value)

    def __eq__(self, other: object) -> bool:
        return (isinstance(other, FieldBoundaryCondition) and other._bc_type == self._bc_type
                and other._value == self._value)  # fmt: skip


class FieldBCs:
    """The conditions on the four faces of a 2D grid (``sections.py:449-540``)."""

    def __init__(self, x_lower, x_upper, y_lower, y_upper) -> None:
        self._bc = {"x": {"min": x_lower, "max": x_upper}, "y": {"min": y_lower, "max": y_upper}}

    has_z = False

    @staticmethod
    def grounded(ndim: int = 2) -> FieldBCs:
        zero = FieldBoundaryCondition.dirichlet(0.0)
        return FieldBCs(zero, zero, zero, zero)

    def get_bc(self, dir: str, side: str) -> FieldBoundaryCondition:  # noqa: A002
        return self._bc[dir][side]

    def to_dict(self) -> dict:
        out = {}
        for axis, sides in self._bc.items():
            lower = sides["min"]
            entry: dict = {"type": lower.bc_type}
            for key, bc in sides.items():
                if callable(bc.value):
                    raise ValueError("a face given by a function has no dictionary form")
                side: Any = float(bc.value)
                if bc.bc_type != lower.bc_type:
                    side = {"value": side, "type": bc.bc_type}
                entry[key] = side
            out[axis] = entry
        return out

    @classmethod
    def from_dict(cls, params: Mapping[str, Any]) -> FieldBCs:
        faces = {}
        for axis in ("x", "y"):
            if axis not in params:
                raise ValueError(f"field boundaries need the {axis!r} axis")
            item = params[axis]
            for key, name in (("min", "lower"), ("max", "upper")):
                side = item[key]
                if not isinstance(side, Mapping):
                    side = {"value": side}
                bc_type = side.get("type", item.get("type"))
                if bc_type is None:
                    raise ValueError(f"field boundary '{axis}/{key}' needs a type")
                faces[f"{axis}_{name}"] = FieldBoundaryCondition(bc_type, float(side["value"]))
        return cls(**faces)


OBJECT_TYPES = ("line", "rectangle", "triangle", "polygon", "circle", "aperture2d")
_GEOMETRY = ("vertices", "midpoint", "side_lengths", "radius", "axis", "position")


def _polygon_inside(vertices: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Points inside the polygon or on its boundary (even-odd rule)."""
    vx, vy = vertices[:, 0], vertices[:, 1]
    n = len(vx)
    inside = np.zeros(np.shape(x), dtype=bool)
    boundary = np.zeros(np.shape(x), dtype=bool)
    for k in range(n):
        x1, y1, x2, y2 = vx[k], vy[k], vx[(k + 1) % n], vy[(k + 1) % n]
        crosses = (y1 > y) != (y2 > y)
        with np.errstate(divide="ignore", invalid="ignore"):
            at = x1 + (y - y1) * (x2 - x1) / (y2 - y1)
        inside ^= crosses & (x < at)
        # on the edge: collinear and within its extent
        cross = (x2 - x1) * (y - y1) - (y2 - y1) * (x - x1)
        length = np.hypot(x2 - x1, y2 - y1)
        near = np.abs(cross) <= 1e-12 * max(length, 1e-300) * max(length, 1.0)
        within = ((x >= min(x1, x2) - 1e-15) & (x <= max(x1, x2) + 1e-15)
                  & (y >= min(y1, y2) - 1e-15) & (y <= max(y1, y2) + 1e-15))  # fmt: skip
        boundary |= near & within
    return inside | boundary


@dataclass
class ObjectParams:
    """An electrode: a shape held at ``bc_value`` [V] (``sections.py:636-784``)."""

    type: str
    bc_type: str
    bc_value: float | None = None
    vertices: Any = None
    midpoint: Any = None
    side_lengths: Any = None
    radius: float | None = None
    axis: Any = None
    position: float | None = None

    def __post_init__(self) -> None:
        if self.type not in OBJECT_TYPES:
            raise ValueError(f"object type must be one of {OBJECT_TYPES}, got {self.type!r}")
        if self.bc_type not in ("dirichlet", "neumann"):
            raise ValueError(f"unknown object condition {self.bc_type!r}")

    def inside(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        """Whether the points lie in the shape (boundary included)."""
        x = np.asarray(x, dtype=float)
        y = np.asarray(y, dtype=float)
        if self.type in ("rectangle", "line"):
            (mx, my), (lx, ly) = self.midpoint, self.side_lengths
            return (np.abs(x - mx) <= 0.5 * lx) & (np.abs(y - my) <= 0.5 * ly)
        if self.type == "circle":
            mx, my = self.midpoint
            return (x - mx) ** 2 + (y - my) ** 2 <= float(self.radius) ** 2
        vertices = np.asarray(self.vertices, dtype=float)
        if self.type in ("polygon", "triangle"):
            return _polygon_inside(vertices, x, y)
        # aperture2d: the polygon and its mirror image across the line axis = position
        axis = int(self.axis) if self.axis is not None else 0
        position = float(self.position or 0.0)
        mirrored = vertices.copy()
        mirrored[:, 1 - axis] = 2.0 * position - mirrored[:, 1 - axis]
        return _polygon_inside(vertices, x, y) | _polygon_inside(mirrored, x, y)

    def to_dict(self) -> dict:
        params: dict = {"type": self.type}
        for key in _GEOMETRY:
            value = getattr(self, key)
            if value is not None:
                params[key] = np.asarray(value).tolist() if not np.isscalar(value) else value
        key = "normal_derivative" if self.bc_type == "neumann" else "potential"
        params["bc"] = {"type": self.bc_type, key: self.bc_value}
        return params

    @classmethod
    def from_dict(cls, params: Mapping[str, Any]) -> ObjectParams:
        bc_type = params["bc"]["type"]
        key = "normal_derivative" if bc_type == "neumann" else "potential"
        if key not in params["bc"]:
            raise ValueError(f"an object with a {bc_type!r} condition needs bc.{key}")
        return cls(type=params["type"], bc_type=bc_type, bc_value=params["bc"][key],
                   **{k: params.get(k) for k in _GEOMETRY})  # fmt: skip


# -- beams, plasma, fields ------------------------------------------------------------------


@dataclass(frozen=True)
class BeamSpecies:
    """A beam emitted from a line with a given energy (``config.py:38-70``)."""

    name: str
    current_density: float
    start: tuple[float, float]
    end: tuple[float, float]
    charge: float = 1.0
    mass: float = 1.007276
    energy: float = 5.0
    parallel_temperature: float = 0.0
    transverse_temperature: float = 0.5
    num_particles: int = 1000

    def __post_init__(self) -> None:
        object.__setattr__(self, "start", tuple(float(v) for v in self.start))
        object.__setattr__(self, "end", tuple(float(v) for v in self.end))
        if len(self.start) != 2 or len(self.end) != 2:
            raise ValueError("start and end are (x, y) points")
        if self.num_particles < 1:
            raise ValueError("num_particles must be at least 1")
        if self.mass <= 0.0:
            raise ValueError("mass must be positive")
        if self.energy <= 0.0:
            raise ValueError("energy must be positive")


@dataclass(frozen=True)
class ParticleBeam:
    """A beam given trajectory by trajectory (``config.py:133-166``): positions and
    velocities (N, 3) [m, m/s], currents (N,) [A], one charge [e] and mass [u]."""

    name: str
    position: tuple
    velocity: tuple
    current: tuple
    charge: float = 1.0
    mass: float = 1.007276

    #: The fields read as nested tuples; each is built from its array at its first read
    #: (a million trajectories take a second to turn into tuples, which a model that
    #: reads the arrays never needs).
    _TUPLE_FIELDS: ClassVar[tuple[str, ...]] = ("position", "velocity", "current")

    def __post_init__(self) -> None:
        position = np.array(self.position, dtype=float).reshape(-1, 3)
        velocity = np.array(self.velocity, dtype=float).reshape(-1, 3)
        current = np.array(self.current, dtype=float).ravel()
        if not position.shape[0] == velocity.shape[0] == current.size:
            raise ValueError("position, velocity and current need one row per trajectory")
        for array in (position, velocity, current):
            array.flags.writeable = False
        object.__setattr__(self, "_arrays", (position, velocity, current))
        for name, array in zip(self._TUPLE_FIELDS, self._arrays, strict=True):
            object.__setattr__(self, name, _PendingRows(array))

    def __getattribute__(self, name: str) -> Any:
        value = object.__getattribute__(self, name)
        if type(value) is _PendingRows:
            value = value.rows()
            object.__setattr__(self, name, value)
        return value

    def arrays(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Positions and velocities (N, 3) and currents (N,) as read-only float arrays."""
        return self._arrays

    def __len__(self) -> int:
        return int(self._arrays[2].size)


class _PendingRows:
    """A `ParticleBeam` field not yet read: the array its tuple is made from."""

    __slots__ = ("array",)

    def __init__(self, array: np.ndarray) -> None:
        self.array = array

    def rows(self) -> tuple:
        if self.array.ndim == 1:
            return tuple(self.array.tolist())
        return tuple(map(tuple, self.array.tolist()))


@dataclass(frozen=True)
class ExtractionPlasma:
    """Boltzmann electrons for positive-ion extraction (``config.py:169-189``)."""

    electron_temperature: float
    plasma_potential: float
    initial_plasma_x: float
    rho_e: float | None = None


@dataclass(frozen=True)
class NegativeExtractionPlasma:
    """Boltzmann positive ions for negative-ion extraction (``config.py:192-215``)."""

    ion_temperature: float
    plasma_potential: float
    initial_plasma_x: float
    rho_p: float | None = None

    def __post_init__(self) -> None:
        if not self.ion_temperature > 0.0:
            raise ValueError(f"ion_temperature must be positive, got {self.ion_temperature}")


@dataclass
class AxialField:
    """A measured on-axis field ``bz`` [T] sampled at ``z0 + dz k`` [m]
    (``config.py:370-382``; SI numbers)."""

    z0: float
    dz: float
    bz: tuple

    def __post_init__(self) -> None:
        self.z0, self.dz = float(self.z0), float(self.dz)
        self.bz = tuple(float(b) for b in self.bz)


@dataclass(frozen=True)
class Solenoid:
    """A thin-walled solenoid on the axis: centre, length, radius [m], peak [T]."""

    centre: float
    length: float
    radius: float
    peak: float


@dataclass(frozen=True)
class RefinementParams:
    """A box refined to ``level`` (cells ``2**level`` times smaller than the grid's;
    ``config.py:437-464``).  ``lower`` and ``upper`` are its corners ``(x, y)`` [m]
    (``(x, r)`` in cylindrical geometry), widened to the cells of the level below; a
    level's boxes lie inside those of the level below."""

    level: int
    lower: tuple[float, ...]
    upper: tuple[float, ...]

    def __post_init__(self) -> None:
        if int(self.level) != self.level or self.level < 1:
            raise ValueError(f"level must be a positive integer, got {self.level}")
        object.__setattr__(self, "level", int(self.level))
        lower = tuple(float(v) for v in self.lower)
        upper = tuple(float(v) for v in self.upper)
        if (len(lower) not in (2, 3) or len(upper) != len(lower)
                or not all(a < b for a, b in zip(lower, upper))):  # fmt: skip
            raise ValueError(f"a refined box needs lower < upper, got {lower}, {upper}")
        object.__setattr__(self, "lower", lower)
        object.__setattr__(self, "upper", upper)


@dataclass(frozen=True)
class SpaceChargeCompensation:
    """The beam's space charge reduced by ``fraction`` between ``x_min`` and ``x_max``."""

    x_min: float
    x_max: float
    fraction: float

    def __post_init__(self) -> None:
        if not 0.0 <= self.fraction <= 1.0:
            raise ValueError(f"fraction must be in [0, 1], got {self.fraction}")


def beam_from_value(value: Any):
    if isinstance(value, (BeamSpecies, ParticleBeam)):
        return value
    params = dict(value)
    kind = params.pop("type", "line")
    classes = {"line": BeamSpecies, "particles": ParticleBeam}
    if kind not in classes:
        raise ValueError(f"beam type must be one of {sorted(classes)}, got {kind!r}")
    return classes[kind](**params)


def plasma_from_value(value: Any):
    if value is None or isinstance(value, (ExtractionPlasma, NegativeExtractionPlasma)):
        return value
    params = dict(value)
    kind = params.pop("type", "positive")
    if kind not in ("positive", "negative"):
        raise ValueError(f"plasma type must be 'positive' or 'negative', got {kind!r}")
    return (NegativeExtractionPlasma if kind == "negative" else ExtractionPlasma)(**params)


def _coerce(cls, value):
    if value is None or isinstance(value, cls):
        return value
    return cls(**value)


@dataclass(kw_only=True)
class BeamOpticsConfig:
    """Steady ion beams in a self-consistent field (``config.py:558-832``)."""

    model_name: ClassVar[str] = "BeamOptics"

    grid: GridParams = field(default_factory=GridParams)
    objects: dict[str, ObjectParams] = field(default_factory=dict)
    bcs_field: FieldBCs | None = None
    beams: Sequence = field(default_factory=list)
    plasma: ExtractionPlasma | NegativeExtractionPlasma | None = None
    solenoids: list[Solenoid] = field(default_factory=list)
    axial_field: Any = None
    field_order: int = 3
    field_map: Any = None
    compensation: list[SpaceChargeCompensation] = field(default_factory=list)
    charge_changing: Any = None
    iterations: int = 20
    tolerance: float = 1.0e-3
    relaxation: float = 1.0
    step_fraction: float = 0.5
    max_steps: int = 100_000
    integrator: str = "rk4"
    relativistic: bool = False
    mixing: str = "linear"
    anderson_depth: int = 5
    coarse_particles: float = 1.0
    coarse_tolerance: float = 0.0
    field_backend: str = "lu"
    refinement: list = field(default_factory=list)
    adaptive_refinement: Any = None
    symmetry_plane: bool = False
    symmetry_planes: list[str] = field(default_factory=list)
    self_magnetic_field: bool = False
    diagnostic_planes: list[float] = field(default_factory=list)
    save_trajectories: int = 0

    def __post_init__(self) -> None:
        if isinstance(self.grid, Mapping):
            self.grid = GridParams.from_dict(self.grid)
        self.objects = {name: obj if isinstance(obj, ObjectParams) else ObjectParams.from_dict(obj)
                        for name, obj in (self.objects or {}).items()}  # fmt: skip
        if self.bcs_field is None:
            self.bcs_field = FieldBCs.grounded()
        elif isinstance(self.bcs_field, Mapping):
            self.bcs_field = FieldBCs.from_dict(self.bcs_field)
        if self.grid.coordinates not in ("cartesian", "cylindrical"):
            raise ValueError(
                f"BeamOptics needs cartesian or cylindrical coordinates, got {self.grid.coordinates!r}"
            )
        deltas = self.grid.deltas
        if max(deltas) - min(deltas) > 1e-9 * max(deltas):
            raise ValueError(f"BeamOptics needs equal node spacing, got {deltas}")
        self.beams = [beam_from_value(beam) for beam in self.beams]
        self.plasma = plasma_from_value(self.plasma)
        self.solenoids = [_coerce(Solenoid, s) for s in self.solenoids]
        if self.axial_field is not None:
            self.axial_field = _coerce(AxialField, self.axial_field)
        if not 0 <= int(self.field_order) <= 6:
            raise ValueError(f"field_order must be 0 to 6, got {self.field_order}")
        self.compensation = [_coerce(SpaceChargeCompensation, c) for c in self.compensation]
        self.refinement = [
            box if isinstance(box, RefinementParams)
            else RefinementParams(**box) if isinstance(box, Mapping) else RefinementParams(*box)
            for box in (self.refinement or [])
        ]  # fmt: skip
        if any(len(box.lower) != 2 for box in self.refinement):
            raise ValueError("a 2D grid takes refined boxes of (x, y) corners")
        self.diagnostic_planes = [float(p) for p in self.diagnostic_planes]
        if (self.solenoids or self.axial_field) and self.grid.coordinates != "cylindrical":
            raise ValueError("solenoids need cylindrical coordinates (or a 3D grid, on the x axis)")
        if not 0.0 < self.relaxation <= 1.0:
            raise ValueError(f"relaxation must be in (0, 1], got {self.relaxation}")
        if self.iterations < 1:
            raise ValueError("iterations must be at least 1")
        if self.mixing not in ("linear", "anderson"):
            raise ValueError(f"mixing must be 'linear' or 'anderson', got {self.mixing!r}")
        if self.anderson_depth < 1:
            raise ValueError("anderson_depth must be at least 1")
        if not 0.0 < self.coarse_particles <= 1.0:
            raise ValueError(f"coarse_particles must be in (0, 1], got {self.coarse_particles}")
        if self.coarse_particles < 1.0 and not self.coarse_tolerance > 0.0:
            raise ValueError("coarse_particles < 1 needs a positive coarse_tolerance")
        if self.field_backend not in ("lu", "petsc", "amg", "multigrid", "auto"):
            raise ValueError(
                "field_backend must be 'lu', 'petsc', 'amg', 'multigrid' or 'auto', got "
                f"{self.field_backend!r}"
            )
        if self.integrator not in ("rk4", "boris"):
            raise ValueError(f"integrator must be 'rk4' or 'boris', got {self.integrator!r}")
        if self.symmetry_plane and self.grid.coordinates == "cylindrical":
            raise ValueError("symmetry_plane needs a planar (cartesian) grid")
        unsupported = {
            "field_map": self.field_map, "charge_changing": self.charge_changing,
            "adaptive_refinement": self.adaptive_refinement,
            "self_magnetic_field": self.self_magnetic_field,
        }  # fmt: skip
        given = sorted(name for name, value in unsupported.items() if value)
        if given:
            raise NotImplementedError(f"this build does not take {', '.join(given)}")

    def replace(self, **changes: Any) -> BeamOpticsConfig:
        return replace(self, **changes)

    def to_dict(self) -> dict:
        params: dict = {"type": self.model_name}
        for entry in fields(self):
            value = getattr(self, entry.name)
            if value is None:
                continue
            params[entry.name] = value
        params["grid"] = self.grid.to_dict()
        params["objects"] = {name: obj.to_dict() for name, obj in self.objects.items()}
        params["bcs_field"] = self.bcs_field.to_dict()
        params["beams"] = []
        for beam in self.beams:
            entry = asdict(beam)
            entry["type"] = "particles" if isinstance(beam, ParticleBeam) else "line"
            params["beams"].append(entry)
        if self.plasma is not None:
            entry = asdict(self.plasma)
            entry["type"] = "negative" if isinstance(self.plasma, NegativeExtractionPlasma) else "positive"
            params["plasma"] = entry
        params["solenoids"] = [asdict(s) for s in self.solenoids]
        if self.axial_field is not None:
            params["axial_field"] = asdict(self.axial_field)
        params["compensation"] = [asdict(c) for c in self.compensation]
        params["refinement"] = [asdict(box) for box in self.refinement]
        return params

    @classmethod
    def from_dict(cls, params: Mapping[str, Any]) -> BeamOpticsConfig:
        params = dict(params)
        model_name = params.pop("type", cls.model_name)
        if model_name != cls.model_name:
            raise ValueError(f"{cls.__name__} configures {cls.model_name!r}, not {model_name!r}")
        for ignored in ("random", "solver"):
            params.pop(ignored, None)
        known = {entry.name for entry in fields(cls)}
        unknown = set(params) - known
        if unknown:
            raise KeyError(f"unknown {cls.model_name} settings {sorted(unknown)}; known: {sorted(known)}")
        return cls(**params)
