"""Design search over the differentiable solver: L-BFGS with adjoint gradients, recorded.

The interface of the reference's ``optimization/design.py`` (``Parameter``, ``Design``,
``Evaluation``) and ``optimization/record.py`` (``Record``): a record is one JSON line per
evaluation in the order evaluated -- the design's key, its parameters, objectives,
constraints, flags, wall time, diagnostics and generation -- and a search given an
existing record takes the designs recorded there instead of evaluating them again.  The
key of a design is the first 16 hex digits of the SHA-1 of the JSON text
``[names, normalized values to 10 decimals]`` (``design.py:119-128``), so records made by
either code resume in the other.

Where the reference searches by differential evolution (``optimization/search.py``),
`lbfgs_search` minimises one objective by L-BFGS-B over the parameters scaled to [0, 1],
each evaluation carrying its gradient (from the adjoint of the converged solve,
`einzel_evaluator`) in its diagnostics.
"""

from __future__ import annotations

import hashlib
import json
import math
import time
from collections.abc import Callable, Iterable, Iterator, Mapping, Sequence
from dataclasses import dataclass, field, replace
from pathlib import Path
from typing import Any

import numpy as np

#: Decimals of the normalized parameters that identify a design in a record.
KEY_DECIMALS = 10


@dataclass(frozen=True)
class Parameter:
    """A design parameter between ``lower`` and ``upper`` (SI values, ``unit`` a label)."""

    name: str
    lower: float
    upper: float
    unit: str = ""

    def __post_init__(self) -> None:
        lo, hi = float(self.lower), float(self.upper)
        object.__setattr__(self, "lower", lo)
        object.__setattr__(self, "upper", hi)
        if not (math.isfinite(lo) and math.isfinite(hi)):
            raise ValueError(f"the bounds of {self.name!r} must be finite")
        if not lo < hi:
            raise ValueError(f"{self.name!r} needs lower < upper, got {lo} and {hi}")


@dataclass(frozen=True)
class Design:
    """Named, bounded parameters, and ``build(values)`` turning ``{name: value}`` into what
    the evaluation takes (the values themselves without it)."""

    parameters: tuple[Parameter, ...]
    build: Callable[[dict[str, float]], Any] | None = None

    def __post_init__(self) -> None:
        parameters = tuple(self.parameters)
        object.__setattr__(self, "parameters", parameters)
        if not parameters:
            raise ValueError("a design needs at least one parameter")
        names = [p.name for p in parameters]
        if len(set(names)) != len(names):
            raise ValueError(f"parameter names must be unique, got {names}")

    @property
    def names(self) -> tuple[str, ...]:
        return tuple(p.name for p in self.parameters)

    @property
    def bounds(self) -> list[tuple[float, float]]:
        return [(p.lower, p.upper) for p in self.parameters]

    def vector(self, values) -> np.ndarray:
        """The values (by name, or in order) as an array."""
        if isinstance(values, Mapping):
            absent = sorted(set(self.names) - set(values))
            if absent:
                raise KeyError(f"missing parameters {absent}")
            return np.array([float(values[name]) for name in self.names])
        x = np.asarray(values, dtype=float).ravel()
        if x.size != len(self):
            raise ValueError(f"need {len(self)} values, got {x.size}")
        return x

    def values(self, x) -> dict[str, float]:
        return {name: float(v) for name, v in zip(self.names, self.vector(x), strict=True)}

    def normalized(self, x) -> np.ndarray:
        """The values mapped to [0, 1] between the bounds."""
        lo, hi = np.array(self.bounds, dtype=float).T
        return (self.vector(x) - lo) / (hi - lo)

    def from_normalized(self, u) -> np.ndarray:
        lo, hi = np.array(self.bounds, dtype=float).T
        return lo + np.asarray(u, dtype=float) * (hi - lo)

    def key(self, x) -> str:
        """The design's identity in a record: designs within about 1e-10 of the parameter
        ranges share it."""
        digits = np.round(self.normalized(x), KEY_DECIMALS) + 0.0  # +0.0: no "-0.0"
        text = json.dumps([list(self.names), [f"{v:.{KEY_DECIMALS}f}" for v in digits]])
        return hashlib.sha1(text.encode()).hexdigest()[:16]

    def configuration(self, values) -> Any:
        named = self.values(values)
        return named if self.build is None else self.build(named)

    def __len__(self) -> int:
        return len(self.parameters)


def _json_plain(value: Any) -> Any:
    """NumPy scalars and arrays as Python numbers and lists, recursively."""
    if isinstance(value, Mapping):
        return {str(k): _json_plain(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_json_plain(v) for v in value]
    if isinstance(value, np.ndarray):
        return value.tolist()
    if isinstance(value, np.generic):
        return value.item()
    return value


@dataclass(frozen=True)
class Evaluation:
    """One design's outcome: objectives (minimised) and constraints (satisfied at <= 0),
    the model's convergence, an exception's message, the wall time [s], diagnostics, the
    parameters and the search generation (None outside a population search)."""

    objectives: Mapping[str, float]
    constraints: Mapping[str, float] = field(default_factory=dict)
    converged: bool = True
    wall_time: float = float("nan")
    failure: str | None = None
    diagnostics: Mapping[str, Any] = field(default_factory=dict)
    parameters: Mapping[str, float] = field(default_factory=dict)
    generation: int | None = None

    def __post_init__(self) -> None:
        for name in ("objectives", "constraints", "parameters"):
            object.__setattr__(self, name, {k: float(v) for k, v in getattr(self, name).items()})
        object.__setattr__(self, "diagnostics", dict(self.diagnostics))
        object.__setattr__(self, "converged", bool(self.converged))

    @property
    def ok(self) -> bool:
        """Converged, no failure, finite objectives."""
        finite = all(math.isfinite(v) for v in self.objectives.values())
        return self.converged and self.failure is None and finite

    @property
    def violation(self) -> float:
        """The sum of the positive constraint values (a NaN constraint: infinity)."""
        return float(sum(math.inf if math.isnan(v) else max(v, 0.0)
                         for v in self.constraints.values()))  # fmt: skip

    @property
    def feasible(self) -> bool:
        return self.ok and self.violation == 0.0

    def rank(self, objective: str) -> tuple[int, float]:
        """Lower is better: feasible by the objective, then ok ones by their violation,
        then the failed."""
        if self.feasible:
            return (0, self.objectives[objective])
        return (1, self.violation) if self.ok else (2, 0.0)

    def to_dict(self) -> dict[str, Any]:
        return {"parameters": dict(self.parameters), "objectives": dict(self.objectives),
                "constraints": dict(self.constraints), "converged": self.converged,
                "feasible": self.feasible, "wall_time": self.wall_time,
                "failure": self.failure, "diagnostics": _json_plain(self.diagnostics),
                "generation": self.generation}  # fmt: skip

    @classmethod
    def from_dict(cls, data: Mapping[str, Any]) -> Evaluation:
        return cls(objectives=data["objectives"], constraints=data.get("constraints", {}),
                   converged=data.get("converged", True),
                   wall_time=data.get("wall_time", float("nan")), failure=data.get("failure"),
                   diagnostics=data.get("diagnostics", {}),
                   parameters=data.get("parameters", {}), generation=data.get("generation"))  # fmt: skip


class Record:
    """A design's evaluations in memory and, with a ``path``, appended line by line to a
    JSON-lines file (an interrupted search keeps what it finished).  An existing file is
    read first; its parameter names must be the design's."""

    def __init__(self, design: Design, path: str | Path | None = None) -> None:
        self.design = design
        self.path = None if path is None else Path(path)
        self._evaluations: list[Evaluation] = []
        self._by_key: dict[str, Evaluation] = {}
        if self.path is None or not self.path.exists():
            return
        for number, line in enumerate(self.path.read_text().splitlines(), 1):
            if not line.strip():
                continue
            data = json.loads(line)
            if set(data["parameters"]) != set(design.names):
                raise ValueError(f"{self.path}:{number} has the parameters "
                                 f"{list(data['parameters'])}, the design {list(design.names)}")  # fmt: skip
            self._keep(Evaluation.from_dict(data))

    def _keep(self, evaluation: Evaluation) -> str:
        key = self.design.key(evaluation.parameters)
        self._evaluations.append(evaluation)
        self._by_key.setdefault(key, evaluation)
        return key

    def get(self, key: str) -> Evaluation | None:
        return self._by_key.get(key)

    def append(self, evaluations: Iterable[Evaluation]) -> None:
        lines = [json.dumps({"key": self._keep(e), **e.to_dict()}) for e in evaluations]
        if self.path is not None and lines:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            with self.path.open("a") as out:
                out.write("\n".join(lines) + "\n")

    def __iter__(self) -> Iterator[Evaluation]:
        return iter(self._evaluations)

    def __len__(self) -> int:
        return len(self._evaluations)


# -- L-BFGS over adjoint gradients -------------------------------------------------------------


@dataclass
class SearchResult:
    """The best evaluation of a search, all of them, and how many were computed (the rest
    came from the record)."""

    best: Evaluation
    evaluations: list[Evaluation]
    computed: int
    message: str


def lbfgs_search(design: Design, evaluate: Callable[[dict[str, float]], Evaluation],
                 start, *, objective: str, record: Record | None = None,
                 max_evaluations: int = 30, tolerance: float = 1e-9) -> SearchResult:  # fmt: skip
    """Minimise ``objective`` by L-BFGS-B between the design's bounds.

    ``evaluate(values)`` returns an `Evaluation` whose diagnostics hold ``"gradient"``:
    ``{name: d objective / d parameter}``.  A design already in ``record`` (by key) is
    taken from it; new evaluations are appended to it.  The search runs in the normalized
    coordinates ([0, 1] per parameter), where the gradient is scaled by the ranges.
    """
    from scipy.optimize import minimize

    record = record if record is not None else Record(design)
    span = np.array([hi - lo for lo, hi in design.bounds])
    seen: list[Evaluation] = []
    computed = 0

    def value_and_gradient(u: np.ndarray) -> tuple[float, np.ndarray]:
        nonlocal computed
        x = design.from_normalized(np.clip(u, 0.0, 1.0))
        key = design.key(x)
        result = record.get(key)
        if result is None or "gradient" not in result.diagnostics:
            if len(seen) >= max_evaluations:
                raise _Budget
            start_time = time.perf_counter()
            values = design.values(x)
            try:
                result = evaluate(values)
            except Exception as error:  # noqa: BLE001 - a failed design is recorded
                result = Evaluation({objective: math.nan}, converged=False,
                                    failure=f"{type(error).__name__}: {error}")  # fmt: skip
            result = replace(result, parameters=values,
                             wall_time=time.perf_counter() - start_time)  # fmt: skip
            record.append([result])
            computed += 1
        seen.append(result)
        if not result.ok:
            return math.inf, np.zeros(len(design))
        gradient = result.diagnostics["gradient"]
        g = np.array([float(gradient[name]) for name in design.names]) * span
        return float(result.objectives[objective]), g

    u0 = design.normalized(design.vector(start))
    message = ""
    try:
        out = minimize(value_and_gradient, u0, jac=True, method="L-BFGS-B",
                       bounds=[(0.0, 1.0)] * len(design),
                       options={"maxfun": max_evaluations, "ftol": tolerance, "gtol": 1e-12})  # fmt: skip
        message = str(out.message)
    except _Budget:
        message = "evaluation budget reached"
    best = min(seen, key=lambda e: e.rank(objective))
    return SearchResult(best, seen, computed, message)


class _Budget(Exception):
    """The search's evaluations are used up."""


def einzel_evaluator(base, names: Sequence[str] = ("v_mid",), plane: float = 79e-3,
                     tolerance: float = 1e-6, iterations: int = 60,
                     field_limit: float | None = None):  # fmt: skip
    """An evaluation function of an einzel design for `lbfgs_search`: the rms angle and
    the current at ``plane`` of the lens with the named parameters set (``v_mid`` the middle
    plate, ``v1``-``v3`` the plates, ``current`` the beam current), and the gradient of the
    rms angle with respect to them from the adjoint of the converged solve.  The largest
    surface field [V/m] is a diagnostic and, with ``field_limit``, the constraint
    ``field / field_limit - 1`` (the reference's einzel constraint, ``einzel.py:348``)."""
    from beamtracer_b200.adjoint import adjoint_design_gradient
    from beamtracer_b200.einzel import GRADIENT_PARAMETERS, resolved_voltages

    columns = {"v1": 0, "v2": 1, "v3": 2, "current": 3, "v_mid": 1}

    def evaluate(values: dict[str, float]) -> Evaluation:
        voltages = list(resolved_voltages(base))
        current = base.current
        for name, value in values.items():
            if name == "current":
                current = value
            else:
                voltages[columns[name]] = value
        design = replace(base, voltages=tuple(voltages), current=current)
        grad = adjoint_design_gradient(design, plane, tolerance=tolerance, iterations=iterations)
        moments = grad["moments"]
        angle = grad["rms_angle"]
        field = max(grad["surface_fields"].values(), default=0.0)
        constraints = {} if field_limit is None else {"surface_field": field / field_limit - 1.0}
        return Evaluation(
            objectives={"rms_angle": moments["rms_angle"], "current": -moments["current"]},
            constraints=constraints, converged=grad["converged"],
            diagnostics={"gradient": {name: float(angle[columns[name]]) for name in values},
                         "emittance": moments["emittance"], "rms_size": moments["rms_size"],
                         "field": field,
                         "adjoint_iterations": grad["adjoint_iterations"],
                         "parameters_order": list(GRADIENT_PARAMETERS)},
        )  # fmt: skip

    return evaluate
