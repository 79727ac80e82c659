"""An einzel lens and its beam: the design problem the batched sweep and the benchmark use.

A cylindrical ``(x, r)`` lens of three plates -- ``|x - x_c| <= t/2``, ``r >= a`` at
``x_c`` = 20, 40 and 60 mm (scaled with the length) held at 0, ``V_mid``, 0 -- with Neumann
faces, and a 10 keV H+ beam of rings launched at x = 1 mm with a seeded truncated-Gaussian
radius and angles correlated to give a chosen rms divergence and emittance in the
cylindrical moments of ``plane_moments`` (the reference's ``optimization/einzel.py``
``EinzelLens`` is the caller this stands for).  Everything is drawn from
``numpy.random.default_rng(seed)``: ``V_mid`` first (when not given), then the radii and
the angles.
"""

from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np
from scipy import constants

from beamtracer_b200.config import (
    BeamOpticsConfig,
    FieldBCs,
    FieldBoundaryCondition,
    GridParams,
    ObjectParams,
    ParticleBeam,
)

PROTON_MASS_U = 1.007276


@dataclass(frozen=True)
class EinzelDesign:
    """The lens and beam settings; lengths in m, voltages in V, current in A."""

    shape: tuple[int, int] = (801, 201)
    length: float = 80e-3
    radius: float = 20e-3
    centres: tuple[float, float, float] = (20e-3, 40e-3, 60e-3)
    thickness: float = 2e-3
    aperture: float = 5e-3
    voltages: tuple[float, float, float] | None = None  # None: (0, V_mid, 0), V_mid seeded
    v_mid_range: tuple[float, float] = (5e3, 9e3)
    energy: float = 10e3  # eV
    current: float = 1e-3
    trajectories: int = 20_000
    launch_x: float = 1e-3
    rms_radius: float = 2e-3
    max_radius: float = 4e-3
    rms_angle: float = 5e-3
    emittance: float = 2e-6
    planes: tuple[float, ...] = (70e-3, 79e-3)
    seed: int = 2


def einzel_beam(design: EinzelDesign, rng: np.random.Generator) -> ParticleBeam:
    """The rings: radius ``rms_radius |g|`` cut at ``max_radius`` (redrawn), angles
    ``r' = kappa r + s g1``, ``a' = s g2`` with ``s = emittance / sigma_x`` and
    ``kappa = sqrt(2 (rms_angle^2 - s^2) / <r^2>)``; speed of ``energy``, equal currents."""
    n = design.trajectories
    radii = np.empty(0)
    while radii.size < n:
        draw = design.rms_radius * np.abs(rng.standard_normal(2 * n))
        radii = np.concatenate([radii, draw[draw <= design.max_radius]])
    r = radii[:n]
    g1, g2 = rng.standard_normal(n), rng.standard_normal(n)
    mean_r2 = float(np.mean(r * r))
    sigma_x = np.sqrt(mean_r2 / 2.0)
    s = design.emittance / sigma_x
    kappa = np.sqrt(max(2.0 * (design.rms_angle**2 - s * s) / mean_r2, 0.0))
    rp = kappa * r + s * g1
    ap = s * g2
    m = PROTON_MASS_U * constants.atomic_mass
    v0 = np.sqrt(2.0 * design.energy * constants.e / m)
    vx = v0 / np.sqrt(1.0 + rp * rp + ap * ap)
    position = np.stack([np.full(n, design.launch_x), r, np.zeros(n)], axis=1)
    velocity = np.stack([vx, rp * vx, ap * vx], axis=1)
    current = np.full(n, design.current / n)
    return ParticleBeam("H+", position, velocity, current, charge=1.0, mass=PROTON_MASS_U)


def _plate(centre: float, design: EinzelDesign, voltage: float) -> ObjectParams:
    mid_r = 0.5 * (design.aperture + design.radius)
    return ObjectParams(type="rectangle", midpoint=(centre, mid_r),
                        side_lengths=(design.thickness, design.radius - design.aperture),
                        bc_type="dirichlet", bc_value=float(voltage))  # fmt: skip


def resolved_voltages(design: EinzelDesign) -> tuple[float, float, float]:
    """The plates' voltages: the design's, or (0, V_mid, 0) with ``V_mid`` the seed's first
    draw (every design draws it, so the beam does not depend on whether it is used)."""
    if design.voltages is not None:
        return tuple(float(v) for v in design.voltages)  # type: ignore[return-value]
    rng = np.random.default_rng(design.seed)
    return (0.0, float(rng.uniform(*design.v_mid_range)), 0.0)


def einzel_config(design: EinzelDesign = EinzelDesign(), **settings) -> BeamOpticsConfig:
    """The `BeamOpticsConfig` of a lens design (``settings`` override the iteration's)."""
    voltages = resolved_voltages(design)
    rng = np.random.default_rng(design.seed)
    rng.uniform(*design.v_mid_range)  # V_mid's draw, made whether or not it is used
    beam = einzel_beam(design, rng)
    neumann = FieldBoundaryCondition.neumann(0.0)
    params = {"iterations": 20, "tolerance": 1e-3, "relaxation": 1.0, **settings}
    return BeamOpticsConfig(
        grid=GridParams(ndim=2, num_gridpoints=design.shape, lower_bound=(0.0, 0.0),
                        upper_bound=(design.length, design.radius), coordinates="cylindrical"),
        bcs_field=FieldBCs(neumann, neumann, neumann, neumann),
        objects={f"plate{k}": _plate(c, design, v)
                 for k, (c, v) in enumerate(zip(design.centres, voltages, strict=True))},
        beams=[beam],
        diagnostic_planes=list(design.planes),
        **params,
    )  # fmt: skip


# -- the batched design sweep -----------------------------------------------------------------

#: The meshes of the sweep's candidates (nodes along x, r) on 80 x 20 mm.
SWEEP_MESHES = ((257, 65), (513, 129), (1025, 257))


def sweep_designs(count: int = 256, seed: int = 5) -> list[EinzelDesign]:
    """Candidate lenses drawn from ``numpy.random.default_rng(seed)``: per candidate
    ``V_mid`` in U(3, 12) kV, aperture in U(3, 7) mm, plate gap in U(10, 25) mm about the
    middle plate at 40 mm, beam current in U(0.1, 2) mA, one of `SWEEP_MESHES`, and
    U{2000..20000} trajectories."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        v_mid = float(rng.uniform(3e3, 12e3))
        aperture = float(rng.uniform(3e-3, 7e-3))
        gap = float(rng.uniform(10e-3, 25e-3))
        current = float(rng.uniform(0.1e-3, 2e-3))
        shape = SWEEP_MESHES[int(rng.integers(len(SWEEP_MESHES)))]
        trajectories = int(rng.integers(2000, 20001))
        out.append(EinzelDesign(shape=shape, centres=(40e-3 - gap, 40e-3, 40e-3 + gap),
                                aperture=aperture, voltages=(0.0, v_mid, 0.0),
                                current=current, trajectories=trajectories, seed=seed + 1 + k))
    return out


def design_cost(design: EinzelDesign) -> float:
    """The relative cost of solving a candidate: its nodes times its trajectories."""
    return float(design.shape[0] * design.shape[1]) * float(design.trajectories)


def share_of_designs(designs: list[EinzelDesign], rank: int, world: int) -> list[int]:
    """The candidates one of ``world`` ranks solves: the longest first, each to the rank
    with the least work so far (ties to the lower rank) -- every candidate exactly once,
    no collective needed to agree on it."""
    load = [0.0] * world
    mine = []
    for k in sorted(range(len(designs)), key=lambda i: (-design_cost(designs[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += design_cost(designs[k])
        if r == rank:
            mine.append(k)
    return sorted(mine)


def evaluate_design(design: EinzelDesign, plane: float = 79e-3, **settings) -> dict:
    """Solve a candidate to convergence; its beam moments at ``plane`` and its stats."""
    from beamtracer_b200.model import BeamOptics

    model = BeamOptics(einzel_config(design, **settings)).run()
    moments = model.beam_moments(plane)
    return {"current": moments.current, "rms_size": moments.rms_size,
            "rms_angle": moments.rms_angle, "emittance": moments.emittance,
            "iterations": len(model.state.history), "converged": model.stats["converged"]}  # fmt: skip


def sweep(designs: list[EinzelDesign], rank: int = 0, world: int = 1, concurrency: int = 1,
          **settings) -> dict[int, dict]:  # fmt: skip
    """This rank's share of the candidates (`share_of_designs`):
    ``{candidate index: evaluate_design(...)}``.  With ``concurrency`` > 1 that many host
    threads solve candidates at once, each on its own CUDA stream and library context, so
    one candidate's trace overlaps another's field solve on the same GPU; every solve is
    deterministic, so the results do not depend on it.  Ranks need no collective; a caller
    that wants every result gathers the dictionaries."""
    mine = share_of_designs(designs, rank, world)
    if concurrency <= 1:
        return {k: evaluate_design(designs[k], **settings) for k in mine}
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch

    device = torch.cuda.current_device()
    local = threading.local()

    def solve(k: int) -> tuple[int, dict]:
        torch.cuda.set_device(device)
        if getattr(local, "stream", None) is None:
            local.stream = torch.cuda.Stream()
        with torch.cuda.stream(local.stream):
            result = evaluate_design(designs[k], **settings)
        local.stream.synchronize()
        return k, result

    # the costliest first, so the threads finish together
    order = sorted(mine, key=lambda k: -design_cost(designs[k]))
    with ThreadPoolExecutor(max_workers=concurrency) as pool:
        return dict(sorted(pool.map(solve, order)))


# -- design gradients (central differences through the solver) --------------------------------

#: The design parameters of a gradient: the three plate voltages and the beam current.
GRADIENT_PARAMETERS = ("v1", "v2", "v3", "current")


def _perturbed(design: EinzelDesign, parameter: str, delta: float) -> EinzelDesign:
    voltages = list(resolved_voltages(design))
    if parameter == "current":
        return replace(design, voltages=tuple(voltages), current=design.current + delta)
    voltages[GRADIENT_PARAMETERS.index(parameter)] += delta
    return replace(design, voltages=tuple(voltages))


def _evaluate_all(designs: list[EinzelDesign], plane: float, concurrency: int,
                  **settings) -> list[dict]:  # fmt: skip
    """`evaluate_design` of every design, ``concurrency`` at once on their own streams."""
    if concurrency <= 1:
        return [evaluate_design(d, plane, **settings) for d in designs]
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch

    device = torch.cuda.current_device()
    local = threading.local()

    def solve(design: EinzelDesign) -> dict:
        torch.cuda.set_device(device)
        if getattr(local, "stream", None) is None:
            local.stream = torch.cuda.Stream()
        with torch.cuda.stream(local.stream):
            result = evaluate_design(design, plane, **settings)
        local.stream.synchronize()
        return result

    with ThreadPoolExecutor(max_workers=concurrency) as pool:
        return list(pool.map(solve, designs))


def design_gradient(design: EinzelDesign, plane: float = 79e-3, rel_step: float = 1e-4,
                    tolerance: float = 1e-7, iterations: int = 60,
                    concurrency: int = 1) -> dict:  # fmt: skip
    """The gradients of the rms angle and the current at ``plane`` with respect to
    `GRADIENT_PARAMETERS`, by central differences of converged solves: voltage steps of
    ``rel_step`` times the largest plate voltage, a current step of ``rel_step`` times the
    current; every solve converged to ``tolerance`` [V] (tighter than the steps' effect).
    The 2 x 4 solves are independent: ``concurrency`` of them run at once, each on its own
    stream (the results do not depend on it)."""
    scale = max(abs(v) for v in resolved_voltages(design))
    steps = [rel_step * (design.current if name == "current" else scale)
             for name in GRADIENT_PARAMETERS]  # fmt: skip
    designs = []
    for name, step in zip(GRADIENT_PARAMETERS, steps, strict=True):
        designs += [_perturbed(design, name, step), _perturbed(design, name, -step)]
    results = _evaluate_all(designs, plane, concurrency, tolerance=tolerance,
                            iterations=iterations)  # fmt: skip
    out = {"rms_angle": np.zeros(len(GRADIENT_PARAMETERS)),
           "current": np.zeros(len(GRADIENT_PARAMETERS)), "solves": len(designs)}  # fmt: skip
    for k, step in enumerate(steps):
        plus, minus = results[2 * k], results[2 * k + 1]
        out["rms_angle"][k] = (plus["rms_angle"] - minus["rms_angle"]) / (2.0 * step)
        out["current"][k] = (plus["current"] - minus["current"]) / (2.0 * step)
    return out
