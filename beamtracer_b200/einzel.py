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

from dataclasses import dataclass

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


def einzel_config(design: EinzelDesign = EinzelDesign(), **settings) -> BeamOpticsConfig:
    """The `BeamOpticsConfig` of a lens design (``settings`` override the iteration's)."""
    rng = np.random.default_rng(design.seed)
    voltages = design.voltages
    if voltages is None:
        voltages = (0.0, float(rng.uniform(*design.v_mid_range)), 0.0)
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
