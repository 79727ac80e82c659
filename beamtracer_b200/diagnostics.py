"""Beam quantities at a diagnostic plane: current, rms sizes and angles, emittance, Twiss.

The interface of the reference's ``solver/diagnostics.py`` (``BeamMoments``,
``plane_moments``, ``mismatch``; ``diagnostics.py:15-170``).  The moments are weighted by
the crossings' currents.  A ring (cylindrical geometry) is projected on one transverse
plane and averaged over its azimuth, which gives, without dividing by the radius,

    <x^2> = <y^2 + z^2> / 2,   <x x'> = <(y v_y + z v_z) / v_x> / 2,
    <x'^2> = <(v_y^2 + v_z^2) / v_x^2> / 2

(the rotation to (v_r, v_theta) keeps v_y^2 + v_z^2, and r v_r = y v_y + z v_z); planar
moments are taken about the means.  The rms ellipse of the 2 x 2 second-moment matrix gives
the emittance (the square root of its determinant) and the Twiss parameters.
"""

from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np
from scipy import constants


@dataclass(frozen=True)
class BeamMoments:
    """Current-weighted second moments of a beam in one transverse plane."""

    current: float
    rms_size: float
    rms_angle: float
    correlation: float
    emittance: float
    normalized_emittance: float
    alpha: float
    beta: float
    gamma: float
    mean_energy: float
    count: int

    def as_dict(self) -> dict[str, float]:
        return {f.name: getattr(self, f.name) for f in fields(self)}


def _empty_moments() -> BeamMoments:
    """No crossings, or no current: zero current and count, every moment NaN."""
    nan = float("nan")
    return BeamMoments(0.0, *([nan] * 9), 0)


def _second_moments(weight: np.ndarray, point: np.ndarray, velocity: np.ndarray,
                    cylindrical: bool, axis: str) -> tuple[float, float, float]:  # fmt: skip
    """``(<x^2>, <x x'>, <x'^2>)`` of the crossings under the normalised weights."""

    def mean(values: np.ndarray) -> float:
        return float(np.dot(weight, values))

    vx = velocity[0]
    if cylindrical:
        y, z = point[1], point[2]
        vy, vz = velocity[1], velocity[2]
        return (0.5 * mean(y * y + z * z), 0.5 * mean((y * vy + z * vz) / vx),
                0.5 * mean((vy * vy + vz * vz) / (vx * vx)))  # fmt: skip
    if axis not in ("y", "z"):
        raise ValueError(f"axis must be 'y' or 'z', got {axis!r}")
    k = 1 if axis == "y" else 2
    u = point[k]
    slope = velocity[k] / vx
    du, dslope = u - mean(u), slope - mean(slope)
    return mean(du * du), mean(du * dslope), mean(dslope * dslope)


def plane_moments(hits, *, cylindrical: bool, mass, species: int | None = None,
                  forward_only: bool = True, axis: str = "y") -> BeamMoments:  # fmt: skip
    """The `BeamMoments` of the crossings ``hits`` (a `PlaneHits`) of a plane.

    ``mass`` [kg] per species (indexed by ``hits.species``) or one value; only ``species``
    and, with ``forward_only``, crossings in the +x direction count.  No crossings or no
    current give NaN moments; a zero emittance gives NaN Twiss parameters.
    """
    keep = np.ones(np.shape(hits.current), dtype=bool)
    if species is not None:
        keep &= np.asarray(hits.species) == species
    if forward_only:
        keep &= np.asarray(hits.direction) > 0
    current = np.abs(np.asarray(hits.current, dtype=float)[keep])
    total = float(current.sum())
    if total == 0.0:
        return _empty_moments()
    weight = current / total
    point = np.asarray(hits.point, dtype=float)[:, keep]
    velocity = np.asarray(hits.velocity, dtype=float)[:, keep]
    xx, xp, pp = _second_moments(weight, point, velocity, cylindrical, axis)
    emittance = float(np.sqrt(max(xx * pp - xp * xp, 0.0)))

    # relativistic factors of every crossing (NaN at or above the speed of light)
    speed2 = np.einsum("ij,ij->j", velocity, velocity)
    with np.errstate(invalid="ignore", divide="ignore"):
        lorentz = 1.0 / np.sqrt(1.0 - speed2 / constants.c**2)
    masses = np.asarray(mass, dtype=float)
    m = masses[np.asarray(hits.species)[keep]] if masses.ndim else masses
    # (gamma - 1) m c^2 in a form without cancellation at low speed
    kinetic = m * lorentz * lorentz * speed2 / (lorentz + 1.0) / constants.e
    beta_gamma = float(np.dot(weight, lorentz * velocity[0])) / constants.c
    if emittance > 0.0:
        alpha, beta, gamma = -xp / emittance, xx / emittance, pp / emittance
    else:
        alpha = beta = gamma = float("nan")
    return BeamMoments(
        current=total, rms_size=float(np.sqrt(xx)), rms_angle=float(np.sqrt(pp)),
        correlation=float(xp), emittance=emittance,
        normalized_emittance=emittance * beta_gamma, alpha=float(alpha), beta=float(beta),
        gamma=float(gamma), mean_energy=float(np.dot(weight, kinetic)), count=int(current.size),
    )  # fmt: skip


def mismatch(alpha: float, beta: float, alpha0: float, beta0: float) -> float:
    """The mismatch parameter of a beam (alpha, beta) against the design (alpha0, beta0)
    (Midttun et al., IPAC'17, eq. 1; the interface of ``diagnostics.py:138-170``): with
    ``R = (beta gamma0 + beta0 gamma) / 2 - alpha alpha0``, ``M = sqrt(R + sqrt(R^2 - 1)) - 1``,
    evaluated through ``D = 2 (R - 1)`` so that a matched beam gives exactly 0."""
    g, g0 = (1.0 + alpha * alpha) / beta, (1.0 + alpha0 * alpha0) / beta0
    d = (alpha - alpha0) ** 2 - (g - g0) * (beta - beta0)
    return float(np.sqrt(1.0 + 0.5 * (d + np.sqrt(d * (d + 4.0)))) - 1.0)
