"""Beam quantities at a diagnostic plane: current, rms sizes and angles, emittance, Twiss.

The interface of the reference's ``solver/diagnostics.py`` (``BeamMoments``,
``plane_moments``, ``mismatch``; ``diagnostics.py:15-170``): current-weighted moments over
the forward crossings of a plane, in cylindrical geometry of every ring projected on one
transverse plane (``<x^2> = <r^2>/2``, ``<x'^2> = <r'^2 + a'^2>/2``, ``<x x'> = <r r'>/2``),
in planar geometry about the means.
"""

from __future__ import annotations

from dataclasses import dataclass

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
        return dict(self.__dict__)


def plane_moments(hits, *, cylindrical: bool, mass, species: int | None = None,
                  forward_only: bool = True, axis: str = "y") -> BeamMoments:  # fmt: skip
    """The `BeamMoments` of the crossings ``hits`` (a `PlaneHits`) of a plane.

    ``mass`` [kg] per species (indexed by ``hits.species``) or one value; only ``species``
    and, with ``forward_only``, crossings in the +x direction count.  No crossings or no
    current give NaN moments, zero emittance NaN Twiss parameters.
    """
    keep = np.ones(hits.current.size, dtype=bool)
    if species is not None:
        keep &= hits.species == species
    if forward_only:
        keep &= hits.direction > 0
    w = np.abs(hits.current[keep])
    point = hits.point[:, keep]
    vel = hits.velocity[:, keep]
    masses = np.asarray(mass, dtype=float)
    m = masses[hits.species[keep]] if masses.ndim else np.full(w.size, float(masses))
    total = float(w.sum())
    if w.size == 0 or total == 0.0:
        nan = float("nan")
        return BeamMoments(0.0, nan, nan, nan, nan, nan, nan, nan, nan, nan, 0)
    vx = vel[0]
    if cylindrical:
        r = np.hypot(point[1], point[2])
        with np.errstate(invalid="ignore", divide="ignore"):
            cy = np.where(r > 0, point[1] / r, 1.0)
            cz = np.where(r > 0, point[2] / r, 0.0)
        vr = vel[1] * cy + vel[2] * cz
        vt = vel[2] * cy - vel[1] * cz
        rp, ap = vr / vx, vt / vx
        xx = np.sum(w * r * r) / (2.0 * total)
        pp = np.sum(w * (rp * rp + ap * ap)) / (2.0 * total)
        xp = np.sum(w * r * rp) / (2.0 * total)
    else:
        if axis not in ("y", "z"):
            raise ValueError(f"axis must be 'y' or 'z', got {axis!r}")
        a = 1 if axis == "y" else 2
        y = point[a]
        yp = vel[a] / vx
        my = np.sum(w * y) / total
        myp = np.sum(w * yp) / total
        xx = np.sum(w * (y - my) ** 2) / total
        pp = np.sum(w * (yp - myp) ** 2) / total
        xp = np.sum(w * (y - my) * (yp - myp)) / total
    emittance = float(np.sqrt(max(xx * pp - xp * xp, 0.0)))
    speed2 = np.sum(vel * vel, axis=0)
    with np.errstate(invalid="ignore", divide="ignore"):
        lorentz = 1.0 / np.sqrt(1.0 - speed2 / constants.c**2)
    beta_gamma = float(np.sum(w * lorentz * vx) / total) / constants.c
    energy = m * lorentz**2 * speed2 / (lorentz + 1.0) / constants.e
    twiss = (-xp, xx, pp) if emittance > 0 else (np.nan, np.nan, np.nan)
    scale = emittance if emittance > 0 else 1.0
    return BeamMoments(
        current=total,
        rms_size=float(np.sqrt(xx)),
        rms_angle=float(np.sqrt(pp)),
        correlation=float(xp),
        emittance=emittance,
        normalized_emittance=emittance * beta_gamma,
        alpha=float(twiss[0] / scale),
        beta=float(twiss[1] / scale),
        gamma=float(twiss[2] / scale),
        mean_energy=float(np.sum(w * energy) / total),
        count=int(w.size),
    )


def mismatch(alpha: float, beta: float, alpha0: float, beta0: float) -> float:
    """The mismatch parameter of a beam (alpha, beta) against the design (alpha0, beta0)
    (Midttun et al., IPAC'17, eq. 1; ``diagnostics.py:138-170``)."""
    gamma = (1.0 + alpha**2) / beta
    gamma0 = (1.0 + alpha0**2) / beta0
    delta = (alpha - alpha0) ** 2 - (gamma - gamma0) * (beta - beta0)
    return float(np.sqrt(1.0 + (delta + np.sqrt(delta * (delta + 4.0))) / 2.0) - 1.0)
