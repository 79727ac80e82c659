"""Seeded cases of the host-side functions both the device path and the oracle share: the
beam seeding, the plane moments and the axisymmetric magnetic field.

``make_golden.py`` runs the reference's own functions on them; ``tests/test_host_goldens.py``
runs this package's on the same cases and compares.
"""

from __future__ import annotations

import numpy as np

#: beam_with_energy cases: (positional args, keyword args).  The generator case is drawn
#: with ``numpy.random.default_rng(seed)`` passed as ``sampling``.
BEAM_CASES = {
    "line_cyl": ((200, 50.0, 1.0, 1.007276, 5.0, 0.0, 0.5, (0.0, 0.0), (0.0, 0.9e-3)),
                 {"cylindrical": True}),
    "line_planar": ((40, 10.0, 1.0, 1.007276, 0.01, 0.0, 0.0, (0.0, 0.0), (0.0, 5e-3)),
                    {"cylindrical": False}),
    "slanted_warm": ((333, 120.0, -1.0, 1.00794, 30.0, 0.2, 1.5, (1e-3, 2e-3), (3e-3, -1e-3)),
                     {"cylindrical": False, "species": 2}),
    "relativistic": ((64, 5.0, 1.0, 1.0, 2.0e6, 10.0, 25.0, (0.0, 0.0), (0.0, 4e-3)),
                     {"cylindrical": True, "relativistic": True}),
    "generator": ((500, 300.0, 1.0, 1.007276, 5.0, 0.0, 1.0, (0.0, 3.5e-3), (0.0, 6.5e-3)),
                  {"cylindrical": False, "seed": 3}),
}  # fmt: skip


def moment_hits(seed: int, cylindrical: bool, n: int = 400) -> dict[str, np.ndarray]:
    """Seeded plane crossings: points, velocities, currents (some negative), species (0-2)
    and directions (mostly forward)."""
    rng = np.random.default_rng(seed)
    if cylindrical:
        r = rng.uniform(0.0, 3e-3, n)
        phase = rng.uniform(0.0, 2 * np.pi, n)
        point = np.stack([np.full(n, 0.079), r * np.cos(phase), r * np.sin(phase)])
        point[1:, :3] = 0.0  # crossings on the axis
    else:
        point = np.stack([np.full(n, 0.04), rng.normal(5e-3, 1e-3, n), rng.normal(0, 5e-4, n)])
    vx = rng.uniform(1.3e6, 1.4e6, n)
    velocity = np.stack([vx, rng.normal(0.0, 7e3, n) + 2e6 * point[1],
                         rng.normal(0.0, 4e3, n)])  # fmt: skip
    current = rng.uniform(0.5, 1.5, n) * 1e-7 * np.where(rng.uniform(size=n) < 0.1, -1, 1)
    species = rng.integers(0, 3, n).astype(np.int32)
    direction = np.where(rng.uniform(size=n) < 0.08, -1, 1).astype(np.int8)
    return {"point": point, "velocity": velocity, "current": current, "species": species,
            "direction": direction}  # fmt: skip


#: plane_moments cases: (hit seed, cylindrical, species, forward_only, axis, mass kind)
MOMENT_CASES = {
    "cyl_all": (11, True, None, True, "y", "array"),
    "cyl_species1": (11, True, 1, True, "y", "array"),
    "cyl_both_ways": (12, True, None, False, "y", "scalar"),
    "planar_y": (13, False, None, True, "y", "array"),
    "planar_z": (13, False, 2, True, "z", "scalar"),
    "planar_fast": (14, False, None, True, "y", "array"),  # relativistic speeds
}

#: Masses [kg] of the three species.
MOMENT_MASSES = np.array([1.007276, 1.00794, 4.0026]) * 1.66053906892e-27

#: AxisymmetricMagneticField cases: (centre, length, radius, peak, z0, hz, samples, order)
FIELD_CASES = {
    "order1": (20e-3, 40e-3, 10e-3, 0.2, -0.4e-3, 0.05e-3, 900, 1),
    "order3": (5e-3, 4e-3, 3e-3, 0.5, -0.3e-3, 0.05e-3, 180, 3),
    "order6": (0.0, 30e-3, 8e-3, -1.1, -30e-3, 0.25e-3, 241, 6),
}


def field_points(seed: int, z0: float, hz: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Points inside and beyond the sampled profile, radii up to 4 mm."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(z0 - 5 * hz, z0 + (n + 4) * hz, 600)
    r = rng.uniform(0.0, 4e-3, 600)
    r[:5] = 0.0
    return z, r


#: A configuration's solenoid sampling: (x_min, x_max, node spacing, solenoids, order).
SAMPLING_CASE = (0.0, 8e-3, 0.1e-3, ((5e-3, 4e-3, 3e-3, 0.5), (6.5e-3, 2e-3, 1e-3, -0.1)), 3)


#: Designs for the record's keys: (parameters (name, lower, upper), points to key).
RECORD_DESIGNS = {
    "v_mid": ((("v_mid", 3e3, 12e3),), [[3e3], [7.123456789e3], [12e3], [5.5e3 + 1e-9]]),
    "lens": ((("v_mid", 3e3, 12e3), ("aperture", 3e-3, 7e-3), ("gap", 10e-3, 25e-3)),
             [[4e3, 5e-3, 12e-3], [11.9e3, 3e-3, 25e-3], [7e3, 6.999999e-3, 17.5e-3]]),
}  # fmt: skip

#: The design whose evaluations make the reference record.
RECORD_CASE = "lens"


def record_evaluations(names, points) -> list[dict]:
    """Evaluations of the record case: objectives, a constraint, flags and diagnostics,
    one failed evaluation and one with a non-finite objective."""
    out = []
    for k, x in enumerate(points):
        values = dict(zip(names, map(float, x), strict=True))
        out.append({
            "objectives": {"rms_angle": 1e-3 * (k + 1), "emittance": 2e-6 / (k + 1)},
            "constraints": {"transmission": 0.05 * k - 0.05},
            "converged": k != 1, "wall_time": 0.25 * k,
            "failure": "RuntimeError: no convergence" if k == 1 else None,
            "diagnostics": {"iterations": 7 + k, "note": f"case {k}", "ok_flag": True,
                            "current": float("nan") if k == 2 else 1e-3},
            "parameters": values, "generation": None if k == 0 else k,
        })  # fmt: skip
    return out
