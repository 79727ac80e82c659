"""Design gradients and the batched sweep through the device solver.

The gradient of the rms angle and the current at the last plane with respect to the plate
voltages and the beam current, by central differences of converged solves of the lens at
401 x 101 with 8,000 rings, must equal the oracle's central differences of its own
converged solves: the two solvers agree to about 1e-12 per solve, far inside what a 1e-4
step resolves.
"""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.einzel import (
    GRADIENT_PARAMETERS,
    EinzelDesign,
    _perturbed,
    design_gradient,
    einzel_config,
    evaluate_design,
    resolved_voltages,
    sweep,
    sweep_designs,
)

pytestmark = pytest.mark.gpu

#: The differentiation workload: the lens at 401 x 101 with 8,000 rings (seed 2).
C4 = EinzelDesign(shape=(401, 101), trajectories=8000, seed=2)


def _oracle_moments(design: EinzelDesign, plane: float, tolerance: float, iterations: int):
    """The oracle's converged moments at ``plane``, its problem built on the host alone."""
    from scipy import constants

    from beamtracer_b200.diagnostics import plane_moments
    from beamtracer_b200.tracer import PlaneHits
    from oracle import vlasov as oracle_vlasov
    from tests.vlasov_cases import config_problem

    config = einzel_config(design, tolerance=tolerance, iterations=iterations)
    problem, particles, j_over_v = config_problem(config)
    out = oracle_vlasov.vlasov(problem, particles, j_over_v, iterations=iterations,
                               tolerance=tolerance)  # fmt: skip
    k = list(problem.planes).index(plane)
    point, velocity, current, species, direction = oracle_vlasov.plane_hits(
        problem, out["trace"], particles.current, particles.species)[k]  # fmt: skip
    hits = PlaneHits(plane, point, velocity, current, species, direction)
    mass = np.array([b.mass for b in config.beams]) * constants.atomic_mass
    return plane_moments(hits, cylindrical=True, mass=mass)


def test_gradient_matches_the_oracle_central_differences():
    plane, tol, its, rel = 79e-3, 1e-7, 60, 1e-4
    gpu = design_gradient(C4, plane, rel_step=rel, tolerance=tol, iterations=its)
    assert gpu["solves"] == 2 * len(GRADIENT_PARAMETERS)
    scale = max(abs(v) for v in resolved_voltages(C4))
    for k, name in enumerate(GRADIENT_PARAMETERS):
        step = rel * (C4.current if name == "current" else scale)
        plus = _oracle_moments(_perturbed(C4, name, step), plane, tol, its)
        minus = _oracle_moments(_perturbed(C4, name, -step), plane, tol, its)
        angle = (plus.rms_angle - minus.rms_angle) / (2 * step)
        current = (plus.current - minus.current) / (2 * step)
        assert gpu["rms_angle"][k] == pytest.approx(angle, rel=1e-5, abs=1e-12), name
        assert gpu["current"][k] == pytest.approx(current, rel=1e-5, abs=1e-12), name
    assert np.all(np.isfinite(gpu["rms_angle"])) and gpu["rms_angle"][1] != 0.0
    concurrent = design_gradient(C4, plane, rel_step=rel, tolerance=tol, iterations=its,
                                 concurrency=8)  # fmt: skip
    np.testing.assert_array_equal(concurrent["rms_angle"], gpu["rms_angle"])
    np.testing.assert_array_equal(concurrent["current"], gpu["current"])


def test_sweep_solves_this_ranks_share():
    designs = [EinzelDesign(shape=(129, 33), trajectories=300, seed=9 + k,
                            voltages=(0.0, 4e3 + 1e3 * k, 0.0)) for k in range(3)]  # fmt: skip
    results = sweep(designs, rank=0, world=1)
    assert sorted(results) == [0, 1, 2]
    again = evaluate_design(designs[1])
    assert results[1] == again  # deterministic
    assert all(r["current"] > 0 for r in results.values())


def test_sweep_candidates_solve():
    design = sweep_designs(4)[0]
    small = EinzelDesign(**{**design.__dict__, "shape": (129, 33), "trajectories": 300})
    result = evaluate_design(small)
    assert np.isfinite(result["rms_angle"])


def test_concurrent_sweep_equals_the_sequential_one():
    """Three candidates solved at once on three streams give the sequential results bit
    for bit (every solve is deterministic and keeps to its own stream)."""
    designs = [EinzelDesign(shape=((129, 33), (257, 65))[k % 2], trajectories=300 + 100 * k,
                            seed=20 + k, voltages=(0.0, 3e3 + 1e3 * k, 0.0)) for k in range(5)]  # fmt: skip
    sequential = sweep(designs)
    concurrent = sweep(designs, concurrency=3)
    assert concurrent == sequential
