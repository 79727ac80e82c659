"""Design gradients and the batched sweep through the device solver.

The gradient of the rms angle and the current at the last plane with respect to the plate
voltages and the beam current, by central differences of converged solves of the lens at
401 x 101 with 8,000 rings, must equal the oracle's central differences of its own
converged solves: the two solvers agree to about 1e-12 per solve, far inside what a 1e-4
step resolves.  The adjoint of one converged solve (``beamtracer_b200.adjoint``) must give
both within 1e-4.
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


PLANE, TOL, ITS, REL = 79e-3, 1e-7, 60, 1e-4


@pytest.fixture(scope="module")
def gpu_fd():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    return design_gradient(C4, PLANE, rel_step=REL, tolerance=TOL, iterations=ITS)


@pytest.fixture(scope="module")
def oracle_fd():
    scale = max(abs(v) for v in resolved_voltages(C4))
    out = {"rms_angle": np.zeros(4), "current": np.zeros(4)}
    for k, name in enumerate(GRADIENT_PARAMETERS):
        step = REL * (C4.current if name == "current" else scale)
        plus = _oracle_moments(_perturbed(C4, name, step), PLANE, TOL, ITS)
        minus = _oracle_moments(_perturbed(C4, name, -step), PLANE, TOL, ITS)
        out["rms_angle"][k] = (plus.rms_angle - minus.rms_angle) / (2 * step)
        out["current"][k] = (plus.current - minus.current) / (2 * step)
    return out


def test_gradient_matches_the_oracle_central_differences(gpu_fd, oracle_fd):
    assert gpu_fd["solves"] == 2 * len(GRADIENT_PARAMETERS)
    for k, name in enumerate(GRADIENT_PARAMETERS):
        assert gpu_fd["rms_angle"][k] == pytest.approx(oracle_fd["rms_angle"][k], rel=1e-5,
                                                       abs=1e-12), name  # fmt: skip
        assert gpu_fd["current"][k] == pytest.approx(oracle_fd["current"][k], rel=1e-5,
                                                     abs=1e-12), name  # fmt: skip
    assert np.all(np.isfinite(gpu_fd["rms_angle"])) and gpu_fd["rms_angle"][1] != 0.0
    concurrent = design_gradient(C4, PLANE, rel_step=REL, tolerance=TOL, iterations=ITS,
                                 concurrency=8)  # fmt: skip
    np.testing.assert_array_equal(concurrent["rms_angle"], gpu_fd["rms_angle"])
    np.testing.assert_array_equal(concurrent["current"], gpu_fd["current"])


def test_adjoint_gradient_matches_central_differences(gpu_fd, oracle_fd):
    """The adjoint of one converged solve (``torch.autograd`` through the hand-written
    reverse) against the central differences of eight solves, on the device and in the
    oracle: within 1e-4 relative."""
    from beamtracer_b200.adjoint import adjoint_design_gradient

    adjoint = adjoint_design_gradient(C4, PLANE, tolerance=TOL, iterations=ITS)
    assert adjoint["adjoint_iterations"] >= 2
    scale = np.abs(gpu_fd["rms_angle"]).max()
    for k, name in enumerate(GRADIENT_PARAMETERS):
        for fd in (gpu_fd, oracle_fd):
            assert adjoint["rms_angle"][k] == pytest.approx(fd["rms_angle"][k], rel=1e-4,
                                                            abs=1e-6 * scale), name  # fmt: skip
            assert adjoint["current"][k] == pytest.approx(fd["current"][k], rel=1e-4,
                                                          abs=1e-12), name  # fmt: skip


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


def test_lbfgs_search_over_the_middle_plate(tmp_path):
    """L-BFGS over V_mid in [3, 12] kV with the adjoint's gradients lowers the rms angle
    at 79 mm, records every evaluation with its gradient, and a search from that record
    evaluates nothing again."""
    import json

    from beamtracer_b200.optimization import (
        Design,
        Parameter,
        Record,
        einzel_evaluator,
        lbfgs_search,
    )

    base = EinzelDesign(shape=(201, 51), trajectories=400, seed=4)
    design = Design((Parameter("v_mid", 3e3, 12e3),))
    evaluate = einzel_evaluator(base, ("v_mid",))
    path = tmp_path / "lbfgs.jsonl"
    result = lbfgs_search(design, evaluate, {"v_mid": 5e3}, objective="rms_angle",
                          record=Record(design, path), max_evaluations=8)  # fmt: skip
    first = result.evaluations[0]
    assert first.ok and result.best.ok
    assert result.best.objectives["rms_angle"] < first.objectives["rms_angle"]
    lines = [json.loads(x) for x in path.read_text().splitlines()]
    assert len(lines) == result.computed >= 2
    assert all(x["converged"] and "gradient" in x["diagnostics"] for x in lines)
    again = lbfgs_search(design, evaluate, {"v_mid": 5e3}, objective="rms_angle",
                         record=Record(design, path), max_evaluations=8)  # fmt: skip
    assert again.computed == 0
