"""``BeamOptics(config).run()`` on the B200 against the oracle's Vlasov iteration.

Per iteration the GPU and the oracle trace the same beam through potentials that agree
to the field solves' tolerance, so the charge densities agree to about 1e-10 of their
largest value; the converged potentials and plane moments agree to well inside 1e-6.
The reference's own known answers (Child--Langmuir, the current at the plane) hold.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import vlasov as oracle_vlasov
from tests.vlasov_cases import child_langmuir_density, diode, extraction, oracle_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def beam_optics():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200 import BeamOptics

    return BeamOptics


def _run_both(model, iterations, **kwargs):
    gpu_states = []
    model.run(lambda it, state: gpu_states.append(
        (state.potential.copy(), state.charge_density.copy())))  # fmt: skip
    problem = oracle_problem(model)
    particles, j_over_v = model._particles()
    ora = []
    oracle_vlasov.vlasov(problem, particles, j_over_v, iterations=iterations,
                         tolerance=model.config.tolerance, relaxation=model.config.relaxation,
                         callback=lambda it, out: ora.append(
                             (out["potential"].copy(), out["charge_density"].copy())),
                         **kwargs)  # fmt: skip
    return gpu_states, ora


def test_diode_iterations_match_the_oracle(beam_optics):
    config = diode(current_density=10.0, iterations=6, tolerance=0.0, relaxation=0.5)
    model = beam_optics(config)
    gpu, ora = _run_both(model, 6)
    assert len(gpu) == len(ora) == 6
    for (phi_g, rho_g), (phi_o, rho_o) in zip(gpu, ora):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-9 * 1000.0)
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-10 * np.abs(rho_o).max())


def test_child_langmuir_diode(beam_optics):
    """phi = -V (x/d)^(4/3) at the Child--Langmuir density (test_beam_optics.py:107-134)."""
    d, voltage = 10e-3, 1000.0
    j_cl = child_langmuir_density(d, voltage)
    model = beam_optics(diode(current_density=0.95 * j_cl, iterations=60, relaxation=0.5,
                              tolerance=1e-3))  # fmt: skip
    model.run()
    assert model.stats["converged"]
    assert model.stats["transmitted"] == 40
    x = model.mesh.x
    phi = model.potential[:, 10]
    inside = (x > 1e-3) & (x < 9e-3)
    assert np.all(phi[inside] > -voltage * x[inside] / d)
    cl = -voltage * (x[inside] / d) ** (4 / 3)
    assert np.max(np.abs(phi[inside] - cl)) < 0.06 * voltage
    moments = model.beam_moments(9.9e-3)
    assert moments.current == pytest.approx(0.95 * j_cl * 5e-3, rel=1e-6)


def test_extraction_with_plasma_matches_the_oracle(beam_optics):
    config = extraction(1.0, iterations=5, tolerance=0.0)
    model = beam_optics(config)
    gpu, ora = _run_both(model, 5, plasma=oracle_vlasov.Plasma(5.0, 5.0, 0.6e-3, -1))
    for k, ((phi_g, rho_g), (phi_o, rho_o)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-7 * 2000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-7 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip
    stats = model.stats
    assert stats["transmitted"] > 0


def test_negative_extraction_mirrors_positive(beam_optics):
    """Boltzmann ions about -U_p for negative ions are Boltzmann electrons about U_p."""
    from beamtracer_b200.config import NegativeExtractionPlasma

    positive = beam_optics(extraction(1.0)).run()
    negative_config = extraction(-1.0).replace(plasma=NegativeExtractionPlasma(5.0, -5.0, 0.6e-3))
    negative = beam_optics(negative_config).run()
    assert negative.stats == positive.stats
    assert negative.stats["converged"]
    np.testing.assert_allclose(negative.potential, -positive.potential, rtol=0, atol=1e-7)
    a, b = positive.beam_moments(7.5e-3), negative.beam_moments(7.5e-3)
    assert a.current == pytest.approx(b.current)
    assert a.emittance == pytest.approx(b.emittance, rel=1e-6)


@pytest.mark.parametrize("integrator", ["rk4", "boris"])
def test_extraction_through_a_solenoid_matches_the_oracle(beam_optics, integrator):
    """The plasma extraction case inside a solenoid: the trace takes the reference's
    NumPy tracer's magnetic step, every electrode cell decided by the exact inside test."""
    from beamtracer_b200.config import Solenoid

    config = extraction(1.0, iterations=4, tolerance=0.0, integrator=integrator,
                        solenoids=[Solenoid(5e-3, 4e-3, 3e-3, 0.5)])  # fmt: skip
    model = beam_optics(config)
    assert model.tracer.magnetic is not None
    gpu, ora = _run_both(model, 4, plasma=oracle_vlasov.Plasma(5.0, 5.0, 0.6e-3, -1))
    for k, ((phi_g, rho_g), (phi_o, rho_o)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-7 * 2000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-7 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip
    assert model.stats["transmitted"] > 0


def test_solenoid_extraction_matches_the_oracle():
    """The planar plasma + solenoid workload (x-graded mesh, Newton solve, Boris step in
    the solenoid's field) on a coarse mesh: every iteration against the oracle."""
    from beamtracer_b200.solenoid_extraction import SolenoidExtractionDesign, solenoid_extraction
    from tests.vlasov_cases import mesh_problem

    case = solenoid_extraction(SolenoidExtractionDesign().small())
    gpu = []
    case.run(lambda it, state: gpu.append((state.potential.copy(), state.charge_density.copy())),
             iterations=3, tolerance=0.0)  # fmt: skip
    problem = mesh_problem(case.mesh, integrator=1, magnetic=case.magnetic)
    d = case.design
    ora = []
    oracle_vlasov.vlasov(problem, case.particles, case.j_over_v, iterations=3,
                         relaxation=d.relaxation,
                         plasma=oracle_vlasov.Plasma(d.electron_temperature, d.plasma_potential,
                                                     d.plasma_x, -1, density=case.plasma.rho_e),
                         callback=lambda it, out: ora.append(
                             (out["potential"].copy(), out["charge_density"].copy())))  # fmt: skip
    assert len(gpu) == len(ora) == 3
    for k, ((phi_g, rho_g), (phi_o, rho_o)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-7 * 1e4, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-7 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip
