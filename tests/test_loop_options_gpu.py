"""The Vlasov loop's options on the device against the oracle: Anderson mixing, the
space-charge compensation, the coarse-particle phase and the density stopping rule.

The oracle restates the reference's loop (``solver/vlasov.py:327-427``), its Anderson
mixer with NumPy's ``lstsq(rcond=1e-10)`` (``vlasov.py:138-173``), ``compensate``
(``vlasov.py:176-184``) and ``thin_particles`` (``vlasov.py:202-215``).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import vlasov as oracle_vlasov
from tests.vlasov_cases import diode, extraction, oracle_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def beam_optics():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200 import BeamOptics

    return BeamOptics


def _iterations(model, iterations, run_kwargs=None, **oracle_kwargs):
    gpu = []
    model.run(lambda it, state: gpu.append((state.potential.copy(), state.charge_density.copy(),
                                            state.history[-1]["trajectories"])),
              **(run_kwargs or {}))  # fmt: skip
    particles, j_over_v = model._particles()
    config = model.config
    ora = []
    oracle_vlasov.vlasov(oracle_problem(model), particles, j_over_v, iterations=iterations,
                         tolerance=config.tolerance, relaxation=config.relaxation,
                         callback=lambda it, out: ora.append(
                             (out["potential"].copy(), out["charge_density"].copy(),
                              int(out["trace"].status.size))),
                         **oracle_kwargs)  # fmt: skip
    return gpu, ora


@pytest.mark.parametrize("depth", [1, 3])
def test_device_mixer_equals_lstsq_mixing(depth):
    """Fed the same iterates, the device mixer and the reference's lstsq mixing agree to
    rounding; the ring of iterates wraps and a repeated iterate (a rank-deficient history)
    is cut off as lstsq cuts it."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.vlasov import AndersonMixer

    rng = np.random.default_rng(7)
    n = 5000
    target = rng.normal(size=n)
    device = AndersonMixer(depth, relaxation=0.7)
    host = oracle_vlasov.Anderson(depth, 0.7)
    rho = rng.normal(size=n)
    for step in range(9):
        # a contraction towards `target` with some nonlinearity
        deposit = target + 0.5 * np.tanh(rho - target) + 0.01 * rng.normal(size=n)
        if step == 5:
            deposit = host.xs[-1] + host.fs[-1] if host.xs else deposit  # repeat an iterate
            rho = host.xs[-1].copy()
        want = host.update(rho, deposit)
        got = device.update(torch.from_numpy(rho).cuda(), torch.from_numpy(deposit).cuda())
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0,
                                   atol=1e-10 * np.abs(want).max(), err_msg=f"step {step}")
        rho = want


def test_anderson_iterations_match_the_oracle(beam_optics):
    config = diode(current_density=14.0, iterations=8, tolerance=0.0, relaxation=0.5,
                   mixing="anderson", anderson_depth=3)  # fmt: skip
    gpu, ora = _iterations(beam_optics(config), 8, mixing="anderson", anderson_depth=3)
    assert len(gpu) == len(ora) == 8
    for k, ((phi_g, rho_g, _), (phi_o, rho_o, _)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-9 * 1000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-9 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip


def test_compensation_matches_the_oracle(beam_optics):
    from beamtracer_b200.config import SpaceChargeCompensation

    regions = [SpaceChargeCompensation(2e-3, 6e-3, 0.5), SpaceChargeCompensation(5e-3, 8e-3, 0.3)]
    config = diode(current_density=10.0, iterations=5, tolerance=0.0, relaxation=0.5,
                   compensation=regions)  # fmt: skip
    gpu, ora = _iterations(beam_optics(config), 5,
                           compensation=[(c.x_min, c.x_max, c.fraction) for c in regions])
    for k, ((phi_g, rho_g, _), (phi_o, rho_o, _)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-9 * 1000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-10 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip


def test_coarse_phase_matches_the_oracle(beam_optics):
    config = extraction(1.0, iterations=8, tolerance=0.0, coarse_particles=0.5,
                        coarse_tolerance=5.0)  # fmt: skip
    model = beam_optics(config)
    gpu, ora = _iterations(model, 8, plasma=oracle_vlasov.Plasma(5.0, 5.0, 0.6e-3, -1),
                           coarse_particles=0.5, coarse_tolerance=5.0)  # fmt: skip
    assert len(gpu) == len(ora) == 8
    traced = [t for *_, t in gpu]
    assert traced[0] == 50 and traced[-1] == 100  # every other trajectory, then all
    assert [t for *_, t in ora] == traced
    for k, ((phi_g, rho_g, _), (phi_o, rho_o, _)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-7 * 2000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-7 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip


def test_density_stopping_rule_matches_the_oracle(beam_optics):
    """The planar diode's stopping rule: the largest change of the density relative to its
    largest value below 1e-8; both stop at the same iteration with the same beam."""
    config = diode(current_density=10.0, iterations=60, tolerance=0.0, relaxation=0.5)
    model = beam_optics(config)
    gpu, ora = _iterations(model, 60, run_kwargs={"density_tolerance": 1e-8},
                           density_tolerance=1e-8)  # fmt: skip
    assert len(gpu) == len(ora) < 60
    assert model.convergence_history[-1]["relative_density_change"] < 1e-8
    assert model.convergence_history[-2]["relative_density_change"] >= 1e-8
    np.testing.assert_allclose(gpu[-1][1], ora[-1][1], rtol=0,
                               atol=1e-10 * np.abs(ora[-1][1]).max())  # fmt: skip
