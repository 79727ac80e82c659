"""Parity at the benchmark's full sizes: the device solves against the oracle's.

- The einzel lens at 801 x 201 with 20,000 rings (the benchmark's workload), solved to
  convergence through ``BeamOptics(config).run()``: the potential and the current, rms
  size, rms angle and emittance at 70 and 79 mm within 1e-6 of the oracle's converged
  solve (relative), and, stage-wise, the density the beam deposits in the oracle's
  converged potential within 1e-10 of its largest value.
- The contracted-multiply-add build of the trace on the same lens: its stage-wise density
  within 1e-10 of the exact build's, its converged solve within 1e-6 of the oracle's.
- The planar plasma + solenoid extraction at 1025 x 513 with 100,000 trajectories: the
  first iteration's potential against the oracle's, and the stage-wise density in the
  device's second (Newton) potential within 1e-10.

The oracle's problems are built on the host alone (``tests.vlasov_cases.config_problem``,
``mesh_problem``): no device classification feeds them.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import vlasov as oracle_vlasov
from tests.vlasov_cases import config_problem, mesh_problem

pytestmark = pytest.mark.gpu

MOMENTS = ("current", "rms_size", "rms_angle", "emittance")


@pytest.fixture(scope="module")
def lens():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.einzel import EinzelDesign, einzel_config
    from beamtracer_b200.model import BeamOptics

    config = einzel_config(EinzelDesign(seed=2))
    model = BeamOptics(config).run()
    problem, particles, j_over_v = config_problem(config)
    oracle = oracle_vlasov.vlasov(problem, particles, j_over_v, iterations=config.iterations,
                                  tolerance=config.tolerance, relaxation=config.relaxation)
    return config, model, problem, particles, oracle


def _oracle_moments(problem, oracle, particles, mass):
    from beamtracer_b200.diagnostics import plane_moments
    from beamtracer_b200.tracer import PlaneHits

    hits = oracle_vlasov.plane_hits(problem, oracle["trace"], particles.current,
                                    particles.species)  # fmt: skip
    return {x: plane_moments(PlaneHits(x, *h), cylindrical=True, mass=mass)
            for x, h in zip(problem.planes, hits)}  # fmt: skip


def test_lens_converges_as_the_oracle(lens):
    config, model, problem, particles, oracle = lens
    assert len(model.convergence_history) == len(oracle["history"])
    assert model.stats["converged"]
    ref = oracle["potential"]
    phi_rel = np.max(np.abs(model.potential - ref)) / np.max(np.abs(ref))
    assert phi_rel <= 1e-6, phi_rel
    ora = _oracle_moments(problem, oracle, particles, model.species_mass)
    for x in config.diagnostic_planes:
        gpu = model.beam_moments(x)
        for name in MOMENTS:
            want = getattr(ora[x], name)
            assert want > 0.0, (x, name)
            assert getattr(gpu, name) == pytest.approx(want, rel=1e-6), (x, name)
        assert gpu.count == ora[x].count


def test_lens_density_stagewise(lens):
    """G(phi) of the oracle's converged potential, on the device and in the oracle."""
    from beamtracer_b200.fields import StaggeredElectricField

    config, model, problem, particles, oracle = lens
    phi = oracle["potential"]
    model.tracer.electric = StaggeredElectricField(model.mesh, phi)
    result = model.tracer.trace(particles)
    rho_o, trace_o = oracle_vlasov.density_of(problem, phi, particles)
    np.testing.assert_array_equal(result.status, trace_o.status.astype(np.int8))
    np.testing.assert_allclose(result.charge_density, rho_o, rtol=0,
                               atol=1e-10 * np.abs(rho_o).max())  # fmt: skip


def test_contracted_trace_matches_at_full_size(lens):
    """The trace with fused multiply-adds (the benchmark's build): stage-wise against the
    exact build, and converged against the oracle, at the bounds of the exact build."""
    from beamtracer_b200.fields import StaggeredElectricField
    from beamtracer_b200.model import BeamOptics

    config, model, problem, particles, oracle = lens
    phi = oracle["potential"]
    model.tracer.electric = StaggeredElectricField(model.mesh, phi)
    want = model.tracer.trace(particles)
    fast = BeamOptics(config, contracted_trace=True)
    fast.tracer.electric = StaggeredElectricField(fast.mesh, phi)
    got = fast.tracer.trace(particles)
    assert (got.status == want.status).mean() > 0.999
    np.testing.assert_allclose(got.charge_density, want.charge_density, rtol=0,
                               atol=1e-10 * np.abs(want.charge_density).max())  # fmt: skip
    solved = BeamOptics(config, contracted_trace=True).run()
    ref = oracle["potential"]
    assert np.max(np.abs(solved.potential - ref)) / np.max(np.abs(ref)) <= 1e-6
    ora = _oracle_moments(problem, oracle, particles, model.species_mass)
    for x in config.diagnostic_planes:
        gpu = solved.beam_moments(x)
        for name in MOMENTS:
            assert getattr(gpu, name) == pytest.approx(getattr(ora[x], name), rel=1e-6), (x, name)


def test_solenoid_extraction_full_size_stagewise():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.fields import StaggeredElectricField
    from beamtracer_b200.solenoid_extraction import SolenoidExtractionDesign, solenoid_extraction

    design = SolenoidExtractionDesign()
    assert design.shape == (1025, 513) and design.trajectories == 100_000
    case = solenoid_extraction(design)
    gpu = []
    case.run(lambda it, state: gpu.append((state.potential.copy(), state.charge_density.copy())),
             iterations=2, tolerance=0.0)  # fmt: skip
    problem = mesh_problem(case.mesh, integrator=1, magnetic=case.magnetic)
    ora = []
    oracle_vlasov.vlasov(problem, case.particles, case.j_over_v, iterations=1,
                         relaxation=design.relaxation,
                         plasma=oracle_vlasov.Plasma(design.electron_temperature,
                                                     design.plasma_potential, design.plasma_x,
                                                     -1, density=case.plasma.rho_e),
                         callback=lambda it, out: ora.append(
                             (out["potential"].copy(), out["charge_density"].copy())))  # fmt: skip
    span = abs(design.extraction_voltage)
    np.testing.assert_allclose(gpu[0][0], ora[0][0], rtol=0, atol=1e-9 * span)
    # the Newton potential of the second iteration, traced by both
    phi = gpu[1][0]
    case.tracer.electric = StaggeredElectricField(case.mesh, phi)
    result = case.tracer.trace(case.particles)
    rho_o, trace_o = oracle_vlasov.density_of(problem, phi, case.particles)
    np.testing.assert_array_equal(result.status, trace_o.status.astype(np.int8))
    assert (result.status == 0).sum() > 0
    np.testing.assert_allclose(result.charge_density, rho_o, rtol=0,
                               atol=1e-10 * np.abs(rho_o).max())  # fmt: skip
