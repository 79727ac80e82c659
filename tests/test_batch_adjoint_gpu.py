"""The design sweep's forward plus adjoint: the gradients taken of the candidates of one
batched solve equal the gradients each candidate's own solve gives."""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_the_gradients_of_a_batch_equal_each_solves() -> None:
    from beamtracer_b200.adjoint import adjoint_design_gradient, batch_design_gradients
    from beamtracer_b200.batch import BatchedVlasov
    from beamtracer_b200.einzel import einzel_config, sweep_designs

    designs = [replace(d, shape=(257, 65), trajectories=1500 + 500 * k)
               for k, d in enumerate(sweep_designs(3))]  # fmt: skip
    batch = BatchedVlasov([einzel_config(d, tolerance=1e-6, iterations=60) for d in designs]).run()
    assert all(c.converged for c in batch.candidates)
    got = batch_design_gradients(batch, designs)
    # one candidate at a time: the same gradients to rounding (the reverse sweep's
    # scatter adds with atomics)
    again = batch_design_gradients(batch, designs, concurrency=1)
    batch.close()
    for mine, once in zip(got, again):
        for name in ("rms_angle", "current"):
            scale = np.abs(once[name]).max()
            np.testing.assert_allclose(mine[name], once[name], rtol=0, atol=1e-9 * scale)
    for design, mine in zip(designs, got):
        alone = adjoint_design_gradient(design)
        for name in ("rms_angle", "current"):
            scale = np.abs(alone[name]).max()
            assert scale > 0.0
            np.testing.assert_allclose(mine[name], alone[name], rtol=0, atol=1e-4 * scale,
                                       err_msg=name)  # fmt: skip
        for name, value in alone["moments"].items():
            assert mine["moments"][name] == pytest.approx(value, rel=1e-6, abs=1e-15)
