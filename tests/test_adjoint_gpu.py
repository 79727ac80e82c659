"""The pieces of the adjoint, each against what it reverses.

- the edge field's transpose: ``<D phi, e> = <phi, D^T e>`` to rounding;
- the transposed field solve: ``<A^-1 b, g> = <b, A^-T g>`` on the free nodes, and the held
  nodes' sensitivity against the (exactly linear) change of a solve with the voltages;
- the reverse sweep of the trace: its replay ends where the trace ended, bit for bit, and
  its edge-field adjoint of a seeded quantity of the node charges and crossings equals the
  central difference of that quantity along a random direction of the edge fields.
"""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.einzel import EinzelDesign, einzel_config

pytestmark = pytest.mark.gpu

SMALL = EinzelDesign(shape=(201, 51), trajectories=400, seed=4)


@pytest.fixture(scope="module")
def model():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.model import BeamOptics

    return BeamOptics(einzel_config(SMALL, tolerance=1e-7, iterations=60)).run()


def test_edge_field_adjoint_is_the_transpose(model):
    import torch

    from beamtracer_b200.adjoint import edge_field_adjoint
    from beamtracer_b200.fields import MeshArrays, StaggeredElectricField

    mesh = model.mesh
    rng = np.random.default_rng(11)
    phi = torch.from_numpy(rng.normal(size=mesh.shape)).cuda()
    field = StaggeredElectricField(mesh, phi)
    ex = torch.from_numpy(rng.normal(size=field.fx_device.shape)).cuda()
    ey = torch.from_numpy(rng.normal(size=field.fy_device.shape)).cuda()
    back = edge_field_adjoint(MeshArrays(mesh), ex, ey, field.extrapolation)
    left = float((field.fx_device * ex).sum() + (field.fy_device * ey).sum())
    right = float((phi * back).sum())
    assert right == pytest.approx(left, rel=1e-12)
    # the same bits on every call
    again = edge_field_adjoint(MeshArrays(mesh), ex, ey, field.extrapolation)
    assert torch.equal(back, again)


def test_transposed_solve_is_the_transpose(model):
    import torch

    from beamtracer_b200 import _lib
    from beamtracer_b200.poisson import IonOpticsPoisson

    mesh = model.mesh
    eps0 = 8.8541878188e-12
    forward = IonOpticsPoisson(mesh, transposed=True)  # zero held values and face terms
    _lib.check(_lib.lib().bt_poisson_set_transposed(forward._handle, 0))  # ... and A itself
    transposed = IonOpticsPoisson(mesh, transposed=True)
    free = torch.from_numpy(~mesh.fixed).cuda()
    rng = np.random.default_rng(12)
    b = torch.from_numpy(rng.normal(size=mesh.shape)).cuda() * free
    g = torch.from_numpy(rng.normal(size=mesh.shape)).cuda() * free
    u = torch.zeros_like(b)
    w = torch.zeros_like(b)
    forward.solve_device(u, eps0 * b)
    transposed.solve_device(w, eps0 * g)
    assert float((u * ~free).abs().max()) == 0.0 and float((w * ~free).abs().max()) == 0.0
    left, right = float((u * g).sum()), float((b * w).sum())
    assert right == pytest.approx(left, rel=1e-9)
    # the operator is not symmetric next to the electrodes and in cylindrical rows
    assert float((u - w).abs().max()) > 1e-6 * float(u.abs().max())


def test_held_node_sensitivity(model):
    """d<w, phi>/dV_e of the field solve with the voltages (linear in them) against the
    adjoint's sum over the electrode's nodes."""
    import torch

    from beamtracer_b200.einzel import resolved_voltages
    from beamtracer_b200.model import config_mesh
    from beamtracer_b200.poisson import IonOpticsPoisson

    eps0 = 8.8541878188e-12
    mesh = model.mesh
    rng = np.random.default_rng(13)
    weight = torch.from_numpy(rng.normal(size=mesh.shape)).cuda()
    transposed = IonOpticsPoisson(mesh, transposed=True)
    z = torch.zeros_like(weight)
    transposed.solve_device(z, eps0 * weight)
    held = torch.empty_like(weight)
    transposed.fixed_adjoint(z, weight, held)
    solid = torch.from_numpy(mesh.solid.astype(np.int64)).cuda()
    voltages = resolved_voltages(SMALL)

    def objective(v):
        from dataclasses import replace

        m = config_mesh(einzel_config(replace(SMALL, voltages=tuple(v))))
        phi = torch.zeros(m.shape, dtype=torch.float64, device="cuda")
        IonOpticsPoisson(m).solve_device(phi, None)
        return float((weight * phi).sum())

    for e in range(3):
        step = 10.0
        plus, minus = list(voltages), list(voltages)
        plus[e] += step
        minus[e] -= step
        fd = (objective(plus) - objective(minus)) / (2 * step)
        assert float(held[solid == e].sum()) == pytest.approx(fd, rel=1e-7), e


def test_trace_adjoint_matches_finite_differences(model):
    import torch

    from beamtracer_b200.adjoint import TraceAdjoint

    engine = model.tracer.engine()
    field = model.state.electric
    fx, fy = field.fx_device.clone(), field.fy_device.clone()
    adjoint = TraceAdjoint(engine, fx, fy)
    end = torch.empty((6, engine.n), dtype=torch.float64, device="cuda")
    adjoint.record(end)
    assert torch.equal(end[:3], engine.x) and torch.equal(end[3:], engine.v)

    rng = np.random.default_rng(14)
    nx, ny = model.mesh.shape
    # seeds of the size of the outputs they weigh: node charges, crossing points (m) and
    # velocities (m/s)
    charge_seed = torch.from_numpy(rng.normal(size=(nx, ny))).cuda() / float(engine.charge.abs().max())
    filled = (torch.arange(engine.hits.shape[2], device="cuda")[None, None, :]
              < engine.counts[:, :, None])  # fmt: skip
    assert int(filled.sum()) > 0
    hit_seed = torch.from_numpy(rng.normal(size=engine.hits.shape)).cuda() * filled[..., None]
    hit_seed[..., 0] = 0.0
    hit_seed[..., 6:] = 0.0
    hit_seed[..., 1:3] *= 1e3
    hit_seed[..., 3:6] *= 1e-6
    bars = {"charge": adjoint.sweep(charge_seed, None), "hits": adjoint.sweep(None, hit_seed)}

    # a direction of the typical field's size on every edge
    dfx = torch.from_numpy(rng.normal(size=fx.shape)).cuda() * float(fx.abs().median())
    dfy = torch.from_numpy(rng.normal(size=fy.shape)).cuda() * float(fy.abs().median())
    steps, status, counts = engine.steps.clone(), engine.status.clone(), engine.counts.clone()

    def outputs(eps):
        engine.run(fx + eps * dfx, fy + eps * dfy)
        # no trajectory took another number of steps, ended otherwise or crossed otherwise:
        # the quantity is smooth between the two runs
        assert torch.equal(engine.steps, steps) and torch.equal(engine.status, status)
        assert torch.equal(engine.counts, counts)
        return {"charge": float((charge_seed.reshape(-1) * engine.charge[0]).sum()),
                "hits": float((hit_seed * engine.hits).sum())}  # fmt: skip

    eps = 1e-6
    plus, minus = outputs(eps), outputs(-eps)
    engine.run(fx, fy)  # the engine's buffers back to the converged trace
    for part, (fx_bar, fy_bar) in bars.items():
        predicted = float((fx_bar * dfx).sum() + (fy_bar * dfy).sum())
        central = (plus[part] - minus[part]) / (2 * eps)
        assert predicted == pytest.approx(central, rel=1e-5), part
