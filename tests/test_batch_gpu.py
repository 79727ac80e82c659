"""The batched sweep against the plain form run candidate by candidate.

Candidates of different meshes, plate positions, apertures, voltages, currents and
trajectory counts go through one `BatchedVlasov`.  Every trajectory of a batched trace must
end where its own candidate's trace ends it, bit for bit (steps, status, state, plane
crossings): a trajectory reads only its own candidate's mesh.  The node charges are the
same records summed in the same order, grouped into deposits differently: within 1e-12 of
the largest.  Converged, every candidate must take the iterations its own
`BeamOptics(config).run()` takes and give its moments within 1e-9 (the bound of the design
sweep is 1e-6).  The batched field solve must meet each single solve's residual criterion:
its potential within 1e-9 of the span of the single solve's.
"""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.einzel import EinzelDesign, einzel_config, evaluate_design

pytestmark = pytest.mark.gpu

#: Small candidates: three meshes, different plates, beams and trajectory counts.
DESIGNS = [
    EinzelDesign(shape=(161, 41), trajectories=600, aperture=4.0e-3, current=0.5e-3,
                 voltages=(0.0, 6e3, 0.0), seed=11),
    EinzelDesign(shape=(241, 61), trajectories=1500, aperture=6.0e-3, current=1.5e-3,
                 centres=(25e-3, 40e-3, 55e-3), voltages=(0.0, 9e3, 0.0), seed=12),
    EinzelDesign(shape=(161, 41), trajectories=900, aperture=3.3e-3, current=0.2e-3,
                 centres=(18e-3, 40e-3, 62e-3), voltages=(0.0, 4e3, 0.0), seed=13),
    EinzelDesign(shape=(321, 81), trajectories=2000, aperture=5.1e-3, current=1.0e-3,
                 voltages=(0.0, 11e3, 0.0), seed=14),
]  # fmt: skip


def _batch(designs, **kwargs):
    from beamtracer_b200.batch import BatchedVlasov

    return BatchedVlasov([einzel_config(d) for d in designs], **kwargs)


@pytest.mark.parametrize("contracted", [False, True])
def test_batched_trace_equals_each_alone(contracted):
    import torch

    batch = _batch(DESIGNS, contracted=contracted)
    members = list(range(len(DESIGNS)))
    # a field per candidate: the vacuum field of its plates
    from beamtracer_b200.fields import StaggeredElectricField

    for k, c in enumerate(batch.candidates):
        c.poisson.solve_device(batch.node_view(batch.phi, k), batch.node_view(batch.rho, k))
        StaggeredElectricField(c.mesh, batch.node_view(batch.phi, k), arrays=c.arrays,
                               out=batch.edge_views(k))  # fmt: skip
    batch.trace(members)
    for k, c in enumerate(batch.candidates):
        e = c.engine
        e.contracted = contracted
        fx, fy = batch.edge_views(k)
        e.run(fx.contiguous(), fy.contiguous())
        t = slice(c.traj0, c.traj0 + c.n_traj)
        assert torch.equal(batch.steps[t], e.steps)
        assert torch.equal(batch.status[t], e.status)
        assert torch.equal(batch.electrode[t], e.electrode)
        assert torch.equal(batch.x[:, t], e.x)
        assert torch.equal(batch.v[:, t], e.v)
        assert torch.equal(batch.counts[t], e.counts)
        for p in range(len(batch.planes)):
            for j in torch.nonzero(e.counts[:, p]).flatten().tolist():
                n = int(e.counts[j, p])
                assert torch.equal(batch.hits[c.traj0 + j, p, :n], e.hits[j, p, :n])
        mine = batch.charge[0, c.node0 : c.node0 + c.n_nodes]
        alone = e.charge[0]
        scale = float(alone.abs().max())
        assert scale > 0
        assert float((mine - alone).abs().max()) <= 1e-12 * scale
    assert (batch.status >= 0).all()


def test_batched_field_solve_equals_each_solve():
    import torch

    batch = _batch(DESIGNS)
    rng = np.random.default_rng(3)
    batch.rho.copy_(torch.from_numpy(rng.uniform(0.0, 2e-5, batch.n_nodes)))
    members = [0, 1, 3]  # candidate 2 is left out and must keep its potential
    keep = batch.node_view(batch.phi, 2).clone()
    for sweep in range(2):  # from zero, then from the last potential with a new density
        batch.poisson_batch.solve(batch.phi, batch.rho, members)
        assert (batch.poisson_batch.cycles[members] > 0).all()
        for k in members:
            c = batch.candidates[k]
            alone = torch.zeros(c.shape, dtype=torch.float64, device="cuda")
            c.poisson.solve_device(alone, batch.node_view(batch.rho, k))
            got = batch.node_view(batch.phi, k)
            # both meet |r| <= 1e-13 max(|b|, |r0|), which bounds the smooth error to about
            # 1e-9 of the potential's span (the single solve's bound against LU)
            scale = float(alone.abs().max())
            assert float((got - alone).abs().max()) <= 1e-9 * scale, (sweep, k)
        assert torch.equal(batch.node_view(batch.phi, 2), keep)
        batch.rho.mul_(1.5)
    assert batch.poisson_batch.tiling["tuned"]


@pytest.mark.parametrize("tiling", [((32, 16), (16, 16), 2), ((64, 16), (32, 32), 2),
                                    ((16, 32), (16, 32), 1)])
def test_batched_field_solve_with_every_tiling(tiling):
    import torch

    batch = _batch(DESIGNS)
    batch.poisson_batch.set_tiling(*tiling)
    rng = np.random.default_rng(4)
    batch.rho.copy_(torch.from_numpy(rng.uniform(0.0, 2e-5, batch.n_nodes)))
    batch.poisson_batch.solve(batch.phi, batch.rho, range(len(DESIGNS)))
    assert batch.poisson_batch.tiling["level0"] == tiling[0]
    for k, c in enumerate(batch.candidates):
        alone = torch.zeros(c.shape, dtype=torch.float64, device="cuda")
        c.poisson.solve_device(alone, batch.node_view(batch.rho, k))
        scale = float(alone.abs().max())
        assert float((batch.node_view(batch.phi, k) - alone).abs().max()) <= 1e-9 * scale


@pytest.mark.parametrize("field", ["batched", "single"])
def test_batched_sweep_matches_each_solve(field):
    batch = _batch(DESIGNS, field=field).run()
    for k, design in enumerate(DESIGNS):
        plain = evaluate_design(design)
        c = batch.candidates[k]
        assert c.done
        assert len(c.history) == plain["iterations"]
        assert int(c.converged) == plain["converged"]
        m = c.moments(79e-3)
        for name in ("current", "rms_size", "rms_angle", "emittance"):
            want = plain[name]
            got = getattr(m, name)
            assert abs(got - want) <= 1e-9 * abs(want), (k, name, got, want)


def test_batch_refuses_what_it_does_not_do():
    from beamtracer_b200.batch import BatchedVlasov

    config = einzel_config(DESIGNS[0])
    with pytest.raises(NotImplementedError):
        BatchedVlasov([config.replace(mixing="anderson")])
    with pytest.raises(ValueError):
        BatchedVlasov([config, einzel_config(DESIGNS[1]).replace(tolerance=1e-4)])
    with pytest.raises(ValueError):
        BatchedVlasov([])
    np.testing.assert_equal(len(BatchedVlasov([config]).candidates), 1)
