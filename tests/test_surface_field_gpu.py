"""The surface field on the device against the reference's (``fields.py:324-377``) and
the oracle's: |E| at the free nodes beside the electrodes and each electrode's largest."""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden.cases import mesh_cases
from tests.gpu_util import GOLDEN
from tests.test_mesh import build_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(mesh_cases()))
def test_surface_field_matches_the_reference(name):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from types import SimpleNamespace

    from beamtracer_b200.fields import surface_field

    mesh = build_mesh(name)
    golden = np.load(GOLDEN / f"mesh_{name}.npz")
    want = np.load(GOLDEN / f"surface_{name}.npz")
    field = SimpleNamespace(fx_device=torch.from_numpy(golden["fx"]).cuda(),
                            fy_device=torch.from_numpy(golden["fy"]).cuda())  # fmt: skip
    magnitude, electrode = surface_field(mesh, field)
    np.testing.assert_array_equal(electrode, want["electrode"])
    np.testing.assert_array_equal(np.isnan(magnitude), np.isnan(want["magnitude"]))
    ok = ~np.isnan(want["magnitude"])
    np.testing.assert_allclose(magnitude[ok], want["magnitude"][ok], rtol=1e-15, atol=0)


def test_lens_surface_fields_match_the_oracle():
    """``BeamOptics.surface_fields()`` of a converged lens: each plate's largest |E| as the
    oracle computes it from the same edge fields."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.einzel import EinzelDesign, einzel_config
    from beamtracer_b200.model import BeamOptics
    from oracle.field import surface_field

    model = BeamOptics(einzel_config(EinzelDesign(shape=(201, 51), trajectories=200))).run()
    fields = model.surface_fields()
    assert list(fields) == ["plate0", "plate1", "plate2"]
    magnitude, electrode = surface_field(model.state.electric.fx, model.state.electric.fy,
                                         model.mesh.solid, model.mesh.near_solid)  # fmt: skip
    for k, name in enumerate(fields):
        want = np.max(magnitude[electrode == k])
        assert fields[name] == pytest.approx(want, rel=1e-15)
    assert fields["plate1"] > 1e5  # the middle plate at kilovolts over 0.4 mm cells
