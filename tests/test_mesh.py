"""The mesh classification and the oracle's edge field against the reference's outputs.

The golden meshes (``tests/golden/mesh_*.npz``) were classified by the reference's own
``solver/mesh.py`` and their edge fields computed by its ``_edge_field``
(``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from oracle.field import edge_fields
from tests.golden.cases import mesh_cases
from tests.gpu_util import GOLDEN

CASES = mesh_cases()


def build_mesh(name: str) -> IonOpticsMesh:
    settings = dict(CASES[name])
    electrodes = [Electrode(f, v) for f, v in settings.pop("electrodes")]
    faces = {k: FaceCondition(*v) for k, v in settings.pop("faces").items()}
    return IonOpticsMesh(electrodes=electrodes, faces=faces, **settings)


@pytest.mark.parametrize("name", sorted(CASES))
def test_classification_matches_the_reference(name):
    mesh = build_mesh(name)
    golden = np.load(GOLDEN / f"mesh_{name}.npz")
    np.testing.assert_array_equal(mesh.solid, golden["solid"])
    np.testing.assert_array_equal(mesh.fixed, golden["fixed"])
    np.testing.assert_array_equal(mesh.fixed_value, golden["fixed_value"])
    np.testing.assert_array_equal(mesh.near_solid, golden["near_solid"])
    np.testing.assert_array_equal(mesh.distance, golden["distance"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_edge_field_matches_the_reference(name):
    mesh = build_mesh(name)
    golden = np.load(GOLDEN / f"mesh_{name}.npz")
    faces = ["extrapolate"] * 4
    if mesh.cylindrical or mesh.symmetry_plane:
        faces[2] = "symmetric"
    fx, fy = edge_fields(golden["phi"], mesh.solid, mesh.near_solid, mesh.distance,
                         mesh.dx, mesh.h, faces)  # fmt: skip
    np.testing.assert_array_equal(fx, golden["fx"])
    np.testing.assert_array_equal(fy, golden["fy"])


def test_mesh_validation():
    with pytest.raises(ValueError, match="axis"):
        IonOpticsMesh(shape=(5, 5), origin=(0.0, 1e-3), h=1e-3)
    with pytest.raises(ValueError, match="3 nodes"):
        IonOpticsMesh(shape=(2, 5), origin=(0.0, 0.0), h=1e-3)
    with pytest.raises(ValueError, match="unknown faces"):
        IonOpticsMesh(shape=(5, 5), origin=(0.0, 0.0), h=1e-3, faces={"z_min": FaceCondition()})


def test_wall_distance_is_bracketed_in_255ths():
    """The case of the reference's ``test_ion_optics.py:39-56``, as a known answer."""
    surface = 5.3e-3
    mesh = IonOpticsMesh(
        shape=(11, 5), origin=(0.0, 0.0), h=1e-3, geometry="planar",
        electrodes=[Electrode(lambda x, y: x >= surface, 10.0)],
    )  # fmt: skip
    assert mesh.near_solid[5].all() and not mesh.near_solid[4].any()
    assert np.allclose(mesh.distance[1, 5], np.floor(0.3 * 255 + 1) / 255, atol=1 / 255)
    assert (mesh.fixed_value[6:] == 10.0).all()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_surface_field_matches_the_reference(name):
    """The oracle's restatement of ``surface_field`` (``fields.py:324-377``) against the
    reference's own on the golden meshes and edge fields."""
    from oracle.field import surface_field

    mesh = build_mesh(name)
    golden = np.load(GOLDEN / f"mesh_{name}.npz")
    want = np.load(GOLDEN / f"surface_{name}.npz")
    magnitude, electrode = surface_field(golden["fx"], golden["fy"], mesh.solid, mesh.near_solid)
    np.testing.assert_array_equal(electrode, want["electrode"])
    np.testing.assert_array_equal(np.isnan(magnitude), np.isnan(want["magnitude"]))
    np.testing.assert_array_equal(magnitude, want["magnitude"])
