"""The 3D mesh classification against the reference's ``IonOpticsMesh3D``.

``tests/golden/mesh3d_plate_sphere.npz`` holds the reference's classification of
``mesh3d_case`` (a plate with a round hole, a sphere, a Dirichlet face and a symmetry
plane): the solid nodes, the near-solid nodes with their bracketed surface distances, the
held nodes and their potentials -- equal here value for value.
"""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.geometry3d import Electrode3D, IonOpticsMesh3D
from beamtracer_b200.mesh import FaceCondition
from tests.golden.cases import mesh3d_case
from tests.gpu_util import GOLDEN


def _mesh(**override) -> IonOpticsMesh3D:
    settings = mesh3d_case()
    settings.update(override)
    return IonOpticsMesh3D(
        shape=settings["shape"], origin=settings["origin"], h=settings["h"],
        electrodes=[Electrode3D(f, v) for f, v in settings["electrodes"]],
        faces={k: FaceCondition(*v) for k, v in settings["faces"].items()},
        symmetry_planes=settings["symmetry_planes"],
    )  # fmt: skip


def test_classification_matches_the_reference():
    golden = np.load(GOLDEN / "mesh3d_plate_sphere.npz")
    mesh = _mesh()
    for name in ("solid", "near_solid", "distance", "fixed", "fixed_value"):
        np.testing.assert_array_equal(getattr(mesh, name), golden[name], err_msg=name)


def test_mesh3d_refuses_bad_settings():
    with pytest.raises(ValueError):
        _mesh(shape=(2, 5, 5))
    with pytest.raises(ValueError):
        _mesh(h=0.0)
    with pytest.raises(ValueError):
        _mesh(symmetry_planes=("x_min",))
    with pytest.raises(ValueError):
        _mesh(faces={"y_min": ("dirichlet", 1.0)})
