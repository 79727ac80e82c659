"""The electrode sub-cell table sampled on the device against the host's NumPy table
(``tracer.py:1092-1114``): the same inside tests in the same order, so the same table."""

from __future__ import annotations

import numpy as np
import pytest

from beamtracer_b200.config import ObjectParams
from beamtracer_b200.mesh import Electrode, IonOpticsMesh
from beamtracer_b200.tracer import electrode_lookup, shape_table

pytestmark = pytest.mark.gpu


def _objects():
    return [
        ObjectParams("rectangle", "dirichlet", 0.0, midpoint=(5e-3, 1.5e-3),
                     side_lengths=(1.0e-3, 2.2e-3)),
        ObjectParams("circle", "dirichlet", 10.0, midpoint=(9.3e-3, 3.1e-3), radius=0.8e-3),
        ObjectParams("polygon", "dirichlet", -5.0,
                     vertices=((12e-3, 0.5e-3), (14.2e-3, 1.1e-3), (13.1e-3, 3.7e-3),
                               (12.4e-3, 2.0e-3))),
        ObjectParams("triangle", "dirichlet", 3.0,
                     vertices=((15e-3, 3e-3), (17.5e-3, 3e-3), (16e-3, 4.6e-3))),
        ObjectParams("aperture2d", "dirichlet", 7.0, axis=0, position=0.0,
                     vertices=((2e-3, 1.0e-3), (2e-3, 5e-3), (2.6e-3, 5e-3), (2.6e-3, 1.0e-3))),
        ObjectParams("line", "dirichlet", 1.0, midpoint=(18.5e-3, 2.5e-3),
                     side_lengths=(0.0, 3.0e-3)),
    ]  # fmt: skip


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
@pytest.mark.parametrize("graded", [False, True])
def test_device_subcells_equal_the_host(geometry, graded):
    from beamtracer_b200.tracer import electrode_lookup_device

    shape, h = (81, 21), 0.25e-3
    nodes = None
    if graded:
        s = np.linspace(0.0, 1.0, shape[0])
        nodes = 20e-3 * (0.3 * s + 0.7 * s * s)
    mesh = IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h, geometry=geometry, x_nodes=nodes,
                         electrodes=[Electrode(o.inside, o.bc_value) for o in _objects()])  # fmt: skip
    assert shape_table(mesh) is not None
    cells, subcells = electrode_lookup(mesh)
    cells_d, subcells_d = electrode_lookup_device(mesh)
    np.testing.assert_array_equal(cells_d.cpu().numpy(), cells)
    np.testing.assert_array_equal(subcells_d.cpu().numpy(), subcells)
    assert (subcells == -2).any() and (subcells >= 0).any()


def test_arbitrary_inside_functions_stay_on_the_host():
    from beamtracer_b200.tracer import electrode_lookup_device

    mesh = IonOpticsMesh(shape=(41, 21), origin=(0.0, 0.0), h=0.25e-3,
                         electrodes=[Electrode(lambda x, y: (x > 4e-3) & (x < 5e-3), 1.0)])  # fmt: skip
    assert shape_table(mesh) is None
    cells, subcells = electrode_lookup(mesh)
    cells_d, subcells_d = electrode_lookup_device(mesh)
    np.testing.assert_array_equal(subcells_d.cpu().numpy(), subcells)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
@pytest.mark.parametrize("graded", [False, True])
def test_device_classification_equals_the_host(geometry, graded):
    """The mesh's solid, near-solid, bracketed distances, held nodes and values sampled on
    the device equal the host's (the same electrodes given as plain inside functions,
    which only the host can call)."""
    shape, h = (81, 21), 0.25e-3
    nodes = None
    if graded:
        s = np.linspace(0.0, 1.0, shape[0])
        nodes = 20e-3 * (0.3 * s + 0.7 * s * s)
    objs = _objects()
    device = IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h, geometry=geometry, x_nodes=nodes,
                           electrodes=[Electrode(o.inside, o.bc_value) for o in objs])  # fmt: skip
    host = IonOpticsMesh(shape=shape, origin=(0.0, 0.0), h=h, geometry=geometry, x_nodes=nodes,
                         electrodes=[Electrode(lambda x, y, o=o: o.inside(x, y), o.bc_value)
                                     for o in objs])  # fmt: skip
    assert shape_table(device) is not None and shape_table(host) is None
    for name in ("solid", "near_solid", "distance", "fixed", "fixed_value"):
        np.testing.assert_array_equal(getattr(device, name), getattr(host, name), err_msg=name)
    assert host.near_solid.any() and (host.distance < 1).any()
