"""Refined boxes on the host: the patches, the composite nodes and the oracle's composite
solve (the cases of the reference's ``tests/unit/test_refinement.py:36-131``)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.constants import epsilon_0

from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from beamtracer_b200.refinement import Refinement, layout_of_mesh, patches_of
from oracle import composite

DIRICHLET_X = {"x_min": FaceCondition("dirichlet", 0.0), "x_max": FaceCondition("dirichlet", 0.0)}


def _plates(geometry: str = "planar") -> IonOpticsMesh:
    return IonOpticsMesh((21, 11), (0.0, 0.0), 1e-3, geometry, faces=DIRICHLET_X,
                         classify_on_device=False)  # fmt: skip


def test_boxes_snap_to_the_level_below_and_their_fields_get_a_margin() -> None:
    mesh = _plates()
    patches = patches_of(mesh, [Refinement(1, (2.6e-3, 0.0), (7.2e-3, 4.1e-3)),
                                Refinement(2, (3e-3, 0), (5e-3, 2e-3))])  # fmt: skip
    one, two = patches[1], patches[2]
    assert one.box == ((4, 16), (0, 10))  # level-1 nodes: base nodes 2..8, 0..5
    assert one.mesh.origin == pytest.approx((2e-3, 0.0))
    assert one.mesh.h == pytest.approx(0.5e-3)
    assert one.field_mesh.origin == pytest.approx((1e-3, 0.0))
    assert one.field_mesh.shape == (one.mesh.shape[0] + 4, one.mesh.shape[1] + 2)
    assert two.box == ((12, 20), (0, 8)) and two.mesh.h == pytest.approx(0.25e-3)
    with pytest.raises(ValueError, match="outside"):
        patches_of(mesh, [Refinement(1, (0.03, 0.0), (0.04, 0.01))])
    with pytest.raises(ValueError, match="level"):
        patches_of(mesh, [Refinement(0, (0.0, 0.0), (0.01, 0.01))])


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_the_volumes_fill_the_domain(geometry) -> None:
    mesh = _plates(geometry)
    plain = layout_of_mesh(mesh)
    refined = layout_of_mesh(mesh, [Refinement(1, (5e-3, 0.0), (12e-3, 6e-3))])
    assert refined.size > plain.size
    total = 20e-3 * 10e-3 if geometry == "planar" else np.pi * 10e-3**2 * 20e-3
    assert plain.volumes.sum() == pytest.approx(total)
    assert refined.volumes.sum() == pytest.approx(total)
    values = np.arange(231.0).reshape(21, 11)
    np.testing.assert_array_equal(plain.from_base(values)[plain.base.index], values)
    with pytest.raises(ValueError, match="composite"):
        refined.from_base(np.zeros(mesh.shape))


def test_the_nodes_hang_on_coarse_edges_and_interpolate_planes_exactly() -> None:
    mesh = _plates()
    layout = layout_of_mesh(mesh, [Refinement(1, (4e-3, 2e-3), (14e-3, 6e-3)),
                                   Refinement(2, (6e-3, 2e-3), (10e-3, 4e-3))])  # fmt: skip
    assert layout.hanging.size > 0
    # no base node hangs, and every hanging node is a node of a box only
    base = set(layout.base.index.ravel().tolist())
    assert not base & set(layout.hanging.tolist())
    plane = 3.0 * layout.x - 7.0 * layout.y + 1.0
    filled = plane.copy()
    filled[layout.hanging] = 0.0
    layout.fill_hanging(filled)
    np.testing.assert_allclose(filled, plane, rtol=0, atol=1e-14)
    # the interpolation reads only nodes that do not hang
    assert not set(layout.interpolation.indices.tolist()) & set(layout.hanging.tolist())


def test_a_box_must_lie_inside_the_level_below() -> None:
    with pytest.raises(ValueError, match="inside those of level 1"):
        layout_of_mesh(_plates(), [Refinement(1, (2e-3, 0.0), (6e-3, 4e-3)),
                                   Refinement(2, (8e-3, 0.0), (10e-3, 2e-3))])  # fmt: skip


def graded_nodes(n: int, lower: float, upper: float) -> np.ndarray:
    """``n`` nodes of a smooth map, cells from 0.7 to 1.3 of the mean (the reference's
    ``test_graded_mesh.py:26-29`` case)."""
    s = np.linspace(0.0, 1.0, n)
    return lower + (upper - lower) * (s + 0.3 * np.sin(2.0 * np.pi * s) / (2.0 * np.pi))


def test_refined_boxes_continue_the_grading() -> None:
    """``test_graded_mesh.py:95-111``: every other node of a box is a base node, the others
    halve the base edges; the box's uniform coordinate is the mesh's."""
    nodes = graded_nodes(21, 0.0, 2.0)
    mesh = IonOpticsMesh((21, 11), (0.0, 0.0), 0.1, "planar", x_nodes=nodes,
                         classify_on_device=False)  # fmt: skip
    base, patch = patches_of(mesh, [Refinement(1, (0.5, 0.2), (1.2, 0.6))])
    first = patch.box[0][0] // 2
    np.testing.assert_allclose(patch.mesh.x[::2], nodes[first : first + patch.mesh.x[::2].size])
    np.testing.assert_allclose(patch.mesh.x[1::2], 0.5 * (patch.mesh.x[:-1:2] + patch.mesh.x[2::2]))
    assert patch.mesh.logical_x0 == pytest.approx(patch.box[0][0] * 0.05)
    x = np.linspace(patch.mesh.x[0], patch.mesh.x[-1], 7)
    np.testing.assert_allclose(patch.mesh.logical_x(x), mesh.logical_x(x))
    assert patch.field_mesh.x[2] == patch.mesh.x[0]


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_graded_volumes_fill_the_domain_and_the_plates_parabola_holds(geometry) -> None:
    rho = 1e-6
    nodes = graded_nodes(41, 0.0, 20e-3)
    mesh = IonOpticsMesh((41, 21), (0.0, 0.0), 0.5e-3, geometry, x_nodes=nodes,
                         faces=DIRICHLET_X, classify_on_device=False)  # fmt: skip
    layout = layout_of_mesh(mesh, [Refinement(1, (4e-3, 0.0), (14e-3, 6e-3)),
                                   Refinement(2, (6e-3, 0.0), (10e-3, 4e-3))])  # fmt: skip
    total = 20e-3 * 10e-3 if geometry == "planar" else np.pi * 10e-3**2 * 20e-3
    assert layout.volumes.sum() == pytest.approx(total)
    if geometry == "planar":
        phi = composite.solve(layout, np.full(layout.size, rho))
        exact = rho / (2 * epsilon_0) * layout.x * (20e-3 - layout.x)
        assert np.abs(phi - exact).max() < 1e-2 * exact.max()


def test_a_uniform_charge_between_plates_on_refined_boxes() -> None:
    """The reference's known answer (``test_refinement.py:105-131``): the parabola of a
    uniform charge between grounded plates, within 1e-2 on two nested boxes, the error
    falling with the cells (first order at the coarse-fine nodes)."""
    rho = 1e-6
    errors = []
    for n in (21, 41):
        mesh = IonOpticsMesh((n, (n + 1) // 2), (0.0, 0.0), 20e-3 / (n - 1), "planar",
                             faces=DIRICHLET_X, classify_on_device=False)  # fmt: skip
        layout = layout_of_mesh(mesh, [Refinement(1, (4e-3, 0.0), (14e-3, 6e-3)),
                                       Refinement(2, (6e-3, 0.0), (10e-3, 4e-3))])  # fmt: skip
        phi = composite.solve(layout, np.full(layout.size, rho))
        exact = rho / (2 * epsilon_0) * layout.x * (20e-3 - layout.x)
        errors.append(np.abs(phi - exact).max() / exact.max())
    assert errors[0] < 1e-2
    assert errors[1] < 0.6 * errors[0]


def test_without_boxes_the_composite_solve_is_the_mesh_solve() -> None:
    from oracle import poisson as oracle_poisson

    plate = lambda x, y: (x >= 8e-3) & (x <= 10e-3) & (y >= 4e-3)  # noqa: E731
    faces = {"x_min": FaceCondition("dirichlet", 0.0), "x_max": FaceCondition("dirichlet", -50.0)}
    for geometry in ("planar", "cylindrical"):
        mesh = IonOpticsMesh((21, 11), (0.0, 0.0), 1e-3, geometry, faces=faces,
                             electrodes=[Electrode(plate, 100.0)], classify_on_device=False)  # fmt: skip
        layout = layout_of_mesh(mesh)
        rho = np.linspace(0.0, 1e-7, layout.size)
        phi = composite.solve(layout, rho)
        direct = oracle_poisson.solve(oracle_poisson.operator_of_mesh(mesh),
                                      layout.on_base(rho)).ravel()  # fmt: skip
        np.testing.assert_allclose(layout.on_base(phi).ravel(), direct, rtol=0, atol=1e-10)


def test_the_setting_is_checked_and_round_trips() -> None:
    """``config.py:437-464``: the level and the corners are checked, and a configuration's
    boxes survive ``to_dict`` / ``from_dict`` (``test_refinement.py:17-27``)."""
    from beamtracer_b200 import BeamOpticsConfig, GridParams, RefinementParams

    with pytest.raises(ValueError, match="level"):
        RefinementParams(0, (0, 0), (1e-3, 1e-3))
    with pytest.raises(ValueError, match="lower < upper"):
        RefinementParams(1, (2e-3, 0), (1e-3, 1e-3))
    grid = GridParams(num_gridpoints=(81, 31), lower_bound=(0.0, 0.0), upper_bound=(8e-3, 3e-3),
                      coordinates="cylindrical")  # fmt: skip
    config = BeamOpticsConfig(grid=grid,
                              refinement=[RefinementParams(1, (0.5e-3, 0.0), (3e-3, 1.5e-3))])
    again = type(config).from_dict(config.to_dict())
    assert again.refinement == config.refinement
    assert again.refinement[0].upper == pytest.approx((3e-3, 1.5e-3))
    with pytest.raises(ValueError, match="2D grid"):
        BeamOpticsConfig(grid=grid, refinement=[RefinementParams(1, (0, 0, 0), (1, 1, 1))])


def test_the_oracle_newton_and_held_region_solve_their_equations() -> None:
    """The oracle's composite Newton iteration and held region: the Boltzmann residual
    vanishes at its solution, the held nodes keep their potential, and without refinement
    Newton's composite solution is the mesh's (``oracle/poisson.py``)."""
    from scipy.constants import epsilon_0 as eps0

    from oracle import poisson as oracle_poisson

    plate = lambda x, y: (x >= 8e-3) & (x <= 10e-3) & (y >= 4e-3)  # noqa: E731
    faces = {"x_min": FaceCondition("dirichlet", 5.0), "x_max": FaceCondition("dirichlet", -50.0)}
    mesh = IonOpticsMesh((21, 11), (0.0, 0.0), 1e-3, "cylindrical", faces=faces,
                         electrodes=[Electrode(plate, -20.0)], classify_on_device=False)  # fmt: skip
    region = lambda x, y: x < 3e-3  # noqa: E731
    rho = np.full(layout_of_mesh(mesh).size, 1e-8)
    for boxes in ([], [Refinement(1, (0.0, 0.0), (6e-3, 4e-3))]):
        layout = layout_of_mesh(mesh, boxes)
        rho = np.full(layout.size, 1e-8)
        held = composite.solve_region(layout, rho, region, 5.0)
        mask = composite.held_region(layout, region)
        np.testing.assert_array_equal(held[mask], 5.0)
        phi, steps = composite.solve_newton(layout, rho, 1e-3 / eps0, 5.0, 5.0, -1, initial=held)
        assert steps >= 2
        K, b = composite.assemble(layout, rho)
        own = (layout.owner >= 0) & ~layout.fixed
        e = 1e-3 / eps0 * np.exp(np.minimum((phi - 5.0) / 5.0, 50.0))
        residual = b - np.where(own, e, 0.0) - K @ phi
        assert np.abs(residual).max() <= 1e-7 * np.abs(b).max()
        if not boxes:
            op = oracle_poisson.operator_of_mesh(mesh)
            direct, _ = oracle_poisson.solve_newton(op, layout.on_base(rho), 1e-3 / eps0, 5.0,
                                                    5.0, -1, tol=1e-11)  # fmt: skip
            np.testing.assert_allclose(layout.on_base(phi), direct, rtol=0, atol=1e-9)


REFINED = ("planar_plates", "cylindrical_lens", "graded_disc")


@pytest.mark.parametrize("name", REFINED)
def test_patches_and_their_fields_match_the_reference(name) -> None:
    """The refined patches and the potential and edge fields of every patch's field mesh
    against the reference's own ``patches_of`` and ``PatchedElectricField`` run on the same
    meshes, boxes and potential (``tests/golden/refinement_*.npz``, made by
    ``tests/golden/make_golden.py``): the boxes and shapes exactly, the positions and the
    fields to rounding."""
    from tests.golden.cases import refinement_cases, refinement_potential
    from tests.gpu_util import GOLDEN
    from tests.test_mesh import build_mesh

    golden = np.load(GOLDEN / f"refinement_{name}.npz")
    mesh = build_mesh(name)
    mesh = IonOpticsMesh(shape=mesh.shape, origin=mesh.origin, h=mesh.h, geometry=mesh.geometry,
                         electrodes=mesh.electrodes, faces=dict(mesh.faces),
                         x_nodes=mesh.x_nodes, classify_on_device=False)  # fmt: skip
    boxes = [Refinement(*b) for b in refinement_cases()[name]]
    layout = layout_of_mesh(mesh, boxes)
    assert len(layout.patches) == int(golden["patches"])
    phi = refinement_potential(layout.x, layout.y)
    values = composite.field_values(layout, phi)
    fields, _ = composite.edge_fields(layout, phi)
    for q, patch in enumerate(layout.patches):
        fm = patch.field_mesh if patch.field_mesh is not None else patch.mesh
        assert patch.level == int(golden[f"p{q}_level"])
        np.testing.assert_array_equal(np.array(patch.box), golden[f"p{q}_box"])
        assert tuple(patch.mesh.shape) == tuple(golden[f"p{q}_shape"])
        assert tuple(fm.shape) == tuple(golden[f"p{q}_field_shape"])
        np.testing.assert_allclose(patch.mesh.origin, golden[f"p{q}_origin"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(fm.origin, golden[f"p{q}_field_origin"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(patch.mesh.x, golden[f"p{q}_x"], rtol=0, atol=1e-15)
        inner = [[s.start or 0, s.stop if s.stop is not None else -1] for s in patch.inner]
        np.testing.assert_array_equal(np.array(inner), golden[f"p{q}_inner"])
        scale = np.abs(golden[f"p{q}_values"]).max()
        np.testing.assert_allclose(values[q], golden[f"p{q}_values"], rtol=0, atol=1e-12 * scale)
        fx, fy = fields[q]
        fscale = max(np.abs(golden[f"p{q}_fx"]).max(), np.abs(golden[f"p{q}_fy"]).max())
        np.testing.assert_allclose(fx, golden[f"p{q}_fx"], rtol=0, atol=1e-10 * fscale)
        np.testing.assert_allclose(fy, golden[f"p{q}_fy"], rtol=0, atol=1e-10 * fscale)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_the_composite_scheme_keeps_the_plates_linear_field(geometry) -> None:
    """The reference's linear plates (``test_ion_optics.py:67-72``, atol 1e-9) on refined
    boxes: with no charge the potential between two plates is linear in x, which every
    patch's rows and the hanging nodes' interpolation reproduce exactly, on and off the axis
    and on a graded axis."""
    faces = {"x_min": FaceCondition("dirichlet", 0.0), "x_max": FaceCondition("dirichlet", 100.0)}
    for x_nodes in (None, graded_nodes(21, 0.0, 20e-3)):
        mesh = IonOpticsMesh((21, 11), (0.0, 0.0), 1e-3, geometry, faces=faces, x_nodes=x_nodes,
                             classify_on_device=False)  # fmt: skip
        layout = layout_of_mesh(mesh, [Refinement(1, (4e-3, 0.0), (14e-3, 6e-3)),
                                       Refinement(2, (6e-3, 2e-3), (10e-3, 4e-3))])  # fmt: skip
        assert layout.hanging.size > 0
        phi = composite.solve(layout)
        np.testing.assert_allclose(phi, 100.0 * layout.x / 20e-3, rtol=0, atol=1e-9)


def random_boxes(seed: int, classify_on_device: bool | None = False):
    """A 17 x 9 mesh (planar for even seeds, cylindrical for odd ones, Dirichlet x faces
    at 0 and 10 V) and seeded nested boxes of levels 1-3, each side inset or on the face
    of the box (or mesh) below."""
    rng = np.random.default_rng(seed)
    geometry = ("planar", "cylindrical")[seed % 2]
    faces = {"x_min": FaceCondition("dirichlet", 0.0), "x_max": FaceCondition("dirichlet", 10.0)}
    mesh = IonOpticsMesh((17, 9), (0.0, 0.0), 1e-3, geometry, faces=faces,
                         classify_on_device=classify_on_device)  # fmt: skip
    boxes, lower, upper = [], np.array([0.0, 0.0]), np.array([16e-3, 8e-3])
    for level in (1, 2, 3):
        span = upper - lower
        lo = lower + rng.uniform(0.0, 0.3, 2) * span * rng.integers(0, 2, 2)
        hi = upper - rng.uniform(0.0, 0.3, 2) * span * rng.integers(0, 2, 2)
        boxes.append(Refinement(level, tuple(lo), tuple(hi)))
        # the next level inside this one's snapped extent
        patch = patches_of(mesh, boxes)[-1]
        x0, y0, x1, y1 = patch.bounds
        lower, upper = np.array([x0, y0]), np.array([x1, y1])
    return mesh, boxes


@pytest.mark.parametrize("seed", range(6))
def test_random_nested_boxes_keep_the_layout_invariants(seed) -> None:
    """Seeded nested boxes of levels 1-3, touching faces or not: the volumes fill the
    domain, every patch node is a composite node, the hanging nodes read only nodes that do
    not hang and interpolate planes exactly, and the composite scheme keeps the plates'
    linear field."""
    mesh, boxes = random_boxes(seed)
    geometry = mesh.geometry
    layout = layout_of_mesh(mesh, boxes)
    total = 16e-3 * 8e-3 if geometry == "planar" else np.pi * 8e-3**2 * 16e-3
    assert layout.volumes.sum() == pytest.approx(total, rel=1e-12)
    assert np.all(layout.volumes > 0.0)
    for patch in layout.patches:
        np.testing.assert_allclose(layout.x[patch.index], patch.mesh.nodes()[0], atol=1e-15)
        np.testing.assert_allclose(layout.y[patch.index], patch.mesh.nodes()[1], atol=1e-15)
    assert not set(layout.interpolation.indices.tolist()) & set(layout.hanging.tolist())
    plane = 2.0 * layout.x + 5.0 * layout.y
    filled = plane.copy()
    filled[layout.hanging] = 0.0
    layout.fill_hanging(filled)
    np.testing.assert_allclose(filled, plane, rtol=0, atol=1e-15)
    phi = composite.solve(layout)
    np.testing.assert_allclose(phi, 10.0 * layout.x / 16e-3, rtol=0, atol=1e-9)
