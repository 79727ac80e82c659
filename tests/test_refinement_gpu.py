"""Refined boxes on the device against the oracle: the sparse maps, the composite field
solve, the patches' field and the Vlasov iteration through them."""

from __future__ import annotations

import numpy as np
import pytest
from scipy import sparse
from scipy.constants import epsilon_0

from beamtracer_b200.mesh import Electrode, FaceCondition, IonOpticsMesh
from beamtracer_b200.refinement import Refinement, layout_of_mesh
from oracle import composite as oracle_composite

pytestmark = pytest.mark.gpu


def _box(x0, x1, y0, y1):
    return lambda x, y: (x >= x0) & (x <= x1) & (y >= y0) & (y <= y1)


def _extraction_mesh(geometry: str) -> IonOpticsMesh:
    """The reference's extraction geometry (``test_beam_optics.py:211-261``) without the
    plasma: 81 x 31 on 8 x 3 mm, two plates, Dirichlet x faces."""
    faces = {"x_min": FaceCondition("dirichlet", 5.0), "x_max": FaceCondition("dirichlet", -2000.0)}
    electrodes = [Electrode(_box(0.5e-3, 1e-3, 1e-3, 3.1e-3), 0.0),
                  Electrode(_box(3e-3, 4e-3, 1.2e-3, 3.1e-3), -2000.0)]  # fmt: skip
    return IonOpticsMesh((81, 31), (0.0, 0.0), 1e-4, geometry, electrodes=electrodes,
                         faces=faces, classify_on_device=False)  # fmt: skip


BOXES = {
    "axis": [Refinement(1, (0.0, 0.0), (2e-3, 1.5e-3)), Refinement(2, (0.0, 0.0), (1.5e-3, 1.2e-3))],
    "inside": [Refinement(1, (2.2e-3, 0.6e-3), (5e-3, 2.2e-3)),
               Refinement(2, (2.6e-3, 0.8e-3), (4.2e-3, 1.6e-3))],
}  # fmt: skip


def test_the_sparse_map_kernel_equals_scipy() -> None:
    import torch

    from beamtracer_b200.composite import DeviceCSR

    rng = np.random.default_rng(4)
    matrix = sparse.random(300, 500, density=0.02, random_state=5, format="csr")
    x = rng.standard_normal(500)
    constant = rng.standard_normal(300)
    y = torch.zeros(300, dtype=torch.float64, device="cuda")
    DeviceCSR(matrix, constant=constant).apply(torch.from_numpy(x).cuda(), y)
    np.testing.assert_allclose(y.cpu().numpy(), matrix @ x + constant, rtol=1e-14, atol=1e-14)
    # rows written to chosen places, added to what is there
    out_rows = rng.permutation(1000)[:300]
    z0 = rng.standard_normal(1000)
    z = torch.from_numpy(z0.copy()).cuda()
    DeviceCSR(matrix, out_rows=out_rows).apply(torch.from_numpy(x).cuda(), z, accumulate=True)
    want = z0.copy()
    want[out_rows] += matrix @ x
    np.testing.assert_allclose(z.cpu().numpy(), want, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
@pytest.mark.parametrize("boxes", ["axis", "inside"])
def test_the_composite_solve_equals_the_oracle(geometry, boxes) -> None:
    import torch

    from beamtracer_b200.poisson import IonOpticsPoisson

    mesh = _extraction_mesh(geometry)
    solver = IonOpticsPoisson(mesh, refinement=BOXES[boxes])
    layout = solver.layout
    assert layout.refined and layout.hanging.size > 0
    np.testing.assert_array_equal(solver.coordinates, np.stack([layout.x, layout.y]))
    rho = 1e-4 * np.exp(-((layout.x - 2e-3) ** 2 + layout.y**2) / (1e-3) ** 2)
    phi = solver.solve(rho)
    ora = oracle_composite.solve(oracle_layout(mesh, BOXES[boxes]), rho)
    span = np.ptp(ora)
    assert np.abs(phi - ora).max() <= 1e-9 * span
    assert solver._composite.sweeps < 120
    # a second solve from the first's potential changes nothing
    again = torch.from_numpy(phi.copy()).cuda()
    solver.solve_device(again, torch.from_numpy(rho).cuda())
    assert np.abs(again.cpu().numpy() - phi).max() <= 1e-10 * span


def oracle_layout(mesh, boxes):
    """The layout of the same mesh classified again on the host."""
    from tests.vlasov_cases import host_twin

    return layout_of_mesh(host_twin(mesh), boxes)


def test_a_uniform_charge_between_plates_on_refined_boxes_on_the_device() -> None:
    """The reference's known answer (``test_refinement.py:105-131``) through the device."""
    from beamtracer_b200.poisson import IonOpticsPoisson

    rho = 1e-6
    errors = []
    for n in (21, 41):
        faces = {"x_min": FaceCondition("dirichlet", 0.0),
                 "x_max": FaceCondition("dirichlet", 0.0)}  # fmt: skip
        mesh = IonOpticsMesh((n, (n + 1) // 2), (0.0, 0.0), 20e-3 / (n - 1), "planar",
                             faces=faces)  # fmt: skip
        solver = IonOpticsPoisson(mesh, refinement=[Refinement(1, (4e-3, 0.0), (14e-3, 6e-3)),
                                                    Refinement(2, (6e-3, 0.0), (10e-3, 4e-3))])  # fmt: skip
        layout = solver.layout
        phi = solver.solve(np.full(layout.size, rho))
        exact = rho / (2 * epsilon_0) * layout.x * (20e-3 - layout.x)
        errors.append(np.abs(phi - exact).max() / exact.max())
    assert errors[0] < 1e-2
    assert errors[1] < 0.6 * errors[0]


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_the_patches_fields_equal_the_oracle(geometry) -> None:
    from beamtracer_b200.composite import PatchedElectricField

    mesh = _extraction_mesh(geometry)
    boxes = BOXES["axis"] + [Refinement(1, (5.2e-3, 0.4e-3), (6.4e-3, 2.4e-3))]
    layout = layout_of_mesh(mesh, boxes)
    rng = np.random.default_rng(7)
    phi = np.where(layout.fixed, layout.fixed_value, 100.0 * rng.standard_normal(layout.size))
    field = PatchedElectricField(layout, phi)
    ora_layout = oracle_layout(mesh, boxes)
    for number, values in enumerate(oracle_composite.field_values(ora_layout, phi)):
        got = field.maps.values[number].cpu().numpy()
        np.testing.assert_allclose(got, values, rtol=0, atol=1e-12 * np.abs(values).max())
    fields, _ = oracle_composite.edge_fields(ora_layout, phi)
    for number, (fx, fy) in enumerate(fields):
        scale = max(np.abs(fx).max(), np.abs(fy).max())
        np.testing.assert_allclose(field.fields[number].fx, fx, rtol=0, atol=1e-11 * scale)
        np.testing.assert_allclose(field.fields[number].fy, fy, rtol=0, atol=1e-11 * scale)
    # at points the finest patch's field is taken
    x = np.array([1.0e-3, 1.4e-3, 5.8e-3, 7.5e-3])
    y = np.array([0.5e-3, 1.1e-3, 1.0e-3, 2.0e-3])
    # (the patches by level: the two level-1 boxes, then the level-2 box)
    assert field.patch_of(x, y).tolist() == [3, 3, 2, 0]


def _device_density(config, layout_host, potential):
    """G(phi) through the product's pieces: the patches' field of a composite potential,
    one trace through them, the composite density."""
    import torch

    from beamtracer_b200.composite import PatchedElectricField, PatchedFieldMaps
    from beamtracer_b200.model import BeamOptics

    model = BeamOptics(config)
    layout = layout_of_mesh(model.mesh, [Refinement(b.level, b.lower, b.upper)
                                         for b in config.refinement])  # fmt: skip
    assert layout.size == layout_host.size
    maps = PatchedFieldMaps(layout)
    PatchedElectricField(layout, torch.from_numpy(potential).cuda(), maps=maps)
    engine = model.tracer.engine()
    engine.set_patches(maps.patch_int, maps.patch_real, maps.n_field_nodes)
    particles, _ = model._particles()
    engine.load(particles)
    engine.run(maps.fx, maps.fy)
    charge = torch.zeros(layout.size, dtype=torch.float64, device="cuda")
    maps.charge_map.apply(engine.charge.reshape(-1), charge)
    return (charge / maps.volumes).cpu().numpy(), engine


def test_the_refined_vlasov_iteration_equals_the_oracle() -> None:
    """The reference's refined planar case (``test_refinement.py:134-165``: IBSimu's
    vlasov2d with a level-1 box over the emitter): per iteration the composite potential
    and density against the oracle's, and stage-wise the density the beam deposits in the
    oracle's potential within 1e-10 of its largest value."""
    from beamtracer_b200 import BeamOptics, RefinementParams
    from tests.vlasov_cases import refined_problem, slit_lens

    config = slit_lens(refinement=[RefinementParams(1, (0.0, 0.0), (0.04, 0.02))])
    gpu = []
    model = BeamOptics(config)
    model.run(lambda it, s: gpu.append((s.composite_potential.copy(),
                                        s.composite_charge_density.copy())))  # fmt: skip
    state = model.state
    assert state.layout.refined and state.composite_potential.size > state.potential.size
    assert state.potential.shape == model.mesh.shape
    fields = model.surface_fields()
    assert set(fields) == set(config.objects) and all(np.isfinite(list(fields.values())))
    assert model.beam_moments(0.115).current > 0.0
    problem, particles, _, layout = refined_problem(config)
    ora = []
    oracle_composite.vlasov(problem, layout, particles, iterations=3,
                            relaxation=config.relaxation, callback=lambda it, o: ora.append(
        (o["potential"].copy(), o["charge_density"].copy())))  # fmt: skip
    assert len(gpu) == len(ora) == 3
    span = np.ptp(ora[0][0])
    for (phi_g, rho_g), (phi_o, rho_o) in zip(gpu, ora):
        assert np.abs(phi_g - phi_o).max() <= 1e-8 * span
        assert np.abs(rho_g - rho_o).max() <= 1e-6 * np.abs(rho_o).max()
    # stage-wise: G(phi) in the oracle's own last potential
    phi_o = ora[-1][0]
    rho_dev, engine = _device_density(config, layout, phi_o)
    rho_ora, t = oracle_composite.density_of(problem, layout, phi_o, particles)
    assert np.abs(rho_dev - rho_ora).max() <= 1e-10 * np.abs(rho_ora).max()
    np.testing.assert_array_equal(engine.status.cpu().numpy(), t.status)


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_the_composite_newton_solve_and_held_region_equal_the_oracle(geometry) -> None:
    """A Boltzmann electron species on refined boxes (``poisson.py:627-757, 860-933``):
    Newton's composite steps against the oracle's; the initial plasma region held
    (``poisson.py:279-309``) against the oracle's."""
    from beamtracer_b200.poisson import BoltzmannElectrons, IonOpticsPoisson

    mesh = _extraction_mesh(geometry)
    solver = IonOpticsPoisson(mesh, refinement=BOXES["axis"])
    layout = solver.layout
    ora_layout = oracle_layout(mesh, BOXES["axis"])
    rho = 2e-4 * np.exp(-((layout.x - 2e-3) ** 2 + layout.y**2) / (1e-3) ** 2)
    region = lambda x, y: x < 0.6e-3  # noqa: E731
    held = solver.solve(rho, fixed_region=region, fixed_potential=5.0)
    ora_held = oracle_composite.solve_region(ora_layout, rho, region, 5.0)
    span = np.ptp(ora_held)
    assert np.abs(held - ora_held).max() <= 1e-9 * span
    plasma = BoltzmannElectrons(1.602e-2, 5.0, 5.0)
    phi = solver.solve(rho, plasma=plasma, initial=held, tolerance=1e-9)
    ora, _ = oracle_composite.solve_newton(ora_layout, rho, 1.602e-2 / epsilon_0, 5.0, 5.0, -1,
                                           initial=ora_held, tol=1e-11)  # fmt: skip
    assert solver.newton_iterations >= 2
    assert np.abs(phi - ora).max() <= 1e-8 * span


def test_the_refined_extraction_with_plasma_equals_the_oracle() -> None:
    """The reference's refined cylindrical case (``test_refinement.py:134-165``): the
    extraction from a plasma with boxes of levels 1 and 2 over the aperture, per iteration
    against the oracle (the held first iteration, then Newton with the Boltzmann
    electrons)."""
    from beamtracer_b200 import BeamOptics, RefinementParams
    from oracle import vlasov as oracle_vlasov
    from tests.vlasov_cases import extraction, refined_problem

    mm = 1e-3
    config = extraction(1.0, iterations=4, tolerance=0.0, refinement=[
        RefinementParams(1, (0.0, 0.0), (2.0 * mm, 1.5 * mm)),
        RefinementParams(2, (0.0, 0.0), (1.5 * mm, 1.2 * mm))])  # fmt: skip
    model = BeamOptics(config)
    gpu = []
    model.run(lambda it, s: gpu.append((s.composite_potential.copy(),
                                        s.composite_charge_density.copy())))  # fmt: skip
    assert model.state.history[-1]["newton_iterations"] >= 1
    problem, particles, j_over_v, layout = refined_problem(config)
    ora = []
    oracle_composite.vlasov(problem, layout, particles, iterations=4,
                            relaxation=config.relaxation,
                            plasma=oracle_vlasov.Plasma(5.0, 5.0, 0.6e-3, -1), j_over_v=j_over_v,
                            callback=lambda it, o: ora.append((o["potential"].copy(),
                                                               o["charge_density"].copy())))  # fmt: skip
    assert len(gpu) == len(ora) == 4
    for k, ((phi_g, rho_g), (phi_o, rho_o)) in enumerate(zip(gpu, ora)):
        np.testing.assert_allclose(phi_g, phi_o, rtol=0, atol=1e-7 * 2000.0, err_msg=f"{k}")
        np.testing.assert_allclose(rho_g, rho_o, rtol=0, atol=1e-7 * np.abs(rho_o).max(),
                                   err_msg=f"{k}")  # fmt: skip


@pytest.mark.parametrize("geometry", ["planar", "cylindrical"])
def test_refined_boxes_on_a_graded_axis_equal_the_oracle(geometry) -> None:
    """Boxes on a graded x (``test_graded_mesh.py:95-155``): the composite solve, the
    patches' fields and, stage-wise, the density a beam deposits through them, against the
    oracle."""
    import torch
    from scipy import constants

    from beamtracer_b200.composite import PatchedElectricField, PatchedFieldMaps
    from beamtracer_b200.poisson import IonOpticsPoisson
    from beamtracer_b200.tracer import BeamParticles, TraceEngine
    from tests.test_refinement import graded_nodes
    from tests.vlasov_cases import host_twin, mesh_problem

    faces = {"x_min": FaceCondition("dirichlet", 5.0), "x_max": FaceCondition("dirichlet", -2000.0)}
    electrodes = [Electrode(_box(0.5e-3, 1e-3, 1e-3, 3.1e-3), 0.0),
                  Electrode(_box(3e-3, 4e-3, 1.2e-3, 3.1e-3), -2000.0)]  # fmt: skip
    mesh = IonOpticsMesh((81, 31), (0.0, 0.0), 1e-4, geometry, x_nodes=graded_nodes(81, 0.0, 8e-3),
                         electrodes=electrodes, faces=faces)  # fmt: skip
    boxes = BOXES["axis"]
    solver = IonOpticsPoisson(mesh, refinement=boxes)
    layout = solver.layout
    ora_layout = layout_of_mesh(host_twin(mesh), boxes)
    np.testing.assert_array_equal(layout.x, ora_layout.x)
    rho = 1e-4 * np.exp(-((layout.x - 2e-3) ** 2 + layout.y**2) / (1e-3) ** 2)
    phi = solver.solve(rho)
    ora = oracle_composite.solve(ora_layout, rho)
    assert np.abs(phi - ora).max() <= 1e-9 * np.ptp(ora)
    # the beam through the patches of the oracle's potential
    n = 200
    mass = constants.m_p
    speed = np.sqrt(2.0 * 5.0 * constants.e / mass)
    position = np.zeros((3, n))
    position[0] = 1e-6
    position[1] = np.linspace(0.02e-3, 0.85e-3, n)
    velocity = np.zeros((3, n))
    velocity[0] = speed
    particles = BeamParticles(position, velocity, np.full(n, constants.e), np.full(n, mass),
                              np.full(n, 1e-6), np.zeros(n, dtype=np.int64))  # fmt: skip
    maps = PatchedFieldMaps(layout)
    PatchedElectricField(layout, torch.from_numpy(ora).cuda(), maps=maps)
    engine = TraceEngine(mesh, planes=(7.5e-3,))
    engine.set_patches(maps.patch_int, maps.patch_real, maps.n_field_nodes)
    engine.load(particles)
    engine.run(maps.fx, maps.fy)
    charge = torch.zeros(layout.size, dtype=torch.float64, device="cuda")
    maps.charge_map.apply(engine.charge.reshape(-1), charge)
    rho_dev = (charge / maps.volumes).cpu().numpy()
    problem = mesh_problem(mesh, planes=(7.5e-3,))
    rho_ora, t = oracle_composite.density_of(problem, ora_layout, ora, particles)
    np.testing.assert_array_equal(engine.status.cpu().numpy(), t.status)
    assert np.abs(rho_ora).max() > 0.0
    assert np.abs(rho_dev - rho_ora).max() <= 1e-10 * np.abs(rho_ora).max()


def test_refined_anderson_mixing_equals_the_oracle() -> None:
    """Anderson mixing on the composite nodes (``vlasov.py:127-173``): the refined slit
    lens per iteration against the oracle's NumPy mixer."""
    from beamtracer_b200 import BeamOptics, RefinementParams
    from tests.vlasov_cases import refined_problem, slit_lens

    config = slit_lens(iterations=5, mixing="anderson", anderson_depth=3, relaxation=0.7,
                       refinement=[RefinementParams(1, (0.0, 0.0), (0.04, 0.02))])  # fmt: skip
    gpu = []
    BeamOptics(config).run(lambda it, s: gpu.append((s.composite_potential.copy(),
                                                     s.composite_charge_density.copy())))  # fmt: skip
    problem, particles, _, layout = refined_problem(config)
    ora = []
    oracle_composite.vlasov(problem, layout, particles, iterations=5, relaxation=0.7,
                            mixing="anderson", anderson_depth=3,
                            callback=lambda it, o: ora.append((o["potential"].copy(),
                                                               o["charge_density"].copy())))  # fmt: skip
    assert len(gpu) == len(ora) == 5
    span = np.ptp(ora[0][0])
    for k, ((phi_g, rho_g), (phi_o, rho_o)) in enumerate(zip(gpu, ora)):
        assert np.abs(phi_g - phi_o).max() <= 1e-8 * span, k
        assert np.abs(rho_g - rho_o).max() <= 1e-6 * np.abs(rho_o).max(), k


def test_a_refined_box_brings_the_beam_to_that_of_the_fine_mesh() -> None:
    """The reference's behavioural case (``test_refinement.py:168-181``): a box around the
    extraction aperture moves the beam's divergence towards that of a mesh of half the
    cells everywhere."""
    from beamtracer_b200 import BeamOptics, GridParams, RefinementParams
    from tests.vlasov_cases import extraction

    def divergence(config) -> float:
        model = BeamOptics(config.replace(iterations=60, tolerance=1e-5)).run()
        return model.beam_moments(7.5e-3).rms_angle

    coarse = extraction(1.0)
    grid = coarse.grid
    fine = coarse.replace(grid=GridParams(num_gridpoints=(161, 61), lower_bound=grid.lower_bound,
                                          upper_bound=grid.upper_bound,
                                          coordinates=grid.coordinates))  # fmt: skip
    box = coarse.replace(refinement=[RefinementParams(1, (0.0, 0.0), (4.5e-3, 2.0e-3))])
    reference = divergence(fine)
    assert abs(divergence(box) - reference) < 0.5 * abs(divergence(coarse) - reference)


@pytest.mark.parametrize("seed", range(6))
def test_random_nested_boxes_solve_as_the_oracle(seed) -> None:
    """Seeded nested boxes of levels 1-3 (on and off the faces and the axis): the device's
    composite solve of a charge against the oracle's LU."""
    from beamtracer_b200.poisson import IonOpticsPoisson
    from tests.test_refinement import random_boxes

    mesh, boxes = random_boxes(seed, classify_on_device=None)
    solver = IonOpticsPoisson(mesh, refinement=boxes)
    layout = solver.layout
    rho = 1e-7 * np.exp(-((layout.x - 8e-3) ** 2 + (layout.y - 3e-3) ** 2) / (3e-3) ** 2)
    phi = solver.solve(rho)
    ora = oracle_composite.solve(oracle_layout(mesh, boxes), rho)
    assert np.abs(phi - ora).max() <= 1e-9 * np.ptp(ora)
