"""The 3D trace kernel on the device against the reference's own 3D kernel.

The golden cases (``tests/golden/trace3d_*.npz``) are the reference's Pyccel source run as
Python on seeded inputs: RK4 and Boris, a refined patch, symmetry planes at the lower y and
z faces, a magnetic field on the nodes, the current deposit and the step limit.  Every
trajectory must end where the reference ends it, bit for bit: state, steps, status,
electrode, plane crossings and kept paths.  The space charge and current are the same
shares summed in another order (records sorted by node, not the reference's per-thread
slabs): within 1e-13 of the largest.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden.cases import copy_args, trace3d_case_names
from tests.gpu_util import load_golden, to_device, to_host

pytestmark = pytest.mark.gpu

#: the exact outputs (argument positions): x, v, steps, status, electrode, hits, counts,
#: paths, path_count
EXACT = (1, 2, 5, 6, 7, 31, 32, 34, 35)
CHARGE, CURRENT = 37, 39


def _run(args, window: int = 0):
    from beamtracer_b200.kernels import KERNELS

    device = to_device(copy_args(args))
    KERNELS["trace_trajectories_3d"](*device, window=window)
    return to_host(device)


def _close(got: np.ndarray, want: np.ndarray, rel: float = 1e-13) -> None:
    scale = max(float(np.abs(want).max()), 1e-300)
    assert float(np.abs(got - want).max()) <= rel * scale


@pytest.mark.parametrize("name", [name for name, _ in trace3d_case_names()])
def test_trace3d_matches_the_reference(name):
    args, out = load_golden(name)
    got = _run(args)
    for i in EXACT:
        np.testing.assert_array_equal(got[i], out[i], err_msg=f"argument {i}")
    # the device adds every share into row 0; the reference into its threads' slabs
    _close(got[CHARGE].sum(axis=0), out[CHARGE].sum(axis=0))
    if args[38]:
        _close(got[CURRENT].sum(axis=0), out[CURRENT].sum(axis=0))


@pytest.mark.parametrize("window", [1, 7, 64])
def test_trace3d_window_changes_nothing(window):
    name = "trace3d_i1_r1_m0_b1_j1"
    args, out = load_golden(name)
    got = _run(args, window)
    for i in EXACT:
        np.testing.assert_array_equal(got[i], out[i], err_msg=f"argument {i}")
    _close(got[CHARGE].sum(axis=0), out[CHARGE].sum(axis=0))


def test_trace3d_of_many_copies_equals_one():
    """16,000 trajectories: 500 copies of one case's 32, each ending as the single copy."""
    name = "trace3d_i0_r1_m1_b1_j0"
    args, out = load_golden(name)
    copies = 500
    n = args[1].shape[1]
    big = copy_args(args)
    big[0] = np.arange(n * copies, dtype=np.int64)
    for i in (1, 2):
        big[i] = np.tile(args[i], (1, copies))
    for i in (3, 4, 5, 6, 7, 33):
        big[i] = np.tile(args[i], copies)
    big[33] = np.full(n * copies, -1, dtype=np.int64)  # no kept paths
    big[31] = np.zeros((n * copies,) + args[31].shape[1:])
    big[32] = np.zeros((n * copies, args[32].shape[1]), dtype=np.int64)
    got = _run(big)
    for c in range(copies):
        t = slice(c * n, (c + 1) * n)
        np.testing.assert_array_equal(got[1][:, t], out[1])
        np.testing.assert_array_equal(got[5][t], out[5])
        np.testing.assert_array_equal(got[6][t], out[6])
        np.testing.assert_array_equal(got[32][t], out[32])
    _close(got[CHARGE].sum(axis=0), copies * out[CHARGE].sum(axis=0), 1e-12)


def test_trace3d_rejects_bad_arguments():
    from beamtracer_b200.kernels import KERNELS

    args, _ = load_golden("trace3d_i0_r0_m0_b0_j0")
    with pytest.raises(TypeError):
        KERNELS["trace_trajectories_3d"](*args[:40])
    bad = copy_args(args)
    bad[11] = bad[11].copy()
    bad[11][-1, 7] = 10**6  # the base patch's nodes outside the charge rows
    with pytest.raises(ValueError):
        KERNELS["trace_trajectories_3d"](*to_device(bad))


def test_edge_field_3d_matches_the_reference():
    """The device's 3D edge fields of the golden mesh's seeded potential equal the
    reference's ``StaggeredElectricField3D`` bit for bit."""
    from beamtracer_b200.geometry3d import StaggeredElectricField3D
    from tests.gpu_util import GOLDEN
    from tests.test_mesh3d import _mesh

    golden = np.load(GOLDEN / "mesh3d_plate_sphere.npz")
    field = StaggeredElectricField3D(_mesh(), golden["phi"])
    for name in ("fx", "fy", "fz"):
        np.testing.assert_array_equal(getattr(field, name), golden[name], err_msg=name)


@pytest.mark.parametrize("integrator", ["rk4", "boris"])
def test_beam_tracer_3d_equals_the_oracle_driven_tracer(integrator):
    """The 3D tracer on the device and the same host logic around the oracle's kernel:
    equal ends, crossings and paths, charge and current within 1e-13 -- including the
    trajectories stopped in cut sub-cells and tested against the electrodes here."""
    from oracle.trace3d import trace_trajectories_3d as oracle_kernel

    from beamtracer_b200.geometry3d import BeamTracer3D, StaggeredElectricField3D
    from beamtracer_b200.tracer import BeamParticles
    from tests.test_mesh3d import _mesh

    mesh = _mesh()
    rng = np.random.default_rng(7)
    # a smooth field pushing +x, with the electrodes' potentials held
    phi = np.where(mesh.fixed, mesh.fixed_value, -2.0e4 * mesh.nodes()[0])
    field = StaggeredElectricField3D(mesh, phi)
    n = 200
    position = np.stack([np.full(n, 0.5e-3), rng.uniform(0.0, 4.5e-3, n),
                         rng.uniform(0.5e-3, 4.5e-3, n)])  # fmt: skip
    velocity = np.stack([np.full(n, 5.0e5), 2.0e4 * rng.normal(size=n),
                         2.0e4 * rng.normal(size=n)])  # fmt: skip
    particles = BeamParticles(position=position, velocity=velocity,
                              charge=np.full(n, 1.602176634e-19),
                              mass=np.full(n, 1.67262192e-27),
                              current=np.full(n, 1.0e-6), species=np.zeros(n, np.int32))  # fmt: skip
    magnetic = 0.05 * np.ones((3, *mesh.shape))
    results = []
    for kernel in (None, oracle_kernel):
        tracer = BeamTracer3D(mesh, field, magnetic, planes=(6.0e-3, 10.5e-3),
                              save_trajectories=7, integrator=integrator,
                              deposit_current=True, max_steps=400)  # fmt: skip
        tracer.kernel = kernel
        results.append(tracer.trace(particles))
    gpu, cpu = results
    np.testing.assert_array_equal(gpu.status, cpu.status)
    np.testing.assert_array_equal(gpu.electrode, cpu.electrode)
    assert gpu.steps == cpu.steps
    assert (cpu.status == 3).any() and (cpu.status == 0).any()
    for a, b in zip(gpu.planes, cpu.planes, strict=True):
        np.testing.assert_array_equal(a.point, b.point)
        np.testing.assert_array_equal(a.velocity, b.velocity)
    for a, b in zip(gpu.trajectories, cpu.trajectories, strict=True):
        np.testing.assert_array_equal(a, b)
    _close(gpu.charge_density, cpu.charge_density)
    _close(gpu.current_density, cpu.current_density)
