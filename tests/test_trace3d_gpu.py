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
