"""The oracle against the golden fixtures made by running the reference's own kernels.

The fixtures (``tests/golden/*.npz``) hold the inputs and outputs of the reference's Pyccel
kernel sources run as Python, and of its NumPy versions; ``tests/golden/make_golden.py``
made them.  The oracle's C restatement must give the same statuses, steps, electrode
indices, hit and path counts exactly, and the same floating-point outputs to rounding
(the one deliberate difference: the radius as sqrt(y^2 + z^2) rather than libm's hypot).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import kernels as oracle
from tests.golden.cases import (
    TRACE_CHARGE,
    TRACE_OUTPUTS,
    copy_args,
    trace3d_case_names,
    trace_case_names,
)

GOLDEN = Path(__file__).resolve().parent / "golden"
EXACT = ("steps", "status", "electrode", "counts", "path_count")


def _load(name: str):
    data = np.load(GOLDEN / f"{name}.npz")
    count = sum(1 for key in data.files if key.startswith("in_"))
    args = [data[f"in_{i}"] for i in range(count)]
    args = [a.item() if a.ndim == 0 else a.copy() for a in args]
    out = [data[f"out_{i}"] for i in range(count)]
    return args, out


@pytest.mark.parametrize("seed", [4, 5, 6])
@pytest.mark.parametrize("version", ["pyccel", "numpy"])
def test_gather_matches_the_reference(seed, version):
    args, expected = _load(f"gather_s{seed}_{version}")
    oracle.staggered_field_2d(*args)
    for i in (7, 8):
        np.testing.assert_allclose(args[i], expected[i], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("seed", [4, 5, 6])
@pytest.mark.parametrize("cylindrical", [0, 1])
@pytest.mark.parametrize("version", ["pyccel", "numpy"])
def test_deposit_matches_the_reference(seed, cylindrical, version):
    args, expected = _load(f"deposit_s{seed}_c{cylindrical}_{version}")
    oracle.deposit_trajectories_2d(*args)
    np.testing.assert_allclose(args[7], expected[7], rtol=1e-13, atol=1e-13)
    # charge is conserved
    assert args[7].sum() == pytest.approx(args[2].sum(), abs=1e-12)


@pytest.mark.parametrize("name", [name for name, _ in trace_case_names()])
def test_trace_matches_the_reference(name):
    args, expected = _load(name)
    oracle.trace_trajectories_2d(*args)
    for key, i in TRACE_OUTPUTS.items():
        if key in EXACT:
            np.testing.assert_array_equal(args[i], expected[i], err_msg=key)
        else:
            np.testing.assert_allclose(args[i], expected[i], rtol=1e-12, atol=1e-12,
                                       err_msg=key)  # fmt: skip
    np.testing.assert_allclose(
        args[TRACE_CHARGE].sum(0), expected[TRACE_CHARGE].sum(0), rtol=1e-12,
        atol=1e-12 * np.abs(expected[TRACE_CHARGE]).max(),
    )  # fmt: skip


@pytest.mark.parametrize("name", [name for name, _ in trace3d_case_names()])
def test_trace3d_matches_the_reference(name):
    """The 3D oracle restates the reference's 3D kernel: every output bit for bit (the
    Boris cases through the stand-in for mpiparticles' Boris push in both)."""
    from oracle.trace3d import trace_trajectories_3d
    from tests.gpu_util import load_golden

    args, out = load_golden(name)
    result = copy_args(args)
    trace_trajectories_3d(*result)
    for i, (got, want) in enumerate(zip(result, out, strict=True)):
        np.testing.assert_array_equal(np.asarray(got), np.asarray(want), err_msg=f"argument {i}")
