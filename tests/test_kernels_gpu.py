"""The CUDA kernels against the oracle and the reference's golden outputs (on a B200).

The gather and the tracer's per-trajectory outputs (positions, velocities, steps,
statuses, electrodes, plane crossings, kept paths) must equal the oracle's bit for bit:
both evaluate the reference's expressions in the same order in FP64 without fused
multiply-adds.  The node charges are sums in a different order (sorted per cell on the
GPU, trajectory by trajectory on the CPU), so they agree to rounding: 1e-12 of the
largest node charge.  The GPU deposit is deterministic: repeated calls agree bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import kernels as oracle
from tests.golden.cases import TRACE_CHARGE, TRACE_OUTPUTS, copy_args, trace_case_names
from tests.gpu_util import load_golden, to_device, to_host

pytestmark = pytest.mark.gpu

EXACT = ("steps", "status", "electrode", "counts", "path_count")


@pytest.fixture(scope="module")
def kernels():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200.kernels import KERNELS

    return KERNELS


@pytest.mark.parametrize("seed", [4, 5, 6])
def test_gather_matches_the_oracle_bit_for_bit(kernels, seed):
    args, golden = load_golden(f"gather_s{seed}_pyccel")
    expected = copy_args(args)
    oracle.staggered_field_2d(*expected)
    device = to_device(args)
    kernels["staggered_field_2d"](*device)
    result = to_host(device)
    for i in (7, 8):
        np.testing.assert_array_equal(result[i], expected[i])
        np.testing.assert_allclose(result[i], golden[i], rtol=1e-13, atol=1e-13)


def test_gather_takes_host_arrays(kernels):
    args, golden = load_golden("gather_s4_pyccel")
    kernels["staggered_field_2d"](*args)
    np.testing.assert_allclose(args[7], golden[7], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("seed", [4, 5, 6])
@pytest.mark.parametrize("cylindrical", [0, 1])
def test_deposit_matches_the_oracle(kernels, seed, cylindrical):
    args, golden = load_golden(f"deposit_s{seed}_c{cylindrical}_pyccel")
    expected = copy_args(args)
    oracle.deposit_trajectories_2d(*expected)
    device = to_device(args)
    kernels["deposit_trajectories_2d"](*device)
    result = to_host(device)
    scale = np.abs(expected[7]).max()
    np.testing.assert_allclose(result[7], expected[7], rtol=0, atol=1e-13 * scale)
    np.testing.assert_allclose(result[7], golden[7], rtol=0, atol=1e-13 * scale)
    assert result[7].sum() == pytest.approx(args[2].sum(), abs=1e-12)


def test_deposit_is_deterministic_and_adds(kernels):
    import torch

    rng = np.random.default_rng(9)
    n, nx, ny = 200_000, 64, 48
    px = torch.from_numpy(rng.uniform(-0.1, 6.5, n)).cuda()
    py = torch.from_numpy(rng.uniform(0.0, 4.9, n)).cuda()
    # a hot cell: a quarter of the charges in one cell, so segments span many warps
    px[: n // 4] = 3.05
    py[: n // 4] = 2.05
    q = torch.from_numpy(rng.normal(size=n)).cuda()
    first = torch.full((nx, ny), 0.25, dtype=torch.float64, device="cuda")
    second = first.clone()
    kernels["deposit_trajectories_2d"](px, py, q, 0.0, 0.0, 0.1, 1, first)
    kernels["deposit_trajectories_2d"](px, py, q, 0.0, 0.0, 0.1, 1, second)
    assert torch.equal(first, second)
    expected = np.full((nx, ny), 0.25)
    oracle.deposit_trajectories_2d(
        px.cpu().numpy(), py.cpu().numpy(), q.cpu().numpy(), 0.0, 0.0, 0.1, 1, expected
    )
    np.testing.assert_allclose(first.cpu().numpy(), expected, rtol=0,
                               atol=1e-11 * np.abs(expected).max())  # fmt: skip


@pytest.mark.parametrize("name", [name for name, _ in trace_case_names()])
def test_trace_matches_the_oracle(kernels, name):
    args, golden = load_golden(name)
    expected = copy_args(args)
    oracle.trace_trajectories_2d(*expected)
    device = to_device(args)
    device[TRACE_CHARGE] = device[TRACE_CHARGE][:1].clone()  # one slab on the GPU
    kernels["trace_trajectories_2d"](*device, window=16)
    result = to_host(device)
    for key, i in TRACE_OUTPUTS.items():
        np.testing.assert_array_equal(result[i], expected[i], err_msg=key)
        if key in EXACT:
            np.testing.assert_array_equal(result[i], golden[i], err_msg=key)
        else:
            np.testing.assert_allclose(result[i], golden[i], rtol=1e-12, atol=1e-12,
                                       err_msg=key)  # fmt: skip
    total = expected[TRACE_CHARGE].sum(0)
    scale = np.abs(total).max()
    np.testing.assert_allclose(result[TRACE_CHARGE][0], total, rtol=0, atol=1e-12 * scale)


@pytest.mark.parametrize("window", [1, 5, 64, 1000])
def test_trace_windows_agree(kernels, window):
    import torch

    args, _ = load_golden("trace_c1_i0_r1_g0_rel0")
    runs = []
    for _ in range(2):
        device = to_device(args)
        device[TRACE_CHARGE] = device[TRACE_CHARGE][:1].clone()
        kernels["trace_trajectories_2d"](*device, window=window)
        runs.append(to_host(device))
    np.testing.assert_array_equal(runs[0][TRACE_CHARGE], runs[1][TRACE_CHARGE])
    reference = to_device(args)
    reference[TRACE_CHARGE] = reference[TRACE_CHARGE][:1].clone()
    kernels["trace_trajectories_2d"](*reference, window=64)
    reference = to_host(reference)
    for key, i in TRACE_OUTPUTS.items():
        np.testing.assert_array_equal(runs[0][i], reference[i], err_msg=key)
    scale = np.abs(reference[TRACE_CHARGE]).max()
    np.testing.assert_allclose(runs[0][TRACE_CHARGE], reference[TRACE_CHARGE], rtol=0,
                               atol=1e-13 * scale)  # fmt: skip
    del torch


@pytest.mark.parametrize("shape", [(200, 300), (500, 400), (1025, 600)])
def test_deposit_sorts_keys_of_every_width(kernels, shape):
    """Meshes of 60,000, 200,000 and 615,000 nodes: 16-, 18- and 20-bit cell keys, sorted
    with two passes of 8-, 9- and 10-bit digits."""
    import torch

    rng = np.random.default_rng(sum(shape))
    nx, ny = shape
    n = 300_000
    px = torch.from_numpy(rng.uniform(-0.05, 0.1 * nx, n)).cuda()
    py = torch.from_numpy(rng.uniform(0.0, 0.1 * ny, n)).cuda()
    q = torch.from_numpy(rng.normal(size=n)).cuda()
    charge = torch.zeros((nx, ny), dtype=torch.float64, device="cuda")
    kernels["deposit_trajectories_2d"](px, py, q, 0.0, 0.0, 0.1, 0, charge)
    expected = np.zeros((nx, ny))
    oracle.deposit_trajectories_2d(
        px.cpu().numpy(), py.cpu().numpy(), q.cpu().numpy(), 0.0, 0.0, 0.1, 0, expected
    )
    np.testing.assert_allclose(charge.cpu().numpy(), expected, rtol=0,
                               atol=1e-12 * np.abs(expected).max())  # fmt: skip


def test_trace_of_many_copies_equals_one(kernels):
    """A golden case tiled 5,625 times (270,000 trajectories, windows of 2,110 blocks: the
    compaction's scanned block offsets): every copy ends as the single case ends, bit for
    bit, and the node charges are 5,625 times the single case's."""
    args, _ = load_golden("trace_c1_i0_r1_g0_rel0")
    n = args[1].shape[1]
    copies = 270_000 // n
    single = to_device(args)
    single[TRACE_CHARGE] = single[TRACE_CHARGE][:1].clone()
    kernels["trace_trajectories_2d"](*single, window=64)
    single = to_host(single)
    tiled = list(args)
    tiled[0] = np.concatenate([args[0] + c * n for c in range(copies)])
    for i in (1, 2):
        tiled[i] = np.tile(args[i], (1, copies))
    for i in (3, 4, 5, 6, 7):
        tiled[i] = np.tile(args[i], copies)
    tiled[25] = np.tile(args[25], (copies, 1, 1, 1))
    tiled[26] = np.tile(args[26], (copies, 1))
    tiled[27] = np.concatenate([args[27], np.full(n * (copies - 1), -1, dtype=np.int64)])
    device = to_device(tiled)
    device[TRACE_CHARGE] = device[TRACE_CHARGE][:1].clone() * 0.0
    kernels["trace_trajectories_2d"](*device, window=64)
    result = to_host(device)
    for key, i in TRACE_OUTPUTS.items():
        if key in ("paths", "path_count"):
            np.testing.assert_array_equal(result[i], single[i], err_msg=key)
            continue
        axis = 1 if key in ("x", "v") else 0
        for c in (0, copies // 2, copies - 1):
            part = np.take(result[i], np.arange(c * n, (c + 1) * n), axis=axis)
            np.testing.assert_array_equal(part, single[i], err_msg=f"{key}, copy {c}")
    expected = copies * (single[TRACE_CHARGE][0] - args[TRACE_CHARGE][0])
    scale = np.abs(expected).max()
    np.testing.assert_allclose(result[TRACE_CHARGE][0], expected, rtol=0, atol=1e-11 * scale)
