"""The deposit entry point that allocates nothing, against the one that does.

``bt_deposit_trajectories_2d_noalloc`` serves callers that may not allocate device memory
(their memory is budgeted by another allocator, or they cannot take cudaMalloc's implicit
device synchronisation where they deposit): its scratch is a fixed static device array.
Called through the C ABI on two deposits in a row, it must give the node charges of
``bt_deposit_trajectories_2d`` (the same kernels in the same order: the same bits, within
the deposit tests' 1e-13 in any case), and it must refuse sizes beyond its array.  This
file is collected last, so a run that stops at its first failure has run everything else.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(seed: int, n: int, nx: int, ny: int, cylindrical: int):
    import torch

    rng = np.random.default_rng(seed)
    h = 0.1
    px = rng.uniform(-0.2, (nx + 0.5) * h, n)
    low = 0.0 if cylindrical else -0.2
    py = rng.uniform(low, (ny + 0.5) * h, n)
    px[: n // 5] = 1.234  # a crowded cell: its records span many warps
    py[: n // 5] = 0.567
    q = rng.normal(size=n)
    return [torch.from_numpy(a).cuda() for a in (px, py, q)]


def _call_noalloc(lib, stream, px, py, q, h, cylindrical, charge):
    from beamtracer_b200 import _lib

    nx, ny = charge.shape
    return lib.bt_deposit_trajectories_2d_noalloc(
        ctypes.c_void_p(stream), _lib.dptr(px), _lib.dptr(py), _lib.dptr(q), px.numel(), 0.0,
        0.0, h, cylindrical, _lib.dptr(charge), nx, ny,
    )  # fmt: skip


def test_noalloc_deposit_matches_the_allocating_one_twice_in_a_row():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200 import _lib
    from beamtracer_b200.kernels import deposit_trajectories_2d

    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(21, 60_000, 200, 300, 1), (22, 65_536, 256, 256, 0)]
    for seed, n, nx, ny, cylindrical in cases:
        px, py, q = _inputs(seed, n, nx, ny, cylindrical)
        expected = torch.full((nx, ny), 0.5, dtype=torch.float64, device="cuda")
        deposit_trajectories_2d(px, py, q, 0.0, 0.0, 0.1, cylindrical, expected)
        result = torch.full((nx, ny), 0.5, dtype=torch.float64, device="cuda")
        _lib.check(_call_noalloc(lib, stream, px, py, q, 0.1, cylindrical, result))
        torch.cuda.synchronize()
        e, r = expected.cpu().numpy(), result.cpu().numpy()
        np.testing.assert_allclose(r, e, rtol=0, atol=1e-13 * np.abs(e).max())
        # the total charge is the charges' sum on top of the start values
        assert r.sum() == pytest.approx(0.5 * nx * ny + q.sum().item(), rel=1e-12)


def test_noalloc_deposit_refuses_sizes_beyond_its_scratch():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200 import _lib

    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    px, py, q = _inputs(3, 65_537, 10, 10, 0)
    charge = torch.zeros((10, 10), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="65536 charges"):
        _lib.check(_call_noalloc(lib, stream, px, py, q, 0.1, 0, charge))
    small = [a[:100] for a in (px, py, q)]
    big_mesh = torch.zeros((300, 300), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="65536 nodes"):
        _lib.check(_call_noalloc(lib, stream, *small, 0.1, 0, big_mesh))
