"""The convergence reductions keep a NaN: a potential or density that blows up must not
read as converged (the reference's ``np.max(np.abs(...))`` propagates NaN, so its
``change < tolerance`` stays false)."""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the GPU tests need a CUDA device")
    from beamtracer_b200 import _lib

    return _lib


def test_max_abs_diff_keeps_nan(lib):
    import torch

    a = torch.zeros(100_000, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    b[12_345] = 3.0
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx = lib.context()
    lib.check(lib.lib().bt_max_abs_diff(ctx.handle, lib.dptr(a), lib.dptr(b), a.numel(),
                                        lib.dptr(out)))  # fmt: skip
    assert float(out) == 3.0
    a[77_777] = float("nan")
    lib.check(lib.lib().bt_max_abs_diff(ctx.handle, lib.dptr(a), lib.dptr(b), a.numel(),
                                        lib.dptr(out)))  # fmt: skip
    assert math.isnan(float(out))


def test_vlasov_mix_keeps_nan(lib):
    import torch

    nx, ny = 64, 33
    charge = torch.ones(nx * ny, dtype=torch.float64, device="cuda")
    volumes = torch.ones_like(charge)
    rho = torch.zeros_like(charge)
    stats = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx = lib.context()
    lib.check(lib.lib().bt_vlasov_mix(ctx.handle, lib.dptr(charge), lib.dptr(volumes), None,
                                      nx, ny, 0.5, 0, lib.dptr(rho), lib.dptr(stats)))  # fmt: skip
    np.testing.assert_allclose(stats.cpu().numpy(), [0.5, 0.5])
    charge[1000] = float("nan")
    lib.check(lib.lib().bt_vlasov_mix(ctx.handle, lib.dptr(charge), lib.dptr(volumes), None,
                                      nx, ny, 0.5, 0, lib.dptr(rho), lib.dptr(stats)))  # fmt: skip
    assert all(math.isnan(v) for v in stats.cpu().numpy())
