"""The library's work is ordered with torch's on torch's current stream (the default stream
included): a library kernel queued behind slow torch work sees that work's results, with
no synchronisation in between."""

from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("side", ["default", "side"])
def test_library_work_follows_torch_work_on_the_same_stream(side):
    import torch

    from beamtracer_b200 import _lib

    stream = torch.cuda.current_stream() if side == "default" else torch.cuda.Stream()
    n = 1 << 20
    with torch.cuda.stream(stream):
        a = torch.zeros(n, dtype=torch.float64, device="cuda")
        b = torch.zeros(n, dtype=torch.float64, device="cuda")
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        m = torch.randn(2048, 2048, device="cuda")
        for _ in range(30):  # slow work ahead of the write the library must see
            m = (m @ m).tanh_()
        b.fill_(3.0)
        ctx = _lib.context()
        _lib.check(_lib.lib().bt_max_abs_diff(ctx.handle, _lib.dptr(a), _lib.dptr(b), n,
                                              _lib.dptr(out)))  # fmt: skip
        result = out.cpu().item()
    assert result == 3.0
