"""Helpers of the GPU tests: golden fixtures and device copies of argument lists."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden(name: str):
    """The inputs and the reference's outputs of a golden fixture."""
    data = np.load(GOLDEN / f"{name}.npz")
    count = sum(1 for key in data.files if key.startswith("in_"))
    args = [data[f"in_{i}"] for i in range(count)]
    args = [a.item() if a.ndim == 0 else a.copy() for a in args]
    out = [data[f"out_{i}"] for i in range(count)]
    return args, out


def to_device(args: list) -> list:
    """Torch CUDA copies of the arrays of an argument list (scalars kept)."""
    import torch

    return [torch.from_numpy(a.copy()).cuda() if isinstance(a, np.ndarray) else a for a in args]


def to_host(args: list) -> list:
    return [a.cpu().numpy() if hasattr(a, "cpu") else a for a in args]
