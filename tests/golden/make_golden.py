"""Generate the golden fixtures of ``tests/golden/`` by running the reference's own code.

Run in the build container, where the reference source tree is readable::

    python tests/golden/make_golden.py [--reference /root/reference]

It loads the reference's kernel sources as plain Python modules -- the Pyccel versions of
``staggered_field_2d``, ``deposit_trajectories_2d`` and ``trace_trajectories_2d`` and the
NumPy versions of the first two (``src/beamtracer/kernels/*/``) -- runs them on the seeded
cases of ``tests/golden/cases.py`` and writes inputs and outputs as ``.npz`` files.  The
one module the trace kernel imports that is absent here, ``mpiparticles``' Lorentz factor,
is stood in for by ``sqrt(1 + |u|^2 inv_c2)`` (the form the kernel's docstring states).

The fixtures are small (kilobytes) and committed; nothing on a GPU machine reads the
reference.
"""

from __future__ import annotations

import argparse
import importlib.util
import math
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from tests.golden.cases import (  # noqa: E402
    copy_args,
    deposit_case,
    gather_case,
    trace_case,
    trace_case_names,
)


def _lorentz_factor(u0, u1, u2, inv_c2):
    return math.sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2)


def _load(path: Path, name: str) -> types.ModuleType:
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def reference_kernels(root: Path) -> dict:
    """The reference's kernel functions, by name and version."""
    shim = types.ModuleType("mpiparticles.kernels.boris_pyccel")
    shim.lorentz_factor = _lorentz_factor
    sys.modules.setdefault("mpiparticles", types.ModuleType("mpiparticles"))
    sys.modules.setdefault("mpiparticles.kernels", types.ModuleType("mpiparticles.kernels"))
    sys.modules["mpiparticles.kernels.boris_pyccel"] = shim
    kernels = root / "src" / "beamtracer" / "kernels"
    out = {}
    for name in ("staggered_field_2d", "deposit_trajectories_2d", "trace_trajectories_2d"):
        for version in ("pyccel", "numpy"):
            path = kernels / name / f"{name}_{version}.py"
            if path.exists():
                module = _load(path, f"_ref_{name}_{version}")
                out[(name, version)] = getattr(module, name)
    return out


def _save(name: str, args: list, result: list, extra: dict | None = None) -> None:
    arrays = {}
    for i, (a, r) in enumerate(zip(args, result, strict=True)):
        arrays[f"in_{i}"] = np.asarray(a)
        arrays[f"out_{i}"] = np.asarray(r)
    for key, value in (extra or {}).items():
        arrays[key] = np.asarray(value)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default="/root/reference")
    root = Path(parser.parse_args().reference)
    ref = reference_kernels(root)

    for seed in (4, 5, 6):
        args = gather_case(seed)
        for version in ("pyccel", "numpy"):
            result = copy_args(args)
            ref[("staggered_field_2d", version)](*result)
            _save(f"gather_s{seed}_{version}", args, result)
        for cylindrical in (0, 1):
            args = deposit_case(seed, cylindrical)
            for version in ("pyccel", "numpy"):
                result = copy_args(args)
                ref[("deposit_trajectories_2d", version)](*result)
                _save(f"deposit_s{seed}_c{cylindrical}_{version}", args, result)

    kernel = ref[("trace_trajectories_2d", "pyccel")]
    for name, combo in trace_case_names():
        args = trace_case(*combo)
        result = copy_args(args)
        kernel(*result)
        _save(name, args, result)
        status = result[6]
        print(name, "statuses", dict(zip(*np.unique(status, return_counts=True))),
              "max steps", int(result[5].max()))  # fmt: skip


if __name__ == "__main__":
    main()
