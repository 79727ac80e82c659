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
    mesh_cases,
    trace_case,
    trace_case_names,
)


def _lorentz_factor(u0, u1, u2, inv_c2):
    return math.sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2)


def _load(path: Path, name: str) -> types.ModuleType:
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
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


def reference_mesh_module(root: Path) -> types.ModuleType:
    """The reference's ``solver/mesh.py`` (its one absent import, ``methodcard.method``, a
    decorator that records documentation, stood in for by the identity)."""
    card = types.ModuleType("methodcard")
    card.method = lambda *a, **k: (lambda obj: obj)
    sys.modules["methodcard"] = card
    return _load(root / "src" / "beamtracer" / "solver" / "mesh.py", "_ref_mesh")


def reference_edge_field(root: Path):
    """The reference's ``_edge_field`` (``solver/fields.py:18-67``), taken out of its module."""
    import ast

    source = (root / "src" / "beamtracer" / "solver" / "fields.py").read_text()
    tree = ast.parse(source)
    node = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "_edge_field")
    namespace = {"np": np}
    exec(compile(ast.Module(body=[node], type_ignores=[]), "fields.py", "exec"), namespace)
    return namespace["_edge_field"]


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

    mesh_module = reference_mesh_module(root)
    edge_field = reference_edge_field(root)
    for name, settings in mesh_cases().items():
        settings = dict(settings)
        electrodes = [mesh_module.Electrode(f, v) for f, v in settings.pop("electrodes")]
        faces = {k: mesh_module.FaceCondition(*v) for k, v in settings.pop("faces").items()}
        mesh = mesh_module.IonOpticsMesh(electrodes=electrodes, faces=faces, **settings)
        rng = np.random.default_rng(21)
        phi = np.where(mesh.fixed, mesh.fixed_value, rng.normal(size=mesh.shape) * 100.0)
        extrapolation = ["extrapolate"] * 4
        if mesh.cylindrical or mesh.symmetry_plane:
            extrapolation[2] = "symmetric"
        solid, near = mesh.solid >= 0, mesh.near_solid
        fx = edge_field(phi, solid, near, mesh.distance[0], mesh.distance[1], mesh.dx,
                        extrapolation[0:2])
        fy = np.ascontiguousarray(
            edge_field(phi.T, solid.T, near.T, mesh.distance[2].T, mesh.distance[3].T,
                       mesh.h, extrapolation[2:4]).T
        )  # fmt: skip
        np.savez_compressed(
            HERE / f"mesh_{name}.npz", solid=mesh.solid, fixed=mesh.fixed,
            fixed_value=mesh.fixed_value, distance=mesh.distance,
            near_solid=mesh.near_solid, phi=phi, fx=fx, fy=fy,
        )  # fmt: skip
        print("mesh", name, "near", int(near.sum()), "solid", int(solid.sum()))

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
