"""Generate the golden fixtures of ``tests/golden/`` by running the reference's own code.

Run in the build container, where the reference source tree is readable::

    python tests/golden/make_golden.py --reference <reference checkout>

(or with ``BEAMTRACER_REFERENCE`` set to the checkout).

It runs the reference's host functions that both arms share -- ``beam_with_energy``,
``plane_moments`` and ``AxisymmetricMagneticField`` with ``solenoid_on_axis``, taken out of
their modules' sources -- on the cases of ``tests/golden/host_cases.py``.  It loads the
reference's kernel sources as plain Python modules -- the Pyccel versions of
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
import os
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


def _relativistic_boris_update(u0, u1, u2, e0, e1, e2, b0, b1, b2, inv_c2):
    """The relativistic Boris push (J. P. Boris, 1970) as the 3D kernel calls
    ``mpiparticles``' ``relativistic_boris_update`` (absent here): a kick by the scaled
    field ``e``, the rotation by ``t = b / gamma`` with ``s = 2 t / (1 + t^2)``, and a
    second kick."""
    m0, m1, m2 = u0 + e0, u1 + e1, u2 + e2
    g = math.sqrt(1.0 + (m0 * m0 + m1 * m1 + m2 * m2) * inv_c2)
    t0, t1, t2 = b0 / g, b1 / g, b2 / g
    f = 2.0 / (1.0 + (t0 * t0 + t1 * t1 + t2 * t2))
    s0, s1, s2 = f * t0, f * t1, f * t2
    p0 = m0 + (m1 * t2 - m2 * t1)
    p1 = m1 + (m2 * t0 - m0 * t2)
    p2 = m2 + (m0 * t1 - m1 * t0)
    return (m0 + (p1 * s2 - p2 * s1) + e0, m1 + (p2 * s0 - p0 * s2) + e1,
            m2 + (p0 * s1 - p1 * s0) + e2)  # fmt: skip


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
    shim.relativistic_boris_update = _relativistic_boris_update
    sys.modules.setdefault("mpiparticles", types.ModuleType("mpiparticles"))
    sys.modules.setdefault("mpiparticles.kernels", types.ModuleType("mpiparticles.kernels"))
    sys.modules["mpiparticles.kernels.boris_pyccel"] = shim
    kernels = root / "src" / "beamtracer" / "kernels"
    out = {}
    for name in ("staggered_field_2d", "deposit_trajectories_2d", "trace_trajectories_2d",
                 "trace_trajectories_3d"):
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


def reference_surface_field(root: Path):
    """The reference's ``surface_field`` and ``_node_component`` (``solver/fields.py:
    323-377``), taken out of their module."""
    namespace = {"np": np, "Any": object}
    reference_definitions(root, "fields", ("_node_component", "surface_field"), namespace)
    return namespace["surface_field"]


def reference_definitions(root: Path, module: str, names: tuple[str, ...],
                          namespace: dict) -> dict:  # fmt: skip
    """Top-level definitions of a reference module, taken out of its source and run in
    ``namespace`` (their decorators that only record documentation left off, ``dataclass``
    kept): the module's absent imports are never executed."""
    import ast

    source = (root / "src" / "beamtracer" / "solver" / f"{module}.py").read_text()
    tree = ast.parse(source)
    picked = []
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            node.decorator_list = [
                d for d in node.decorator_list
                if isinstance(d, ast.Name) and d.id == "dataclass"
                or isinstance(d, ast.Call) and getattr(d.func, "id", "") == "dataclass"
            ]  # fmt: skip
            picked.append(node)
    missing = set(names) - {n.name for n in picked}
    if missing:
        raise RuntimeError(f"{module}.py has no {sorted(missing)}")
    exec(compile(ast.Module(body=picked, type_ignores=[]), f"{module}.py", "exec"), namespace)
    return namespace


def reference_host_functions(root: Path) -> dict:
    """The reference's beam seeding (``tracer.py:87-291``), plane crossings and moments
    (``tracer.py:295-325``, ``diagnostics.py:15-135``) and axisymmetric field
    (``fields.py:192-321``), in one namespace.  ``mpiparticles.lorentz_factor`` (absent) is
    stood in for by ``sqrt(1 + |u|^2 / c^2)`` of (3, N) proper velocities."""
    from collections.abc import Sequence
    from dataclasses import dataclass, field
    from typing import Any

    from scipy import constants

    def lorentz_factor(u, c):
        return np.sqrt(1.0 + np.sum(u * u, axis=0) / (c * c))

    module = types.ModuleType("_ref_host")  # dataclasses look their module up by name
    sys.modules[module.__name__] = module
    namespace = module.__dict__
    namespace.update({"np": np, "constants": constants, "dataclass": dataclass, "field": field,
                      "Sequence": Sequence, "Any": Any, "lorentz_factor": lorentz_factor})  # fmt: skip
    reference_definitions(root, "tracer", ("BeamParticles", "_gaussian_samples", "_beam_speeds",
                                           "beam_with_energy", "PlaneHits"), namespace)
    reference_definitions(root, "diagnostics", ("BeamMoments", "plane_moments"), namespace)
    reference_definitions(root, "fields", ("AxisymmetricMagneticField", "solenoid_on_axis"),
                          namespace)  # fmt: skip
    return namespace


def host_goldens(root: Path) -> None:
    """``host_*.npz``: the reference's beams, moments and magnetic fields on the cases of
    ``tests/golden/host_cases.py``."""
    from tests.golden import host_cases as hc

    ref = reference_host_functions(root)
    beams = {}
    for name, (args, kwargs) in hc.BEAM_CASES.items():
        kwargs = dict(kwargs)
        if "seed" in kwargs:
            kwargs["sampling"] = np.random.default_rng(kwargs.pop("seed"))
        particles, j_over_v = ref["beam_with_energy"](*args, **kwargs)
        for key in ("position", "velocity", "charge", "mass", "current", "species"):
            beams[f"{name}.{key}"] = getattr(particles, key)
        beams[f"{name}.j_over_v"] = np.array(j_over_v)
    np.savez_compressed(HERE / "host_beams.npz", **beams)

    moments = {}
    for name, (seed, cylindrical, species, forward, axis, mass_kind) in hc.MOMENT_CASES.items():
        h = hc.moment_hits(seed, cylindrical)
        if name == "planar_fast":
            h["velocity"] = h["velocity"] * 150.0  # about 0.7 c
        hits = ref["PlaneHits"](0.0)
        hits.append(h["point"], h["velocity"], h["current"], h["species"], h["direction"])
        mass = hc.MOMENT_MASSES if mass_kind == "array" else float(hc.MOMENT_MASSES[0])
        m = ref["plane_moments"](hits, cylindrical=cylindrical, mass=mass, species=species,
                                 forward_only=forward, axis=axis)  # fmt: skip
        moments[name] = np.array([getattr(m, k) for k in m.__dataclass_fields__], dtype=float)
    np.savez_compressed(HERE / "host_moments.npz", **moments)

    fields = {}
    field_class, solenoid = ref["AxisymmetricMagneticField"], ref["solenoid_on_axis"]
    for k, (name, (centre, length, radius, peak, z0, hz, n, order)) in enumerate(
            hc.FIELD_CASES.items()):  # fmt: skip
        z = z0 + hz * np.arange(n)
        profile = solenoid(z, centre, length, radius, peak)
        f = field_class(z0, hz, profile, order=order)
        pz, pr = hc.field_points(30 + k, z0, hz, n)
        bz, br = f(pz, pr)
        fields.update({f"{name}.profile": profile, f"{name}.table": f._samples,
                       f"{name}.bz": bz, f"{name}.br": br})  # fmt: skip
    lo, hi, h, solenoids, order = hc.SAMPLING_CASE
    dz = 0.5 * h
    z = np.arange(lo - 8 * dz, hi + 8.5 * dz, dz)  # the sampling of model.py:180-182
    bz = np.zeros(z.size)
    for centre, length, radius, peak in solenoids:
        bz = bz + solenoid(z, centre, length, radius, peak)
    f = field_class(float(z[0]), dz, bz, order=order)
    pz, pr = hc.field_points(40, lo, h, int((hi - lo) / h))
    fields["sampling.bz"], fields["sampling.br"] = f(pz, pr)
    fields["sampling.z0"], fields["sampling.count"] = np.array(z[0]), np.array(z.size)
    np.savez_compressed(HERE / "host_fields.npz", **fields)
    print("host goldens:", len(beams), "beam arrays,", len(moments), "moment cases,",
          len(fields), "field arrays")


def record_goldens(root: Path) -> None:
    """``record_*``: the design keys and the record lines of the reference's
    ``optimization/design.py`` (``Design.key``, ``Evaluation.to_dict``) and
    ``optimization/record.py`` (``Record.append``) on the cases of
    ``tests/golden/host_cases.py`` -- the record format a search resumes from."""
    import json

    from tests.golden import host_cases as hc

    card = types.ModuleType("methodcard")
    card.method = lambda *a, **k: (lambda obj: obj)
    sys.modules["methodcard"] = card
    units = types.ModuleType("plasmacoll.units")
    units.to_unit = lambda value, unit, name=None: float(value)
    sys.modules.setdefault("plasmacoll", types.ModuleType("plasmacoll"))
    sys.modules["plasmacoll.units"] = units
    opt = root / "src" / "beamtracer" / "optimization"
    design_module = _load(opt / "design.py", "_ref_design")
    for name in ("beamtracer", "beamtracer.optimization"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["beamtracer.optimization.design"] = design_module
    record_module = _load(opt / "record.py", "_ref_record")
    keys = {}
    for name, (parameters, points) in hc.RECORD_DESIGNS.items():
        design = design_module.Design(tuple(design_module.Parameter(*p) for p in parameters))
        keys[name] = [design.key(x) for x in points]
    (HERE / "record_keys.json").write_text(json.dumps(keys, indent=1) + "\n")
    parameters, points = hc.RECORD_DESIGNS[hc.RECORD_CASE]
    design = design_module.Design(tuple(design_module.Parameter(*p) for p in parameters))
    path = HERE / "record_reference.jsonl"
    if path.exists():
        path.unlink()
    record = record_module.Record(design, path)
    evaluations = [design_module.Evaluation(**e) for e in hc.record_evaluations(design.names, points)]
    record.append(evaluations)
    print("record goldens:", sum(len(v) for v in keys.values()), "keys,", len(record), "lines")


def mesh3d_goldens(root: Path) -> None:
    """The reference's ``IonOpticsMesh3D`` (``solver/mesh3d.py``) and
    ``StaggeredElectricField3D`` (``solver/fields3d.py``) on ``mesh3d_case``: the node
    classification and the edge fields of a seeded potential."""
    from collections.abc import Sequence

    from tests.golden.cases import mesh3d_case

    mesh2d = reference_mesh_module(root)
    for name in ("beamtracer", "beamtracer.solver"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["beamtracer.solver.mesh"] = mesh2d
    mesh3d = _load(root / "src" / "beamtracer" / "solver" / "mesh3d.py", "_ref_mesh3d")
    namespace = {"np": np, "Sequence": Sequence, "_edge_field": reference_edge_field(root),
                 "IonOpticsMesh3D": mesh3d.IonOpticsMesh3D}  # fmt: skip
    reference_definitions(root, "fields3d", ("_trilinear", "StaggeredElectricField3D"), namespace)
    settings = mesh3d_case()
    mesh = mesh3d.IonOpticsMesh3D(
        shape=settings["shape"], origin=settings["origin"], h=settings["h"],
        electrodes=[mesh3d.Electrode3D(f, v) for f, v in settings["electrodes"]],
        faces={k: mesh2d.FaceCondition(*v) for k, v in settings["faces"].items()},
        symmetry_planes=settings["symmetry_planes"],
    )  # fmt: skip
    rng = np.random.default_rng(23)
    phi = np.where(mesh.fixed, mesh.fixed_value, rng.normal(size=mesh.shape) * 100.0)
    field = namespace["StaggeredElectricField3D"](mesh, phi)
    np.savez_compressed(HERE / "mesh3d_plate_sphere.npz", solid=mesh.solid,
                        near_solid=mesh.near_solid, distance=mesh.distance, fixed=mesh.fixed,
                        fixed_value=mesh.fixed_value, phi=phi, fx=field.fx, fy=field.fy,
                        fz=field.fz)  # fmt: skip
    print("mesh3d near", int(mesh.near_solid.sum()), "solid", int((mesh.solid >= 0).sum()))


def trace3d_goldens(root: Path) -> None:
    """The reference's 3D trace kernel (its Pyccel source run as Python) on the cases of
    ``trace3d_case_names``.  Its Boris steps go through the stand-in for
    ``relativistic_boris_update`` above (mpiparticles is absent); its Runge--Kutta steps
    need only the Lorentz factor, 1 for these non-relativistic cases."""
    from tests.golden.cases import trace3d_case, trace3d_case_names

    kernel = reference_kernels(root)[("trace_trajectories_3d", "pyccel")]
    for name, combo in trace3d_case_names():
        args = trace3d_case(*combo)
        result = copy_args(args)
        kernel(*result)
        _save(name, args, result)
        status = result[6]
        print(name, "statuses", dict(zip(*np.unique(status, return_counts=True))),
              "max steps", int(result[5].max()))  # fmt: skip


def _save(name: str, args: list, result: list, extra: dict | None = None) -> None:
    arrays = {}
    for i, (a, r) in enumerate(zip(args, result, strict=True)):
        arrays[f"in_{i}"] = np.asarray(a)
        arrays[f"out_{i}"] = np.asarray(r)
    for key, value in (extra or {}).items():
        arrays[key] = np.asarray(value)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def refinement_goldens(root: Path) -> None:
    """The reference's refined patches (``solver/refinement.py:83-152``) and their fields
    (``PatchedElectricField``, ``:319-365``, its edge fields by the reference's
    ``_edge_field``) on the meshes of `mesh_cases` with the boxes of `refinement_cases`, for
    the potential `refinement_potential` at every patch's nodes."""
    from collections.abc import Sequence
    from dataclasses import dataclass
    from typing import Any

    from tests.golden.cases import mesh_cases, refinement_cases, refinement_potential

    mesh_module = reference_mesh_module(root)
    edge_field = reference_edge_field(root)

    class StaggeredElectricField:
        """The reference's edge fields of a potential (``fields.py:116-152``)."""

        def __init__(self, mesh, values, extrapolation) -> None:
            solid, near = mesh.solid >= 0, mesh.near_solid
            self.values = np.array(values, dtype=float)
            self.fx = edge_field(self.values, solid, near, mesh.distance[0], mesh.distance[1],
                                 mesh.dx, extrapolation[0:2])  # fmt: skip
            self.fy = np.ascontiguousarray(edge_field(
                self.values.T, solid.T, near.T, mesh.distance[2].T, mesh.distance[3].T, mesh.h,
                extrapolation[2:4]).T)  # fmt: skip

    namespace = {"np": np, "IonOpticsMesh": mesh_module.IonOpticsMesh, "Any": Any,
                 "StaggeredElectricField": StaggeredElectricField, "dataclass": dataclass,
                 "Sequence": Sequence}  # fmt: skip
    reference_definitions(root, "refinement", (
        "Refinement", "Patch", "_on_plane", "_part", "patches_of", "_extrapolation_of",
        "_bilinear", "PatchedElectricField"), namespace)  # fmt: skip
    for name, settings in mesh_cases().items():
        settings = dict(settings)
        electrodes = [mesh_module.Electrode(f, v) for f, v in settings.pop("electrodes")]
        faces = {k: mesh_module.FaceCondition(*v) for k, v in settings.pop("faces").items()}
        mesh = mesh_module.IonOpticsMesh(electrodes=electrodes, faces=faces, **settings)
        boxes = [namespace["Refinement"](*b) for b in refinement_cases()[name]]
        patches = namespace["patches_of"](mesh, boxes)
        values, start = [], 0
        for patch in patches:
            xn, yn = patch.mesh.nodes()
            patch.index = start + np.arange(xn.size).reshape(xn.shape)
            start += xn.size
            values.append(refinement_potential(xn, yn).ravel())
        layout = types.SimpleNamespace(patches=patches, base=patches[0])
        field = namespace["PatchedElectricField"](layout, np.concatenate(values))
        out = {}
        for q, (patch, f) in enumerate(zip(patches, field.fields)):
            fm = patch.field_mesh if patch.field_mesh is not None else patch.mesh
            out[f"p{q}_level"] = np.array(patch.level)
            out[f"p{q}_box"] = np.array(patch.box, dtype=np.int64)
            out[f"p{q}_shape"] = np.array(patch.mesh.shape)
            out[f"p{q}_origin"] = np.array(patch.mesh.origin)
            out[f"p{q}_x"] = np.asarray(patch.mesh.x, dtype=float)
            out[f"p{q}_field_shape"] = np.array(fm.shape)
            out[f"p{q}_field_origin"] = np.array(fm.origin)
            out[f"p{q}_inner"] = np.array([[s.start or 0, s.stop if s.stop is not None else -1]
                                           for s in patch.inner])  # fmt: skip
            out[f"p{q}_values"] = f.values
            out[f"p{q}_fx"] = f.fx
            out[f"p{q}_fy"] = f.fy
        out["patches"] = np.array(len(patches))
        np.savez_compressed(HERE / f"refinement_{name}.npz", **out)
        print("refinement", name, [p.box for p in patches])


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument(
        "--reference", default=os.environ.get("BEAMTRACER_REFERENCE"),
        help="the reference checkout (default: $BEAMTRACER_REFERENCE)",
    )  # fmt: skip
    parser.add_argument("--only", choices=["trace3d", "refinement"], default=None,
                        help="generate only the 3D fixtures (tracer, mesh, edge fields) or "
                             "the refined patches' fixtures")
    args = parser.parse_args()
    given = args.reference
    if not given:
        parser.error("give --reference or set BEAMTRACER_REFERENCE to the reference checkout")
    root = Path(given)
    if not (root / "src" / "beamtracer").is_dir():
        parser.error(f"{root} holds no src/beamtracer package")
    if args.only == "refinement":
        refinement_goldens(root)
        return
    trace3d_goldens(root)
    mesh3d_goldens(root)
    if args.only == "trace3d":
        return
    refinement_goldens(root)
    host_goldens(root)
    record_goldens(root)
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
        surface = reference_surface_field(root)
        magnitude, electrode = surface(mesh, types.SimpleNamespace(fx=fx, fy=fy))
        np.savez_compressed(HERE / f"surface_{name}.npz", magnitude=magnitude,
                            electrode=electrode)  # fmt: skip
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
