"""Seeded inputs of the kernel-level parity cases (shared by the fixture script and tests).

The trace cases exercise every branch of ``trace_trajectories_2d``: the three geometries
(planar, cylindrical, planar with a symmetry plane), both integrators (RK4, Boris), a
refined patch, a graded x axis, relativistic proper velocities, plane crossings beyond the
hit buffer, kept paths beyond their buffer, and electrode sub-cells that stop a trajectory
(status 3) or pause it (status -2).  They are modelled on the case list of the reference's
kernel tests (``tests/unit/test_compiled_tracer.py:253-347`` and
``tests/unit/test_kernels.py:26-40``), drawn from this file's own generator.
"""

from __future__ import annotations

import numpy as np

#: The scaled 1 / c^2 of the relativistic cases: c = 500 km/s, so trajectories at about
#: 300 km/s have a Lorentz factor near 1.2.
INV_C2 = 1.0 / 5.0e5**2

#: Positions of the outputs in the trace kernel's argument list.
TRACE_OUTPUTS = {
    "x": 1, "v": 2, "steps": 5, "status": 6, "electrode": 7, "hits": 25,
    "counts": 26, "paths": 28, "path_count": 29,
}  # fmt: skip
TRACE_CHARGE = 31
TRACE_NAMES = (
    "active x v qm dq steps status electrode fxs fys patch_int patch_real origin_x "
    "origin_y h upper_x upper_y cylindrical integrator step_fraction max_steps cells "
    "subcells refine planes hits counts path_slot paths path_count num_threads charge "
    "graded x_nodes inv_c2"
).split()


def gather_case(seed: int, n: int = 257, nx: int = 9, ny: int = 7, h: float = 0.1):
    """Edge fields and points inside, on and beyond a small mesh."""
    rng = np.random.default_rng(seed)
    fx = rng.normal(size=(nx + 1, ny))
    fy = rng.normal(size=(nx, ny + 1))
    origin = (rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05))
    px = origin[0] + h * rng.uniform(-3.0, nx + 2.0, n)
    py = origin[1] + h * rng.uniform(-3.0, ny + 2.0, n)
    return [px, py, fx, fy, origin[0], origin[1], h, np.zeros(n), np.zeros(n)]


def deposit_case(seed: int, cylindrical: int, n: int = 257, nx: int = 9, ny: int = 7):
    """Charges at points inside and beyond a small mesh (radii >= 0 when cylindrical)."""
    rng = np.random.default_rng(seed)
    h = 0.1
    origin = (rng.uniform(-0.05, 0.05), 0.0 if cylindrical else rng.uniform(-0.05, 0.05))
    px = origin[0] + h * rng.uniform(-2.0, nx + 1.0, n)
    low = 0.0 if cylindrical else -2.0
    py = origin[1] + h * rng.uniform(low, ny + 1.0, n)
    q = rng.normal(size=n)
    return [px, py, q, origin[0], origin[1], h, cylindrical, np.zeros((nx, ny))]


def trace_case(
    cylindrical: int,
    integrator: int,
    refined: bool = False,
    graded: bool = False,
    relativistic: bool = False,
    seed: int = 11,
    n: int = 48,
    max_steps: int = 500,
) -> list:
    """The 35 positional arguments of ``trace_trajectories_2d`` for one branch combination."""
    rng = np.random.default_rng(seed + 100 * cylindrical + 10 * integrator)
    nx, ny, h = 32, 13, 1.0e-3
    patches = [(nx, ny, 0.0, 0.0, h)]
    if refined:
        # a box of half the spacing, finest first
        patches.insert(0, (23, 15, 9.0e-3, 0.0, 0.5 * h))
    fxs, fys, patch_int, patch_real = [], [], [], []
    fx_off = fy_off = node_off = 0
    for pnx, pny, ox, oy, ph in patches:
        fxs.append((3.0e5 + 1.5e4 * rng.normal(size=(pnx + 1, pny))).ravel())
        fys.append((1.5e4 * rng.normal(size=(pnx, pny + 1))).ravel())
        patch_int.append((pnx, pny, fx_off, fy_off, pnx * pny, node_off))
        patch_real.append(
            (ox, oy, ph, ox, oy, ox + (pnx - 1) * ph, oy + (pny - 1) * ph)
        )
        fx_off += fxs[-1].size
        fy_off += fys[-1].size
        node_off += pnx * pny
    if graded:
        s = np.linspace(0.0, 1.0, nx)
        x_nodes = (nx - 1) * h * (0.4 * s + 0.6 * s * s)
    else:
        x_nodes = np.zeros(2)
    x = np.stack(
        [rng.uniform(0.0, 4.0e-3, n), rng.uniform(0.2e-3, 10.0e-3, n), np.zeros(n)]
    )
    v = np.stack(
        [
            np.full(n, 3.0e5) + 2.0e4 * rng.normal(size=n),
            3.0e4 * rng.normal(size=n),
            3.0e4 * rng.normal(size=n) * (cylindrical == 1),
        ]
    )
    if cylindrical == 2:
        # near the symmetry plane and heading across it
        x[1] *= 0.3
        v[1] = -2.5 * np.abs(v[1])
    x[:, 0] = (-1.0e-3, 1.0e-3, 0.0)  # one starts behind the mesh: backward at once
    cells = np.full((nx - 1, ny - 1), -1, dtype=np.int64)
    cells[21, 2:10] = np.arange(8)
    cells[26, 3:9] = np.arange(8, 14)
    refine = 8
    subcells = rng.choice(
        np.array([-2, -1, -1, -1, -1, -1, -1, 0, 1], dtype=np.int64), size=14 * refine**2
    )
    slot = np.full(n, -1, dtype=np.int64)
    slot[::3] = np.arange(len(slot[::3]))
    slots = int(slot.max()) + 1
    threads = 3
    return [
        np.arange(n, dtype=np.int64), x, v, np.full(n, 9.58e7), rng.uniform(0.5, 1.5, n),
        np.zeros(n, dtype=np.int64), np.full(n, -1, dtype=np.int64),
        np.full(n, -1, dtype=np.int64), np.concatenate(fxs), np.concatenate(fys),
        np.array(patch_int, dtype=np.int64), np.array(patch_real), 0.0, 0.0, h,
        (nx - 1) * h, (ny - 1) * h, cylindrical, integrator, 0.5, max_steps, cells, subcells,
        refine, np.array([6.0e-3, 17.5e-3]), np.zeros((n, 2, 3, 8)),
        np.zeros((n, 2), dtype=np.int64), slot, np.zeros((slots, 40, 2)),
        np.zeros(slots, dtype=np.int64), threads, np.zeros((threads, node_off)),
        int(graded), x_nodes, INV_C2 if relativistic else 0.0,
    ]  # fmt: skip


def trace_case_names() -> list[tuple[str, tuple]]:
    """Every branch combination, named ``trace_c{geometry}_i{integrator}_r_g_rel``."""
    out = []
    for cylindrical in (0, 1, 2):
        for integrator in (0, 1):
            for refined in (False, True):
                for graded in (False, True):
                    for relativistic in (False, True):
                        name = (
                            f"trace_c{cylindrical}_i{integrator}_r{int(refined)}"
                            f"_g{int(graded)}_rel{int(relativistic)}"
                        )
                        out.append(
                            (name, (cylindrical, integrator, refined, graded, relativistic))
                        )
    out.append(("trace_c0_i0_max_steps", (0, 0, False, False, False, 11, 48, 40)))
    out.append(("trace_c1_i1_max_steps", (1, 1, True, False, False, 12, 48, 55)))
    return out


def copy_args(args: list) -> list:
    """A deep copy of an argument list (arrays copied, scalars kept)."""
    return [a.copy() if isinstance(a, np.ndarray) else a for a in args]


# -- meshes -------------------------------------------------------------------------------


def _ring(x0: float, x1: float, r0: float, r1: float):
    """An electrode ``x0 <= x <= x1``, ``r0 <= y <= r1`` (a ring plate in (x, r))."""

    def inside(x, y):
        return (x >= x0) & (x <= x1) & (y >= r0) & (y <= r1)

    return inside


def _disc(cx: float, cy: float, radius: float):
    def inside(x, y):
        return (x - cx) ** 2 + (y - cy) ** 2 <= radius**2

    return inside


def mesh_cases() -> dict[str, dict]:
    """Mesh settings (IonOpticsMesh keyword arguments, electrodes as (inside, potential)),
    covering off-node surfaces on every side, overlapping electrodes, Dirichlet and Neumann
    faces, the axis and a graded x axis."""
    h = 1.0e-3
    s = np.linspace(0.0, 1.0, 41)
    return {
        "planar_plates": dict(
            shape=(31, 17), origin=(0.0, 0.0), h=h, geometry="planar",
            electrodes=[(_ring(10.37e-3, 13.61e-3, 5.23e-3, 16.0e-3), -500.0),
                        (_disc(22.4e-3, 6.1e-3, 3.33e-3), 250.0)],
            faces={"x_min": ("dirichlet", 0.0), "x_max": ("dirichlet", -1000.0)},
        ),
        "cylindrical_lens": dict(
            shape=(81, 21), origin=(0.0, 0.0), h=h, geometry="cylindrical",
            electrodes=[(_ring(19.3e-3, 21.3e-3, 5.05e-3, 20.0e-3), 0.0),
                        (_ring(39.4e-3, 41.4e-3, 5.55e-3, 20.0e-3), 7000.0),
                        (_ring(59.15e-3, 61.15e-3, 5.0e-3, 20.0e-3), 0.0),
                        (_disc(40.4e-3, 12.0e-3, 2.2e-3), 100.0)],
            faces={},
        ),
        "graded_disc": dict(
            shape=(41, 19), origin=(0.0, -9.0e-3), h=h, geometry="planar",
            x_nodes=40 * h * (0.3 * s + 0.7 * s * s),
            electrodes=[(_disc(20.2e-3, 0.3e-3, 4.1e-3), 1000.0)],
            faces={"x_min": ("dirichlet", 0.0), "y_min": ("dirichlet", 50.0)},
        ),
    }


# -- the 3D tracer --------------------------------------------------------------------------


def trace3d_case(
    integrator: int,
    refined: bool = False,
    mirror: bool = False,
    has_b: bool = False,
    has_j: bool = False,
    seed: int = 31,
    n: int = 32,
    max_steps: int = 300,
) -> list:
    """The 41 positional arguments of ``trace_trajectories_3d`` for one branch combination
    (non-relativistic: ``inv_c2`` 0)."""
    rng = np.random.default_rng(seed + 10 * integrator + 3 * int(refined) + 5 * int(mirror))
    nx, ny, nz, h = 20, 9, 9, 1.0e-3
    oy = oz = 0.0 if mirror else -4.0e-3
    patches = [(nx, ny, nz, 0.0, oy, oz, h)]
    if refined:
        # a box of half the spacing, finest first
        patches.insert(0, (15, 9, 9, 6.0e-3, oy + 2.0e-3, oz + 2.0e-3, 0.5 * h))
    fxs, fys, fzs, patch_int, patch_real = [], [], [], [], []
    ofx = ofy = ofz = ofn = 0
    for pnx, pny, pnz, px0, py0, pz0, ph in patches:
        fxs.append((3.0e5 + 1.5e4 * rng.normal(size=(pnx + 1, pny, pnz))).ravel())
        fys.append((1.5e4 * rng.normal(size=(pnx, pny + 1, pnz))).ravel())
        fzs.append((1.5e4 * rng.normal(size=(pnx, pny, pnz + 1))).ravel())
        patch_int.append((pnx, pny, pnz, ofx, ofy, ofz, pnx * pny * pnz, ofn))
        patch_real.append((px0, py0, pz0, ph, px0, py0, pz0, px0 + (pnx - 1) * ph,
                           py0 + (pny - 1) * ph, pz0 + (pnz - 1) * ph))  # fmt: skip
        ofx += fxs[-1].size
        ofy += fys[-1].size
        ofz += fzs[-1].size
        ofn += pnx * pny * pnz
    bn = 0.05 * rng.normal(size=(3, nx, ny, nz)) + np.array([0.2, 0.0, 0.0])[:, None, None, None]
    if not has_b:
        bn = np.zeros((3, 2, 2, 2))
    upper = (0.0 + (nx - 1) * h, oy + (ny - 1) * h, oz + (nz - 1) * h)
    lo = oy + (0.3e-3 if mirror else 1.0e-3)
    x = np.stack([rng.uniform(0.0, 3.0e-3, n), rng.uniform(lo, upper[1] - 1.0e-3, n),
                  rng.uniform(lo, upper[2] - 1.0e-3, n)])  # fmt: skip
    v = np.stack([np.full(n, 3.0e5) + 2.0e4 * rng.normal(size=n),
                  3.0e4 * rng.normal(size=n), 3.0e4 * rng.normal(size=n)])  # fmt: skip
    if mirror:
        # near the symmetry planes and heading across them
        x[1, : n // 2] = oy + 0.2e-3 * rng.uniform(size=n // 2)
        v[1, : n // 2] = -2.5 * np.abs(v[1, : n // 2])
        x[2, n // 2 :] = oz + 0.2e-3 * rng.uniform(size=n - n // 2)
        v[2, n // 2 :] = -2.5 * np.abs(v[2, n // 2 :])
    x[:, 0] = (-1.0e-3, 0.5 * (oy + upper[1]), 0.5 * (oz + upper[2]))  # backward at once
    cells = np.full((nx - 1, ny - 1, nz - 1), -1, dtype=np.int64)
    cells[12, 2:6, 3] = np.arange(4)
    cells[15, 3:7, 2:4] = np.arange(4, 12).reshape(4, 2)
    refine = 4
    subcells = rng.choice(np.array([-2, -1, -1, -1, -1, -1, 0, 1], dtype=np.int64),
                          size=12 * refine**3)  # fmt: skip
    slot = np.full(n, -1, dtype=np.int64)
    slot[::4] = np.arange(len(slot[::4]))
    slots = int(slot.max()) + 1
    threads = 2
    planes = np.array([5.5e-3, 14.25e-3])
    n_nodes = sum(p[0] * p[1] * p[2] for p in patches)
    nb = nx * ny * nz
    return [
        np.arange(n, dtype=np.int64), x, v,
        np.full(n, 9.58e7) * (1.0 + 0.1 * rng.uniform(size=n)),
        1.0e-6 * (1.0 + rng.uniform(size=n)),
        np.zeros(n, dtype=np.int64), np.full(n, -1, dtype=np.int64),
        np.full(n, -1, dtype=np.int64),
        np.concatenate(fxs), np.concatenate(fys), np.concatenate(fzs),
        np.array(patch_int, dtype=np.int64), np.array(patch_real, dtype=np.float64),
        bn, int(has_b), 0.0, oy, oz, h, upper[0], upper[1], upper[2], int(mirror), int(mirror),
        integrator, 0.5, max_steps, cells, subcells, refine, planes,
        np.zeros((n, len(planes), 4, 8)), np.zeros((n, len(planes)), dtype=np.int64),
        slot, np.zeros((slots, 64, 3)), np.zeros(slots, dtype=np.int64), threads,
        np.zeros((threads, n_nodes)), int(has_j),
        np.zeros((threads, 3 * nb)) if has_j else np.zeros((threads, 1)), 0.0,
    ]  # fmt: skip


def trace3d_case_names() -> list[tuple[str, tuple]]:
    """The 3D branch combinations, named ``trace3d_i{integrator}_r_m_b_j``."""
    out = []
    for integrator in (0, 1):
        for refined in (False, True):
            for mirror in (False, True):
                for has_b in (False, True):
                    has_j = refined != mirror
                    name = (f"trace3d_i{integrator}_r{int(refined)}_m{int(mirror)}"
                            f"_b{int(has_b)}_j{int(has_j)}")  # fmt: skip
                    out.append((name, (integrator, refined, mirror, has_b, has_j)))
    out.append(("trace3d_i0_max_steps", (0, False, False, True, False, 32, 32, 25)))
    return out


# -- the 3D mesh ------------------------------------------------------------------------------


def mesh3d_case() -> dict:
    """A 3D mesh with a plate with a round hole (0 V) and a sphere (1.5 kV), a Dirichlet
    face at x max (800 V) and a symmetry plane at y min: the settings both the reference's
    and this package's ``IonOpticsMesh3D`` take (the electrodes as ``(inside, potential)``,
    the faces as ``(kind, value)``)."""

    def plate(x, y, z):
        return (np.abs(x - 4.0e-3) <= 0.6e-3) & (y * y + (z - 2.5e-3) ** 2 >= (2.1e-3) ** 2)

    def sphere(x, y, z):
        return (x - 9.0e-3) ** 2 + (y - 3.0e-3) ** 2 + (z - 3.0e-3) ** 2 <= (1.3e-3) ** 2

    return {
        "shape": (25, 13, 11), "origin": (0.0, 0.0, 0.0), "h": 0.5e-3,
        "electrodes": [(plate, 0.0), (sphere, 1500.0)],
        "faces": {"x_max": ("dirichlet", 800.0), "y_min": ("neumann", 0.0)},
        "symmetry_planes": ("y_min",),
    }  # fmt: skip


# -- refined boxes ------------------------------------------------------------------------


def refinement_cases() -> dict[str, list[tuple[int, tuple[float, float], tuple[float, float]]]]:
    """Nested boxes ``(level, lower, upper)`` on the meshes of `mesh_cases`: around the
    plates' ring electrode, along the lens's axis with a finer box off the axis, and over
    the graded mesh's disc."""
    return {
        "planar_plates": [(1, (8e-3, 3e-3), (18e-3, 12e-3)), (2, (10e-3, 5e-3), (14e-3, 9e-3))],
        "cylindrical_lens": [(1, (15e-3, 0.0), (45e-3, 10e-3)), (2, (36e-3, 2e-3), (44e-3, 8e-3))],
        "graded_disc": [(1, (12e-3, -5e-3), (28e-3, 5e-3))],
    }


def refinement_potential(x, y):
    """A smooth potential [V] to take the patches' fields of."""
    x, y = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
    return 300.0 * np.sin(170.0 * x + 0.3) * np.cos(110.0 * y) + 2.0e4 * x * y
