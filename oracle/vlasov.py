"""ORACLE (test infrastructure): the Vlasov iteration on the CPU.

Restates ``solver/vlasov.py:247-429`` (the loop: solve, edge field, trace, compensate,
mix, repeat until the potential change is below the tolerance) and the host side of
``solver/tracer.py:1186-1304`` (``_trace_compiled``: trajectories starting in an electrode
end at once, paused ones are decided by the electrodes' inside test and resumed, full hit
buffers are grown and the trace repeated, the thread slabs summed) with the oracle's
kernels: the C trace (``oracle/bt_oracle.c``, OpenMP over trajectories), the NumPy edge
field and the SciPy LU field solve.  The node volumes are those of
``solver/refinement.py:274-296`` on an unrefined mesh.

Inputs are the classified mesh arrays and the electrode sub-cell tables (host setup,
checked against the reference's own outputs separately) and the beam.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np
from scipy import constants

from oracle import field as oracle_field
from oracle import kernels, poisson


@dataclass
class Problem:
    """What the iteration needs of a mesh, its electrodes and the trace settings."""

    shape: tuple[int, int]
    x: np.ndarray  # node positions along x
    h: float
    origin: tuple[float, float]
    logical_origin: tuple[float, float]
    logical_upper: tuple[float, float]
    geometry: int  # 0 planar, 1 cylindrical, 2 symmetry plane
    graded: bool
    fixed: np.ndarray
    fixed_value: np.ndarray
    solid: np.ndarray
    near_solid: np.ndarray
    distance: np.ndarray
    neumann: tuple[float, float, float, float]
    cells: np.ndarray
    subcells: np.ndarray
    inside_solid: Callable[[np.ndarray, np.ndarray], np.ndarray]
    planes: tuple[float, ...] = ()
    integrator: int = 0
    step_fraction: float = 0.5
    max_steps: int = 100_000
    inv_c2: float = 0.0
    threads: int = 0  # 0: every host core
    capacity: tuple[int, int] = (4, 1024)
    #: a magnetic field (mode, order, z0, hz, axis_y, samples) for the NumPy tracer's step
    magnetic: Any = None
    extra: dict = field(default_factory=dict)


def volumes(p: Problem) -> np.ndarray:
    nx, ny = p.shape
    cell = np.diff(p.x)[:, None] * np.full(ny - 1, p.h)[None, :]
    if p.geometry == 1:
        centres = p.origin[1] + p.h * (np.arange(ny - 1) + 0.5)
        cell = 2.0 * np.pi * centres[None, :] * cell
    out = np.zeros((nx, ny))
    for di in (0, 1):
        for dj in (0, 1):
            out[di : nx - 1 + di, dj : ny - 1 + dj] += 0.25 * cell
    return out


def _project(p: Problem, x: np.ndarray):
    if p.geometry == 1:
        return x[0], np.hypot(x[1], x[2])
    if p.geometry == 2:
        return x[0], p.origin[1] + np.abs(x[1] - p.origin[1])
    return x[0], x[1]


def _logical_x(p: Problem, x):
    if not p.graded:
        return x
    i = np.clip(np.searchsorted(p.x, x, side="right") - 1, 0, p.x.size - 2)
    return p.logical_origin[0] + p.h * (i + (x - p.x[i]) / (p.x[i + 1] - p.x[i]))


@dataclass
class Trace:
    charge: np.ndarray  # node charges (nx, ny)
    status: np.ndarray
    electrode: np.ndarray
    steps: np.ndarray
    hits: np.ndarray
    counts: np.ndarray


def trace(p: Problem, fx, fy, particles, patches=None) -> Trace:
    """One trace of ``particles`` (positions, velocities, charge, mass, current arrays).

    ``patches``: ``(patch_int, patch_real, nodes)`` of refined boxes (finest first, the base
    last; ``fx``, ``fy`` their edge fields flattened in that order); the charges are then
    the flat node charges of every patch."""
    nx, ny = p.shape
    n = particles.position.shape[1]
    x0 = np.array(particles.position, dtype=float, order="C")
    v0 = np.array(particles.velocity, dtype=float, order="C")
    if p.inv_c2 > 0.0:
        v0 = np.ascontiguousarray(v0 / np.sqrt(1.0 - np.sum(v0 * v0, axis=0) * p.inv_c2))
    qm = np.ascontiguousarray(particles.charge / particles.mass, dtype=float)
    dq = np.ascontiguousarray(np.sign(particles.charge) * np.abs(particles.current), dtype=float)
    status0 = np.full(n, -1, dtype=np.int64)
    electrode0 = np.full(n, -1, dtype=np.int64)
    hit = p.inside_solid(*_project(p, x0))
    dead = hit >= 0
    status0[dead] = 3
    electrode0[dead] = hit[dead]
    start = np.flatnonzero(status0 == -1).astype(np.int64)
    threads = p.threads or kernels.host_cores()
    threads = max(1, min(threads, max(start.size, 1)))
    planes = np.array(p.planes or (np.nan,), dtype=float)
    patch_int = np.array([[nx, ny, 0, 0, nx * ny, 0]], dtype=np.int64)
    patch_real = np.array([[*p.logical_origin, p.h, *p.logical_origin, *p.logical_upper]])
    nodes = nx * ny
    if patches is not None:
        patch_int, patch_real, nodes = patches
    x_nodes = np.ascontiguousarray(p.x if p.graded else np.zeros(2))
    fxs, fys = np.ascontiguousarray(fx).ravel(), np.ascontiguousarray(fy).ravel()
    while True:
        capacity, path_capacity = p.capacity
        x, v = x0.copy(), v0.copy()
        status, electrode = status0.copy(), electrode0.copy()
        steps = np.zeros(n, dtype=np.int64)
        charge = np.zeros((threads, nodes))
        hits = np.zeros((n, planes.size, capacity, 8))
        counts = np.zeros((n, planes.size), dtype=np.int64)
        slot = np.full(n, -1, dtype=np.int64)
        paths = np.zeros((1, path_capacity, 2))
        path_count = np.ones(1, dtype=np.int64)
        active = start
        while active.size:
            kernels.trace_trajectories_2d(
                active, x, v, qm, dq, steps, status, electrode, fxs, fys, patch_int,
                patch_real, *p.logical_origin, p.h, *p.logical_upper, p.geometry,
                p.integrator, p.step_fraction, p.max_steps, p.cells, p.subcells, 8, planes,
                hits, counts, slot, paths, path_count, threads, charge, int(p.graded),
                x_nodes, p.inv_c2, magnetic=p.magnetic,
            )  # fmt: skip
            paused = active[status[active] == -2]
            if not paused.size:
                break
            inside_hit = p.inside_solid(*_project(p, x[:, paused]))
            inside = inside_hit >= 0
            status[paused[inside]] = 3
            electrode[paused[inside]] = inside_hit[inside]
            active = paused[~inside]
            status[active] = -1
        most = int(counts.max()) if counts.size else 0
        if most <= capacity:
            break
        p.capacity = (max(capacity, most), path_capacity)
    total = charge.sum(axis=0)
    return Trace(total if patches is not None else total.reshape(nx, ny), status, electrode,
                 steps, hits, counts)  # fmt: skip


def plane_hits(p: Problem, t: Trace, current, species):
    """Per plane (point (3, m), velocity (3, m), current, species, direction), in the
    order of the steps then the trajectories (``tracer.py:1276-1293``)."""
    out = []
    slots = np.arange(t.hits.shape[2])
    for k_plane, _ in enumerate(p.planes):
        k, c = np.nonzero(slots[None, :] < t.counts[:, k_plane, None])
        record = t.hits[k, k_plane, c]
        order = np.lexsort((k, record[:, 7]))
        k, record = k[order], record[order]
        out.append((record[:, 0:3].T.copy(), record[:, 3:6].T.copy(), current[k], species[k],
                    record[:, 6].astype(np.int8)))  # fmt: skip
    return out


@dataclass
class Plasma:
    temperature: float
    potential: float
    initial_x: float
    sign: int  # -1 electrons, +1 ions
    density: float | None = None


def edge_faces(p: Problem) -> list[str]:
    """The edge field's face rules: extrapolated, mirrored on the axis or symmetry plane."""
    faces = ["extrapolate"] * 4
    if p.geometry in (1, 2):
        faces[2] = "symmetric"
    return faces


def density_of(p: Problem, potential: np.ndarray, particles) -> tuple[np.ndarray, Trace]:
    """G(phi): the beam's charge density (node charges over node volumes) when traced
    through the edge field of ``potential`` -- one iteration's stage after its field solve
    (``vlasov.py:368-397`` before compensation and mixing); and the trace."""
    fx, fy = oracle_field.edge_fields(potential, p.solid, p.near_solid, p.distance,
                                      np.diff(p.x), p.h, edge_faces(p))  # fmt: skip
    t = trace(p, fx, fy, particles)
    return t.charge / volumes(p), t


class Anderson:
    """Anderson mixing of type II (``vlasov.py:127-173``): from the last ``depth + 1``
    iterates x and residuals f = G(x) - x, gamma = argmin |f - dF gamma| by NumPy's
    least squares with singular values below 1e-10 of the largest cut off, and
    x + w f - (dX + w dF) gamma."""

    def __init__(self, depth: int, relaxation: float) -> None:
        self.depth, self.relaxation = int(depth), float(relaxation)
        self.xs: list[np.ndarray] = []
        self.fs: list[np.ndarray] = []

    def reset(self) -> None:
        self.xs, self.fs = [], []

    def update(self, rho: np.ndarray, deposit: np.ndarray) -> np.ndarray:
        x = np.asarray(rho, dtype=float).ravel()
        f = np.asarray(deposit, dtype=float).ravel() - x
        self.xs = (self.xs + [x])[-(self.depth + 1):]
        self.fs = (self.fs + [f])[-(self.depth + 1):]
        w = self.relaxation
        new = x + w * f
        if len(self.xs) > 1:
            dx = np.diff(np.array(self.xs), axis=0).T
            df = np.diff(np.array(self.fs), axis=0).T
            gamma = np.linalg.lstsq(df, f, rcond=1e-10)[0]
            new = new - (dx + w * df) @ gamma
        return new.reshape(np.shape(rho))


def thin(particles, stride: int):
    """Every ``stride``-th trajectory of each species, the kept currents scaled to keep the
    species' total (``vlasov.py:202-215``)."""
    from types import SimpleNamespace

    keep = np.zeros(particles.current.size, dtype=bool)
    scale = np.ones(particles.current.size)
    for s in np.unique(particles.species):
        members = np.flatnonzero(particles.species == s)
        kept = members[::stride]
        keep[kept] = True
        total, part = np.abs(particles.current[members]).sum(), np.abs(particles.current[kept]).sum()
        scale[kept] = total / part if part > 0.0 else 1.0
    return SimpleNamespace(position=particles.position[:, keep],
                           velocity=particles.velocity[:, keep],
                           charge=particles.charge[keep], mass=particles.mass[keep],
                           current=particles.current[keep] * scale[keep],
                           species=particles.species[keep])  # fmt: skip


def vlasov(p: Problem, particles, j_over_v: float, *, iterations: int, tolerance: float = 0.0,
           relaxation: float = 1.0, plasma: Plasma | None = None, compensation=(),
           density_tolerance: float | None = None, callback=None, mixing: str = "linear",
           anderson_depth: int = 5, coarse_particles: float = 1.0,
           coarse_tolerance: float = 0.0) -> dict[str, Any]:  # fmt: skip
    """The Vlasov iteration (``vlasov.py:327-427``: linear or Anderson mixing, the coarse
    phase of every k-th trajectory until the potential changes by less than
    ``coarse_tolerance``); the last iteration's potential, density, trace and history."""
    mixer = Anderson(anderson_depth, relaxation) if mixing == "anderson" else None
    stride = int(np.ceil(1.0 / coarse_particles - 1e-9))
    coarse = stride > 1
    nx, ny = p.shape
    op = poisson.assemble(p.x, p.h, p.geometry == 1, p.fixed, p.fixed_value, p.distance,
                          p.neumann)  # fmt: skip
    vol = volumes(p)
    factor = np.ones(nx)
    for x_min, x_max, fraction in compensation:
        factor[(p.x >= x_min) & (p.x <= x_max)] *= 1.0 - fraction
    faces = edge_faces(p)
    rho = np.zeros((nx, ny))
    potential = None
    history = []
    boltzmann = None
    out: dict[str, Any] = {}
    for iteration in range(iterations):
        if plasma is not None and iteration == 0:
            xn = np.broadcast_to(p.x[:, None], (nx, ny))
            region = (xn < plasma.initial_x) & ~np.asarray(p.fixed, bool)
            fixed = np.asarray(p.fixed, bool) | region
            value = np.where(region, plasma.potential, p.fixed_value)
            op0 = poisson.assemble(p.x, p.h, p.geometry == 1, fixed, value, p.distance, p.neumann)
            new = poisson.solve(op0, rho)
        elif plasma is not None:
            if boltzmann is None:
                density = plasma.density if plasma.density is not None else j_over_v
                boltzmann = density / constants.epsilon_0
            new, _ = poisson.solve_newton(op, rho, boltzmann, plasma.temperature,
                                          plasma.potential, plasma.sign, initial=potential,
                                          tol=1e-11)  # fmt: skip
        else:
            new = poisson.solve(op, rho)
        change = float("inf") if potential is None else float(np.max(np.abs(new - potential)))
        potential = new
        fx, fy = oracle_field.edge_fields(potential, p.solid, p.near_solid, p.distance,
                                          np.diff(p.x), p.h, faces)  # fmt: skip
        if coarse and change < coarse_tolerance:
            coarse = False
            if mixer is not None:
                mixer.reset()
        t = trace(p, fx, fy, thin(particles, stride) if coarse else particles)
        deposit = t.charge / vol * factor[:, None]
        old = rho
        if iteration == 0:
            rho = deposit
        elif mixer is not None:
            rho = mixer.update(rho, deposit)
        else:
            rho = (1.0 - relaxation) * rho + relaxation * deposit
        scale = np.max(np.abs(rho))
        density_change = float(np.max(np.abs(rho - old)) / scale) if scale > 0 else 0.0
        history.append({"iteration": iteration, "max_potential_change": change,
                        "relative_density_change": density_change if iteration else float("inf"),
                        "steps": int(t.steps.max()) if t.steps.size else 0})  # fmt: skip
        out = {"potential": potential, "charge_density": rho, "deposit": deposit, "trace": t,
               "history": history, "fields": (fx, fy)}  # fmt: skip
        if callback is not None:
            callback(iteration, out)
        if coarse:
            continue
        if change < tolerance:
            break
        if density_tolerance is not None and iteration > 0 and density_change < density_tolerance:
            break
    return out
