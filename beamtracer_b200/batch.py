"""Batched design sweeps: many candidate lenses converged together on one GPU.

The reference's design search solves its candidates one at a time, each a whole
`BeamOptics(config).run()` (``optimization/einzel.py:389-403``, ``EinzelLens.problem``).
Each of those solves leaves a B200 mostly idle: one candidate's trace is a few thousand
trajectories (one warp per scheduler), its field solve a chain of small launches.  Here the
candidates are laid end to end in device memory and every stage of a Vlasov iteration
covers all of them at once:

- the trace: one window launch advances every candidate's live trajectories
  (``bt_trace_trajectories_2d_batch``: each trajectory reads its candidate's mesh from a
  table), and one deposit sorts and reduces the records of all of them by their
  concatenated node keys;
- the field solve: one multigrid V-cycle over all candidates' levels per level and
  colour, the coarse levels in one block per candidate (``bt_poisson_batch_*``), iterated
  until each candidate's residual meets the single solve's criterion;
- the edge fields, the mixing and the convergence tests: one launch each over the
  candidates' concatenated nodes.

A candidate leaves the batch after the iteration in which it converges, as its own solve
would stop there; its moments are taken from that iteration's trace.

Layout in HBM (all FP64 unless said): candidate c's nodes at ``[node0[c], node0[c] +
nx ny)`` of the potential, density and charge; its edge fields at ``fx0[c]``, ``fy0[c]``
of the concatenated ``(nx + 1) ny`` and ``nx (ny + 1)`` arrays; its trajectories at
``[traj0[c], traj0[c] + n)`` of the state arrays ((3, N) positions and velocities).
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from beamtracer_b200 import _lib
from beamtracer_b200.config import BeamOpticsConfig
from beamtracer_b200.diagnostics import BeamMoments, plane_moments
from beamtracer_b200.fields import MeshArrays, StaggeredElectricField
from beamtracer_b200.mesh import IonOpticsMesh
from beamtracer_b200.poisson import IonOpticsPoisson
from beamtracer_b200.tracer import (
    _ALIVE,
    _PAUSED,
    ELECTRODE,
    INTEGRATORS,
    SUBCELLS,
    PlaneHits,
    TraceEngine,
    _project,
    geometry_code,
)


@dataclass
class Candidate:
    """One candidate of a batch: its configuration, mesh, solver and place in the batch."""

    config: BeamOpticsConfig
    mesh: IonOpticsMesh
    poisson: IonOpticsPoisson
    arrays: MeshArrays
    engine: TraceEngine
    mass: np.ndarray
    node0: int = 0
    fx0: int = 0
    fy0: int = 0
    traj0: int = 0
    n_traj: int = 0
    #: the Vlasov iterations run, their largest potential changes; set when it leaves
    history: list[dict[str, float]] = field(default_factory=list)
    done: bool = False
    converged: bool = False
    planes: list[PlaneHits] | None = None

    @property
    def shape(self) -> tuple[int, int]:
        return self.mesh.shape

    @property
    def n_nodes(self) -> int:
        nx, ny = self.mesh.shape
        return nx * ny

    def moments(self, x: float, species: int | None = None, axis: str = "y") -> BeamMoments:
        """The current, emittance and Twiss parameters at the plane ``x`` (as
        `BeamOptics.beam_moments`)."""
        if self.planes is None:
            raise RuntimeError("the candidate has not finished")
        match = [hits for hits in self.planes if np.isclose(hits.position_x, x)]
        if not match:
            raise KeyError(f"no diagnostic plane at x = {x}")
        return plane_moments(match[0], cylindrical=self.mesh.cylindrical, mass=self.mass,
                             species=species, axis=axis)  # fmt: skip


def _supported(config: BeamOpticsConfig) -> None:
    """Refuse what the batched loop does not do (each of these runs through `BeamOptics`)."""
    refused = {
        "a plasma": config.plasma is not None,
        "magnetic fields": bool(config.solenoids) or config.axial_field is not None,
        "compensation": bool(config.compensation),
        "Anderson mixing": config.mixing != "linear",
        "a coarse-particle phase": config.coarse_particles < 1.0,
        "relativity": bool(config.relativistic),
    }
    given = [name for name, on in refused.items() if on]
    if given:
        raise NotImplementedError("a batched sweep takes no " + ", ".join(given))


class BatchedVlasov:
    """The Vlasov iterations of many configurations run together (see the module).

    Every configuration must share the diagnostic planes, the integrator, the step fraction,
    the step limit, the iteration limit, the tolerance and the relaxation; meshes, electrodes
    and beams may differ.  ``window``: trace steps per launch; ``contracted``: the trace
    build with fused multiply-adds (moments agree with the exact build to rounding);
    ``builders``: host threads that set the candidates up.
    """

    def __init__(self, configs: Sequence[BeamOpticsConfig], *, window: int = 64,
                 contracted: bool = False, capacity: tuple[int, int] = (4, 1024),
                 field: str = "batched", builders: int = 6) -> None:  # fmt: skip
        import torch

        from beamtracer_b200.model import config_mesh, config_particles

        if not configs:
            raise ValueError("a batch needs at least one configuration")
        first = configs[0]
        shared = ("diagnostic_planes", "integrator", "step_fraction", "max_steps",
                  "iterations", "tolerance", "relaxation")  # fmt: skip
        for config in configs:
            if type(config) is not BeamOpticsConfig:
                raise TypeError(f"a batch takes BeamOpticsConfig, got {type(config).__name__}")
            _supported(config)
            for name in shared:
                if getattr(config, name) != getattr(first, name):
                    raise ValueError(f"every configuration of a batch needs the same {name}")
        if field not in ("batched", "single"):
            raise ValueError(f"field must be 'batched' or 'single', got {field!r}")
        self.field = field
        self.torch = torch
        self.window = int(window)
        self.contracted = bool(contracted)
        self.planes = tuple(float(p) for p in first.diagnostic_planes)
        self.iterations = int(first.iterations)
        self.tolerance = float(first.tolerance)
        self.relaxation = float(first.relaxation)
        self.ctx = _lib.context()
        dev = "cuda"
        self.candidates: list[Candidate] = []
        node = fx = fy = traj = 0
        device = torch.cuda.current_device()
        #: the library contexts of the threads that built candidates (their solvers are
        #: bound to them: kept for the batch's life)
        self._builder_contexts: list[Any] = []

        def build(config: BeamOpticsConfig) -> Candidate:
            torch.cuda.set_device(device)
            mesh = config_mesh(config)
            if mesh.graded:
                raise NotImplementedError("a batch takes uniform meshes")
            particles, _ = config_particles(config)
            engine = TraceEngine(mesh, planes=self.planes, integrator=config.integrator,
                                 step_fraction=config.step_fraction, max_steps=config.max_steps,
                                 capacity=capacity, window=self.window)  # fmt: skip
            engine.load(particles, buffers=False)
            mass = np.array([beam.mass for beam in config.beams]) * _atomic_mass()
            cand = Candidate(config, mesh, IonOpticsPoisson(mesh), MeshArrays(mesh), engine, mass)
            cand.n_traj = len(particles)
            torch.cuda.current_stream().synchronize()
            return cand, _lib.context()

        if builders > 1 and len(configs) > 1:
            # the candidates' host work (meshes, tables, beams) on several threads; each
            # thread's device work queues on its own context
            from concurrent.futures import ThreadPoolExecutor

            with ThreadPoolExecutor(max_workers=min(builders, len(configs))) as pool:
                built = list(pool.map(build, configs))
        else:
            built = [build(config) for config in configs]
        contexts = {id(c): c for _, c in built}
        self._builder_contexts = list(contexts.values())
        cylindrical = None
        for cand, _ in built:
            mesh = cand.mesh
            if cylindrical is None:
                cylindrical = (mesh.cylindrical, mesh.symmetry_plane)
            elif cylindrical != (mesh.cylindrical, mesh.symmetry_plane):
                raise ValueError("every configuration of a batch needs the same geometry")
            nx, ny = mesh.shape
            cand.node0, cand.fx0, cand.fy0, cand.traj0 = node, fx, fy, traj
            node += nx * ny
            fx += (nx + 1) * ny
            fy += nx * (ny + 1)
            traj += cand.n_traj
            self.candidates.append(cand)
        self.n_nodes, self.n_traj = node, traj
        first_engine = self.candidates[0].engine
        self.integrator = INTEGRATORS.index(first_engine.integrator)
        self.step_fraction = first_engine.step_fraction
        self.max_steps = first_engine.max_steps
        self.geometry = geometry_code(self.candidates[0].mesh)
        # the concatenated state
        f64 = dict(dtype=torch.float64, device=dev)
        self.phi = torch.zeros(node, **f64)
        self.rho = torch.zeros(node, **f64)
        self.previous = torch.zeros(node, **f64)
        self.fx = torch.zeros(fx, **f64)
        self.fy = torch.zeros(fy, **f64)
        self.charge = torch.zeros((1, node), **f64)
        cands = self.candidates
        self.volumes = torch.cat([c.engine.volumes.reshape(-1) for c in cands])
        self.x0 = torch.cat([c.engine.x0 for c in cands], dim=1).contiguous()
        self.v0 = torch.cat([c.engine.v0 for c in cands], dim=1).contiguous()
        self.status0 = torch.cat([c.engine.status0 for c in cands])
        self.electrode0 = torch.cat([c.engine.electrode0 for c in cands])
        self.qm = torch.cat([c.engine.qm for c in cands])
        self.dq = torch.cat([c.engine.dq for c in cands])
        self.start_active = [c.engine.start_active + c.traj0 for c in cands]
        self.candidate_of = np.concatenate(
            [np.full(c.n_traj, k, dtype=np.int32) for k, c in enumerate(cands)])
        self.candidate_dev = torch.from_numpy(self.candidate_of).to(dev)
        self.x = torch.empty_like(self.x0)
        self.v = torch.empty_like(self.v0)
        self.steps = torch.zeros(traj, dtype=torch.int64, device=dev)
        self.status = torch.empty_like(self.status0)
        self.electrode = torch.empty_like(self.electrode0)
        # the candidates' meshes as one-patch rows, their cell tables end to end (the
        # sub-cell block numbers shifted past the blocks of the candidates before)
        rows_int, rows_real, cells, subcells, cell_offset = [], [], [], [], []
        blocks = cell0 = 0
        block = SUBCELLS * SUBCELLS
        for c in cands:
            nx, ny = c.mesh.shape
            lo_x, lo_y = c.mesh.logical_origin
            up_x, up_y = c.mesh.logical_upper
            rows_int.append([nx, ny, c.fx0, c.fy0, nx * ny, c.node0])
            rows_real.append([lo_x, lo_y, c.mesh.h, lo_x, lo_y, up_x, up_y])
            table = c.engine.cells.reshape(-1)
            used = int(table.max().item()) + 1 if table.numel() else 0
            cells.append(torch.where(table >= 0, table + blocks, table))
            subcells.append(c.engine.subcells.reshape(-1)[: used * block])
            cell_offset.append(cell0)
            blocks += used
            cell0 += (nx - 1) * (ny - 1)
        self.patch_int = torch.tensor(rows_int, dtype=torch.int64, device=dev)
        self.patch_real = torch.tensor(rows_real, dtype=torch.float64, device=dev)
        self.cells = torch.cat(cells)
        self.subcells = torch.cat(subcells) if blocks else torch.full((1,), -1, dtype=torch.int64,
                                                                     device=dev)  # fmt: skip
        self.cell_offset = torch.tensor(cell_offset, dtype=torch.int64, device=dev)
        # the candidates' electrode shapes end to end, for the trace's own electrode test
        # (None when one candidate's electrodes are not configuration shapes: its paused
        # trajectories are tested here, on the host)
        self.shapes = self._shape_tables()
        self.planes_dev = torch.tensor(self.planes or (np.nan,), dtype=torch.float64, device=dev)
        self.capacity = tuple(capacity)
        self._allocate_hits()
        self.path_slot = torch.full((traj,), -1, dtype=torch.int64, device=dev)
        self.paths = torch.zeros((1, 1, 2), **f64)
        self.path_count = torch.ones(1, dtype=torch.int64, device=dev)
        self.x_nodes = torch.zeros(2, **f64)
        # per candidate: max |phi - previous|, max |rho_new - rho_old|, max |rho_new|
        self.scalars = torch.zeros((len(cands), 4), **f64)
        self.trace_launches = 0
        for c in cands:
            c.poisson.rebind(self.ctx)  # built on other threads' contexts
        self.poisson_batch = PoissonBatch([c.poisson for c in cands], [c.node0 for c in cands])

    def _shape_tables(self):
        torch = self.torch
        from beamtracer_b200.shapes import shape_table

        kinds, offsets, params, first = [], [], [], [0]
        for c in self.candidates:
            table = shape_table(c.mesh) if c.mesh.electrodes else (
                np.zeros(0, np.int32), np.zeros(0, np.int64), np.zeros(0))  # fmt: skip
            if table is None:
                return None
            kind, offset, param = table
            kinds.append(kind)
            offsets.append(offset + sum(p.size for p in params))
            params.append(param)
            first.append(first[-1] + kind.size)
        if first[-1] == 0:
            return None  # no electrodes: nothing to test
        dev = "cuda"
        return (torch.from_numpy(np.array(first, dtype=np.int64)).to(dev),
                torch.from_numpy(np.concatenate(kinds).astype(np.int32)).to(dev),
                torch.from_numpy(np.concatenate(offsets).astype(np.int64)).to(dev),
                torch.from_numpy(np.concatenate(params).astype(np.float64)).to(dev))  # fmt: skip

    # -- the trace ---------------------------------------------------------------------

    def _allocate_hits(self) -> None:
        torch = self.torch
        capacity, _ = self.capacity
        P = len(self.planes_dev)
        self.hits = torch.zeros((self.n_traj, P, capacity, 8), dtype=torch.float64, device="cuda")
        self.counts = torch.zeros((self.n_traj, P), dtype=torch.int64, device="cuda")

    def _reset(self) -> None:
        # every trajectory back to its start (a finished candidate's crossings were taken
        # when it finished)
        self.x.copy_(self.x0)
        self.v.copy_(self.v0)
        self.status.copy_(self.status0)
        self.electrode.copy_(self.electrode0)
        self.steps.zero_()
        self.counts.zero_()
        self.charge.zero_()

    def _trace_call(self, active) -> None:
        d = _lib.dptr
        a = _lib.TraceArgs(
            d(active), int(active.numel()), d(self.x), d(self.v), self.n_traj, d(self.qm),
            d(self.dq), d(self.steps), d(self.status), d(self.electrode), d(self.fx),
            d(self.fy), d(self.patch_int), d(self.patch_real), len(self.candidates), 0.0, 0.0,
            0.0, 0.0, 0.0, self.geometry, self.integrator, self.step_fraction, self.max_steps,
            d(self.cells), d(self.subcells), SUBCELLS, d(self.planes_dev),
            int(self.planes_dev.numel()), d(self.hits), int(self.hits.shape[2]), d(self.counts),
            d(self.path_slot), d(self.paths), 1, d(self.path_count), 1, d(self.charge),
            self.n_nodes, 0, d(self.x_nodes), 2, 0.0,
        )  # fmt: skip
        shapes = (d(t) for t in self.shapes) if self.shapes is not None else (None,) * 4
        b = _lib.TraceBatch(len(self.candidates), d(self.candidate_dev), d(self.cell_offset), 0,
                            *shapes)  # fmt: skip
        lib = _lib.lib()
        entry = lib.bt_trace_trajectories_2d_batch_fast if self.contracted else lib.bt_trace_trajectories_2d_batch
        _lib.check(entry(self.ctx.handle, ctypes.byref(a), ctypes.byref(b), self.window))
        self.trace_launches += 1

    def trace(self, members: Sequence[int]) -> None:
        """Trace the beams of the candidates ``members`` through the edge fields in
        ``fx``, ``fy``; their node charges land in ``charge``, their ends and plane
        crossings in the state arrays."""
        torch = self.torch
        while True:
            self._reset()
            active = torch.cat([self.start_active[k] for k in members])
            while active.numel():
                self._trace_call(active)
                paused_mask = self.status[active] == _PAUSED
                flags = torch.stack([paused_mask.sum(), self.counts.max()]).cpu().tolist()
                most = flags[1]
                if flags[0] == 0:
                    break
                # the exact inside tests of the trajectories that stopped in a cell an
                # electrode surface cuts, each against its own candidate's electrodes
                paused = active[paused_mask]
                ids = paused.cpu().numpy()
                points = self.x[:, paused].cpu().numpy()
                hit = np.full(ids.size, -1, dtype=np.int64)
                owner = self.candidate_of[ids]
                for k in np.unique(owner):
                    sel = owner == k
                    mesh = self.candidates[int(k)].mesh
                    hit[sel] = mesh.inside_solid(*_project(mesh, points[:, sel]))
                inside = torch.from_numpy(hit >= 0).to("cuda")
                hit_dev = torch.from_numpy(hit).to("cuda")
                stopped = paused[inside]
                self.status[stopped] = ELECTRODE
                self.electrode[stopped] = hit_dev[inside]
                active = paused[~inside]
                self.status[active] = _ALIVE
            else:
                most = int(self.counts.max())
            capacity, paths = self.capacity
            if most <= capacity:
                return
            self.capacity = (max(capacity, most), paths)
            self._allocate_hits()

    def plane_hits(self, k: int) -> list[PlaneHits]:
        """Candidate k's crossings of every plane, as its own trace returns them: ordered by
        step, then trajectory (`TraceEngine.result`)."""
        torch = self.torch
        c = self.candidates[k]
        t = slice(c.traj0, c.traj0 + c.n_traj)
        hits, counts = self.hits[t], self.counts[t]
        particles = c.engine.particles
        current = particles.current.astype(float)
        species = particles.species
        slots = torch.arange(hits.shape[2], device=hits.device)
        out = []
        for p, position in enumerate(self.planes):
            j, s = (slots[None, :] < counts[:, p, None]).nonzero(as_tuple=True)
            record = hits[j, p, s]
            order = torch.sort(record[:, 7], stable=True).indices
            record = torch.cat([record[order], j[order, None].to(torch.float64)], dim=1)
            record = record.cpu().numpy()
            j = record[:, 8].astype(np.int64)
            plane = PlaneHits(position)
            plane.append(record[:, 0:3].T.copy(), record[:, 3:6].T.copy(), current[j],
                         species[j], record[:, 6].astype(np.int8))  # fmt: skip
            out.append(plane)
        return out

    # -- the iteration -------------------------------------------------------------------

    def run(self) -> BatchedVlasov:
        """Iterate every candidate to convergence (``vlasov.py:327-427`` for each: solve
        the field, trace, deposit, mix linearly; stop when the potential changes by less
        than the tolerance) or to the iteration limit."""
        lib, ctx, d = _lib.lib(), self.ctx, _lib.dptr
        cands = self.candidates
        for iteration in range(self.iterations):
            members = [k for k, c in enumerate(cands) if not c.done]
            if not members:
                break
            self.previous.copy_(self.phi)
            self.solve_fields(members)
            for k in members:
                c = cands[k]
                phi, prev = self.node_view(self.phi, k), self.node_view(self.previous, k)
                _lib.check(lib.bt_max_abs_diff(ctx.handle, d(phi), d(prev), c.n_nodes,
                                               d(self.scalars[k])))  # fmt: skip
                StaggeredElectricField(c.mesh, phi, arrays=c.arrays, out=self.edge_views(k))
            self.trace(members)
            for k in members:
                c = cands[k]
                nx, ny = c.shape
                charge = self.charge[0, c.node0 : c.node0 + c.n_nodes]
                volumes = self.volumes[c.node0 : c.node0 + c.n_nodes]
                _lib.check(lib.bt_vlasov_mix(
                    ctx.handle, d(charge), d(volumes), None, nx, ny, self.relaxation,
                    int(iteration == 0), d(self.node_view(self.rho, k)),
                    d(self.scalars[k]) + 8))  # fmt: skip
            host = self.scalars.cpu().numpy()
            for k in members:
                c = cands[k]
                change = float(host[k, 0]) if iteration > 0 else float("inf")
                c.history.append({"iteration": iteration, "max_potential_change": change})
                if change < self.tolerance or iteration == self.iterations - 1:
                    c.done = True
                    c.converged = change < self.tolerance
                    c.planes = self.plane_hits(k)
        return self

    def solve_fields(self, members: Sequence[int]) -> None:
        """The potential of every member candidate from its density, each from its last
        potential: one batched multigrid iteration over all of them
        (``bt_poisson_batch_solve``), or one candidate at a time (``field="single"``)."""
        if self.field == "single":
            for k in members:
                c = self.candidates[k]
                c.poisson.solve_device(self.node_view(self.phi, k), self.node_view(self.rho, k))
            return
        self.poisson_batch.solve(self.phi, self.rho, members)

    def close(self) -> None:
        """Release the batched field solver (the candidates' own solvers stay usable)."""
        self.poisson_batch.close()

    # -- views ---------------------------------------------------------------------------

    def node_view(self, array, k: int):
        c = self.candidates[k]
        return array[c.node0 : c.node0 + c.n_nodes].view(c.shape)

    def edge_views(self, k: int):
        c = self.candidates[k]
        nx, ny = c.shape
        fx = self.fx[c.fx0 : c.fx0 + (nx + 1) * ny].view(nx + 1, ny)
        fy = self.fy[c.fy0 : c.fy0 + nx * (ny + 1)].view(nx, ny + 1)
        return fx, fy


class PoissonBatch:
    """The field solves of many candidates' solvers at once (``bt_poisson_batch_*``):
    candidate k's nodes at ``offsets[k]`` of the concatenated potential and density."""

    def __init__(self, solvers: Sequence[IonOpticsPoisson], offsets: Sequence[int]) -> None:
        self.solvers = list(solvers)  # kept alive: the batch reads their hierarchies
        self.count = len(self.solvers)
        handles = (_lib.P * self.count)(*[s._handle.value for s in self.solvers])
        self._offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        handle = _lib.P()
        ctx = _lib.context()
        _lib.check(_lib.lib().bt_poisson_batch_create(
            ctx.handle, ctypes.cast(handles, _lib.P), self.count, self._offsets.ctypes.data,
            ctypes.byref(handle)))  # fmt: skip
        self._handle = handle
        self.cycles = np.zeros(self.count, dtype=np.int32)
        self.residual = np.zeros(self.count)

    def solve(self, phi, rho, members: Sequence[int], tolerance: float = 1e-13,
              max_cycles: int = 400) -> None:  # fmt: skip
        """Solve the members' fields in place on the concatenated device arrays."""
        flags = np.zeros(self.count, dtype=np.uint8)
        flags[list(members)] = 1
        d = _lib.dptr
        _lib.check(_lib.lib().bt_poisson_batch_solve(
            self._handle, d(phi), d(rho), flags.ctypes.data, float(tolerance), int(max_cycles),
            self.cycles.ctypes.data, self.residual.ctypes.data))  # fmt: skip

    @property
    def tiling(self) -> dict:
        """The V-cycle's smoothing tiles (chosen by timing at the first solve)."""
        t = np.zeros(6, dtype=np.int32)
        _lib.check(_lib.lib().bt_poisson_batch_tiling(self._handle, 0, t.ctypes.data))
        return {"level0": (int(t[0]), int(t[1])), "nine_point": (int(t[2]), int(t[3])),
                "nine_point_launches": int(t[4]), "tuned": bool(t[5])}  # fmt: skip

    def set_tiling(self, level0=(32, 32), nine_point=(16, 32), launches: int = 1) -> None:
        """Fix the smoothing tiles (no tuning)."""
        t = np.array([*level0, *nine_point, launches, 1], dtype=np.int32)
        _lib.check(_lib.lib().bt_poisson_batch_tiling(self._handle, 1, t.ctypes.data))

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None and self._handle.value:
            _lib.lib().bt_poisson_batch_destroy(self._handle)
            self._handle = None

    def __del__(self) -> None:  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def _atomic_mass() -> float:
    from scipy import constants

    return constants.atomic_mass


def batched_sweep(designs, rank: int = 0, world: int = 1, plane: float = 79e-3,
                  **settings) -> dict[int, dict]:  # fmt: skip
    """This rank's share of the einzel candidates ``designs`` (`einzel.share_of_designs`)
    converged together in one `BatchedVlasov`: ``{candidate index: result}`` with the
    result of `einzel.evaluate_design` (moments at ``plane``, iterations, convergence)."""
    from beamtracer_b200.einzel import einzel_config, share_of_designs

    mine = share_of_designs(designs, rank, world)
    if not mine:
        return {}
    batch = BatchedVlasov([einzel_config(designs[k], **settings) for k in mine]).run()
    out = {}
    for j, k in enumerate(mine):
        c = batch.candidates[j]
        m = c.moments(plane)
        out[k] = {"current": m.current, "rms_size": m.rms_size, "rms_angle": m.rms_angle,
                  "emittance": m.emittance, "iterations": len(c.history),
                  "converged": int(c.converged)}  # fmt: skip
    batch.close()
    return out
