"""Gradients through the converged Vlasov iteration: a hand-written adjoint behind
``torch.autograd.Function``.

The design workload asks for the gradients of plane moments (the rms divergence and the
transmitted current at a plane) with respect to the electrode voltages and the beam
current.  The reference differentiates by finite differences of whole solves
(``optimization/einzel.py``); here the converged fixed point ``rho = G(rho; V, I)`` --
``G`` the density the beam deposits when traced in the potential of ``rho`` -- is
differentiated implicitly:

- the adjoint density solves ``lambda = (dJ/drho)^T + G_rho^T lambda``, by the fixed-point
  iteration ``lambda <- M^T D^T T^T (lambda / Vol, dJ/dhits)`` (it contracts as the forward
  iteration does): ``T^T`` the reverse sweep of the trace (``bt_adjoint_sweep``: RK4 steps
  recomputed from checkpoints every 64 steps; gather and deposit each other's adjoints),
  ``D^T`` the edge field's transpose (``bt_edge_field_adjoint``) and ``M^T`` the
  transposed linear field solve, which reuses the multigrid (``bt_poisson_set_transposed``);
- ``dJ/dV_e`` is the sensitivity to the potentials held by electrode e, ``dJ/dI`` the
  direct term of the crossings' currents plus ``lambda . G / I`` (the deposit is linear
  in the current).

The scope is the lens workload's: RK4, one uniform patch, no magnetic field, no plasma,
not relativistic, planar or cylindrical.
"""

from __future__ import annotations

import ctypes
import functools
import math
from dataclasses import dataclass, replace
from typing import Any

import numpy as np

from beamtracer_b200 import _lib

#: Steps between the trace's checkpoints (the reverse sweep's memory bound).
SEGMENT = 64


class TraceAdjoint:
    """The reverse of one trace held by a `TraceEngine` through the edge fields ``fx``,
    ``fy`` (device arrays): its checkpoints, and sweeps that turn adjoints of the trace's
    node charges and plane crossings into the adjoint of the edge fields."""

    def __init__(self, engine, fx, fy) -> None:
        import torch

        from beamtracer_b200.tracer import geometry_code

        mesh = engine.mesh
        code = geometry_code(mesh)
        problems = {
            "a graded mesh": mesh.graded, "a symmetry plane": code == 2,
            "a magnetic field": engine.magnetic is not None,
            "the Boris integrator": engine.integrator != "rk4",
            "a relativistic trace": engine.inv_c2 > 0.0,
        }  # fmt: skip
        given = [name for name, present in problems.items() if present]
        if given:
            raise NotImplementedError("the trace's adjoint does not take " + ", ".join(given))
        self.engine = engine
        self.fx, self.fy = fx.reshape(-1).contiguous(), fy.reshape(-1).contiguous()
        n = engine.n
        nx, ny = mesh.shape
        most = int(engine.steps.max()) if n else 0
        self.segments = max(1, math.ceil(most / SEGMENT))
        self.checkpoints = torch.empty(self.segments * 6 * max(n, 1), dtype=torch.float64,
                                       device="cuda")  # fmt: skip
        d = _lib.dptr
        lo_x, lo_y = mesh.logical_origin
        self.args = _lib.AdjointArgs(
            d(engine.x0), d(engine.v0), d(engine.qm), d(engine.dq), d(engine.steps), n,
            d(self.fx), d(self.fy), nx, ny, float(lo_x), float(lo_y), float(mesh.h), code,
            float(engine.step_fraction), d(engine.planes_dev), len(engine.planes),
            d(engine.counts), int(engine.hits.shape[2]), d(self.checkpoints), self.segments,
        )  # fmt: skip
        self.shape = mesh.shape

    def record(self, end_state=None) -> None:
        """Replay the trace and keep its checkpoints (``end_state``: (6, n) device array for
        the replay's end states, or None)."""
        ctx = _lib.context()
        _lib.check(_lib.lib().bt_adjoint_checkpoints(ctx.handle, ctypes.byref(self.args),
                                                     _lib.dptr(end_state)))  # fmt: skip

    def sweep(self, charge_seed=None, hit_seed=None):
        """``(fx_bar, fy_bar)``: the edge fields' adjoint of a quantity whose adjoint of the
        node charges is ``charge_seed`` ((nx, ny) device) and of the hit buffers
        ``hit_seed`` ((n, planes, capacity, 8) device, slots 1-5); either may be None."""
        import torch

        nx, ny = self.shape
        fx_bar = torch.zeros((nx + 1) * ny, dtype=torch.float64, device="cuda")
        fy_bar = torch.zeros(nx * (ny + 1), dtype=torch.float64, device="cuda")
        ctx = _lib.context()
        _lib.check(_lib.lib().bt_adjoint_sweep(
            ctx.handle, ctypes.byref(self.args), _lib.dptr(charge_seed), _lib.dptr(hit_seed),
            _lib.dptr(fx_bar), _lib.dptr(fy_bar)))  # fmt: skip
        return fx_bar.reshape(nx + 1, ny), fy_bar.reshape(nx, ny + 1)


def edge_field_adjoint(arrays, fx_bar, fy_bar, extrapolation):
    """``D^T (fx_bar, fy_bar)``: the potential's adjoint (device (nx, ny)) from the edge
    fields' on a mesh's device arrays (`MeshArrays`)."""
    import torch

    mesh = arrays.mesh
    nx, ny = mesh.shape
    out = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
    faces = (ctypes.c_int32 * 4)(*[int(f == "symmetric") for f in extrapolation])
    ctx = _lib.context()
    _lib.check(_lib.lib().bt_edge_field_adjoint(
        ctx.handle, _lib.dptr(fx_bar.contiguous()), _lib.dptr(fy_bar.contiguous()),
        _lib.dptr(arrays.solid), _lib.dptr(arrays.near), _lib.dptr(arrays.distance),
        _lib.dptr(arrays.dx), nx, ny, float(mesh.h), faces, _lib.dptr(out)))  # fmt: skip
    return out


@dataclass
class FixedPointAdjoint:
    """The adjoint of a converged solve: the adjoint density ``lam`` (nx, ny), the
    potential's adjoint ``phi_bar`` and ``z = A_ff^-T phi_bar``, and the iterations."""

    lam: Any
    phi_bar: Any
    z: Any
    iterations: int
    change: float


class SolveAdjoint:
    """The adjoint of a converged `BeamOptics` solve (linear mixing or its fixed point; a
    linear field solve): built once per solve, applied to any objective of its crossings."""

    def __init__(self, model) -> None:
        from scipy import constants

        from beamtracer_b200.fields import MeshArrays
        from beamtracer_b200.poisson import IonOpticsPoisson

        if model.config.plasma is not None:
            raise NotImplementedError("the adjoint takes a linear field solve (no plasma)")
        state = model.state
        self.model = model
        self.mesh = model.mesh
        self.engine = model.tracer.engine()
        self.trace = TraceAdjoint(self.engine, state.electric.fx_device, state.electric.fy_device)
        self.trace.record()
        self.arrays = MeshArrays(self.mesh)
        self.extrapolation = state.electric.extrapolation
        self.transposed = IonOpticsPoisson(self.mesh, transposed=True)
        self.eps0 = constants.epsilon_0
        #: the deposit of the last trace: G at the fixed point
        self.deposit = self.engine.density().clone()

    def hit_seed(self, plane: int, point_bar, velocity_bar):
        """The adjoint of the crossings of plane ``plane`` (in the order of the state's
        `PlaneHits`) laid out as the hit buffers (n, planes, capacity, 8)."""
        import torch

        engine = self.engine
        _ = self.model.state.trace  # the crossings' slots are recorded with the result
        k, c = engine.hit_slots[plane]
        seed = torch.zeros_like(engine.hits)
        values = torch.cat([torch.as_tensor(point_bar, dtype=torch.float64)[1:3],
                            torch.as_tensor(velocity_bar, dtype=torch.float64)]).T.cuda()  # fmt: skip
        seed[k, plane, c, 1:6] = values
        return seed

    def solve(self, hit_seed, tolerance: float = 1e-8, max_iterations: int = 100,
              depth: int = 4) -> FixedPointAdjoint:  # fmt: skip
        """``lambda = (dJ/drho)^T + G_rho^T lambda`` from the crossings' adjoint
        ``hit_seed`` (hit-buffer layout): the map is affine, so its fixed point is found by
        Anderson mixing of depth ``depth`` (`AndersonMixer`; for an affine map a Krylov
        method) until the residual ``|K(lambda) - lambda|`` is below ``tolerance`` of
        ``|K(lambda)|``; every transposed solve starts from the last one's solution."""
        import torch

        from beamtracer_b200.vlasov import AndersonMixer

        nx, ny = self.mesh.shape
        volumes = self.engine.volumes.reshape(nx, ny)
        lam = torch.zeros((nx, ny), dtype=torch.float64, device="cuda")
        z = torch.zeros_like(lam)
        mixer = AndersonMixer(depth, relaxation=1.0) if depth > 0 else None
        change = float("inf")
        for iteration in range(1, max_iterations + 1):
            charge_seed = (lam / volumes).contiguous() if iteration > 1 else None
            fx_bar, fy_bar = self.trace.sweep(charge_seed, hit_seed)
            phi_bar = edge_field_adjoint(self.arrays, fx_bar, fy_bar, self.extrapolation)
            self.transposed.solve_device(z, self.eps0 * phi_bar, linear_tolerance=1e-12)
            image = z / self.eps0
            scale = float(image.abs().max())
            change = float((image - lam).abs().max()) / scale if scale > 0 else 0.0
            if change <= tolerance:
                lam = image
                break
            lam = mixer.update(lam, image) if mixer is not None else image
        # phi_bar and z are those of the last evaluation, whose input is within the
        # tolerance of the fixed point
        return FixedPointAdjoint(lam, phi_bar, z, iteration, change)

    def parameter_gradient(self, adjoint: FixedPointAdjoint, current: float) -> np.ndarray:
        """``[dJ/dV_e for every electrode] + [dJ/dI]`` through the fixed point (without the
        crossings' direct current term, which the caller adds)."""
        import torch

        held = torch.empty_like(adjoint.lam)
        self.transposed.fixed_adjoint(adjoint.z, adjoint.phi_bar, held)
        solid = torch.from_numpy(np.ascontiguousarray(self.mesh.solid, dtype=np.int64)).cuda()
        grads = [float(held[solid == e].sum()) for e in range(len(self.mesh.electrodes))]
        grads.append(float((adjoint.lam * self.deposit).sum()) / current)
        return np.array(grads)


# -- differentiable moments ------------------------------------------------------------------


def moments_torch(point, velocity, current, direction, cylindrical: bool = True) -> dict:
    """The current, rms size, rms angle, correlation and emittance of the forward crossings
    (torch tensors, differentiable): the formulas of `plane_moments` (rings projected on a
    transverse plane in cylindrical geometry, moments about the means in planar)."""
    import torch

    keep = direction > 0
    w = current[keep].abs()
    total = w.sum()
    wn = w / total
    p, v = point[:, keep], velocity[:, keep]
    if cylindrical:
        xx = 0.5 * (wn * (p[1] * p[1] + p[2] * p[2])).sum()
        xp = 0.5 * (wn * ((p[1] * v[1] + p[2] * v[2]) / v[0])).sum()
        pp = 0.5 * (wn * ((v[1] * v[1] + v[2] * v[2]) / (v[0] * v[0]))).sum()
    else:
        y, yp = p[1], v[1] / v[0]
        dy, dyp = y - (wn * y).sum(), yp - (wn * yp).sum()
        xx, xp, pp = (wn * dy * dy).sum(), (wn * dy * dyp).sum(), (wn * dyp * dyp).sum()
    emittance = torch.sqrt(torch.clamp(xx * pp - xp * xp, min=0.0))
    return {"current": total, "rms_size": torch.sqrt(xx), "rms_angle": torch.sqrt(pp),
            "correlation": xp, "emittance": emittance}  # fmt: skip


# -- the einzel lens as a differentiable function ----------------------------------------------


class LensProblem:
    """An einzel design whose plate voltages and beam current are parameters: ``solve``
    converges it for a parameter vector ``(V_1, V_2, V_3, I)``, ``gradient`` reverses it."""

    def __init__(self, design, plane: float = 79e-3, tolerance: float = 1e-6,
                 iterations: int = 60, adjoint_tolerance: float = 1e-8) -> None:  # fmt: skip
        self.design = design
        self.plane = float(plane)
        self.tolerance = float(tolerance)
        self.iterations = int(iterations)
        self.adjoint_tolerance = float(adjoint_tolerance)
        #: the fixed-point iterations of the last adjoint solve
        self.adjoint_iterations = 0
        #: whether the last forward solve met its tolerance
        self.converged = False
        #: the largest |E| on every electrode's surface in the last forward solve [V/m]
        self.surface_fields: dict[str, float] = {}

    def config(self, params: np.ndarray):
        from beamtracer_b200.einzel import einzel_config

        design = replace(self.design, voltages=tuple(float(v) for v in params[:3]),
                         current=float(params[3]))  # fmt: skip
        return einzel_config(design, tolerance=self.tolerance, iterations=self.iterations)

    def solve(self, params: np.ndarray):
        from beamtracer_b200.model import BeamOptics

        return BeamOptics(self.config(params)).run()

    def plane_index(self, model) -> int:
        planes = [p.position_x for p in model.state.trace.planes]
        return int(np.argmin([abs(p - self.plane) for p in planes]))


class LensMoments:
    """``torch.autograd.Function`` of a `LensProblem`: parameters ``(V_1, V_2, V_3, I)`` ->
    the crossings of the plane (point, velocity, current, direction); the backward pass is
    the adjoint of the converged solve (`SolveAdjoint`)."""

    @staticmethod
    @functools.cache
    def function():
        import torch

        class _Lens(torch.autograd.Function):
            @staticmethod
            def forward(ctx, params, problem):
                values = params.detach().cpu().numpy().astype(np.float64)
                model = problem.solve(values)
                problem.converged = bool(model.stats["converged"])
                problem.surface_fields = model.surface_fields()
                hits = model.plane(problem.plane)
                ctx.problem, ctx.model, ctx.values = problem, model, values
                ctx.hits_current = np.array(hits.current, dtype=np.float64)
                ctx.adjoint = None
                as_tensor = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))  # noqa: E731
                direction = as_tensor(hits.direction)
                ctx.mark_non_differentiable(direction)
                return as_tensor(hits.point), as_tensor(hits.velocity), as_tensor(hits.current), direction

            @staticmethod
            def backward(ctx, point_bar, velocity_bar, current_bar, _direction_bar):
                problem, model = ctx.problem, ctx.model
                current = float(ctx.values[3])
                grad = np.zeros(4)
                # the crossings' currents are the rings' currents: proportional to I
                grad[3] += float((current_bar.numpy() * ctx.hits_current).sum()) / current
                if bool((point_bar != 0).any()) or bool((velocity_bar != 0).any()):
                    if ctx.adjoint is None:
                        ctx.adjoint = SolveAdjoint(model)
                    adjoint = ctx.adjoint
                    seed = adjoint.hit_seed(problem.plane_index(model), point_bar, velocity_bar)
                    fixed = adjoint.solve(seed, tolerance=problem.adjoint_tolerance)
                    grad += adjoint.parameter_gradient(fixed, current)
                    problem.adjoint_iterations = fixed.iterations
                return torch.from_numpy(grad).to(torch.float64), None

        return _Lens

    @classmethod
    def apply(cls, params, problem):
        return cls.function().apply(params, problem)


def adjoint_design_gradient(design, plane: float = 79e-3, tolerance: float = 1e-6,
                            iterations: int = 60, adjoint_tolerance: float = 1e-8) -> dict:  # fmt: skip
    """The gradients of the rms angle and the current at ``plane`` with respect to the three
    plate voltages and the beam current (`GRADIENT_PARAMETERS`) by the adjoint of one
    solve converged to ``tolerance`` [V] (the gradient is linearised there: unlike central
    differences, which divide the solves' error by the step, it needs no tighter solve),
    through ``torch.autograd``."""
    import torch

    from beamtracer_b200.einzel import resolved_voltages

    problem = LensProblem(design, plane, tolerance, iterations, adjoint_tolerance)
    start = [*resolved_voltages(design), design.current]
    params = torch.tensor(start, dtype=torch.float64, requires_grad=True)
    point, velocity, current, direction = LensMoments.apply(params, problem)
    moments = moments_torch(point, velocity, current, direction, cylindrical=True)
    (angle,) = torch.autograd.grad(moments["rms_angle"], params, retain_graph=True)
    (transmitted,) = torch.autograd.grad(moments["current"], params)
    return {"rms_angle": angle.numpy().copy(), "current": transmitted.numpy().copy(),
            "moments": {k: float(v.detach()) for k, v in moments.items()}, "solves": 1,
            "adjoint_iterations": problem.adjoint_iterations,
            "converged": problem.converged, "surface_fields": dict(problem.surface_fields)}  # fmt: skip


# -- gradients of the candidates of a batch ----------------------------------------------------


class _CandidateSolve:
    """What `SolveAdjoint` and `LensMoments` read of a converged solve, for candidate ``k``
    of a finished `BatchedVlasov`: its mesh and configuration, the edge fields of its last
    iteration (kept in the batch's buffers) and its beam traced alone through them (the
    same trajectories as in the batch, bit for bit)."""

    def __init__(self, batch, k: int) -> None:
        from types import SimpleNamespace

        from beamtracer_b200.fields import default_extrapolation

        c = batch.candidates[k]
        if c.planes is None:
            raise RuntimeError("the candidate has not finished")
        self.config = c.config
        self.mesh = c.mesh
        fx, fy = batch.edge_views(k)
        engine = c.engine
        engine.run(fx, fy)
        self.tracer = SimpleNamespace(engine=lambda: engine)
        electric = SimpleNamespace(fx_device=fx, fy_device=fy,
                                   extrapolation=tuple(default_extrapolation(c.mesh)))  # fmt: skip
        self.state = SimpleNamespace(electric=electric, trace=engine.result())
        self.stats = {"converged": bool(c.converged)}

    def surface_fields(self) -> dict[str, float]:
        return {}

    def plane(self, x: float):
        match = [hits for hits in self.state.trace.planes if np.isclose(hits.position_x, x)]
        if not match:
            raise KeyError(f"no diagnostic plane at x = {x}")
        return match[0]


class _BatchLensProblem(LensProblem):
    """A `LensProblem` whose forward solve is candidate ``k`` of a finished batch (solved
    there at the design's own parameters)."""

    def __init__(self, batch, k: int, design, plane: float, adjoint_tolerance: float) -> None:
        super().__init__(design, plane, adjoint_tolerance=adjoint_tolerance)
        self.batch, self.k = batch, k

    def solve(self, params: np.ndarray):
        return _CandidateSolve(self.batch, self.k)


def batch_design_gradients(batch, designs, plane: float = 79e-3, adjoint_tolerance: float = 1e-8,
                           concurrency: int = 8) -> list[dict]:  # fmt: skip
    """The gradients of the rms angle and the current at ``plane`` with respect to the
    plate voltages and the beam current (`GRADIENT_PARAMETERS`) of every candidate of a
    finished `BatchedVlasov` of einzel ``designs`` (in its order): the adjoint of each
    candidate's converged solve, as `adjoint_design_gradient` takes it of a solve of its
    own (the batch's candidates should be converged as tightly, e.g. to 1e-6 V).  With
    ``concurrency`` > 1 that many host threads take candidates at once, each on its own
    CUDA stream and library context; the gradients agree with one candidate at a time to
    rounding (the reverse sweep's scatter adds with atomics)."""
    import threading

    import torch

    from beamtracer_b200.einzel import design_cost, resolved_voltages

    device = torch.cuda.current_device()
    torch.cuda.synchronize()  # the batch's fields, read by every thread
    local = threading.local()

    def gradient(k: int) -> tuple[int, dict]:
        design = designs[k]
        torch.cuda.set_device(device)
        if getattr(local, "stream", None) is None:
            local.stream = torch.cuda.Stream() if concurrency > 1 else torch.cuda.current_stream()
        with torch.cuda.stream(local.stream):
            problem = _BatchLensProblem(batch, k, design, plane, adjoint_tolerance)
            start = [*resolved_voltages(design), design.current]
            params = torch.tensor(start, dtype=torch.float64, requires_grad=True)
            point, velocity, current, direction = LensMoments.apply(params, problem)
            moments = moments_torch(point, velocity, current, direction, cylindrical=True)
            (angle,) = torch.autograd.grad(moments["rms_angle"], params, retain_graph=True)
            (transmitted,) = torch.autograd.grad(moments["current"], params)
        local.stream.synchronize()
        return k, {"rms_angle": angle.numpy().copy(), "current": transmitted.numpy().copy(),
                   "moments": {name: float(v.detach()) for name, v in moments.items()},
                   "adjoint_iterations": problem.adjoint_iterations,
                   "converged": problem.converged}  # fmt: skip

    # the costliest first, so the threads finish together
    order = sorted(range(len(designs)), key=lambda k: -design_cost(designs[k]))
    if concurrency <= 1:
        done = dict(gradient(k) for k in order)
    else:
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=concurrency) as pool:
            done = dict(pool.map(gradient, order))
    return [done[k] for k in range(len(designs))]
