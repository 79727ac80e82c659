"""Benchmark: converged Vlasov solves per second of the einzel lens at 801 x 201.

The workload is the einzel lens of the reference's configuration list at scale: a
cylindrical (x, r) mesh of 801 x 201 nodes on 80 x 20 mm, three plates at 0 / V_mid / 0
(V_mid seeded uniform in 5-9 kV), Neumann faces, a 10 keV H+ beam of 1 mA in 20,000 rings
(seeded Gaussian radius, rms 2 mm cut at 4 mm, 5 mrad rms angle, 2 mm mrad emittance),
planes at 70 and 79 mm; the reference's iteration defaults (at most 20 iterations, linear
mixing with relaxation 1, until the potential changes by less than 1 mV).  A step is one
converged solve from a zero charge density.

- ``value``: steps per second with the mesh, operator and beam resident on the device
  (CUDA events around each step on the launching stream; L2 flushed between steps);
- ``e2e``: the same through the public call ``BeamOptics(config).run()`` plus
  ``beam_moments()``, from host inputs to host results;
- ``roofline``: the dominant kernel's launches timed live (CUDA events) against its
  algorithmic work;
- ``cpu_baseline``: the oracle (the reference's kernel restated in C, OpenMP over every
  host core, and SciPy's sparse LU for the field) on one converged solve of the same lens,
  its problem built on the host alone;
- ``parity``: the device solve's potential and plane moments against that oracle solve's
  (relative differences; the bound is 1e-6 of the moments).

``--impl reference`` times that CPU path alone (the reference's Pyccel build cannot be
made here) and prints its moments.  Under torchrun every rank solves its own lens (weak
scaling, no collective).
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "converged einzel-lens Vlasov solves/s (801x201 cyl., 20k rings)"
UNIT = "solves/s"
WORKLOAD = "einzel lens 801x201 cylindrical, 20,000 rings, 3 plates, tol 1 mV"
#: FP64 operations of one RK4 step of the trace kernel, counted from its source
#: (trace.cu): four field gathers (2 x 3 bilinear lerps of 3 ops + cell arithmetic),
#: the stage updates, the step size, the Hermite midpoint and the deposit weights.
FLOPS_PER_RK4_STEP = 370
#: Deposit bytes per record (key 4 B + u, w, q 24 B written by the trace, read by the
#: reduction) and per node (charge read and written).
DEPOSIT_BYTES_PER_RECORD = 28 * 2
NOMINAL_FP64_TFLOPS = 37.0
#: The trace's algorithmic bytes per step: its deposit record (u32 key, u, w, q f64).  The
#: kernel writes a 4-byte key per step and a 32-byte record (the four node charges) per run
#: of steps in one cell.
TRACE_BYTES_PER_STEP = 28
#: DRAM bytes read + written per trace_window launch at this workload: ncu's
#: dram__bytes_read.sum + dram__bytes_write.sum over launches 21-25 of one converged solve
#: (1.957 MB read, 0.124 MB written on average; the records it writes stay in L2 and drain
#: during the deposit).
TRACE_DRAM_BYTES_PER_LAUNCH = 2.081e6
#: Timed end-to-end calls (after one untimed call); their median is reported.
E2E_RUNS = 5


def _env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )  # fmt: skip
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc) -> None:
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [line for line in out.splitlines() if line.strip()]
        else:
            self.lines = []

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8], strict=False):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}  # fmt: skip


def build_workload(seed: int, small: bool = False):
    from beamtracer_b200.einzel import EinzelDesign, einzel_config

    if small:
        return einzel_config(EinzelDesign(seed=seed, shape=(401, 101), trajectories=2000))
    return einzel_config(EinzelDesign(seed=seed))


def run_profile_adjoint(args) -> None:
    """One adjoint gradient of the lens at 401 x 101 with 2,000 rings to warm up, then one
    inside the NVTX range "profiled_adjoint" (the range a profiler's capture selects)."""
    import torch

    from beamtracer_b200.adjoint import adjoint_design_gradient
    from beamtracer_b200.einzel import EinzelDesign

    torch.cuda.set_device(0)
    design = EinzelDesign(shape=(401, 101), trajectories=2000, seed=2)
    adjoint_design_gradient(design)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("profiled_adjoint")
    out = adjoint_design_gradient(design)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": "adjoint", "iterations": out["adjoint_iterations"]}))


def run_profile(args) -> None:
    """One converged solve to warm up, then one inside the NVTX range "profiled_solve"
    (the range a profiler's capture selects)."""
    import torch

    from beamtracer_b200.model import BeamOptics
    from beamtracer_b200.poisson import IonOpticsPoisson
    from beamtracer_b200.vlasov import vlasov_iterate

    torch.cuda.set_device(0)
    config = build_workload(2, small=args.small)
    model = BeamOptics(config, contracted_trace=args.trace == "contracted")
    model.tracer.window = args.window
    poisson = IonOpticsPoisson(model.mesh, backend=config.field_backend)

    def solve():
        return vlasov_iterate(model.mesh, model._particles, model.tracer,
                              iterations=config.iterations, tolerance=config.tolerance,
                              relaxation=config.relaxation, poisson=poisson)  # fmt: skip

    solve()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("profiled_solve")
    state = solve()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": "ok", "small": args.small,
                      "iterations": len(state.history),
                      "total_steps": sum(h["total_steps"] for h in state.history)}))  # fmt: skip


#: The workload's identity, the same in both arms' lines.
def workload_config() -> dict:
    return {"workload": WORKLOAD, "trajectories": 20000, "mesh": [801, 201],
            "seed": 2, "l2": "256 MiB written between timed steps"}  # fmt: skip


MOMENT_NAMES = ("current", "rms_size", "rms_angle", "emittance")


def oracle_solve(config) -> tuple[float, dict, dict]:
    """The oracle's converged solve of a configuration, built on the host alone (no device
    classification, no library load): its seconds, its output and its moments per plane."""
    from beamtracer_b200.diagnostics import plane_moments
    from beamtracer_b200.tracer import PlaneHits
    from oracle import vlasov as oracle_vlasov
    from tests.vlasov_cases import config_problem

    problem, particles, j_over_v = config_problem(config)
    start = time.perf_counter()
    out = oracle_vlasov.vlasov(problem, particles, j_over_v, iterations=config.iterations,
                               tolerance=config.tolerance, relaxation=config.relaxation)
    seconds = time.perf_counter() - start
    from scipy import constants

    mass = np.array([beam.mass for beam in config.beams]) * constants.atomic_mass
    moments = {}
    for plane, hits in zip(problem.planes, oracle_vlasov.plane_hits(
            problem, out["trace"], particles.current, particles.species)):  # fmt: skip
        m = plane_moments(PlaneHits(plane, *hits), cylindrical=problem.geometry == 1, mass=mass)
        moments[f"{plane * 1e3:g}mm"] = {k: getattr(m, k) for k in MOMENT_NAMES}
    return seconds, out, moments


def parity_report(potential: np.ndarray, moments: dict, oracle_out: dict,
                  oracle_moments: dict) -> dict:  # fmt: skip
    """The device solve against the oracle's: the potential's largest difference relative
    to the oracle's largest magnitude, and every moment's relative difference."""
    ref = oracle_out["potential"]
    phi_rel = float(np.max(np.abs(potential - ref)) / np.max(np.abs(ref)))
    per = {plane: {k: abs(moments[plane][k] - v) / abs(v) for k, v in values.items()}
           for plane, values in oracle_moments.items()}  # fmt: skip
    worst = max(max(d.values()) for d in per.values())
    return {"against": "the oracle's converged solve of the same lens (FP64, same seed)",
            "potential_max_rel": phi_rel, "moments_max_rel": worst, "moments_rel": per,
            "oracle_iterations": len(oracle_out["history"]), "bound": 1e-6,
            "within_bound": bool(phi_rel <= 1e-6 and worst <= 1e-6)}  # fmt: skip


def run_reference(args, rank: int) -> None:
    """The reference arm: the oracle's converged solve of the same lens on every host core
    (the field by SciPy's LU, the trace and deposit by the C port), each step one solve run
    until the potential changes by less than the tolerance, as the device solve is.  The
    problem is built on the host alone."""
    if rank != 0:
        return
    from oracle import kernels as oracle_kernels

    config = build_workload(2)
    if args.warmup > 0:
        oracle_solve(config)  # the oracle's build and caches
    runs = [oracle_solve(config) for _ in range(max(args.steps, 1))]
    seconds = float(np.mean([r[0] for r in runs]))
    iterations = len(runs[-1][1]["history"])
    base = {"value": 1.0 / seconds, "unit": UNIT, "cores": oracle_kernels.host_cores(),
            "kind": "port",
            "sample": f"converged solves of the oracle ({iterations} iterations: SciPy LU "
                      f"field, C trace and deposit), {seconds:.2f} s each"}  # fmt: skip
    line = {
        "impl": "reference", "metric": METRIC, "value": 1.0 / seconds, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(), "iterations_per_solve": iterations,
        "cpu_baseline": base,
        "e2e": {"value": 1.0 / seconds, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "moments": runs[-1][2],
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def design_measurements(stream) -> dict:
    """The metric's design half, measured in the default run: gradient evaluations per
    second of the lens at 401 x 101 with 8,000 rings by the adjoint of one solve and by the
    plain form (central differences of 8 solves, 8 at once), and candidates per second of
    16 seeded sweep candidates solved one at a time and 8 at once on their own streams.
    Device time with CUDA events on the launching stream; one untimed call first."""
    import torch

    from beamtracer_b200.adjoint import adjoint_design_gradient
    from beamtracer_b200.einzel import EinzelDesign, design_gradient, sweep, sweep_designs

    def timed(fn, repeats: int) -> tuple[float, object]:
        fn()
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(repeats):
            out = fn()
        stop.record(stream)
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / repeats, out

    c4 = EinzelDesign(shape=(401, 101), trajectories=8000, seed=2)
    adj_ms, adj = timed(lambda: adjoint_design_gradient(c4), 3)
    fd_ms, fd = timed(lambda: design_gradient(c4, concurrency=8), 3)
    diff = float(np.max(np.abs(adj["rms_angle"] - fd["rms_angle"])) / np.max(np.abs(fd["rms_angle"])))
    from beamtracer_b200.batch import batched_sweep

    designs = sweep_designs(32)
    one_ms, _ = timed(lambda: sweep(designs, concurrency=1), 1)
    many_ms, _ = timed(lambda: sweep(designs, concurrency=8), 1)
    batch_ms, _ = timed(lambda: batched_sweep(designs), 1)
    return {
        "gradient": {"workload": "einzel 401x101, 8,000 rings, d(rms angle, current)/d(V1, V2, "
                                 "V3, I) at 79 mm", "unit": "gradient evals/s",
                     "adjoint": 1e3 / adj_ms, "plain_form": 1e3 / fd_ms,
                     "speedup_over_plain": fd_ms / adj_ms, "max_rel_diff": diff,
                     "adjoint_iterations": adj["adjoint_iterations"]},
        "sweep": {"workload": "32 seeded einzel candidates (257x65..1025x257, 2k-20k rings)",
                  "unit": "candidates/s", "batched": 32e3 / batch_ms,
                  "concurrent_8_streams": 32e3 / many_ms, "one_at_a_time": 32e3 / one_ms,
                  "speedup_over_plain": one_ms / batch_ms, "target_speedup": 20.0},
    }  # fmt: skip


def run_plasma(args) -> None:
    """The planar plasma + solenoid extraction (1025 x 513, x graded, 100,000 H+, Newton
    field solve, Boris step in the solenoid's field): converged solves per second, device
    resident and through ``solenoid_extraction(design).run()`` from host inputs."""
    import torch

    from beamtracer_b200 import _lib
    from beamtracer_b200.poisson import IonOpticsPoisson
    from beamtracer_b200.solenoid_extraction import SolenoidExtractionDesign, solenoid_extraction

    torch.cuda.set_device(0)
    design = SolenoidExtractionDesign()
    case = solenoid_extraction(design, window=args.window)
    poisson = IonOpticsPoisson(case.mesh)
    ctx = _lib.context()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        state = case.run(poisson=poisson)
    torch.cuda.synchronize()
    ctx.set_timing(True)
    ctx.reset_timers()
    launches_before = ctx.launch_count()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]  # fmt: skip
    steps_total = 0
    with ClockSampler(0) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))
            events[k][0].record(stream)
            state = case.run(poisson=poisson)
            events[k][1].record(stream)
            steps_total += sum(h["total_steps"] for h in state.history)
        torch.cuda.synchronize()
    total_ms = float(sum(a.elapsed_time(b) for a, b in events))
    timers = {name: ctx.read_timer(name) for name in
              ("trace_window", "deposit", "field_solve", "vcycle", "hierarchy",
               "edge_field")}  # fmt: skip
    ctx.set_timing(False)
    launches = ctx.launch_count() - launches_before
    e2e_ms = []
    for k in range(3):
        gc.collect()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        solenoid_extraction(design, window=args.window).run()
        stop.record(stream)
        torch.cuda.synchronize()
        if k:
            e2e_ms.append(start.elapsed_time(stop))
    nx, ny = design.shape
    line = {
        "metric": "converged plasma+solenoid extraction solves/s (1025x513 planar graded, "
                  "100k H+)", "value": args.steps / (total_ms / 1e3), "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "solenoid extraction 1025x513 planar, x graded, 100,000 H+, "
                               "Boltzmann electrons, Boris in a 0.2 T solenoid",
                   "mesh": [nx, ny], "trajectories": design.trajectories,
                   "iterations_per_solve": len(state.history),
                   "newton_steps_per_solve": sum(h["newton_iterations"] for h in state.history),
                   "l2": "256 MiB written between timed steps"},
        "kernels": {name: {"ms": ms, "launches": n, "share": ms / total_ms}
                    for name, (ms, n) in timers.items()},
        "steps_per_solve": steps_total / args.steps,
        "e2e": {"value": 1e3 / float(np.median(e2e_ms)), "unit": UNIT,
                "runs_ms": [round(v, 2) for v in e2e_ms]},
        "gpu_launches": launches, "clocks": clocks.summary(),
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def run_refined(args) -> None:
    """Refined boxes: the reference's refined extraction (``tests/unit/test_refinement.py``:
    81 x 31 cylindrical, boxes of levels 1 and 2 over the aperture, a Boltzmann electron
    plasma, 100 ions), converged solves per second through ``BeamOptics(config).run()``,
    beside the oracle's converged solve of the same case (composite LU, the C trace on the
    host cores) and the two potentials' largest difference."""
    import torch

    from beamtracer_b200 import BeamOptics, RefinementParams
    from oracle import composite as oracle_composite
    from oracle import kernels as oracle_kernels
    from oracle import vlasov as oracle_vlasov
    from tests.vlasov_cases import extraction, refined_problem

    torch.cuda.set_device(0)
    mm = 1e-3
    config = extraction(1.0, refinement=[RefinementParams(1, (0.0, 0.0), (2.0 * mm, 1.5 * mm)),
                                         RefinementParams(2, (0.0, 0.0), (1.5 * mm, 1.2 * mm))])
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        BeamOptics(config).run()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            model = BeamOptics(config).run()
            stop.record(stream)
            torch.cuda.synchronize()
            times.append(start.elapsed_time(stop))
    state = model.state
    iterations = len(state.history)
    problem, particles, j_over_v, layout = refined_problem(config)
    t0 = time.perf_counter()
    out = oracle_composite.vlasov(problem, layout, particles, iterations=iterations,
                                  relaxation=config.relaxation,
                                  plasma=oracle_vlasov.Plasma(5.0, 5.0, 0.6e-3, -1),
                                  j_over_v=j_over_v)  # fmt: skip
    cpu_s = time.perf_counter() - t0
    phi_o = out["potential"]
    total_ms = float(sum(times))
    line = {
        "metric": "converged refined-box extraction solves/s (81x31 cyl. + boxes of levels 1, 2; "
                  "Boltzmann plasma)", "value": args.steps / (total_ms / 1e3), "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "refined extraction: the reference's refined cylindrical case",
                   "composite_nodes": layout.size, "patches": len(layout.patches),
                   "iterations_per_solve": iterations,
                   "newton_steps_per_solve": sum(h["newton_iterations"] for h in state.history)},
        "e2e": {"value": args.steps / (total_ms / 1e3), "unit": UNIT,
                "note": "the timed call is the public BeamOptics(config).run() from host inputs"},
        "cpu_baseline": {"value": 1.0 / cpu_s, "unit": UNIT, "cores": oracle_kernels.host_cores(),
                         "kind": "port", "sample": f"one solve of {iterations} iterations by the "
                         "oracle (composite LU, C trace with OpenMP)"},
        "parity": {"potential_max_rel": float(np.abs(state.composite_potential - phi_o).max()
                                              / np.ptp(phi_o))},
        "clocks": clocks.summary(),
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def sweep_with_gradients(designs, stream, concurrency: int = 8) -> dict:
    """The sweep's forward plus adjoint (one GPU): every candidate converged to 1e-6 V and
    its gradients of the rms angle and the current at 79 mm with respect to the plate
    voltages and the beam current -- batched (one `BatchedVlasov`, then the adjoint of each
    candidate's converged solve) and in the plain form (each candidate's own solve and
    adjoint, one at a time); both timed once with CUDA events, configuration building
    included, and their gradients compared."""
    import torch

    from beamtracer_b200.adjoint import adjoint_design_gradient, batch_design_gradients
    from beamtracer_b200.batch import BatchedVlasov
    from beamtracer_b200.einzel import einzel_config

    def timed(fn):
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        out = fn()
        stop.record(stream)
        torch.cuda.synchronize()
        return out, start.elapsed_time(stop)

    def batched():
        batch = BatchedVlasov([einzel_config(d, tolerance=1e-6, iterations=60)
                               for d in designs]).run()  # fmt: skip
        grads = batch_design_gradients(batch, designs, concurrency=concurrency)
        batch.close()
        return grads

    grads, batched_ms = timed(batched)
    plain, plain_ms = timed(lambda: [adjoint_design_gradient(d) for d in designs])
    worst, worst_k, diffs = 0.0, -1, []
    for k, (mine, alone) in enumerate(zip(grads, plain)):
        diff = 0.0
        for name in ("rms_angle", "current"):
            scale = float(np.abs(alone[name]).max())
            if scale > 0.0:
                diff = max(diff, float(np.abs(mine[name] - alone[name]).max()) / scale)
        diffs.append(diff)
        if diff > worst:
            worst, worst_k = diff, k
    n = len(designs)
    worst_case = None
    if worst_k >= 0:
        d = designs[worst_k]
        worst_case = {"candidate": worst_k, "mesh": list(d.shape), "trajectories": d.trajectories,
                      "converged_batched": bool(grads[worst_k]["converged"]),
                      "converged_plain": bool(plain[worst_k]["converged"]),
                      "adjoint_iterations": [grads[worst_k]["adjoint_iterations"],
                                             plain[worst_k]["adjoint_iterations"]]}  # fmt: skip
    return {"unit": "candidates/s", "batched": n * 1e3 / batched_ms,
            "plain_form": n * 1e3 / plain_ms, "speedup_over_plain": plain_ms / batched_ms,
            "max_rel_gradient_diff": worst, "worst_candidate": worst_case,
            "median_rel_gradient_diff": float(np.median(diffs)) if diffs else 0.0,
            "candidates_within_1e-4": int(sum(v <= 1e-4 for v in diffs)),
            "forward_tolerance_v": 1e-6,
            "concurrency": concurrency,
            "note": "batched forward in one BatchedVlasov, then each candidate's adjoint; "
                    "plain: each candidate's own solve and adjoint"}


def run_design(args, rank: int, world: int, local: int) -> None:
    """Design workloads: ``gradient`` -- the gradient of the rms angle and the current at
    79 mm with respect to the three plate voltages and the beam current of the einzel lens
    at 401 x 101 with 8,000 rings, by central differences of converged solves (8 solves an
    evaluation); ``sweep`` -- the seeded candidates of the batched design sweep (meshes of
    257 x 65 to 1025 x 257, 2,000-20,000 rings), every rank solving its cost-balanced share
    with no collective.  Device time with CUDA events, the max over ranks."""
    import torch
    import torch.distributed as dist

    from beamtracer_b200.einzel import EinzelDesign, design_gradient, share_of_designs, sweep, sweep_designs

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))  # fmt: skip
    stream = torch.cuda.current_stream()
    fd_line = None
    if args.workload == "gradient":
        from beamtracer_b200.adjoint import adjoint_design_gradient

        design = EinzelDesign(shape=(401, 101), trajectories=8000, seed=2 + rank)

        def fd_step():
            return design_gradient(design, concurrency=args.concurrency)

        def step():
            return adjoint_design_gradient(design)

        # the plain form first: central differences of 8 converged solves, 8 at once
        for _ in range(args.warmup):
            fd_result = fd_step()
        torch.cuda.synchronize()
        fd_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                     for _ in range(args.steps)]  # fmt: skip
        for k in range(args.steps):
            fd_events[k][0].record(stream)
            fd_result = fd_step()
            fd_events[k][1].record(stream)
        torch.cuda.synchronize()
        fd_ms = float(sum(a.elapsed_time(b) for a, b in fd_events)) / args.steps
        fd_line = {"method": "central differences of 8 converged solves (relative step 1e-4), "
                             f"{args.concurrency} at once on their own streams",
                   "value": world * 1e3 / fd_ms, "ms_per_step": fd_ms,
                   "rms_angle": [float(v) for v in fd_result["rms_angle"]],
                   "current": [float(v) for v in fd_result["current"]]}  # fmt: skip
        units_per_step, unit = world, "gradient evals/s"
        metric = "einzel design-gradient evals/s (401x101 cyl., 8k rings, 4 parameters)"
        workload = ("einzel lens 401x101, 8,000 rings: d(rms angle, current)/d(V1, V2, V3, J) "
                    "by the adjoint of one converged solve (torch.autograd through the "
                    "hand-written reverse)")
    else:
        from beamtracer_b200.batch import batched_sweep

        designs = sweep_designs(args.sweep_count)

        def step():
            return batched_sweep(designs, rank, world)

        # the plain form first: the same share, one candidate at a time
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        plain = sweep(designs, rank, world, concurrency=1)
        stop.record(stream)
        torch.cuda.synchronize()
        plain_ms = start.elapsed_time(stop)
        fd_line = {"method": "the plain form: BeamOptics(config).run() one candidate at a time",
                   "value": args.sweep_count * 1e3 / plain_ms, "ms_per_step": plain_ms}  # fmt: skip
        units_per_step, unit = args.sweep_count, "candidates/s"
        metric = "einzel design-sweep candidates/s (257x65..1025x257, 2k-20k rings)"
        workload = (f"{args.sweep_count} seeded einzel candidates (seed 5), cost-balanced "
                    "shares, each rank's share converged together in one batch (batched "
                    "trace, deposit and multigrid), configuration building included")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    from beamtracer_b200 import _lib

    ctx = _lib.context()
    ctx.set_timing(True)
    ctx.reset_timers()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]  # fmt: skip
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            events[k][0].record(stream)
            result = step()
            events[k][1].record(stream)
        torch.cuda.synchronize()
    total_ms = float(sum(a.elapsed_time(b) for a, b in events))
    # the calling thread's context times the launches it queued (the concurrent sweep's
    # worker threads have their own)
    kernels = {name: {"ms": ms, "launches": n} for name, (ms, n) in
               ((name, ctx.read_timer(name)) for name in
                ("trace_window", "deposit", "field_solve", "vcycle", "hierarchy",
                 "adjoint_checkpoints", "adjoint_sweep")) if n}  # fmt: skip
    ctx.set_timing(False)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": metric, "value": units_per_step * args.steps / (total_ms / 1e3), "unit": unit,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak" if args.workload == "gradient" else "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload,
                   "share_of_rank0": len(share_of_designs(designs, 0, world))
                   if args.workload == "sweep" else None},
        "clocks": clocks.summary(), "kernels": kernels,
    }  # fmt: skip
    if args.workload == "sweep":
        worst = 0.0
        for k, want in plain.items():
            for name in ("current", "rms_size", "rms_angle", "emittance"):
                ref = want[name]
                worst = max(worst, abs(result[k][name] - ref) / abs(ref) if ref else abs(result[k][name]))
        line["plain_form"] = fd_line
        line["speedup_over_plain"] = line["value"] / fd_line["value"]
        line["target_speedup"] = 20.0
        line["max_rel_moment_diff_vs_plain"] = worst
        line["iteration_mismatches"] = sum(result[k]["iterations"] != plain[k]["iterations"]
                                           for k in plain)  # fmt: skip
        if args.adjoint and world == 1:
            line["forward_plus_adjoint"] = sweep_with_gradients(designs, stream,
                                                                args.concurrency)
    if args.workload == "gradient":
        line["gradient"] = {k: [float(v) for v in result[k]] for k in ("rms_angle", "current")}
        line["adjoint_iterations"] = result["adjoint_iterations"]
        fd_angle = np.array(fd_line["rms_angle"])
        line["plain_form"] = fd_line
        line["speedup_over_plain"] = line["value"] / fd_line["value"]
        line["max_rel_diff_vs_plain"] = float(
            np.max(np.abs(np.array(line["gradient"]["rms_angle"]) - fd_angle))
            / np.max(np.abs(fd_angle)))  # fmt: skip
    print(json.dumps(line), flush=True)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="b200", choices=["b200", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-design", action="store_true",
                        help="leave out the design measurements of the default run")
    parser.add_argument("--window", type=int, default=64)
    parser.add_argument("--trace", default="exact", choices=["exact", "contracted"],
                        help="the trace's build: multiply-adds as written (bit-exact with the "
                             "oracle) or contracted into fused multiply-adds")
    parser.add_argument("--profile", action="store_true",
                        help="one warm solve, then one in the NVTX range 'profiled_solve'")
    parser.add_argument("--small", action="store_true",
                        help="with --profile: the lens at 401 x 101 with 2,000 rings")
    parser.add_argument("--profile-adjoint", action="store_true",
                        help="one warm adjoint gradient, then one in the NVTX range "
                             "'profiled_adjoint' (401 x 101, 2,000 rings)")
    parser.add_argument("--workload", default="einzel",
                        choices=["einzel", "plasma", "gradient", "sweep", "refined"],
                        help="plasma: the planar plasma + solenoid extraction (one GPU); "
                             "refined: the refined-box extraction (one GPU); "
                             "gradient: einzel design gradients; sweep: the design sweep")
    parser.add_argument("--sweep-count", type=int, default=32,
                        help="with --workload sweep: the candidates of one step")
    parser.add_argument("--adjoint", action="store_true",
                        help="with --workload sweep: also time the forward plus adjoint of "
                             "every candidate, batched and in the plain form")
    parser.add_argument("--concurrency", type=int, default=8,
                        help="with --workload sweep or gradient: solves at once per GPU")
    args = parser.parse_args()
    if args.profile_adjoint:
        run_profile_adjoint(args)
        return
    if args.profile:
        run_profile(args)
        return
    if args.workload == "plasma" and args.impl == "b200":
        run_plasma(args)
        return
    if args.workload == "refined" and args.impl == "b200":
        run_refined(args)
        return
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload in ("gradient", "sweep"):
        run_design(args, rank, world, local)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    distributed = world > 1
    if distributed:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))  # fmt: skip
    from beamtracer_b200 import _lib
    from beamtracer_b200.model import BeamOptics
    from beamtracer_b200.vlasov import vlasov_iterate

    config = build_workload(2 + rank)
    contracted = args.trace == "contracted"
    model = BeamOptics(config, contracted_trace=contracted)
    model.tracer.window = args.window
    from beamtracer_b200.poisson import IonOpticsPoisson

    poisson = IonOpticsPoisson(model.mesh, backend=config.field_backend)
    ctx = _lib.context()
    stream = torch.cuda.current_stream()

    def solve_once():
        return vlasov_iterate(model.mesh, model._particles, model.tracer,
                              iterations=config.iterations, tolerance=config.tolerance,
                              relaxation=config.relaxation, poisson=poisson)  # fmt: skip

    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        state = solve_once()
    torch.cuda.synchronize()
    iterations = len(state.history)
    ctx.set_timing(True)
    ctx.reset_timers()
    launches_before = ctx.launch_count()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]  # fmt: skip
    steps_total = 0
    if distributed:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))
            events[k][0].record(stream)
            state = solve_once()
            events[k][1].record(stream)
            steps_total += sum(h["total_steps"] for h in state.history)
        torch.cuda.synchronize()
    if distributed:
        dist.barrier()
    launches = ctx.launch_count() - launches_before
    records = ctx.deposit_records()
    step_ms = [a.elapsed_time(b) for a, b in events]
    total_ms = float(sum(step_ms))
    if distributed:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)
    timers = {name: ctx.read_timer(name) for name in
              ("trace_window", "deposit", "field_solve", "vcycle", "hierarchy", "edge_field",
               "vlasov_mix")}  # fmt: skip
    ctx.set_timing(False)
    history = state.history

    # the dominant kernel and its roofline
    kernels = {name: {"ms": ms, "launches": n, "share": ms / total_ms if total_ms else 0.0}
               for name, (ms, n) in timers.items()}  # fmt: skip
    trace_ms, trace_launches = timers["trace_window"]
    flops = FLOPS_PER_RK4_STEP * steps_total
    fp64_peak = ctx.fp64_peak()
    fp64 = {"bound": "fp64", "achieved": flops / (trace_ms / 1e3) / 1e12 if trace_ms else None,
            "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": (flops / (trace_ms / 1e3) / 1e12) / fp64_peak if trace_ms else None,
            "peak_source": "measured here: independent DFMA chains on every SM, CUDA events "
                           f"(nominal {NOMINAL_FP64_TFLOPS} TFLOP/s)",
            "kernel": "trace_window", "flops_per_step": FLOPS_PER_RK4_STEP,
            "steps_per_launch": steps_total / max(trace_launches, 1)}  # fmt: skip
    peaks = _peaks()
    dep_ms, dep_launches = timers["deposit"]
    dep_bytes = records * DEPOSIT_BYTES_PER_RECORD
    deposit = {"bound": "hbm", "kernel": "deposit",
               "achieved": dep_bytes / (dep_ms / 1e3) / 1e9 if dep_ms else None,
               "peak": peaks["hbm_gbs"], "unit": "GB/s",
               "frac": (dep_bytes / (dep_ms / 1e3) / 1e9) / peaks["hbm_gbs"] if dep_ms else None,
               "peak_source": peaks["source"], "records": records,
               "records_per_step": records / max(steps_total, 1),
               "traffic": None}  # fmt: skip
    # the dominant kernel, the trace: its algorithmic bytes are the deposit records it
    # writes (the edge fields it reads stay in L1/L2); its limit is the latency of its
    # dependent FP64 chain at one warp per scheduler (roofline_fp64)
    per_launch = TRACE_BYTES_PER_STEP * steps_total / max(trace_launches, 1)
    trace_gbs = per_launch / (trace_ms / max(trace_launches, 1) / 1e3) / 1e9 if trace_ms else None
    hbm = {"bound": "hbm", "kernel": "trace_window", "achieved": trace_gbs,
           "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": trace_gbs / peaks["hbm_gbs"] if trace_gbs else None,
           "peak_source": peaks["source"], "traffic": TRACE_DRAM_BYTES_PER_LAUNCH,
           "algorithmic_bytes_per_launch": per_launch,
           "limiter": "FP64 dependency latency at one warp per scheduler"}  # fmt: skip

    # end to end: the public call from host inputs to host results; one untimed call first
    # (its first-use allocations), then the median of E2E_RUNS calls (the host is shared,
    # so a single call can stall on it), each started from a collected heap
    e2e_ms = []
    h2d = d2h = 0
    for k in range(1 + E2E_RUNS):
        m = None
        gc.collect()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        m = BeamOptics(config, contracted_trace=contracted)
        m.run()
        moments = {f"{x * 1e3:g}mm": m.beam_moments(x) for x in config.diagnostic_planes}
        stop.record(stream)
        torch.cuda.synchronize()
        if k:
            e2e_ms.append(start.elapsed_time(stop))
        engine = m.tracer.engine()
        n = engine.n
        nn = m.mesh.shape[0] * m.mesh.shape[1]
        h2d = (nn * (1 + 8 + 32 + 4 + 1 + 8) + engine.cells.numel() * 8
               + engine.subcells.numel() * 8 + n * (48 + 16 + 24 + 8))  # fmt: skip
        d2h = (engine.counts.numel() * 8 + engine.hits.numel() * 8 + n * 24
               + engine.paths.numel() * 8 + 2 * nn * 8)  # fmt: skip
    e2e_value = world * 1e3 / float(np.median(e2e_ms))

    gpu_moments = {plane: {k: getattr(mo, k) for k in MOMENT_NAMES}
                   for plane, mo in moments.items()}  # fmt: skip
    design_lines = None
    if rank == 0 and world == 1 and not args.no_design:
        design_lines = design_measurements(stream)
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import kernels as oracle_kernels

        seconds, oracle_out, oracle_moments = oracle_solve(config)
        cpu = {"value": 1.0 / seconds, "unit": UNIT, "cores": oracle_kernels.host_cores(),
               "kind": "port",
               "sample": f"one converged solve of the same lens by the oracle "
                         f"({len(oracle_out['history'])} iterations: SciPy LU field, C trace "
                         f"and deposit with OpenMP), {seconds:.2f} s"}  # fmt: skip
        parity = parity_report(m.potential, gpu_moments, oracle_out, oracle_moments)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "solve": {"iterations_per_solve": len(history),
                  "vcycles_per_solve": sum(h["krylov_steps"] for h in history),
                  "window": args.window, "trace_build": args.trace},
        "roofline": hbm, "roofline_fp64": fp64, "roofline_deposit": deposit,
        "kernels": kernels,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms": float(np.median(e2e_ms)),
                "runs_ms": [round(v, 2) for v in e2e_ms]},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
        "moments": gpu_moments,
        "parity": parity,
        "design": design_lines,
    }  # fmt: skip
    if rank == 0:
        print(json.dumps(line), flush=True)
    if distributed:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
