"""Loading the CUDA library ``libbt200.so`` and calling its C ABI through ctypes.

The library is built in-tree (`beamtracer_b200.build`).  There is no fallback: without the
library, or without a CUDA device, every call raises.
"""

from __future__ import annotations

import ctypes
import functools
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libbt200.so"

BT_OK = 0
BT_ERR_ARG = -1
BT_ERR_CUDA = -2
BT_ERR_CAPACITY = -3
BT_ERR_NOCONV = -4
BT_ERR_TIMEOUT = -5
BT_ERR_ALLOC = -6

P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int32
F64 = ctypes.c_double


class BTError(RuntimeError):
    """A failure reported by the CUDA library."""

    def __init__(self, code: int, message: str) -> None:
        super().__init__(f"{message} (code {code})")
        self.code = code


class CapacityError(BTError):
    """An output buffer was too small."""


class ConvergenceError(BTError):
    """An iterative solve did not converge."""


class TraceArgs(ctypes.Structure):
    """``bt_trace_args`` of ``include/bt200.h``."""

    _fields_ = [
        ("active", P), ("n_active", I64), ("x", P), ("v", P), ("n", I64),
        ("qm", P), ("dq", P), ("steps", P), ("status", P), ("electrode", P),
        ("fxs", P), ("fys", P), ("patch_int", P), ("patch_real", P),
        ("n_patches", I64), ("origin_x", F64), ("origin_y", F64), ("h", F64),
        ("upper_x", F64), ("upper_y", F64), ("cylindrical", I64),
        ("integrator", I64), ("step_fraction", F64), ("max_steps", I64),
        ("cells", P), ("subcells", P), ("refine", I64), ("planes", P),
        ("n_planes", I64), ("hits", P), ("capacity", I64), ("counts", P),
        ("path_slot", P), ("paths", P), ("path_capacity", I64), ("path_count", P),
        ("num_threads", I64), ("charge", P), ("n_nodes", I64), ("graded", I64),
        ("x_nodes", P), ("n_x_nodes", I64), ("inv_c2", F64),
    ]  # fmt: skip


class Trace3DArgs(ctypes.Structure):
    """``bt_trace3d_args`` of ``include/bt200.h``."""

    _fields_ = [
        ("active", P), ("n_active", I64), ("x", P), ("v", P), ("n", I64), ("qm", P),
        ("dq", P), ("steps", P), ("status", P), ("electrode", P), ("fxs", P), ("fys", P),
        ("fzs", P), ("patch_int", P), ("patch_real", P), ("n_patches", I64), ("bn", P),
        ("has_b", I64), ("origin_x", F64), ("origin_y", F64), ("origin_z", F64), ("h", F64),
        ("upper_x", F64), ("upper_y", F64), ("upper_z", F64), ("mirror_y", I64),
        ("mirror_z", I64), ("integrator", I64), ("step_fraction", F64), ("max_steps", I64),
        ("cells", P), ("subcells", P), ("refine", I64), ("planes", P), ("n_planes", I64),
        ("hits", P), ("capacity", I64), ("counts", P), ("path_slot", P), ("paths", P),
        ("path_capacity", I64), ("path_count", P), ("num_threads", I64), ("charge", P),
        ("n_nodes", I64), ("has_j", I64), ("current", P), ("inv_c2", F64),
    ]  # fmt: skip


class TraceBatch(ctypes.Structure):
    """``bt_trace_batch`` of ``include/bt200.h``."""

    _fields_ = [
        ("n_candidates", I64), ("candidate", P), ("cell_offset", P), ("group", I64),
        ("shape_first", P), ("shape_kind", P), ("shape_offset", P), ("shape_params", P),
    ]  # fmt: skip


class MagneticDesc(ctypes.Structure):
    """``bt_magnetic`` of ``include/bt200.h``."""

    _fields_ = [
        ("mode", I32), ("order", I32), ("n", I64), ("z0", F64), ("hz", F64),
        ("axis_y", F64), ("samples", P),
    ]  # fmt: skip


class ShapesDesc(ctypes.Structure):
    """``bt_shapes`` of ``include/bt200.h``."""

    _fields_ = [("count", I64), ("kind", P), ("offset", P), ("params", P)]


class AdjointArgs(ctypes.Structure):
    """``bt_adjoint_args`` of ``include/bt200.h``."""

    _fields_ = [
        ("x0", P), ("v0", P), ("qm", P), ("dq", P), ("steps", P), ("n", I64), ("fx", P),
        ("fy", P), ("nx", I64), ("ny", I64), ("origin_x", F64), ("origin_y", F64), ("h", F64),
        ("cylindrical", I64), ("step_fraction", F64), ("planes", P), ("n_planes", I64),
        ("counts", P), ("capacity", I64), ("checkpoints", P), ("segments", I64),
    ]  # fmt: skip


class MeshDesc(ctypes.Structure):
    """``bt_mesh_desc`` of ``include/bt200.h``."""

    _fields_ = [
        ("nx", I64), ("ny", I64), ("h", F64), ("x", P), ("origin_y", F64),
        ("cylindrical", I32), ("fixed", P), ("fixed_value", P), ("distance", P),
        ("neumann", P),
    ]  # fmt: skip


#: Every symbol the C ABI exports (``include/bt200.h``), with its argument types.
SIGNATURES: dict[str, list] = {
    "bt_ctx_create": [I32, ctypes.POINTER(P)],
    "bt_ctx_destroy": [P],
    "bt_ctx_set_stream": [P, P],
    "bt_ctx_synchronize": [P],
    "bt_ctx_set_timing": [P, I32],
    "bt_ctx_read_timer": [P, ctypes.c_char_p, ctypes.POINTER(F64), ctypes.POINTER(I64)],
    "bt_ctx_reset_timers": [P],
    "bt_ctx_launch_count": [P, ctypes.POINTER(I64)],
    "bt_ctx_deposit_records": [P, ctypes.POINTER(I64)],
    "bt_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "bt_version": [],
    "bt_staggered_field_2d": [P, P, P, I64, P, P, I64, I64, F64, F64, F64, P, P],
    "bt_deposit_trajectories_2d": [P, P, P, P, I64, F64, F64, F64, I64, P, I64, I64],
    "bt_deposit_trajectories_2d_noalloc": [P, P, P, P, I64, F64, F64, F64, I64, P, I64, I64],
    "bt_classify_mesh": [P, ctypes.POINTER(ShapesDesc), I64, I64, P, P, F64, F64, P, P, P],
    "bt_subcell_table": [P, ctypes.POINTER(ShapesDesc), P, P, I64, F64, F64, F64, P, I64, I64,
                         P],
    "bt_trace_trajectories_2d_magnetic": [P, ctypes.POINTER(TraceArgs),
                                          ctypes.POINTER(MagneticDesc), I64],
    "bt_trace_trajectories_2d": [P, ctypes.POINTER(TraceArgs), I64],
    "bt_trace_trajectories_2d_fast": [P, ctypes.POINTER(TraceArgs), I64],
    "bt_trace_trajectories_2d_magnetic_fast": [P, ctypes.POINTER(TraceArgs),
                                               ctypes.POINTER(MagneticDesc), I64],
    "bt_trace_trajectories_2d_batch": [P, ctypes.POINTER(TraceArgs),
                                       ctypes.POINTER(TraceBatch), I64],
    "bt_trace_trajectories_2d_batch_fast": [P, ctypes.POINTER(TraceArgs),
                                            ctypes.POINTER(TraceBatch), I64],
    "bt_trace_trajectories_3d": [P, ctypes.POINTER(Trace3DArgs), I64],
    "bt_measure_fp64_peak": [P, ctypes.POINTER(F64)],
    "bt_trace_last_stats": [P, ctypes.POINTER(I64), ctypes.POINTER(I64), ctypes.POINTER(I64)],
    "bt_edge_field": [P, P, P, P, P, P, I64, I64, F64, P, P, P],
    "bt_edge_field_adjoint": [P, P, P, P, P, P, P, I64, I64, F64, P, P],
    "bt_edge_field_3d": [P, P, P, P, P, I64, I64, I64, F64, P, P, P, P],
    "bt_surface_field": [P, P, P, P, P, I64, I64, I32, P, P, P],
    "bt_adjoint_checkpoints": [P, ctypes.POINTER(AdjointArgs), P],
    "bt_adjoint_sweep": [P, ctypes.POINTER(AdjointArgs), P, P, P, P],
    "bt_poisson_set_transposed": [P, I32],
    "bt_poisson_fixed_adjoint": [P, P, P, P],
    "bt_poisson_residual": [P, P, P, P],
    "bt_csr_apply": [P, I64, P, P, P, P, P, I32, P, P],
    "bt_poisson_solve_reaction": [P, P, P, P, F64, ctypes.POINTER(I32)],
    "bt_boltzmann_terms": [P, I64, P, P, F64, F64, F64, I32, P, P],
    "bt_newton_residual": [P, I64, P, P, P, P, P],
    "bt_poisson_vcycle": [P, P, P, I32, P],
    "bt_vlasov_mix": [P, P, P, P, I64, I64, F64, I32, P, P],
    "bt_max_abs_diff": [P, P, P, I64, P],
    "bt_anderson_mix": [P, P, P, P, I64, I64, I32, I32, I32, F64, P, P, P, P, P],
    "bt_poisson_create": [P, ctypes.POINTER(MeshDesc), ctypes.POINTER(P)],
    "bt_poisson_destroy": [P],
    "bt_poisson_set_region": [P, P, F64],
    "bt_poisson_set_options": [P, I32, I32, I32, I64],
    "bt_poisson_set_context": [P, P],
    "bt_poisson_batch_create": [P, P, I64, P, ctypes.POINTER(P)],
    "bt_poisson_batch_destroy": [P],
    "bt_poisson_batch_solve": [P, P, P, P, F64, I32, P, P],
    "bt_poisson_batch_tiling": [P, I32, P],
    "bt_poisson_solve": [
        P, P, P, F64, F64, F64, I32, F64, F64, I32,
        ctypes.POINTER(I32), ctypes.POINTER(I32),
    ],  # fmt: skip
}


@functools.cache
def lib() -> ctypes.CDLL:
    """The loaded library (built first if missing and nvcc is available)."""
    if not LIBRARY.exists():
        from beamtracer_b200.build import build

        build()
    handle = ctypes.CDLL(str(LIBRARY))
    for name, args in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    handle.bt_last_error.restype = ctypes.c_size_t
    handle.bt_version.restype = ctypes.c_char_p
    return handle


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib().bt_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    """Raise the error of a failed call."""
    if code == BT_OK:
        return
    message = last_error()
    if code == BT_ERR_ARG:
        raise ValueError(message)
    if code == BT_ERR_CAPACITY:
        raise CapacityError(code, message)
    if code == BT_ERR_NOCONV:
        raise ConvergenceError(code, message)
    raise BTError(code, message)


class Context:
    """A library context on one CUDA device (its own stream unless told otherwise)."""

    def __init__(self, device: int = 0) -> None:
        self.device = int(device)
        handle = P()
        check(lib().bt_ctx_create(self.device, ctypes.byref(handle)))
        self.handle = handle

    def use_stream(self, stream: int) -> None:
        """Queue work on ``stream`` (a ``cudaStream_t`` as an int; 0: CUDA's default stream,
        which is torch's default stream)."""
        check(lib().bt_ctx_set_stream(self.handle, P(stream) if stream else None))

    def set_timing(self, on: bool) -> None:
        """Record the launch times of the library's kernels (CUDA events on its stream)."""
        check(lib().bt_ctx_set_timing(self.handle, int(bool(on))))

    def read_timer(self, name: str) -> tuple[float, int]:
        """The summed launch time [ms] and the launches of a timed kernel since the reset."""
        ms, count = F64(), I64()
        check(lib().bt_ctx_read_timer(self.handle, name.encode(), ctypes.byref(ms),
                                      ctypes.byref(count)))  # fmt: skip
        return ms.value, count.value

    def launch_count(self) -> int:
        """The kernels this context has launched since its creation."""
        count = I64()
        check(lib().bt_ctx_launch_count(self.handle, ctypes.byref(count)))
        return count.value

    def deposit_records(self) -> int:
        """The records the deposits reduced while timing was on, since the last reset."""
        count = I64()
        check(lib().bt_ctx_deposit_records(self.handle, ctypes.byref(count)))
        return count.value

    def fp64_peak(self) -> float:
        """The FP64 pipe's measured peak [TFLOP/s] on this context's device."""
        value = F64()
        check(lib().bt_measure_fp64_peak(self.handle, ctypes.byref(value)))
        return value.value

    def reset_timers(self) -> None:
        check(lib().bt_ctx_reset_timers(self.handle))

    def synchronize(self) -> None:
        check(lib().bt_ctx_synchronize(self.handle))

    def close(self) -> None:
        if self.handle:
            lib().bt_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_local = threading.local()


def context(device: int | None = None) -> Context:
    """The calling thread's context on ``device`` (default: torch's current device).

    Its work runs on torch's current stream, so it is ordered with torch's own.
    """
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("beamtracer_b200 needs a CUDA device")
    if device is None:
        device = torch.cuda.current_device()
    contexts = getattr(_local, "contexts", None)
    if contexts is None:
        contexts = _local.contexts = {}
    ctx = contexts.get(device)
    if ctx is None:
        ctx = contexts[device] = Context(device)
    ctx.use_stream(torch.cuda.current_stream(device).cuda_stream)
    return ctx


def exported_symbols() -> list[str]:
    """The names the C ABI must export."""
    return list(SIGNATURES)


def dptr(array) -> int:
    """The device address of a CUDA array (``__cuda_array_interface__``), 0 for None."""
    if array is None:
        return 0
    return int(array.__cuda_array_interface__["data"][0])


def is_device_array(array) -> bool:
    return hasattr(array, "__cuda_array_interface__")


def np_ptr(array: np.ndarray | None) -> int:
    return 0 if array is None else int(array.ctypes.data)
