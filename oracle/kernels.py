"""ORACLE (test infrastructure): the reference's three cunumpy kernels, restated in C.

Each function takes the positional arguments of the reference kernel of the same name
(NumPy arrays, written in place) and runs the C restatement in ``bt_oracle.c``:

- ``staggered_field_2d(px, py, fx, fy, origin_x, origin_y, h, ex, ey)``
  (``kernels/staggered_field_2d/staggered_field_2d_pyccel.py:13-55``)
- ``deposit_trajectories_2d(px, py, q, origin_x, origin_y, h, cylindrical, charge)``
  (``kernels/deposit_trajectories_2d/deposit_trajectories_2d_pyccel.py:13-59``)
- ``trace_trajectories_2d(active, x, v, qm, dq, steps, status, electrode, fxs, fys,
  patch_int, patch_real, origin_x, origin_y, h, upper_x, upper_y, cylindrical, integrator,
  step_fraction, max_steps, cells, subcells, refine, planes, hits, counts, path_slot,
  paths, path_count, num_threads, charge, graded, x_nodes, inv_c2)``
  (``kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:42-507``)
"""

from __future__ import annotations

import ctypes
import functools

import numpy as np

from oracle.build import build

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_int64)
_I64 = ctypes.c_int64
_F64 = ctypes.c_double


class _TraceArgs(ctypes.Structure):
    _fields_ = [
        ("active", _L), ("n_active", _I64), ("x", _D), ("v", _D), ("n", _I64),
        ("qm", _D), ("dq", _D), ("steps", _L), ("status", _L), ("electrode", _L),
        ("fxs", _D), ("fys", _D), ("patch_int", _L), ("patch_real", _D),
        ("n_patches", _I64), ("origin_x", _F64), ("origin_y", _F64), ("h", _F64),
        ("upper_x", _F64), ("upper_y", _F64), ("cylindrical", _I64),
        ("integrator", _I64), ("step_fraction", _F64), ("max_steps", _I64),
        ("cells", _L), ("subcells", _L), ("refine", _I64), ("planes", _D),
        ("n_planes", _I64), ("hits", _D), ("capacity", _I64), ("counts", _L),
        ("path_slot", _L), ("paths", _D), ("path_capacity", _I64), ("path_count", _L),
        ("num_threads", _I64), ("charge", _D), ("n_nodes", _I64), ("graded", _I64),
        ("x_nodes", _D), ("n_x_nodes", _I64), ("inv_c2", _F64),
    ]  # fmt: skip


class _Magnetic(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("order", ctypes.c_int32), ("n", _I64), ("z0", _F64),
        ("hz", _F64), ("axis_y", _F64), ("samples", _D),
    ]  # fmt: skip


@functools.cache
def library() -> ctypes.CDLL:
    """The compiled oracle (built on first use)."""
    lib = ctypes.CDLL(str(build()))
    lib.bto_staggered_field_2d.argtypes = [
        _D, _D, _I64, _D, _D, _I64, _I64, _F64, _F64, _F64, _D, _D,
    ]
    lib.bto_deposit_trajectories_2d.argtypes = [
        _D, _D, _D, _I64, _F64, _F64, _F64, _I64, _D, _I64, _I64,
    ]
    lib.bto_trace_trajectories_2d.argtypes = [ctypes.POINTER(_TraceArgs)]
    lib.bto_trace_magnetic_2d.argtypes = [ctypes.POINTER(_TraceArgs), ctypes.POINTER(_Magnetic)]
    lib.bto_num_procs.restype = ctypes.c_int
    return lib


def _f64(a: np.ndarray, name: str) -> np.ndarray:
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous float64 array")
    return a


def _i64(a: np.ndarray, name: str) -> np.ndarray:
    if a.dtype != np.int64 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous int64 array")
    return a


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D if a.dtype == np.float64 else _L)


def staggered_field_2d(px, py, fx, fy, origin_x, origin_y, h, ex, ey) -> None:
    """``(E_x, E_y)`` at the points from the edge fields (restated Pyccel kernel)."""
    arrays = [_f64(a, n) for a, n in zip((px, py, fx, fy, ex, ey), "px py fx fy ex ey".split())]
    px, py, fx, fy, ex, ey = arrays
    nx, ny = fy.shape[0], fx.shape[1]
    library().bto_staggered_field_2d(
        _p(px), _p(py), px.size, _p(fx), _p(fy), nx, ny,
        float(origin_x), float(origin_y), float(h), _p(ex), _p(ey),
    )  # fmt: skip


def deposit_trajectories_2d(px, py, q, origin_x, origin_y, h, cylindrical, charge) -> None:
    """Add the charges ``q`` at ``(px, py)`` to ``charge`` (restated Pyccel kernel)."""
    for a, n in ((px, "px"), (py, "py"), (q, "q"), (charge, "charge")):
        _f64(a, n)
    nx, ny = charge.shape
    library().bto_deposit_trajectories_2d(
        _p(px), _p(py), _p(q), px.size, float(origin_x), float(origin_y), float(h),
        int(cylindrical), _p(charge), nx, ny,
    )  # fmt: skip


def trace_trajectories_2d(
    active, x, v, qm, dq, steps, status, electrode, fxs, fys, patch_int, patch_real,
    origin_x, origin_y, h, upper_x, upper_y, cylindrical, integrator, step_fraction,
    max_steps, cells, subcells, refine, planes, hits, counts, path_slot, paths,
    path_count, num_threads, charge, graded, x_nodes, inv_c2, magnetic=None,
) -> None:  # fmt: skip
    """Trace the ``active`` trajectories to their ends (restated Pyccel kernel).

    With ``magnetic = (mode, order, z0, hz, axis_y, samples)`` the step is the reference's
    NumPy tracer's in that field instead (``tracer.py:851-1054``): acceleration
    ``q/m (E + v x B)``, Boris with the magnetic rotation, and every step ending in a cell
    that touches an electrode pauses (status -2) for the caller's exact inside test.
    """
    for a, n in ((active, "active"), (steps, "steps"), (status, "status"),
                 (electrode, "electrode"), (patch_int, "patch_int"), (cells, "cells"),
                 (subcells, "subcells"), (counts, "counts"), (path_slot, "path_slot"),
                 (path_count, "path_count")):  # fmt: skip
        _i64(a, n)
    for a, n in ((x, "x"), (v, "v"), (qm, "qm"), (dq, "dq"), (fxs, "fxs"), (fys, "fys"),
                 (patch_real, "patch_real"), (planes, "planes"), (hits, "hits"),
                 (paths, "paths"), (charge, "charge"), (x_nodes, "x_nodes")):  # fmt: skip
        _f64(a, n)
    args = _TraceArgs(
        _p(active), active.size, _p(x), _p(v), x.shape[1], _p(qm), _p(dq), _p(steps),
        _p(status), _p(electrode), _p(fxs), _p(fys), _p(patch_int), _p(patch_real),
        patch_int.shape[0], float(origin_x), float(origin_y), float(h), float(upper_x),
        float(upper_y), int(cylindrical), int(integrator), float(step_fraction),
        int(max_steps), _p(cells), _p(subcells), int(refine), _p(planes), planes.size,
        _p(hits), hits.shape[2], _p(counts), _p(path_slot), _p(paths), paths.shape[1],
        _p(path_count), int(num_threads), _p(charge), charge.shape[1], int(graded),
        _p(x_nodes), x_nodes.size, float(inv_c2),
    )  # fmt: skip
    if charge.shape[0] < int(num_threads):
        raise ValueError("charge needs one slab per thread")
    if magnetic is None:
        library().bto_trace_trajectories_2d(ctypes.byref(args))
        return
    mode, order, z0, hz, axis_y, samples = magnetic
    samples = _f64(np.ascontiguousarray(samples, dtype=np.float64), "samples")
    if samples.ndim != 2 or samples.shape[1] != int(order) + 1 or samples.shape[0] < 8:
        raise ValueError("samples must be (n >= 8, order + 1)")
    if float(inv_c2) != 0.0 or patch_int.shape[0] != 1:
        raise ValueError("the magnetic trace is non-relativistic on one patch")
    mag = _Magnetic(int(mode), int(order), samples.shape[0], float(z0), float(hz),
                    float(axis_y), _p(samples))  # fmt: skip
    library().bto_trace_magnetic_2d(ctypes.byref(args), ctypes.byref(mag))


def host_cores() -> int:
    """The host cores OpenMP sees."""
    return int(library().bto_num_procs())
