"""The reference's kernel plugin interface, on the B200.

``KERNELS[name](*args)`` takes the positional arguments of the reference kernel of the same
name (``kernels/catalog.py:39-44`` and the kernels' Pyccel signatures) and runs the CUDA
kernel of this package:

- ``staggered_field_2d(px, py, fx, fy, origin_x, origin_y, h, ex, ey)``
- ``deposit_trajectories_2d(px, py, q, origin_x, origin_y, h, cylindrical, charge)``
- ``trace_trajectories_2d(active, x, v, qm, dq, steps, status, electrode, fxs, fys,
  patch_int, patch_real, origin_x, origin_y, h, upper_x, upper_y, cylindrical, integrator,
  step_fraction, max_steps, cells, subcells, refine, planes, hits, counts, path_slot, paths,
  path_count, num_threads, charge, graded, x_nodes, inv_c2)``
- ``trace_trajectories_3d(active, x, v, qm, dq, steps, status, electrode, fxs, fys, fzs,
  patch_int, patch_real, bn, has_b, origin_x, origin_y, origin_z, h, upper_x, upper_y,
  upper_z, mirror_y, mirror_z, integrator, step_fraction, max_steps, cells, subcells,
  refine, planes, hits, counts, path_slot, paths, path_count, num_threads, charge, has_j,
  current, inv_c2)``

The arrays are written in place.  Device arrays (anything with
``__cuda_array_interface__``: torch CUDA tensors, CuPy arrays) are used where they lie, as
the reference runs its CUDA versions on CuPy arrays; NumPy arrays are copied to the device,
the kernel runs there, and the outputs are copied back.  There is no CPU version: without
a CUDA device a call raises.  Floating-point arrays are float64 and integer arrays int64,
C-contiguous.  As the reference's CUDA version, the trace deposits into ``charge[0]``
(``num_threads`` only sizes the host versions' slabs).
"""

from __future__ import annotations

import ctypes

import numpy as np

from beamtracer_b200 import _lib

_F8 = "<f8"
_I8 = "<i8"


def _check_device(array, typestr: str, name: str) -> None:
    iface = array.__cuda_array_interface__
    if iface["typestr"] != typestr:
        kind = "float64" if typestr == _F8 else "int64"
        raise TypeError(f"{name} must be {kind}, got {iface['typestr']}")
    strides = iface.get("strides")
    if strides is not None:
        shape = iface["shape"]
        expected, step = [], 8
        for extent in reversed(shape):
            expected.insert(0, step)
            step *= extent
        if tuple(strides) != tuple(expected) and int(np.prod(shape)) > 1:
            raise TypeError(f"{name} must be C-contiguous")


def _check_host(array: np.ndarray, dtype, name: str) -> None:
    if not isinstance(array, np.ndarray) or array.dtype != dtype:
        raise TypeError(f"{name} must be a {np.dtype(dtype).name} array")
    if not array.flags.c_contiguous:
        raise TypeError(f"{name} must be C-contiguous")


class _Staging:
    """Device copies of host arrays for one call, written back afterwards."""

    def __init__(self) -> None:
        import torch

        self.torch = torch
        self.back: list[tuple[np.ndarray, object]] = []

    def device(self, array, dtype, name: str, output: bool = False):
        if _lib.is_device_array(array):
            _check_device(array, _F8 if dtype == np.float64 else _I8, name)
            return array
        _check_host(array, dtype, name)
        tensor = self.torch.from_numpy(array).to("cuda", non_blocking=False)
        if output:
            self.back.append((array, tensor))
        return tensor

    def finish(self) -> None:
        for array, tensor in self.back:
            array[...] = tensor.cpu().numpy()


def _size(array) -> int:
    if _lib.is_device_array(array):
        return int(np.prod(array.__cuda_array_interface__["shape"]))
    return int(np.asarray(array).size)


def _shape(array) -> tuple:
    if _lib.is_device_array(array):
        return tuple(array.__cuda_array_interface__["shape"])
    return tuple(np.shape(array))


def staggered_field_2d(px, py, fx, fy, origin_x, origin_y, h, ex, ey) -> None:
    """``(E_x, E_y)`` at the points ``(px, py)`` from the edge fields ``fx``, ``fy``."""
    s = _Staging()
    px, py = s.device(px, np.float64, "px"), s.device(py, np.float64, "py")
    fx, fy = s.device(fx, np.float64, "fx"), s.device(fy, np.float64, "fy")
    ex = s.device(ex, np.float64, "ex", output=True)
    ey = s.device(ey, np.float64, "ey", output=True)
    nx, ny = _shape(fy)[0], _shape(fx)[1]
    n = _size(px)
    if not (_size(py) == _size(ex) == _size(ey) == n):
        raise ValueError("px, py, ex and ey need one entry per point")
    if _shape(fx) != (nx + 1, ny) or _shape(fy) != (nx, ny + 1):
        raise ValueError("fx must be (nx + 1, ny) and fy (nx, ny + 1)")
    ctx = _lib.context()
    _lib.check(
        _lib.lib().bt_staggered_field_2d(
            ctx.handle, _lib.dptr(px), _lib.dptr(py), n, _lib.dptr(fx), _lib.dptr(fy),
            nx, ny, float(origin_x), float(origin_y), float(h), _lib.dptr(ex),
            _lib.dptr(ey),
        )
    )  # fmt: skip
    s.finish()


def deposit_trajectories_2d(px, py, q, origin_x, origin_y, h, cylindrical, charge) -> None:
    """Add the charges ``q`` at ``(px, py)`` to the node charges ``charge``, area-weighted."""
    s = _Staging()
    px, py = s.device(px, np.float64, "px"), s.device(py, np.float64, "py")
    q = s.device(q, np.float64, "q")
    charge = s.device(charge, np.float64, "charge", output=True)
    nx, ny = _shape(charge)
    n = _size(px)
    if not (_size(py) == _size(q) == n):
        raise ValueError("px, py and q need one entry per charge")
    ctx = _lib.context()
    _lib.check(
        _lib.lib().bt_deposit_trajectories_2d(
            ctx.handle, _lib.dptr(px), _lib.dptr(py), _lib.dptr(q), n, float(origin_x),
            float(origin_y), float(h), int(cylindrical), _lib.dptr(charge), nx, ny,
        )
    )  # fmt: skip
    s.finish()


_TRACE_ARRAYS = {
    # name: (position, dtype, output)
    "active": (0, np.int64, False), "x": (1, np.float64, True), "v": (2, np.float64, True),
    "qm": (3, np.float64, False), "dq": (4, np.float64, False),
    "steps": (5, np.int64, True), "status": (6, np.int64, True),
    "electrode": (7, np.int64, True), "fxs": (8, np.float64, False),
    "fys": (9, np.float64, False), "patch_int": (10, np.int64, False),
    "patch_real": (11, np.float64, False), "cells": (21, np.int64, False),
    "subcells": (22, np.int64, False), "planes": (24, np.float64, False),
    "hits": (25, np.float64, True), "counts": (26, np.int64, True),
    "path_slot": (27, np.int64, False), "paths": (28, np.float64, True),
    "path_count": (29, np.int64, True), "charge": (31, np.float64, True),
    "x_nodes": (33, np.float64, False),
}  # fmt: skip


def trace_trajectories_2d(*args, window: int = 0, magnetic=None) -> None:
    """Trace the ``active`` trajectories until they end, or reach a cut electrode sub-cell.

    The 35 arguments of the reference kernel, in its order (see the module docstring);
    ``window`` is the number of steps a launch advances every trajectory (0: the library's
    default).  ``magnetic``, a `MagneticProfile` on the device, selects the reference's
    NumPy tracer's step in that field (``tracer.py:851-1054``): every step ending in a cell
    that touches an electrode then pauses (status -2) for the caller's inside test.
    """
    if len(args) != 35:
        raise TypeError(f"trace_trajectories_2d takes 35 arguments, got {len(args)}")
    s = _Staging()
    arrays = list(args)
    for name, (i, dtype, output) in _TRACE_ARRAYS.items():
        arrays[i] = s.device(args[i], dtype, name, output=output)
    (active, x, v, qm, dq, steps, status, electrode, fxs, fys, patch_int, patch_real,
     origin_x, origin_y, h, upper_x, upper_y, cylindrical, integrator, step_fraction,
     max_steps, cells, subcells, refine, planes, hits, counts, path_slot, paths,
     path_count, num_threads, charge, graded, x_nodes, inv_c2) = arrays  # fmt: skip
    n = _shape(x)[1]
    hits_shape = _shape(hits)
    charge_shape = _shape(charge)
    if _shape(x) != (3, n) or _shape(v) != (3, n):
        raise ValueError("x and v must be (3, n)")
    if len(hits_shape) != 4 or hits_shape[:2] != (n, _size(planes)) or hits_shape[3] != 8:
        raise ValueError("hits must be (n, planes, capacity, 8)")
    if len(charge_shape) != 2:
        raise ValueError("charge must be (threads, nodes)")
    a = _lib.TraceArgs(
        _lib.dptr(active), _size(active), _lib.dptr(x), _lib.dptr(v), n, _lib.dptr(qm),
        _lib.dptr(dq), _lib.dptr(steps), _lib.dptr(status), _lib.dptr(electrode),
        _lib.dptr(fxs), _lib.dptr(fys), _lib.dptr(patch_int), _lib.dptr(patch_real),
        _shape(patch_int)[0], float(origin_x), float(origin_y), float(h), float(upper_x),
        float(upper_y), int(cylindrical), int(integrator), float(step_fraction),
        int(max_steps), _lib.dptr(cells), _lib.dptr(subcells), int(refine),
        _lib.dptr(planes), _size(planes), _lib.dptr(hits), hits_shape[2],
        _lib.dptr(counts), _lib.dptr(path_slot), _lib.dptr(paths), _shape(paths)[1],
        _lib.dptr(path_count), int(num_threads), _lib.dptr(charge), charge_shape[1],
        int(graded), _lib.dptr(x_nodes), _size(x_nodes), float(inv_c2),
    )  # fmt: skip
    ctx = _lib.context()
    if magnetic is None:
        _lib.check(_lib.lib().bt_trace_trajectories_2d(ctx.handle, ctypes.byref(a), int(window)))
    else:
        m = magnetic.descriptor()
        _lib.check(_lib.lib().bt_trace_trajectories_2d_magnetic(
            ctx.handle, ctypes.byref(a), ctypes.byref(m), int(window)))  # fmt: skip
    s.finish()


_TRACE3D_ARRAYS = {
    # name: (position, dtype, output)
    "active": (0, np.int64, False), "x": (1, np.float64, True), "v": (2, np.float64, True),
    "qm": (3, np.float64, False), "dq": (4, np.float64, False),
    "steps": (5, np.int64, True), "status": (6, np.int64, True),
    "electrode": (7, np.int64, True), "fxs": (8, np.float64, False),
    "fys": (9, np.float64, False), "fzs": (10, np.float64, False),
    "patch_int": (11, np.int64, False), "patch_real": (12, np.float64, False),
    "bn": (13, np.float64, False), "cells": (27, np.int64, False),
    "subcells": (28, np.int64, False), "planes": (30, np.float64, False),
    "hits": (31, np.float64, True), "counts": (32, np.int64, True),
    "path_slot": (33, np.int64, False), "paths": (34, np.float64, True),
    "path_count": (35, np.int64, True), "charge": (37, np.float64, True),
    "current": (39, np.float64, True),
}  # fmt: skip


def trace_trajectories_3d(*args, window: int = 0) -> None:
    """Trace the ``active`` trajectories of a 3D mesh until they end, or reach a cut
    electrode sub-cell (status -2): the 41 arguments of the reference kernel
    (``trace_trajectories_3d_pyccel.py:19-61``), in its order; ``window`` is the number of
    steps a launch advances every trajectory (0: the library's default).  The space charge
    goes to ``charge[0]``, the current elements (``has_j``) to ``current[0]``."""
    if len(args) != 41:
        raise TypeError(f"trace_trajectories_3d takes 41 arguments, got {len(args)}")
    s = _Staging()
    arrays = list(args)
    for name, (i, dtype, output) in _TRACE3D_ARRAYS.items():
        arrays[i] = s.device(args[i], dtype, name, output=output)
    (active, x, v, qm, dq, steps, status, electrode, fxs, fys, fzs, patch_int, patch_real, bn,
     has_b, origin_x, origin_y, origin_z, h, upper_x, upper_y, upper_z, mirror_y, mirror_z,
     integrator, step_fraction, max_steps, cells, subcells, refine, planes, hits, counts,
     path_slot, paths, path_count, num_threads, charge, has_j, current, inv_c2) = arrays  # fmt: skip
    n = _shape(x)[1]
    hits_shape = _shape(hits)
    if _shape(x) != (3, n) or _shape(v) != (3, n):
        raise ValueError("x and v must be (3, n)")
    if len(hits_shape) != 4 or hits_shape[:2] != (n, _size(planes)) or hits_shape[3] != 8:
        raise ValueError("hits must be (n, planes, capacity, 8)")
    if len(_shape(charge)) != 2 or len(_shape(patch_int)) != 2 or _shape(patch_int)[1] != 8:
        raise ValueError("charge must be (threads, nodes) and patch_int (patches, 8)")
    if len(_shape(paths)) != 3 or _shape(paths)[2] != 3:
        raise ValueError("paths must be (slots, capacity, 3)")
    a = _lib.Trace3DArgs(
        _lib.dptr(active), _size(active), _lib.dptr(x), _lib.dptr(v), n, _lib.dptr(qm),
        _lib.dptr(dq), _lib.dptr(steps), _lib.dptr(status), _lib.dptr(electrode),
        _lib.dptr(fxs), _lib.dptr(fys), _lib.dptr(fzs), _lib.dptr(patch_int),
        _lib.dptr(patch_real), _shape(patch_int)[0], _lib.dptr(bn), int(has_b),
        float(origin_x), float(origin_y), float(origin_z), float(h), float(upper_x),
        float(upper_y), float(upper_z), int(mirror_y), int(mirror_z), int(integrator),
        float(step_fraction), int(max_steps), _lib.dptr(cells), _lib.dptr(subcells),
        int(refine), _lib.dptr(planes), _size(planes), _lib.dptr(hits), hits_shape[2],
        _lib.dptr(counts), _lib.dptr(path_slot), _lib.dptr(paths), _shape(paths)[1],
        _lib.dptr(path_count), int(num_threads), _lib.dptr(charge), _shape(charge)[1],
        int(has_j), _lib.dptr(current), float(inv_c2),
    )  # fmt: skip
    ctx = _lib.context()
    _lib.check(_lib.lib().bt_trace_trajectories_3d(ctx.handle, ctypes.byref(a), int(window)))
    s.finish()


def last_trace_stats() -> dict[str, int]:
    """Windows, deposit records and deposit flushes of the calling thread's last trace."""
    windows, records, flushes = _lib.I64(), _lib.I64(), _lib.I64()
    ctx = _lib.context()
    _lib.check(
        _lib.lib().bt_trace_last_stats(
            ctx.handle, ctypes.byref(windows), ctypes.byref(records), ctypes.byref(flushes)
        )
    )
    return {"windows": windows.value, "records": records.value, "flushes": flushes.value}


#: The kernels by name, as the reference's ``KERNELS`` catalogue.
KERNELS = {
    "staggered_field_2d": staggered_field_2d,
    "deposit_trajectories_2d": deposit_trajectories_2d,
    "trace_trajectories_2d": trace_trajectories_2d,
    "trace_trajectories_3d": trace_trajectories_3d,
}
KERNEL_NAMES = tuple(KERNELS)
