"""The configuration's electrode shapes as device tables (``bt_shapes``): the inside tests
of ``config.ObjectParams`` (rectangles, lines, circles, polygons, triangles, mirrored
apertures) with every parameter the device test reads computed here, in the host test's
expressions, so the device's answers are the host's."""

from __future__ import annotations

from typing import Any

import numpy as np


def _polygon_words(vertices: np.ndarray) -> list[float]:
    """A polygon for the device's inside test: its edge count, then per edge its ends, the
    boundary threshold and the extent the host's test uses (``config._polygon_inside``)."""
    vx, vy = vertices[:, 0], vertices[:, 1]
    n = len(vx)
    words = [float(n)]
    for k in range(n):
        x1, y1, x2, y2 = vx[k], vy[k], vx[(k + 1) % n], vy[(k + 1) % n]
        length = np.hypot(x2 - x1, y2 - y1)
        threshold = 1e-12 * max(length, 1e-300) * max(length, 1.0)
        words += [x1, y1, x2, y2, threshold, min(x1, x2) - 1e-15, max(x1, x2) + 1e-15,
                  min(y1, y2) - 1e-15, max(y1, y2) + 1e-15]  # fmt: skip
    return [float(w) for w in words]


def shape_table(mesh: Any):
    """The electrodes as device shapes ``(kind, offset, params)`` arrays, or None when one
    is not a configuration shape (an arbitrary inside function: tested on the host)."""
    from beamtracer_b200.config import ObjectParams

    kinds, offsets, params = [], [], []
    for electrode in mesh.electrodes:
        obj = getattr(electrode.inside, "__self__", None)
        if not isinstance(obj, ObjectParams):
            return None
        offsets.append(len(params))
        if obj.type in ("rectangle", "line"):
            (mx, my), (lx, ly) = obj.midpoint, obj.side_lengths
            kinds.append(0)
            params += [float(mx), float(my), 0.5 * lx, 0.5 * ly]
        elif obj.type == "circle":
            mx, my = obj.midpoint
            kinds.append(1)
            params += [float(mx), float(my), float(obj.radius) ** 2]
        else:
            vertices = np.asarray(obj.vertices, dtype=float)
            if obj.type in ("polygon", "triangle"):
                kinds.append(2)
                params += _polygon_words(vertices)
            else:
                axis = int(obj.axis) if obj.axis is not None else 0
                position = float(obj.position or 0.0)
                mirrored = vertices.copy()
                mirrored[:, 1 - axis] = 2.0 * position - mirrored[:, 1 - axis]
                kinds.append(3)
                params += _polygon_words(vertices) + _polygon_words(mirrored)
    return (np.array(kinds, dtype=np.int32), np.array(offsets, dtype=np.int64),
            np.array(params or [0.0], dtype=np.float64))  # fmt: skip
