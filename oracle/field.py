"""ORACLE (test infrastructure): the staggered edge field, restated in NumPy.

Restates ``solver/fields.py:18-67`` (``_edge_field``) and the two calls of
``StaggeredElectricField.__init__`` (``fields.py:116-152``): E_x on the (nx + 1, ny) edges
along x, E_y on the (nx, ny + 1) edges along y.  The same expressions in the same order, so
the same bits.
"""

from __future__ import annotations

import numpy as np


def _line_field(phi, solid, near, dist_lo, dist_hi, lengths, faces):
    """The edge field along axis 0 of (n, m) arrays; ``lengths`` the n - 1 edge lengths."""
    n = phi.shape[0]
    lengths = np.broadcast_to(np.asarray(lengths, dtype=float), (n - 1,))[:, None]
    before = np.ones_like(lengths)
    before[1:] = lengths[:-1]
    after = np.ones_like(lengths)
    after[:-1] = lengths[1:]
    a, b = phi[:-1], phi[1:]  # the nodes at either end of the interior edges
    sa, sb = solid[:-1], solid[1:]
    na, nb = near[:-1], near[1:]
    out = np.zeros((n + 1, phi.shape[1]))
    edge = (a - b) / lengths
    # a free node and its electrode neighbour: over the distance to the surface
    cut = na & sb
    edge[cut] = ((a - b) / (dist_hi[:-1] * lengths))[cut]
    cut = nb & sa
    edge[cut] = ((a - b) / (dist_lo[1:] * lengths))[cut]
    # both ends in an electrode: from the one surface beside the edge, if only one
    both = sa & sb
    if both.any():
        shape = a.shape
        near_prev = np.zeros(shape, dtype=bool)
        near_prev[1:] = near[:-2]
        near_next = np.zeros(shape, dtype=bool)
        near_next[:-1] = near[2:]
        phi_prev = np.zeros(shape)
        phi_prev[1:] = phi[:-2]
        phi_next = np.zeros(shape)
        phi_next[:-1] = phi[2:]
        d_prev = np.ones(shape)
        d_prev[1:] = dist_hi[:-2]
        d_next = np.ones(shape)
        d_next[:-1] = dist_lo[2:]
        inside = np.zeros(shape)
        one = near_prev & ~near_next
        inside[one] = ((phi_prev - a) / (d_prev * before))[one]
        one = near_next & ~near_prev
        inside[one] = ((b - phi_next) / (d_next * after))[one]
        edge[both] = inside[both]
    out[1:-1] = edge
    for end, first, second, face in ((0, 1, 2, faces[0]), (n, n - 1, n - 2, faces[1])):
        if face == "symmetric":
            out[end] = -out[first]
        else:
            out[end] = 2.0 * out[first] - out[second]
    return out


def edge_fields(phi, solid, near, distance, dx, h, extrapolation):
    """``(fx, fy)`` of the potential ``phi`` (nx, ny) on a mesh's classified nodes.

    ``solid`` the electrode index (or -1) per node, ``near`` the near-solid mask,
    ``distance`` (4, nx, ny), ``dx`` the x edge lengths, ``h`` the y spacing,
    ``extrapolation`` "extrapolate"/"symmetric" for x_min, x_max, y_min, y_max.
    """
    phi = np.asarray(phi, dtype=float)
    is_solid = np.asarray(solid) >= 0
    near = np.asarray(near, dtype=bool)
    fx = _line_field(phi, is_solid, near, distance[0], distance[1], dx, extrapolation[0:2])
    fy = _line_field(phi.T, is_solid.T, near.T, distance[2].T, distance[3].T, h,
                     extrapolation[2:4]).T  # fmt: skip
    return fx, np.ascontiguousarray(fy)


def surface_field(fx, fy, solid, near):
    """|E| at the free nodes next to an electrode and that electrode (``fields.py:324-377``):
    per axis the edge towards the solid neighbour, the larger with both solid, else the
    mean; NaN and -1 away from the electrodes."""
    solid = np.asarray(solid)
    nx, ny = solid.shape
    pad = np.pad(solid, 1, constant_values=-1)
    neighbours = [pad[0:nx, 1:ny + 1], pad[2:nx + 2, 1:ny + 1], pad[1:nx + 1, 0:ny],
                  pad[1:nx + 1, 2:ny + 2]]  # fmt: skip

    def component(low, high, solid_low, solid_high):
        larger = np.where(np.abs(low) >= np.abs(high), low, high)
        one = np.where(solid_low, low, np.where(solid_high, high, 0.5 * (low + high)))
        return np.where(solid_low & solid_high, larger, one)

    flags = [n >= 0 for n in neighbours]
    ex = component(fx[:-1], fx[1:], flags[0], flags[1])
    ey = component(fy[:, :-1], fy[:, 1:], flags[2], flags[3])
    near = np.asarray(near, dtype=bool)
    magnitude = np.where(near, np.hypot(ex, ey), np.nan)
    electrode = np.full(solid.shape, -1, dtype=np.int32)
    for n in neighbours:
        electrode = np.where(electrode < 0, n, electrode)
    return magnitude, np.where(near, electrode, -1).astype(np.int32)
