"""Refined boxes of a 2D mesh: their patches and the composite nodes (host side).

The interface of the reference's ``solver/refinement.py:23-387`` (`Refinement`, `Patch`,
`patches_of`, `Layout`): a box of finer cells halves the cells of the level below once per
level; every patch, the base mesh included, is a uniform `IonOpticsMesh` of its own (its
electrodes classified at its spacing), and a refined patch's field is taken on a mesh two
of its cells wider on every side inside the domain (`Patch.field_mesh`).  patchwork, which
builds the reference's composite mesh, is not in this container; the composite nodes here
are built from their definition:

- the composite nodes are the nodes of every patch, identified on the lattice of the
  finest level, numbered in the order of ``(i, j)`` on that lattice (x major);
- a leaf cell is a cell of a level that no box of the next level covers; a node's control
  volume is a quarter of every leaf cell it is a corner of (of the cell's ring volume
  ``2 pi r_c |K|`` in cylindrical geometry), the volumes ``solver/refinement.py:160-163``
  describes;
- a node belongs to a patch's *inside* unless it lies on a side of the patch's box that is
  not a face of the domain; the *owner* of a node is the finest patch whose inside holds
  it, and its equation is that patch's row of the field operator;
- a node no patch's inside holds is *hanging*: it lies on a coarse cell's edge, and its
  value is the linear interpolation of the edge's two ends (recursively, where an end
  hangs itself).

Boxes of a level must lie inside the boxes of the level below (nested).  Along a graded x
axis a box is placed in the uniform coordinate of the node indices, and a level's nodes lie
evenly between the base nodes (``solver/refinement.py:60-82``).
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass, field
from typing import Any

import numpy as np
from scipy import sparse

from beamtracer_b200.mesh import IonOpticsMesh


@dataclass(frozen=True)
class Refinement:
    """A box ``lower``-``upper`` [m] (``(x, y)`` corners) refined to ``level`` (>= 1)."""

    level: int
    lower: tuple[float, ...]
    upper: tuple[float, ...]


@dataclass
class Patch:
    """A uniform part of the composite mesh (``solver/refinement.py:32-57``).

    ``box`` is ``((i0, i1), (j0, j1))``: the patch's first and last node along ``x`` and
    ``y`` in its level's node indices; ``index`` the composite node of every node of
    ``mesh`` (set by `layout_of`); ``field_mesh`` the mesh of the patch's field (two of its
    cells wider on every side inside the domain; None for the base), ``inner`` the box's
    nodes in it.
    """

    level: int
    box: tuple[tuple[int, int], tuple[int, int]]
    mesh: IonOpticsMesh
    index: np.ndarray | None = None
    field_mesh: IonOpticsMesh | None = None
    inner: tuple[slice, slice] = (slice(None), slice(None))

    @property
    def bounds(self) -> tuple[float, float, float, float]:
        """The patch's node extent ``(x_lower, y_lower, x_upper, y_upper)`` [m]."""
        (x0, y0), (x1, y1) = self.mesh.origin, self.mesh.upper
        return x0, y0, x1, y1


def _parent_span(lower: float, upper: float, start: float, end: float, step: float,
                 cells: int) -> tuple[int, int]:
    """The parent level's cells ``[c0, c1]`` a box side ``[lower, upper]`` widens to."""
    lo = (max(start, lower) - start) / step
    hi = (min(end, upper) - start) / step
    c0 = max(int(np.floor(lo + 1e-9)), 0)
    c1 = min(int(np.ceil(hi - 1e-9)), cells)
    return c0, c1


def _patch_faces(mesh: IonOpticsMesh, touches: dict[str, bool]) -> dict:
    """The domain's face conditions on the sides of a patch that lie on them."""
    return {face: mesh.faces[face] for face, on in touches.items() if on}


def patches_of(mesh: IonOpticsMesh, refinement: Sequence[Refinement]) -> list[Patch]:
    """The base patch and one patch per refined box, coarse to fine (stable by level).

    A box is widened to the cells of the level below, so it starts and ends on that level's
    nodes, and clipped to the mesh (``solver/refinement.py:85-152``).
    """
    nx, ny = mesh.shape
    origin = mesh.origin
    upper = mesh.upper
    patches = [Patch(0, ((0, nx - 1), (0, ny - 1)), mesh)]
    for box in sorted(refinement, key=lambda b: int(b.level)):
        level = int(box.level)
        if level < 1:
            raise ValueError(f"a refined box needs a level of at least 1, got {box.level}")
        parent = 2 ** (level - 1)  # the parent level's cells per base cell
        spans = []
        for axis, n in enumerate((nx, ny)):
            lower, upper_ = float(box.lower[axis]), float(box.upper[axis])
            start, end = origin[axis], upper[axis]
            if axis == 0 and mesh.graded:
                # along a graded x, the box in the uniform coordinate of the node indices
                clip = lambda v: min(max(v, origin[0]), upper[0])  # noqa: E731
                lower = float(mesh.logical_x(clip(lower)))
                upper_ = float(mesh.logical_x(clip(upper_)))
                start, end = mesh.logical_origin[0], mesh.logical_upper[0]
            c0, c1 = _parent_span(lower, upper_, start, end, mesh.h / parent, (n - 1) * parent)
            if c1 <= c0:
                raise ValueError(f"the refined box {box} is outside the mesh")
            spans.append((2 * c0, 2 * c1))
        h = mesh.h / 2**level
        last = ((nx - 1) * 2**level, (ny - 1) * 2**level)
        shape = tuple(spans[a][1] - spans[a][0] + 1 for a in range(2))
        touches = {"x_min": spans[0][0] == 0, "x_max": spans[0][1] == last[0],
                   "y_min": spans[1][0] == 0, "y_max": spans[1][1] == last[1]}  # fmt: skip
        y0 = origin[1] + spans[1][0] * h
        plane = bool(mesh.symmetry_plane and spans[1][0] == 0)

        def part(first_x: int, first_y: int, size: tuple[int, int]) -> IonOpticsMesh:
            graded = {}
            x0 = origin[0] + first_x * h
            if mesh.graded:
                # the level's nodes evenly between the base nodes of a graded x
                nodes = np.asarray(mesh.position_x(np.arange(first_x, first_x + size[0])
                                                   / 2**level), dtype=float)  # fmt: skip
                x0 = float(nodes[0])
                graded = {"x_nodes": nodes, "logical_x0": mesh.logical_x0 + first_x * h}
            return IonOpticsMesh(
                shape=size, origin=(x0, origin[1] + first_y * h), h=h,
                geometry=mesh.geometry, electrodes=mesh.electrodes,
                faces=_patch_faces(mesh, touches), patch=True, symmetry_plane=plane,
                classify_on_device=mesh.classify_on_device, **graded,
            )  # fmt: skip

        patch_mesh = part(spans[0][0], spans[1][0], shape)
        below = [min(2, spans[a][0]) for a in range(2)]
        above = [min(2, last[a] - spans[a][1]) for a in range(2)]
        field_mesh = part(spans[0][0] - below[0], spans[1][0] - below[1],
                          (shape[0] + below[0] + above[0], shape[1] + below[1] + above[1]))  # fmt: skip
        inner = (slice(below[0], below[0] + shape[0]), slice(below[1], below[1] + shape[1]))
        assert abs(patch_mesh.origin[1] - y0) <= 1e-12 * max(1.0, abs(y0))
        patches.append(Patch(level, (spans[0], spans[1]), patch_mesh, None, field_mesh, inner))
    return patches


def _inside(patch: Patch, base_shape: tuple[int, int]) -> np.ndarray:
    """The patch's nodes off the sides of its box that are not faces of the domain."""
    nxp, nyp = patch.mesh.shape
    scale = 2**patch.level
    keep = []
    for axis, n in enumerate((nxp, nyp)):
        first, last = patch.box[axis]
        ok = np.zeros(n, dtype=bool)
        ok[1:-1] = True
        ok[0] = first == 0
        ok[-1] = last == (base_shape[axis] - 1) * scale
        keep.append(ok)
    return keep[0][:, None] & keep[1][None, :]


@dataclass
class Layout:
    """The composite nodes of a refined mesh (``solver/refinement.py:155-231``).

    ``x``, ``y`` the nodes' coordinates; ``volumes`` their control volumes; ``owner`` the
    patch whose row is each node's equation (-1: hanging), ``owner_node`` its flat node in
    that patch; ``hanging`` the hanging nodes and ``interpolation`` (CSR, hanging x nodes)
    their values from the nodes that are not hanging; ``fixed``, ``fixed_value`` the nodes
    held by an electrode or a Dirichlet face.
    """

    patches: list[Patch]
    x: np.ndarray
    y: np.ndarray
    volumes: np.ndarray
    owner: np.ndarray
    owner_node: np.ndarray
    hanging: np.ndarray
    interpolation: sparse.csr_matrix
    fixed: np.ndarray
    fixed_value: np.ndarray
    lattice: np.ndarray = field(repr=False, default=None)
    hierarchy: Any = None

    @property
    def size(self) -> int:
        """The number of composite nodes."""
        return int(self.x.size)

    @property
    def base(self) -> Patch:
        return self.patches[0]

    @property
    def refined(self) -> bool:
        return len(self.patches) > 1

    def on_base(self, values: np.ndarray) -> np.ndarray:
        """The ``(nx, ny)`` array of composite values on the base mesh."""
        return np.asarray(values)[self.base.index]

    def from_base(self, array: np.ndarray) -> np.ndarray:
        """Composite values of an ``(nx, ny)`` array, without refinement only."""
        if self.refined:
            raise ValueError(
                "with refinement give values on the composite nodes (`Layout.x`, `Layout.y`)"
            )
        out = np.empty(self.size)
        out[self.base.index.ravel()] = np.asarray(array, dtype=float).ravel()
        return out

    def deposit_total(self, charges: Sequence[np.ndarray]) -> np.ndarray:
        """The composite node charges of per-patch node charges (shared nodes added, in
        patch order)."""
        total = np.zeros(self.size)
        for patch, charge in zip(self.patches, charges, strict=True):
            np.add.at(total, patch.index.ravel(), np.asarray(charge, dtype=float).ravel())
        return total

    def fill_hanging(self, values: np.ndarray) -> None:
        """Set the hanging nodes of a composite array from the nodes they hang from."""
        if self.hanging.size:
            values[self.hanging] = self.interpolation @ values

    def field(self, potential: np.ndarray):
        """The electric field of a composite potential (`PatchedElectricField`)."""
        from beamtracer_b200.composite import PatchedElectricField

        return PatchedElectricField(self, potential)


def _check_nested(covers: list[np.ndarray]) -> None:
    """Every level's boxes inside those of the level below (cell masks per level)."""
    for level in range(2, len(covers)):
        fine = covers[level]
        coarse = covers[level - 1]
        shrunk = fine.reshape(coarse.shape[0], 2, coarse.shape[1], 2).any(axis=(1, 3))
        if np.any(shrunk & ~coarse):
            raise ValueError(f"the boxes of level {level} must lie inside those of level "
                             f"{level - 1}")  # fmt: skip


def layout_of(mesh: IonOpticsMesh, patches: list[Patch]) -> Layout:
    """The composite nodes of ``patches`` (see the module), setting every `Patch.index`."""
    finest = max(p.level for p in patches)
    nx, ny = mesh.shape
    span = (ny - 1) * 2**finest + 1
    coords = []
    for patch in patches:
        s = 2 ** (finest - patch.level)
        nxp, nyp = patch.mesh.shape
        i = (patch.box[0][0] + np.arange(nxp)) * s
        j = (patch.box[1][0] + np.arange(nyp)) * s
        coords.append((i, j))
    keys = np.unique(np.concatenate([(i[:, None] * span + j[None, :]).ravel()
                                     for i, j in coords]))  # fmt: skip
    for patch, (i, j) in zip(patches, coords):
        patch.index = np.searchsorted(keys, i[:, None] * span + j[None, :]).astype(np.int64)
    n = keys.size
    I, J = keys // span, keys % span
    hf = mesh.h / 2**finest
    x = (np.asarray(mesh.position_x(I / 2**finest), dtype=float) if mesh.graded
         else mesh.origin[0] + I * hf)  # fmt: skip
    y = mesh.origin[1] + J * hf
    # owners: the finest patch whose inside holds the node
    owner = np.full(n, -1, dtype=np.int64)
    owner_node = np.full(n, -1, dtype=np.int64)
    for number in sorted(range(len(patches)), key=lambda q: patches[q].level):
        patch = patches[number]
        inside = _inside(patch, mesh.shape)
        owner[patch.index[inside]] = number
        owner_node[patch.index[inside]] = np.flatnonzero(inside.ravel())
    hanging = np.flatnonzero(owner < 0)
    interpolation = _hanging_interpolation(hanging, I, J, keys, span, finest, owner)
    # held nodes, from each owner's own classification
    fixed = np.zeros(n, dtype=bool)
    fixed_value = np.zeros(n)
    for number, patch in enumerate(patches):
        mine = np.flatnonzero(owner == number)
        local = owner_node[mine]
        fixed[mine] = np.asarray(patch.mesh.fixed).ravel()[local]
        fixed_value[mine] = np.asarray(patch.mesh.fixed_value).ravel()[local]
    volumes, covers = _leaf_volumes(mesh, patches, keys, span, finest)
    _check_nested(covers)
    return Layout(patches, x, y, volumes, owner, owner_node, hanging, interpolation, fixed,
                  fixed_value, np.stack([I, J], axis=1))  # fmt: skip


def _hanging_interpolation(hanging, I, J, keys, span, finest, owner) -> sparse.csr_matrix:
    """Each hanging node's value from nodes that do not hang (linear along the coarse edge
    it lies on, substituted while an end hangs itself)."""
    n = keys.size
    if not hanging.size:
        return sparse.csr_matrix((0, n))

    def node(i: int, j: int) -> int:
        k = int(np.searchsorted(keys, i * span + j))
        if k >= n or keys[k] != i * span + j:  # pragma: no cover - a layout invariant
            raise RuntimeError("a hanging node's edge end is not a composite node")
        return k

    memo: dict[int, dict[int, float]] = {}

    def expand(k: int) -> dict[int, float]:
        if owner[k] >= 0:
            return {k: 1.0}
        if k in memo:
            return memo[k]
        i, j = int(I[k]), int(J[k])
        # the coarsest level whose lattice holds the node: a node of level m hangs on an
        # edge of level m - 1 along the axis where it is off that level's lattice
        q = 2**finest
        while q > 1 and not (i % q == 0 and j % q == 0):
            q //= 2
        if i % (2 * q) == 0:
            ends = (node(i, j - q), node(i, j + q))
        else:
            ends = (node(i - q, j), node(i + q, j))
        out: dict[int, float] = {}
        for end in ends:
            for src, w in expand(end).items():
                out[src] = out.get(src, 0.0) + 0.5 * w
        memo[k] = out
        return out

    rows, cols, vals = [], [], []
    for r, k in enumerate(hanging):
        for src, w in sorted(expand(int(k)).items()):
            rows.append(r)
            cols.append(src)
            vals.append(w)
    return sparse.csr_matrix((vals, (rows, cols)), shape=(hanging.size, n))


def _leaf_volumes(mesh, patches, keys, span, finest):
    """The control volumes (quarters of the leaf cells at their corners) and the cell
    masks of every level's boxes."""
    nx, ny = mesh.shape
    covers = []
    for level in range(finest + 1):
        cover = np.zeros(((nx - 1) * 2**level, (ny - 1) * 2**level), dtype=bool)
        for patch in patches:
            if patch.level == level:
                (i0, i1), (j0, j1) = patch.box
                cover[i0:i1, j0:j1] = True
        covers.append(cover)
    volumes = np.zeros(keys.size)
    for level, cover in enumerate(covers):
        leaf = cover.copy()
        if level < finest:
            finer = covers[level + 1]
            leaf &= ~finer.reshape(cover.shape[0], 2, cover.shape[1], 2).any(axis=(1, 3))
        ci, cj = np.nonzero(leaf)
        if not ci.size:
            continue
        h = mesh.h / 2**level
        if mesh.graded:  # the cell's width between its two nodes along the graded x
            width = (np.asarray(mesh.position_x((ci + 1) / 2**level), dtype=float)
                     - np.asarray(mesh.position_x(ci / 2**level), dtype=float))  # fmt: skip
        else:
            width = np.full(ci.size, h)
        if mesh.cylindrical:
            rc = mesh.origin[1] + (cj + 0.5) * h
            cell = 2.0 * np.pi * rc * width * h
        else:
            cell = width * h
        s = 2 ** (finest - level)
        for di in (0, 1):
            for dj in (0, 1):
                corner = np.searchsorted(keys, (ci + di) * s * span + (cj + dj) * s)
                volumes += np.bincount(corner, weights=0.25 * cell, minlength=keys.size)
    return volumes, covers


def layout_of_mesh(mesh: IonOpticsMesh, refinement: Sequence[Refinement] = ()) -> Layout:
    """The layout of a mesh with the boxes ``refinement`` (none: the mesh's own nodes)."""
    return layout_of(mesh, patches_of(mesh, refinement))
