"""Refined boxes on the B200: the composite field solve and the patches' electric field.

The reference solves the field of refined boxes with patchwork's composite ``NodalPoisson``
(``solver/poisson.py:169-335``) and takes a trajectory's field and deposit on the finest
patch holding it (``solver/refinement.py:299-387``, ``tracer.py:1141-1183``).  Here:

- every patch keeps its own device field solver (`IonOpticsPoisson` of its mesh): its rows
  are the equations of the composite nodes it owns (`beamtracer_b200.refinement`), and its
  multigrid solves the corrections;
- the composite system is solved by restarted GMRES right-preconditioned with one fast
  adaptive composite (FAC) sweep: coarse to fine, the composite residual is taken on a
  patch's nodes, the patch's homogeneous problem (its held nodes and, for a box, its sides
  inside the domain at zero) is solved inexactly by one V-cycle of its multigrid, and the
  correction is added to the composite nodes in the patch's box (bilinear between the
  patch's nodes at the finer nodes); with a Boltzmann species every Newton step's
  correction is solved the same way, each patch's multigrid rebuilt with the step's
  reaction;
- the maps between composite nodes and patch arrays are row-compressed matrices applied
  by one kernel (``bt_csr_apply``) in a fixed order: the patches' potentials and the wider
  meshes of their fields (the margin bilinear from the coarser patches, finest wins, as
  ``solver/refinement.py:299-325``), the composite charges from the patches' deposits, the
  hanging nodes.
"""

from __future__ import annotations

import ctypes

import numpy as np
from scipy import sparse

from beamtracer_b200 import _lib
from beamtracer_b200.refinement import Layout, _inside


class DeviceCSR:
    """A row-compressed matrix on the device: ``y[out] = (y[out] or c) + A x`` per row."""

    def __init__(self, matrix: sparse.csr_matrix, out_rows=None, constant=None) -> None:
        import torch

        matrix = sparse.csr_matrix(matrix)
        matrix.sort_indices()
        self.rows = int(matrix.shape[0])
        self.cols = int(matrix.shape[1])
        dev = "cuda"
        self.ptr = torch.from_numpy(matrix.indptr.astype(np.int64)).to(dev)
        self.col = torch.from_numpy(matrix.indices.astype(np.int64)).to(dev)
        self.val = torch.from_numpy(matrix.data.astype(np.float64)).to(dev)
        self.out = (None if out_rows is None
                    else torch.from_numpy(np.asarray(out_rows, dtype=np.int64)).to(dev))  # fmt: skip
        self.constant = (None if constant is None
                         else torch.from_numpy(np.asarray(constant, dtype=np.float64)).to(dev))  # fmt: skip
        # the map's own arrays live as long as it does: their addresses, once
        d = _lib.dptr
        self._args = (d(self.out), d(self.ptr), d(self.col), d(self.val), d(self.constant))

    def apply(self, x, y, accumulate: bool = False, handle=None) -> None:
        """``handle``: the library context to queue on (default: the calling thread's)."""
        d = _lib.dptr
        handle = _lib.context().handle if handle is None else handle
        _lib.check(_lib.lib().bt_csr_apply(handle, self.rows, *self._args, int(accumulate),
                                           d(x), d(y)))  # fmt: skip


def _selection(index: np.ndarray, size: int, value: float = 1.0) -> sparse.csr_matrix:
    """Rows picking ``index`` out of ``size`` entries (times ``value``)."""
    index = np.asarray(index, dtype=np.int64).ravel()
    return sparse.csr_matrix((np.full(index.size, value), (np.arange(index.size), index)),
                             shape=(index.size, size))  # fmt: skip


def prolongation(layout: Layout, number: int,
                 held: np.ndarray | None = None) -> tuple[sparse.csr_matrix, np.ndarray]:
    """The composite nodes in patch ``number``'s box not ``held`` (default: the layout's
    held nodes) and, per node, the bilinear weights of the patch's nodes at it (the node's
    own value where it is one of them)."""
    held = layout.fixed if held is None else held
    patch = layout.patches[number]
    finest = max(p.level for p in layout.patches)
    s = 2 ** (finest - patch.level)
    (i0, _), (j0, _) = patch.box
    nxp, nyp = patch.mesh.shape
    li = layout.lattice[:, 0] / s - i0
    lj = layout.lattice[:, 1] / s - j0
    mine = np.flatnonzero((li >= 0) & (li <= nxp - 1) & (lj >= 0) & (lj <= nyp - 1)
                          & ~held)  # fmt: skip
    a = np.clip(np.floor(li[mine]).astype(np.int64), 0, nxp - 2)
    b = np.clip(np.floor(lj[mine]).astype(np.int64), 0, nyp - 2)
    u, w = li[mine] - a, lj[mine] - b
    rows = np.tile(np.arange(mine.size), 4)
    cols = np.concatenate([a * nyp + b, a * nyp + b + 1, (a + 1) * nyp + b, (a + 1) * nyp + b + 1])
    vals = np.concatenate([(1 - u) * (1 - w), (1 - u) * w, u * (1 - w), u * w])
    keep = vals != 0.0
    matrix = sparse.csr_matrix((vals[keep], (rows[keep], cols[keep])),
                               shape=(mine.size, nxp * nyp))  # fmt: skip
    return matrix, mine


class _Held:
    """What depends on the held composite nodes (the mesh's, plus an initial plasma region):
    the rows that carry an equation, the values to hold, the corrections' spread and the
    nodes each patch's correction holds."""

    def __init__(self, layout: Layout, held: np.ndarray, values: np.ndarray,
                 offsets: np.ndarray) -> None:  # fmt: skip
        import torch

        n = layout.size
        base_shape = layout.base.mesh.shape
        own = (layout.owner >= 0) & ~held
        rows = np.flatnonzero(own)
        cols = offsets[layout.owner[rows]] + layout.owner_node[rows]
        self.owned = DeviceCSR(sparse.csr_matrix((np.ones(rows.size), (rows, cols)),
                                                 shape=(n, int(offsets[-1]))))  # fmt: skip
        self.own = torch.from_numpy(own.astype(np.uint8)).cuda()
        kept = np.flatnonzero(held)
        self.setter = DeviceCSR(sparse.csr_matrix((kept.size, 1)), out_rows=kept,
                                constant=values[kept])  # fmt: skip
        self.prolong = []
        self.sides = []
        for number, patch in enumerate(layout.patches):
            matrix, where = prolongation(layout, number, held)
            self.prolong.append(DeviceCSR(matrix, out_rows=where))
            local = held[patch.index] & ~np.asarray(patch.mesh.fixed, dtype=bool)
            sides = local if number == 0 else (~_inside(patch, base_shape) | local)
            self.sides.append(sides if sides.any() else None)


class CompositePoisson:
    """The field of a refined layout solved on the device (see the module).

    ``solve_device(phi, rho)`` takes composite device vectors: ``phi`` the first guess (its
    held and hanging nodes are set) and the result, ``rho`` [C/m^3] or None.  With
    ``fixed_region`` (a mask of the composite nodes, or a function of their ``(x, y)``) those
    nodes are held at ``fixed_potential`` as well; with ``plasma`` (a Boltzmann species:
    ``amplitude`` rho_0 / eps0, ``temperature``, ``up``, ``sign``) Newton's method from
    ``phi``, each step's correction by the same Krylov solve with the Jacobian's reaction
    in every patch's solver, until its largest update is below ``newton_tolerance``.
    """

    def __init__(self, layout: Layout, *, tolerance: float = 1e-13, restart: int = 30,
                 max_restarts: int = 20, newton_sweep_tolerance: float = 1e-10) -> None:  # fmt: skip
        import torch

        from beamtracer_b200.poisson import IonOpticsPoisson

        self.layout = layout
        #: the linear solves' relative residual (of the first residual)
        self.tolerance = float(tolerance)
        #: GMRES's restart length and restarts
        self.restart = int(restart)
        self.max_restarts = int(max_restarts)
        #: a Newton step's relative residual (an inexact Newton step: the steps continue
        #: until their own update is below Newton's tolerance)
        self.newton_sweep_tolerance = float(newton_sweep_tolerance)
        patches = layout.patches
        n = layout.size
        #: every patch's own operator (its rows: the equations of the nodes it owns)
        self.rows = [IonOpticsPoisson(p.mesh) for p in patches]
        #: the corrections' solvers: held values and face terms zero, a box's sides held
        self.corrections = [IonOpticsPoisson(p.mesh, homogeneous=True) for p in patches]
        sizes = [int(np.prod(p.mesh.shape)) for p in patches]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        total = int(self.offsets[-1])
        dev = "cuda"
        f64 = torch.float64
        self._phi_p = torch.zeros(total, dtype=f64, device=dev)
        self._rho_p = torch.zeros(total, dtype=f64, device=dev)
        self._res_p = torch.zeros(total, dtype=f64, device=dev)
        self._rhs_p = torch.zeros(total, dtype=f64, device=dev)
        self._e_p = torch.zeros(total, dtype=f64, device=dev)
        self._reaction_p = torch.zeros(total, dtype=f64, device=dev)
        self._r = torch.zeros(n, dtype=f64, device=dev)
        self._r0 = torch.zeros(n, dtype=f64, device=dev)
        self._reaction = torch.zeros(n, dtype=f64, device=dev)
        self._delta = torch.zeros(n, dtype=f64, device=dev)
        self._w = torch.zeros(n, dtype=f64, device=dev)
        #: the Krylov basis and its preconditioned images
        self._basis = torch.zeros((self.restart + 1, n), dtype=f64, device=dev)
        self._images = torch.zeros((self.restart, n), dtype=f64, device=dev)
        self._zero = torch.zeros(max(n, 1), dtype=f64, device=dev)
        self._scalars = torch.zeros(2, dtype=f64, device=dev)
        self._gather = [DeviceCSR(_selection(p.index, n)) for p in patches]
        self._hang = (DeviceCSR(layout.interpolation, out_rows=layout.hanging)
                      if layout.hanging.size else None)  # fmt: skip
        self._plain = _Held(layout, layout.fixed, layout.fixed_value, self.offsets)
        self._views: dict = {}
        #: per patch, the patches whose rows its correction reads: it and the finer ones
        #: (every patch for the base)
        self._finer = [[p for p in range(len(patches)) if patches[p].level >= patches[q].level]
                       for q in range(len(patches))]  # fmt: skip
        #: the library context of the solve in progress (the calling thread's)
        self._h = None
        #: the sides each correction solver holds now (the object last given to it)
        self._held_sides: list = [None] * len(patches)
        self._region_key: object = None
        self._region: _Held | None = None
        #: FAC sweeps of the last solve, and their corrections' V-cycles; Newton steps
        self.sweeps = 0
        self.krylov_steps = 0
        self.newton_iterations = 0

    def _view(self, buffer, number: int):
        """Patch ``number``'s part of a buffer over every patch's nodes (made once)."""
        key = (id(buffer), number)
        view = self._views.get(key)
        if view is None:
            lo, hi = self.offsets[number], self.offsets[number + 1]
            view = buffer[lo:hi].view(self.layout.patches[number].mesh.shape)
            self._views[key] = view
        return view

    def _hold(self, number: int, sides) -> None:
        """Hold a correction solver's ``sides`` (skipped when they are the ones it holds)."""
        if self._held_sides[number] is not sides:
            self.corrections[number].hold(sides)
            self._held_sides[number] = sides

    def fill_hanging(self, phi) -> None:
        if self._hang is not None:
            self._hang.apply(phi, phi, handle=self._h)

    def _held(self, region, potential: float) -> _Held:
        if region is None:
            return self._plain
        layout = self.layout
        mask = np.asarray(region(layout.x, layout.y) if callable(region) else region, dtype=bool)
        if mask.shape != (layout.size,):
            raise ValueError("the held region needs the layout's composite nodes")
        mask = mask & ~layout.fixed
        mask[layout.hanging] = False
        key = (np.packbits(mask).tobytes(), float(potential))
        if key != self._region_key:
            values = np.where(mask, float(potential), layout.fixed_value)
            self._region = _Held(layout, layout.fixed | mask, values, self.offsets)
            self._region_key = key
        return self._region

    def residual(self, phi, r, held: _Held | None = None, patches=None) -> None:
        """``r`` <- the composite residual of ``phi`` (zero on held and hanging nodes), with
        the charge density last given to `solve_device`.  ``patches``: only these patches'
        rows are evaluated again (the others keep their last values): a patch's correction
        reads the residual at its inside nodes alone, which it and the finer patches own."""
        held = held or self._plain
        self.fill_hanging(phi)
        lib = _lib.lib()
        for number in range(len(self.rows)) if patches is None else patches:
            solver = self.rows[number]
            phi_p = self._view(self._phi_p, number)
            self._gather[number].apply(phi, phi_p, handle=self._h)
            _lib.check(lib.bt_poisson_residual(solver._handle, _lib.dptr(phi_p),
                                               _lib.dptr(self._view(self._rho_p, number)),
                                               _lib.dptr(self._view(self._res_p, number))))  # fmt: skip
        held.owned.apply(self._res_p, r, handle=self._h)

    def _step_residual(self, delta, r, held: _Held, patches=None) -> None:
        """``r`` <- the residual of a Newton step's correction ``delta``: the step's own
        residual less (K + diag(reaction)) delta, at the nodes with an equation
        (``patches`` as in `residual`)."""
        self.fill_hanging(delta)
        lib = _lib.lib()
        for number in range(len(self.corrections)) if patches is None else patches:
            solver = self.corrections[number]
            d_p = self._view(self._phi_p, number)
            self._gather[number].apply(delta, d_p, handle=self._h)
            self._hold(number, held.sides[number])
            _lib.check(lib.bt_poisson_residual(solver._handle, _lib.dptr(d_p), None,
                                               _lib.dptr(self._view(self._res_p, number))))  # fmt: skip
        held.owned.apply(self._res_p, r, handle=self._h)
        d = _lib.dptr
        _lib.check(lib.bt_newton_residual(self._h, self.layout.size, d(held.own),
                                          d(self._r0), d(self._reaction), d(delta), d(r)))  # fmt: skip

    def _max(self, a, b=None) -> float:
        n = self.layout.size
        _lib.check(_lib.lib().bt_max_abs_diff(self._h, _lib.dptr(a),
                                              _lib.dptr(self._zero if b is None else b), n,
                                              _lib.dptr(self._scalars)))  # fmt: skip
        return float(self._scalars[0])

    def _sweep(self, x, held: _Held, reaction: bool, rebuild: bool) -> None:
        """One FAC sweep on ``x`` for ``J x = r0`` (J the composite operator, plus the
        reaction when ``reaction``): coarse to fine, the residual at each patch's nodes,
        one V-cycle of its homogeneous problem, the correction spread over its box."""
        lib = _lib.lib()
        for number, solver in enumerate(self.corrections):
            self._step_residual(x, self._r, held, self._finer[number])
            rhs = self._view(self._rhs_p, number)
            e = self._view(self._e_p, number)
            self._gather[number].apply(self._r, rhs, handle=self._h)
            self._hold(number, held.sides[number])
            react = None
            if reaction:
                react = self._view(self._reaction_p, number)
                self._gather[number].apply(self._reaction, react, handle=self._h)
            _lib.check(lib.bt_poisson_vcycle(solver._handle, _lib.dptr(rhs), _lib.dptr(react),
                                             int(rebuild), _lib.dptr(e)))  # fmt: skip
            held.prolong[number].apply(e.reshape(-1), x, True, self._h)
        self.fill_hanging(x)

    def _krylov(self, x, held: _Held, reaction: bool, tolerance: float, floor: float) -> int:
        """``x`` (zero on entry) <- the solution of ``J x = r0`` (``self._r0`` on the nodes
        with an equation) by restarted GMRES, right-preconditioned by one FAC sweep from
        zero: the sweeps alone diverge on some nestings of three levels, the Krylov method
        converges whenever the preconditioned operator is regular.  Stops at a residual of
        ``tolerance`` of the first (at least ``floor``), or where it stalls within 1e4 of
        that (its rounding floor); returns the sweeps taken."""
        import torch

        n = self.layout.size
        m = self.restart
        basis = self._basis
        images = self._images
        r0 = self._r0
        goal = None
        sweeps = 0
        rebuild = reaction
        rhs = r0.clone()
        for _cycle in range(self.max_restarts):
            # r = rhs - J x
            self._r0.copy_(rhs)
            self._step_residual(x, self._w, held)
            beta = float(torch.linalg.vector_norm(self._w))
            if goal is None:
                goal = max(tolerance * beta, floor)
                if not goal > 0.0:
                    goal = 1e-300
            if not np.isfinite(beta):
                raise RuntimeError("the composite field solve diverged (a non-finite residual)")
            if beta <= goal:
                break
            basis[0].copy_(self._w / beta)
            hess = np.zeros((m + 1, m))
            g = np.zeros(m + 1)
            g[0] = beta
            rot = []
            k = 0
            for j in range(m):
                # z_j = M v_j: one sweep from zero on the right-hand side v_j
                self._r0.copy_(basis[j])
                images[j].zero_()
                self._sweep(images[j], held, reaction, rebuild)
                rebuild = False
                sweeps += 1
                # w = J z_j (the residual of z_j against a zero right-hand side, negated)
                self._r0.zero_()
                self._step_residual(images[j], self._w, held)
                self._w.neg_()
                # classical Gram-Schmidt, twice
                h = torch.mv(basis[: j + 1], self._w)
                self._w.sub_(torch.mv(basis[: j + 1].T, h))
                h2 = torch.mv(basis[: j + 1], self._w)
                self._w.sub_(torch.mv(basis[: j + 1].T, h2))
                col = (h + h2).cpu().numpy()
                norm = float(torch.linalg.vector_norm(self._w))
                hess[: j + 1, j] = col
                hess[j + 1, j] = norm
                for i, (c, sn) in enumerate(rot):
                    a, b = hess[i, j], hess[i + 1, j]
                    hess[i, j], hess[i + 1, j] = c * a + sn * b, -sn * a + c * b
                a, b = hess[j, j], hess[j + 1, j]
                radius = float(np.hypot(a, b))
                c, sn = (a / radius, b / radius) if radius > 0.0 else (1.0, 0.0)
                rot.append((c, sn))
                hess[j, j], hess[j + 1, j] = radius, 0.0
                g[j], g[j + 1] = c * g[j], -sn * g[j]
                k = j + 1
                if abs(g[j + 1]) <= goal or norm == 0.0:
                    break
                basis[j + 1].copy_(self._w / norm)
            y = np.linalg.solve(np.triu(hess[:k, :k]), g[:k]) if k else np.zeros(0)
            update = torch.from_numpy(y).to(images.device)
            x.add_(torch.mv(images[:k].T, update))
            self.fill_hanging(x)
            if abs(g[k]) <= goal:
                continue  # confirmed by the true residual at the top of the next cycle
            if abs(g[k]) > 0.5 * beta and abs(g[k]) <= 1e4 * goal:
                break  # stalled at the rounding floor
        else:
            self._r0.copy_(rhs)
            self._step_residual(x, self._w, held)
            left = float(torch.linalg.vector_norm(self._w))
            if not left <= 1e4 * goal:
                raise RuntimeError("the composite field solve did not converge")
        self._r0.copy_(rhs)
        self.sweeps = sweeps
        return sweeps

    def solve_device(self, phi, rho=None, *, fixed_region=None, fixed_potential: float = 0.0,
                     plasma: tuple[float, float, float, int] | None = None,
                     newton_tolerance: float = 1e-6, max_newton: int = 100) -> None:  # fmt: skip
        n = self.layout.size
        if tuple(phi.shape) != (n,) or (rho is not None and tuple(rho.shape) != (n,)):
            raise ValueError(f"the composite solve takes ({n},) composite vectors")
        self._h = _lib.context().handle
        held = self._held(fixed_region, fixed_potential)
        if rho is None:
            self._rho_p.zero_()
        else:
            for number in range(len(self.rows)):
                self._gather[number].apply(rho, self._view(self._rho_p, number),
                                           handle=self._h)
        held.setter.apply(phi, phi, handle=self._h)
        self.fill_hanging(phi)
        self.newton_iterations = 0
        # the scale of the right-hand side: the residual of the held values alone, whose
        # 1e-13 is the rounding floor the solves stop at
        import torch

        self._w.zero_()
        held.setter.apply(self._w, self._w, handle=self._h)
        self.residual(self._w, self._r, held)
        floor = 1e-13 * float(torch.linalg.vector_norm(self._r))
        if plasma is None:
            # phi += J^-1 (b - K phi), J = K on the nodes with an equation
            self.residual(phi, self._r0, held)
            self._reaction.zero_()
            self._delta.zero_()
            self.krylov_steps = self._krylov(self._delta, held, False, self.tolerance, floor)
            phi.add_(self._delta)
            self.fill_hanging(phi)
            return
        amplitude, temperature, up, sign = plasma
        lib = _lib.lib()
        cycles = 0
        d = _lib.dptr
        for step in range(1, int(max_newton) + 1):
            self.residual(phi, self._r0, held)
            _lib.check(lib.bt_boltzmann_terms(self._h, n, d(held.own), d(phi),
                                              float(amplitude), float(temperature), float(up),
                                              int(sign), d(self._r0), d(self._reaction)))  # fmt: skip
            self._delta.zero_()
            cycles += self._krylov(self._delta, held, True, self.newton_sweep_tolerance, floor)
            phi.add_(self._delta)
            self.fill_hanging(phi)
            update = self._max(self._delta)
            if not np.isfinite(update):
                raise RuntimeError("the composite Newton update is not finite")
            self.newton_iterations = step
            if update < newton_tolerance:
                break
        self.krylov_steps = cycles

    def close(self) -> None:
        for solver in (*self.rows, *self.corrections):
            solver.close()


def _extrapolation(mesh) -> list[str]:
    """Linear extrapolation on every face, mirror on the y_min face where it is the axis or
    a symmetry plane (``solver/refinement.py:289-295``)."""
    faces = ["extrapolate"] * 4
    on_axis = mesh.cylindrical and abs(mesh.origin[1]) <= 1e-12 * mesh.h
    if on_axis or mesh.symmetry_plane:
        faces[2] = "symmetric"
    return faces


class PatchedFieldMaps:
    """What the electric field of a layout needs on the device, built once per layout: per
    patch the map from composite potentials to its field mesh's nodes, the field meshes'
    classification, the edge fields' flat buffers and the tracer's patch tables (finest
    first, the base last: ``tracer.py:1141-1183``), and the map from the deposit's patch
    charges (their boxes' nodes) to composite charges."""

    def __init__(self, layout: Layout) -> None:
        import torch

        from beamtracer_b200.fields import MeshArrays

        self.layout = layout
        patches = layout.patches
        n = layout.size
        self.meshes = [p.field_mesh if p.field_mesh is not None else p.mesh for p in patches]
        matrices, constants = [], []
        for number, patch in enumerate(patches):
            mesh = self.meshes[number]
            nxf, nyf = mesh.shape
            if patch.field_mesh is None:
                matrix = _selection(patch.index, n)
                constant = np.zeros(nxf * nyf)
            else:
                # the margin bilinear, its electrode nodes at their potential, the box's
                # own nodes from the composite nodes (in that order of precedence)
                matrix, constant = self._margin(matrices, constants, mesh)
                solid = np.asarray(mesh.solid).ravel() >= 0
                inner = np.zeros((nxf, nyf), dtype=bool)
                inner[patch.inner] = True
                inner = inner.ravel()
                keep = sparse.diags((~solid & ~inner).astype(float))
                own = sparse.csr_matrix((np.ones(patch.index.size),
                                         (np.flatnonzero(inner), patch.index.ravel())),
                                        shape=(nxf * nyf, n))  # fmt: skip
                matrix = (keep @ matrix + own).tocsr()
                constant = np.where(inner, 0.0, np.where(
                    solid, np.asarray(mesh.fixed_value).ravel(), constant))
            matrix.eliminate_zeros()
            matrices.append(matrix)
            constants.append(constant)
        self.potential_maps = [DeviceCSR(m, constant=c) for m, c in zip(matrices, constants)]
        self.arrays = [MeshArrays(mesh) for mesh in self.meshes]
        # flat edge-field buffers and the tracer's tables, finest first
        order = list(range(len(patches)))[::-1]
        fx_sizes = [(self.meshes[q].shape[0] + 1) * self.meshes[q].shape[1] for q in order]
        fy_sizes = [self.meshes[q].shape[0] * (self.meshes[q].shape[1] + 1) for q in order]
        node_sizes = [self.meshes[q].shape[0] * self.meshes[q].shape[1] for q in order]
        fx_off = np.concatenate([[0], np.cumsum(fx_sizes)]).astype(np.int64)
        fy_off = np.concatenate([[0], np.cumsum(fy_sizes)]).astype(np.int64)
        node_off = np.concatenate([[0], np.cumsum(node_sizes)]).astype(np.int64)
        dev = "cuda"
        self.fx = torch.zeros(int(fx_off[-1]), dtype=torch.float64, device=dev)
        self.fy = torch.zeros(int(fy_off[-1]), dtype=torch.float64, device=dev)
        self.values = [torch.zeros(m.shape, dtype=torch.float64, device=dev) for m in self.meshes]
        self.field_views = {}
        ints, reals = [], []
        for slot, q in enumerate(order):
            mesh = self.meshes[q]
            nxf, nyf = mesh.shape
            self.field_views[q] = (
                self.fx[fx_off[slot]:fx_off[slot + 1]].view(nxf + 1, nyf),
                self.fy[fy_off[slot]:fy_off[slot + 1]].view(nxf, nyf + 1),
            )
            ints.append([nxf, nyf, fx_off[slot], fy_off[slot], nxf * nyf, node_off[slot]])
            # along a graded x the kernel locates points by their uniform coordinate
            x0, y0, x1, y1 = patches[q].bounds
            base = layout.base.mesh
            lx0, lx1 = float(base.logical_x(x0)), float(base.logical_x(x1))
            reals.append([*mesh.logical_origin, mesh.h, lx0, y0, lx1, y1])
        self.patch_int = torch.tensor(ints, dtype=torch.int64, device=dev)
        self.patch_real = torch.tensor(reals, dtype=torch.float64, device=dev)
        self.n_field_nodes = int(node_off[-1])
        # composite charges: each node sums its boxes' node charges, coarse to fine
        rows, cols = [], []
        for q, patch in enumerate(patches):
            slot = order.index(q)
            nxf, nyf = self.meshes[q].shape
            local = np.arange(nxf * nyf).reshape(nxf, nyf)[patch.inner]
            rows.append(patch.index.ravel())
            cols.append(node_off[slot] + local.ravel())
        rows = np.concatenate(rows)
        cols = np.concatenate(cols)
        order_rows = np.argsort(rows, kind="stable")
        self.charge_map = DeviceCSR(sparse.csr_matrix(
            (np.ones(rows.size), (rows[order_rows], cols[order_rows])),
            shape=(n, self.n_field_nodes)))  # fmt: skip
        self.volumes = torch.from_numpy(np.ascontiguousarray(layout.volumes)).to(dev)

    def _margin(self, matrices, constants, mesh):
        """The field mesh's nodes from the patches done so far (finest containing wins)."""
        xn, yn = mesh.nodes()
        x, y = xn.ravel(), yn.ravel()
        total = x.size
        n = self.layout.size
        matrix = sparse.csr_matrix((total, n))
        constant = np.zeros(total)
        for number, (done, c_done) in enumerate(zip(matrices, constants)):
            patch = self.layout.patches[number]
            dmesh = self.meshes[number]
            x0, y0, x1, y1 = patch.bounds
            inside = np.flatnonzero((x >= x0) & (x <= x1) & (y >= y0) & (y <= y1))
            if not inside.size:
                continue
            nxd, nyd = dmesh.shape
            s = np.asarray(dmesh.index_x(x[inside]), dtype=float)
            t = (y[inside] - dmesh.origin[1]) / dmesh.h
            i = np.clip(np.floor(s).astype(np.int64), 0, nxd - 2)
            j = np.clip(np.floor(t).astype(np.int64), 0, nyd - 2)
            u, w = s - i, t - j
            rows = np.tile(np.arange(inside.size), 4)
            cols = np.concatenate([i * nyd + j, i * nyd + j + 1, (i + 1) * nyd + j,
                                   (i + 1) * nyd + j + 1])  # fmt: skip
            vals = np.concatenate([(1 - u) * (1 - w), (1 - u) * w, u * (1 - w), u * w])
            weights = sparse.csr_matrix((vals, (rows, cols)), shape=(inside.size, nxd * nyd))
            part = (weights @ done).tocsr()
            part_c = weights @ c_done
            pick = sparse.csr_matrix((np.ones(inside.size), (inside, np.arange(inside.size))),
                                     shape=(total, inside.size))  # fmt: skip
            drop = np.ones(total)
            drop[inside] = 0.0
            matrix = (sparse.diags(drop) @ matrix + pick @ part).tocsr()
            constant = drop * constant + pick @ part_c
        return matrix, constant


class PatchedElectricField:
    """The electric field of a composite potential: a `StaggeredElectricField` per patch on
    its field mesh (``solver/refinement.py:328-387``).  At a point the field is that of the
    finest patch containing it; ``fx``, ``fy`` are the base patch's."""

    def __init__(self, layout: Layout, potential, *, maps: PatchedFieldMaps | None = None) -> None:
        import torch

        from beamtracer_b200.fields import StaggeredElectricField

        self.layout = layout
        self.patches = layout.patches
        self.maps = maps or PatchedFieldMaps(layout)
        if _lib.is_device_array(potential):
            phi = potential
        else:
            phi = torch.from_numpy(np.ascontiguousarray(potential, dtype=np.float64)).cuda()
        if tuple(phi.shape) != (layout.size,):
            raise ValueError("the potential needs the layout's composite nodes")
        self.fields = []
        for number, mesh in enumerate(self.maps.meshes):
            values = self.maps.values[number]
            self.maps.potential_maps[number].apply(phi, values)
            self.fields.append(StaggeredElectricField(
                mesh, values, _extrapolation(mesh), arrays=self.maps.arrays[number],
                out=self.maps.field_views[number]))  # fmt: skip
        self.mesh = layout.base.mesh
        self.fx_device = self.maps.fx
        self.fy_device = self.maps.fy

    @property
    def fx(self) -> np.ndarray:
        return self.fields[0].fx

    @property
    def fy(self) -> np.ndarray:
        return self.fields[0].fy

    def patch_of(self, x, y) -> np.ndarray:
        """The finest patch containing each point."""
        x, y = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
        which = np.zeros(np.shape(x), dtype=np.int64)
        for number, patch in enumerate(self.patches[1:], start=1):
            x0, y0, x1, y1 = patch.bounds
            which[(x >= x0) & (x <= x1) & (y >= y0) & (y <= y1)] = number
        return which

    def __call__(self, x, y) -> tuple[np.ndarray, np.ndarray]:
        """``(E_x, E_y)`` [V/m] at the points ``(x, y)``."""
        x = np.ascontiguousarray(x, dtype=float).ravel()
        y = np.ascontiguousarray(y, dtype=float).ravel()
        ex, ey = self.fields[0](x, y)
        ex, ey = np.array(ex), np.array(ey)
        which = self.patch_of(x, y)
        for number in range(1, len(self.patches)):
            inside = which == number
            if inside.any():
                ex[inside], ey[inside] = self.fields[number](x[inside], y[inside])
        return ex, ey


def composite_density(maps: PatchedFieldMaps, charge, out) -> None:
    """``out`` (composite) <- the patches' node charges ``charge`` (flat, finest first) summed
    on the composite nodes (coarse to fine), not yet divided by the volumes."""
    maps.charge_map.apply(charge.reshape(-1), out)
