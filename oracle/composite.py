"""ORACLE (test infrastructure): the field solve on refined boxes, with SciPy's sparse LU.

The composite operator of a `beamtracer_b200.refinement.Layout` assembled on the host and
solved directly.  The reference solves refined boxes with patchwork's composite
``NodalPoisson`` (``solver/poisson.py:169-335``, ``solver/refinement.py:155-296``);
patchwork (``patchwork-amr 0.2.0`` at ``e8ed9cb2``) is not in this container, so the
composite scheme is restated from its definition and pinned only by the reference's
known answers for refined boxes (``tests/unit/test_refinement.py:57-131``: the volumes fill
the domain; a uniform charge between plates within 1e-2 of the parabola, the error falling
with the cells):

- a node's equation is its owner patch's row of the operator of ``oracle/poisson.py``
  (``A phi = rho / eps0 + c``) on that patch's mesh, its neighbours the patch's nodes;
- a held node (electrode, Dirichlet face) keeps its value;
- a hanging node equals the interpolation of the nodes it hangs from.
"""

from __future__ import annotations

import numpy as np
from scipy import sparse
from scipy.constants import epsilon_0
from scipy.sparse.linalg import splu

from oracle import poisson as oracle_poisson


def _patch_rows(patch):
    """The patch's neighbour coefficients ``(cw, ce, cs, cn)`` and face source."""
    mesh = patch.mesh
    op = oracle_poisson.operator_of_mesh(mesh)
    return op.coefficients, op.c.reshape(mesh.shape)


def assemble(layout, rho=None):
    """The composite matrix and right-hand side for the charge density ``rho`` (composite
    nodes, C/m^3, or None).  The matrix, the held values and the face sources depend on
    the layout alone and are assembled once per layout."""
    n = layout.size
    rho = np.zeros(n) if rho is None else np.asarray(rho, dtype=float)
    cached = _ASSEMBLED.get(id(layout))
    if cached is None or cached[0] is not layout:
        cached = (layout, *_assemble_fixed(layout))
        _ASSEMBLED.clear()  # one layout at a time: no stale entries under a reused id
        _ASSEMBLED[id(layout)] = cached
    _, K, b0, charged = cached
    b = b0.copy()
    b[charged] += rho[charged] / epsilon_0
    return K, b


#: the last layout's assembled matrix, fixed right-hand side and charged rows
_ASSEMBLED: dict = {}


def _assemble_fixed(layout):
    """The composite matrix, the right-hand side without charge and the rows that take
    ``rho / eps0`` (the nodes with an equation of their own)."""
    n = layout.size
    rho = np.zeros(n)
    hang_row = {int(k): r for r, k in enumerate(layout.hanging)}
    interp = layout.interpolation.tocsr()

    def expand(k):
        r = hang_row.get(int(k))
        if r is None:
            return [(int(k), 1.0)]
        lo, hi = interp.indptr[r], interp.indptr[r + 1]
        return list(zip(interp.indices[lo:hi].tolist(), interp.data[lo:hi].tolist()))

    rows, cols, vals = [], [], []
    b = np.zeros(n)
    rows_of = [_patch_rows(p) for p in layout.patches]
    for k in range(n):
        p = int(layout.owner[k])
        if p < 0:  # hanging: phi_k - sum w phi_src = 0
            rows.append(k)
            cols.append(k)
            vals.append(1.0)
            for src, w in expand(k):
                rows.append(k)
                cols.append(src)
                vals.append(-w)
            continue
        if layout.fixed[k]:
            rows.append(k)
            cols.append(k)
            vals.append(1.0)
            b[k] = layout.fixed_value[k]
            continue
        patch = layout.patches[p]
        (cw, ce, cs, cn), src = rows_of[p]
        nyp = patch.mesh.shape[1]
        a, c = divmod(int(layout.owner_node[k]), nyp)
        diag = cw[a, c] + ce[a, c] + cs[a, c] + cn[a, c]
        rows.append(k)
        cols.append(k)
        vals.append(diag)
        for coef, da, dc in ((cw, -1, 0), (ce, 1, 0), (cs, 0, -1), (cn, 0, 1)):
            value = coef[a, c]
            if value == 0.0:
                continue
            for node, w in expand(patch.index[a + da, c + dc]):
                rows.append(k)
                cols.append(node)
                vals.append(-value * w)
        b[k] = rho[k] / epsilon_0 + src[a, c]
    K = sparse.csr_matrix((vals, (rows, cols)), shape=(n, n))
    charged = (layout.owner >= 0) & ~np.asarray(layout.fixed, dtype=bool)
    return K, b, charged


def solve(layout, rho=None) -> np.ndarray:
    """The composite potential for the charge density ``rho`` (composite nodes).

    LU of the row-equilibrated matrix (its held and hanging rows are of order 1, its
    operator rows of order ``1 / h^2``) and three steps of iterative refinement: the plain
    factorisation of the mixed rows is off by ~1e-7 of the potential's scale."""
    K, b = assemble(layout, rho)
    scale = 1.0 / abs(K).max(axis=1).toarray().ravel()
    Ks = (sparse.diags(scale) @ K).tocsc()
    lu = splu(Ks)
    phi = lu.solve(scale * b)
    for _ in range(3):
        phi += lu.solve(scale * (b - K @ phi))
    return phi


def residual(layout, phi, rho=None) -> np.ndarray:
    """``b - K phi`` of the composite system (held and hanging rows included)."""
    K, b = assemble(layout, rho)
    return b - K @ np.asarray(phi, dtype=float)


# -- the field and the Vlasov iteration on refined boxes -----------------------------------


def _faces(mesh) -> list[str]:
    """``solver/refinement.py:289-295``: mirrored on y_min on the axis or a symmetry plane."""
    faces = ["extrapolate"] * 4
    if (mesh.cylindrical and abs(mesh.origin[1]) <= 1e-12 * mesh.h) or mesh.symmetry_plane:
        faces[2] = "symmetric"
    return faces


def field_values(layout, potential) -> list[np.ndarray]:
    """The potential on every patch's field mesh (``solver/refinement.py:335-365``): a box's
    own nodes from the composite potential, its margin bilinear in the patches done before
    it (the last containing the node wins), electrode nodes of the margin at their
    potential."""
    potential = np.asarray(potential, dtype=float)
    arrays, meshes = [], []
    for patch in layout.patches:
        values = potential[patch.index]
        mesh = patch.mesh if patch.field_mesh is None else patch.field_mesh
        if patch.field_mesh is not None:
            xn, yn = mesh.nodes()
            x, y = xn.ravel(), yn.ravel()
            full = np.zeros(x.size)
            for done, (dmesh, dvalues) in zip(layout.patches, zip(meshes, arrays)):
                x0, y0, x1, y1 = done.bounds
                inside = (x >= x0) & (x <= x1) & (y >= y0) & (y <= y1)
                if not inside.any():
                    continue
                nxd, nyd = dmesh.shape
                s = np.asarray(dmesh.index_x(x[inside]), dtype=float)
                t = (y[inside] - dmesh.origin[1]) / dmesh.h
                i = np.clip(np.floor(s).astype(np.int64), 0, nxd - 2)
                j = np.clip(np.floor(t).astype(np.int64), 0, nyd - 2)
                u, w = s - i, t - j
                full[inside] = ((1 - u) * (1 - w) * dvalues[i, j] + (1 - u) * w * dvalues[i, j + 1]
                                + u * (1 - w) * dvalues[i + 1, j] + u * w * dvalues[i + 1, j + 1])  # fmt: skip
            full = full.reshape(mesh.shape)
            solid = np.asarray(mesh.solid) >= 0
            full[solid] = np.asarray(mesh.fixed_value)[solid]
            full[patch.inner] = values
            values = full
        arrays.append(values)
        meshes.append(mesh)
    return arrays


def edge_fields(layout, potential):
    """Every patch's edge fields ``(fx, fy)`` (coarse to fine) and field meshes."""
    from oracle import field as oracle_field

    out = []
    meshes = []
    for patch, values in zip(layout.patches, field_values(layout, potential)):
        mesh = patch.mesh if patch.field_mesh is None else patch.field_mesh
        out.append(oracle_field.edge_fields(values, np.asarray(mesh.solid),
                                            np.asarray(mesh.near_solid), np.asarray(mesh.distance),
                                            np.diff(mesh.x), mesh.h, _faces(mesh)))  # fmt: skip
        meshes.append(mesh)
    return out, meshes


def trace_tables(layout, fields, meshes):
    """The kernel's patch tables and flat edge fields, finest first (``tracer.py:1141-1183``)."""
    order = list(range(len(meshes)))[::-1]
    ints, reals, fxs, fys = [], [], [], []
    fx_off = fy_off = node_off = 0
    for q in order:
        mesh = meshes[q]
        fx, fy = fields[q]
        nxf, nyf = mesh.shape
        ints.append([nxf, nyf, fx_off, fy_off, nxf * nyf, node_off])
        fx_off += fx.size
        fy_off += fy.size
        node_off += nxf * nyf
        x0, y0, x1, y1 = layout.patches[q].bounds
        base = layout.base.mesh
        reals.append([*mesh.logical_origin, mesh.h, float(base.logical_x(x0)), y0,
                      float(base.logical_x(x1)), y1])  # fmt: skip
        fxs.append(np.ravel(fx))
        fys.append(np.ravel(fy))
    return (np.array(ints, dtype=np.int64), np.array(reals, dtype=float), node_off,
            np.concatenate(fxs), np.concatenate(fys), order)  # fmt: skip


def composite_charge(layout, meshes, order, flat) -> np.ndarray:
    """The patches' node charges (flat, finest first) on the composite nodes, each box's own
    nodes only (``tracer.py:1266-1276``)."""
    offsets = {}
    start = 0
    for q in order:
        offsets[q] = start
        start += meshes[q].shape[0] * meshes[q].shape[1]
    charges = []
    for q, patch in enumerate(layout.patches):
        block = flat[offsets[q]:offsets[q] + meshes[q].shape[0] * meshes[q].shape[1]]
        charges.append(block.reshape(meshes[q].shape)[patch.inner])
    return layout.deposit_total(charges)


def density_of(p, layout, potential, particles):
    """G(phi) on refined boxes: the composite density the beam deposits in the potential."""
    from oracle import vlasov as oracle_vlasov

    fields, meshes = edge_fields(layout, potential)
    patch_int, patch_real, nodes, fxs, fys, order = trace_tables(layout, fields, meshes)
    t = oracle_vlasov.trace(p, fxs, fys, particles, patches=(patch_int, patch_real, nodes))
    return composite_charge(layout, meshes, order, t.charge) / layout.volumes, t


def vlasov(p, layout, particles, *, iterations: int, tolerance: float = 0.0,
           relaxation: float = 1.0, plasma=None, j_over_v: float = 0.0, mixing: str = "linear",
           anderson_depth: int = 5, callback=None) -> dict:  # fmt: skip
    """The Vlasov iteration on refined boxes (``vlasov.py:327-427``, linear or Anderson
    mixing as the mesh's loop mixes): the first iteration with a plasma holds the nodes
    below its initial x at the plasma potential, the later ones solve with its Boltzmann
    species by Newton's method from the last potential; the composite potential and
    density of the last iteration and the
    history."""
    from scipy import constants

    from oracle import vlasov as oracle_vlasov

    mixer = oracle_vlasov.Anderson(anderson_depth, relaxation) if mixing == "anderson" else None
    rho = np.zeros(layout.size)
    potential = None
    history = []
    out: dict = {}
    for iteration in range(iterations):
        if plasma is not None and iteration == 0:
            new = solve_region(layout, rho, lambda x, y: x < plasma.initial_x, plasma.potential)
        elif plasma is not None:
            density = plasma.density if plasma.density is not None else j_over_v
            new, _ = solve_newton(layout, rho, density / constants.epsilon_0,
                                  plasma.temperature, plasma.potential, plasma.sign,
                                  initial=potential, tol=1e-11)  # fmt: skip
        else:
            new = solve(layout, rho)
        change = float("inf") if potential is None else float(np.max(np.abs(new - potential)))
        potential = new
        deposit, t = density_of(p, layout, potential, particles)
        if iteration == 0:
            rho = deposit
        elif mixer is not None:
            rho = mixer.update(rho, deposit)
        else:
            rho = (1.0 - relaxation) * rho + relaxation * deposit
        history.append({"iteration": iteration, "max_potential_change": change})
        out = {"potential": potential, "charge_density": rho, "deposit": deposit, "trace": t,
               "history": history}  # fmt: skip
        if callback is not None:
            callback(iteration, out)
        if change < tolerance:
            break
    return out


def held_region(layout, region) -> np.ndarray:
    """The nodes an initial plasma region holds (``poisson.py:279-309``): ``region(x, y)``
    at the composite nodes, less those already held and the hanging ones."""
    mask = np.asarray(region(layout.x, layout.y), dtype=bool) & ~layout.fixed
    mask[layout.hanging] = False
    return mask


def _with_region(K, b, region_mask, value):
    K = K.tolil()
    for k in np.flatnonzero(region_mask):
        K.rows[k] = [int(k)]
        K.data[k] = [1.0]
    b = b.copy()
    b[region_mask] = value
    return K.tocsr(), b


def _equilibrated_solve(K, b, refine: int = 3) -> np.ndarray:
    scale = 1.0 / abs(K).max(axis=1).toarray().ravel()
    lu = splu((sparse.diags(scale) @ K).tocsc())
    x = lu.solve(scale * b)
    for _ in range(refine):
        x += lu.solve(scale * (b - K @ x))
    return x


def solve_region(layout, rho, region, value) -> np.ndarray:
    """The composite potential with the nodes of ``region`` held at ``value``."""
    K, b = assemble(layout, rho)
    K, b = _with_region(K, b, held_region(layout, region), value)
    return _equilibrated_solve(K, b)


def solve_newton(layout, rho, amplitude, temperature, up, sign, initial=None, tol=1e-11,
                 max_newton=100):  # fmt: skip
    """The composite potential with the Boltzmann species ``sign * amplitude
    exp(-sign (phi - up) / T)`` in the source of every node with an equation of its own
    (``poisson.py:860-933``): Newton from ``initial`` (default: the linear solution), a
    full step each, until the largest update is below ``tol``."""
    K, b = assemble(layout, rho)
    own = (layout.owner >= 0) & ~layout.fixed
    phi = _equilibrated_solve(K, b) if initial is None else np.array(initial, dtype=float)
    steps = 0
    for steps in range(1, max_newton + 1):
        e = amplitude * np.exp(np.minimum(-sign * (phi - up) / temperature, 50.0))
        residual = b + np.where(own, sign * e, 0.0) - K @ phi
        jac = (K + sparse.diags(np.where(own, e / temperature, 0.0))).tocsr()
        delta = _equilibrated_solve(jac, residual)
        phi += delta
        if np.max(np.abs(delta)) < tol:
            break
    return phi, steps
