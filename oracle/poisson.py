"""ORACLE (test infrastructure): the field solve, restated with SciPy's sparse LU.

The operator is the finite-volume Laplacian the reference solves with patchwork's
``NodalPoisson`` (``solver/poisson.py:1-24, 491-534``; patchwork itself, ``patchwork-amr
0.2.0`` at ``e8ed9cb2``, is not in this container, so its operator is restated from the
reference's documented form -- parity of the cut rows is pinned only by the analytic
cases of the reference's tests).  Per free node, in the form ``A phi = rho / eps0 + c``
with ``A = -laplacian``:

- along x (and along y in planar geometry), a node with four cells takes Shortley and
  Weller's row with the bracketed surface distances ``alpha``, ``beta`` (fractions of the
  node's two edges): ``2 / ((d- + d+) d-)`` and ``2 / ((d- + d+) d+)`` on its neighbours,
  ``d = alpha h-``, ``beta h+``; a node on a domain face takes the cut edge's two-point flux
  over its control length ``(h- + h+) / 2``: ``1 / (L d-)``, ``1 / (L d+)``;
- along the radius (cylindrical, ``r_j = j h``): ``(2/alpha - 1/j) / ((alpha + beta) h^2)`` and
  ``(2/beta + 1/j) / ((alpha + beta) h^2)`` with four cells, ``(1 - 1/2j) / (alpha h^2)`` and
  ``(1 + 1/2j) / (beta h^2)`` on a face; ``4 / (beta h^2)`` towards ``r_1`` on the axis;
- on a Neumann face the missing neighbour is the mirror image: the inner neighbour's
  coefficient doubles (``2 / (h d)``), and the outward normal derivative g adds
  ``2 g / h`` to the source (``(1 + 1/2j) 2 g / h`` on the cylinder's outer wall);
- a fixed node (electrode, Dirichlet face, initial-plasma region) has the row
  ``phi = value``.

The Boltzmann species (``poisson.py:76-141, 860-933``) adds
``s a exp(min(-s (phi - U_p) / T, 50))`` (``a = rho_0 / eps0``) to the source of every free
node; Newton's method (a full Newton step with a fresh LU factorisation each step) stops
when the largest update is below the tolerance.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy import sparse
from scipy.constants import epsilon_0
from scipy.sparse.linalg import splu


@dataclass
class Operator:
    """The assembled operator of a mesh: ``A`` (CSR), the face source ``c``, the fixed nodes."""

    A: sparse.csr_matrix
    c: np.ndarray
    fixed: np.ndarray
    value: np.ndarray
    shape: tuple[int, int]
    coefficients: tuple[np.ndarray, ...]  # cW, cE, cS, cN (nx, ny)


def coefficients(x, h, cylindrical, fixed, distance, neumann=(0.0, 0.0, 0.0, 0.0), j0=0):
    """The four neighbour coefficients and the face source of every node (see the module).

    ``j0`` is the radial index ``r_0 / h`` of the first row (a refined patch off the axis,
    cylindrical geometry): the radial weights take ``j + j0``, and a first row off the axis
    takes the face row ``2 / (beta h^2)`` (a patch's side inside the domain, whose rows the
    composite operator does not use)."""
    x = np.asarray(x, dtype=float)
    nx, ny = fixed.shape
    cw, ce, cs, cn = (np.zeros((nx, ny)) for _ in range(4))
    src = np.zeros((nx, ny))
    i = np.arange(nx)[:, None] * np.ones((1, ny), dtype=int)
    j = np.ones((nx, 1), dtype=int) * np.arange(ny)[None, :]
    hx = np.diff(x)
    h_lo = np.where(i > 0, hx[np.clip(i - 1, 0, nx - 2)], 0.0)
    h_hi = np.where(i < nx - 1, hx[np.clip(i, 0, nx - 2)], 0.0)
    alpha_x, beta_x, alpha_y, beta_y = distance
    four = (i > 0) & (i < nx - 1) & (j > 0) & (j < ny - 1)
    # -- x
    inner = (i > 0) & (i < nx - 1)
    dm = alpha_x * h_lo
    dp = beta_x * h_hi
    with np.errstate(divide="ignore", invalid="ignore"):
        sw_m = 2.0 / ((dm + dp) * dm)
        sw_p = 2.0 / ((dm + dp) * dp)
        length = 0.5 * (h_lo + h_hi)
        tp_m = 1.0 / (length * dm)
        tp_p = 1.0 / (length * dp)
        cw = np.where(inner, np.where(four, sw_m, tp_m), 0.0)
        ce = np.where(inner, np.where(four, sw_p, tp_p), 0.0)
        first, last = i == 0, i == nx - 1
        ce = np.where(first, 2.0 / (h_hi * dp), ce)
        cw = np.where(last, 2.0 / (h_lo * dm), cw)
        src += np.where(first, 2.0 * neumann[0] / np.where(first, h_hi, 1.0), 0.0)
        src += np.where(last, 2.0 * neumann[1] / np.where(last, h_lo, 1.0), 0.0)
        # -- y
        a, b = alpha_y, beta_y
        mid = (j > 0) & (j < ny - 1)
        bottom, top = j == 0, j == ny - 1
        if not cylindrical:
            dm, dp = a * h, b * h
            cs = np.where(mid, np.where(four, 2.0 / ((dm + dp) * dm), 1.0 / (h * dm)), 0.0)
            cn = np.where(mid, np.where(four, 2.0 / ((dm + dp) * dp), 1.0 / (h * dp)), 0.0)
            cn = np.where(bottom, 2.0 / (h * dp), cn)
            cs = np.where(top, 2.0 / (h * dm), cs)
            src += np.where(bottom, 2.0 * neumann[2] / h, 0.0)
            src += np.where(top, 2.0 * neumann[3] / h, 0.0)
        else:
            jj = np.maximum(j + j0, 1).astype(float)
            h2 = h * h
            sw_s = (2.0 / a - 1.0 / jj) / ((a + b) * h2)
            sw_n = (2.0 / b + 1.0 / jj) / ((a + b) * h2)
            tp_s = (1.0 - 0.5 / jj) / (a * h2)
            tp_n = (1.0 + 0.5 / jj) / (b * h2)
            cs = np.where(mid, np.where(four, sw_s, tp_s), 0.0)
            cn = np.where(mid, np.where(four, sw_n, tp_n), 0.0)
            cn = np.where(bottom, (4.0 if j0 == 0 else 2.0) / (b * h2), cn)
            cs = np.where(top, 2.0 / (a * h2), cs)
            src += np.where(top, (1.0 + 0.5 / jj) * 2.0 * neumann[3] / h, 0.0)
    free = ~np.asarray(fixed, dtype=bool)
    out = [np.where(free, c, 0.0) for c in (cw, ce, cs, cn)]
    return (*out, np.where(free, src, 0.0))


def assemble(x, h, cylindrical, fixed, value, distance, neumann=(0.0, 0.0, 0.0, 0.0), j0=0):
    """The operator of a classified mesh (``fixed``, ``value`` and ``distance`` as the
    mesh's ``fixed``, ``fixed_value``, ``distance``)."""
    fixed = np.asarray(fixed, dtype=bool)
    nx, ny = fixed.shape
    cw, ce, cs, cn, src = coefficients(x, h, cylindrical, fixed, distance, neumann, j0)
    n = nx * ny
    idx = np.arange(n).reshape(nx, ny)
    diag = cw + ce + cs + cn
    diag = np.where(fixed, 1.0, diag)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [diag.ravel()]
    for coef, di, dj in ((cw, -1, 0), (ce, 1, 0), (cs, 0, -1), (cn, 0, 1)):
        m = coef != 0.0
        ii, jj = np.nonzero(m)
        rows.append(idx[ii, jj])
        cols.append(idx[ii + di, jj + dj])
        vals.append(-coef[ii, jj])
    A = sparse.csr_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)
    )
    return Operator(A, src.ravel(), fixed.ravel(), np.asarray(value, float).ravel(), (nx, ny),
                    (cw, ce, cs, cn))  # fmt: skip


def _rhs(op: Operator, rho) -> np.ndarray:
    b = op.c.copy()
    if rho is not None:
        b += np.asarray(rho, dtype=float).ravel() / epsilon_0
    b[op.fixed] = op.value[op.fixed]
    return b


def _reduced_solve(matrix: sparse.csr_matrix, rhs: np.ndarray, fixed: np.ndarray,
                   known: np.ndarray) -> np.ndarray:
    """Solve ``matrix x = rhs`` with the entries at ``fixed`` known: LU on the free block."""
    free = ~fixed
    out = np.where(fixed, known, 0.0)
    block = matrix[free][:, free].tocsc()
    coupled = matrix[free][:, fixed] @ known[fixed]
    out[free] = splu(block).solve(rhs[free] - coupled)
    return out


def solve(op: Operator, rho=None) -> np.ndarray:
    """The potential of the charge density ``rho`` (nx, ny) [C/m^3] (the linear solve)."""
    b = _rhs(op, rho)
    return _reduced_solve(op.A, b, op.fixed, op.value).reshape(op.shape)


def solve_newton(
    op: Operator, rho, amplitude, temperature, up, sign, initial=None, tol=1e-10,
    max_newton=100,
):  # fmt: skip
    """The potential with the Boltzmann species ``sign * amplitude exp(-sign (phi - up) / T)``
    (``amplitude = rho_0 / eps0``) in the source; Newton from ``initial`` (default: the
    linear solution).  Returns the potential and the Newton steps taken."""
    b = _rhs(op, rho)
    free = ~op.fixed
    phi = solve(op, rho).ravel() if initial is None else np.array(initial, float).ravel()
    phi[op.fixed] = op.value[op.fixed]
    steps = 0
    for steps in range(1, max_newton + 1):
        e = amplitude * np.exp(np.minimum(-sign * (phi - up) / temperature, 50.0))
        residual = op.A @ phi - b - np.where(free, sign * e, 0.0)
        residual[op.fixed] = 0.0
        jac = (op.A + sparse.diags(np.where(free, e / temperature, 0.0))).tocsr()
        delta = _reduced_solve(jac, -residual, op.fixed, np.zeros_like(phi))
        phi += delta
        if np.max(np.abs(delta)) < tol:
            break
    return phi.reshape(op.shape), steps


def operator_of_mesh(mesh, region=None, region_value=0.0) -> Operator:
    """The operator of a classified ``IonOpticsMesh``; ``region`` (nx, ny) bool: extra nodes
    held at ``region_value`` (the initial plasma), except those the mesh already fixes."""
    fixed = np.array(mesh.fixed, dtype=bool)
    value = np.array(mesh.fixed_value, dtype=float)
    if region is not None:
        extra = np.asarray(region, dtype=bool) & ~fixed
        fixed |= extra
        value[extra] = region_value
    neumann = [
        0.0 if mesh.faces[f].kind != "neumann" or callable(mesh.faces[f].value)
        else float(mesh.faces[f].value)
        for f in ("x_min", "x_max", "y_min", "y_max")
    ]  # fmt: skip
    j0 = int(round(mesh.origin[1] / mesh.h)) if mesh.cylindrical else 0
    return assemble(mesh.x, mesh.h, mesh.cylindrical, fixed, value, mesh.distance, neumann, j0)
