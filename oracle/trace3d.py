"""Oracle (test infrastructure only): the 3D trajectory tracer restated in plain Python.

It restates the reference's ``kernels/trace_trajectories_3d/trace_trajectories_3d_pyccel.py``
(lines 19-657): the same arguments, the same steps and the same floating-point expressions in
the same order -- the results must be the same numbers -- organised as small functions.  Only
the tests call it, on small cases (pure-Python loops); the product never imports ``oracle/``.

The one function the reference kernel takes from a dependency absent here,
``mpiparticles``' ``relativistic_boris_update``, is `boris_push` below: the relativistic
Boris push as published (J. P. Boris, 1970; kick, rotation by ``t = b / gamma`` with
``s = 2 t / (1 + t^2)``, kick).  The Runge--Kutta path needs only the Lorentz factor; the
Boris path's parity with the reference is as good as that stand-in.
"""

from __future__ import annotations

from math import floor, sqrt


def lorentz(u0: float, u1: float, u2: float, inv_c2: float) -> float:
    """gamma of a proper velocity (1 for inv_c2 = 0)."""
    return sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2)


def boris_push(u0, u1, u2, e0, e1, e2, b0, b1, b2, inv_c2):
    """The relativistic Boris push of u by the scaled fields e (kicks) and b (rotation)."""
    m0, m1, m2 = u0 + e0, u1 + e1, u2 + e2
    g = sqrt(1.0 + (m0 * m0 + m1 * m1 + m2 * m2) * inv_c2)
    t0, t1, t2 = b0 / g, b1 / g, b2 / g
    f = 2.0 / (1.0 + (t0 * t0 + t1 * t1 + t2 * t2))
    s0, s1, s2 = f * t0, f * t1, f * t2
    p0 = m0 + (m1 * t2 - m2 * t1)
    p1 = m1 + (m2 * t0 - m0 * t2)
    p2 = m2 + (m0 * t1 - m1 * t0)
    return (m0 + (p1 * s2 - p2 * s1) + e0, m1 + (p2 * s0 - p0 * s2) + e1,
            m2 + (p0 * s1 - p1 * s0) + e2)  # fmt: skip


def _clamp(i: int, lo: int, hi: int) -> int:
    return lo if i < lo else (hi if i > hi else i)


def _finest(patch_real, n_patches: int, p0: float, p1: float, p2: float) -> int:
    """The first (finest) patch whose node box holds the point, else the base (last)."""
    for q in range(n_patches - 1):
        r = patch_real[q]
        if r[4] <= p0 <= r[7] and r[5] <= p1 <= r[8] and r[6] <= p2 <= r[9]:
            return q
    return n_patches - 1


def _trilinear(f, ci: int, dj: int, di: int, a: float, b: float, c: float) -> float:
    """The reference's nested trilinear form (``:231-236``) at corner index ci."""
    return ((1.0 - a) * ((1.0 - b) * ((1.0 - c) * f[ci] + c * f[ci + 1])
                         + b * ((1.0 - c) * f[ci + dj] + c * f[ci + dj + 1]))
            + a * ((1.0 - b) * ((1.0 - c) * f[ci + di] + c * f[ci + di + 1])
                   + b * ((1.0 - c) * f[ci + di + dj] + c * f[ci + di + dj + 1])))  # fmt: skip


class _Args:
    """The kernel's 41 arguments by name (``trace_trajectories_3d_pyccel.py:19-61``)."""

    NAMES = ("active x v qm dq steps status electrode fxs fys fzs patch_int patch_real bn "
             "has_b origin_x origin_y origin_z h upper_x upper_y upper_z mirror_y mirror_z "
             "integrator step_fraction max_steps cells subcells refine planes hits counts "
             "path_slot paths path_count num_threads charge has_j current inv_c2").split()

    def __init__(self, args) -> None:
        for name, value in zip(self.NAMES, args, strict=True):
            setattr(self, name, value)


def _fields(a: _Args, p0: float, p1: float, p2: float):
    """E (and B) at a point: mirrored below a symmetry plane, from the finest patch
    (``:173-335``)."""
    s1 = s2 = 1.0
    if a.mirror_y != 0 and p1 < a.origin_y:
        p1, s1 = 2.0 * a.origin_y - p1, -1.0
    if a.mirror_z != 0 and p2 < a.origin_z:
        p2, s2 = 2.0 * a.origin_z - p2, -1.0
    pp = _finest(a.patch_real, a.patch_int.shape[0], p0, p1, p2)
    pnx, pny, pnz, ofx, ofy, ofz = (int(v) for v in a.patch_int[pp, :6])
    pox, poy, poz, phh = (float(v) for v in a.patch_real[pp, :4])
    sx, sy, sz = (p0 - pox) / phh, (p1 - poy) / phh, (p2 - poz) / phh
    # E_x at (sx + 1/2, sy, sz)
    s = sx + 0.5
    i = _clamp(floor(s), 0, pnx - 1)
    j = _clamp(floor(sy), 0, pny - 2)
    k = _clamp(floor(sz), 0, pnz - 2)
    c = sz - k
    e0 = _trilinear(a.fxs, ofx + i * pny * pnz + j * pnz + k, pnz, pny * pnz, s - i, sy - j, c)
    # E_y at (sx, sy + 1/2, sz)
    i = _clamp(floor(sx), 0, pnx - 2)
    s = sy + 0.5
    j = _clamp(floor(s), 0, pny - 1)
    ax = sx - i
    di = (pny + 1) * pnz
    e1 = s1 * _trilinear(a.fys, ofy + i * di + j * pnz + k, pnz, di, ax, s - j, c)
    # E_z at (sx, sy, sz + 1/2)
    j = _clamp(floor(sy), 0, pny - 2)
    s = sz + 0.5
    k = _clamp(floor(s), 0, pnz - 1)
    di = pny * (pnz + 1)
    e2 = s2 * _trilinear(a.fzs, ofz + i * di + j * (pnz + 1) + k, pnz + 1, di, ax, sy - j, s - k)
    b = (0.0, 0.0, 0.0)
    if a.has_b != 0:
        nx, ny, nz = (int(v) for v in a.patch_int[-1, :3])
        tx, ty, tz = (p0 - a.origin_x) / a.h, (p1 - a.origin_y) / a.h, (p2 - a.origin_z) / a.h
        i = _clamp(floor(tx), 0, nx - 2)
        j = _clamp(floor(ty), 0, ny - 2)
        k = _clamp(floor(tz), 0, nz - 2)
        u, w, z = tx - i, ty - j, tz - k
        weights = ((1.0 - u) * (1.0 - w) * (1.0 - z), (1.0 - u) * (1.0 - w) * z,
                   (1.0 - u) * w * (1.0 - z), (1.0 - u) * w * z, u * (1.0 - w) * (1.0 - z),
                   u * (1.0 - w) * z, u * w * (1.0 - z), u * w * z)  # fmt: skip
        corners = ((0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0),
                   (1, 1, 1))  # fmt: skip
        comp = []
        for n0 in range(3):
            f = 0.0
            for q, (ci, cj, ck) in enumerate(corners):
                term = weights[q] * a.bn[n0, i + ci, j + cj, k + ck]
                f = term if q == 0 else f + term
            comp.append(f)
        b = (s1 * s2 * comp[0], s2 * comp[1], s1 * comp[2])
    return (e0, e1, e2), b


def _deposit_box(a: _Args, m0: float, m1: float, m2: float):
    """The patch, corner node and weights of a deposit point (``:466-510``)."""
    if a.mirror_y != 0 and m1 < a.origin_y:
        m1 = 2.0 * a.origin_y - m1
    if a.mirror_z != 0 and m2 < a.origin_z:
        m2 = 2.0 * a.origin_z - m2
    pp = _finest(a.patch_real, a.patch_int.shape[0], m0, m1, m2)
    pnx, pny, pnz = (int(v) for v in a.patch_int[pp, :3])
    ofn = int(a.patch_int[pp, 7])
    r = a.patch_real[pp]
    phh = r[3]
    sx, sy, sz = (m0 - r[0]) / phh, (m1 - r[1]) / phh, (m2 - r[2]) / phh
    out = []
    for s, n in ((sx, pnx), (sy, pny), (sz, pnz)):
        i = floor(s)
        w = s - i
        if i < 0:
            w, i = 0.0, 0
        elif i >= n - 1:
            w, i = 1.0, n - 2
        out.append((i, w))
    (i, wa), (j, wb), (k, wc) = out
    return ofn + i * pny * pnz + j * pnz + k, pnz, pny * pnz, wa, wb, wc


def _add8(target, t: int, cc: int, dj: int, di: int, a: float, b: float, c: float, q: float):
    """The eight trilinear shares of q, in the reference's order (``:512-519``)."""
    target[t, cc] += (1.0 - a) * (1.0 - b) * (1.0 - c) * q
    target[t, cc + 1] += (1.0 - a) * (1.0 - b) * c * q
    target[t, cc + dj] += (1.0 - a) * b * (1.0 - c) * q
    target[t, cc + dj + 1] += (1.0 - a) * b * c * q
    target[t, cc + di] += a * (1.0 - b) * (1.0 - c) * q
    target[t, cc + di + 1] += a * (1.0 - b) * c * q
    target[t, cc + di + dj] += a * b * (1.0 - c) * q
    target[t, cc + di + dj + 1] += a * b * c * q


def _step(a: _Args, k: int, x, v, hloc: float, cache):
    """One step from (x, v): RK4 (four field evaluations) or Boris (kick--rotate--kick
    half steps around the drift, the end's fields kept for the next start); returns the new
    state, dt, 1/gamma at both ends and the cache (``:167-447``)."""
    x0, x1, x2 = x
    v0, v1, v2 = v
    qmk = a.qm[k]
    inv_c2 = a.inv_c2
    gv = 1.0 / lorentz(v0, v1, v2, inv_c2)

    def accel(kx0, kx1, kx2, e, b):
        gk = 1.0 / lorentz(kx0, kx1, kx2, inv_c2)
        return gk, (qmk * (e[0] + gk * kx1 * b[2] - gk * kx2 * b[1]),
                    qmk * (e[1] + gk * kx2 * b[0] - gk * kx0 * b[2]),
                    qmk * (e[2] + gk * kx0 * b[1] - gk * kx1 * b[0]))  # fmt: skip

    if a.integrator != 0 and cache is not None:
        e, b = cache
    else:
        e, b = _fields(a, x0, x1, x2)
    _, g = accel(v0, v1, v2, e, b)
    speed = gv * sqrt(v0 * v0 + v1 * v1 + v2 * v2)
    acc = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
    dt = -1.0
    if speed > 0.0:
        dt = hloc / speed
    if acc > 0.0:
        d2 = sqrt(2.0 * hloc / acc)
        if dt < 0.0 or d2 < dt:
            dt = d2
    if dt < 0.0:
        dt = hloc
    dt = a.step_fraction * dt
    hdt = 0.5 * dt
    if a.integrator != 0:
        tau = 0.5 * hdt * qmk
        k0, k1, k2 = boris_push(v0, v1, v2, tau * e[0], tau * e[1], tau * e[2],
                                tau * b[0], tau * b[1], tau * b[2], inv_c2)  # fmt: skip
        gk = 1.0 / lorentz(k0, k1, k2, inv_c2)
        y = (x0 + dt * gk * k0, x1 + dt * gk * k1, x2 + dt * gk * k2)
        e, b = _fields(a, *y)
        w = boris_push(k0, k1, k2, tau * e[0], tau * e[1], tau * e[2],
                       tau * b[0], tau * b[1], tau * b[2], inv_c2)  # fmt: skip
        return y, w, dt, gv, (e, b)
    dt6 = dt / 6.0
    sx = [gv * v0, gv * v1, gv * v2]
    sv = list(g)
    q = (x0 + hdt * gv * v0, x1 + hdt * gv * v1, x2 + hdt * gv * v2)
    kx = (v0 + hdt * g[0], v1 + hdt * g[1], v2 + hdt * g[2])
    for stage in (1, 2, 3):
        e, b = _fields(a, *q)
        gk, g = accel(*kx, e, b)
        if stage < 3:
            for c in range(3):
                sx[c] = sx[c] + 2.0 * gk * kx[c]
                sv[c] = sv[c] + 2.0 * g[c]
            f = hdt if stage == 1 else dt
            q = (x0 + f * gk * kx[0], x1 + f * gk * kx[1], x2 + f * gk * kx[2])
            kx = (v0 + f * g[0], v1 + f * g[1], v2 + f * g[2])
        else:
            for c in range(3):
                sx[c] = sx[c] + gk * kx[c]
                sv[c] = sv[c] + g[c]
    y = (x0 + dt6 * sx[0], x1 + dt6 * sx[1], x2 + dt6 * sx[2])
    w = (v0 + dt6 * sv[0], v1 + dt6 * sv[1], v2 + dt6 * sv[2])
    return y, w, dt, gv, None


def _end_test(a: _Args, k: int, px: float, py: float, pz: float) -> int:
    """-1 to continue, else the end status of a step ending at (px, py, pz) (mirrored):
    off the mesh (0-2), in an electrode's sub-cell (3) or in one its surface cuts (-2)
    (``:599-641``)."""
    if px >= a.upper_x:
        return 0
    if px < a.origin_x:
        return 1
    if py > a.upper_y or py < a.origin_y or pz > a.upper_z or pz < a.origin_z:
        return 2
    nx, ny, nz = (int(c) for c in a.patch_int[-1, :3])
    R = a.refine
    ux, uy, uz = (px - a.origin_x) / a.h, (py - a.origin_y) / a.h, (pz - a.origin_z) / a.h
    i, j, kz = min(int(ux), nx - 2), min(int(uy), ny - 2), min(int(uz), nz - 2)
    cell = a.cells[i, j, kz]
    if cell < 0:
        return -1
    si = _clamp(int((ux - i) * R), 0, R - 1)
    sj = _clamp(int((uy - j) * R), 0, R - 1)
    sk = _clamp(int((uz - kz) * R), 0, R - 1)
    e = a.subcells[((cell * R + si) * R + sj) * R + sk]
    if e >= 0:
        a.electrode[k] = e
        return 3
    return -2 if e == -2 else -1


def trace_trajectories_3d(*args) -> None:
    """The reference kernel's effect on its arguments (updated in place)."""
    a = _Args(args)
    n_patches = a.patch_int.shape[0]
    nx, ny, nz = (int(c) for c in a.patch_int[-1, :3])
    capacity, path_capacity = a.hits.shape[2], a.paths.shape[1]
    for t in range(a.num_threads):
        for m in range(t, a.active.shape[0], a.num_threads):
            k = int(a.active[m])
            x = (a.x[0, k], a.x[1, k], a.x[2, k])
            v = (a.v[0, k], a.v[1, k], a.v[2, k])
            slot = int(a.path_slot[k])
            ns = int(a.steps[k])
            st = -1
            cache = None
            while ns < a.max_steps:
                p1, p2 = x[1], x[2]
                if a.mirror_y != 0 and p1 < a.origin_y:
                    p1 = 2.0 * a.origin_y - p1
                if a.mirror_z != 0 and p2 < a.origin_z:
                    p2 = 2.0 * a.origin_z - p2
                hloc = a.h
                q = _finest(a.patch_real, n_patches, x[0], p1, p2)
                if q < n_patches - 1:
                    hloc = a.patch_real[q, 3]
                y, w, dt, gv, cache = _step(a, k, x, v, hloc, cache)
                gw = 1.0 / lorentz(w[0], w[1], w[2], a.inv_c2)
                mid = [0.5 * (x[c] + y[c]) + dt * (gv * v[c] - gw * w[c]) / 8.0 for c in range(3)]
                cc, dj, di, wa, wb, wc = _deposit_box(a, *mid)
                _add8(a.charge, t, cc, dj, di, wa, wb, wc, a.dq[k] * dt)
                if a.has_j != 0:
                    jd = [a.dq[k] * (y[c] - x[c]) for c in range(3)]
                    if a.mirror_y != 0 and 0.5 * (x[1] + y[1]) < a.origin_y:
                        jd[1] = -jd[1]
                    if a.mirror_z != 0 and 0.5 * (x[2] + y[2]) < a.origin_z:
                        jd[2] = -jd[2]
                    m1, m2 = mid[1], mid[2]
                    if a.mirror_y != 0 and m1 < a.origin_y:
                        m1 = 2.0 * a.origin_y - m1
                    if a.mirror_z != 0 and m2 < a.origin_z:
                        m2 = 2.0 * a.origin_z - m2
                    box = []
                    for s, n in (((mid[0] - a.origin_x) / a.h, nx), ((m1 - a.origin_y) / a.h, ny),
                                 ((m2 - a.origin_z) / a.h, nz)):  # fmt: skip
                        i = floor(s)
                        f = s - i
                        if i < 0:
                            f, i = 0.0, 0
                        elif i >= n - 1:
                            f, i = 1.0, n - 2
                        box.append((i, f))
                    (bi, ba), (bj, bb), (bk, bc) = box
                    for jc in range(3):
                        _add8(a.current, t, jc * nx * ny * nz + bi * ny * nz + bj * nz + bk, nz,
                              ny * nz, ba, bb, bc, jd[jc])  # fmt: skip
                ns += 1
                for p, xp in enumerate(a.planes):
                    before, after = x[0] - xp, y[0] - xp
                    if (before < 0.0) != (after < 0.0):
                        s = before / (before - after)
                        c = int(a.counts[k, p])
                        if c < capacity:
                            a.hits[k, p, c] = (
                                xp, x[1] + s * (y[1] - x[1]), x[2] + s * (y[2] - x[2]),
                                gv * v[0] + s * (gw * w[0] - gv * v[0]),
                                gv * v[1] + s * (gw * w[1] - gv * v[1]),
                                gv * v[2] + s * (gw * w[2] - gv * v[2]),
                                1.0 if after >= 0.0 else -1.0, 1.0 * ns)  # fmt: skip
                        a.counts[k, p] = c + 1
                x, v = y, w
                px, py, pz = x
                if a.mirror_y != 0 and py < a.origin_y:
                    py = 2.0 * a.origin_y - py
                if a.mirror_z != 0 and pz < a.origin_z:
                    pz = 2.0 * a.origin_z - pz
                if slot >= 0:
                    c = int(a.path_count[slot])
                    if c < path_capacity:
                        a.paths[slot, c] = (px, py, pz)
                    a.path_count[slot] = c + 1
                st = _end_test(a, k, px, py, pz)
                if st != -1:
                    break
            if st == -1:
                st = 4
            a.x[:, k] = x
            a.v[:, k] = v
            a.steps[k] = ns
            a.status[k] = st
