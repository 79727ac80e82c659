// The trajectory tracer: kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:42-507
// re-designed for the B200.
//
// One thread per live trajectory advances it by at most `window` steps per launch (RK4 or
// Boris's kick-drift-kick through the staggered edge fields of the patches, plane
// crossings, kept paths, exit and electrode sub-cell tests: the reference's step, term by
// term, in FP64 with no contracted multiply-add, so a trajectory ends bit for bit where the
// reference's CPU kernel ends it; the only fused multiply-adds are those of `div_known`,
// whose quotients are the IEEE division's).  Instead of adding its charge to the mesh with
// atomics, every step writes one deposit record (cell, u, w, dq dt) to a slot fixed by
// (window, step, trajectory); between windows the live trajectories are compacted in order,
// and the records are sorted by cell and reduced per cell in record order (deposit.cu), so
// the node charges are deterministic.  The deposits run on a side stream under the next
// windows, in the order the record buffers were filled.  Short windows bound the tail of a
// warp (its threads wait only for the longest trajectory of the window, not of the whole
// trace).
#include <algorithm>

#include "common.cuh"

namespace bt {

namespace {

struct Trace {
    bt_trace_args a;
    i64 nx, ny;       // the last patch's node counts
    bt_magnetic mag;  // the magnetic field of the MAG kernels
    // A batch of candidate meshes (the BATCH kernels): every trajectory's candidate, and
    // where each candidate's cell table starts in a.cells.  Row c of a.patch_int /
    // a.patch_real is candidate c's one patch (shape, offsets, origin, spacing, extent).
    const int32_t *cand;
    const i64 *cell_off;
    // the candidates' electrode shapes (candidate c's: shape_first[c] .. shape_first[c + 1]
    // - 1 of `shapes`), or shape_first NULL: pause for the caller's test
    const i64 *shape_first;
    Shapes shapes;
};

__device__ __forceinline__ i64 node_cell(double x, const double *__restrict__ nodes, i64 n) {
    i64 lo = 0, hi = n - 1;
    if (x >= nodes[n - 1]) {
        lo = n - 2;
    } else if (x > nodes[0]) {
        while (hi - lo > 1) {
            const i64 mid = (lo + hi) / 2;
            if (nodes[mid] <= x)
                lo = mid;
            else
                hi = mid;
        }
    }
    return lo;
}

__device__ __forceinline__ double uniform_x(double x, const double *__restrict__ nodes, i64 n,
                                            double x0, double h) {
    const i64 c = node_cell(x, nodes, n);
    return x0 + h * ((double)c + (x - nodes[c]) / (nodes[c + 1] - nodes[c]));
}

__device__ __forceinline__ i64 finest_patch(const bt_trace_args &a, i64 P, double px, double py) {
    for (i64 qq = 0; qq < P - 1; ++qq) {
        const double *pr = a.patch_real + qq * 7;
        if (px >= __ldg(pr + 3) && px <= __ldg(pr + 5) && py >= __ldg(pr + 4) &&
            py <= __ldg(pr + 6))
            return qq;
    }
    return P - 1;
}

// A patch's shape: node counts, its offsets into the edge-field and node arrays, origin and
// spacing (one row of patch_int / patch_real), and the spacing's reciprocal for `div_known`
// (0: divide plainly).
struct PatchGeom {
    i64 pnx, pny, ofx, ofy, ofn;
    double pox, poy, phh, rphh;
};

__device__ __forceinline__ PatchGeom patch_geom(const bt_trace_args &a, i64 pp) {
    const i64 *pi = a.patch_int + pp * 6;
    const double *pr = a.patch_real + pp * 7;
    return {__ldg(pi + 0), __ldg(pi + 1), __ldg(pi + 2), __ldg(pi + 3), __ldg(pi + 5),
            __ldg(pr + 0), __ldg(pr + 1), __ldg(pr + 2), 0.0};
}

// Cell indices are 32-bit: a patch has fewer than 2^31 nodes along an axis (the deposit keys
// are 32-bit).  floor and truncation saturate outside that range, where the clamps that
// follow them give what the 64-bit conversions give.
__device__ __forceinline__ int clamp_index(int i, int lo, int hi) { return min(max(i, lo), hi); }

// E at the point (sx, sy) in cells of patch g from its origin (the finest patch holding the
// point; trace_trajectories_2d_pyccel.py:212-269).
__device__ __forceinline__ void edge_field_cells(const bt_trace_args &a, const PatchGeom &g,
                                                 double sx, double sy, double &ex, double &ey) {
    const int pnx = (int)g.pnx, pny = (int)g.pny;
    double s = sx + 0.5;
    int i = clamp_index(__double2int_rd(s), 0, pnx - 1);
    int j = clamp_index(__double2int_rd(sy), 0, pny - 2);
    double u = s - (double)i;
    double w = sy - (double)j;
    const double *fx = a.fxs + g.ofx + (i64)i * pny + j;
    double f00 = __ldg(fx), f01 = __ldg(fx + 1), f10 = __ldg(fx + pny), f11 = __ldg(fx + pny + 1);
    double low = f00 + w * (f01 - f00);
    double high = f10 + w * (f11 - f10);
    ex = low + u * (high - low);
    s = sy + 0.5;
    i = clamp_index(__double2int_rd(sx), 0, pnx - 2);
    j = clamp_index(__double2int_rd(s), 0, pny - 1);
    u = sx - (double)i;
    w = s - (double)j;
    const double *fy = a.fys + g.ofy + (i64)i * (pny + 1) + j;
    f00 = __ldg(fy);
    f01 = __ldg(fy + 1);
    f10 = __ldg(fy + pny + 1);
    f11 = __ldg(fy + pny + 2);
    low = f00 + w * (f01 - f00);
    high = f10 + w * (f11 - f10);
    ey = low + u * (high - low);
}

// E at (lq, qy), the uniform x and the mesh y, on patch g.
__device__ __forceinline__ void edge_field(const bt_trace_args &a, const PatchGeom &g, double lq,
                                           double qy, double &ex, double &ey) {
    edge_field_cells(a, g, div_known(lq - g.pox, g.phh, g.rphh),
                     div_known(qy - g.poy, g.phh, g.rphh), ex, ey);
}

// (B_z, B_r) of an on-axis profile at axial position z and radius r (fields.py:250-279,
// term by term: the derivatives interpolated between samples, then the series in r).
__device__ __forceinline__ void axial_field(const bt_magnetic &m, double z, double r,
                                            double &bz_out, double &br_out) {
    const i64 n = m.n;
    const int K = m.order + 1;
    const double s = (z - m.z0) / m.hz;
    i64 i = (i64)floor(s);
    if (i < 3)
        i = 3;
    else if (i > n - 5)
        i = n - 5;
    const double t = s - (double)i;
    const double *lo = m.samples + i * K, *hi = lo + K;
    double d[7];
#pragma unroll
    for (int k = 0; k < 7; ++k)
        if (k < K) {
            const double a = __ldg(lo + k);
            d[k] = a + t * (__ldg(hi + k) - a);
        }
    const double r2 = r * r;
    const double bz_c[4] = {1.0, -1.0 / 4.0, 1.0 / 64.0, -1.0 / 2304.0};
    const double br_c[3] = {-1.0 / 2.0, 1.0 / 16.0, -1.0 / 384.0};
    double bz = d[0], br = 0.0, power = 1.0;
#pragma unroll
    for (int k = 1; k <= 3; ++k)
        if (k <= m.order / 2) {
            power = power * r2;
            bz = bz + bz_c[k] * power * d[2 * k];
        }
    power = r;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < (m.order + 1) / 2) {
            br = br + br_c[k] * power * d[2 * k + 1];
            power = power * r2;
        }
    bz_out = bz;
    br_out = br;
}

// The Cartesian B at (q0, q1, q2): mode 1 on a cylindrical mesh ((cy, cz) the radial unit
// vector, r the radius), mode 2 a planar mesh with the solenoid axis on y = axis_y.
__device__ __forceinline__ void magnetic_at(const bt_magnetic &m, double q0, double q1, double r,
                                            double cy, double cz, double *b) {
    double bz, br;
    if (m.mode == 1) {
        axial_field(m, q0, r, bz, br);
        b[0] = bz;
        b[1] = br * cy;
        b[2] = br * cz;
    } else {
        const double yr = q1 - m.axis_y;
        axial_field(m, q0, fabs(yr), bz, br);
        b[0] = bz;
        b[1] = yr < 0.0 ? -br : br;
        b[2] = 0.0;
    }
}

// v <- Boris's kick over tau in the fields e, b (non-relativistic; tracer.py:605-621):
// v- = v + (tau/2) q/m E, t = (tau/2) q/m B, v+ = v- + (v- + v- x t) x 2t / (1 + t^2),
// then + (tau/2) q/m E; the operations in the oracle's order.
__device__ __forceinline__ void kick(double *v, const double *e, const double *b, double tau,
                                     double qm) {
    const double f = 0.5 * tau * qm;
    const double m0 = v[0] + f * e[0], m1 = v[1] + f * e[1], m2 = v[2] + f * e[2];
    const double t0 = f * b[0], t1 = f * b[1], t2 = f * b[2];
    const double d = 2.0 / (1.0 + (t0 * t0 + t1 * t1 + t2 * t2));
    const double s0 = d * t0, s1 = d * t1, s2 = d * t2;
    const double p0 = m0 + (m1 * t2 - m2 * t1);
    const double p1 = m1 + (m2 * t0 - m0 * t2);
    const double p2 = m2 + (m0 * t1 - m1 * t0);
    const double w0 = m0 + (p1 * s2 - p2 * s1);
    const double w1 = m1 + (p2 * s0 - p0 * s2);
    const double w2 = m2 + (p0 * s1 - p1 * s0);
    v[0] = w0 + f * e[0];
    v[1] = w1 + f * e[1];
    v[2] = w2 + f * e[2];
}

// 1 / gamma of a proper velocity: exactly 1 without relativity (inv_c2 = 0), which the
// non-general kernels fold away.
template <bool GENERAL>
__device__ __forceinline__ double inv_gamma(double u0, double u1, double u2, double inv_c2) {
    return GENERAL ? 1.0 / lorentz(u0, u1, u2, inv_c2) : 1.0;
}

// The kernel is specialised on the geometry (0 planar, 1 cylindrical, 2 symmetry plane),
// the integrator (0 RK4, 1 Boris) and GENERAL: refined patches, a graded x axis or
// relativity.  Without them the mesh is one patch, whose shape is read once, and gamma is
// exactly 1; the operations on every value are the general kernel's, so the results are.
// MAG: the reference's NumPy tracer's step in a magnetic field instead (tracer.py:851-1054):
// q/m (E + v x B) at every stage, Boris with the rotation, and every step that ends in a
// cell touching an electrode pauses (status -2) for the caller's exact inside test.
//
// The live trajectories are act[0, *live); the grid covers `stride` >= *live threads, the
// live count when the host last read it, and the records of step s of thread m go to slot
// s * stride + m.  Threads past the live count fill their slots with the sentinel.  A
// window with live trajectories sets *records_end to `end`, the end of its slots, so the
// deposit sorts no window that had none.
//
// At most 168 registers, so that an SM holds three blocks: measured as fast as the
// registers the compiler wants on a window of one block per SM (the einzel lens) and
// faster on larger windows and on concurrent solves, whose warps hide each other's latency.
//
// One thread's window (m < stride): whether its trajectory is still live afterwards.
template <int CYL, int INTEG, bool GENERAL, bool MAG, bool BATCH>
__device__ __forceinline__ bool trace_thread(const Trace &tr, const i64 *__restrict__ act,
                                             i64 m, i64 n_act, i64 stride, int S,
                                             uint32_t *__restrict__ keys,
                                             DepositRec *__restrict__ rec, uint32_t sentinel) {
    if (m >= n_act) {
        for (int s = 0; s < S; ++s) keys[(i64)s * stride + m] = sentinel;
        return false;
    }
    const bt_trace_args &a = tr.a;
    const i64 k = act[m];
    const i64 P = GENERAL ? a.n_patches : 1;
    // the one patch of a non-general mesh (of the trajectory's candidate in a batch)
    const i64 cand = BATCH ? (i64)__ldg(tr.cand + k) : 0;
    PatchGeom base = patch_geom(a, cand);
    base.rphh = known_reciprocal(base.phh);
    const double rh = BATCH ? base.rphh : known_reciprocal(a.h);
    const i64 nx = BATCH ? base.pnx : tr.nx, ny = BATCH ? base.pny : tr.ny;
    const double origin_x = BATCH ? base.pox : a.origin_x;
    const double origin_y = BATCH ? base.poy : a.origin_y;
    const double h = BATCH ? base.phh : a.h;
    const double upper_x = BATCH ? __ldg(a.patch_real + cand * 7 + 5) : a.upper_x;
    const double upper_y = BATCH ? __ldg(a.patch_real + cand * 7 + 6) : a.upper_y;
    const i64 *__restrict__ cells = BATCH ? a.cells + __ldg(tr.cell_off + cand) : a.cells;
    constexpr int cyl = CYL;
    const double inv_c2 = a.inv_c2;
    const i64 n = a.n;
    const bool graded = GENERAL && a.graded != 0;
    double x0 = a.x[k], x1 = a.x[n + k], x2 = a.x[2 * n + k];
    double v0 = a.v[k], v1 = a.v[n + k], v2 = a.v[2 * n + k];
    const double qmk = a.qm[k];
    const double dqk = a.dq[k];
    const i64 slot = a.path_slot[k];
    i64 ns = a.steps[k];
    i64 st = -1;
    constexpr int nstage = INTEG == 0 ? 4 : 2;
    int have = 0;
    double ca0 = 0.0, ca1 = 0.0, ca2 = 0.0;
    double cE[3] = {0, 0, 0}, cB[3] = {0, 0, 0};  // with B: the fields at the step's end
    // A one-patch mesh whose patch is the mesh: the first gather of a step is at the point
    // where the exit test of the step before found the radius and the cell coordinates;
    // they are kept (the same expressions on the same values).
    const bool reuse = !GENERAL && !MAG && base.pox == origin_x && base.poy == origin_y &&
                       base.phh == h;
    double start_r = 0.0, start_sx = 0.0, start_sy = 0.0;
    if (reuse) {
        start_r = x1;
        if (cyl == 1)
            start_r = radius(x1, x2);
        else if (cyl == 2)
            start_r = origin_y + fabs(x1 - origin_y);
        start_sx = div_known(x0 - origin_x, h, rh);
        start_sy = div_known(start_r - origin_y, h, rh);
    }
    // The records of consecutive steps in one cell are summed into one (the run's): it goes
    // to the slot of the run's last step, the slots of its other steps hold the sentinel.
    i64 run_slot = -1;
    uint32_t run_key = sentinel;
    double r00 = 0.0, r01 = 0.0, r10 = 0.0, r11 = 0.0;
    int s = 0;
    for (; s < S; ++s) {
        if (ns >= a.max_steps) break;
        double rr = x1;
        if (cyl == 1)
            rr = radius(x1, x2);
        else if (cyl == 2)
            rr = origin_y + fabs(x1 - origin_y);
        double lx = x0;
        if (graded) lx = uniform_x(x0, a.x_nodes, a.n_x_nodes, origin_x, h);
        double hloc = h;
        for (i64 qq = 0; qq < P - 1; ++qq) {
            const double *pr = a.patch_real + qq * 7;
            if (lx >= __ldg(pr + 3) && lx <= __ldg(pr + 5) && rr >= __ldg(pr + 4) &&
                rr <= __ldg(pr + 6)) {
                hloc = __ldg(pr + 2);
                break;
            }
        }
        if (graded) {
            const i64 cg = node_cell(x0, a.x_nodes, a.n_x_nodes);
            if (MAG) {
                // the NumPy tracer's spacing: the smaller of the cell's edge and h
                const double dxc = a.x_nodes[cg + 1] - a.x_nodes[cg];
                if (dxc < hloc) hloc = dxc;
            } else {
                const double d2 = (a.x_nodes[cg + 1] - a.x_nodes[cg]) / h;
                if (d2 < 1.0) hloc = hloc * d2;
            }
        }
        const double gv = inv_gamma<GENERAL>(v0, v1, v2, inv_c2);
        double q0 = x0, q1 = x1, q2 = x2;
        double kx0 = v0, kx1 = v1, kx2 = v2;
        double sx0 = 0, sx1 = 0, sx2 = 0, sv0 = 0, sv1 = 0, sv2 = 0;
        double w0 = 0, w1 = 0, w2 = 0, y0, y1, y2;
        double dt = 0.0, hdt = 0.0, dt6 = 0.0;
        for (int stage = 0; stage < nstage; ++stage) {
            double gk = inv_gamma<GENERAL>(kx0, kx1, kx2, inv_c2);
            double g0, g1, g2;
            double E[3], B[3];
            if (MAG && stage == 0 && have != 0) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    E[c] = cE[c];
                    B[c] = cB[c];
                }
            }
            if (MAG && !(stage == 0 && have != 0)) {
                double qy = q1, cy = 0.0, cz = 0.0;
                if (cyl == 1) {
                    const double r = radius(q1, q2);
                    if (r > 0.0) {
                        cy = q1 / r;
                        cz = q2 / r;
                    }
                    qy = r;
                }
                double lq = q0;
                if (graded) lq = uniform_x(q0, a.x_nodes, a.n_x_nodes, origin_x, h);
                double ex, ey;
                const PatchGeom g = GENERAL ? patch_geom(a, finest_patch(a, P, lq, qy)) : base;
                edge_field(a, g, lq, qy, ex, ey);
                if (cyl != 0) {
                    E[0] = ex;
                    E[1] = ey * cy;
                    E[2] = ey * cz;
                } else {
                    E[0] = ex;
                    E[1] = ey;
                    E[2] = 0.0;
                }
                magnetic_at(tr.mag, q0, q1, qy, cy, cz, B);
            }
            if (MAG) {
                // q/m (E + v x B) at the stage velocity (tracer.py:519-529)
                const double c0 = kx1 * B[2] - kx2 * B[1];
                const double c1 = kx2 * B[0] - kx0 * B[2];
                const double c2 = kx0 * B[1] - kx1 * B[0];
                g0 = qmk * (E[0] + c0);
                g1 = qmk * (E[1] + c1);
                g2 = qmk * (E[2] + c2);
            } else if (stage == 0 && have != 0) {
                g0 = ca0;
                g1 = ca1;
                g2 = ca2;
            } else {
                const bool kept = reuse && stage == 0;
                double qy = q1, cy = 0.0, cz = 0.0;
                if (cyl == 1) {
                    const double r = kept ? start_r : radius(q1, q2);
                    if (r > 0.0) {
                        cy = q1 / r;
                        cz = q2 / r;
                    }
                    qy = r;
                } else if (cyl == 2) {
                    cy = 1.0;
                    if (q1 < origin_y) cy = -1.0;
                    qy = origin_y + fabs(q1 - origin_y);
                }
                double lq = q0;
                if (graded) lq = uniform_x(q0, a.x_nodes, a.n_x_nodes, origin_x, h);
                double ex, ey;
                const PatchGeom g = GENERAL ? patch_geom(a, finest_patch(a, P, lq, qy)) : base;
                if (kept)
                    edge_field_cells(a, g, start_sx, start_sy, ex, ey);
                else
                    edge_field(a, g, lq, qy, ex, ey);
                if (cyl != 0) {
                    g0 = qmk * ex;
                    g1 = qmk * (ey * cy);
                    g2 = qmk * (ey * cz);
                } else {
                    g0 = qmk * ex;
                    g1 = qmk * ey;
                    g2 = qmk * 0.0;
                }
            }
            if (stage == 0) {
                const double a0 = g0, a1 = g1, a2 = g2;
                const double speed = gv * sqrt(v0 * v0 + v1 * v1 + v2 * v2);
                const double accel = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
                dt = -1.0;
                if (speed > 0.0) dt = hloc / speed;
                if (accel > 0.0) {
                    const double d2 = sqrt(2.0 * hloc / accel);
                    if (dt < 0.0 || d2 < dt) dt = d2;
                }
                if (dt < 0.0) dt = hloc;
                dt = a.step_fraction * dt;
                hdt = 0.5 * dt;
                dt6 = div_known(dt, 6.0, 1.0 / 6.0);
                if (INTEG != 0 && MAG) {
                    // Boris with B: the kick over half the step, then the drift
                    double u[3] = {v0, v1, v2};
                    kick(u, E, B, hdt, qmk);
                    kx0 = u[0];
                    kx1 = u[1];
                    kx2 = u[2];
                    q0 = x0 + dt * kx0;
                    q1 = x1 + dt * kx1;
                    q2 = x2 + dt * kx2;
                    continue;
                }
                if (INTEG != 0) {
                    kx0 = v0 + hdt * a0;
                    kx1 = v1 + hdt * a1;
                    kx2 = v2 + hdt * a2;
                    gk = inv_gamma<GENERAL>(kx0, kx1, kx2, inv_c2);
                    q0 = x0 + dt * gk * kx0;
                    q1 = x1 + dt * gk * kx1;
                    q2 = x2 + dt * gk * kx2;
                    continue;
                }
                sx0 = gv * v0;
                sx1 = gv * v1;
                sx2 = gv * v2;
                sv0 = a0;
                sv1 = a1;
                sv2 = a2;
                q0 = x0 + hdt * gv * v0;
                q1 = x1 + hdt * gv * v1;
                q2 = x2 + hdt * gv * v2;
                kx0 = v0 + hdt * a0;
                kx1 = v1 + hdt * a1;
                kx2 = v2 + hdt * a2;
            } else if (INTEG != 0 && MAG) {
                // Boris with B: the second kick in the fields at the end of the step
                double u[3] = {kx0, kx1, kx2};
                kick(u, E, B, hdt, qmk);
                w0 = u[0];
                w1 = u[1];
                w2 = u[2];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    cE[c] = E[c];
                    cB[c] = B[c];
                }
                have = 1;
            } else if (INTEG != 0) {
                w0 = kx0 + hdt * g0;
                w1 = kx1 + hdt * g1;
                w2 = kx2 + hdt * g2;
                ca0 = g0;
                ca1 = g1;
                ca2 = g2;
                have = 1;
            } else if (stage == 1 || stage == 2) {
                sx0 = sx0 + 2.0 * gk * kx0;
                sx1 = sx1 + 2.0 * gk * kx1;
                sx2 = sx2 + 2.0 * gk * kx2;
                sv0 = sv0 + 2.0 * g0;
                sv1 = sv1 + 2.0 * g1;
                sv2 = sv2 + 2.0 * g2;
                const double f = stage == 1 ? hdt : dt;
                q0 = x0 + f * gk * kx0;
                q1 = x1 + f * gk * kx1;
                q2 = x2 + f * gk * kx2;
                kx0 = v0 + f * g0;
                kx1 = v1 + f * g1;
                kx2 = v2 + f * g2;
            } else {
                sx0 = sx0 + gk * kx0;
                sx1 = sx1 + gk * kx1;
                sx2 = sx2 + gk * kx2;
                sv0 = sv0 + g0;
                sv1 = sv1 + g1;
                sv2 = sv2 + g2;
            }
        }
        if (INTEG == 0) {
            y0 = x0 + dt6 * sx0;
            y1 = x1 + dt6 * sx1;
            y2 = x2 + dt6 * sx2;
            w0 = v0 + dt6 * sv0;
            w1 = v1 + dt6 * sv1;
            w2 = v2 + dt6 * sv2;
        } else {
            y0 = q0;
            y1 = q1;
            y2 = q2;
        }

        // the deposit record of the step's Hermite midpoint (:372-423)
        const double gw = inv_gamma<GENERAL>(w0, w1, w2, inv_c2);
        // (a / 8 is a * 0.125 exactly)
        double m0 = 0.5 * (x0 + y0) + dt * (gv * v0 - gw * w0) * 0.125;
        double m1 = 0.5 * (x1 + y1) + dt * (gv * v1 - gw * w1) * 0.125;
        const double m2 = 0.5 * (x2 + y2) + dt * (gv * v2 - gw * w2) * 0.125;
        if (cyl == 1)
            m1 = radius(m1, m2);
        else if (cyl == 2)
            m1 = origin_y + fabs(m1 - origin_y);
        if (graded) m0 = uniform_x(m0, a.x_nodes, a.n_x_nodes, origin_x, h);
        {
            const PatchGeom g = GENERAL ? patch_geom(a, finest_patch(a, P, m0, m1)) : base;
            const int pnx = (int)g.pnx, pny = (int)g.pny;
            const double pox = g.pox, poy = g.poy, phh = g.phh, rphh = g.rphh;
            int i = __double2int_rd(div_known(m0 - pox, phh, rphh));
            int j = __double2int_rd(div_known(m1 - poy, phh, rphh));
            double u = div_known(m0 - (pox + phh * (double)i), phh, rphh);
            double w;
            if (cyl == 1) {
                const double low = poy + phh * (double)j;
                const double high = low + phh;
                w = (m1 * m1 - low * low) / (high * high - low * low);
            } else {
                w = div_known(m1 - (poy + phh * (double)j), phh, rphh);
            }
            if (i < 0) {
                u = 0.0;
                i = 0;
            } else if (i >= pnx - 1) {
                u = 1.0;
                i = pnx - 2;
            }
            if (j < 0) {
                w = 0.0;
                j = 0;
            } else if (j >= pny - 1) {
                w = 1.0;
                j = pny - 2;
            }
            const uint32_t key = (uint32_t)(g.ofn + (i64)i * pny + j);
            const double q = dqk * dt;
            const double c00 = (1.0 - u) * (1.0 - w) * q, c01 = (1.0 - u) * w * q;
            const double c10 = u * (1.0 - w) * q, c11 = u * w * q;
            if (run_slot >= 0 && key == run_key) {
                // the step stays in the run's cell: its charge joins the run's record
                keys[run_slot] = sentinel;
                r00 = r00 + c00;
                r01 = r01 + c01;
                r10 = r10 + c10;
                r11 = r11 + c11;
            } else {
                if (run_slot >= 0) {
                    keys[run_slot] = run_key;
                    rec[run_slot] = DepositRec{r00, r01, r10, r11};
                }
                run_key = key;
                r00 = c00;
                r01 = c01;
                r10 = c10;
                r11 = c11;
            }
            run_slot = (i64)s * stride + m;
        }
        ns = ns + 1;

        for (i64 p = 0; p < a.n_planes; ++p) {
            const double xp = a.planes[p];
            const double before = x0 - xp;
            const double after = y0 - xp;
            if ((before < 0.0) != (after < 0.0)) {
                const double sc = before / (before - after);
                i64 *cnt = a.counts + k * a.n_planes + p;
                const i64 c = *cnt;
                if (c < a.capacity) {
                    double *hit = a.hits + ((k * a.n_planes + p) * a.capacity + c) * 8;
                    hit[0] = xp;
                    hit[1] = x1 + sc * (y1 - x1);
                    hit[2] = x2 + sc * (y2 - x2);
                    hit[3] = gv * v0 + sc * (gw * w0 - gv * v0);
                    hit[4] = gv * v1 + sc * (gw * w1 - gv * v1);
                    hit[5] = gv * v2 + sc * (gw * w2 - gv * v2);
                    hit[6] = after >= 0.0 ? 1.0 : -1.0;
                    hit[7] = 1.0 * (double)ns;
                }
                *cnt = c + 1;
            }
        }
        x0 = y0;
        x1 = y1;
        x2 = y2;
        v0 = w0;
        v1 = w1;
        v2 = w2;

        double px = x0, py = x1;
        if (cyl == 1)
            py = radius(x1, x2);
        else if (cyl == 2)
            py = origin_y + fabs(x1 - origin_y);
        if (slot >= 0) {
            const i64 c = a.path_count[slot];
            if (c < a.path_capacity) {
                a.paths[(slot * a.path_capacity + c) * 2 + 0] = px;
                a.paths[(slot * a.path_capacity + c) * 2 + 1] = py;
            }
            a.path_count[slot] = c + 1;
        }
        if (graded) px = uniform_x(px, a.x_nodes, a.n_x_nodes, origin_x, h);
        if (px >= upper_x) {
            st = 0;
        } else if (px < origin_x) {
            st = 1;
        } else if (py > upper_y || (cyl == 0 && py < origin_y)) {
            st = 2;
        } else {
            const double ux = div_known(px - origin_x, h, rh);
            const double uy = div_known(py - origin_y, h, rh);
            start_r = py;
            start_sx = ux;
            start_sy = uy;
            // a point below the mesh (only a malformed geometry puts one there) takes
            // its first cell, where the reference indexes outside the table
            const int i = max(min(__double2int_rz(ux), (int)nx - 2), 0);
            const int j = max(min(__double2int_rz(uy), (int)ny - 2), 0);
            const i64 cell = __ldg(cells + (i64)i * (ny - 1) + j);
            if (MAG && cell >= 0) {
                st = -2;  // the caller tests the electrodes' shapes
            } else if (cell >= 0) {
                const i64 R = a.refine;
                i64 si = (i64)((ux - (double)i) * (double)R);
                if (si < 0)
                    si = 0;
                else if (si > R - 1)
                    si = R - 1;
                i64 sj = (i64)((uy - (double)j) * (double)R);
                if (sj < 0)
                    sj = 0;
                else if (sj > R - 1)
                    sj = R - 1;
                const i64 e = __ldg(a.subcells + (cell * R + si) * R + sj);
                if (e >= 0) {
                    st = 3;
                    a.electrode[k] = e;
                } else if (e == -2 && BATCH && tr.shape_first) {
                    // the candidate's own electrodes, tested here at the point's mesh
                    // coordinates: the caller's test of a paused trajectory
                    const i64 s0 = __ldg(tr.shape_first + cand);
                    const Shapes S{__ldg(tr.shape_first + cand + 1) - s0, tr.shapes.kind + s0,
                                   tr.shapes.offset + s0, tr.shapes.params};
                    const i64 hit = inside_solid(S, px, py);
                    if (hit >= 0) {
                        st = 3;
                        a.electrode[k] = hit;
                    }
                } else if (e == -2) {
                    st = -2;
                }
            }
        }
        if (st != -1) {
            ++s;
            break;
        }
    }
    if (run_slot >= 0) {
        keys[run_slot] = run_key;
        rec[run_slot] = DepositRec{r00, r01, r10, r11};
    }
    // the slots of the steps not taken hold no record
    for (; s < S; ++s) keys[(i64)s * stride + m] = sentinel;
    if (st == -1 && ns >= a.max_steps) st = 4;
    a.x[k] = x0;
    a.x[n + k] = x1;
    a.x[2 * n + k] = x2;
    a.v[k] = v0;
    a.v[n + k] = v1;
    a.v[2 * n + k] = v2;
    a.steps[k] = ns;
    a.status[k] = st;
    return st == -1;
}

// The window: every thread's trajectory, then each block's count of live trajectories and
// every thread's flag, for compact_live.  BATCH: the trajectories of many candidate meshes
// in one launch (Trace::cand).
template <int CYL, int INTEG, bool GENERAL, bool MAG, bool BATCH>
__global__ void __launch_bounds__(128, 3)
    trace_window(Trace tr, const i64 *__restrict__ act, const i64 *__restrict__ live, i64 stride,
                 int S, uint32_t *__restrict__ keys, DepositRec *__restrict__ rec,
                 uint32_t sentinel, i64 *__restrict__ records_end, i64 end,
                 uint32_t *__restrict__ block_live, uint8_t *__restrict__ alive) {
    const i64 m = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n_act = *live;
    if (m == 0 && n_act > 0) *records_end = end;
    bool still = false;
    if (m < stride)
        still = trace_thread<CYL, INTEG, GENERAL, MAG, BATCH>(tr, act, m, n_act, stride, S, keys,
                                                              rec, sentinel);
    const int count = __syncthreads_count(still);
    if (m < stride) alive[m] = still ? 1 : 0;
    if (threadIdx.x == 0) block_live[blockIdx.x] = (uint32_t)count;
}

// -- order-preserving compaction of the live trajectories ----------------------------------

// Windows of more blocks than this have their blocks' offsets scanned by block_offsets
// (each compact_live block would otherwise add up all the counts before its own).
constexpr int kSumBlocks = 2048;

// offsets[b] = the live trajectories of the window's blocks before b (one block, in chunks
// of 1024).
__global__ void __launch_bounds__(1024) block_offsets(const uint32_t *__restrict__ block_live,
                                                      int nblocks, uint32_t *__restrict__ offsets) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int start = 0; start < nblocks; start += 1024) {
        const int b = start + t;
        const uint32_t v = b < nblocks ? block_live[b] : 0u;
        uint32_t x = v;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sums[lane];
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const uint32_t inclusive = x + (warp > 0 ? warp_sums[warp - 1] : 0u) + carry;
        if (b < nblocks) offsets[b] = inclusive - v;
        __syncthreads();
        if (t == 1023) carry = inclusive;
        __syncthreads();
    }
}

// act_out = the live trajectories of act, in order, and *live_out their count, from a
// window's per-block counts and flags (the window's grid of 128-thread blocks); `offsets`,
// when not NULL, holds each block's count of the live trajectories before it.
__global__ void __launch_bounds__(128) compact_live(const i64 *__restrict__ act,
                                                    const uint8_t *__restrict__ alive,
                                                    const uint32_t *__restrict__ block_live,
                                                    const uint32_t *__restrict__ offsets,
                                                    i64 stride, i64 *__restrict__ act_out,
                                                    i64 *__restrict__ live_out) {
    __shared__ uint32_t part[4], warp_first[4];
    const int b = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    uint32_t before = 0;  // the live trajectories of the blocks before this one
    if (offsets)
        before = t == 0 ? offsets[b] : 0u;
    else
        for (int q = t; q < b; q += 128) before += block_live[q];
    for (int off = 16; off > 0; off >>= 1) before += __shfl_down_sync(0xffffffffu, before, off);
    if (lane == 0) part[warp] = before;
    const i64 m = (i64)b * 128 + t;
    const bool a = m < stride && alive[m] != 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, a);
    if (lane == 0) warp_first[warp] = __popc(ballot);
    __syncthreads();
    const uint32_t offset = part[0] + part[1] + part[2] + part[3];
    uint32_t rank = offset;
    for (int w = 0; w < warp; ++w) rank += warp_first[w];
    rank += __popc(ballot & ((1u << lane) - 1u));
    if (a) act_out[rank] = act[m];
    if (b == (int)gridDim.x - 1 && t == 0) *live_out = offset + block_live[b];
}

__global__ void set_count(i64 *__restrict__ count, i64 value) { *count = value; }

}  // namespace

}  // namespace bt

namespace bt {
namespace {

// Windows launched between two reads of the live count.
constexpr int kGroup = 4;

// Record slots per deposit batch, at most: a batch is a group's windows when they hold
// fewer.  A batch is deposited at the end of its group, under the next group's windows,
// so only the last group's deposit is left when the trace ends.
constexpr int64_t kBatchRecords = (int64_t)1 << 24;

// Points the context's launches at `side` for its lifetime.
struct SideStream {
    bt_ctx *ctx;
    cudaStream_t saved;
    SideStream(bt_ctx *c, cudaStream_t side) : ctx(c), saved(c->stream) { ctx->stream = side; }
    ~SideStream() { ctx->stream = saved; }
};

// Windows between reads of the live count for a batch: as many as keep a group's record
// slots within kBatchGroupRecords (at least one, at most kGroup).
constexpr int64_t kBatchGroupRecords = (int64_t)1 << 26;

void trace_all(bt_ctx *ctx, const bt_trace_args *args, const bt_magnetic *mag, int64_t window,
               const bt_trace_batch *batch = nullptr) {
    {
        BT_REQUIRE(ctx && args, "trace: null argument");
        const bt_trace_args &a = *args;
        BT_REQUIRE(a.n_patches >= 1 && a.patch_int && a.patch_real, "trace: no patches");
        BT_REQUIRE(a.n_active >= 0 && a.n >= 0, "trace: negative sizes");
        BT_REQUIRE(a.capacity >= 0 && a.path_capacity >= 0 && a.n_planes >= 0,
                   "trace: negative buffer sizes");
        BT_REQUIRE(a.refine >= 1, "trace: refine must be positive");
        BT_REQUIRE(!a.graded || a.n_x_nodes >= 2, "trace: a graded axis needs its nodes");
        BT_REQUIRE(a.n_nodes < (int64_t)0xffffffffLL, "trace: too many nodes for 32-bit keys");
        bt::Trace tr;
        tr.a = a;
        tr.mag = mag ? *mag : bt_magnetic{};
        if (mag) {
            BT_REQUIRE(mag->mode == 1 || mag->mode == 2, "trace: magnetic mode must be 1 or 2");
            BT_REQUIRE(mag->order >= 0 && mag->order <= 6, "trace: magnetic order must be 0 to 6");
            BT_REQUIRE(mag->n >= 8 && mag->samples, "trace: the profile needs 8 samples");
            BT_REQUIRE(mag->hz > 0.0, "trace: the profile spacing must be positive");
            BT_REQUIRE((mag->mode == 1) == (a.cylindrical == 1),
                       "trace: mode 1 needs a cylindrical mesh, mode 2 a planar one");
            BT_REQUIRE(a.inv_c2 == 0.0 && a.n_patches == 1,
                       "trace: the magnetic trace is non-relativistic on one patch");
            BT_REQUIRE(a.cylindrical != 2, "trace: no magnetic field with a symmetry plane");
        }
        tr.cand = nullptr;
        tr.cell_off = nullptr;
        tr.shape_first = nullptr;
        tr.shapes = bt::Shapes{0, nullptr, nullptr, nullptr};
        if (batch) {
            // every candidate's one patch: shapes of at least 2 x 2 nodes whose node ranges
            // tile [0, n_nodes) in order (the deposit finds a node's candidate by bisection)
            BT_REQUIRE(!mag, "trace: a batch takes no magnetic field");
            BT_REQUIRE(batch->n_candidates >= 1 && batch->n_candidates == a.n_patches,
                       "trace: a batch needs one patch row per candidate");
            BT_REQUIRE(batch->candidate && batch->cell_offset, "trace: null batch table");
            BT_REQUIRE(!a.graded && a.inv_c2 == 0.0,
                       "trace: a batch takes uniform, non-relativistic meshes");
            std::vector<int64_t> rows((size_t)6 * a.n_patches);
            BT_CUDA(cudaMemcpyAsync(rows.data(), a.patch_int, sizeof(int64_t) * rows.size(),
                                    cudaMemcpyDeviceToHost, ctx->stream));
            BT_CUDA(cudaStreamSynchronize(ctx->stream));
            int64_t next = 0;
            for (int64_t c = 0; c < a.n_patches; ++c) {
                const int64_t *r = rows.data() + 6 * c;
                BT_REQUIRE(r[0] >= 2 && r[1] >= 2, "trace: a candidate needs at least 2 x 2 nodes");
                BT_REQUIRE(r[4] == r[0] * r[1] && r[5] == next,
                           "trace: the candidates' nodes must follow one another from 0");
                next += r[4];
            }
            BT_REQUIRE(next == a.n_nodes, "trace: the candidates' nodes must fill n_nodes");
            tr.cand = batch->candidate;
            tr.cell_off = batch->cell_offset;
            if (batch->shape_first) {
                BT_REQUIRE(batch->shape_kind && batch->shape_offset && batch->shape_params,
                           "trace: a batch's shapes need their kind, offset and parameters");
                tr.shape_first = batch->shape_first;
                tr.shapes = bt::Shapes{0, batch->shape_kind, batch->shape_offset,
                                       batch->shape_params};
            }
            tr.nx = tr.ny = 0;
        } else {
            // the last patch's shape, for the exit and electrode tests
            int64_t last[6];
            BT_CUDA(cudaMemcpyAsync(last, a.patch_int + (a.n_patches - 1) * 6, sizeof(last),
                                    cudaMemcpyDeviceToHost, ctx->stream));
            BT_CUDA(cudaStreamSynchronize(ctx->stream));
            tr.nx = last[0];
            tr.ny = last[1];
            BT_REQUIRE(tr.nx >= 2 && tr.ny >= 2, "trace: the mesh needs at least 2 x 2 nodes");
        }
        BT_REQUIRE(a.cylindrical >= 0 && a.cylindrical <= 2, "trace: geometry must be 0, 1 or 2");
        const int S = window > 0 ? (int)window : 64;
        const bool general = !batch && (a.n_patches > 1 || a.graded != 0 || a.inv_c2 != 0.0);
        ctx->last_windows = ctx->last_records = ctx->last_flushes = 0;
        if (a.n_active == 0) return;
        bt::TraceScratch &ts = ctx->trace;
        cudaStream_t st = ctx->stream;
        const uint32_t sentinel = (uint32_t)a.n_nodes;
        // Two record buffers: the windows fill one while the records of the other are sorted
        // and reduced into charge[0] on the side stream, in the order the buffers were
        // filled, so the deposit runs under the next windows and the sums are the same
        // whatever the timing.  A buffer is deposited at the end of the group that brought
        // it to `flush_at` records (or on filling up within a group).  A batch's windows
        // are large: its groups hold fewer of them, so the buffers stay within a few GB.
        const int64_t per_window = a.n_active * (int64_t)S;
        int group = kGroup;
        if (batch) {
            const int64_t fit = std::max<int64_t>(1, kBatchGroupRecords / std::max<int64_t>(per_window, 1));
            group = (int)std::min<int64_t>(batch->group > 0 ? batch->group : fit, kGroup);
        }
        const int64_t flush_at = std::min<int64_t>(kBatchRecords, group * per_window);
        const int64_t capacity = flush_at + group * per_window;
        uint32_t *keys[2];
        bt::DepositRec *rec[2];
        for (int b = 0; b < 2; ++b) {
            keys[b] = ts.rec_keys[b].as<uint32_t>(capacity);
            rec[b] = ts.rec[b].as<bt::DepositRec>(capacity);
        }
        if (!ts.side) {
            BT_CUDA(cudaStreamCreateWithFlags(&ts.side, cudaStreamNonBlocking));
            for (int b = 0; b < 2; ++b) {
                BT_CUDA(cudaEventCreateWithFlags(&ts.filled[b], cudaEventDisableTiming));
                BT_CUDA(cudaEventCreateWithFlags(&ts.drained[b], cudaEventDisableTiming));
            }
        }
        int64_t *act_a = ts.active_a.as<int64_t>(a.n_active);
        int64_t *act_b = ts.active_b.as<int64_t>(a.n_active);
        // the window's per-block live counts, and room after them for their offsets
        uint32_t *block_live =
            ts.block_counts.as<uint32_t>(2 * (size_t)bt::blocks_for(a.n_active, 128));
        uint8_t *alive = ts.alive.as<uint8_t>(a.n_active);
        // live[2]: the live count before and after a window's compaction; records_end[2]:
        // where the slots of each buffer's last window with live trajectories end
        int64_t *live = ts.n_alive.as<int64_t>(4);
        int64_t *records_end = live + 2;
        int64_t *n_alive_host = static_cast<int64_t *>(ctx->host.get(sizeof(int64_t)));
        BT_CUDA(cudaMemcpyAsync(act_a, a.active, sizeof(int64_t) * a.n_active,
                                cudaMemcpyDeviceToDevice, st));
        BT_CUDA(cudaMemsetAsync(records_end, 0, 2 * sizeof(int64_t), st));
        BT_LAUNCH(ctx, bt::set_count, 1, 1, 0, st, live, a.n_active);
        // A batch's deposits add their per-cell sums up over the whole trace and reach the
        // nodes once at its end (a flush then costs only its records, not every node of
        // every candidate).
        if (batch) bt::deposit_cells_reset(ctx, a.n_nodes);
        bt::NodeLayout layout{a.patch_int, a.n_patches, tr.nx, tr.ny, a.n_nodes, batch != nullptr};
        int64_t bound = a.n_active, used = 0;
        int lv = 0;
        int cur = 0;
        bool pending[2] = {false, false};
        // deposit buffer `cur` on the side stream and switch the windows to the other one
        auto flush = [&] {
            if (used == 0) return;
            BT_CUDA(cudaEventRecord(ts.filled[cur], st));
            BT_CUDA(cudaStreamWaitEvent(ts.side, ts.filled[cur], 0));
            {
                SideStream on_side(ctx, ts.side);
                bt::Timed timed(ctx, "deposit");
                bt::deposit_records(ctx, keys[cur], rec[cur], used, records_end + cur, sentinel,
                                    a.charge, layout, batch != nullptr);
            }
            BT_CUDA(cudaMemsetAsync(records_end + cur, 0, sizeof(int64_t), ts.side));
            BT_CUDA(cudaEventRecord(ts.drained[cur], ts.side));
            pending[cur] = true;
            ctx->last_records += used;
            ctx->last_flushes += 1;
            used = 0;
            cur ^= 1;
            if (pending[cur]) BT_CUDA(cudaStreamWaitEvent(st, ts.drained[cur], 0));
        };
        // The windows go in groups of kGroup between reads of the live count: each reads
        // the count on the device, and a window after the last trajectory ended does no work.
        while (bound > 0) {
            for (int g = 0; g < group; ++g) {
                const int64_t need = bound * (int64_t)S;
                if (used + need > capacity) flush();
                unsigned grid = 0;
                {
                    bt::Timed timed(ctx, "trace_window");
                    grid = (unsigned)bt::blocks_for(bound, 128);
                    const int64_t launched = ctx->launch_count;
#define BT_TRACE_CASE_B(C, I, G, M, B)                                                          \
    if (a.cylindrical == C && (a.integrator != 0) == (I != 0) && general == G &&                 \
        (mag != nullptr) == M && (batch != nullptr) == B)                                        \
        BT_LAUNCH(ctx, (bt::trace_window<C, I, G, M, B>), grid, 128, 0, st, tr, act_a,            \
                  live + lv, bound, S, keys[cur] + used, rec[cur] + used, sentinel,               \
                  records_end + cur, used + need, block_live, alive);
#define BT_TRACE_CASE(C, I, G, M) BT_TRACE_CASE_B(C, I, G, M, false)
                    BT_TRACE_CASE(0, 0, false, false) BT_TRACE_CASE(0, 0, true, false)
                    BT_TRACE_CASE(0, 1, false, false) BT_TRACE_CASE(0, 1, true, false)
                    BT_TRACE_CASE(1, 0, false, false) BT_TRACE_CASE(1, 0, true, false)
                    BT_TRACE_CASE(1, 1, false, false) BT_TRACE_CASE(1, 1, true, false)
                    BT_TRACE_CASE(2, 0, false, false) BT_TRACE_CASE(2, 0, true, false)
                    BT_TRACE_CASE(2, 1, false, false) BT_TRACE_CASE(2, 1, true, false)
                    BT_TRACE_CASE(0, 0, false, true) BT_TRACE_CASE(0, 0, true, true)
                    BT_TRACE_CASE(0, 1, false, true) BT_TRACE_CASE(0, 1, true, true)
                    BT_TRACE_CASE(1, 0, false, true) BT_TRACE_CASE(1, 0, true, true)
                    BT_TRACE_CASE(1, 1, false, true) BT_TRACE_CASE(1, 1, true, true)
                    BT_TRACE_CASE_B(0, 0, false, false, true) BT_TRACE_CASE_B(0, 1, false, false, true)
                    BT_TRACE_CASE_B(1, 0, false, false, true) BT_TRACE_CASE_B(1, 1, false, false, true)
                    BT_TRACE_CASE_B(2, 0, false, false, true) BT_TRACE_CASE_B(2, 1, false, false, true)
#undef BT_TRACE_CASE
#undef BT_TRACE_CASE_B
                    BT_REQUIRE(ctx->launch_count > launched,
                               "trace: no kernel for these settings");
                }
                BT_CHECK_LAUNCH();
                used += need;
                ctx->last_windows += 1;
                uint32_t *offsets = nullptr;
                if (grid > (unsigned)bt::kSumBlocks) {
                    offsets = block_live + grid;
                    BT_LAUNCH(ctx, bt::block_offsets, 1, 1024, 0, st, block_live, (int)grid,
                              offsets);
                }
                BT_LAUNCH(ctx, bt::compact_live, grid, 128, 0, st, act_a, alive, block_live,
                          offsets, bound, act_b, live + (lv ^ 1));
                BT_CHECK_LAUNCH();
                std::swap(act_a, act_b);
                lv ^= 1;
            }
            BT_CUDA(cudaMemcpyAsync(n_alive_host, live + lv, sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, st));
            BT_CUDA(cudaStreamSynchronize(st));
            bound = *n_alive_host;
            if (used >= flush_at) flush();
        }
        flush();
        // the caller's stream continues once every deposit is in charge[0]
        for (int b = 0; b < 2; ++b)
            if (pending[b]) BT_CUDA(cudaStreamWaitEvent(st, ts.drained[b], 0));
        if (batch) bt::deposit_cells_finish(ctx, a.charge, layout);
    }
}

}  // namespace
}  // namespace bt

// trace_fast.cu compiles this file again with contracted multiply-adds; its entry points
// carry the suffix _fast.
#ifdef BT_TRACE_FAST
#define BT_TRACE_ENTRY(name) name##_fast
#else
#define BT_TRACE_ENTRY(name) name
#endif

extern "C" int BT_TRACE_ENTRY(bt_trace_trajectories_2d)(bt_ctx *ctx, const bt_trace_args *args,
                                                        int64_t window) {
    return bt::guarded([&] { bt::trace_all(ctx, args, nullptr, window); });
}

extern "C" int BT_TRACE_ENTRY(bt_trace_trajectories_2d_magnetic)(bt_ctx *ctx,
                                                                 const bt_trace_args *args,
                                                                 const bt_magnetic *magnetic,
                                                                 int64_t window) {
    return bt::guarded([&] {
        BT_REQUIRE(magnetic, "trace: null magnetic field");
        bt::trace_all(ctx, args, magnetic, window);
    });
}

extern "C" int BT_TRACE_ENTRY(bt_trace_trajectories_2d_batch)(bt_ctx *ctx,
                                                              const bt_trace_args *args,
                                                              const bt_trace_batch *batch,
                                                              int64_t window) {
    return bt::guarded([&] {
        BT_REQUIRE(batch, "trace: null batch");
        bt::trace_all(ctx, args, nullptr, window, batch);
    });
}

#ifndef BT_TRACE_FAST
extern "C" int bt_trace_last_stats(bt_ctx *ctx, int64_t *windows, int64_t *records,
                                   int64_t *deposit_flushes) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "trace stats: null context");
        if (windows) *windows = ctx->last_windows;
        if (records) *records = ctx->last_records;
        if (deposit_flushes) *deposit_flushes = ctx->last_flushes;
    });
}
#endif
