/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain-C, FP64 restatement of the reference beamtracer's CPU kernels of the Vlasov
 * iteration's trajectory path.  It is the checker that the CUDA kernels of
 * beamtracer_b200 are compared with, and the CPU baseline that bench.py times (OpenMP
 * over trajectories, one charge slab per thread, as the reference's Pyccel/OpenMP build
 * splits the work).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.
 *
 * Restated from (paths inside the reference project):
 *   staggered_field_2d      src/beamtracer/kernels/staggered_field_2d/staggered_field_2d_pyccel.py:13-55
 *   deposit_trajectories_2d src/beamtracer/kernels/deposit_trajectories_2d/deposit_trajectories_2d_pyccel.py:13-59
 *   trace_trajectories_2d   src/beamtracer/kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:42-507
 *   node_cell / uniform_x   trace_trajectories_2d_pyccel.py:19-39
 *   lorentz_factor          mpiparticles (absent; restated as sqrt(1 + |u|^2 inv_c2), the
 *                           form the tracer's docstring gives, trace_trajectories_2d_pyccel.py:108-111)
 *
 * The arithmetic follows the reference's expressions term by term (built with
 * -ffp-contract=off so no multiply-add is fused).  One deliberate difference: the radius
 * sqrt(y^2 + z^2) is formed by that expression instead of libm's hypot (the two differ by
 * at most one unit in the last place); the CUDA kernels form it the same way, so the two
 * agree bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

static inline double bto_radius(double y, double z) { return sqrt(y * y + z * z); }

static inline double bto_lorentz(double u0, double u1, double u2, double inv_c2) {
    return sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2);
}

static inline i64 bto_floor(double s) { return (i64)floor(s); }

/* staggered_field_2d_pyccel.py:13-55 */
void bto_staggered_field_2d(const double *px, const double *py, i64 n, const double *fx,
                            const double *fy, i64 nx, i64 ny, double origin_x,
                            double origin_y, double h, double *ex, double *ey) {
    /* fx (nx + 1, ny), fy (nx, ny + 1) */
#pragma omp parallel for schedule(static)
    for (i64 k = 0; k < n; ++k) {
        double sx = (px[k] - origin_x) / h;
        double sy = (py[k] - origin_y) / h;
        double s = sx + 0.5;
        i64 i = bto_floor(s);
        if (i < 0) i = 0;
        if (i > nx - 1) i = nx - 1;
        i64 j = bto_floor(sy);
        if (j < 0) j = 0;
        if (j > ny - 2) j = ny - 2;
        double u = s - (double)i;
        double w = sy - (double)j;
        double low = fx[i * ny + j] + w * (fx[i * ny + j + 1] - fx[i * ny + j]);
        double high = fx[(i + 1) * ny + j] + w * (fx[(i + 1) * ny + j + 1] - fx[(i + 1) * ny + j]);
        ex[k] = low + u * (high - low);
        double t = sy + 0.5;
        i = bto_floor(sx);
        if (i < 0) i = 0;
        if (i > nx - 2) i = nx - 2;
        j = bto_floor(t);
        if (j < 0) j = 0;
        if (j > ny - 1) j = ny - 1;
        u = sx - (double)i;
        w = t - (double)j;
        i64 m = ny + 1;
        low = fy[i * m + j] + w * (fy[i * m + j + 1] - fy[i * m + j]);
        high = fy[(i + 1) * m + j] + w * (fy[(i + 1) * m + j + 1] - fy[(i + 1) * m + j]);
        ey[k] = low + u * (high - low);
    }
}

/* deposit_trajectories_2d_pyccel.py:13-59; charge (nx, ny) is added to in order k = 0..n-1 */
void bto_deposit_trajectories_2d(const double *px, const double *py, const double *q, i64 n,
                                 double origin_x, double origin_y, double h, i64 cylindrical,
                                 double *charge, i64 nx, i64 ny) {
    for (i64 k = 0; k < n; ++k) {
        double x = px[k], y = py[k];
        i64 i = bto_floor((x - origin_x) / h);
        i64 j = bto_floor((y - origin_y) / h);
        double t = (x - (origin_x + h * (double)i)) / h;
        double u;
        if (cylindrical != 0) {
            double r1 = origin_y + h * (double)j;
            double r2 = r1 + h;
            u = (y * y - r1 * r1) / (r2 * r2 - r1 * r1);
        } else {
            u = (y - (origin_y + h * (double)j)) / h;
        }
        if (i < 0) {
            t = 0.0;
            i = 0;
        } else if (i >= nx - 1) {
            t = 1.0;
            i = nx - 2;
        }
        if (j < 0) {
            u = 0.0;
            j = 0;
        } else if (j >= ny - 1) {
            u = 1.0;
            j = ny - 2;
        }
        double value = q[k];
        charge[i * ny + j] += (1.0 - t) * (1.0 - u) * value;
        charge[i * ny + j + 1] += (1.0 - t) * u * value;
        charge[(i + 1) * ny + j] += t * (1.0 - u) * value;
        charge[(i + 1) * ny + j + 1] += t * u * value;
    }
}

/* trace_trajectories_2d_pyccel.py:19-33 */
static i64 bto_node_cell(double x, const double *nodes, i64 n) {
    i64 lo = 0, hi = n - 1;
    if (x >= nodes[n - 1]) {
        lo = n - 2;
    } else if (x > nodes[0]) {
        while (hi - lo > 1) {
            i64 mid = (lo + hi) / 2;
            if (nodes[mid] <= x)
                lo = mid;
            else
                hi = mid;
        }
    }
    return lo;
}

/* trace_trajectories_2d_pyccel.py:36-39 */
static double bto_uniform_x(double x, const double *nodes, i64 n, double x0, double h) {
    i64 c = bto_node_cell(x, nodes, n);
    return x0 + h * ((double)c + (x - nodes[c]) / (nodes[c + 1] - nodes[c]));
}

/* The arguments of trace_trajectories_2d (trace_trajectories_2d_pyccel.py:42-78), with the
 * array shapes spelled out. */
typedef struct {
    const i64 *active;
    i64 n_active;
    double *x, *v; /* (3, n) */
    i64 n;
    const double *qm, *dq;
    i64 *steps, *status, *electrode;
    const double *fxs, *fys;
    const i64 *patch_int;     /* (P, 6) */
    const double *patch_real; /* (P, 7) */
    i64 n_patches;
    double origin_x, origin_y, h, upper_x, upper_y;
    i64 cylindrical, integrator;
    double step_fraction;
    i64 max_steps;
    const i64 *cells; /* (nx - 1, ny - 1) of the last patch */
    const i64 *subcells;
    i64 refine;
    const double *planes;
    i64 n_planes;
    double *hits; /* (n, P, capacity, 8) */
    i64 capacity;
    i64 *counts; /* (n, P) */
    const i64 *path_slot;
    double *paths; /* (slots, path_capacity, 2) */
    i64 path_capacity;
    i64 *path_count;
    i64 num_threads;
    double *charge; /* (num_threads, n_nodes) */
    i64 n_nodes;
    i64 graded;
    const double *x_nodes;
    i64 n_x_nodes;
    double inv_c2;
} bto_trace_args;

/* An axisymmetric magnetic field from its on-axis profile (solver/fields.py:192-279): the
 * derivatives d^k B_z / dz^k, k = 0..order, at the samples z0 + hz i (n rows of order + 1).
 * mode 1: a cylindrical mesh, B = B_z x + B_r r^; mode 2: a planar mesh with the solenoid's
 * axis on the line y = axis_y, B = (B_z, sign(y - axis_y) B_r, 0) at r = |y - axis_y|. */
typedef struct bto_magnetic {
    int32_t mode, order;
    i64 n;
    double z0, hz, axis_y;
    const double *samples;
} bto_magnetic;

/* (B_z, B_r) at axial position z and radius r (fields.py:250-279, term by term). */
static void bto_axial_field(const bto_magnetic *m, double z, double r, double *bz_out,
                            double *br_out) {
    static const double bz_c[4] = {1.0, -1.0 / 4.0, 1.0 / 64.0, -1.0 / 2304.0};
    static const double br_c[3] = {-1.0 / 2.0, 1.0 / 16.0, -1.0 / 384.0};
    const i64 n = m->n;
    const int K = m->order + 1;
    double s = (z - m->z0) / m->hz;
    i64 i = bto_floor(s);
    if (i < 3)
        i = 3;
    else if (i > n - 5)
        i = n - 5;
    double t = s - (double)i;
    const double *lo = m->samples + i * K, *hi = lo + K;
    double d[7];
    for (int k = 0; k < K; ++k) d[k] = lo[k] + t * (hi[k] - lo[k]);
    double r2 = r * r;
    double bz = d[0], br = 0.0, power = 1.0;
    for (int k = 1; k <= m->order / 2; ++k) {
        power = power * r2;
        bz = bz + bz_c[k] * power * d[2 * k];
    }
    power = r;
    for (int k = 0; k < (m->order + 1) / 2; ++k) {
        br = br + br_c[k] * power * d[2 * k + 1];
        power = power * r2;
    }
    *bz_out = bz;
    *br_out = br;
}

/* The Cartesian B at a point (q0, q1, q2); (cy, cz) its radial unit vector on a
 * cylindrical mesh, r its radius. */
static void bto_magnetic_at(const bto_magnetic *m, double q0, double q1, double r, double cy,
                            double cz, double *b) {
    double bz, br;
    if (m->mode == 1) {
        bto_axial_field(m, q0, r, &bz, &br);
        b[0] = bz;
        b[1] = br * cy;
        b[2] = br * cz;
    } else {
        double yr = q1 - m->axis_y;
        bto_axial_field(m, q0, fabs(yr), &bz, &br);
        b[0] = bz;
        b[1] = yr < 0.0 ? -br : br;
        b[2] = 0.0;
    }
}

/* v <- Boris's kick over tau in the fields e, b (non-relativistic; tracer.py:605-616 with
 * its equations :620-621): v- = v + (tau/2) q/m E, t = (tau/2) q/m B,
 * v+ = v- + (v- + v- x t) x 2t / (1 + t^2), then + (tau/2) q/m E.  The association of the
 * operations is this restatement's own (mpiparticles' source is not available). */
static void bto_kick(double *v, const double *e, const double *b, double tau, double qm) {
    double f = 0.5 * tau * qm;
    double m0 = v[0] + f * e[0], m1 = v[1] + f * e[1], m2 = v[2] + f * e[2];
    double t0 = f * b[0], t1 = f * b[1], t2 = f * b[2];
    double d = 2.0 / (1.0 + (t0 * t0 + t1 * t1 + t2 * t2));
    double s0 = d * t0, s1 = d * t1, s2 = d * t2;
    double p0 = m0 + (m1 * t2 - m2 * t1);
    double p1 = m1 + (m2 * t0 - m0 * t2);
    double p2 = m2 + (m0 * t1 - m1 * t0);
    double w0 = m0 + (p1 * s2 - p2 * s1);
    double w1 = m1 + (p2 * s0 - p0 * s2);
    double w2 = m2 + (p0 * s1 - p1 * s0);
    v[0] = w0 + f * e[0];
    v[1] = w1 + f * e[1];
    v[2] = w2 + f * e[2];
}

/* The field E at (lq, qy) [uniform x, mesh y] from the finest patch holding it
 * (trace_trajectories_2d_pyccel.py:212-269). */
static void bto_edge_field(const bto_trace_args *a, double lq, double qy, double *ex_out,
                           double *ey_out) {
    const i64 P = a->n_patches;
    i64 pp = P - 1;
    for (i64 qq = 0; qq < P - 1; ++qq) {
        const double *pr = a->patch_real + qq * 7;
        if (lq >= pr[3] && lq <= pr[5] && qy >= pr[4] && qy <= pr[6]) {
            pp = qq;
            break;
        }
    }
    const i64 *pi = a->patch_int + pp * 6;
    const double *pr = a->patch_real + pp * 7;
    i64 pnx = pi[0], pny = pi[1], ofx = pi[2], ofy = pi[3];
    double pox = pr[0], poy = pr[1], phh = pr[2];
    double sx = (lq - pox) / phh;
    double sy = (qy - poy) / phh;
    double s = sx + 0.5;
    i64 i = bto_floor(s);
    if (i < 0)
        i = 0;
    else if (i > pnx - 1)
        i = pnx - 1;
    i64 j = bto_floor(sy);
    if (j < 0)
        j = 0;
    else if (j > pny - 2)
        j = pny - 2;
    double u = s - (double)i;
    double w = sy - (double)j;
    i64 c = ofx + i * pny + j;
    const double *fxs = a->fxs;
    double low = fxs[c] + w * (fxs[c + 1] - fxs[c]);
    double high = fxs[c + pny] + w * (fxs[c + pny + 1] - fxs[c + pny]);
    *ex_out = low + u * (high - low);
    s = sy + 0.5;
    i = bto_floor(sx);
    if (i < 0)
        i = 0;
    else if (i > pnx - 2)
        i = pnx - 2;
    j = bto_floor(s);
    if (j < 0)
        j = 0;
    else if (j > pny - 1)
        j = pny - 1;
    u = sx - (double)i;
    w = s - (double)j;
    c = ofy + i * (pny + 1) + j;
    const double *fys = a->fys;
    low = fys[c] + w * (fys[c + 1] - fys[c]);
    high = fys[c + pny + 1] + w * (fys[c + pny + 2] - fys[c + pny + 1]);
    *ey_out = low + u * (high - low);
}

/* One trajectory from its state to its end (trace_trajectories_2d_pyccel.py:134-507). */
static void bto_trace_one(const bto_trace_args *a, const bto_magnetic *mag, i64 k,
                          double *charge) {
    const i64 P = a->n_patches;
    const i64 nx = a->patch_int[(P - 1) * 6 + 0];
    const i64 ny = a->patch_int[(P - 1) * 6 + 1];
    const double origin_x = a->origin_x, origin_y = a->origin_y, h = a->h;
    const i64 cyl = a->cylindrical;
    const double inv_c2 = a->inv_c2;
    const i64 n = a->n;
    double x0 = a->x[k], x1 = a->x[n + k], x2 = a->x[2 * n + k];
    double v0 = a->v[k], v1 = a->v[n + k], v2 = a->v[2 * n + k];
    const double qmk = a->qm[k];
    const i64 slot = a->path_slot[k];
    i64 ns = a->steps[k];
    i64 st = -1;
    double dt = 0.0, hdt = 0.0, dt6 = 0.0;
    const int nstage = a->integrator == 0 ? 4 : 2;
    int have = 0;
    double ca0 = 0.0, ca1 = 0.0, ca2 = 0.0;
    double cE[3] = {0, 0, 0}, cB[3] = {0, 0, 0};  /* with B: the fields at the step's end */
    while (ns < a->max_steps) {
        /* the spacing of the finest patch at the step's start */
        double rr = x1;
        if (cyl == 1)
            rr = bto_radius(x1, x2);
        else if (cyl == 2)
            rr = origin_y + fabs(x1 - origin_y);
        double lx = x0;
        if (a->graded) lx = bto_uniform_x(x0, a->x_nodes, a->n_x_nodes, origin_x, h);
        double hloc = h;
        for (i64 qq = 0; qq < P - 1; ++qq) {
            const double *pr = a->patch_real + qq * 7;
            if (lx >= pr[3] && lx <= pr[5] && rr >= pr[4] && rr <= pr[6]) {
                hloc = pr[2];
                break;
            }
        }
        if (a->graded) {
            i64 cg = bto_node_cell(x0, a->x_nodes, a->n_x_nodes);
            if (mag) {
                /* the NumPy tracer's spacing: the smaller of the cell's edge and h
                   (mesh.py:197-202) */
                double dxc = a->x_nodes[cg + 1] - a->x_nodes[cg];
                if (dxc < hloc) hloc = dxc;
            } else {
                double d2 = (a->x_nodes[cg + 1] - a->x_nodes[cg]) / h;
                if (d2 < 1.0) hloc = hloc * d2;
            }
        }
        double gv = 1.0 / bto_lorentz(v0, v1, v2, inv_c2);
        double q0 = x0, q1 = x1, q2 = x2;
        double kx0 = v0, kx1 = v1, kx2 = v2;
        double sx0 = 0, sx1 = 0, sx2 = 0, sv0 = 0, sv1 = 0, sv2 = 0;
        double w0 = 0, w1 = 0, w2 = 0, y0, y1, y2;
        for (int stage = 0; stage < nstage; ++stage) {
            double gk = 1.0 / bto_lorentz(kx0, kx1, kx2, inv_c2);
            double g0, g1, g2;
            double E[3], B[3];
            if (mag && stage == 0 && have != 0) {
                for (int c = 0; c < 3; ++c) {
                    E[c] = cE[c];
                    B[c] = cB[c];
                }
            }
            if (mag && !(stage == 0 && have != 0)) {
                /* E and B at the stage point (tracer.py:547-583) */
                double qy = q1, cy = 0.0, cz = 0.0;
                if (cyl == 1) {
                    double r = bto_radius(q1, q2);
                    if (r > 0.0) {
                        cy = q1 / r;
                        cz = q2 / r;
                    }
                    qy = r;
                }
                double lq = q0;
                if (a->graded) lq = bto_uniform_x(q0, a->x_nodes, a->n_x_nodes, origin_x, h);
                double ex, ey;
                bto_edge_field(a, lq, qy, &ex, &ey);
                if (cyl != 0) {
                    E[0] = ex;
                    E[1] = ey * cy;
                    E[2] = ey * cz;
                } else {
                    E[0] = ex;
                    E[1] = ey;
                    E[2] = 0.0;
                }
                bto_magnetic_at(mag, q0, q1, qy, cy, cz, B);
            }
            if (mag) {
                /* q/m (E + v x B) at the stage velocity (tracer.py:519-529) */
                double c0 = kx1 * B[2] - kx2 * B[1];
                double c1 = kx2 * B[0] - kx0 * B[2];
                double c2 = kx0 * B[1] - kx1 * B[0];
                g0 = qmk * (E[0] + c0);
                g1 = qmk * (E[1] + c1);
                g2 = qmk * (E[2] + c2);
            } else if (stage == 0 && have != 0) {
                g0 = ca0;
                g1 = ca1;
                g2 = ca2;
            } else {
                double qy = q1, cy = 0.0, cz = 0.0;
                if (cyl == 1) {
                    double r = bto_radius(q1, q2);
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
                if (a->graded) lq = bto_uniform_x(q0, a->x_nodes, a->n_x_nodes, origin_x, h);
                double ex, ey;
                bto_edge_field(a, lq, qy, &ex, &ey);
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
                double a0 = g0, a1 = g1, a2 = g2;
                double speed = gv * sqrt(v0 * v0 + v1 * v1 + v2 * v2);
                double accel = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
                dt = -1.0;
                if (speed > 0.0) dt = hloc / speed;
                if (accel > 0.0) {
                    double d2 = sqrt(2.0 * hloc / accel);
                    if (dt < 0.0 || d2 < dt) dt = d2;
                }
                if (dt < 0.0) dt = hloc;
                dt = a->step_fraction * dt;
                hdt = 0.5 * dt;
                dt6 = dt / 6.0;
                if (a->integrator != 0 && mag) {
                    /* Boris with B: the kick over half the step, the drift (tracer.py:652-660) */
                    double u[3] = {v0, v1, v2};
                    bto_kick(u, E, B, hdt, qmk);
                    kx0 = u[0];
                    kx1 = u[1];
                    kx2 = u[2];
                    q0 = x0 + dt * kx0;
                    q1 = x1 + dt * kx1;
                    q2 = x2 + dt * kx2;
                    continue;
                }
                if (a->integrator != 0) {
                    /* Boris: the half kick, then the drift to the end of the step */
                    kx0 = v0 + hdt * a0;
                    kx1 = v1 + hdt * a1;
                    kx2 = v2 + hdt * a2;
                    gk = 1.0 / bto_lorentz(kx0, kx1, kx2, inv_c2);
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
            } else if (a->integrator != 0 && mag) {
                /* Boris with B: the second kick in the fields at the end of the step */
                double u[3] = {kx0, kx1, kx2};
                bto_kick(u, E, B, hdt, qmk);
                w0 = u[0];
                w1 = u[1];
                w2 = u[2];
                for (int c = 0; c < 3; ++c) {
                    cE[c] = E[c];
                    cB[c] = B[c];
                }
                have = 1;
            } else if (a->integrator != 0) {
                /* Boris: the second half kick at the end of the step */
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
                double f = stage == 1 ? hdt : dt;
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
        if (a->integrator == 0) {
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

        /* space charge: dq dt at the Hermite midpoint, area-weighted (:372-423) */
        double gw = 1.0 / bto_lorentz(w0, w1, w2, inv_c2);
        double m0 = 0.5 * (x0 + y0) + dt * (gv * v0 - gw * w0) / 8.0;
        double m1 = 0.5 * (x1 + y1) + dt * (gv * v1 - gw * w1) / 8.0;
        double m2 = 0.5 * (x2 + y2) + dt * (gv * v2 - gw * w2) / 8.0;
        if (cyl == 1)
            m1 = bto_radius(m1, m2);
        else if (cyl == 2)
            m1 = origin_y + fabs(m1 - origin_y);
        if (a->graded) m0 = bto_uniform_x(m0, a->x_nodes, a->n_x_nodes, origin_x, h);
        i64 pp = P - 1;
        for (i64 qq = 0; qq < P - 1; ++qq) {
            const double *pr = a->patch_real + qq * 7;
            if (m0 >= pr[3] && m0 <= pr[5] && m1 >= pr[4] && m1 <= pr[6]) {
                pp = qq;
                break;
            }
        }
        {
            const i64 *pi = a->patch_int + pp * 6;
            const double *pr = a->patch_real + pp * 7;
            i64 pnx = pi[0], pny = pi[1], ofn = pi[5];
            double pox = pr[0], poy = pr[1], phh = pr[2];
            i64 i = bto_floor((m0 - pox) / phh);
            i64 j = bto_floor((m1 - poy) / phh);
            double u = (m0 - (pox + phh * (double)i)) / phh;
            double w;
            if (cyl == 1) {
                double low = poy + phh * (double)j;
                double high = low + phh;
                w = (m1 * m1 - low * low) / (high * high - low * low);
            } else {
                w = (m1 - (poy + phh * (double)j)) / phh;
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
            double deposit = a->dq[k] * dt;
            i64 c = ofn + i * pny + j;
            charge[c] += (1.0 - u) * (1.0 - w) * deposit;
            charge[c + 1] += (1.0 - u) * w * deposit;
            charge[c + pny] += u * (1.0 - w) * deposit;
            charge[c + pny + 1] += u * w * deposit;
        }
        ns = ns + 1;

        /* plane crossings, linear along the step (:426-442) */
        for (i64 p = 0; p < a->n_planes; ++p) {
            double xp = a->planes[p];
            double before = x0 - xp;
            double after = y0 - xp;
            if ((before < 0.0) != (after < 0.0)) {
                double s = before / (before - after);
                i64 *cnt = a->counts + k * a->n_planes + p;
                i64 c = *cnt;
                if (c < a->capacity) {
                    double *hit = a->hits + ((k * a->n_planes + p) * a->capacity + c) * 8;
                    hit[0] = xp;
                    hit[1] = x1 + s * (y1 - x1);
                    hit[2] = x2 + s * (y2 - x2);
                    hit[3] = gv * v0 + s * (gw * w0 - gv * v0);
                    hit[4] = gv * v1 + s * (gw * w1 - gv * v1);
                    hit[5] = gv * v2 + s * (gw * w2 - gv * v2);
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

        /* the end of the step: off the mesh or in an electrode (:450-497) */
        double px = x0, py = x1;
        if (cyl == 1)
            py = bto_radius(x1, x2);
        else if (cyl == 2)
            py = origin_y + fabs(x1 - origin_y);
        if (slot >= 0) {
            i64 c = a->path_count[slot];
            if (c < a->path_capacity) {
                a->paths[(slot * a->path_capacity + c) * 2 + 0] = px;
                a->paths[(slot * a->path_capacity + c) * 2 + 1] = py;
            }
            a->path_count[slot] = c + 1;
        }
        if (a->graded) px = bto_uniform_x(px, a->x_nodes, a->n_x_nodes, origin_x, h);
        if (px >= a->upper_x) {
            st = 0;
        } else if (px < origin_x) {
            st = 1;
        } else if (py > a->upper_y || (cyl == 0 && py < origin_y)) {
            st = 2;
        } else {
            i64 i = (i64)((px - origin_x) / h);
            if (i > nx - 2) i = nx - 2;
            i64 j = (i64)((py - origin_y) / h);
            if (j > ny - 2) j = ny - 2;
            /* a point below the mesh (only a malformed geometry puts one there) takes
               its first cell, where the reference indexes outside the table */
            if (i < 0) i = 0;
            if (j < 0) j = 0;
            i64 cell = a->cells[i * (ny - 1) + j];
            if (cell >= 0 && mag) {
                /* the NumPy tracer tests the exact electrode shapes in every cell touching
                   one (tracer.py:1019-1024): the caller decides */
                st = -2;
            } else if (cell >= 0) {
                i64 R = a->refine;
                i64 si = (i64)(((px - origin_x) / h - (double)i) * (double)R);
                if (si < 0)
                    si = 0;
                else if (si > R - 1)
                    si = R - 1;
                i64 sj = (i64)(((py - origin_y) / h - (double)j) * (double)R);
                if (sj < 0)
                    sj = 0;
                else if (sj > R - 1)
                    sj = R - 1;
                i64 e = a->subcells[(cell * R + si) * R + sj];
                if (e >= 0) {
                    st = 3;
                    a->electrode[k] = e;
                } else if (e == -2) {
                    st = -2;
                }
            }
        }
        if (st != -1) break;
    }
    if (st == -1) st = 4;
    a->x[k] = x0;
    a->x[n + k] = x1;
    a->x[2 * n + k] = x2;
    a->v[k] = v0;
    a->v[n + k] = v1;
    a->v[2 * n + k] = v2;
    a->steps[k] = ns;
    a->status[k] = st;
}

/* trace_trajectories_2d: thread t traces every num_threads-th active trajectory into its
 * own charge slab (trace_trajectories_2d_pyccel.py:129-135). */
void bto_trace_trajectories_2d(const bto_trace_args *a) {
    const i64 T = a->num_threads;
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (i64 t = 0; t < T; ++t) {
        double *slab = a->charge + t * a->n_nodes;
        for (i64 m = t; m < a->n_active; m += T) bto_trace_one(a, NULL, a->active[m], slab);
    }
}

/* The NumPy tracer's step in a magnetic field (tracer.py:851-1054 with _rk4 / _boris and
 * AxisymmetricMagneticField), each trajectory to its end or to a cell touching an
 * electrode (status -2, where the caller tests the electrodes' shapes).  Needs inv_c2 = 0
 * and one patch. */
void bto_trace_magnetic_2d(const bto_trace_args *a, const bto_magnetic *m) {
    const i64 T = a->num_threads;
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (i64 t = 0; t < T; ++t) {
        double *slab = a->charge + t * a->n_nodes;
        for (i64 q = t; q < a->n_active; q += T) bto_trace_one(a, m, a->active[q], slab);
    }
}

int bto_num_procs(void) {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}
