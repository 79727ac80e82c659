// The adjoint of the trace: the reverse of trace.cu's RK4 step for the differentiation form
// of the design workload (planar or cylindrical, RK4, one uniform patch, no magnetic
// field, not relativistic).  No counterpart in the reference, which differentiates by
// finite differences of whole solves.
//
// The trace maps the edge fields (fx, fy) to the node charges it deposits and the plane
// crossings it records.  Given the adjoints of those outputs -- charge_seed on the nodes,
// hit_seed on the crossings' points and velocities -- the sweep accumulates the adjoint
// of the edge fields: every gather of the field at a stage point is reversed into a
// scatter onto the same four edges with the same bilinear weights, so gather and deposit
// are each other's transposes.
//
// One thread per trajectory.  A first pass replays every trajectory for the steps it took
// in the forward trace and keeps its state every kSegment steps (checkpoints, the memory
// bound: 6 doubles a trajectory every 64 steps).  The sweep walks the segments from the
// last: it replays a segment's steps from its checkpoint into local memory, then reverses
// them one by one (each step recomputed from its start state), carrying the adjoint of the
// trajectory's state backwards.  The replay is the trace's step, term by term, in the same
// order and with the same roundings (--fmad=false), so it visits the same states bit for
// bit.  The non-smooth parts of the step are taken as they fell in the forward trace: the
// branch of the step size's minimum, the cells of every lookup, the crossings, the clamps
// of the deposit at the mesh's edges.  The scatter adds each run of gathers in one cell in
// registers and the runs' sums to the edges by atomic additions (their order varies from
// run to run, so the adjoint is reproducible to rounding, not bit for bit).
#include "common.cuh"

namespace bt {
namespace {

constexpr int kSegment = 64;   // steps between checkpoints
constexpr int kMaxPlanes = 8;  // plane crossings the sweep follows
// One warp a block: a solve's few thousand trajectories spread over every SM (128-thread
// blocks left most of the 148 SMs idle on 8,000 trajectories).
constexpr int kAdjThreads = 32;

struct Grid {
    const double *fx, *fy;
    int nx, ny;
    double ox, oy, h, rh;
};

__device__ __forceinline__ int clamp_cell(int i, int lo, int hi) { return min(max(i, lo), hi); }

// The field lookup of trace.cu (edge_field_cells, the same expressions) at cell coordinates
// (sx, sy), with its cells, weights and the derivatives along them.
struct Lookup {
    int ix, jx, iy, jy;
    double ux, wx, uy, wy;
    double ex, ey;
    double dex_du, dex_dw, dey_du, dey_dw;
};

__device__ __forceinline__ void lookup(const Grid &G, double sx, double sy, Lookup &g) {
    double s = sx + 0.5;
    int i = clamp_cell(__double2int_rd(s), 0, G.nx - 1);
    int j = clamp_cell(__double2int_rd(sy), 0, G.ny - 2);
    double u = s - (double)i;
    double w = sy - (double)j;
    const double *f = G.fx + (i64)i * G.ny + j;
    double f00 = __ldg(f), f01 = __ldg(f + 1), f10 = __ldg(f + G.ny), f11 = __ldg(f + G.ny + 1);
    double low = f00 + w * (f01 - f00);
    double high = f10 + w * (f11 - f10);
    g.ex = low + u * (high - low);
    g.ix = i;
    g.jx = j;
    g.ux = u;
    g.wx = w;
    g.dex_du = high - low;
    g.dex_dw = (1.0 - u) * (f01 - f00) + u * (f11 - f10);
    s = sy + 0.5;
    i = clamp_cell(__double2int_rd(sx), 0, G.nx - 2);
    j = clamp_cell(__double2int_rd(s), 0, G.ny - 1);
    u = sx - (double)i;
    w = s - (double)j;
    f = G.fy + (i64)i * (G.ny + 1) + j;
    f00 = __ldg(f);
    f01 = __ldg(f + 1);
    f10 = __ldg(f + G.ny + 1);
    f11 = __ldg(f + G.ny + 2);
    low = f00 + w * (f01 - f00);
    high = f10 + w * (f11 - f10);
    g.ey = low + u * (high - low);
    g.iy = i;
    g.jy = j;
    g.uy = u;
    g.wy = w;
    g.dey_du = high - low;
    g.dey_dw = (1.0 - u) * (f01 - f00) + u * (f11 - f10);
}

// q/m E at a point, as trace.cu forms it (the radius and its unit vector in cylindrical
// geometry).
template <int CYL>
__device__ __forceinline__ void accel(const Grid &G, double qm, const double *q, double *a) {
    double qy = q[1], cy = 0.0, cz = 0.0;
    if (CYL == 1) {
        const double r = radius(q[1], q[2]);
        if (r > 0.0) {
            cy = q[1] / r;
            cz = q[2] / r;
        }
        qy = r;
    }
    Lookup g;
    lookup(G, div_known(q[0] - G.ox, G.h, G.rh), div_known(qy - G.oy, G.h, G.rh), g);
    if (CYL == 1) {
        a[0] = qm * g.ex;
        a[1] = qm * (g.ey * cy);
        a[2] = qm * (g.ey * cz);
    } else {
        a[0] = qm * g.ex;
        a[1] = qm * g.ey;
        a[2] = qm * 0.0;
    }
}

// One RK4 step of trace.cu (uniform mesh, gamma = 1), keeping what its reverse needs.
struct StepTape {
    double y[3], w[3];     // the end state
    double a[4][3];        // the stage accelerations
    double q[3][3];        // the stage points of stages 2-4
    double u[3][3];        // the stage velocities of stages 2-4
    double dt, speed, accn;
    int branch;            // the step size from 0: h, 1: h / |v|, 2: sqrt(2 h / |a|)
};

template <int CYL>
__device__ __forceinline__ void step_forward(const Grid &G, double qm, double f, const double *x,
                                             const double *v, StepTape &T) {
    accel<CYL>(G, qm, x, T.a[0]);
    const double *a1 = T.a[0];
    const double speed = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double accn = sqrt(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]);
    double dt = -1.0;
    int branch = 0;
    if (speed > 0.0) {
        dt = G.h / speed;
        branch = 1;
    }
    if (accn > 0.0) {
        const double d2 = sqrt(2.0 * G.h / accn);
        if (dt < 0.0 || d2 < dt) {
            dt = d2;
            branch = 2;
        }
    }
    if (dt < 0.0) {
        dt = G.h;
        branch = 0;
    }
    dt = f * dt;
    const double hdt = 0.5 * dt;
    const double dt6 = div_known(dt, 6.0, 1.0 / 6.0);
    double sx[3], sv[3], kx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        sx[c] = v[c];
        sv[c] = a1[c];
        T.q[0][c] = x[c] + hdt * v[c];
        kx[c] = v[c] + hdt * a1[c];
        T.u[0][c] = kx[c];
    }
    accel<CYL>(G, qm, T.q[0], T.a[1]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        sx[c] = sx[c] + 2.0 * kx[c];
        sv[c] = sv[c] + 2.0 * T.a[1][c];
        T.q[1][c] = x[c] + hdt * kx[c];
        kx[c] = v[c] + hdt * T.a[1][c];
        T.u[1][c] = kx[c];
    }
    accel<CYL>(G, qm, T.q[1], T.a[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        sx[c] = sx[c] + 2.0 * kx[c];
        sv[c] = sv[c] + 2.0 * T.a[2][c];
        T.q[2][c] = x[c] + dt * kx[c];
        kx[c] = v[c] + dt * T.a[2][c];
        T.u[2][c] = kx[c];
    }
    accel<CYL>(G, qm, T.q[2], T.a[3]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        sx[c] = sx[c] + kx[c];
        sv[c] = sv[c] + T.a[3][c];
        T.y[c] = x[c] + dt6 * sx[c];
        T.w[c] = v[c] + dt6 * sv[c];
    }
    T.dt = dt;
    T.speed = speed;
    T.accn = accn;
    T.branch = branch;
}

// The edge fields' adjoint, added run by run: consecutive lookups in one cell add into
// registers, a change of cell adds the run to the four edges.
struct Scatter {
    double *fxb, *fyb;
    int ny;
    i64 kx = -1, ky = -1;
    double ax[4] = {0, 0, 0, 0}, ay[4] = {0, 0, 0, 0};

    __device__ __forceinline__ void flush() {
        if (kx >= 0) {
            atomicAdd(fxb + kx, ax[0]);
            atomicAdd(fxb + kx + 1, ax[1]);
            atomicAdd(fxb + kx + ny, ax[2]);
            atomicAdd(fxb + kx + ny + 1, ax[3]);
        }
        if (ky >= 0) {
            atomicAdd(fyb + ky, ay[0]);
            atomicAdd(fyb + ky + 1, ay[1]);
            atomicAdd(fyb + ky + ny + 1, ay[2]);
            atomicAdd(fyb + ky + ny + 2, ay[3]);
        }
        kx = ky = -1;
    }

    __device__ __forceinline__ void add(const Lookup &g, double exb, double eyb) {
        const i64 key_x = (i64)g.ix * ny + g.jx;
        if (key_x != kx) {
            if (kx >= 0) {
                atomicAdd(fxb + kx, ax[0]);
                atomicAdd(fxb + kx + 1, ax[1]);
                atomicAdd(fxb + kx + ny, ax[2]);
                atomicAdd(fxb + kx + ny + 1, ax[3]);
            }
            kx = key_x;
            ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
        }
        ax[0] += exb * ((1.0 - g.ux) * (1.0 - g.wx));
        ax[1] += exb * ((1.0 - g.ux) * g.wx);
        ax[2] += exb * (g.ux * (1.0 - g.wx));
        ax[3] += exb * (g.ux * g.wx);
        const i64 key_y = (i64)g.iy * (ny + 1) + g.jy;
        if (key_y != ky) {
            if (ky >= 0) {
                atomicAdd(fyb + ky, ay[0]);
                atomicAdd(fyb + ky + 1, ay[1]);
                atomicAdd(fyb + ky + ny + 1, ay[2]);
                atomicAdd(fyb + ky + ny + 2, ay[3]);
            }
            ky = key_y;
            ay[0] = ay[1] = ay[2] = ay[3] = 0.0;
        }
        ay[0] += eyb * ((1.0 - g.uy) * (1.0 - g.wy));
        ay[1] += eyb * ((1.0 - g.uy) * g.wy);
        ay[2] += eyb * (g.uy * (1.0 - g.wy));
        ay[3] += eyb * (g.uy * g.wy);
    }
};

// The reverse of accel: ab the adjoint of q/m E at q; adds the point's adjoint to qb and
// the field's to the scatter.
template <int CYL>
__device__ __forceinline__ void accel_reverse(const Grid &G, double qm, const double *q,
                                              const double *ab, double *qb, Scatter &sc) {
    double qy = q[1], cy = 0.0, cz = 0.0, r = 0.0;
    if (CYL == 1) {
        r = radius(q[1], q[2]);
        if (r > 0.0) {
            cy = q[1] / r;
            cz = q[2] / r;
        }
        qy = r;
    }
    Lookup g;
    lookup(G, div_known(q[0] - G.ox, G.h, G.rh), div_known(qy - G.oy, G.h, G.rh), g);
    const double exb = qm * ab[0];
    const double eyb = CYL == 1 ? qm * (ab[1] * cy + ab[2] * cz) : qm * ab[1];
    sc.add(g, exb, eyb);
    const double sxb = exb * g.dex_du + eyb * g.dey_du;  // along x (u of either lookup)
    const double syb = exb * g.dex_dw + eyb * g.dey_dw;  // along y / r
    qb[0] += sxb / G.h;
    if (CYL == 1) {
        if (r > 0.0) {
            const double cyb = qm * g.ey * ab[1], czb = qm * g.ey * ab[2];
            const double rb = syb / G.h - (cyb * q[1] + czb * q[2]) / (r * r);
            qb[1] += cyb / r + rb * (q[1] / r);
            qb[2] += czb / r + rb * (q[2] / r);
        }
    } else {
        qb[1] += syb / G.h;
    }
}

struct Adj {
    bt_adjoint_args a;
    Grid G;
};

// The checkpoints: every trajectory replayed for its forward steps, its state kept at steps
// 0, kSegment, 2 kSegment, ...; its end state (6, n) for the caller's check.
template <int CYL>
__global__ void __launch_bounds__(kAdjThreads) adjoint_checkpoints(Adj A, double *__restrict__ end) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const bt_adjoint_args &a = A.a;
    if (k >= a.n) return;
    const i64 n = a.n;
    double x[3] = {a.x0[k], a.x0[n + k], a.x0[2 * n + k]};
    double v[3] = {a.v0[k], a.v0[n + k], a.v0[2 * n + k]};
    const i64 steps = a.steps[k];
    const double qm = a.qm[k];
    StepTape T;
    for (i64 s = 0; s < steps; ++s) {
        if (s % kSegment == 0) {
            double *c = a.checkpoints + (s / kSegment) * 6 * n + k;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                c[q * n] = x[q];
                c[(3 + q) * n] = v[q];
            }
        }
        step_forward<CYL>(A.G, qm, a.step_fraction, x, v, T);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            x[q] = T.y[q];
            v[q] = T.w[q];
        }
    }
    if (end) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            end[q * n + k] = x[q];
            end[(3 + q) * n + k] = v[q];
        }
    }
}

// The reverse of one step from (x, v): xb, vb hold the adjoint of its end state on entry
// and of its start state on return.  charge_seed: the node charges' adjoint; the hits'
// adjoints of this step's crossings come through hit_seed at the counters cnt.
template <int CYL>
__device__ void step_reverse(const Adj &A, i64 k, double qm, double dq, const double *x,
                             const double *v, double *xb, double *vb,
                             const double *__restrict__ charge_seed,
                             const double *__restrict__ hit_seed, int *cnt, Scatter &sc) {
    const bt_adjoint_args &a = A.a;
    const Grid &G = A.G;
    StepTape T;
    step_forward<CYL>(G, qm, a.step_fraction, x, v, T);
    const double dt = T.dt, hdt = 0.5 * T.dt;
    double yb[3] = {xb[0], xb[1], xb[2]}, wb[3] = {vb[0], vb[1], vb[2]};
    double xs[3] = {0, 0, 0}, vs[3] = {0, 0, 0};  // the start state's adjoint so far
    double dtb = 0.0;

    // the deposit at the step's Hermite midpoint (trace.cu's record, reversed)
    if (charge_seed) {
        double m[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) m[c] = 0.5 * (x[c] + T.y[c]) + dt * (v[c] - T.w[c]) * 0.125;
        const double mr = CYL == 1 ? radius(m[1], m[2]) : m[1];
        int i = __double2int_rd(div_known(m[0] - G.ox, G.h, G.rh));
        int j = __double2int_rd(div_known(mr - G.oy, G.h, G.rh));
        double u = div_known(m[0] - (G.ox + G.h * (double)i), G.h, G.rh);
        double w, dw_dr;
        if (CYL == 1) {
            const double low = G.oy + G.h * (double)j;
            const double high = low + G.h;
            const double span = high * high - low * low;
            w = (mr * mr - low * low) / span;
            dw_dr = 2.0 * mr / span;
        } else {
            w = div_known(mr - (G.oy + G.h * (double)j), G.h, G.rh);
            dw_dr = 1.0 / G.h;
        }
        double du_dx = 1.0 / G.h;
        if (i < 0) {
            u = 0.0;
            i = 0;
            du_dx = 0.0;
        } else if (i >= G.nx - 1) {
            u = 1.0;
            i = G.nx - 2;
            du_dx = 0.0;
        }
        if (j < 0) {
            w = 0.0;
            j = 0;
            dw_dr = 0.0;
        } else if (j >= G.ny - 1) {
            w = 1.0;
            j = G.ny - 2;
            dw_dr = 0.0;
        }
        const i64 node = (i64)i * G.ny + j;
        const double s00 = charge_seed[node], s01 = charge_seed[node + 1];
        const double s10 = charge_seed[node + G.ny], s11 = charge_seed[node + G.ny + 1];
        const double z = s00 * (1.0 - u) * (1.0 - w) + s01 * (1.0 - u) * w +
                         s10 * u * (1.0 - w) + s11 * u * w;
        const double q = dq * dt;
        dtb += dq * z;
        const double ub = q * ((s10 - s00) * (1.0 - w) + (s11 - s01) * w);
        const double wbar = q * ((s01 - s00) * (1.0 - u) + (s11 - s10) * u);
        double mb[3] = {ub * du_dx, 0.0, 0.0};
        const double mrb = wbar * dw_dr;
        if (CYL == 1) {
            if (mr > 0.0) {
                mb[1] = mrb * (m[1] / mr);
                mb[2] = mrb * (m[2] / mr);
            }
        } else {
            mb[1] = mrb;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            xs[c] += 0.5 * mb[c];
            yb[c] += 0.5 * mb[c];
            vs[c] += dt * 0.125 * mb[c];
            wb[c] -= dt * 0.125 * mb[c];
            dtb += (v[c] - T.w[c]) * 0.125 * mb[c];
        }
    }

    // the plane crossings of the step (the interpolation between its ends, reversed)
    if (hit_seed) {
        for (int p = 0; p < (int)a.n_planes; ++p) {
            const double xp = a.planes[p];
            const double before = x[0] - xp, after = T.y[0] - xp;
            if ((before < 0.0) == (after < 0.0)) continue;
            const int c = --cnt[p];
            if (c < 0 || c >= a.capacity) continue;
            const double *g = hit_seed + ((k * a.n_planes + p) * a.capacity + c) * 8;
            const double den = before - after;
            const double sc_ = before / den;
            double scb = 0.0;
#pragma unroll
            for (int q = 1; q < 3; ++q) {  // the point's y, z
                scb += g[q] * (T.y[q] - x[q]);
                xs[q] += g[q] * (1.0 - sc_);
                yb[q] += g[q] * sc_;
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {  // the velocity
                scb += g[3 + q] * (T.w[q] - v[q]);
                vs[q] += g[3 + q] * (1.0 - sc_);
                wb[q] += g[3 + q] * sc_;
            }
            xs[0] += scb * (-after / (den * den));
            yb[0] += scb * (before / (den * den));
        }
    }

    // y = x + dt/6 sx, w = v + dt/6 sv
    double sxb[3], svb[3];
    double dt6b = 0.0;
    {
        // sx and sv from the tape: v + 2 u2 + 2 u3 + u4 and a1 + 2 a2 + 2 a3 + a4
        const double dt6 = div_known(dt, 6.0, 1.0 / 6.0);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double sx = v[c] + 2.0 * T.u[0][c] + 2.0 * T.u[1][c] + T.u[2][c];
            const double sv = T.a[0][c] + 2.0 * T.a[1][c] + 2.0 * T.a[2][c] + T.a[3][c];
            xs[c] += yb[c];
            vs[c] += wb[c];
            sxb[c] = dt6 * yb[c];
            svb[c] = dt6 * wb[c];
            dt6b += yb[c] * sx + wb[c] * sv;
        }
    }
    dtb += dt6b / 6.0;
    double u2b[3], u3b[3], u4b[3], a1b[3], a2b[3], a3b[3], a4b[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vs[c] += sxb[c];
        u2b[c] = 2.0 * sxb[c];
        u3b[c] = 2.0 * sxb[c];
        u4b[c] = sxb[c];
        a1b[c] = svb[c];
        a2b[c] = 2.0 * svb[c];
        a3b[c] = 2.0 * svb[c];
        a4b[c] = svb[c];
    }
    double hdtb = 0.0;
    double qb[3] = {0, 0, 0};
    // a4 = acc(q4), q4 = x + dt u3, u4 = v + dt a3
    accel_reverse<CYL>(G, qm, T.q[2], a4b, qb, sc);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vs[c] += u4b[c];
        dtb += u4b[c] * T.a[2][c];
        a3b[c] += dt * u4b[c];
        xs[c] += qb[c];
        dtb += qb[c] * T.u[1][c];
        u3b[c] += dt * qb[c];
        qb[c] = 0.0;
    }
    // a3 = acc(q3), q3 = x + hdt u2, u3 = v + hdt a2
    accel_reverse<CYL>(G, qm, T.q[1], a3b, qb, sc);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vs[c] += u3b[c];
        hdtb += u3b[c] * T.a[1][c];
        a2b[c] += hdt * u3b[c];
        xs[c] += qb[c];
        hdtb += qb[c] * T.u[0][c];
        u2b[c] += hdt * qb[c];
        qb[c] = 0.0;
    }
    // a2 = acc(q2), q2 = x + hdt v, u2 = v + hdt a1
    accel_reverse<CYL>(G, qm, T.q[0], a2b, qb, sc);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vs[c] += u2b[c];
        hdtb += u2b[c] * T.a[0][c];
        a1b[c] += hdt * u2b[c];
        xs[c] += qb[c];
        hdtb += qb[c] * v[c];
        vs[c] += hdt * qb[c];
        qb[c] = 0.0;
    }
    dtb += 0.5 * hdtb;
    // the step size: f h / |v| or f sqrt(2 h / |a1|)
    if (T.branch == 1) {
        const double coef = -dt / (T.speed * T.speed);
#pragma unroll
        for (int c = 0; c < 3; ++c) vs[c] += dtb * coef * v[c];
    } else if (T.branch == 2) {
        const double coef = -0.5 * dt / (T.accn * T.accn);
#pragma unroll
        for (int c = 0; c < 3; ++c) a1b[c] += dtb * coef * T.a[0][c];
    }
    // a1 = acc(x)
    accel_reverse<CYL>(G, qm, x, a1b, xs, sc);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        xb[c] = xs[c];
        vb[c] = vs[c];
    }
}

// The sweep: every trajectory's steps reversed, from its last to its first.
template <int CYL>
__global__ void __launch_bounds__(kAdjThreads) adjoint_sweep(Adj A, const double *__restrict__ charge_seed,
                                                             const double *__restrict__ hit_seed,
                                                             double *__restrict__ fx_bar,
                                                             double *__restrict__ fy_bar) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const bt_adjoint_args &a = A.a;
    if (k >= a.n) return;
    const i64 n = a.n;
    const i64 steps = a.steps[k];
    if (steps <= 0) return;
    int cnt[kMaxPlanes];
    for (int p = 0; p < (int)a.n_planes; ++p) cnt[p] = (int)a.counts[k * a.n_planes + p];
    const double qm = a.qm[k], dq = a.dq[k];
    Scatter sc{fx_bar, fy_bar, A.G.ny};
    double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0};
    double tape[kSegment][6];  // the segment's start states
    const i64 segments = (steps + kSegment - 1) / kSegment;
    for (i64 seg = segments - 1; seg >= 0; --seg) {
        const double *c = a.checkpoints + seg * 6 * n + k;
        double x[3] = {c[0], c[n], c[2 * n]};
        double v[3] = {c[3 * n], c[4 * n], c[5 * n]};
        const int len = (int)min((i64)kSegment, steps - seg * kSegment);
        StepTape T;
        for (int s = 0; s < len; ++s) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                tape[s][q] = x[q];
                tape[s][3 + q] = v[q];
            }
            if (s + 1 < len) {
                step_forward<CYL>(A.G, qm, a.step_fraction, x, v, T);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    x[q] = T.y[q];
                    v[q] = T.w[q];
                }
            }
        }
        for (int s = len - 1; s >= 0; --s) {
            const double xs[3] = {tape[s][0], tape[s][1], tape[s][2]};
            const double vs[3] = {tape[s][3], tape[s][4], tape[s][5]};
            step_reverse<CYL>(A, k, qm, dq, xs, vs, xb, vb, charge_seed, hit_seed, cnt, sc);
        }
    }
    sc.flush();
}

Adj adj_of(const bt_adjoint_args *a) {
    Adj A{};
    A.a = *a;
    A.G = Grid{a->fx, a->fy, (int)a->nx, (int)a->ny, a->origin_x, a->origin_y, a->h,
               known_reciprocal(a->h)};
    return A;
}

void check_args(const bt_adjoint_args *a) {
    BT_REQUIRE(a, "adjoint: null arguments");
    BT_REQUIRE(a->n >= 0, "adjoint: negative trajectory count");
    BT_REQUIRE(a->nx >= 3 && a->ny >= 3, "adjoint: the mesh needs at least 3 nodes per axis");
    BT_REQUIRE(a->nx < (1LL << 30) && a->ny < (1LL << 30), "adjoint: mesh too large");
    BT_REQUIRE(a->cylindrical == 0 || a->cylindrical == 1,
               "adjoint: planar or cylindrical geometry only (no symmetry plane)");
    BT_REQUIRE(a->h > 0.0, "adjoint: h must be positive");
    BT_REQUIRE(a->n_planes >= 0 && a->n_planes <= kMaxPlanes, "adjoint: at most 8 planes");
    BT_REQUIRE(a->segments >= 0, "adjoint: negative checkpoint count");
    if (a->n > 0)
        BT_REQUIRE(a->x0 && a->v0 && a->qm && a->dq && a->steps && a->fx && a->fy &&
                       a->checkpoints && (a->n_planes == 0 || (a->planes && a->counts)),
                   "adjoint: null array");
}

}  // namespace
}  // namespace bt

extern "C" int bt_adjoint_checkpoints(bt_ctx *ctx, const bt_adjoint_args *a, double *end_state) {
    using namespace bt;
    return guarded([&] {
        BT_REQUIRE(ctx, "adjoint: null context");
        check_args(a);
        if (a->n == 0) return;
        const Adj A = adj_of(a);
        Timed timed(ctx, "adjoint_checkpoints");
        const unsigned grid = blocks_for(a->n, kAdjThreads);
        if (a->cylindrical)
            BT_LAUNCH(ctx, adjoint_checkpoints<1>, grid, kAdjThreads, 0, ctx->stream, A, end_state);
        else
            BT_LAUNCH(ctx, adjoint_checkpoints<0>, grid, kAdjThreads, 0, ctx->stream, A, end_state);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_adjoint_sweep(bt_ctx *ctx, const bt_adjoint_args *a, const double *charge_seed,
                                const double *hit_seed, double *fx_bar, double *fy_bar) {
    using namespace bt;
    return guarded([&] {
        BT_REQUIRE(ctx && fx_bar && fy_bar, "adjoint: null argument");
        check_args(a);
        if (a->n == 0 || (!charge_seed && !hit_seed)) return;
        const Adj A = adj_of(a);
        Timed timed(ctx, "adjoint_sweep");
        const unsigned grid = blocks_for(a->n, kAdjThreads);
        if (a->cylindrical)
            BT_LAUNCH(ctx, adjoint_sweep<1>, grid, kAdjThreads, 0, ctx->stream, A, charge_seed,
                      hit_seed, fx_bar, fy_bar);
        else
            BT_LAUNCH(ctx, adjoint_sweep<0>, grid, kAdjThreads, 0, ctx->stream, A, charge_seed,
                      hit_seed, fx_bar, fy_bar);
        BT_CHECK_LAUNCH();
    });
}
