// The 3D trajectory tracer: kernels/trace_trajectories_3d/trace_trajectories_3d_pyccel.py:19-657
// re-designed for the B200.
//
// One thread per active trajectory advances it by at most `window` steps a launch through
// the staggered edge fields of the patches (finest first, the base mesh last), with a
// magnetic field on the base mesh's nodes, symmetry planes at the lower y and z faces, the
// plane crossings, kept paths, exit and electrode sub-cell tests: the reference's step term
// by term in FP64 with no contracted multiply-add, so a trajectory ends bit for bit where the
// reference's kernel ends it.  Instead of adding to the charge with atomics, every step writes
// its eight node shares as (node, value) records to slots fixed by (window step, trajectory,
// corner); after each window the records are sorted by node (stable) and summed per node in
// record order, so the node charges are the same on every run.  The current elements (has_j)
// take the same way on the base mesh's 3 nx ny nz components.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace bt {
namespace {

struct Fields3 {
    double e[3], b[3];
};

__device__ __forceinline__ int clamp3(int i, int lo, int hi) { return min(max(i, lo), hi); }

// The first (finest) patch whose node box holds the point, else the base (the last).
__device__ __forceinline__ int finest3(const bt_trace3d_args &a, double p0, double p1, double p2) {
    for (int q = 0; q < (int)a.n_patches - 1; ++q) {
        const double *r = a.patch_real + q * 10;
        if (p0 >= __ldg(r + 4) && p0 <= __ldg(r + 7) && p1 >= __ldg(r + 5) && p1 <= __ldg(r + 8) &&
            p2 >= __ldg(r + 6) && p2 <= __ldg(r + 9))
            return q;
    }
    return (int)a.n_patches - 1;
}

// The reference's nested trilinear form at corner index ci (:231-236).
__device__ __forceinline__ double trilinear(const double *__restrict__ f, i64 ci, i64 dj, i64 di,
                                            double a, double b, double c) {
    return (1.0 - a) * ((1.0 - b) * ((1.0 - c) * __ldg(f + ci) + c * __ldg(f + ci + 1)) +
                        b * ((1.0 - c) * __ldg(f + ci + dj) + c * __ldg(f + ci + dj + 1))) +
           a * ((1.0 - b) * ((1.0 - c) * __ldg(f + ci + di) + c * __ldg(f + ci + di + 1)) +
                b * ((1.0 - c) * __ldg(f + ci + di + dj) + c * __ldg(f + ci + di + dj + 1)));
}

// E and B at a point: mirrored below a symmetry plane, E from the finest patch holding it
// (:173-335).
__device__ __forceinline__ Fields3 fields3(const bt_trace3d_args &a, i64 nx, i64 ny, i64 nz,
                                           double p0, double p1, double p2) {
    double s1 = 1.0, s2 = 1.0;
    if (a.mirror_y != 0 && p1 < a.origin_y) {
        p1 = 2.0 * a.origin_y - p1;
        s1 = -1.0;
    }
    if (a.mirror_z != 0 && p2 < a.origin_z) {
        p2 = 2.0 * a.origin_z - p2;
        s2 = -1.0;
    }
    const int pp = finest3(a, p0, p1, p2);
    const i64 *pi = a.patch_int + pp * 8;
    const double *pr = a.patch_real + pp * 10;
    const int pnx = (int)__ldg(pi), pny = (int)__ldg(pi + 1), pnz = (int)__ldg(pi + 2);
    const i64 ofx = __ldg(pi + 3), ofy = __ldg(pi + 4), ofz = __ldg(pi + 5);
    const double phh = __ldg(pr + 3);
    const double sx = (p0 - __ldg(pr)) / phh, sy = (p1 - __ldg(pr + 1)) / phh;
    const double sz = (p2 - __ldg(pr + 2)) / phh;
    Fields3 F;
    // E_x on (pnx + 1, pny, pnz) at (sx + 1/2, sy, sz)
    double s = sx + 0.5;
    int i = clamp3(__double2int_rd(s), 0, pnx - 1);
    int j = clamp3(__double2int_rd(sy), 0, pny - 2);
    int k = clamp3(__double2int_rd(sz), 0, pnz - 2);
    const double c = sz - (double)k;
    F.e[0] = trilinear(a.fxs, ofx + (i64)i * pny * pnz + (i64)j * pnz + k, pnz, (i64)pny * pnz,
                       s - (double)i, sy - (double)j, c);
    // E_y on (pnx, pny + 1, pnz) at (sx, sy + 1/2, sz)
    i = clamp3(__double2int_rd(sx), 0, pnx - 2);
    s = sy + 0.5;
    j = clamp3(__double2int_rd(s), 0, pny - 1);
    const double ax = sx - (double)i;
    i64 di = (i64)(pny + 1) * pnz;
    F.e[1] = s1 * trilinear(a.fys, ofy + i * di + (i64)j * pnz + k, pnz, di, ax, s - (double)j, c);
    // E_z on (pnx, pny, pnz + 1) at (sx, sy, sz + 1/2)
    j = clamp3(__double2int_rd(sy), 0, pny - 2);
    s = sz + 0.5;
    k = clamp3(__double2int_rd(s), 0, pnz - 1);
    di = (i64)pny * (pnz + 1);
    F.e[2] = s2 * trilinear(a.fzs, ofz + i * di + (i64)j * (pnz + 1) + k, pnz + 1, di, ax,
                            sy - (double)j, s - (double)k);
    F.b[0] = F.b[1] = F.b[2] = 0.0;
    if (a.has_b != 0) {
        // B on the base mesh's nodes (3, nx, ny, nz), the weights summed in corner order
        const double tx = (p0 - a.origin_x) / a.h, ty = (p1 - a.origin_y) / a.h;
        const double tz = (p2 - a.origin_z) / a.h;
        const int bi = clamp3(__double2int_rd(tx), 0, (int)nx - 2);
        const int bj = clamp3(__double2int_rd(ty), 0, (int)ny - 2);
        const int bk = clamp3(__double2int_rd(tz), 0, (int)nz - 2);
        const double u = tx - (double)bi, w = ty - (double)bj, z = tz - (double)bk;
        const double wt[8] = {(1.0 - u) * (1.0 - w) * (1.0 - z), (1.0 - u) * (1.0 - w) * z,
                              (1.0 - u) * w * (1.0 - z),         (1.0 - u) * w * z,
                              u * (1.0 - w) * (1.0 - z),         u * (1.0 - w) * z,
                              u * w * (1.0 - z),                 u * w * z};
        const i64 nb = nx * ny * nz, dj = nz, dI = ny * nz;
        const i64 base = (i64)bi * dI + (i64)bj * dj + bk;
        const i64 off[8] = {0, 1, dj, dj + 1, dI, dI + 1, dI + dj, dI + dj + 1};
        double comp[3];
#pragma unroll
        for (int n0 = 0; n0 < 3; ++n0) {
            const double *bn = a.bn + n0 * nb + base;
            double f = wt[0] * __ldg(bn + off[0]);
#pragma unroll
            for (int q = 1; q < 8; ++q) f = f + wt[q] * __ldg(bn + off[q]);
            comp[n0] = f;
        }
        F.b[0] = s1 * s2 * comp[0];
        F.b[1] = s2 * comp[1];
        F.b[2] = s1 * comp[2];
    }
    return F;
}

// The relativistic Boris push (J. P. Boris, 1970) of u by the scaled fields e (the kicks)
// and b (the rotation by t = b / gamma, s = 2 t / (1 + t^2)): what the reference's kernel
// calls mpiparticles' relativistic_boris_update for.
__device__ __forceinline__ void boris_push(double *u, const double *e, const double *b,
                                           double inv_c2) {
    const double m0 = u[0] + e[0], m1 = u[1] + e[1], m2 = u[2] + e[2];
    const double g = sqrt(1.0 + (m0 * m0 + m1 * m1 + m2 * m2) * inv_c2);
    const double t0 = b[0] / g, t1 = b[1] / g, t2 = b[2] / g;
    const double f = 2.0 / (1.0 + (t0 * t0 + t1 * t1 + t2 * t2));
    const double s0 = f * t0, s1 = f * t1, s2 = f * t2;
    const double p0 = m0 + (m1 * t2 - m2 * t1);
    const double p1 = m1 + (m2 * t0 - m0 * t2);
    const double p2 = m2 + (m0 * t1 - m1 * t0);
    u[0] = m0 + (p1 * s2 - p2 * s1) + e[0];
    u[1] = m1 + (p2 * s0 - p0 * s2) + e[1];
    u[2] = m2 + (p0 * s1 - p1 * s0) + e[2];
}

__device__ __forceinline__ double inv_gamma3(double u0, double u1, double u2, double inv_c2) {
    return 1.0 / sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2);
}

// A deposit point's corner node (among `nodes` of a box of (bnx, bny, bnz) from `first`) and
// its trilinear weights, the indices clamped as the reference's (:485-510).
struct Box {
    i64 cc, dj, di;
    double a, b, c;
};

__device__ __forceinline__ void clamp_axis(double s, int n, int &i, double &w) {
    i = __double2int_rd(s);
    w = s - (double)i;
    if (i < 0) {
        w = 0.0;
        i = 0;
    } else if (i >= n - 1) {
        w = 1.0;
        i = n - 2;
    }
}

__device__ __forceinline__ Box box3(i64 first, int bnx, int bny, int bnz, double sx, double sy,
                                    double sz) {
    int i, j, k;
    double a, b, c;
    clamp_axis(sx, bnx, i, a);
    clamp_axis(sy, bny, j, b);
    clamp_axis(sz, bnz, k, c);
    return {first + (i64)i * bny * bnz + (i64)j * bnz + k, bnz, (i64)bny * bnz, a, b, c};
}

// A cell's charge record: the shares of its eight corners, in the corner order (k, then j,
// then i offsets: q = 4 di + 2 dj + dk), two 32-byte sectors.
struct __align__(64) CellRec {
    double c[8];
};

// The eight shares of q, in the reference's corner order (:512-519).
__device__ __forceinline__ void shares8(const Box &B, double q, double *w) {
    const double a = B.a, b = B.b, c = B.c;
    w[0] = (1.0 - a) * (1.0 - b) * (1.0 - c) * q;
    w[1] = (1.0 - a) * (1.0 - b) * c * q;
    w[2] = (1.0 - a) * b * (1.0 - c) * q;
    w[3] = (1.0 - a) * b * c * q;
    w[4] = a * (1.0 - b) * (1.0 - c) * q;
    w[5] = a * (1.0 - b) * c * q;
    w[6] = a * b * (1.0 - c) * q;
    w[7] = a * b * c * q;
}

// The eight shares of q as records, in the reference's corner order (:512-519).
__device__ __forceinline__ void records8(const Box &B, double q, uint32_t *key, double *val) {
    const double a = B.a, b = B.b, c = B.c;
    const i64 o[8] = {0, 1, B.dj, B.dj + 1, B.di, B.di + 1, B.di + B.dj, B.di + B.dj + 1};
    const double w[8] = {(1.0 - a) * (1.0 - b) * (1.0 - c) * q, (1.0 - a) * (1.0 - b) * c * q,
                         (1.0 - a) * b * (1.0 - c) * q,         (1.0 - a) * b * c * q,
                         a * (1.0 - b) * (1.0 - c) * q,         a * (1.0 - b) * c * q,
                         a * b * (1.0 - c) * q,                 a * b * c * q};
#pragma unroll
    for (int q8 = 0; q8 < 8; ++q8) {
        key[q8] = (uint32_t)(B.cc + o[q8]);
        val[q8] = w[q8];
    }
}

}  // namespace
}  // namespace bt

namespace bt {
namespace {

struct Trace3 {
    bt_trace3d_args a;
    i64 nx, ny, nz;       // the base mesh's nodes
    int S;                // steps a window
    uint32_t sentinel;    // a slot with no charge record
    uint32_t jsentinel;   // a slot with no current record
};

// One window of trajectory m (of the active list): at most S steps from its state.  The
// charge of a run of consecutive steps in one cell is summed into one cell record (key: the
// cell's lower corner node), written to the slot (s n_active + m) of the run's last step s;
// with has_j, each step's current shares go to the slots ((s n_active + m) 24 + 8 component
// + corner).  The slots with no record hold the sentinels.  alive[m]: the trajectory has not ended (cleared here when
// it does, with its status written); *live counts the ones still going after the window.
__global__ void __launch_bounds__(128) trace3d_window(Trace3 T, uint8_t *__restrict__ alive,
                                                      uint32_t *__restrict__ keys,
                                                      CellRec *__restrict__ recs,
                                                      uint32_t *__restrict__ jkeys,
                                                      double *__restrict__ jvals,
                                                      unsigned long long *__restrict__ live) {
    const bt_trace3d_args &a = T.a;
    const i64 m = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 na = a.n_active;
    if (m >= na) return;
    const int S = T.S;
    const bool j_on = a.has_j != 0;
    int s = 0;
    if (alive[m]) {
        const i64 k = a.active[m];
        const i64 n = a.n;
        const i64 nx = T.nx, ny = T.ny, nz = T.nz;
        double x0 = a.x[k], x1 = a.x[n + k], x2 = a.x[2 * n + k];
        double v0 = a.v[k], v1 = a.v[n + k], v2 = a.v[2 * n + k];
        const double qmk = a.qm[k], dqk = a.dq[k], inv_c2 = a.inv_c2;
        const i64 slot = a.path_slot[k];
        i64 ns = a.steps[k];
        i64 st = -1;
        bool have = false;
        Fields3 cache{};
        // the current run of steps in one cell: its slot, key and summed shares
        i64 run_slot = -1;
        uint32_t run_key = T.sentinel;
        double run[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (; s < S && ns < a.max_steps; ++s) {
            // the spacing of the finest patch at the step's start (:148-163)
            double p1 = x1, p2 = x2;
            if (a.mirror_y != 0 && p1 < a.origin_y) p1 = 2.0 * a.origin_y - p1;
            if (a.mirror_z != 0 && p2 < a.origin_z) p2 = 2.0 * a.origin_z - p2;
            double hloc = a.h;
            {
                const int q = finest3(a, x0, p1, p2);
                if (q < (int)a.n_patches - 1) hloc = __ldg(a.patch_real + q * 10 + 3);
            }
            const double gv = inv_gamma3(v0, v1, v2, inv_c2);
            Fields3 F = (a.integrator != 0 && have) ? cache : fields3(a, nx, ny, nz, x0, x1, x2);
            double gk = inv_gamma3(v0, v1, v2, inv_c2);
            double g0 = qmk * (F.e[0] + gk * v1 * F.b[2] - gk * v2 * F.b[1]);
            double g1 = qmk * (F.e[1] + gk * v2 * F.b[0] - gk * v0 * F.b[2]);
            double g2 = qmk * (F.e[2] + gk * v0 * F.b[1] - gk * v1 * F.b[0]);
            const double speed = gv * sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            const double accel = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
            double dt = -1.0;
            if (speed > 0.0) dt = hloc / speed;
            if (accel > 0.0) {
                const double d2 = sqrt(2.0 * hloc / accel);
                if (dt < 0.0 || d2 < dt) dt = d2;
            }
            if (dt < 0.0) dt = hloc;
            dt = a.step_fraction * dt;
            const double hdt = 0.5 * dt;
            double y0, y1, y2, w0, w1, w2;
            if (a.integrator != 0) {
                // Boris: a half step's kick--rotate--kick, the drift, the second at the end
                const double tau = 0.5 * hdt * qmk;
                double u[3] = {v0, v1, v2};
                double e[3] = {tau * F.e[0], tau * F.e[1], tau * F.e[2]};
                double b[3] = {tau * F.b[0], tau * F.b[1], tau * F.b[2]};
                boris_push(u, e, b, inv_c2);
                gk = inv_gamma3(u[0], u[1], u[2], inv_c2);
                y0 = x0 + dt * gk * u[0];
                y1 = x1 + dt * gk * u[1];
                y2 = x2 + dt * gk * u[2];
                F = fields3(a, nx, ny, nz, y0, y1, y2);
                e[0] = tau * F.e[0];
                e[1] = tau * F.e[1];
                e[2] = tau * F.e[2];
                b[0] = tau * F.b[0];
                b[1] = tau * F.b[1];
                b[2] = tau * F.b[2];
                boris_push(u, e, b, inv_c2);
                w0 = u[0];
                w1 = u[1];
                w2 = u[2];
                cache = F;
                have = true;
            } else {
                const double dt6 = dt / 6.0;
                double sx0 = gv * v0, sx1 = gv * v1, sx2 = gv * v2;
                double sv0 = g0, sv1 = g1, sv2 = g2;
                double q0 = x0 + hdt * gv * v0, q1 = x1 + hdt * gv * v1, q2 = x2 + hdt * gv * v2;
                double k0 = v0 + hdt * g0, k1 = v1 + hdt * g1, k2 = v2 + hdt * g2;
                for (int stage = 1; stage < 4; ++stage) {
                    F = fields3(a, nx, ny, nz, q0, q1, q2);
                    gk = inv_gamma3(k0, k1, k2, inv_c2);
                    g0 = qmk * (F.e[0] + gk * k1 * F.b[2] - gk * k2 * F.b[1]);
                    g1 = qmk * (F.e[1] + gk * k2 * F.b[0] - gk * k0 * F.b[2]);
                    g2 = qmk * (F.e[2] + gk * k0 * F.b[1] - gk * k1 * F.b[0]);
                    if (stage < 3) {
                        sx0 = sx0 + 2.0 * gk * k0;
                        sx1 = sx1 + 2.0 * gk * k1;
                        sx2 = sx2 + 2.0 * gk * k2;
                        sv0 = sv0 + 2.0 * g0;
                        sv1 = sv1 + 2.0 * g1;
                        sv2 = sv2 + 2.0 * g2;
                        const double f = stage == 1 ? hdt : dt;
                        q0 = x0 + f * gk * k0;
                        q1 = x1 + f * gk * k1;
                        q2 = x2 + f * gk * k2;
                        k0 = v0 + f * g0;
                        k1 = v1 + f * g1;
                        k2 = v2 + f * g2;
                    } else {
                        sx0 = sx0 + gk * k0;
                        sx1 = sx1 + gk * k1;
                        sx2 = sx2 + gk * k2;
                        sv0 = sv0 + g0;
                        sv1 = sv1 + g1;
                        sv2 = sv2 + g2;
                    }
                }
                y0 = x0 + dt6 * sx0;
                y1 = x1 + dt6 * sx1;
                y2 = x2 + dt6 * sx2;
                w0 = v0 + dt6 * sv0;
                w1 = v1 + dt6 * sv1;
                w2 = v2 + dt6 * sv2;
            }
            // the space charge dq dt at the step's Hermite midpoint (:451-519)
            const double gw = inv_gamma3(w0, w1, w2, inv_c2);
            const double m0 = 0.5 * (x0 + y0) + dt * (gv * v0 - gw * w0) / 8.0;
            double m1 = 0.5 * (x1 + y1) + dt * (gv * v1 - gw * w1) / 8.0;
            double m2 = 0.5 * (x2 + y2) + dt * (gv * v2 - gw * w2) / 8.0;
            if (a.mirror_y != 0 && m1 < a.origin_y) m1 = 2.0 * a.origin_y - m1;
            if (a.mirror_z != 0 && m2 < a.origin_z) m2 = 2.0 * a.origin_z - m2;
            {
                const int pp = finest3(a, m0, m1, m2);
                const i64 *pi = a.patch_int + pp * 8;
                const double *pr = a.patch_real + pp * 10;
                const double phh = __ldg(pr + 3);
                const Box B = box3(__ldg(pi + 7), (int)__ldg(pi), (int)__ldg(pi + 1),
                                   (int)__ldg(pi + 2), (m0 - __ldg(pr)) / phh,
                                   (m1 - __ldg(pr + 1)) / phh, (m2 - __ldg(pr + 2)) / phh);
                double w[8];
                shares8(B, dqk * dt, w);
                const uint32_t key = (uint32_t)B.cc;
                const i64 at = (i64)s * na + m;
                if (run_slot >= 0 && key == run_key) {
                    keys[run_slot] = T.sentinel;  // the run moves on to this step's slot
#pragma unroll
                    for (int q = 0; q < 8; ++q) run[q] = run[q] + w[q];
                } else {
                    if (run_slot >= 0) {
                        keys[run_slot] = run_key;
                        CellRec r;
#pragma unroll
                        for (int q = 0; q < 8; ++q) r.c[q] = run[q];
                        recs[run_slot] = r;
                    }
                    run_key = key;
#pragma unroll
                    for (int q = 0; q < 8; ++q) run[q] = w[q];
                }
                run_slot = at;
                keys[at] = T.sentinel;
            }
            if (j_on) {
                // the current element dq (x' - x) on the base mesh (:520-565)
                double jd[3] = {dqk * (y0 - x0), dqk * (y1 - x1), dqk * (y2 - x2)};
                if (a.mirror_y != 0 && 0.5 * (x1 + y1) < a.origin_y) jd[1] = -jd[1];
                if (a.mirror_z != 0 && 0.5 * (x2 + y2) < a.origin_z) jd[2] = -jd[2];
                const Box B = box3(0, (int)nx, (int)ny, (int)nz, (m0 - a.origin_x) / a.h,
                                   (m1 - a.origin_y) / a.h, (m2 - a.origin_z) / a.h);
                const i64 at = ((i64)s * na + m) * 24;
                const i64 nb = nx * ny * nz;
#pragma unroll
                for (int jc = 0; jc < 3; ++jc) {
                    Box C = B;
                    C.cc = B.cc + jc * nb;
                    records8(C, jd[jc], jkeys + at + 8 * jc, jvals + at + 8 * jc);
                }
            }
            ns = ns + 1;
            for (i64 p = 0; p < a.n_planes; ++p) {
                const double xp = a.planes[p];
                const double before = x0 - xp, after = y0 - xp;
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
            // the end of the step: off the mesh or in an electrode (:587-641)
            const double px = x0;
            double py = x1, pz = x2;
            if (a.mirror_y != 0 && py < a.origin_y) py = 2.0 * a.origin_y - py;
            if (a.mirror_z != 0 && pz < a.origin_z) pz = 2.0 * a.origin_z - pz;
            if (slot >= 0) {
                const i64 c = a.path_count[slot];
                if (c < a.path_capacity) {
                    double *path = a.paths + (slot * a.path_capacity + c) * 3;
                    path[0] = px;
                    path[1] = py;
                    path[2] = pz;
                }
                a.path_count[slot] = c + 1;
            }
            if (px >= a.upper_x) {
                st = 0;
            } else if (px < a.origin_x) {
                st = 1;
            } else if (py > a.upper_y || py < a.origin_y || pz > a.upper_z || pz < a.origin_z) {
                st = 2;
            } else {
                const double ux = (px - a.origin_x) / a.h, uy = (py - a.origin_y) / a.h;
                const double uz = (pz - a.origin_z) / a.h;
                const int i = min(__double2int_rz(ux), (int)nx - 2);
                const int j = min(__double2int_rz(uy), (int)ny - 2);
                const int kz = min(__double2int_rz(uz), (int)nz - 2);
                const i64 cell = __ldg(a.cells + ((i64)i * (ny - 1) + j) * (nz - 1) + kz);
                if (cell >= 0) {
                    const int R = (int)a.refine;
                    const int si = clamp3(__double2int_rz((ux - (double)i) * (double)R), 0, R - 1);
                    const int sj = clamp3(__double2int_rz((uy - (double)j) * (double)R), 0, R - 1);
                    const int sk = clamp3(__double2int_rz((uz - (double)kz) * (double)R), 0, R - 1);
                    const i64 e = __ldg(a.subcells + ((cell * R + si) * R + sj) * R + sk);
                    if (e >= 0) {
                        st = 3;
                        a.electrode[k] = e;
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
            CellRec r;
#pragma unroll
            for (int q = 0; q < 8; ++q) r.c[q] = run[q];
            recs[run_slot] = r;
        }
        if (st == -1 && ns >= a.max_steps) st = 4;
        a.x[k] = x0;
        a.x[n + k] = x1;
        a.x[2 * n + k] = x2;
        a.v[k] = v0;
        a.v[n + k] = v1;
        a.v[2 * n + k] = v2;
        a.steps[k] = ns;
        if (st != -1) {
            a.status[k] = st;
            alive[m] = 0;
        } else {
            atomicAdd(live, 1ull);
        }
    }
    // the slots of the steps not taken hold no record
    for (; s < S; ++s) {
        keys[(i64)s * na + m] = T.sentinel;
        if (j_on) {
            const i64 jt = ((i64)s * na + m) * 24;
            for (int q = 0; q < 24; ++q) jkeys[jt + q] = T.jsentinel;
        }
    }
}

// target[key] += the values of each run of equal sorted keys, in record order (one thread
// a run, from its head).
__global__ void run_sums(const uint32_t *__restrict__ K, const uint32_t *__restrict__ I,
                         const double *__restrict__ vals, const i64 *__restrict__ count,
                         i64 n_host, double *__restrict__ target) {
    const i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n = count ? *count : n_host;
    if (r >= n) return;
    const uint32_t key = K[r];
    if (r > 0 && K[r - 1] == key) return;
    double s = target[key];
    for (i64 q = r; q < n && K[q] == key; ++q) s += vals[I[q]];
    target[key] = s;
}

// cells[key] = the sum of each run of equal sorted keys' records, in record order (one
// thread a run, from its head); the cells of no record hold zeros.
__global__ void cell_runs(const uint32_t *__restrict__ K, const uint32_t *__restrict__ I,
                          const CellRec *__restrict__ recs, const i64 *__restrict__ count,
                          CellRec *__restrict__ cells) {
    const i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n = *count;
    if (r >= n) return;
    const uint32_t key = K[r];
    if (r > 0 && K[r - 1] == key) return;
    CellRec sum = recs[I[r]];
    for (i64 q = r + 1; q < n && K[q] == key; ++q) {
        const CellRec add = recs[I[q]];
#pragma unroll
        for (int c = 0; c < 8; ++c) sum.c[c] = sum.c[c] + add.c[c];
    }
    cells[key] = sum;
}

// charge[node] += its shares of the eight cells it is a corner of, in a fixed order (the
// corner q = 4 di + 2 dj + dk of the cell at node - (di, dj, dk)), within its patch.
__global__ void node_gather3(const CellRec *__restrict__ cells, const i64 *__restrict__ patch_int,
                             int n_patches, i64 n_nodes, double *__restrict__ charge) {
    const i64 node = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= n_nodes) return;
    int p = 0;
    while (p < n_patches - 1 &&
           !(node >= patch_int[p * 8 + 7] && node < patch_int[p * 8 + 7] + patch_int[p * 8 + 6]))
        ++p;
    const i64 *pi = patch_int + p * 8;
    const i64 pnx = pi[0], pny = pi[1], pnz = pi[2], local = node - pi[7];
    if (local < 0 || local >= pnx * pny * pnz) return;
    const i64 i = local / (pny * pnz), j = (local / pnz) % pny, k = local % pnz;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int di = q >> 2, dj = (q >> 1) & 1, dk = q & 1;
        const i64 ci = i - di, cj = j - dj, ck = k - dk;
        if (ci < 0 || cj < 0 || ck < 0 || ci > pnx - 2 || cj > pny - 2 || ck > pnz - 2) continue;
        s = s + cells[node - di * pny * pnz - dj * pnz - dk].c[q];
    }
    charge[node] += s;
}

__global__ void fill_flags(uint8_t *__restrict__ flags, i64 n, uint8_t value) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) flags[t] = value;
}

}  // namespace
}  // namespace bt

namespace bt {
namespace {

int key_bits(uint64_t max_key) {
    int b = 0;
    while (b < 32 && (max_key >> b) != 0) ++b;
    return b;
}

// Sort a window's records by node and add each node's run, in record order, to target.
void deposit_runs(bt_ctx *ctx, const uint32_t *keys, const double *vals, i64 n, uint32_t sentinel,
                  double *target) {
    uint32_t *sk = nullptr, *sv = nullptr;
    const i64 *count = nullptr;
    radix_sort_pairs(ctx, keys, n, nullptr, key_bits(sentinel), sentinel, &sk, &sv, &count);
    BT_LAUNCH(ctx, run_sums, blocks_for(n, 256), 256, 0, ctx->stream, sk, sv, vals, count, n,
              target);
    BT_CHECK_LAUNCH();
}

void trace3d_all(bt_ctx *ctx, const bt_trace3d_args *args, int64_t window) {
    BT_REQUIRE(ctx && args, "trace3d: null argument");
    const bt_trace3d_args &a = *args;
    BT_REQUIRE(a.n_patches >= 1 && a.patch_int && a.patch_real, "trace3d: no patches");
    BT_REQUIRE(a.n_active >= 0 && a.n >= 0, "trace3d: negative sizes");
    BT_REQUIRE(a.capacity >= 0 && a.path_capacity >= 0 && a.n_planes >= 0,
               "trace3d: negative buffer sizes");
    BT_REQUIRE(a.refine >= 1, "trace3d: refine must be positive");
    BT_REQUIRE(a.h > 0.0, "trace3d: h must be positive");
    BT_REQUIRE(a.integrator == 0 || a.integrator == 1, "trace3d: integrator must be 0 or 1");
    BT_REQUIRE(!a.has_b || a.bn, "trace3d: has_b needs bn");
    BT_REQUIRE(!a.has_j || a.current, "trace3d: has_j needs current");
    BT_REQUIRE(a.charge, "trace3d: null charge");
    BT_REQUIRE(a.n_nodes >= 8 && a.n_nodes < (int64_t)0xffffffffLL,
               "trace3d: the charge rows need 8 to 2^32 - 2 nodes");
    if (a.n_active == 0) return;
    Trace3 T;
    T.a = a;
    // the patches' shapes: every deposit key must fall inside the charge rows
    std::vector<int64_t> rows((size_t)8 * a.n_patches);
    BT_CUDA(cudaMemcpyAsync(rows.data(), a.patch_int, sizeof(int64_t) * rows.size(),
                            cudaMemcpyDeviceToHost, ctx->stream));
    BT_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int64_t p = 0; p < a.n_patches; ++p) {
        const int64_t *r = rows.data() + 8 * p;
        BT_REQUIRE(r[0] >= 2 && r[1] >= 2 && r[2] >= 2, "trace3d: a patch needs 2 x 2 x 2 nodes");
        BT_REQUIRE(r[3] >= 0 && r[4] >= 0 && r[5] >= 0 && r[7] >= 0 &&
                       r[7] + r[0] * r[1] * r[2] <= a.n_nodes,
                   "trace3d: a patch's nodes must lie inside the charge rows");
    }
    const int64_t *base = rows.data() + 8 * (a.n_patches - 1);
    T.nx = base[0];
    T.ny = base[1];
    T.nz = base[2];
    BT_REQUIRE(T.nx >= 2 && T.ny >= 2 && T.nz >= 2, "trace3d: the mesh needs 2 x 2 x 2 nodes");
    const i64 nb = T.nx * T.ny * T.nz;
    BT_REQUIRE(!a.has_j || 3 * nb < (int64_t)0xffffffffLL, "trace3d: too many current nodes");
    T.S = window > 0 ? (int)window : 32;
    T.sentinel = (uint32_t)a.n_nodes;
    T.jsentinel = (uint32_t)(3 * nb);
    const i64 na = a.n_active;
    const i64 slots = (i64)T.S * na, jslots = a.has_j ? (i64)T.S * na * 24 : 0;
    BT_REQUIRE(slots < (i64)0xffffffffLL && jslots < (i64)0xffffffffLL,
               "trace3d: too many records a window (use a shorter window)");
    uint32_t *keys = ctx->t3_keys.as<uint32_t>(slots);
    CellRec *recs = ctx->t3_vals.as<CellRec>(slots);
    CellRec *cells = ctx->t3_cells.as<CellRec>(a.n_nodes);
    uint32_t *jkeys = a.has_j ? ctx->t3_jkeys.as<uint32_t>(jslots) : nullptr;
    double *jvals = a.has_j ? ctx->t3_jvals.as<double>(jslots) : nullptr;
    uint8_t *alive = ctx->t3_alive.as<uint8_t>(na);
    auto *live = ctx->t3_live.as<unsigned long long>(1);
    unsigned long long *host = static_cast<unsigned long long *>(ctx->host.get(64));
    cudaStream_t st = ctx->stream;
    BT_LAUNCH(ctx, fill_flags, blocks_for(na, 256), 256, 0, st, alive, na, (uint8_t)1);
    // every trajectory ends by max_steps: at most that many windows (and one more)
    const i64 max_windows = a.max_steps / T.S + 2;
    for (i64 w = 0; w < max_windows; ++w) {
        BT_CUDA(cudaMemsetAsync(live, 0, sizeof(unsigned long long), st));
        {
            Timed timed(ctx, "trace3d_window");
            BT_LAUNCH(ctx, trace3d_window, blocks_for(na, 128), 128, 0, st, T, alive, keys, recs,
                      jkeys, jvals, live);
        }
        BT_CHECK_LAUNCH();
        {
            // the window's cell records: sorted by cell, summed per cell, gathered per node
            uint32_t *sk = nullptr, *sv = nullptr;
            const i64 *count = nullptr;
            radix_sort_pairs(ctx, keys, slots, nullptr, key_bits(T.sentinel), T.sentinel, &sk, &sv,
                             &count);
            BT_CUDA(cudaMemsetAsync(cells, 0, sizeof(CellRec) * a.n_nodes, st));
            BT_LAUNCH(ctx, cell_runs, blocks_for(slots, 256), 256, 0, st, sk, sv, recs, count, cells);
            BT_LAUNCH(ctx, node_gather3, blocks_for(a.n_nodes, 256), 256, 0, st, cells, a.patch_int,
                      (int)a.n_patches, a.n_nodes, a.charge);
            BT_CHECK_LAUNCH();
        }
        if (a.has_j) deposit_runs(ctx, jkeys, jvals, jslots, T.jsentinel, a.current);
        BT_CUDA(cudaMemcpyAsync(host, live, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        BT_CUDA(cudaStreamSynchronize(st));
        if (*host == 0) return;
    }
    BT_REQUIRE(false, "trace3d: trajectories still live after max_steps steps");
}

}  // namespace
}  // namespace bt

extern "C" int bt_trace_trajectories_3d(bt_ctx *ctx, const bt_trace3d_args *args,
                                        int64_t window) {
    return bt::guarded([&] { bt::trace3d_all(ctx, args, window); });
}
