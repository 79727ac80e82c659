// The field solve on the B200: the finite-volume operator of the reference's field
// (patchwork's NodalPoisson as solver/poisson.py:1-24, 491-534 documents it), solved by
// GMRES preconditioned with a geometric multigrid V-cycle, and Newton's method for the
// Boltzmann plasma species (poisson.py:860-933).
//
// The operator, per free node, A phi = rho / eps0 + c (A = -laplacian, FD-scaled rows):
// Shortley-Weller rows with the bracketed surface distances at nodes with four cells, the
// cut edge's two-point flux at nodes on a face, (1 -/+ 1/2j) radial weights and 4 (phi_1 -
// phi_0) on the axis, mirror images on Neumann faces; fixed nodes keep their values.
//
// Multigrid: vertex-centred coarsening (coarse node I at fine node 2I, the last coarse
// node on the last fine node), bilinear prolongation P that is zero at fixed fine nodes,
// Galerkin coarse operators A_1 = P^T W A_0 P (W the control volumes, which make W A_0
// nearly symmetric) and A_{l+1} = P^T A_l P: 9-point stencils on every coarse level, built
// on the device (and rebuilt for every Newton step's Jacobian).  Smoothing: red-black
// Gauss-Seidel on the 5-point fine level, four-colour Gauss-Seidel on the 9-point levels;
// the coarsest level (at most 64 nodes) is inverted by Gauss-Jordan in shared memory.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace bt {
namespace {

constexpr int kCoarsest = 256;  // the coarsest level is inverted densely (at most this size)
constexpr double kEps0 = 8.8541878188e-12;  // scipy.constants.epsilon_0 (CODATA 2022)

struct Axis {
    i64 n = 0, nc = 0;
    bool coarsened = false;
    Buffer lo, w, cidx;  // per fine node: coarse index and its weight; per coarse: fine index
    Buffer r0, rw;       // per coarse node: its first fine node and kRestrict weights from there
};

constexpr int kRestrict = 4;  // fine nodes per axis that one coarse node restricts from

struct Level {
    i64 nx = 0, ny = 0, n = 0;
    Buffer c4;      // level 0: cw, ce, cs, cn (4 n)
    Buffer diag;    // level 0: the diagonal (with the reaction)
    Buffer base;    // level 0: the diagonal without the reaction
    Buffer weight;  // level 0: the control volumes W
    Buffer a9;      // coarse levels: 9 coefficients per node, (dI + 1) * 3 + (dJ + 1)
    Buffer active;  // uint8: free (level 0) or a nonzero row (coarse)
    Buffer x, b, r;
    Buffer x2;              // the second x of staged smoothing (it writes the other buffer)
    double *cur = nullptr;  // which of x, x2 holds the level's x while a V-cycle is recorded
    Axis ax, ay;            // the map to the next coarser level
};

__device__ __forceinline__ double pw(const int32_t *lo, const double *w, i64 k, i64 I) {
    const i64 l = lo[k];
    if (l == I) return w[k];
    if (l + 1 == I) return 1.0 - w[k];
    return 0.0;
}

// -- the fine operator (mirrors oracle/poisson.py:coefficients) ---------------------------

__global__ void build_fine(i64 nx, i64 ny, const double *__restrict__ x, double h, int cyl,
                           i64 j0, const uint8_t *__restrict__ fixed, const double *__restrict__ dist,
                           double g0, double g1, double g2, double g3,
                           double *__restrict__ c4, double *__restrict__ base,
                           double *__restrict__ src, double *__restrict__ weight,
                           uint8_t *__restrict__ active) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n = nx * ny;
    if (t >= n) return;
    const i64 i = t / ny, j = t - i * ny;
    const double h_lo = i > 0 ? x[i] - x[i - 1] : 0.0;
    const double h_hi = i < nx - 1 ? x[i + 1] - x[i] : 0.0;
    const double ax = dist[t], bx = dist[n + t], ay = dist[2 * n + t], by = dist[3 * n + t];
    const bool four = i > 0 && i < nx - 1 && j > 0 && j < ny - 1;
    double cw = 0.0, ce = 0.0, cs = 0.0, cn = 0.0, s = 0.0;
    // x
    if (i > 0 && i < nx - 1) {
        const double dm = ax * h_lo, dp = bx * h_hi;
        if (four) {
            cw = 2.0 / ((dm + dp) * dm);
            ce = 2.0 / ((dm + dp) * dp);
        } else {
            const double L = 0.5 * (h_lo + h_hi);
            cw = 1.0 / (L * dm);
            ce = 1.0 / (L * dp);
        }
    } else if (i == 0) {
        ce = 2.0 / (h_hi * (bx * h_hi));
        s += 2.0 * g0 / h_hi;
    } else {
        cw = 2.0 / (h_lo * (ax * h_lo));
        s += 2.0 * g1 / h_lo;
    }
    // y
    const bool mid = j > 0 && j < ny - 1;
    if (!cyl) {
        const double dm = ay * h, dp = by * h;
        if (mid) {
            if (four) {
                cs = 2.0 / ((dm + dp) * dm);
                cn = 2.0 / ((dm + dp) * dp);
            } else {
                cs = 1.0 / (h * dm);
                cn = 1.0 / (h * dp);
            }
        } else if (j == 0) {
            cn = 2.0 / (h * dp);
            s += 2.0 * g2 / h;
        } else {
            cs = 2.0 / (h * dm);
            s += 2.0 * g3 / h;
        }
    } else {
        // the radial index of the row: j0 = r_0 / h for a refined patch off the axis
        const double jj = j + j0 > 1 ? (double)(j + j0) : 1.0;
        const double h2 = h * h;
        if (mid) {
            if (four) {
                cs = (2.0 / ay - 1.0 / jj) / ((ay + by) * h2);
                cn = (2.0 / by + 1.0 / jj) / ((ay + by) * h2);
            } else {
                cs = (1.0 - 0.5 / jj) / (ay * h2);
                cn = (1.0 + 0.5 / jj) / (by * h2);
            }
        } else if (j == 0) {
            // the axis; off the axis (a patch's side inside the domain, a row the
            // composite operator does not use) a face row
            cn = (j0 == 0 ? 4.0 : 2.0) / (by * h2);
        } else {
            cs = 2.0 / (ay * h2);
            s += (1.0 + 0.5 / jj) * 2.0 * g3 / h;
        }
    }
    const bool free = fixed[t] == 0;
    c4[t] = free ? cw : 0.0;
    c4[n + t] = free ? ce : 0.0;
    c4[2 * n + t] = free ? cs : 0.0;
    c4[3 * n + t] = free ? cn : 0.0;
    base[t] = free ? cw + ce + cs + cn : 1.0;
    src[t] = free ? s : 0.0;
    active[t] = free ? 1 : 0;
    // the control volume (divided by 2 pi in cylindrical geometry)
    const double lx = 0.5 * (h_lo + h_hi);  // half an edge at an x face
    double ly = (j > 0 && j < ny - 1) ? h : 0.5 * h;
    if (cyl) ly = j + j0 == 0 ? 0.125 * h * h : (double)(j + j0) * h * ly;
    weight[t] = lx * ly;
}

// The transposed operator, scaled by the control volumes: B = W^-1 A^T W, whose
// neighbour coefficients are B[t][nb] = A[nb][t] W_nb / W_t (A[nb][t] the coefficient of
// the neighbour's row pointing back at t; zero for a held node's row or a held neighbour,
// whose rows hold none); the diagonal stays.  W A is symmetric away from the cut rows next
// to electrodes and the faces, so B equals A there and the multigrid built for A serves
// it: A^T z = g is solved as B y = W^-1 g, z = W y.
__global__ void transpose_c4(i64 nx, i64 ny, const double *__restrict__ c4,
                             const double *__restrict__ weight,
                             const uint8_t *__restrict__ active, double *__restrict__ c4t) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n = nx * ny;
    if (t >= n) return;
    const i64 i = t / ny, j = t - i * ny;
    const bool free = active[t] != 0;
    const double wt = weight[t];
    c4t[t] = free && i > 0 ? c4[n + (t - ny)] * weight[t - ny] / wt : 0.0;  // west's east
    c4t[n + t] = free && i < nx - 1 ? c4[t + ny] * weight[t + ny] / wt : 0.0;  // east's west
    c4t[2 * n + t] = free && j > 0 ? c4[3 * n + (t - 1)] * weight[t - 1] / wt : 0.0;
    c4t[3 * n + t] = free && j < ny - 1 ? c4[2 * n + (t + 1)] * weight[t + 1] / wt : 0.0;
}

// v <- v / W (divide) or v * W on the free nodes: to and from the scaled transposed system.
__global__ void scale_by_weight(i64 n, const double *__restrict__ weight,
                                const uint8_t *__restrict__ active, int divide,
                                double *__restrict__ v) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !active[t]) return;
    v[t] = divide ? v[t] / weight[t] : v[t] * weight[t];
}

// The sensitivity to the held potentials of a quantity whose sensitivity to phi is
// phi_bar, given z = A_ff^-T phi_bar (free nodes): the free rows read the held neighbours'
// potentials through their coefficients, so out_d = phi_bar_d + sum over the free
// neighbours i of c(i -> d) z_i; 0 on free nodes.
__global__ void fixed_adjoint(i64 nx, i64 ny, const double *__restrict__ c4,
                              const uint8_t *__restrict__ active, const double *__restrict__ z,
                              const double *__restrict__ phi_bar, double *__restrict__ out) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 n = nx * ny;
    if (t >= n) return;
    if (active[t]) {
        out[t] = 0.0;
        return;
    }
    const i64 i = t / ny, j = t - i * ny;
    double s = phi_bar[t];
    if (i < nx - 1 && active[t + ny]) s += c4[t + ny] * z[t + ny];              // east's west
    if (i > 0 && active[t - ny]) s += c4[n + (t - ny)] * z[t - ny];             // west's east
    if (j < ny - 1 && active[t + 1]) s += c4[2 * n + (t + 1)] * z[t + 1];       // north's south
    if (j > 0 && active[t - 1]) s += c4[3 * n + (t - 1)] * z[t - 1];            // south's north
    out[t] = s;
}

__global__ void add_diag(i64 n, const double *__restrict__ base, const double *__restrict__ reaction,
                         const uint8_t *__restrict__ active, double *__restrict__ diag) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    diag[t] = base[t] + ((reaction && active[t]) ? reaction[t] : 0.0);
}

// -- Galerkin coarse operator -----------------------------------------------------------

struct Fine {
    i64 nx, ny;
    const double *c4, *diag, *a9, *weight;  // c4/diag for the 5-point level, a9 otherwise
    const uint8_t *active;
    const int32_t *lox, *loy;
    const double *wx, *wy;
    const int32_t *cix, *ciy;  // fine index of each coarse node
    const int32_t *rx0, *ry0;  // restriction: first fine node of each coarse node
    const double *rxw, *ryw;   //   and kRestrict weights from it (zero: not a neighbour)
    i64 ncx, ncy;
};

__device__ __forceinline__ double fine_coef(const Fine &F, i64 f, int di, int dj) {
    if (F.a9) return F.a9[(i64)((di + 1) * 3 + (dj + 1)) * (F.nx * F.ny) + f];
    const i64 n = F.nx * F.ny;
    if (di == 0 && dj == 0) return F.diag[f];
    if (di == -1 && dj == 0) return -F.c4[f];
    if (di == 1 && dj == 0) return -F.c4[n + f];
    if (di == 0 && dj == -1) return -F.c4[2 * n + f];
    if (di == 0 && dj == 1) return -F.c4[3 * n + f];
    return 0.0;
}

__global__ void galerkin(Fine F, double *__restrict__ a9c, uint8_t *__restrict__ active_c) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 nc = F.ncx * F.ncy;
    if (t >= nc) return;
    const i64 I = t / F.ncy, J = t - I * F.ncy;
    double acc[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[q] = 0.0;
    const i64 k0 = I > 0 ? F.cix[I - 1] : 0, k1 = I < F.ncx - 1 ? F.cix[I + 1] : F.nx - 1;
    const i64 l0 = J > 0 ? F.ciy[J - 1] : 0, l1 = J < F.ncy - 1 ? F.ciy[J + 1] : F.ny - 1;
    const int span = F.a9 ? 1 : 0;  // the 9-point fine stencil reaches diagonals
    for (i64 k = k0; k <= k1; ++k) {
        const double pk = pw(F.lox, F.wx, k, I);
        if (pk == 0.0) continue;
        for (i64 l = l0; l <= l1; ++l) {
            const double pl = pw(F.loy, F.wy, l, J);
            if (pl == 0.0) continue;
            const i64 f = k * F.ny + l;
            if (!F.active[f]) continue;
            const double wgt = pk * pl * (F.weight ? F.weight[f] : 1.0);
            for (int di = -1; di <= 1; ++di) {
                const i64 k2 = k + di;
                if (k2 < 0 || k2 >= F.nx) continue;
                for (int dj = -1; dj <= 1; ++dj) {
                    if (!span && di != 0 && dj != 0) continue;
                    const i64 l2 = l + dj;
                    if (l2 < 0 || l2 >= F.ny) continue;
                    const i64 f2 = k2 * F.ny + l2;
                    if (!F.active[f2]) continue;
                    const double a = fine_coef(F, f, di, dj);
                    if (a == 0.0) continue;
                    const i64 ix = F.lox[k2], iy = F.loy[l2];
                    const double wx = F.wx[k2], wy = F.wy[l2];
                    for (int sx = 0; sx < 2; ++sx) {
                        const double px = sx ? 1.0 - wx : wx;
                        const i64 I2 = ix + sx;
                        if (px == 0.0 || I2 - I < -1 || I2 - I > 1) continue;
                        for (int sy = 0; sy < 2; ++sy) {
                            const double py = sy ? 1.0 - wy : wy;
                            const i64 J2 = iy + sy;
                            if (py == 0.0 || J2 - J < -1 || J2 - J > 1) continue;
                            acc[(I2 - I + 1) * 3 + (J2 - J + 1)] += wgt * a * px * py;
                        }
                    }
                }
            }
        }
    }
    const bool on = acc[4] != 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) a9c[(i64)q * nc + t] = on ? acc[q] : (q == 4 ? 1.0 : 0.0);
    active_c[t] = on ? 1 : 0;
}

// -- smoothing, residual, transfer ---------------------------------------------------------

__global__ void smooth5(i64 nx, i64 ny, const double *__restrict__ c4,
                        const double *__restrict__ diag, const uint8_t *__restrict__ active,
                        const double *__restrict__ b, double *__restrict__ x, int colour) {
    const i64 n = nx * ny;
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    // thread t handles the t-th node of the colour
    const i64 half = (ny + 1) / 2;
    const i64 i = t / half;
    if (i >= nx) return;
    const i64 j = 2 * (t - i * half) + ((i + colour) & 1);
    if (j >= ny) return;
    const i64 f = i * ny + j;
    if (!active[f]) return;
    double s = b[f];
    if (i > 0) s += c4[f] * x[f - ny];
    if (i < nx - 1) s += c4[n + f] * x[f + ny];
    if (j > 0) s += c4[2 * n + f] * x[f - 1];
    if (j < ny - 1) s += c4[3 * n + f] * x[f + 1];
    x[f] = s / diag[f];
}

// How the item functions load the vectors they read (plain loads; a kernel whose blocks
// shared vectors through global memory within one launch would bypass L1 here).
struct PlainLoad {
    __device__ __forceinline__ double operator()(const double *p) const { return *p; }
};

// The nodes of one of four colours (i % 2, j % 2) of a 9-point level: item t of `count`.
__host__ __device__ __forceinline__ i64 colour_count(i64 nx, i64 ny, int colour) {
    const int ci = colour >> 1, cj = colour & 1;
    return ((nx - ci + 1) / 2) * ((ny - cj + 1) / 2);
}

template <class Load>
__device__ __forceinline__ void smooth9_item(i64 t, i64 nx, i64 ny, const double *__restrict__ a9,
                                             const uint8_t *__restrict__ active,
                                             const double *__restrict__ b, double *x, int colour,
                                             Load load) {
    const i64 n = nx * ny;
    const int ci = colour >> 1, cj = colour & 1;
    const i64 hy = (ny - cj + 1) / 2;
    const i64 i = 2 * (t / hy) + ci, j = 2 * (t % hy) + cj;
    const i64 f = i * ny + j;
    if (!active[f]) return;
    double s = load(b + f);
#pragma unroll
    for (int di = -1; di <= 1; ++di) {
#pragma unroll
        for (int dj = -1; dj <= 1; ++dj) {
            if (di == 0 && dj == 0) continue;
            const i64 i2 = i + di, j2 = j + dj;
            if (i2 < 0 || i2 >= nx || j2 < 0 || j2 >= ny) continue;
            s -= a9[(i64)((di + 1) * 3 + (dj + 1)) * n + f] * load(x + i2 * ny + j2);
        }
    }
    x[f] = s / a9[4 * n + f];
}

__global__ void smooth9(i64 nx, i64 ny, const double *__restrict__ a9,
                        const uint8_t *__restrict__ active, const double *__restrict__ b,
                        double *__restrict__ x, int colour) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= colour_count(nx, ny, colour)) return;
    smooth9_item(t, nx, ny, a9, active, b, x, colour, PlainLoad{});
}

// -- smoothing staged through shared memory -------------------------------------------------
//
// One launch runs up to kMaxPhases colour phases of Gauss-Seidel on a tile of interior
// nodes plus a halo as wide as the phases (phase k is exact on the halo's rings k + 1 and
// inward, so after the last phase the interior is exactly what per-colour launches give).
// The tile's coefficients, right-hand side, active flags and x are read from global memory
// once, each phase then runs from shared memory, and the interior is written to a second x
// buffer: no block reads what another block of the same launch writes.  Coefficients and b
// are stored compacted by colour, so the threads of a phase read consecutive words; x keeps
// the tile's natural layout.
constexpr int kMaxPhases = 8;
constexpr int kStageThreads = 512;
constexpr int kStage5X = 32, kStage5Y = 32;  // 5-point level: interior rows x columns
constexpr int kStage9X = 16, kStage9Y = 32;  // 9-point levels

struct Phases {
    int count;
    int colour[kMaxPhases];
};

// The halo of `count` phases: rounded up to even, so the tile's origin has even (i, j)
// and a node's colour follows from its place in the tile.
__host__ __device__ inline int stage_halo(int count) { return (count + 1) & ~1; }

// (P xc)[f], the prolongation of the coarse correction xc to the fine node f of an active
// fine node (the bilinear weights of the fine node's coarse neighbours, in (sx, sy) order).
template <class Load>
__device__ __forceinline__ double prolong_sum(const Fine &F, i64 f, const double *xc, Load load) {
    const i64 k = f / F.ny, l = f - k * F.ny;
    const i64 ix = F.lox[k], iy = F.loy[l];
    const double wx = F.wx[k], wy = F.wy[l];
    double s = 0.0;
    for (int sx = 0; sx < 2; ++sx) {
        const double px = sx ? 1.0 - wx : wx;
        if (px == 0.0 || ix + sx >= F.ncx) continue;
        for (int sy = 0; sy < 2; ++sy) {
            const double py = sy ? 1.0 - wy : wy;
            if (py == 0.0 || iy + sy >= F.ncy) continue;
            s += px * py * load(xc + (ix + sx) * F.ncy + iy + sy);
        }
    }
    return s;
}

__host__ __device__ inline size_t stage_smem(bool nine, int tx, int ty, int halo) {
    const size_t m = (size_t)(tx + 2 * halo) * (ty + 2 * halo);
    return m * sizeof(double) * (nine ? 11 : 7) + m;
}

// One tile (bx, by) of the staged smoothing (the body of smooth_staged and of its batched
// form).
template <bool NINE, int R>
__device__ __forceinline__ void smooth_staged_tile(
    i64 nx, i64 ny, const double *__restrict__ c4, const double *__restrict__ diag,
    const double *__restrict__ a9, const uint8_t *__restrict__ active,
    const double *__restrict__ b, const double *__restrict__ xin, double *__restrict__ xout,
    int tx, int ty, const Phases &ph, const Fine &F, const double *__restrict__ xc, i64 bx,
    i64 by, bool zero_in = false) {
    // zero_in: x starts at zero (xin is not read)
    // xc, when not NULL: the coarse correction, prolonged onto x as it is read (the values
    // prolong_add would leave in xin)
    extern __shared__ double sm[];
    constexpr int Q = NINE ? 9 : 5;  // coefficients per node (5-point: w, e, s, n, diagonal)
    constexpr int K = NINE ? 4 : 2;  // colours
    const int halo = stage_halo(ph.count);
    const int wx = tx + 2 * halo, wy = ty + 2 * halo, m = wx * wy, per = m / K, hy = wy / 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    double *coef = sm;          // [Q][m], position slot(a, c)
    double *bs = coef + Q * m;  // [m], position slot(a, c)
    double *xs = bs + m;        // [m], natural a * wy + c
    uint8_t *act = reinterpret_cast<uint8_t *>(xs + m);
    // the compacted position of tile node (a, c): its colour's block, then its index there
    auto slot = [&](int a, int c) -> int {
        if (NINE) return (((a & 1) << 1) | (c & 1)) * per + (a >> 1) * hy + (c >> 1);
        return ((a + c) & 1) * per + ((a * wy + c) >> 1);
    };
    const i64 i0 = bx * tx - halo, j0 = by * ty - halo;
    const i64 n = nx * ny;
    // Every array of a node is loaded at once, whether or not the node is active (the
    // flag selects afterwards): one round trip to memory a node, not two.  An inactive
    // node's coefficients are stored but never read.
#pragma unroll 4
    for (int e = tid; e < m; e += nt) {
        const int a = e / wy, c = e - a * wy;
        const i64 i = i0 + a, j = j0 + c;
        const int pos = slot(a, c);
        double xv = 0.0, bv = 0.0;
        uint8_t av = 0;
        if (i >= 0 && i < nx && j >= 0 && j < ny) {
            const i64 f = i * ny + j;
            xv = zero_in ? 0.0 : xin[f];
            av = active[f];
            const double bf = b[f];
            if (NINE) {
                double q9[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) q9[q] = a9[(i64)q * n + f];
#pragma unroll
                for (int q = 0; q < 9; ++q) coef[q * m + pos] = q9[q];
            } else {
                double q5[5];
#pragma unroll
                for (int q = 0; q < 4; ++q) q5[q] = c4[(i64)q * n + f];
                q5[4] = diag[f];
#pragma unroll
                for (int q = 0; q < 5; ++q) coef[q * m + pos] = q5[q];
            }
            if (av) {
                if (xc) xv = xv + prolong_sum(F, f, xc, PlainLoad{});
                bv = bf;
            }
        }
        xs[e] = xv;
        bs[pos] = bv;
        act[pos] = av;
    }
    __syncthreads();
    // The nodes this thread updates: node u = tid + r nt of each colour's compacted list,
    // with its place in x's layout and its ring (its distance from the tile's edge; -1 for
    // a node it never updates: past the list, outside the mesh, or held).  A neighbour
    // outside the mesh holds x = 0 in the tile and adds nothing: no bounds tests.
    int xi[K][R], ring[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int u = tid + r * nt;
            int a = 0, c = 0;
            if (NINE) {
                const int ua = u / hy;
                a = 2 * ua + (k >> 1);
                c = 2 * (u - ua * hy) + (k & 1);
            } else {
                a = u / hy;
                c = 2 * (u - a * hy) + ((a + k) & 1);
            }
            const i64 i = i0 + a, j = j0 + c;
            const bool mine = u < per && i >= 0 && i < nx && j >= 0 && j < ny && act[k * per + u];
            xi[k][r] = a * wy + c;
            ring[k][r] = mine ? min(min(a, wx - 1 - a), min(c, wy - 1 - c)) : -1;
        }
    }
    for (int kk = 0; kk < ph.count; ++kk) {
        const int colour = ph.colour[kk];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (k != colour) continue;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (ring[k][r] <= kk) continue;  // phase kk is exact from ring kk + 1 inward
                const int pos = k * per + tid + r * nt, q = xi[k][r];
                double s = bs[pos];
                if (NINE) {
                    s -= coef[pos] * xs[q - wy - 1];
                    s -= coef[m + pos] * xs[q - wy];
                    s -= coef[2 * m + pos] * xs[q - wy + 1];
                    s -= coef[3 * m + pos] * xs[q - 1];
                    s -= coef[5 * m + pos] * xs[q + 1];
                    s -= coef[6 * m + pos] * xs[q + wy - 1];
                    s -= coef[7 * m + pos] * xs[q + wy];
                    s -= coef[8 * m + pos] * xs[q + wy + 1];
                } else {
                    s += coef[pos] * xs[q - wy];
                    s += coef[m + pos] * xs[q + wy];
                    s += coef[2 * m + pos] * xs[q - 1];
                    s += coef[3 * m + pos] * xs[q + 1];
                }
                xs[q] = s / coef[4 * m + pos];
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < tx * ty; e += nt) {
        const int ea = e / ty;
        const int a = halo + ea, c = halo + (e - ea * ty);
        const i64 i = i0 + a, j = j0 + c;
        if (i < nx && j < ny) xout[i * ny + j] = xs[a * wy + c];
    }
}

template <bool NINE, int R>
__global__ void __launch_bounds__(kStageThreads) smooth_staged(
    i64 nx, i64 ny, const double *__restrict__ c4, const double *__restrict__ diag,
    const double *__restrict__ a9, const uint8_t *__restrict__ active,
    const double *__restrict__ b, const double *__restrict__ xin, double *__restrict__ xout,
    int tx, int ty, Phases ph, Fine F, const double *__restrict__ xc) {
    smooth_staged_tile<NINE, R>(nx, ny, c4, diag, a9, active, b, xin, xout, tx, ty, ph, F, xc,
                                blockIdx.x, blockIdx.y);
}

// y = A x (level 0, 5-point) on active rows, 0 elsewhere; with b: r = b - A x.  Node f of
// an (nx, ny) level; returns y[f].
__device__ __forceinline__ double apply5_item(i64 f, i64 nx, i64 ny, const double *__restrict__ c4,
                                              const double *__restrict__ diag,
                                              const uint8_t *__restrict__ active,
                                              const double *__restrict__ x,
                                              const double *__restrict__ b,
                                              double *__restrict__ y) {
    const i64 n = nx * ny;
    if (!active[f]) {
        y[f] = 0.0;
        return 0.0;
    }
    const i64 i = f / ny, j = f - i * ny;
    double s = diag[f] * x[f];
    if (i > 0) s -= c4[f] * x[f - ny];
    if (i < nx - 1) s -= c4[n + f] * x[f + ny];
    if (j > 0) s -= c4[2 * n + f] * x[f - 1];
    if (j < ny - 1) s -= c4[3 * n + f] * x[f + 1];
    const double out = b ? b[f] - s : s;
    y[f] = out;
    return out;
}

__global__ void apply5(i64 nx, i64 ny, const double *__restrict__ c4,
                       const double *__restrict__ diag, const uint8_t *__restrict__ active,
                       const double *__restrict__ x, const double *__restrict__ b,
                       double *__restrict__ y) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nx * ny) return;
    apply5_item(f, nx, ny, c4, diag, active, x, b, y);
}

template <class Load>
__device__ __forceinline__ void residual9_item(i64 f, i64 nx, i64 ny, const double *__restrict__ a9,
                                               const uint8_t *__restrict__ active,
                                               const double *x, const double *b, double *r,
                                               Load load) {
    const i64 n = nx * ny;
    if (!active[f]) {
        r[f] = 0.0;
        return;
    }
    const i64 i = f / ny, j = f - i * ny;
    double s = load(b + f);
    for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj) {
            const i64 i2 = i + di, j2 = j + dj;
            if (i2 < 0 || i2 >= nx || j2 < 0 || j2 >= ny) continue;
            s -= a9[(i64)((di + 1) * 3 + (dj + 1)) * n + f] * load(x + i2 * ny + j2);
        }
    r[f] = s;
}

__global__ void residual9(i64 nx, i64 ny, const double *__restrict__ a9,
                          const uint8_t *__restrict__ active, const double *__restrict__ x,
                          const double *__restrict__ b, double *__restrict__ r) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nx * ny) return;
    residual9_item(f, nx, ny, a9, active, x, b, r, PlainLoad{});
}

// bc[t] = (R r)[t] over the active fine nodes (weighted by the control volumes on level 0),
// xc[t] = 0.  The terms are those of the fine nodes with a nonzero prolongation weight, in
// ascending (k, l) order; the weights and the fine values are independent loads.
template <class Load>
__device__ __forceinline__ void restrict_item(i64 t, const Fine &F, const double *r, double *bc,
                                              double *xc, Load load) {
    const i64 I = t / F.ncy, J = t - I * F.ncy;
    const i64 k0 = F.rx0[I], l0 = F.ry0[J];
    double px[kRestrict], py[kRestrict];
#pragma unroll
    for (int a = 0; a < kRestrict; ++a) {
        px[a] = F.rxw[kRestrict * I + a];
        py[a] = F.ryw[kRestrict * J + a];
    }
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < kRestrict; ++a) {
        if (px[a] == 0.0) continue;
#pragma unroll
        for (int c = 0; c < kRestrict; ++c) {
            if (py[c] == 0.0) continue;
            const i64 f = (k0 + a) * F.ny + l0 + c;
            if (!F.active[f]) continue;
            s += px[a] * py[c] * (F.weight ? F.weight[f] : 1.0) * load(r + f);
        }
    }
    bc[t] = s;
    xc[t] = 0.0;
}

__global__ void restrict_residual(Fine F, const double *__restrict__ r, double *__restrict__ bc,
                                  double *__restrict__ xc) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= F.ncx * F.ncy) return;
    restrict_item(t, F, r, bc, xc, PlainLoad{});
}

template <class Load>
__device__ __forceinline__ void prolong_item(i64 f, const Fine &F, const double *xc, double *x,
                                             Load load) {
    if (!F.active[f]) return;
    x[f] = load(x + f) + prolong_sum(F, f, xc, load);
}

__global__ void prolong_add(Fine F, const double *__restrict__ xc, double *__restrict__ x) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F.nx * F.ny) return;
    prolong_item(f, F, xc, x, PlainLoad{});
}

// The coarsest level: the dense matrix of its 9-point operator, inverted in place in `M`
// (global memory, n x n) by Gauss-Jordan with partial pivoting, one block.  The pivot is the
// largest |M[r][k]| (the first such row).  `status` is set to 1 on a zero pivot (a singular
// operator: no node of the mesh is held).
constexpr int kInvertThreads = 1024;

// The coarsest operator is a 9-point stencil: ordered along its shorter side first its
// matrix is banded with half-bandwidth b = min(nx, ny) + 1 (at most 17 for 256 nodes), and
// its LU factors without pivoting fit shared memory (n rows of 2b + 1).  One block
// factorises it (b^2 updates a step between two barriers), then one thread a column
// solves L U x = e_c into the dense inverse the V-cycle applies.  A pivot smaller than
// 1e-12 of its row (a matrix that needs pivoting, or a singular one) sets *fallback and the
// pivoting Gauss-Jordan below computes the inverse instead.
constexpr int kBandThreads = 512;
constexpr int kBandMax = 17;

__host__ __device__ __forceinline__ int band_half(i64 nx, i64 ny) {
    return (int)(nx < ny ? nx : ny) + 1;
}

__host__ __device__ __forceinline__ size_t band_smem(i64 nx, i64 ny) {
    return sizeof(double) * (size_t)(nx * ny) * (size_t)(2 * band_half(nx, ny) + 1);
}

__global__ void __launch_bounds__(kBandThreads) coarsest_band_invert(
    i64 nx, i64 ny, const double *__restrict__ a9, double *__restrict__ M,
    int *__restrict__ fallback) {
    extern __shared__ double band[];  // row r: band[r * W + (c - r + b)], |c - r| <= b
    const int n = (int)(nx * ny);
    const bool across = nx < ny;  // order x fastest when x is the shorter side
    const int b = band_half(nx, ny), W = 2 * b + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    auto order_of = [&](int node) {
        return across ? (node % (int)ny) * (int)nx + node / (int)ny : node;
    };
    auto node_of = [&](int o) { return across ? (o % (int)nx) * (int)ny + o / (int)nx : o; };
    for (int e = tid; e < n * W; e += nt) band[e] = 0.0;
    __syncthreads();
    for (int node = tid; node < n; node += nt) {
        const int i = node / (int)ny, j = node % (int)ny, r = order_of(node);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj) {
                const int i2 = i + di, j2 = j + dj;
                if (i2 < 0 || i2 >= nx || j2 < 0 || j2 >= ny) continue;
                const int c = order_of(i2 * (int)ny + j2);
                band[r * W + (c - r + b)] = a9[(i64)((di + 1) * 3 + (dj + 1)) * n + node];
            }
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = band[k * W + b];
        if (tid == 0) {
            double row = 0.0;
            for (int q = 0; q < W; ++q) row = fmax(row, fabs(band[k * W + q]));
            if (!(fabs(piv) > 1e-12 * row)) *fallback = 1;
        }
        const int last = min(n - 1, k + b);
        for (int r = k + 1 + tid; r <= last; r += nt) band[r * W + (k - r + b)] /= piv;
        __syncthreads();
        const int m = last - k;  // rows and columns k + 1 .. last
        for (int e = tid; e < m * m; e += nt) {
            const int r = k + 1 + e / m, c = k + 1 + e % m;
            band[r * W + (c - r + b)] -= band[r * W + (k - r + b)] * band[k * W + (c - k + b)];
        }
        __syncthreads();
    }
    if (*fallback) return;
    for (int col = tid; col < n; col += nt) {
        const int oc = order_of(col);
        // L y = e (unit lower, band b), y in M's column col: y_r = 0 for r < oc
        for (int o = 0; o < oc; ++o) M[(i64)node_of(o) * n + col] = 0.0;
        for (int o = oc; o < n; ++o) {
            double y = o == oc ? 1.0 : 0.0;
            for (int q = max(oc, o - b); q < o; ++q)
                y -= band[o * W + (q - o + b)] * M[(i64)node_of(q) * n + col];
            M[(i64)node_of(o) * n + col] = y;
        }
        // U x = y, in place
        for (int o = n - 1; o >= 0; --o) {
            double x = M[(i64)node_of(o) * n + col];
            for (int q = o + 1; q <= min(n - 1, o + b); ++q)
                x -= band[o * W + (q - o + b)] * M[(i64)node_of(q) * n + col];
            M[(i64)node_of(o) * n + col] = x / band[o * W + b];
        }
    }
}

__global__ void __launch_bounds__(kInvertThreads) coarsest_invert(
    i64 nx, i64 ny, const double *__restrict__ a9, double *M, int *__restrict__ status,
    const int *__restrict__ fallback) {
    if (fallback && *fallback == 0) return;  // the banded factorisation made the inverse
    __shared__ int perm[kCoarsest];
    __shared__ double best_v[kInvertThreads / 32];
    __shared__ int best_r[kInvertThreads / 32];
    __shared__ int pivot_row;
    const int n = (int)(nx * ny);
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < n * n; e += nt) {
        const int row = e / n, col = e % n;
        const i64 i = row / ny, j = row % ny, i2 = col / ny, j2 = col % ny;
        const i64 di = i2 - i, dj = j2 - j;
        double v = 0.0;
        if (di >= -1 && di <= 1 && dj >= -1 && dj <= 1)
            v = a9[(i64)((di + 1) * 3 + (dj + 1)) * n + row];
        M[e] = v;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        // the pivot: a block-wide arg-max of |M[r][k]|, r >= k, the lowest r on ties
        double v = -1.0;
        int r = n;
        for (int q = k + tid; q < n; q += nt) {
            const double a = fabs(M[(i64)q * n + k]);
            if (a > v) {
                v = a;
                r = q;
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double v2 = __shfl_down_sync(0xffffffffu, v, off);
            const int r2 = __shfl_down_sync(0xffffffffu, r, off);
            if (v2 > v || (v2 == v && r2 < r)) {
                v = v2;
                r = r2;
            }
        }
        if (lane == 0) {
            best_v[warp] = v;
            best_r[warp] = r;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = best_v[0];
            int br = best_r[0];
            for (int w = 1; w < nt / 32; ++w)
                if (best_v[w] > bv || (best_v[w] == bv && best_r[w] < br)) {
                    bv = best_v[w];
                    br = best_r[w];
                }
            if (br >= n) br = k;
            pivot_row = br;
            perm[k] = br;
            if (!(bv > 0.0)) *status = 1;
        }
        __syncthreads();
        const int p = pivot_row;
        if (p != k)
            for (int c = tid; c < n; c += nt) {
                const double t = M[(i64)k * n + c];
                M[(i64)k * n + c] = M[(i64)p * n + c];
                M[(i64)p * n + c] = t;
            }
        __syncthreads();
        const double piv = M[(i64)k * n + k];
        __syncthreads();
        for (int c = tid; c < n; c += nt) M[(i64)k * n + c] = (c == k ? 1.0 : M[(i64)k * n + c]) / piv;
        __syncthreads();
        for (int e = tid; e < n * n; e += nt) {
            const int rr = e / n, c = e % n;
            if (rr == k || c == k) continue;
            M[e] -= M[(i64)rr * n + k] * M[(i64)k * n + c];
        }
        __syncthreads();
        for (int rr = tid; rr < n; rr += nt)
            if (rr != k) M[(i64)rr * n + k] = -M[(i64)rr * n + k] * M[(i64)k * n + k];
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        const int p = perm[k];
        if (p != k)
            for (int rr = tid; rr < n; rr += nt) {
                const double t = M[(i64)rr * n + k];
                M[(i64)rr * n + k] = M[(i64)rr * n + p];
                M[(i64)rr * n + p] = t;
            }
        __syncthreads();
    }
}

// x = inv b on the active rows, 0 on held ones (the inverse's held rows are unit rows up to
// the rounding that pivoting mixes into them; a correction never moves a held node).
__global__ void coarsest_apply(int n, const double *__restrict__ inv, const uint8_t *__restrict__ active,
                               const double *__restrict__ b, double *__restrict__ x) {
    const int r = threadIdx.x;
    if (r >= n) return;
    double s = 0.0;
    for (int c = 0; c < n; ++c) s += inv[r * n + c] * b[c];
    x[r] = active[r] ? s : 0.0;
}

// The 9-point form of the 5-point level-0 operator, for a mesh whose first level is
// already the coarsest (the dense inverse reads 9-point rows).
__global__ void five_to_nine(i64 n, const double *__restrict__ c4, const double *__restrict__ diag,
                             const uint8_t *__restrict__ active, double *__restrict__ a9) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    for (int q = 0; q < 9; ++q) a9[(i64)q * n + f] = 0.0;
    if (!active[f]) {
        a9[4 * n + f] = 1.0;
        return;
    }
    a9[4 * n + f] = diag[f];
    a9[1 * n + f] = -c4[2 * n + f];  // (0, -1)
    a9[7 * n + f] = -c4[3 * n + f];  // (0, +1)
    a9[3 * n + f] = -c4[f];          // (-1, 0)
    a9[5 * n + f] = -c4[n + f];      // (+1, 0)
}

// -- the small levels in one launch, in shared memory ---------------------------------------

constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 16;
constexpr size_t kTailSmemMax = 200 * 1024;

struct TailLevel {
    i64 nx, ny, n;
    const double *a9;
    const uint8_t *active;
    double *x, *b;  // the level's global vectors (read: b of the first, written: x of the first)
    Fine next;      // the map to the next coarser level (unused on the coarsest)
};

// Where a tail level lives in shared memory.  The block's shared memory is a static image
// -- the levels' coefficients and transfer weights (doubles), transfer indices (int32s) and
// active flags (bytes), copied in one piece from a device buffer kept in step with the
// hierarchy -- then the levels' x (with a ring of zeros), b and r (doubles).  a9, wx, wy,
// rxw, ryw count doubles from the start; lox, loy, rx0, ry0 int32s from the int block; act
// bytes from the byte block; x, b, r doubles from the dynamic block.
struct TailPlan {
    int nx, ny, n, ncx, ncy;
    int x, b, r, a9;         // x: (nx + 2) (ny + 2) with a ring of zeros; b, r: n; a9: 9 n
    int wx, wy, rxw, ryw;    // transfer weights to the next level
    int lox, loy, rx0, ry0;  // transfer indices (ints)
    int act;                 // active flags (bytes)
};

struct TailLayout {
    std::vector<TailPlan> plan;
    int doubles = 0, ints = 0, bytes = 0, dynamic = 0;
    // the static image's bytes, rounded up to whole 16-byte words, and where the dynamic
    // doubles start
    size_t image() const {
        const size_t b = sizeof(double) * (size_t)doubles + sizeof(int32_t) * (size_t)ints + bytes;
        return (b + 15) & ~(size_t)15;
    }
    size_t total() const { return image() + sizeof(double) * (size_t)dynamic; }
};

__device__ __forceinline__ void tail_smooth(const TailPlan &P, const double *sm, double *smd,
                                            const uint8_t *act, int colour, int tid, int nt) {
    const int nx = P.nx, ny = P.ny, n = P.n, W = ny + 2;
    const int ci = colour >> 1, cj = colour & 1;
    const int hx = (nx - ci + 1) >> 1, hy = (ny - cj + 1) >> 1;
    double *x = smd + P.x;
    const double *b = smd + P.b, *a9 = sm + P.a9;
    for (int t = tid; t < hx * hy; t += nt) {
        const int ti = t / hy;
        const int i = 2 * ti + ci, j = 2 * (t - ti * hy) + cj;
        const int f = i * ny + j;
        if (!act[f]) continue;
        const int q = (i + 1) * W + j + 1;
        double s = b[f];
        s -= a9[f] * x[q - W - 1];
        s -= a9[n + f] * x[q - W];
        s -= a9[2 * n + f] * x[q - W + 1];
        s -= a9[3 * n + f] * x[q - 1];
        s -= a9[5 * n + f] * x[q + 1];
        s -= a9[6 * n + f] * x[q + W - 1];
        s -= a9[7 * n + f] * x[q + W];
        s -= a9[8 * n + f] * x[q + W + 1];
        x[q] = s / a9[4 * n + f];
    }
}

__device__ __forceinline__ void tail_residual(const TailPlan &P, const double *sm, double *smd,
                                              const uint8_t *act, int tid, int nt) {
    const int ny = P.ny, n = P.n, W = ny + 2;
    const double *x = smd + P.x, *b = smd + P.b, *a9 = sm + P.a9;
    double *r = smd + P.r;
    for (int f = tid; f < n; f += nt) {
        if (!act[f]) {
            r[f] = 0.0;
            continue;
        }
        const int i = f / ny;
        const int q = f + 2 * i + W + 1;
        double s = b[f];
        s -= a9[f] * x[q - W - 1];
        s -= a9[n + f] * x[q - W];
        s -= a9[2 * n + f] * x[q - W + 1];
        s -= a9[3 * n + f] * x[q - 1];
        s -= a9[4 * n + f] * x[q];
        s -= a9[5 * n + f] * x[q + 1];
        s -= a9[6 * n + f] * x[q + W - 1];
        s -= a9[7 * n + f] * x[q + W];
        s -= a9[8 * n + f] * x[q + W + 1];
        r[f] = s;
    }
}

// b of the next level = R r of this one (the next level's x is zero already).
__device__ __forceinline__ void tail_restrict(const TailPlan &P, const TailPlan &C,
                                              const double *sm, double *smd, const int32_t *smi,
                                              const uint8_t *act, int tid, int nt) {
    const int ny = P.ny, ncy = P.ncy;
    const double *r = smd + P.r, *rxw = sm + P.rxw, *ryw = sm + P.ryw;
    const int32_t *rx0 = smi + P.rx0, *ry0 = smi + P.ry0;
    double *bc = smd + C.b;
    for (int t = tid; t < C.n; t += nt) {
        const int I = t / ncy, J = t - I * ncy;
        const int k0 = rx0[I], l0 = ry0[J];
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < kRestrict; ++a) {
            const double px = rxw[kRestrict * I + a];
            if (px == 0.0) continue;
#pragma unroll
            for (int c = 0; c < kRestrict; ++c) {
                const double py = ryw[kRestrict * J + c];
                if (py == 0.0) continue;
                const int f = (k0 + a) * ny + l0 + c;
                if (!act[f]) continue;
                s += px * py * 1.0 * r[f];
            }
        }
        bc[t] = s;
    }
}

// x of this level += P x of the next level.
__device__ __forceinline__ void tail_prolong(const TailPlan &P, const TailPlan &C,
                                             const double *sm, double *smd, const int32_t *smi,
                                             const uint8_t *act, int tid, int nt) {
    const int ny = P.ny, n = P.n, W = ny + 2, ncx = P.ncx, ncy = P.ncy, Wc = ncy + 2;
    double *x = smd + P.x;
    const double *xc = smd + C.x, *wxs = sm + P.wx, *wys = sm + P.wy;
    const int32_t *lox = smi + P.lox, *loy = smi + P.loy;
    for (int f = tid; f < n; f += nt) {
        if (!act[f]) continue;
        const int k = f / ny, l = f - k * ny;
        const int ix = lox[k], iy = loy[l];
        const double wx = wxs[k], wy = wys[l];
        double s = 0.0;
        for (int sx = 0; sx < 2; ++sx) {
            const double px = sx ? 1.0 - wx : wx;
            if (px == 0.0 || ix + sx >= ncx) continue;
            for (int sy = 0; sy < 2; ++sy) {
                const double py = sy ? 1.0 - wy : wy;
                if (py == 0.0 || iy + sy >= ncy) continue;
                s += px * py * xc[(ix + sx + 1) * Wc + iy + sy + 1];
            }
        }
        const int q = f + 2 * k + W + 1;
        x[q] = x[q] + s;
    }
}

// levels[0] reads b from, and writes x to, global memory; `image` holds the static part
// of the shared memory (image_words 16-byte words); inv is the coarsest level's inverse.
// (The body of vcycle_tail and of its batched form.)
__device__ __forceinline__ void vcycle_tail_run(const TailLevel *__restrict__ levels,
                                                const TailPlan *__restrict__ plans, int count,
                                                const uint4 *__restrict__ image,
                                                int image_words, int doubles, int ints,
                                                const double *__restrict__ inv, int sweeps) {
    extern __shared__ __align__(16) double sm[];
    __shared__ TailPlan plan[kTailMaxLevels];
    int32_t *smi = reinterpret_cast<int32_t *>(sm + doubles);
    uint8_t *smb = reinterpret_cast<uint8_t *>(smi + ints);
    double *smd = sm + 2 * image_words;  // the dynamic doubles follow the image
    const int tid = threadIdx.x, nt = blockDim.x;
    {
        const int *src = reinterpret_cast<const int *>(plans);
        int *dst = reinterpret_cast<int *>(plan);
        const int words = count * (int)(sizeof(TailPlan) / sizeof(int));
        for (int e = tid; e < words; e += nt) dst[e] = src[e];
    }
    // the static image in one piece, x zero, level 0's b
    uint4 *dst = reinterpret_cast<uint4 *>(sm);
#pragma unroll 4
    for (int e = tid; e < image_words; e += nt) dst[e] = image[e];
    for (int l = 0; l < count; ++l) {
        const TailPlan &P = plans[l];
        for (int e = tid; e < (P.nx + 2) * (P.ny + 2); e += nt) smd[P.x + e] = 0.0;
    }
    {
        const TailPlan &P = plans[0];
        const double *b0 = levels[0].b;
        for (int f = tid; f < P.n; f += nt) smd[P.b + f] = b0[f];
    }
    __syncthreads();
    for (int l = 0; l + 1 < count; ++l) {
        const TailPlan &P = plan[l];
        const uint8_t *act = smb + P.act;
        for (int s = 0; s < sweeps; ++s)
            for (int c = 0; c < 4; ++c) {
                tail_smooth(P, sm, smd, act, c, tid, nt);
                __syncthreads();
            }
        tail_residual(P, sm, smd, act, tid, nt);
        __syncthreads();
        tail_restrict(P, plan[l + 1], sm, smd, smi, act, tid, nt);
        __syncthreads();
    }
    {
        // the coarsest level: x = inv b, a warp per row, its lanes over the columns
        const TailPlan &C = plan[count - 1];
        const int n = C.n, W = C.ny + 2, lane = tid & 31;
        const double *b = smd + C.b;
        const uint8_t *act = smb + C.act;
        for (int row = tid >> 5; row < n; row += nt >> 5) {
            double s = 0.0;
            for (int c = lane; c < n; c += 32) s += __ldg(inv + (i64)row * n + c) * b[c];
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if (lane == 0) smd[C.x + row + 2 * (row / C.ny) + W + 1] = act[row] ? s : 0.0;
        }
        __syncthreads();
    }
    for (int l = count - 2; l >= 0; --l) {
        const TailPlan &P = plan[l];
        const uint8_t *act = smb + P.act;
        tail_prolong(P, plan[l + 1], sm, smd, smi, act, tid, nt);
        __syncthreads();
        for (int s = 0; s < sweeps; ++s)
            for (int c = 3; c >= 0; --c) {
                tail_smooth(P, sm, smd, act, c, tid, nt);
                __syncthreads();
            }
    }
    {
        const TailPlan &P = plan[0];
        const int W = P.ny + 2;
        double *x0 = levels[0].x;
        for (int f = tid; f < P.n; f += nt) x0[f] = smd[P.x + f + 2 * (f / P.ny) + W + 1];
    }
}

__global__ void __launch_bounds__(kTailThreads, 1)
vcycle_tail(const TailLevel *__restrict__ levels, const TailPlan *__restrict__ plans, int count,
            const uint4 *__restrict__ image, int image_words, int doubles, int ints,
            const double *__restrict__ inv, int sweeps) {
    vcycle_tail_run(levels, plans, count, image, image_words, doubles, ints, inv, sweeps);
}

// The shared-memory layout of tail levels first .. (the coarsest): the static image
// (coefficients of every level but the coarsest, transfer tables, active flags), then the
// dynamic x, b, r of every level.
TailLayout tail_layout(const std::vector<Level> &levels, int first) {
    TailLayout T;
    const int last = (int)levels.size() - 1;
    for (int l = first; l <= last; ++l) {
        const Level &L = levels[l];
        TailPlan P{};
        P.nx = (int)L.nx;
        P.ny = (int)L.ny;
        P.n = (int)L.n;
        if (l < last) {
            P.ncx = (int)levels[l + 1].nx;
            P.ncy = (int)levels[l + 1].ny;
            P.a9 = T.doubles;
            T.doubles += 9 * P.n;
            P.wx = T.doubles;
            T.doubles += P.nx;
            P.wy = T.doubles;
            T.doubles += P.ny;
            P.rxw = T.doubles;
            T.doubles += kRestrict * P.ncx;
            P.ryw = T.doubles;
            T.doubles += kRestrict * P.ncy;
            P.lox = T.ints;
            T.ints += P.nx;
            P.loy = T.ints;
            T.ints += P.ny;
            P.rx0 = T.ints;
            T.ints += P.ncx;
            P.ry0 = T.ints;
            T.ints += P.ncy;
        }
        P.act = T.bytes;
        T.bytes += P.n;
        P.x = T.dynamic;
        T.dynamic += (P.nx + 2) * (P.ny + 2);
        P.b = T.dynamic;
        T.dynamic += P.n;
        P.r = T.dynamic;
        T.dynamic += P.n;
        T.plan.push_back(P);
    }
    return T;
}

// -- dot products: partial sums per block, the last block adds them in block order --------

constexpr int kDotMax = 32;      // at most this many vectors against one
constexpr int kDotBlocks = 296;  // two per SM
constexpr int kDotThreads = 256;

// What a dot pass does: the sums out[q] = <V_q, w> (kPlain), or first w -= sum_q h[q] V_q
// (classical Gram-Schmidt's orthogonalisation, written back to w) and then the sums
// <V_q, w> (kOrthDots) or <w, w> (kOrthNorm) of the new w, q < m.  Every thread adds its
// grid-stride elements in order, the warps and blocks are added in a fixed order, and the
// block that finishes last (a ticket counter, reset by it) adds the blocks' partials in
// block order: the same bits on every run, in one launch.
enum DotMode { kPlain = 0, kOrthDots = 1, kOrthNorm = 2 };

template <int MQ, int MODE>
__global__ void __launch_bounds__(kDotThreads) dot_pass(
    const double *__restrict__ V, const double *__restrict__ h, double *w, i64 n, int m,
    double *__restrict__ partial, unsigned *__restrict__ ticket, double *__restrict__ out) {
    constexpr int NACC = MODE == kOrthNorm ? 1 : MQ;
    __shared__ double warp_part[kDotThreads / 32][NACC];
    __shared__ bool is_last;
    const int sums = MODE == kOrthNorm ? 1 : m;
    double acc[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) acc[q] = 0.0;
    for (i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (i64)gridDim.x * blockDim.x) {
        double s = w[f];
        if (MODE == kPlain) {
#pragma unroll
            for (int q = 0; q < MQ; ++q)
                if (q < m) acc[q] += V[(i64)q * n + f] * s;
        } else {
            double vq[MQ];
#pragma unroll
            for (int q = 0; q < MQ; ++q)
                if (q < m) {
                    vq[q] = V[(i64)q * n + f];
                    s -= h[q] * vq[q];
                }
            w[f] = s;
            if (MODE == kOrthDots) {
#pragma unroll
                for (int q = 0; q < MQ; ++q)
                    if (q < m) acc[q] += vq[q] * s;
            } else {
                acc[0] += s * s;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NACC; ++q) {
        if (q >= sums) break;
        double v = acc[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) warp_part[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < sums) {
        double v = 0.0;
        for (int wi = 0; wi < kDotThreads / 32; ++wi) v += warp_part[wi][threadIdx.x];
        partial[(i64)blockIdx.x * kDotMax + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // the last block: warp w adds the blocks' partials of q = w, w + 8, ... (lanes stride
    // the blocks, then a fixed tree)
    // the blocks' partials are read together, then added in block order
    constexpr int kPer = (kDotBlocks + 31) / 32;
    const int blocks = (int)gridDim.x;
    for (int q = warp; q < sums; q += kDotThreads / 32) {
        double part[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int b = lane + 32 * k;
            part[k] = b < blocks ? __ldcg(partial + (i64)b * kDotMax + q) : 0.0;
        }
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kPer; ++k)
            if (lane + 32 * k < blocks) v += part[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) out[q] = v;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// -- vector kernels of GMRES and Newton ----------------------------------------------------

// The Arnoldi process of one GMRES restart cycle, on the device: the Hessenberg matrix H
// ((m + 1) x m, row-major), the Givens rotations (cs, sn) and the rotated right-hand side
// g.  `j` counts the steps taken; once `done` (the residual estimate |g[j]| at the
// tolerance, or a breakdown) later steps change nothing, so the host may queue steps past
// the end and the cycle's solution is the same.
struct Arnoldi {
    int j, done;
    double tol;
    double resid[kDotMax + 1];  // |g[j]| after step j
};

__global__ void arnoldi_begin(Arnoldi *__restrict__ a, double *__restrict__ g, int m,
                              double beta, double tol) {
    if (threadIdx.x != 0) return;
    a->j = 0;
    a->done = 0;
    a->tol = tol;
    a->resid[0] = beta;
    g[0] = beta;
    for (int q = 1; q <= m; ++q) g[q] = 0.0;
}

// Step j: the new Hessenberg column from the two Gram-Schmidt passes' coefficients h1, h2
// and the new vector's squared norm, rotated by the earlier rotations; the new rotation and
// g, whose last entry is the residual norm up to its sign.
__global__ void arnoldi_step(Arnoldi *__restrict__ a, double *__restrict__ H,
                             double *__restrict__ cs, double *__restrict__ sn,
                             double *__restrict__ g, const double *__restrict__ h1,
                             const double *__restrict__ h2, const double *__restrict__ norm2,
                             int j, int m) {
    // the warp reads the column's coefficients and the rotations together; one thread then
    // rotates the column in shared memory and writes it out
    __shared__ double col[kDotMax + 2], c[kDotMax], sv[kDotMax];
    __shared__ int skip;
    const int t = threadIdx.x;
    if (t == 0) skip = a->done || a->j != j;
    __syncthreads();
    if (skip) return;
    for (int q = t; q <= j; q += blockDim.x) col[q] = h1[q] + h2[q];
    for (int q = t; q < j; q += blockDim.x) {
        c[q] = cs[q];
        sv[q] = sn[q];
    }
    __syncthreads();
    if (t != 0) return;
    const double hn = sqrt(norm2[0]);
    col[j + 1] = hn;
    for (int q = 0; q < j; ++q) {
        const double x = col[q], y = col[q + 1];
        col[q] = c[q] * x + sv[q] * y;
        col[q + 1] = -sv[q] * x + c[q] * y;
    }
    const double x = col[j], y = col[j + 1];
    const double rr = hypot(x, y);
    const double cj = rr > 0.0 ? x / rr : 1.0;
    const double sj = rr > 0.0 ? y / rr : 0.0;
    col[j] = rr;
    col[j + 1] = 0.0;
    for (int q = 0; q <= j + 1; ++q) H[q * m + j] = col[q];
    cs[j] = cj;
    sn[j] = sj;
    const double gj = g[j];
    g[j + 1] = -sj * gj;
    g[j] = cj * gj;
    a->j = j + 1;
    a->resid[j + 1] = fabs(g[j + 1]);
    if (fabs(g[j + 1]) <= a->tol || hn == 0.0) a->done = 1;
}

// y = H^-1 g on the leading j x j upper triangle (j the steps taken)
__global__ void arnoldi_solve(const Arnoldi *__restrict__ a, const double *__restrict__ H,
                              const double *__restrict__ g, double *__restrict__ y, int m) {
    if (threadIdx.x != 0) return;
    const int j = a->j;
    for (int q = j - 1; q >= 0; --q) {
        double s = g[q];
        for (int c = q + 1; c < j; ++c) s -= H[q * m + c] * y[c];
        y[q] = s / H[q * m + q];
    }
}

// v = w / sqrt(norm2[0]) (zero for a zero norm: GMRES stops there)
__global__ void scale_by_norm(const double *__restrict__ w, const double *__restrict__ norm2, i64 n,
                              double *__restrict__ v) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    const double s = norm2[0];
    v[f] = s > 0.0 ? w[f] / sqrt(s) : 0.0;
}

__global__ void scale_into(const double *__restrict__ w, double a, i64 n, double *__restrict__ v) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < n) v[f] = a * w[f];
}

// x += sum_q y[q] Z[q], q below the cycle's steps
__global__ void combine(const double *__restrict__ Z, const double *__restrict__ y,
                        const Arnoldi *__restrict__ a, i64 n, double *__restrict__ x) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    const int m = a->j;
    double s = x[f];
    for (int q = 0; q < m; ++q) s += y[q] * Z[(i64)q * n + f];
    x[f] = s;
}

// the larger of two values, NaN if either is (a NaN update must not read as converged)
__device__ __forceinline__ double max_nan(double m, double v) {
    return (v > m || v != v) ? v : m;
}

// max |v| over the array (one block, deterministic; NaN if any entry is NaN)
__global__ void max_abs(const double *__restrict__ v, i64 n, double *__restrict__ out) {
    __shared__ double part[256];
    double s = 0.0;
    for (i64 f = threadIdx.x; f < n; f += blockDim.x) s = max_nan(s, fabs(v[f]));
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] = max_nan(part[threadIdx.x], part[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

// the right-hand side: rho / eps0 + c on free nodes, 0 on fixed ones; phi's fixed values set
__global__ void prepare(i64 n, const double *__restrict__ rho, const double *__restrict__ src,
                        const uint8_t *__restrict__ active, const double *__restrict__ value,
                        double *__restrict__ b, double *__restrict__ phi) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    if (active[f]) {
        b[f] = (rho ? rho[f] / kEps0 : 0.0) + src[f];
    } else {
        b[f] = 0.0;
        phi[f] = value[f];
    }
}

// The Boltzmann species at phi: e = a exp(min(-s (phi - up) / T, 50)); the Newton
// residual r = b + s e - A phi (the negative of F) and the reaction e / T, on free nodes.
__global__ void boltzmann(i64 nx, i64 ny, const double *__restrict__ c4,
                          const double *__restrict__ base, const uint8_t *__restrict__ active,
                          const double *__restrict__ phi, const double *__restrict__ b,
                          double amplitude, double temperature, double up, double sign,
                          double *__restrict__ r, double *__restrict__ reaction) {
    const i64 n = nx * ny;
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    if (!active[f]) {
        r[f] = 0.0;
        reaction[f] = 0.0;
        return;
    }
    const i64 i = f / ny, j = f - i * ny;
    double s = base[f] * phi[f];
    if (i > 0) s -= c4[f] * phi[f - ny];
    if (i < nx - 1) s -= c4[n + f] * phi[f + ny];
    if (j > 0) s -= c4[2 * n + f] * phi[f - 1];
    if (j < ny - 1) s -= c4[3 * n + f] * phi[f + 1];
    const double e = amplitude * exp(fmin(-sign * (phi[f] - up) / temperature, 50.0));
    r[f] = b[f] + sign * e - s;
    reaction[f] = e / temperature;
}

__global__ void add_into(const double *__restrict__ d, i64 n, double *__restrict__ x) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < n) x[f] += d[f];
}

// w = r - w
__global__ void subtract_from(const double *__restrict__ r, i64 n, double *__restrict__ w) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < n) w[f] = r[f] - w[f];
}

void build_axis(Axis &A, i64 n) {
    A.n = n;
    A.coarsened = n > 3;
    A.nc = A.coarsened ? n / 2 + 1 : n;
    std::vector<int32_t> lo(n), cidx(A.nc);
    std::vector<double> w(n);
    for (i64 I = 0; I < A.nc; ++I) cidx[I] = (int32_t)(A.coarsened ? std::min<i64>(2 * I, n - 1) : I);
    for (i64 k = 0; k < n; ++k) {
        if (!A.coarsened) {
            lo[k] = (int32_t)k;
            w[k] = 1.0;
            continue;
        }
        i64 I = std::min<i64>(k / 2, A.nc - 2);
        const double c0 = cidx[I], c1 = cidx[I + 1];
        lo[k] = (int32_t)I;
        w[k] = (c1 - (double)k) / (c1 - c0);
    }
    // the restriction tables: the prolongation weights read by coarse node
    std::vector<int32_t> r0(A.nc, 0);
    std::vector<double> rw((size_t)kRestrict * A.nc, 0.0);
    for (i64 I = 0; I < A.nc; ++I) {
        i64 first = -1;
        for (i64 k = 0; k < n; ++k) {
            const double p = lo[k] == I ? w[k] : (lo[k] + 1 == I ? 1.0 - w[k] : 0.0);
            if (p == 0.0) continue;
            if (first < 0) first = k;
            BT_REQUIRE(k - first < kRestrict, "poisson: a coarse node restricts from too many nodes");
            rw[(size_t)kRestrict * I + (k - first)] = p;
        }
        r0[I] = (int32_t)std::max<i64>(first, 0);
    }
    cudaMemcpy(A.r0.as<int32_t>(A.nc), r0.data(), A.nc * sizeof(int32_t), cudaMemcpyHostToDevice);
    cudaMemcpy(A.rw.as<double>(kRestrict * A.nc), rw.data(), rw.size() * sizeof(double),
               cudaMemcpyHostToDevice);
    cudaMemcpy(A.lo.as<int32_t>(n), lo.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice);
    cudaMemcpy(A.w.as<double>(n), w.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(A.cidx.as<int32_t>(A.nc), cidx.data(), A.nc * sizeof(int32_t),
               cudaMemcpyHostToDevice);
}

}  // namespace
}  // namespace bt

struct bt_poisson {
    bt_ctx *ctx = nullptr;
    i64 nx = 0, ny = 0, n = 0;
    double h = 0.0;
    int cyl = 0;
    i64 j0 = 0;  // the radial index of the first row (origin_y / h; cylindrical)
    double neumann[4] = {0, 0, 0, 0};
    bt::Buffer x, fixed, value, distance, region;  // mesh; region: the extra held nodes
    bt::Buffer fixed_eff, value_eff, src;
    double region_value = 0.0;
    bool has_region = false;
    std::vector<bt::Level> levels;
    bt::Buffer inv, status;
    bool built = false;        // hierarchy matches the current diagonal
    bool transposed = false;   // the fine operator is A's transpose (bt_poisson_set_transposed)
    bt::Buffer c4_plain;       // A's own coefficients while the operator is transposed
    bool reaction_on = false;  // level-0 diagonal holds a reaction
    int restart = 30;
    // the V-cycle's settings (bt_poisson_set_options)
    int fine_sweeps = 2;    // red-black sweeps on level 0, before and after
    int coarse_sweeps = 2;  // four-colour sweeps on the 9-point levels
    int staged = 1;         // smoothing staged through shared memory (else a launch per colour)
    i64 tail_nodes = 4096;  // levels at most this large may go to the one-block tail
    int tail_start = -1;    // the first level of the V-cycle's one-block tail
    size_t tail_smem = 0;   // its shared memory
    int tail_doubles = 0, tail_ints = 0, tail_words = 0;  // its layout (bt::TailLayout)
    bt::Buffer tail_levels;  // its TailLevel descriptors
    bt::Buffer tail_plans;   // and TailPlan layouts
    bt::Buffer tail_image;   // the static part of its shared memory (tail_words 16-byte words)
    bt::Buffer dot_partial;  // per-block partial dot products
    bt::Buffer dot_ticket;   // the dot passes' finishing-block counter (zero between passes)
    bool ticket_ready = false;
    bt::Buffer arnoldi;      // the device Arnoldi state of GMRES (bt::Arnoldi, H, rotations)
    // the V-cycle from a zero guess on level 0's b into its x, captured once as a graph
    cudaGraph_t vgraph = nullptr;
    cudaGraphExec_t vexec = nullptr;
    i64 vgraph_kernels = 0;
    ~bt_poisson() {
        if (vexec) cudaGraphExecDestroy(vexec);
        if (vgraph) cudaGraphDestroy(vgraph);
    }
    // GMRES: the Krylov basis V, its preconditioned images Z, two work vectors; the solve:
    // its right-hand side, the residual GMRES reduces, the correction, the Newton reaction
    // and scalars.
    bt::Buffer V, Z, work, work2, rhs, r0, delta, reaction, scalars;
};

namespace bt {
namespace {

void refresh_tail_image(bt_poisson *p);

Fine fine_of(Level &L, Level &C, bool first) {
    Fine F{};
    F.nx = L.nx;
    F.ny = L.ny;
    if (first) {
        F.c4 = L.c4.as<double>(4 * L.n);
        F.diag = L.diag.as<double>(L.n);
        F.a9 = nullptr;
        F.weight = L.weight.as<double>(L.n);
    } else {
        F.c4 = nullptr;
        F.diag = nullptr;
        F.a9 = L.a9.as<double>(9 * L.n);
        F.weight = nullptr;
    }
    F.active = L.active.as<uint8_t>(L.n);
    F.lox = L.ax.lo.as<int32_t>(L.nx);
    F.loy = L.ay.lo.as<int32_t>(L.ny);
    F.wx = L.ax.w.as<double>(L.nx);
    F.wy = L.ay.w.as<double>(L.ny);
    F.cix = L.ax.cidx.as<int32_t>(L.ax.nc);
    F.ciy = L.ay.cidx.as<int32_t>(L.ay.nc);
    F.rx0 = L.ax.r0.as<int32_t>(L.ax.nc);
    F.ry0 = L.ay.r0.as<int32_t>(L.ay.nc);
    F.rxw = L.ax.rw.as<double>(kRestrict * L.ax.nc);
    F.ryw = L.ay.rw.as<double>(kRestrict * L.ay.nc);
    F.ncx = C.nx;
    F.ncy = C.ny;
    return F;
}

void build_operator(bt_poisson *p) {
    cudaStream_t st = p->ctx->stream;
    Level &L = p->levels[0];
    const i64 n = p->n;
    BT_LAUNCH(p->ctx, build_fine, blocks_for(n, 256), 256, 0, st, p->nx, p->ny, p->x.as<double>(p->nx), p->h, p->cyl, p->j0, p->fixed_eff.as<uint8_t>(n),
        p->distance.as<double>(4 * n), p->neumann[0], p->neumann[1], p->neumann[2],
        p->neumann[3], L.c4.as<double>(4 * n), L.base.as<double>(n), p->src.as<double>(n),
        L.weight.as<double>(n), L.active.as<uint8_t>(n));
    if (p->transposed) {
        double *plain = p->c4_plain.as<double>(4 * n);
        BT_CUDA(cudaMemcpyAsync(plain, L.c4.as<double>(4 * n), sizeof(double) * 4 * n,
                                cudaMemcpyDeviceToDevice, st));
        BT_LAUNCH(p->ctx, transpose_c4, blocks_for(n, 256), 256, 0, st, p->nx, p->ny, plain,
                  L.weight.as<double>(n), L.active.as<uint8_t>(n), L.c4.as<double>(4 * n));
    }
    BT_CHECK_LAUNCH();
    p->built = false;
    p->reaction_on = true;  // force the diagonal to be set
}

// Set the level-0 diagonal (with `reaction`, or without) and rebuild the coarse levels.
void build_hierarchy(bt_poisson *p, const double *reaction) {
    cudaStream_t st = p->ctx->stream;
    Timed timed(p->ctx, "hierarchy");
    Level &L0 = p->levels[0];
    BT_LAUNCH(p->ctx, add_diag, blocks_for(p->n, 256), 256, 0, st, p->n, L0.base.as<double>(p->n), reaction,
                                                    L0.active.as<uint8_t>(p->n),
                                                    L0.diag.as<double>(p->n));
    for (size_t l = 0; l + 1 < p->levels.size(); ++l) {
        Level &L = p->levels[l], &C = p->levels[l + 1];
        Fine F = fine_of(L, C, l == 0);
        BT_LAUNCH(p->ctx, galerkin, blocks_for(C.n, 128), 128, 0, st, F, C.a9.as<double>(9 * C.n),
                                                        C.active.as<uint8_t>(C.n));
    }
    Level &Lc = p->levels.back();
    if (p->levels.size() == 1)
        BT_LAUNCH(p->ctx, five_to_nine, blocks_for(Lc.n, 256), 256, 0, st, Lc.n,
                  Lc.c4.as<double>(4 * Lc.n), Lc.diag.as<double>(Lc.n), Lc.active.as<uint8_t>(Lc.n),
                  Lc.a9.as<double>(9 * Lc.n));
    int *status = p->status.as<int>(2);  // [0] singular, [1] the banded path fell back
    BT_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(int), st));
    double *inv = p->inv.as<double>(Lc.n * Lc.n);
    const double *a9c = Lc.a9.as<double>(9 * Lc.n);
    if (band_half(Lc.nx, Lc.ny) <= kBandMax) {
        BT_LAUNCH(p->ctx, coarsest_band_invert, 1, kBandThreads, band_smem(Lc.nx, Lc.ny), st,
                  Lc.nx, Lc.ny, a9c, inv, status + 1);
        BT_LAUNCH(p->ctx, coarsest_invert, 1, kInvertThreads, 0, st, Lc.nx, Lc.ny, a9c, inv,
                  status, status + 1);
    } else {
        BT_LAUNCH(p->ctx, coarsest_invert, 1, kInvertThreads, 0, st, Lc.nx, Lc.ny, a9c, inv,
                  status, (const int *)nullptr);
    }
    BT_CHECK_LAUNCH();
    refresh_tail_image(p);
    p->built = true;
    p->reaction_on = reaction != nullptr;
}

// The tail: the longest run of coarsest levels (never level 0, whose operator is 5-point),
// each at most tail_nodes large, whose shared-memory image fits one block; its descriptors
// and layout, and the shared memory of the staged smoother.
void setup_tail(bt_poisson *p) {
    const int levels = (int)p->levels.size();
    p->tail_start = -1;
    p->tail_smem = 0;
    for (int l = levels - 1; l >= 1 && levels - l <= kTailMaxLevels; --l) {
        if (p->levels[l].n > p->tail_nodes || tail_layout(p->levels, l).total() > kTailSmemMax)
            break;
        p->tail_start = l;
    }
    const int big5 = (int)stage_smem(false, kStage5X, kStage5Y, kMaxPhases);
    const int big9 = (int)stage_smem(true, kStage9X, kStage9Y, kMaxPhases);
    BT_CUDA(cudaFuncSetAttribute(smooth_staged<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big5));
    BT_CUDA(cudaFuncSetAttribute(smooth_staged<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big5));
    BT_CUDA(cudaFuncSetAttribute(smooth_staged<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big9));
    // the largest band any solver's coarsest level needs (the attribute is the kernel's,
    // shared by every solver of the process: never set it to one mesh's own size)
    BT_CUDA(cudaFuncSetAttribute(coarsest_band_invert, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kCoarsest * (2 * kBandMax + 1))));
    if (p->tail_start <= 0) return;
    const TailLayout T = tail_layout(p->levels, p->tail_start);
    p->tail_smem = T.total();
    p->tail_doubles = T.doubles;
    p->tail_ints = T.ints;
    p->tail_words = (int)(T.image() / 16);
    std::vector<TailLevel> tail;
    for (int l = p->tail_start; l < levels; ++l) {
        Level &L = p->levels[l];
        TailLevel t{};
        t.nx = L.nx;
        t.ny = L.ny;
        t.n = L.n;
        t.a9 = L.a9.as<double>(9 * L.n);
        t.active = L.active.as<uint8_t>(L.n);
        t.x = L.x.as<double>(L.n);
        t.b = L.b.as<double>(L.n);
        if (l + 1 < levels) t.next = fine_of(L, p->levels[l + 1], false);
        tail.push_back(t);
    }
    // the largest any solver asks for: solvers of other meshes may launch concurrently
    BT_CUDA(cudaFuncSetAttribute(vcycle_tail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTailSmemMax));
    BT_CUDA(cudaMemcpy(p->tail_levels.as<TailLevel>(tail.size()), tail.data(),
                       sizeof(TailLevel) * tail.size(), cudaMemcpyHostToDevice));
    BT_CUDA(cudaMemcpy(p->tail_plans.as<TailPlan>(T.plan.size()), T.plan.data(),
                       sizeof(TailPlan) * T.plan.size(), cudaMemcpyHostToDevice));
    p->tail_image.get(T.image());
    refresh_tail_image(p);
}

// Copy the tail levels' coefficients, transfer tables and active flags into the tail's
// static image (after the hierarchy's coefficients change).
void refresh_tail_image(bt_poisson *p) {
    if (p->tail_start <= 0) return;
    cudaStream_t st = p->ctx->stream;
    const TailLayout T = tail_layout(p->levels, p->tail_start);
    char *image = static_cast<char *>(p->tail_image.get(T.image()));
    double *d = reinterpret_cast<double *>(image);
    int32_t *ints = reinterpret_cast<int32_t *>(d + T.doubles);
    uint8_t *bytes = reinterpret_cast<uint8_t *>(ints + T.ints);
    auto copy = [&](void *dst, const void *src, size_t n) {
        if (n) BT_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, st));
    };
    const int levels = (int)p->levels.size();
    for (int l = p->tail_start; l < levels; ++l) {
        Level &L = p->levels[l];
        const TailPlan &P = T.plan[l - p->tail_start];
        copy(bytes + P.act, L.active.as<uint8_t>(L.n), L.n);
        if (l + 1 == levels) continue;
        const Fine F = fine_of(L, p->levels[l + 1], false);
        copy(d + P.a9, L.a9.as<double>(9 * L.n), sizeof(double) * 9 * L.n);
        copy(d + P.wx, F.wx, sizeof(double) * P.nx);
        copy(d + P.wy, F.wy, sizeof(double) * P.ny);
        copy(d + P.rxw, F.rxw, sizeof(double) * kRestrict * P.ncx);
        copy(d + P.ryw, F.ryw, sizeof(double) * kRestrict * P.ncy);
        copy(ints + P.lox, F.lox, sizeof(int32_t) * P.nx);
        copy(ints + P.loy, F.loy, sizeof(int32_t) * P.ny);
        copy(ints + P.rx0, F.rx0, sizeof(int32_t) * P.ncx);
        copy(ints + P.ry0, F.ry0, sizeof(int32_t) * P.ncy);
    }
}

void drop_graphs(bt_poisson *p) {
    if (p->vexec) cudaGraphExecDestroy(p->vexec);
    if (p->vgraph) cudaGraphDestroy(p->vgraph);
    p->vexec = nullptr;
    p->vgraph = nullptr;
}

// The smoothing of level l before (pre) or after the coarse correction: red-black sweeps
// on level 0, four-colour sweeps on 9-point levels, the colours reversed afterwards; the
// phases in shared-memory staged launches (up to kMaxPhases each) that move x between the
// level's two buffers, or one in-place launch per colour.
// The level's smoothing sweeps; with xc, after adding the prolonged coarse correction
// (P of the fine-coarse pair `pf`) to x: in the first staged launch's read of x, or by
// prolong_add.
void smooth(bt_poisson *p, size_t l, bool pre, const Fine *pf = nullptr,
            const double *xc = nullptr) {
    cudaStream_t st = p->ctx->stream;
    Level &L = p->levels[l];
    const int T = 256;
    const double *b = L.b.as<double>(L.n);
    const uint8_t *act = L.active.as<uint8_t>(L.n);
    const bool five = l == 0;
    const int colours = five ? 2 : 4;
    const int sweeps = five ? p->fine_sweeps : p->coarse_sweeps;
    std::vector<int> order;
    for (int sw = 0; sw < sweeps; ++sw)
        for (int c = 0; c < colours; ++c) order.push_back(pre ? c : colours - 1 - c);
    if (p->staged) {
        const int tx = five ? kStage5X : kStage9X, ty = five ? kStage5Y : kStage9Y;
        const dim3 tiles((unsigned)((L.nx + tx - 1) / tx), (unsigned)((L.ny + ty - 1) / ty));
        for (size_t start = 0; start < order.size(); start += kMaxPhases) {
            Phases ph{};
            ph.count = (int)std::min<size_t>(kMaxPhases, order.size() - start);
            for (int k = 0; k < ph.count; ++k) ph.colour[k] = order[start + k];
            const int halo = stage_halo(ph.count);
            const size_t smem = stage_smem(!five, tx, ty, halo);
            const int per = (tx + 2 * halo) * (ty + 2 * halo) / colours;
            const int own = (per + kStageThreads - 1) / kStageThreads;
            double *x = L.x.as<double>(L.n);
            double *in = L.cur, *out = L.cur == x ? L.x2.as<double>(L.n) : x;
            const Fine F = start == 0 && xc ? *pf : Fine{};
            const double *add = start == 0 ? xc : nullptr;
            if (five && own <= 2)
                BT_LAUNCH(p->ctx, (smooth_staged<false, 2>), tiles, kStageThreads, smem, st, L.nx,
                          L.ny, L.c4.as<double>(4 * L.n), L.diag.as<double>(L.n),
                          (const double *)nullptr, act, b, in, out, tx, ty, ph, F, add);
            else if (five && own == 3)
                BT_LAUNCH(p->ctx, (smooth_staged<false, 3>), tiles, kStageThreads, smem, st, L.nx,
                          L.ny, L.c4.as<double>(4 * L.n), L.diag.as<double>(L.n),
                          (const double *)nullptr, act, b, in, out, tx, ty, ph, F, add);
            else if (!five && own == 1)
                BT_LAUNCH(p->ctx, (smooth_staged<true, 1>), tiles, kStageThreads, smem, st, L.nx,
                          L.ny, (const double *)nullptr, (const double *)nullptr,
                          L.a9.as<double>(9 * L.n), act, b, in, out, tx, ty, ph, F, add);
            else
                BT_REQUIRE(false, "poisson: staged smoothing tile too large for its block");
            L.cur = out;
        }
        return;
    }
    double *x = L.cur;
    if (xc) BT_LAUNCH(p->ctx, prolong_add, blocks_for(L.n, T), T, 0, st, *pf, xc, x);
    for (int c : order) {
        if (five) {
            const i64 per = L.nx * ((L.ny + 1) / 2);
            BT_LAUNCH(p->ctx, smooth5, blocks_for(per, T), T, 0, st, L.nx, L.ny,
                      L.c4.as<double>(4 * L.n), L.diag.as<double>(L.n), act, b, x, c);
        } else {
            const i64 per = colour_count(L.nx, L.ny, c);
            BT_LAUNCH(p->ctx, smooth9, blocks_for(per, T), T, 0, st, L.nx, L.ny,
                      L.a9.as<double>(9 * L.n), act, b, x, c);
        }
    }
}

// x = V-cycle(b) on level l (x starts at zero on entry for l > 0; level 0's x given).  The
// staged smoother moves a level's x between its two buffers; the cycle leaves it in the
// first.
void vcycle(bt_poisson *p, size_t l) {
    cudaStream_t st = p->ctx->stream;
    Level &L = p->levels[l];
    const int T = 256;
    if ((int)l == p->tail_start) {
        const int count = (int)(p->levels.size() - l);
        const Level &Lc = p->levels.back();
        BT_LAUNCH(p->ctx, vcycle_tail, 1, kTailThreads, p->tail_smem, st,
                  p->tail_levels.as<TailLevel>(count), p->tail_plans.as<TailPlan>(count), count,
                  static_cast<const uint4 *>(p->tail_image.get(16 * (size_t)p->tail_words)),
                  p->tail_words, p->tail_doubles, p->tail_ints, p->inv.as<double>(Lc.n * Lc.n),
                  p->coarse_sweeps);
        return;
    }
    if (l + 1 == p->levels.size()) {
        BT_LAUNCH(p->ctx, coarsest_apply, 1, kCoarsest, 0, st, (int)L.n, p->inv.as<double>(L.n * L.n),
                  L.active.as<uint8_t>(L.n), L.b.as<double>(L.n), L.x.as<double>(L.n));
        return;
    }
    Level &C = p->levels[l + 1];
    double *b = L.b.as<double>(L.n), *r = L.r.as<double>(L.n);
    const uint8_t *act = L.active.as<uint8_t>(L.n);
    L.cur = L.x.as<double>(L.n);
    smooth(p, l, true);
    if (l == 0)
        BT_LAUNCH(p->ctx, apply5, blocks_for(L.n, T), T, 0, st, L.nx, L.ny, L.c4.as<double>(4 * L.n),
                  L.diag.as<double>(L.n), act, L.cur, b, r);
    else
        BT_LAUNCH(p->ctx, residual9, blocks_for(L.n, T), T, 0, st, L.nx, L.ny,
                  L.a9.as<double>(9 * L.n), act, L.cur, b, r);
    Fine F = fine_of(L, C, l == 0);
    BT_LAUNCH(p->ctx, restrict_residual, blocks_for(C.n, T), T, 0, st, F, r, C.b.as<double>(C.n),
                                                          C.x.as<double>(C.n));
    vcycle(p, l + 1);
    smooth(p, l, false, &F, C.x.as<double>(C.n));
    if (L.cur != L.x.as<double>(L.n))
        BT_CUDA(cudaMemcpyAsync(L.x.as<double>(L.n), L.cur, sizeof(double) * L.n,
                                cudaMemcpyDeviceToDevice, st));
    L.cur = L.x.as<double>(L.n);
    BT_CHECK_LAUNCH();
}

// Capture the V-cycle (level 0's x zeroed, then the cycle on its b) as a graph: every
// buffer it touches keeps its address for the solver's life, so one capture serves every
// solve and every Newton Jacobian (whose coefficients change in place).
void capture_vcycle(bt_poisson *p) {
    // captured on the context's own stream (the default stream cannot capture); the
    // graph then runs on whichever stream the context queues on
    cudaStream_t st = p->ctx->own_stream;
    cudaStream_t queue = p->ctx->stream;
    Level &L = p->levels[0];
    const i64 before = p->ctx->launch_count;
    p->ctx->stream = st;
    BT_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
        BT_CUDA(cudaMemsetAsync(L.x.as<double>(L.n), 0, sizeof(double) * L.n, st));
        vcycle(p, 0);
    } catch (...) {
        cudaGraph_t broken = nullptr;
        cudaStreamEndCapture(st, &broken);
        if (broken) cudaGraphDestroy(broken);
        p->ctx->stream = queue;
        throw;
    }
    p->ctx->stream = queue;
    BT_CUDA(cudaStreamEndCapture(st, &p->vgraph));
    BT_CUDA(cudaGraphInstantiate(&p->vexec, p->vgraph, 0));
    p->vgraph_kernels = p->ctx->launch_count - before;
    p->ctx->launch_count = before;  // counted when the graph runs
}

// z = M v: one V-cycle from zero
void precondition(bt_poisson *p, const double *v, double *z) {
    Level &L = p->levels[0];
    cudaStream_t st = p->ctx->stream;
    if (!p->vexec) capture_vcycle(p);
    BT_CUDA(cudaMemcpyAsync(L.b.as<double>(L.n), v, sizeof(double) * L.n, cudaMemcpyDeviceToDevice, st));
    {
        Timed timed(p->ctx, "vcycle");
        BT_CUDA(cudaGraphLaunch(p->vexec, st));
    }
    p->ctx->launch_count += p->vgraph_kernels;
    BT_CUDA(cudaMemcpyAsync(z, L.x.as<double>(L.n), sizeof(double) * L.n, cudaMemcpyDeviceToDevice, st));
}

void apply(bt_poisson *p, const double *x, double *y) {
    Level &L = p->levels[0];
    BT_LAUNCH(p->ctx, apply5, blocks_for(L.n, 256), 256, 0, p->ctx->stream, L.nx, L.ny, L.c4.as<double>(4 * L.n), L.diag.as<double>(L.n),
        L.active.as<uint8_t>(L.n), x, nullptr, y);
}

double read_scalar(bt_poisson *p, const double *dev) {
    double *host = static_cast<double *>(p->ctx->host.get(sizeof(double) * 64));
    BT_CUDA(cudaMemcpyAsync(host, dev, sizeof(double), cudaMemcpyDeviceToHost, p->ctx->stream));
    BT_CUDA(cudaStreamSynchronize(p->ctx->stream));
    return host[0];
}

// One dot pass (dot_pass) over the n-vectors w and V's rows q < m; out gets its sums.
template <int MODE>
void dot_launch(bt_poisson *p, const double *V, const double *h, double *w, int m, double *out) {
    double *partial = p->dot_partial.as<double>((size_t)kDotBlocks * kDotMax);
    unsigned *ticket = p->dot_ticket.as<unsigned>(1);
    cudaStream_t st = p->ctx->stream;
    if (!p->ticket_ready) {
        BT_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
        p->ticket_ready = true;
    }
    BT_REQUIRE(m >= 1 && m <= kDotMax, "poisson: a dot pass takes 1 to 32 vectors");
#define BT_DOT(MQ)                                                                              \
    BT_LAUNCH(p->ctx, (dot_pass<MQ, MODE>), kDotBlocks, kDotThreads, 0, st, V, h, w, p->n, m,  \
              partial, ticket, out)
    if (m <= 1)
        BT_DOT(1);
    else if (m <= 8)
        BT_DOT(8);
    else if (m <= 16)
        BT_DOT(16);
    else
        BT_DOT(32);
#undef BT_DOT
}

// out[q] = <V_q, w> for q < m (V's rows of n values), deterministic
void dots(bt_poisson *p, const double *V, const double *w, int m, double *out) {
    dot_launch<kPlain>(p, V, nullptr, const_cast<double *>(w), m, out);
}

double norm2(bt_poisson *p, const double *v) {
    double *s = p->scalars.as<double>(8);
    dots(p, v, v, 1, s);
    return std::sqrt(read_scalar(p, s));
}

// The steps a cycle still needs by the rate of its last (up to three) steps, one fewer so
// that a queued step rarely runs past the end: at least 1.
int steps_to_queue(const Arnoldi &a) {
    const int j = a.j;
    const int k = std::min(j, 3);
    const double r = a.resid[j];
    if (k == 0 || !(r > 0.0) || !(a.resid[j - k] > 0.0)) return 1;
    const double rate = std::pow(r / a.resid[j - k], 1.0 / k);
    if (!(rate < 0.95)) return 1;
    const double left = std::log(a.tol / r) / std::log(rate);
    if (!(left < 1e6)) return 1;
    return std::max(1, (int)std::ceil(left) - 1);
}

// Solve A d = r0 for d (d zero on entry) by restarted right-preconditioned GMRES until
// ||r0 - A d|| <= abs_tol or max_iter V-cycles; returns the V-cycles run and the final
// residual norm.  The Arnoldi process runs on the device (Gram-Schmidt twice, the Givens
// rotations in arnoldi_step); the host queues steps in batches sized by the residual's
// rate and reads the state between them, and the cycle's solution is the same as if it
// read it after every step.
int gmres(bt_poisson *p, const double *r0, double *d, double abs_tol, int max_iter,
          double *final_norm) {
    const i64 n = p->n;
    const int m = p->restart;  // at most kDotMax - 1: a basis of m + 1 vectors
    cudaStream_t st = p->ctx->stream;
    double *V = p->V.as<double>((size_t)(m + 1) * n);
    double *Z = p->Z.as<double>((size_t)m * n);
    double *w = p->work.as<double>(n);
    // the device state: Arnoldi, H, cs, sn, g, y and the passes' coefficients and norm
    const size_t head = (sizeof(Arnoldi) + 255) / 256 * 256;
    const size_t doubles = (size_t)(m + 1) * m + 3 * m + 1 + 2 * (m + 2) + 1;
    unsigned char *state = p->arnoldi.as<unsigned char>(head + sizeof(double) * doubles);
    Arnoldi *a = reinterpret_cast<Arnoldi *>(state);
    double *H = reinterpret_cast<double *>(state + head);
    double *cs = H + (size_t)(m + 1) * m, *sn = cs + m, *g = sn + m, *y = g + m + 1;
    double *h1 = y + m, *h2 = h1 + (m + 2), *hn = h2 + (m + 2);
    Arnoldi *host = static_cast<Arnoldi *>(p->ctx->host.get(sizeof(Arnoldi)));
    int total = 0;
    BT_CUDA(cudaMemcpyAsync(w, r0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    double beta = norm2(p, w);
    double previous = INFINITY;
    // stop at the tolerance, or where a whole restart cycle no longer halves the true
    // residual: the rounding floor of the residual itself
    while (beta > abs_tol && total < max_iter && beta < 0.5 * previous) {
        previous = beta;
        if (!std::isfinite(beta)) throw Error{BT_ERR_NOCONV, "field solve: the residual is not finite"};
        BT_LAUNCH(p->ctx, scale_into, blocks_for(n, 256), 256, 0, st, w, 1.0 / beta, n, V);
        BT_LAUNCH(p->ctx, arnoldi_begin, 1, 32, 0, st, a, g, m, beta, abs_tol);
        int j = 0, batch = 2;
        for (;;) {
            const int count = std::min(batch, std::min(m - j, max_iter - total));
            for (int b = 0; b < count; ++b, ++j, ++total) {
                double *v = V + (i64)j * n, *z = Z + (i64)j * n;
                precondition(p, v, z);
                apply(p, z, w);
                dot_launch<kPlain>(p, V, nullptr, w, j + 1, h1);
                dot_launch<kOrthDots>(p, V, h1, w, j + 1, h2);
                dot_launch<kOrthNorm>(p, V, h2, w, j + 1, hn);
                BT_LAUNCH(p->ctx, scale_by_norm, blocks_for(n, 256), 256, 0, st, w, hn, n,
                          V + (i64)(j + 1) * n);
                BT_LAUNCH(p->ctx, arnoldi_step, 1, 32, 0, st, a, H, cs, sn, g, h1, h2, hn, j, m);
            }
            BT_CHECK_LAUNCH();
            BT_CUDA(cudaMemcpyAsync(host, a, sizeof(Arnoldi), cudaMemcpyDeviceToHost, st));
            BT_CUDA(cudaStreamSynchronize(st));
            if (host->done || j >= m || total >= max_iter) break;
            batch = steps_to_queue(*host);
        }
        // d += Z y, y = H^-1 g over the steps taken
        BT_LAUNCH(p->ctx, arnoldi_solve, 1, 32, 0, st, a, H, g, y, m);
        BT_LAUNCH(p->ctx, combine, blocks_for(n, 256), 256, 0, st, Z, y, a, n, d);
        // the true residual r0 - A d
        apply(p, d, w);
        BT_LAUNCH(p->ctx, subtract_from, blocks_for(n, 256), 256, 0, st, r0, n, w);
        BT_CHECK_LAUNCH();
        beta = norm2(p, w);
    }
    if (final_norm) *final_norm = beta;
    return total;
}

}  // namespace
}  // namespace bt

extern "C" int bt_poisson_create(bt_ctx *ctx, const bt_mesh_desc *m, bt_poisson **out) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && m && out, "poisson: null argument");
        BT_REQUIRE(m->nx >= 3 && m->ny >= 3, "poisson: the mesh needs at least 3 nodes per axis");
        BT_REQUIRE(m->x && m->fixed && m->fixed_value && m->distance, "poisson: null mesh array");
        BT_REQUIRE(m->h > 0.0, "poisson: h must be positive");
        auto p = new bt_poisson;
        try {
            p->ctx = ctx;
            p->nx = m->nx;
            p->ny = m->ny;
            p->n = m->nx * m->ny;
            p->h = m->h;
            p->cyl = m->cylindrical;
            if (p->cyl) {
                const double rows = m->origin_y / m->h;
                p->j0 = (i64)llround(rows);
                BT_REQUIRE(p->j0 >= 0 && std::fabs(rows - (double)p->j0) <= 1e-6,
                           "poisson: a cylindrical mesh starts on the axis or a multiple of h "
                           "above it");
            }
            for (int q = 0; q < 4; ++q) p->neumann[q] = m->neumann ? m->neumann[q] : 0.0;
            const i64 n = p->n;
            BT_CUDA(cudaMemcpy(p->x.as<double>(p->nx), m->x, sizeof(double) * p->nx, cudaMemcpyHostToDevice));
            BT_CUDA(cudaMemcpy(p->fixed.as<uint8_t>(n), m->fixed, n, cudaMemcpyHostToDevice));
            BT_CUDA(cudaMemcpy(p->value.as<double>(n), m->fixed_value, sizeof(double) * n, cudaMemcpyHostToDevice));
            BT_CUDA(cudaMemcpy(p->distance.as<double>(4 * n), m->distance, sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
            BT_CUDA(cudaMemcpy(p->fixed_eff.as<uint8_t>(n), m->fixed, n, cudaMemcpyHostToDevice));
            BT_CUDA(cudaMemcpy(p->value_eff.as<double>(n), m->fixed_value, sizeof(double) * n, cudaMemcpyHostToDevice));
            // the levels
            p->levels.reserve(48);
            i64 nx = p->nx, ny = p->ny;
            while (true) {
                p->levels.emplace_back();
                bt::Level &L = p->levels.back();
                L.nx = nx;
                L.ny = ny;
                L.n = nx * ny;
                L.x.as<double>(L.n);
                L.x2.as<double>(L.n);
                L.b.as<double>(L.n);
                L.r.as<double>(L.n);
                L.active.as<uint8_t>(L.n);
                if (p->levels.size() == 1) {
                    L.c4.as<double>(4 * L.n);
                    L.diag.as<double>(L.n);
                    L.base.as<double>(L.n);
                    L.weight.as<double>(L.n);
                } else {
                    L.a9.as<double>(9 * L.n);
                }
                const bool more = L.n > bt::kCoarsest && (nx > 3 || ny > 3);
                if (!more) break;
                bt::build_axis(L.ax, nx);
                bt::build_axis(L.ay, ny);
                nx = L.ax.nc;
                ny = L.ay.nc;
            }
            BT_REQUIRE(p->levels.back().n <= bt::kCoarsest, "poisson: coarsest level too large");
            bt::setup_tail(p);
            p->src.as<double>(n);
            bt::build_operator(p);
            BT_CUDA(cudaStreamSynchronize(ctx->stream));
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

extern "C" int bt_poisson_destroy(bt_poisson *p) {
    return bt::guarded([&] {
        if (!p) return;
        cudaStreamSynchronize(p->ctx->stream);
        delete p;
    });
}

extern "C" int bt_poisson_set_region(bt_poisson *p, const uint8_t *mask, double value) {
    return bt::guarded([&] {
        BT_REQUIRE(p, "poisson: null solver");
        const i64 n = p->n;
        std::vector<uint8_t> fixed(n);
        std::vector<double> val(n);
        BT_CUDA(cudaMemcpy(fixed.data(), p->fixed.as<uint8_t>(n), n, cudaMemcpyDeviceToHost));
        BT_CUDA(cudaMemcpy(val.data(), p->value.as<double>(n), sizeof(double) * n, cudaMemcpyDeviceToHost));
        if (mask)
            for (i64 f = 0; f < n; ++f)
                if (mask[f] && !fixed[f]) {
                    fixed[f] = 1;
                    val[f] = value;
                }
        BT_CUDA(cudaMemcpy(p->fixed_eff.as<uint8_t>(n), fixed.data(), n, cudaMemcpyHostToDevice));
        BT_CUDA(cudaMemcpy(p->value_eff.as<double>(n), val.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        p->has_region = mask != nullptr;
        p->region_value = value;
        bt::build_operator(p);
    });
}

extern "C" int bt_poisson_solve(bt_poisson *p, double *phi, const double *rho, double amplitude,
                                double temperature, double up, int32_t sign, double tol,
                                double newton_tol, int32_t max_newton, int32_t *newton_steps,
                                int32_t *cycles) {
    return bt::guarded([&] {
        BT_REQUIRE(p && phi, "poisson: null argument");
        BT_REQUIRE(tol > 0.0, "poisson: the tolerance must be positive");
        const i64 n = p->n;
        cudaStream_t st = p->ctx->stream;
        bt::Level &L0 = p->levels[0];
        double *b = p->rhs.as<double>(n);
        double *r0 = p->r0.as<double>(n);
        double *d = p->delta.as<double>(n);
        double *reaction = p->reaction.as<double>(n);
        double *scal = p->scalars.as<double>(16);
        const int max_cycles = 4000;
        bt::Timed timed(p->ctx, "field_solve");
        BT_LAUNCH(p->ctx, bt::prepare, bt::blocks_for(n, 256), 256, 0, st, n, rho, p->src.as<double>(n), L0.active.as<uint8_t>(n), p->value_eff.as<double>(n),
            b, phi);
        BT_CHECK_LAUNCH();
        int total_cycles = 0, steps = 0;
        BT_REQUIRE(!p->transposed || !(amplitude > 0.0),
                   "poisson: the transposed solver takes linear solves only");
        const double *weight = L0.weight.as<double>(n);
        const uint8_t *active = L0.active.as<uint8_t>(n);
        if (p->transposed) {  // A^T z = b as B y = W^-1 b, y = W^-1 z (transpose_c4)
            BT_LAUNCH(p->ctx, bt::scale_by_weight, bt::blocks_for(n, 256), 256, 0, st, n, weight, active, 1, b);
            BT_LAUNCH(p->ctx, bt::scale_by_weight, bt::blocks_for(n, 256), 256, 0, st, n, weight, active, 1, phi);
        }
        if (!(amplitude > 0.0)) {
            if (!p->built || p->reaction_on) bt::build_hierarchy(p, nullptr);
            // r0 = b - A phi; the tolerance is relative to the larger of |b| and |r0|
            BT_LAUNCH(p->ctx, bt::apply5, bt::blocks_for(n, 256), 256, 0, st, p->nx, p->ny, L0.c4.as<double>(4 * n), L0.diag.as<double>(n),
                L0.active.as<uint8_t>(n), phi, b, r0);
            BT_CHECK_LAUNCH();
            const double scale = std::max(bt::norm2(p, b), bt::norm2(p, r0));
            BT_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, st));
            double left = 0.0;
            const double goal = tol * (scale > 0.0 ? scale : 1.0);
            total_cycles = bt::gmres(p, r0, d, goal, max_cycles, &left);
            BT_LAUNCH(p->ctx, bt::add_into, bt::blocks_for(n, 256), 256, 0, st, d, n, phi);
            if (p->transposed)
                BT_LAUNCH(p->ctx, bt::scale_by_weight, bt::blocks_for(n, 256), 256, 0, st, n, weight, active, 0, phi);
            BT_CHECK_LAUNCH();
            // a residual stalled within 1e4 of the goal is the floor of its own rounding
            if (!(left <= 1e4 * goal))
                throw bt::Error{BT_ERR_NOCONV, "field solve: GMRES did not reach the tolerance"};
        } else {
            BT_REQUIRE(temperature > 0.0, "poisson: the temperature must be positive");
            BT_REQUIRE(sign == 1 || sign == -1, "poisson: the species' sign must be +-1");
            const int limit = max_newton > 0 ? max_newton : 100;
            bool converged = false;
            for (steps = 1; steps <= limit; ++steps) {
                BT_LAUNCH(p->ctx, bt::boltzmann, bt::blocks_for(n, 256), 256, 0, st, p->nx, p->ny, L0.c4.as<double>(4 * n), L0.base.as<double>(n),
                    L0.active.as<uint8_t>(n), phi, b, amplitude, temperature, up, (double)sign,
                    r0, reaction);
                BT_CHECK_LAUNCH();
                bt::build_hierarchy(p, reaction);
                const double fnorm = bt::norm2(p, r0);
                BT_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, st));
                double left = 0.0;
                total_cycles += bt::gmres(p, r0, d, tol * (fnorm > 0.0 ? fnorm : 1.0),
                                          max_cycles, &left);
                BT_LAUNCH(p->ctx, bt::add_into, bt::blocks_for(n, 256), 256, 0, st, d, n, phi);
                BT_LAUNCH(p->ctx, bt::max_abs, 1, 256, 0, st, d, n, scal + 8);
                BT_CHECK_LAUNCH();
                const double change = bt::read_scalar(p, scal + 8);
                if (!std::isfinite(change))
                    throw bt::Error{BT_ERR_NOCONV, "field solve: Newton's update is not finite"};
                if (change < newton_tol) {
                    converged = true;
                    break;
                }
            }
            if (!converged) steps = limit;
        }
        int status = 0;
        BT_CUDA(cudaMemcpyAsync(&status, p->status.as<int>(1), sizeof(int), cudaMemcpyDeviceToHost, st));
        BT_CUDA(cudaStreamSynchronize(st));
        if (status)
            throw bt::Error{BT_ERR_NOCONV, "field solve: the coarsest operator is singular (is any node held?)"};
        if (newton_steps) *newton_steps = steps;
        if (cycles) *cycles = total_cycles;
    });
}

namespace bt {
namespace {
// r = rho / eps0 + c - A phi on the free nodes of the level-0 operator (its diagonal
// without a Newton reaction), 0 on the held ones
__global__ void linear_residual(i64 nx, i64 ny, const double *__restrict__ c4,
                                const double *__restrict__ base, const double *__restrict__ src,
                                const uint8_t *__restrict__ active, const double *__restrict__ phi,
                                const double *__restrict__ rho, double *__restrict__ r) {
    const i64 n = nx * ny;
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    if (!active[f]) {
        r[f] = 0.0;
        return;
    }
    const i64 i = f / ny, j = f - i * ny;
    double s = base[f] * phi[f];
    if (i > 0) s -= c4[f] * phi[f - ny];
    if (i < nx - 1) s -= c4[n + f] * phi[f + ny];
    if (j > 0) s -= c4[2 * n + f] * phi[f - 1];
    if (j < ny - 1) s -= c4[3 * n + f] * phi[f + 1];
    r[f] = (rho ? rho[f] / kEps0 : 0.0) + src[f] - s;
}
}  // namespace
}  // namespace bt

extern "C" int bt_poisson_residual(bt_poisson *p, const double *phi, const double *rho,
                                   double *r) {
    return bt::guarded([&] {
        BT_REQUIRE(p && phi && r, "poisson residual: null argument");
        BT_REQUIRE(!p->transposed, "poisson residual: the solver is transposed");
        const i64 n = p->n;
        bt::Level &L0 = p->levels[0];
        BT_LAUNCH(p->ctx, bt::linear_residual, bt::blocks_for(n, 256), 256, 0, p->ctx->stream, p->nx, p->ny,
                  L0.c4.as<double>(4 * n), L0.base.as<double>(n), p->src.as<double>(n),
                  L0.active.as<uint8_t>(n), phi, rho, r);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_poisson_solve_reaction(bt_poisson *p, double *phi, const double *rho,
                                         const double *reaction, double tol, int32_t *cycles) {
    return bt::guarded([&] {
        BT_REQUIRE(p && phi && reaction, "poisson: null argument");
        BT_REQUIRE(tol > 0.0, "poisson: the tolerance must be positive");
        BT_REQUIRE(!p->transposed, "poisson: the transposed solver takes no reaction");
        const i64 n = p->n;
        cudaStream_t st = p->ctx->stream;
        bt::Level &L0 = p->levels[0];
        double *b = p->rhs.as<double>(n);
        double *r0 = p->r0.as<double>(n);
        double *d = p->delta.as<double>(n);
        bt::Timed timed(p->ctx, "field_solve");
        BT_LAUNCH(p->ctx, bt::prepare, bt::blocks_for(n, 256), 256, 0, st, n, rho, p->src.as<double>(n),
                  L0.active.as<uint8_t>(n), p->value_eff.as<double>(n), b, phi);
        bt::build_hierarchy(p, reaction);
        BT_LAUNCH(p->ctx, bt::apply5, bt::blocks_for(n, 256), 256, 0, st, p->nx, p->ny, L0.c4.as<double>(4 * n),
                  L0.diag.as<double>(n), L0.active.as<uint8_t>(n), phi, b, r0);
        BT_CHECK_LAUNCH();
        const double scale = std::max(bt::norm2(p, b), bt::norm2(p, r0));
        BT_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, st));
        double left = 0.0;
        const double goal = tol * (scale > 0.0 ? scale : 1.0);
        const int total = bt::gmres(p, r0, d, goal, 4000, &left);
        BT_LAUNCH(p->ctx, bt::add_into, bt::blocks_for(n, 256), 256, 0, st, d, n, phi);
        BT_CHECK_LAUNCH();
        if (!(left <= 1e4 * goal))
            throw bt::Error{BT_ERR_NOCONV, "field solve: GMRES did not reach the tolerance"};
        int status = 0;
        BT_CUDA(cudaMemcpyAsync(&status, p->status.as<int>(1), sizeof(int), cudaMemcpyDeviceToHost, st));
        BT_CUDA(cudaStreamSynchronize(st));
        if (status)
            throw bt::Error{BT_ERR_NOCONV, "field solve: the coarsest operator is singular (is any node held?)"};
        if (cycles) *cycles = total;
    });
}

extern "C" int bt_poisson_vcycle(bt_poisson *p, const double *b, const double *reaction,
                                 int32_t rebuild, double *z) {
    return bt::guarded([&] {
        BT_REQUIRE(p && b && z, "poisson: null argument");
        BT_REQUIRE(!p->transposed, "poisson: the transposed solver takes no V-cycle here");
        if (rebuild || !p->built || p->reaction_on != (reaction != nullptr))
            bt::build_hierarchy(p, reaction);
        bt::precondition(p, b, z);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_poisson_set_transposed(bt_poisson *p, int32_t on) {
    return bt::guarded([&] {
        BT_REQUIRE(p, "poisson: null solver");
        if ((on != 0) == p->transposed) return;
        BT_CUDA(cudaStreamSynchronize(p->ctx->stream));
        p->transposed = on != 0;
        bt::build_operator(p);
    });
}

extern "C" int bt_poisson_fixed_adjoint(bt_poisson *p, const double *z, const double *phi_bar,
                                        double *out) {
    return bt::guarded([&] {
        BT_REQUIRE(p && z && phi_bar && out, "poisson: null argument");
        const i64 n = p->n;
        bt::Level &L0 = p->levels[0];
        const double *c4 = p->transposed ? p->c4_plain.as<double>(4 * n) : L0.c4.as<double>(4 * n);
        BT_LAUNCH(p->ctx, bt::fixed_adjoint, bt::blocks_for(n, 256), 256, 0, p->ctx->stream,
                  p->nx, p->ny, c4, L0.active.as<uint8_t>(n), z, phi_bar, out);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_poisson_set_options(bt_poisson *p, int32_t fine_sweeps, int32_t coarse_sweeps,
                                      int32_t staged, int64_t tail_nodes) {
    return bt::guarded([&] {
        BT_REQUIRE(p, "poisson: null solver");
        BT_REQUIRE(fine_sweeps >= 1 && fine_sweeps <= 4, "poisson: fine_sweeps must be 1 to 4");
        BT_REQUIRE(coarse_sweeps >= 1 && coarse_sweeps <= 4,
                   "poisson: coarse_sweeps must be 1 to 4");
        BT_REQUIRE(tail_nodes >= 1, "poisson: tail_nodes must be positive");
        BT_CUDA(cudaStreamSynchronize(p->ctx->stream));
        p->fine_sweeps = fine_sweeps;
        p->coarse_sweeps = coarse_sweeps;
        p->staged = staged != 0;
        p->tail_nodes = tail_nodes;
        bt::drop_graphs(p);
        bt::setup_tail(p);
    });
}

// -- the batched field solve --------------------------------------------------------------
//
// Many candidates' linear field solves at once: each candidate keeps its own solver (its
// operator and multigrid hierarchy, built as for a single solve), and one launch per level
// step covers the level of every candidate that has it -- a table of (candidate, level)
// entries and the first block of each, so a block finds its entry by bisection.  The
// candidates' hierarchies are aligned at their finest levels: step l holds level l of every
// candidate whose one-block tail starts below l; the tails of all candidates run in one
// launch of one block each.  The iteration is multigrid's own: d <- d + V(r0 - A d), each
// candidate until its residual meets the single solve's criterion (|r| <= tol max(|b|,
// |r0|)) or stops falling (its rounding floor); a candidate that has stopped leaves every
// launch (its live flag), so the tables stay fixed for the batch's life.

namespace bt {
namespace {

constexpr int kBatchThreads = 256;

// One (candidate, level) of a level step: the level's arrays and its transfer to the next.
struct BatchLevel {
    int cand;
    i64 nx, ny, n;
    const double *c4, *diag, *a9;  // level 0: c4, diag; coarse levels: a9
    const uint8_t *active;
    double *x, *x2, *b, *r;
    Fine F;           // to the next level
    double *xc, *bc;  // the next level's x and b
    i64 ncn;          // the next level's nodes
};

// One candidate's finest level for the outer iteration.
struct BatchFine {
    int cand;
    i64 nx, ny, n;
    const double *c4, *diag, *src, *value;
    const uint8_t *active;
    double *phi;        // its part of the batch's potential
    const double *rho;  // and of the density
    double *b, *r0, *d;
    double *vb, *vx;    // level 0's b and x: the V-cycle's input and output
};

struct BatchTail {
    int cand;
    const TailLevel *levels;
    const TailPlan *plans;
    int count;
    const uint4 *image;
    int words, doubles, ints;
    const double *inv;
    int sweeps;
};

// The entry of block `block`: the last whose first block is at or before it.
__device__ __forceinline__ int find_entry(const int *__restrict__ start, int n, int block) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= block)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Smoothing phases of every entry's level, a staged tile a block: from one of the level's
// x buffers (0: x, 1: x2) into the other; `zero_in`: x starts at zero (not read);
// `prolong`: the prolonged coarse correction is added as x is read.
template <bool NINE, int R>
__global__ void __launch_bounds__(kStageThreads)
    batch_smooth(const BatchLevel *__restrict__ E, const int *__restrict__ ids,
                 const int *__restrict__ start, int ne, const uint8_t *__restrict__ live,
                 int tx, int ty, Phases ph, int from, int prolong, int zero_in) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchLevel &L = E[ids[slot]];
    if (!live[L.cand]) return;
    const i64 local = (i64)blockIdx.x - start[slot];
    const i64 tiles_y = (L.ny + ty - 1) / ty;
    const i64 bx = local / tiles_y, by = local - bx * tiles_y;
    const double *in = from ? L.x2 : L.x;
    double *out = from ? L.x : L.x2;
    const Fine none{};
    smooth_staged_tile<NINE, R>(L.nx, L.ny, L.c4, L.diag, L.a9, L.active, L.b, in, out, tx, ty,
                                ph, prolong ? L.F : none, prolong ? L.xc : nullptr, bx, by,
                                zero_in != 0);
}

// r = b - A x on every entry's level (x in the buffer `from` names: 0 x, 1 x2), then
// (after the launch) its restriction.
template <bool NINE>
__global__ void batch_residual(const BatchLevel *__restrict__ E, const int *__restrict__ ids,
                               const int *__restrict__ start,
                               int ne, const uint8_t *__restrict__ live, int from) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchLevel &L = E[ids[slot]];
    if (!live[L.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    if (f >= L.n) return;
    const double *x = from ? L.x2 : L.x;
    if (NINE)
        residual9_item(f, L.nx, L.ny, L.a9, L.active, x, L.b, L.r, PlainLoad{});
    else
        apply5_item(f, L.nx, L.ny, L.c4, L.diag, L.active, x, L.b, L.r);
}

// b of the next level = R r, its x = 0.
__global__ void batch_restrict(const BatchLevel *__restrict__ E, const int *__restrict__ ids,
                               const int *__restrict__ start,
                               int ne, const uint8_t *__restrict__ live) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchLevel &L = E[ids[slot]];
    if (!live[L.cand]) return;
    const i64 t = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    if (t >= L.ncn) return;
    restrict_item(t, L.F, L.r, L.bc, L.xc, PlainLoad{});
}

// Every candidate's coarse levels, one block each.
__global__ void __launch_bounds__(kTailThreads, 1)
    batch_tail(const BatchTail *__restrict__ T, const int *__restrict__ ids,
               const uint8_t *__restrict__ live) {
    const BatchTail &t = T[ids[blockIdx.x]];
    if (!live[t.cand]) return;
    vcycle_tail_run(t.levels, t.plans, t.count, t.image, t.words, t.doubles, t.ints, t.inv,
                    t.sweeps);
}

// The per-block partial sums of the finest levels' squares: part[2 block + q].
__device__ __forceinline__ void block_sums(double a, double b, double *__restrict__ part) {
    __shared__ double sa[kBatchThreads / 32], sb[kBatchThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < kBatchThreads / 32; ++w) {
            ta += sa[w];
            tb += sb[w];
        }
        part[2 * blockIdx.x] = ta;
        part[2 * blockIdx.x + 1] = tb;
    }
}

// The right-hand side and the held potentials (prepare), then r0 = b - A phi (a second
// launch: it reads the neighbours' held values).
__global__ void batch_prepare(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                              int ne, const uint8_t *__restrict__ live) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchFine &F = E[ids[slot]];
    if (!live[F.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    if (f >= F.n) return;
    if (F.active[f]) {
        F.b[f] = (F.rho ? F.rho[f] / kEps0 : 0.0) + F.src[f];
    } else {
        F.b[f] = 0.0;
        F.phi[f] = F.value[f];
    }
}

// r0 = b - A phi, the V-cycle's first input r0, d = 0; the partial sums of |b|^2, |r0|^2.
__global__ void batch_initial(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                              int ne, const uint8_t *__restrict__ live, double *__restrict__ part) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchFine &F = E[ids[slot]];
    if (!live[F.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    double bb = 0.0, rr = 0.0;
    if (f < F.n) {
        const double r = apply5_item(f, F.nx, F.ny, F.c4, F.diag, F.active, F.phi, F.b, F.r0);
        F.vb[f] = r;
        F.d[f] = 0.0;
        const double b = F.b[f];
        bb = b * b;
        rr = r * r;
    }
    block_sums(bb, rr, part);
}

// d += the V-cycle's correction.
__global__ void batch_correct(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                              int ne, const uint8_t *__restrict__ live) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchFine &F = E[ids[slot]];
    if (!live[F.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    if (f < F.n) F.d[f] += F.vx[f];
}

// The true residual r = r0 - A d as the next V-cycle's input; the partial sums of |r|^2.
__global__ void batch_residual0(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                                int ne, const uint8_t *__restrict__ live,
                                double *__restrict__ part) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchFine &F = E[ids[slot]];
    if (!live[F.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    double rr = 0.0;
    if (f < F.n) {
        const double r = apply5_item(f, F.nx, F.ny, F.c4, F.diag, F.active, F.d, F.r0, F.vb);
        rr = r * r;
    }
    block_sums(rr, 0.0, part);
}

// phi += d.
__global__ void batch_finish(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                             int ne, const uint8_t *__restrict__ solving) {
    const int slot = find_entry(start, ne, blockIdx.x);
    const BatchFine &F = E[ids[slot]];
    if (!solving[F.cand]) return;
    const i64 f = ((i64)blockIdx.x - start[slot]) * kBatchThreads + threadIdx.x;
    if (f < F.n) F.phi[f] += F.d[f];
}

// Per live candidate (a warp each): its blocks' partial sums added in block order.  First
// call (cycle 0): the goal tol max(|b|, |r0|) and the first residual; later: the residual
// after the cycle, and whether the candidate stops -- at the goal, or after three cycles
// that did not halve its best residual (its rounding floor).  state[4 e ..]: goal, best,
// last residual, cycles without halving; cycles[e]: the cycles it ran.
__global__ void batch_check(const BatchFine *__restrict__ E, const int *__restrict__ ids,
                              const int *__restrict__ start,
                            int ne, const double *__restrict__ part, double tol, int cycle,
                            uint8_t *__restrict__ live, double *__restrict__ state,
                            int32_t *__restrict__ cycles, int32_t *__restrict__ remaining) {
    const int slot = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (slot >= ne) return;
    const int e = ids[slot];
    const BatchFine &F = E[e];
    if (!live[F.cand]) return;
    const int b0 = start[slot];
    const int b1 = slot + 1 < ne ? start[slot + 1] : b0 + (int)((F.n + kBatchThreads - 1) / kBatchThreads);
    double s0 = 0.0, s1 = 0.0;
    for (int k = b0 + lane; k < b1; k += 32) {
        s0 += part[2 * k];
        s1 += part[2 * k + 1];
    }
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, off);
        s1 += __shfl_down_sync(0xffffffffu, s1, off);
    }
    if (lane != 0) return;
    double *st = state + 4 * e;
    if (cycle == 0) {
        const double scale = fmax(sqrt(s0), sqrt(s1));
        const double r = sqrt(s1);
        st[0] = tol * (scale > 0.0 ? scale : 1.0);
        st[1] = r;
        st[2] = r;
        st[3] = 0.0;
        cycles[e] = 0;
        if (!(r > st[0])) {
            live[F.cand] = 0;
            atomicSub(remaining, 1);
        }
        return;
    }
    const double r = sqrt(s0);
    cycles[e] = cycle;
    st[2] = r;
    if (r < 0.5 * st[1]) {
        st[1] = r;
        st[3] = 0.0;
    } else {
        st[3] += 1.0;
    }
    if (!(r > st[0]) || st[3] >= 3.0 || r != r) {
        live[F.cand] = 0;
        atomicSub(remaining, 1);
    }
}

}  // namespace
}  // namespace bt


struct bt_poisson_batch {
    bt_ctx *ctx = nullptr;
    std::vector<bt_poisson *> solvers;
    std::vector<i64> offset;  // each candidate's first node in the batch's arrays
    int steps = 0;            // level steps above the tails
    // A level step: all its entries (device) with their candidates and block counts (host),
    // and the launch tables of the entries whose candidates are live: their numbers and,
    // per kind of launch, each one's first block.
    struct Step {
        bt::Buffer entries;
        std::vector<int> cand, nx, ny, nodes, coarse;
        bt::Buffer ids, smooth_start, node_start, coarse_start;
        int n = 0, smooth_blocks = 0, node_blocks = 0, coarse_blocks = 0;
    };
    std::vector<Step> level;
    bt::Buffer tails, tail_ids;  // one block per live candidate
    int n_tails = 0;
    size_t tail_smem = 0;
    bt::Buffer fine, fine_ids, fine_start;
    std::vector<bt::BatchFine> fine_host;  // the device table's copy
    std::vector<int> fine_nodes;           // blocks of each candidate's finest level
    int n_fine = 0, fine_blocks = 0;
    std::vector<uint8_t> compacted;        // the live set of the launch tables
    bt::Buffer live, solving, part, state, cycles, remaining;
    bt::HostBuffer host;
    int fine_sweeps = 2, coarse_sweeps = 2;
    // The smoothing tiles (interior nodes along x and y) of level 0 and of the 9-point
    // levels, and the launches a 9-point smoothing is split into (1 or 2); chosen by timing
    // at the first solve unless set (tuned == false: still to be chosen).
    int tile5[2] = {32, 32}, tile9[2] = {16, 32}, split9 = 1;
    bool tuned = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~bt_poisson_batch() {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace bt {
namespace {

template <class T>
void upload(Buffer &dst, const std::vector<T> &src, cudaStream_t st) {
    if (src.empty()) return;
    BT_CUDA(cudaMemcpyAsync(dst.as<T>(src.size()), src.data(), sizeof(T) * src.size(),
                            cudaMemcpyHostToDevice, st));
}

// The launch tables of the candidates flagged in `alive` (host): the finished ones launch
// no blocks.  Queued on the stream, after the launches that read the old tables.
void compact(bt_poisson_batch *B, const uint8_t *alive) {
    cudaStream_t st = B->ctx->stream;
    const int count = (int)B->solvers.size();
    for (auto &S : B->level) {
        std::vector<int> ids, smooth, node, coarse;
        int sb = 0, nb = 0, cb = 0;
        const bool five = &S == &B->level[0];
        const int tx = five ? B->tile5[0] : B->tile9[0], ty = five ? B->tile5[1] : B->tile9[1];
        for (int e = 0; e < (int)S.cand.size(); ++e) {
            if (!alive[S.cand[e]]) continue;
            ids.push_back(e);
            smooth.push_back(sb);
            node.push_back(nb);
            coarse.push_back(cb);
            sb += ((S.nx[e] + tx - 1) / tx) * ((S.ny[e] + ty - 1) / ty);
            nb += S.nodes[e];
            cb += S.coarse[e];
        }
        S.n = (int)ids.size();
        S.smooth_blocks = sb;
        S.node_blocks = nb;
        S.coarse_blocks = cb;
        upload(S.ids, ids, st);
        upload(S.smooth_start, smooth, st);
        upload(S.node_start, node, st);
        upload(S.coarse_start, coarse, st);
    }
    std::vector<int> tails, fine, start;
    int fb = 0;
    for (int c = 0; c < count; ++c) {
        if (!alive[c]) continue;
        tails.push_back(c);
        fine.push_back(c);
        start.push_back(fb);
        fb += B->fine_nodes[c];
    }
    B->n_tails = (int)tails.size();
    B->n_fine = (int)fine.size();
    B->fine_blocks = fb;
    upload(B->tail_ids, tails, st);
    upload(B->fine_ids, fine, st);
    upload(B->fine_start, start, st);
    B->compacted.assign(alive, alive + count);
}

// The staged smoother's nodes a thread per colour for a tile (tx, ty) and `count` phases.
int stage_own(bool nine, int tx, int ty, int count) {
    const int halo = stage_halo(count);
    const int per = (tx + 2 * halo) * (ty + 2 * halo) / (nine ? 4 : 2);
    return (per + kStageThreads - 1) / kStageThreads;
}

int fine_own(int count) { return stage_own(false, kStage5X, kStage5Y, count); }

Phases batch_phases(int sweeps, int colours, bool pre, int first, int count) {
    Phases ph{};
    std::vector<int> order;
    for (int s = 0; s < sweeps; ++s)
        for (int c = 0; c < colours; ++c) order.push_back(pre ? c : colours - 1 - c);
    ph.count = count;
    for (int k = 0; k < count; ++k) ph.colour[k] = order[first + k];
    return ph;
}

// One staged launch over step l's live entries: phases [first, first + count) of the
// smoothing, from buffer `from` into the other.
void batch_smooth_launch(bt_poisson_batch *B, int l, bool pre, int first, int count, int from,
                         int prolong, int zero_in) {
    bt_ctx *ctx = B->ctx;
    auto &S = B->level[l];
    const bool nine = l > 0;
    const uint8_t *live = B->live.as<uint8_t>(B->solvers.size());
    const BatchLevel *E = S.entries.as<BatchLevel>(S.cand.size());
    const int *ids = S.ids.as<int>(S.n), *start = S.smooth_start.as<int>(S.n);
    const int tx = nine ? B->tile9[0] : B->tile5[0], ty = nine ? B->tile9[1] : B->tile5[1];
    const Phases ph = batch_phases(nine ? B->coarse_sweeps : B->fine_sweeps, nine ? 4 : 2, pre,
                                   first, count);
    const size_t smem = stage_smem(nine, tx, ty, stage_halo(count));
    const int own = stage_own(nine, tx, ty, count);
#define BT_BATCH_SMOOTH(N, R)                                                                 \
    BT_LAUNCH(ctx, (batch_smooth<N, R>), S.smooth_blocks, kStageThreads, smem, ctx->stream, E, \
              ids, start, S.n, live, tx, ty, ph, from, prolong, zero_in)
    if (!nine && own == 1)
        BT_BATCH_SMOOTH(false, 1);
    else if (!nine && own == 2)
        BT_BATCH_SMOOTH(false, 2);
    else if (!nine && own == 3)
        BT_BATCH_SMOOTH(false, 3);
    else if (nine && own == 1)
        BT_BATCH_SMOOTH(true, 1);
    else if (nine && own == 2)
        BT_BATCH_SMOOTH(true, 2);
    else
        BT_REQUIRE(false, "poisson batch: a smoothing tile too large for its block");
#undef BT_BATCH_SMOOTH
}

// The smoothing of step l's live entries before (pre) or after the coarse correction;
// returns the buffer that holds the result (0: x, 1: x2).  Level 0's pre-smoothing starts
// from zero; the post-smoothing adds the prolonged correction as it reads.  Before the
// correction the input is the pre-smoothing's result `from`.
int batch_smooth_step(bt_poisson_batch *B, int l, bool pre, int from = 0) {
    auto &S = B->level[l];
    if (S.n == 0) return from;
    const bool nine = l > 0;
    const int phases = nine ? 4 * B->coarse_sweeps : 2 * B->fine_sweeps;
    const int split = nine ? B->split9 : 1;
    const int per = (phases + split - 1) / split;
    int in = pre ? 0 : from;
    for (int first = 0, k = 0; first < phases; first += per, ++k) {
        const int count = std::min(per, phases - first);
        batch_smooth_launch(B, l, pre, first, count, in, (!pre && k == 0) ? 1 : 0,
                            (pre && k == 0 && !nine) ? 1 : 0);
        in ^= 1;
    }
    return in;
}

// One V-cycle of every live candidate: level 0's b (its residual) into level 0's x.
void batch_vcycle(bt_poisson_batch *B) {
    bt_ctx *ctx = B->ctx;
    cudaStream_t st = ctx->stream;
    const uint8_t *live = B->live.as<uint8_t>(B->solvers.size());
    std::vector<int> held(B->steps, 0);  // where each step's pre-smoothing left x
    for (int l = 0; l < B->steps; ++l) {
        auto &S = B->level[l];
        if (S.n == 0) continue;
        const BatchLevel *E = S.entries.as<BatchLevel>(S.cand.size());
        const int *ids = S.ids.as<int>(S.n);
        held[l] = batch_smooth_step(B, l, true);
        if (l == 0)
            BT_LAUNCH(ctx, batch_residual<false>, S.node_blocks, kBatchThreads, 0, st, E, ids,
                      S.node_start.as<int>(S.n), S.n, live, held[l]);
        else
            BT_LAUNCH(ctx, batch_residual<true>, S.node_blocks, kBatchThreads, 0, st, E, ids,
                      S.node_start.as<int>(S.n), S.n, live, held[l]);
        BT_LAUNCH(ctx, batch_restrict, S.coarse_blocks, kBatchThreads, 0, st, E, ids,
                  S.coarse_start.as<int>(S.n), S.n, live);
    }
    if (B->n_tails)
        BT_LAUNCH(ctx, batch_tail, (unsigned)B->n_tails, kTailThreads, B->tail_smem, st,
                  B->tails.as<BatchTail>(B->solvers.size()), B->tail_ids.as<int>(B->n_tails),
                  live);
    for (int l = B->steps - 1; l >= 0; --l) {
        // the post-smoothing must leave x in the level's x buffer (the next coarser level's
        // x, or level 0's output)
        const int at = batch_smooth_step(B, l, false, held[l]);
        BT_REQUIRE(B->level[l].n == 0 || at == 0, "poisson batch: smoothing left x in x2");
    }
    BT_CHECK_LAUNCH();
}

}  // namespace
}  // namespace bt

namespace bt {
namespace {

// The project's autotuner of the batched V-cycle: the staged smoothing tiles of level 0 and
// of the 9-point levels (and whether a 9-point smoothing is one launch of all its phases,
// with a halo as wide as them, or two of half as many), timed on this batch's own V-cycle
// (two cycles each, CUDA events on the stream) from the residual of its first solve; the
// fastest is kept.  The choices trade a tile's re-read halo against blocks per SM.
void tune_tiling(bt_poisson_batch *B) {
    cudaStream_t st = B->ctx->stream;
    const std::vector<uint8_t> set = B->compacted;
    auto time_cycle = [&]() {
        compact(B, set.data());
        BT_CUDA(cudaEventRecord(B->ev[0], st));
        for (int k = 0; k < 2; ++k) batch_vcycle(B);
        BT_CUDA(cudaEventRecord(B->ev[1], st));
        BT_CUDA(cudaEventSynchronize(B->ev[1]));
        float ms = 0.0f;
        BT_CUDA(cudaEventElapsedTime(&ms, B->ev[0], B->ev[1]));
        return ms;
    };
    const int tiles5[][2] = {{32, 32}, {32, 16}, {16, 32}, {64, 16}};
    float best = 1e30f;
    int pick5[2] = {B->tile5[0], B->tile5[1]};
    for (const auto &t : tiles5) {
        if (stage_own(false, t[0], t[1], 2 * B->fine_sweeps) > 3) continue;
        B->tile5[0] = t[0];
        B->tile5[1] = t[1];
        const float ms = time_cycle();
        if (ms < best) {
            best = ms;
            pick5[0] = t[0];
            pick5[1] = t[1];
        }
    }
    B->tile5[0] = pick5[0];
    B->tile5[1] = pick5[1];
    const int tiles9[][3] = {{16, 32, 1}, {16, 32, 2}, {16, 16, 2}, {32, 16, 2}, {32, 32, 2}};
    best = 1e30f;
    int pick9[3] = {B->tile9[0], B->tile9[1], B->split9};
    for (const auto &t : tiles9) {
        const int phases = 4 * B->coarse_sweeps;
        const int count = (phases + t[2] - 1) / t[2];
        if (stage_own(true, t[0], t[1], count) > 2 ||
            stage_smem(true, t[0], t[1], stage_halo(count)) > 200 * 1024)
            continue;
        B->tile9[0] = t[0];
        B->tile9[1] = t[1];
        B->split9 = t[2];
        const float ms = time_cycle();
        if (ms < best) {
            best = ms;
            pick9[0] = t[0];
            pick9[1] = t[1];
            pick9[2] = t[2];
        }
    }
    B->tile9[0] = pick9[0];
    B->tile9[1] = pick9[1];
    B->split9 = pick9[2];
    compact(B, set.data());
    B->tuned = true;
}

}  // namespace
}  // namespace bt

extern "C" int bt_poisson_batch_create(bt_ctx *ctx, bt_poisson *const *solvers, int64_t count,
                                       const int64_t *offset, bt_poisson_batch **out) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && solvers && offset && out, "poisson batch: null argument");
        BT_REQUIRE(count >= 1 && count <= (1 << 20), "poisson batch: 1 to 2^20 candidates");
        auto B = new bt_poisson_batch;
        try {
            B->ctx = ctx;
            cudaStream_t st = ctx->stream;
            B->solvers.assign(solvers, solvers + count);
            B->offset.assign(offset, offset + count);
            bt_poisson *first = B->solvers[0];
            BT_REQUIRE(first, "poisson batch: null solver");
            B->fine_sweeps = first->fine_sweeps;
            B->coarse_sweeps = first->coarse_sweeps;
            for (i64 c = 0; c < count; ++c) {
                bt_poisson *p = B->solvers[c];
                BT_REQUIRE(p, "poisson batch: null solver");
                BT_REQUIRE(p->ctx == ctx, "poisson batch: every solver must share the context");
                BT_REQUIRE(!p->transposed, "poisson batch: the transposed solver is not batched");
                BT_REQUIRE(p->staged, "poisson batch: needs the staged smoother");
                BT_REQUIRE(p->fine_sweeps == B->fine_sweeps && p->coarse_sweeps == B->coarse_sweeps,
                           "poisson batch: every solver needs the same smoothing sweeps");
                BT_REQUIRE(B->coarse_sweeps * 4 <= bt::kMaxPhases && B->fine_sweeps * 2 <= bt::kMaxPhases,
                           "poisson batch: a smoothing must fit one staged launch");
                BT_REQUIRE(bt::fine_own(2 * B->fine_sweeps) <= 3,
                           "poisson batch: the fine smoothing tile is too large for its block");
                BT_REQUIRE(p->tail_start >= 1,
                           "poisson batch: a candidate's mesh is too small for the batched cycle");
                B->steps = std::max(B->steps, p->tail_start);
                B->tail_smem = std::max(B->tail_smem, p->tail_smem);
            }
            B->level.resize(B->steps);
            for (int l = 0; l < B->steps; ++l) {
                std::vector<bt::BatchLevel> E;
                auto &S = B->level[l];
                const bool five = l == 0;
                for (i64 c = 0; c < count; ++c) {
                    bt_poisson *p = B->solvers[c];
                    if (l >= p->tail_start) continue;
                    bt::Level &L = p->levels[l], &C = p->levels[l + 1];
                    bt::BatchLevel e{};
                    e.cand = (int)c;
                    e.nx = L.nx;
                    e.ny = L.ny;
                    e.n = L.n;
                    if (five) {
                        e.c4 = L.c4.as<double>(4 * L.n);
                        e.diag = L.diag.as<double>(L.n);
                    } else {
                        e.a9 = L.a9.as<double>(9 * L.n);
                    }
                    e.active = L.active.as<uint8_t>(L.n);
                    e.x = L.x.as<double>(L.n);
                    e.x2 = L.x2.as<double>(L.n);
                    e.b = L.b.as<double>(L.n);
                    e.r = L.r.as<double>(L.n);
                    e.F = bt::fine_of(L, C, five);
                    e.xc = C.x.as<double>(C.n);
                    e.bc = C.b.as<double>(C.n);
                    e.ncn = C.n;
                    E.push_back(e);
                    S.cand.push_back((int)c);
                    S.nx.push_back((int)L.nx);
                    S.ny.push_back((int)L.ny);
                    S.nodes.push_back((int)bt::blocks_for(L.n, bt::kBatchThreads));
                    S.coarse.push_back((int)bt::blocks_for(C.n, bt::kBatchThreads));
                }
                bt::upload(S.entries, E, st);
            }
            std::vector<bt::BatchTail> T;
            std::vector<bt::BatchFine> F;
            int all_blocks = 0;
            for (i64 c = 0; c < count; ++c) {
                bt_poisson *p = B->solvers[c];
                const int first_tail = p->tail_start;
                const int levels = (int)p->levels.size();
                const bt::Level &Lc = p->levels.back();
                bt::BatchTail t{};
                t.cand = (int)c;
                t.levels = p->tail_levels.as<bt::TailLevel>(levels - first_tail);
                t.plans = p->tail_plans.as<bt::TailPlan>(levels - first_tail);
                t.count = levels - first_tail;
                t.image = static_cast<const uint4 *>(p->tail_image.get(16 * (size_t)p->tail_words));
                t.words = p->tail_words;
                t.doubles = p->tail_doubles;
                t.ints = p->tail_ints;
                t.inv = p->inv.as<double>(Lc.n * Lc.n);
                t.sweeps = p->coarse_sweeps;
                T.push_back(t);
                bt::Level &L0 = p->levels[0];
                const i64 n = p->n;
                bt::BatchFine f{};
                f.cand = (int)c;
                f.nx = p->nx;
                f.ny = p->ny;
                f.n = n;
                f.c4 = L0.c4.as<double>(4 * n);
                f.diag = L0.diag.as<double>(n);
                f.src = p->src.as<double>(n);
                f.value = p->value_eff.as<double>(n);
                f.active = L0.active.as<uint8_t>(n);
                f.b = p->rhs.as<double>(n);
                f.r0 = p->r0.as<double>(n);
                f.d = p->delta.as<double>(n);
                f.vb = L0.b.as<double>(n);
                f.vx = L0.x.as<double>(n);
                F.push_back(f);
                B->fine_nodes.push_back((int)bt::blocks_for(n, bt::kBatchThreads));
                all_blocks += B->fine_nodes.back();
            }
            B->fine_host = F;
            bt::upload(B->tails, T, st);
            bt::upload(B->fine, F, st);
            {
                // the largest staged tile the tuner tries (bt::tune_tiling)
                const int big = 200 * 1024;
                BT_CUDA(cudaFuncSetAttribute(bt::batch_smooth<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
                BT_CUDA(cudaFuncSetAttribute(bt::batch_smooth<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
                BT_CUDA(cudaFuncSetAttribute(bt::batch_smooth<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
                BT_CUDA(cudaFuncSetAttribute(bt::batch_smooth<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
                BT_CUDA(cudaFuncSetAttribute(bt::batch_smooth<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
                BT_CUDA(cudaFuncSetAttribute(bt::batch_tail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)bt::kTailSmemMax));
            }
            for (auto &e : B->ev) BT_CUDA(cudaEventCreate(&e));
            B->live.as<uint8_t>(count);
            B->solving.as<uint8_t>(count);
            B->part.as<double>(2 * (size_t)all_blocks);
            B->state.as<double>(4 * (size_t)count);
            B->cycles.as<int32_t>(count);
            B->remaining.as<int32_t>(1);
            BT_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            delete B;
            throw;
        }
        *out = B;
    });
}

extern "C" int bt_poisson_batch_destroy(bt_poisson_batch *B) {
    return bt::guarded([&] {
        if (!B) return;
        cudaStreamSynchronize(B->ctx->stream);
        delete B;
    });
}

extern "C" int bt_poisson_batch_solve(bt_poisson_batch *B, double *phi, const double *rho,
                                      const uint8_t *members, double tol, int32_t max_cycles,
                                      int32_t *cycles, double *residual) {
    return bt::guarded([&] {
        BT_REQUIRE(B && phi && members, "poisson batch: null argument");
        BT_REQUIRE(tol > 0.0, "poisson batch: the tolerance must be positive");
        BT_REQUIRE(max_cycles >= 1, "poisson batch: max_cycles must be positive");
        bt_ctx *ctx = B->ctx;
        cudaStream_t st = ctx->stream;
        const i64 count = (i64)B->solvers.size();
        bt::Timed timed(ctx, "field_solve");
        // every member's hierarchy of its plain operator
        int members_n = 0;
        for (i64 c = 0; c < count; ++c) {
            if (!members[c]) continue;
            ++members_n;
            bt_poisson *p = B->solvers[c];
            if (!p->built || p->reaction_on) bt::build_hierarchy(p, nullptr);
        }
        if (members_n == 0) return;
        {
            // point the finest entries at this call's potential and density
            std::vector<bt::BatchFine> &F = B->fine_host;
            bool moved = false;
            for (i64 c = 0; c < count; ++c) {
                double *ph = phi + B->offset[c];
                const double *rh = rho ? rho + B->offset[c] : nullptr;
                if (F[c].phi != ph || F[c].rho != rh) moved = true;
                F[c].phi = ph;
                F[c].rho = rh;
            }
            if (moved) bt::upload(B->fine, F, st);
        }
        uint8_t *live = B->live.as<uint8_t>(count);
        uint8_t *solving = B->solving.as<uint8_t>(count);
        BT_CUDA(cudaMemcpyAsync(live, members, count, cudaMemcpyHostToDevice, st));
        BT_CUDA(cudaMemcpyAsync(solving, members, count, cudaMemcpyHostToDevice, st));
        int32_t *remaining = B->remaining.as<int32_t>(1);
        uint8_t *flags = static_cast<uint8_t *>(B->host.get((size_t)count + 64));
        int32_t *host_remaining = reinterpret_cast<int32_t *>(flags + ((count + 15) / 16) * 16);
        *host_remaining = members_n;
        BT_CUDA(cudaMemcpyAsync(remaining, host_remaining, sizeof(int32_t), cudaMemcpyHostToDevice, st));
        bt::compact(B, members);
        const bt::BatchFine *F = B->fine.as<bt::BatchFine>(count);
        double *part = B->part.as<double>(1);
        double *state = B->state.as<double>(4 * (size_t)count);
        int32_t *cyc = B->cycles.as<int32_t>(count);
        const int T = bt::kBatchThreads;
        auto fine_launch = [&](auto kernel, auto... more) {
            if (B->fine_blocks)
                BT_LAUNCH(ctx, kernel, B->fine_blocks, T, 0, st, F, B->fine_ids.as<int>(B->n_fine),
                          B->fine_start.as<int>(B->n_fine), B->n_fine, more...);
        };
        auto check = [&](int cycle) {
            BT_LAUNCH(ctx, bt::batch_check, bt::blocks_for((i64)B->n_fine * 32, 256), 256, 0, st, F,
                      B->fine_ids.as<int>(B->n_fine), B->fine_start.as<int>(B->n_fine),
                      B->n_fine, (const double *)part, tol, cycle, live, state, cyc, remaining);
        };
        fine_launch(bt::batch_prepare, (const uint8_t *)live);
        fine_launch(bt::batch_initial, (const uint8_t *)live, part);
        check(0);
        BT_CHECK_LAUNCH();
        if (!B->tuned) bt::tune_tiling(B);
        for (int cycle = 1; cycle <= max_cycles; ++cycle) {
            BT_CUDA(cudaMemcpyAsync(flags, live, count, cudaMemcpyDeviceToHost, st));
            BT_CUDA(cudaStreamSynchronize(st));
            int alive = 0, before = 0;
            for (i64 c = 0; c < count; ++c) {
                alive += flags[c] != 0;
                before += B->compacted[c] != 0;
            }
            if (alive == 0) break;
            // launch tables of the live candidates only, once enough of them have finished
            if (10 * alive <= 9 * before) bt::compact(B, flags);
            {
                bt::Timed vt(ctx, "vcycle");
                bt::batch_vcycle(B);
            }
            fine_launch(bt::batch_correct, (const uint8_t *)live);
            fine_launch(bt::batch_residual0, (const uint8_t *)live, part);
            check(cycle);
            BT_CHECK_LAUNCH();
        }
        bt::compact(B, members);
        fine_launch(bt::batch_finish, (const uint8_t *)solving);
        BT_CHECK_LAUNCH();
        std::vector<double> S(4 * count);
        std::vector<int32_t> C(count);
        BT_CUDA(cudaMemcpyAsync(S.data(), state, sizeof(double) * 4 * count, cudaMemcpyDeviceToHost, st));
        BT_CUDA(cudaMemcpyAsync(C.data(), cyc, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, st));
        BT_CUDA(cudaStreamSynchronize(st));
        for (i64 c = 0; c < count; ++c) {
            if (!members[c]) continue;
            if (cycles) cycles[c] = C[c];
            if (residual) residual[c] = S[4 * c + 2];
            // a residual stalled within 1e4 of the goal is the floor of its own rounding
            if (!(S[4 * c + 2] <= 1e4 * S[4 * c]))
                throw bt::Error{BT_ERR_NOCONV, "batched field solve: a candidate did not reach the tolerance"};
        }
    });
}

extern "C" int bt_poisson_batch_tiling(bt_poisson_batch *B, int32_t set, int32_t *tiling) {
    return bt::guarded([&] {
        BT_REQUIRE(B && tiling, "poisson batch: null argument");
        if (set) {
            if (tiling[0] <= 0) {
                B->tuned = false;
                return;
            }
            for (int q = 0; q < 5; ++q)
                BT_REQUIRE(tiling[q] > 0, "poisson batch: tile sizes and split must be positive");
            BT_REQUIRE(tiling[4] <= 2, "poisson batch: a 9-point smoothing splits into 1 or 2 launches");
            const int phases9 = 4 * B->coarse_sweeps, count9 = (phases9 + tiling[4] - 1) / tiling[4];
            BT_REQUIRE(bt::stage_own(false, tiling[0], tiling[1], 2 * B->fine_sweeps) <= 3 &&
                           bt::stage_smem(false, tiling[0], tiling[1], bt::stage_halo(2 * B->fine_sweeps)) <= 200 * 1024,
                       "poisson batch: the level-0 tile is too large for its block");
            BT_REQUIRE(bt::stage_own(true, tiling[2], tiling[3], count9) <= 2 &&
                           bt::stage_smem(true, tiling[2], tiling[3], bt::stage_halo(count9)) <= 200 * 1024,
                       "poisson batch: the 9-point tile is too large for its block");
            B->tile5[0] = tiling[0];
            B->tile5[1] = tiling[1];
            B->tile9[0] = tiling[2];
            B->tile9[1] = tiling[3];
            B->split9 = tiling[4];
            B->tuned = true;
            return;
        }
        tiling[0] = B->tile5[0];
        tiling[1] = B->tile5[1];
        tiling[2] = B->tile9[0];
        tiling[3] = B->tile9[1];
        tiling[4] = B->split9;
        tiling[5] = B->tuned ? 1 : 0;
    });
}

extern "C" int bt_poisson_set_context(bt_poisson *p, bt_ctx *ctx) {
    return bt::guarded([&] {
        BT_REQUIRE(p && ctx, "poisson: null argument");
        if (p->ctx == ctx) return;
        BT_REQUIRE(p->ctx->device == ctx->device, "poisson: the new context is on another device");
        // the old context's queued work first; its captured V-cycle is its own
        BT_CUDA(cudaStreamSynchronize(p->ctx->stream));
        bt::drop_graphs(p);
        p->ctx = ctx;
    });
}
