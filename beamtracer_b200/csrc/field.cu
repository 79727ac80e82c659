// The staggered edge field of a potential (solver/fields.py:18-67, 116-152): E_x on the
// (nx + 1, ny) edges along x and E_y on the (nx, ny + 1) edges along y, the difference
// over the edge's length, over the bracketed distance to an electrode surface next to
// one, extrapolated from the single surface across an edge inside an electrode, and
// mirrored or extrapolated linearly on the faces.  Same expressions as the reference,
// so the same bits.
#include "common.cuh"

namespace bt {
namespace {

struct Line {
    const double *phi;
    const int32_t *solid;
    const uint8_t *near;
    const double *dist_lo;  // the distance towards -axis
    const double *dist_hi;  // towards +axis
    const double *len;      // (n - 1,) edge lengths along the axis, or NULL for h
    double h;
    i64 n;       // nodes along the axis
    i64 stride;  // of the axis in the (nx, ny) arrays
};

__device__ __forceinline__ double edge_len(const Line &L, i64 t) {  // edge t .. t + 1
    return L.len ? L.len[t] : L.h;
}

// The potential at a node index: the array itself for the field, or a unit vector at one
// node for the field's transpose (every edge is linear in the potential and its branches
// depend on the node classes only, so evaluating it on a unit vector gives that node's
// coefficient).
struct PhiArray {
    const double *phi;
    __device__ __forceinline__ double operator()(i64 idx) const { return phi[idx]; }
};
struct PhiUnit {
    i64 node;
    __device__ __forceinline__ double operator()(i64 idx) const { return idx == node ? 1.0 : 0.0; }
};

// The edge between nodes e - 1 and e (1 <= e <= n - 1) of the line starting at `base`.
template <class Phi>
__device__ double interior_edge(const Line &L, const Phi &phi, i64 base, i64 e) {
    const i64 s = L.stride;
    const i64 ia = base + (e - 1) * s, ib = base + e * s;
    const double a = phi(ia), b = phi(ib);
    const double h = edge_len(L, e - 1);
    const bool sa = L.solid[ia] >= 0, sb = L.solid[ib] >= 0;
    const bool na = L.near[ia] != 0, nb = L.near[ib] != 0;
    double field = (a - b) / h;
    if (na && sb) field = (a - b) / (L.dist_hi[ia] * h);
    if (nb && sa) field = (a - b) / (L.dist_lo[ib] * h);
    if (sa && sb) {
        const bool has0 = e >= 2, has3 = e + 1 <= L.n - 1;
        const bool near0 = has0 && L.near[base + (e - 2) * s] != 0;
        const bool near3 = has3 && L.near[base + (e + 1) * s] != 0;
        const double phi0 = has0 ? phi(base + (e - 2) * s) : 0.0;
        const double phi3 = has3 ? phi(base + (e + 1) * s) : 0.0;
        const double d0 = has0 ? L.dist_hi[base + (e - 2) * s] : 1.0;
        const double d3 = has3 ? L.dist_lo[base + (e + 1) * s] : 1.0;
        const double h_before = e - 1 >= 1 ? edge_len(L, e - 2) : 1.0;
        const double h_after = e - 1 < L.n - 2 ? edge_len(L, e) : 1.0;
        double inside = 0.0;
        if (near0 && !near3) inside = (phi0 - a) / (d0 * h_before);
        if (near3 && !near0) inside = (b - phi3) / (d3 * h_after);
        field = inside;
    }
    return field;
}

template <class Phi>
__device__ double edge(const Line &L, const Phi &phi, i64 base, i64 e, int sym_lo, int sym_hi) {
    const i64 n = L.n;
    if (e == 0) {
        const double first = interior_edge(L, phi, base, 1);
        return sym_lo ? -first : 2.0 * first - interior_edge(L, phi, base, 2);
    }
    if (e == n) {
        const double first = interior_edge(L, phi, base, n - 1);
        return sym_hi ? -first : 2.0 * first - interior_edge(L, phi, base, n - 2);
    }
    return interior_edge(L, phi, base, e);
}

// The transpose of the field along one line at node k of the line (its index `node`):
// sum over the edges that read the node -- interior edges k - 1 .. k + 2, and the face
// edges, which read the first or last four nodes -- of the edge's adjoint times the
// node's coefficient in it.
__device__ double line_adjoint(const Line &L, const double *__restrict__ bar, i64 bar_stride,
                               i64 base, i64 k, i64 node, int sym_lo, int sym_hi) {
    const PhiUnit unit{node};
    double sum = 0.0;
    const i64 lo = max((i64)1, k - 1), hi = min(L.n - 1, k + 2);
    for (i64 e = lo; e <= hi; ++e) sum += bar[e * bar_stride] * edge(L, unit, base, e, sym_lo, sym_hi);
    if (k <= 3) sum += bar[0] * edge(L, unit, base, 0, sym_lo, sym_hi);
    if (k >= L.n - 4) sum += bar[L.n * bar_stride] * edge(L, unit, base, L.n, sym_lo, sym_hi);
    return sum;
}

// phi_bar = D^T (fx_bar, fy_bar): the potential's adjoint from the edge fields' (one
// thread per node, the sums in a fixed order).
__global__ void edge_field_adjoint(Line lx, Line ly, i64 nx, i64 ny, int sx_lo, int sx_hi,
                                   int sy_lo, int sy_hi, const double *__restrict__ fx_bar,
                                   const double *__restrict__ fy_bar,
                                   double *__restrict__ phi_bar) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nx * ny) return;
    const i64 i = t / ny, j = t - i * ny;
    // along x: the line of column j, fx_bar[e, j] at e * ny + j
    const double ax = line_adjoint(lx, fx_bar + j, ny, j, i, t, sx_lo, sx_hi);
    // along y: the line of row i, fy_bar[i, e] at i * (ny + 1) + e
    const double ay = line_adjoint(ly, fy_bar + i * (ny + 1), 1, i * ny, j, t, sy_lo, sy_hi);
    phi_bar[t] = ax + ay;
}

__global__ void edge_field_x(Line L, i64 ny, int sym_lo, int sym_hi, double *__restrict__ fx) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 total = (L.n + 1) * ny;
    if (t >= total) return;
    const i64 e = t / ny, j = t - e * ny;
    fx[t] = edge(L, PhiArray{L.phi}, j, e, sym_lo, sym_hi);
}

__global__ void edge_field_y(Line L, i64 nx, int sym_lo, int sym_hi, double *__restrict__ fy) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 m = L.n + 1;  // ny + 1
    if (t >= nx * m) return;
    const i64 i = t / m, e = t - i * m;
    fy[t] = edge(L, PhiArray{L.phi}, i * L.n, e, sym_lo, sym_hi);
}

// The edges along one axis of a 3D mesh (n nodes along it, `stride` between them): edge e
// of the line through the other two coordinates (u, w), u over `count_u` values with line
// step `step_u`, w over `count_w` with step `step_w`; out (n + 1 edges, in the mesh's C
// order with the axis lengthened by one).
__global__ void edge_field_3d(Line L, i64 count_u, i64 step_u, i64 count_w, i64 step_w,
                              i64 out_u, i64 out_w, i64 out_e, int sym_lo, int sym_hi,
                              double *__restrict__ out) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 m = L.n + 1;
    if (t >= m * count_u * count_w) return;
    const i64 e = t % m, uw = t / m, u = uw / count_w, w = uw - u * count_w;
    out[u * out_u + w * out_w + e * out_e] =
        edge(L, PhiArray{L.phi}, u * step_u + w * step_w, e, sym_lo, sym_hi);
}

}  // namespace
}  // namespace bt

extern "C" int bt_edge_field_3d(bt_ctx *ctx, const double *phi, const int32_t *solid,
                                const uint8_t *near, const double *distance, int64_t nx,
                                int64_t ny, int64_t nz, double h,
                                const int32_t extrapolation[6], double *fx, double *fy,
                                double *fz) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && phi && solid && near && distance && fx && fy && fz && extrapolation,
                   "edge field 3d: null argument");
        BT_REQUIRE(nx >= 3 && ny >= 3 && nz >= 3, "edge field 3d: 3 nodes per axis at least");
        const i64 nn = nx * ny * nz;
        const int T = 256;
        // along x: lines (j, k), nodes i at stride ny nz; fx (nx + 1, ny, nz)
        bt::Line lx{phi, solid, near, distance, distance + nn, nullptr, h, nx, ny * nz};
        BT_LAUNCH(ctx, bt::edge_field_3d, bt::blocks_for((nx + 1) * ny * nz, T), T, 0, ctx->stream,
                  lx, ny, nz, nz, (i64)1, nz, (i64)1, ny * nz, extrapolation[0], extrapolation[1],
                  fx);
        // along y: lines (i, k), stride nz; fy (nx, ny + 1, nz)
        bt::Line ly{phi, solid, near, distance + 2 * nn, distance + 3 * nn, nullptr, h, ny, nz};
        BT_LAUNCH(ctx, bt::edge_field_3d, bt::blocks_for(nx * (ny + 1) * nz, T), T, 0, ctx->stream,
                  ly, nx, ny * nz, nz, (i64)1, (ny + 1) * nz, (i64)1, nz, extrapolation[2],
                  extrapolation[3], fy);
        // along z: lines (i, j), stride 1; fz (nx, ny, nz + 1)
        bt::Line lz{phi, solid, near, distance + 4 * nn, distance + 5 * nn, nullptr, h, nz, 1};
        BT_LAUNCH(ctx, bt::edge_field_3d, bt::blocks_for(nx * ny * (nz + 1), T), T, 0, ctx->stream,
                  lz, nx, ny * nz, ny, nz, ny * (nz + 1), nz + 1, (i64)1, extrapolation[4],
                  extrapolation[5], fz);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_edge_field(bt_ctx *ctx, const double *phi, const int32_t *solid,
                             const uint8_t *near, const double *distance, const double *dx,
                             int64_t nx, int64_t ny, double h, const int32_t extrapolation[4],
                             double *fx, double *fy) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && phi && solid && near && distance && fx && fy && extrapolation,
                   "edge field: null argument");
        BT_REQUIRE(nx >= 3 && ny >= 3, "edge field: the mesh needs at least 3 nodes per axis");
        const i64 nn = nx * ny;
        bt::Line lx{phi, solid, near, distance, distance + nn, dx, h, nx, ny};
        bt::Line ly{phi, solid, near, distance + 2 * nn, distance + 3 * nn, nullptr, h, ny, 1};
        bt::Timed timed(ctx, "edge_field");
        BT_LAUNCH(ctx, bt::edge_field_x, bt::blocks_for((nx + 1) * ny, 256), 256, 0, ctx->stream, lx, ny, extrapolation[0], extrapolation[1], fx);
        BT_LAUNCH(ctx, bt::edge_field_y, bt::blocks_for(nx * (ny + 1), 256), 256, 0, ctx->stream, ly, nx, extrapolation[2], extrapolation[3], fy);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_edge_field_adjoint(bt_ctx *ctx, const double *fx_bar, const double *fy_bar,
                                     const int32_t *solid, const uint8_t *near,
                                     const double *distance, const double *dx, int64_t nx,
                                     int64_t ny, double h, const int32_t extrapolation[4],
                                     double *phi_bar) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && fx_bar && fy_bar && solid && near && distance && phi_bar && extrapolation,
                   "edge field adjoint: null argument");
        BT_REQUIRE(nx >= 3 && ny >= 3, "edge field adjoint: the mesh needs at least 3 nodes per axis");
        const i64 nn = nx * ny;
        bt::Line lx{nullptr, solid, near, distance, distance + nn, dx, h, nx, ny};
        bt::Line ly{nullptr, solid, near, distance + 2 * nn, distance + 3 * nn, nullptr, h, ny, 1};
        BT_LAUNCH(ctx, bt::edge_field_adjoint, bt::blocks_for(nn, 256), 256, 0, ctx->stream, lx, ly,
                  nx, ny, extrapolation[0], extrapolation[1], extrapolation[2], extrapolation[3],
                  fx_bar, fy_bar, phi_bar);
        BT_CHECK_LAUNCH();
    });
}

// -- the surface field (solver/fields.py:324-377) --------------------------------------------

namespace bt {
namespace {

// One component at a node from its two edges (fields.py:323-338): the edge towards an
// electrode neighbour (the field at the surface), the larger of the two with electrodes on
// both sides, else their mean.
__device__ __forceinline__ double node_component(double low, double high, bool solid_low,
                                                 bool solid_high) {
    if (solid_low && solid_high) return fabs(low) >= fabs(high) ? low : high;
    if (solid_low) return low;
    if (solid_high) return high;
    return 0.5 * (low + high);
}

// |E| at every free node next to an electrode (NaN elsewhere) and that electrode (the first
// of the -x, +x, -y, +y neighbours that is one; -1 elsewhere); the largest |E| of each
// electrode by an atomic maximum on the bits of the non-negative doubles (order-free).
__global__ void surface_field(const double *__restrict__ fx, const double *__restrict__ fy,
                              const int32_t *__restrict__ solid, const uint8_t *__restrict__ near,
                              i64 nx, i64 ny, int n_electrodes, double *__restrict__ magnitude,
                              int32_t *__restrict__ electrode,
                              unsigned long long *__restrict__ largest) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nx * ny) return;
    const i64 i = t / ny, j = t - i * ny;
    const int32_t nb[4] = {i > 0 ? solid[t - ny] : -1, i < nx - 1 ? solid[t + ny] : -1,
                           j > 0 ? solid[t - 1] : -1, j < ny - 1 ? solid[t + 1] : -1};
    if (!near[t]) {
        magnitude[t] = __longlong_as_double(0x7ff8000000000000LL);  // a quiet NaN
        electrode[t] = -1;
        return;
    }
    const double ex = node_component(fx[t], fx[t + ny], nb[0] >= 0, nb[1] >= 0);
    const double ey = node_component(fy[i * (ny + 1) + j], fy[i * (ny + 1) + j + 1], nb[2] >= 0,
                                     nb[3] >= 0);
    const double m = hypot(ex, ey);
    int32_t e = -1;
    for (int q = 0; q < 4 && e < 0; ++q) e = nb[q];
    magnitude[t] = m;
    electrode[t] = e;
    if (largest && e >= 0 && e < n_electrodes && m == m)
        atomicMax(largest + e, (unsigned long long)__double_as_longlong(m));
}

}  // namespace
}  // namespace bt

extern "C" int bt_surface_field(bt_ctx *ctx, const double *fx, const double *fy,
                                const int32_t *solid, const uint8_t *near, int64_t nx, int64_t ny,
                                int32_t n_electrodes, double *magnitude, int32_t *electrode,
                                double *largest) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && fx && fy && solid && near && magnitude && electrode,
                   "surface field: null argument");
        BT_REQUIRE(nx >= 2 && ny >= 2, "surface field: the mesh needs at least 2 nodes per axis");
        BT_REQUIRE(n_electrodes >= 0, "surface field: negative electrode count");
        if (largest && n_electrodes > 0)
            BT_CUDA(cudaMemsetAsync(largest, 0, sizeof(double) * n_electrodes, ctx->stream));
        BT_LAUNCH(ctx, bt::surface_field, bt::blocks_for(nx * ny, 256), 256, 0, ctx->stream, fx,
                  fy, solid, near, nx, ny, n_electrodes, magnitude, electrode,
                  reinterpret_cast<unsigned long long *>(largest));
        BT_CHECK_LAUNCH();
    });
}
