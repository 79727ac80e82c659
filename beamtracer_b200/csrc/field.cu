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

// The edge between nodes e - 1 and e (1 <= e <= n - 1) of the line starting at `base`.
__device__ double interior_edge(const Line &L, i64 base, i64 e) {
    const i64 s = L.stride;
    const i64 ia = base + (e - 1) * s, ib = base + e * s;
    const double a = L.phi[ia], b = L.phi[ib];
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
        const double phi0 = has0 ? L.phi[base + (e - 2) * s] : 0.0;
        const double phi3 = has3 ? L.phi[base + (e + 1) * s] : 0.0;
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

__device__ double edge(const Line &L, i64 base, i64 e, int sym_lo, int sym_hi) {
    const i64 n = L.n;
    if (e == 0) {
        const double first = interior_edge(L, base, 1);
        return sym_lo ? -first : 2.0 * first - interior_edge(L, base, 2);
    }
    if (e == n) {
        const double first = interior_edge(L, base, n - 1);
        return sym_hi ? -first : 2.0 * first - interior_edge(L, base, n - 2);
    }
    return interior_edge(L, base, e);
}

__global__ void edge_field_x(Line L, i64 ny, int sym_lo, int sym_hi, double *__restrict__ fx) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 total = (L.n + 1) * ny;
    if (t >= total) return;
    const i64 e = t / ny, j = t - e * ny;
    fx[t] = edge(L, j, e, sym_lo, sym_hi);
}

__global__ void edge_field_y(Line L, i64 nx, int sym_lo, int sym_hi, double *__restrict__ fy) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const i64 m = L.n + 1;  // ny + 1
    if (t >= nx * m) return;
    const i64 i = t / m, e = t - i * m;
    fy[t] = edge(L, i * L.n, e, sym_lo, sym_hi);
}

}  // namespace
}  // namespace bt

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
