// Electrode shapes on the device: the inside tests of the configuration's objects
// (config.py's rectangles, lines, circles, polygons, triangles and mirrored apertures; the
// reference's simgeometry tests, restated with closed boundaries) and the sub-cell table
// the tracer's electrode test reads (solver/tracer.py:1092-1114): for every sub-cell of the
// cells touching an electrode, the electrode holding its four corners and its centre, -1
// for none, -2 where they disagree.  The tests evaluate the same expressions in the same
// order as the host's NumPy ones, with the per-edge thresholds computed on the host, so the
// table is the host's bit for bit.
#include "common.cuh"

namespace bt {
namespace {

// The position along x of the fractional node index `index` (mesh.position_x).
__device__ double position_x(double index, double origin_x, double h, const double *nodes,
                             i64 n_nodes) {
    if (!nodes) return origin_x + h * index;
    i64 i = (i64)floor(index);
    if (i < 0) i = 0;
    if (i > n_nodes - 2) i = n_nodes - 2;
    return nodes[i] + (index - (double)i) * (nodes[i + 1] - nodes[i]);
}

__global__ void subcell_kernel(Shapes S, const i64 *__restrict__ ci, const i64 *__restrict__ cj,
                               i64 n_cells, double origin_x, double origin_y, double h,
                               const double *__restrict__ nodes, i64 n_nodes, int R,
                               i64 *__restrict__ out) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cells * R * R) return;
    const i64 k = t / (R * R);
    const int a = (int)(t / R % R), b = (int)(t % R);
    const double fi = (double)ci[k], fj = (double)cj[k];
    auto at = [&](double fa, double fb) {
        const double px = position_x(fi + fa, origin_x, h, nodes, n_nodes);
        const double py = origin_y + h * (fj + fb);
        return inside_solid(S, px, py);
    };
    const double r = (double)R;
    const i64 centre = at(((double)a + 0.5) / r, ((double)b + 0.5) / r);
    const bool same = at((double)a / r, (double)b / r) == centre &&
                      at((double)(a + 1) / r, (double)b / r) == centre &&
                      at((double)a / r, (double)(b + 1) / r) == centre &&
                      at((double)(a + 1) / r, (double)(b + 1) / r) == centre;
    out[t] = same ? centre : -2;
}

// The electrode of every node (solver/mesh.py _classify: the first holding it, or -1).
__global__ void node_solid(Shapes S, i64 nx, i64 ny, const double *__restrict__ x, double origin_y,
                           double h, int32_t *__restrict__ solid) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nx * ny) return;
    const i64 i = f / ny, j = f - i * ny;
    solid[f] = (int32_t)inside_solid(S, x[i], origin_y + h * (double)j);
}

// Per direction d (-x, +x, -y, +y): a free node whose neighbour there is an electrode is
// near it, and the surface's place on the edge between them is bracketed by eight
// bisections of that electrode's own inside test on a scale of 255 (never 0): the
// reference's _bracket, expression for expression.  distance (4, nx, ny) is 1 elsewhere.
__global__ void node_bracket(Shapes S, i64 nx, i64 ny, const double *__restrict__ x,
                             const double *__restrict__ dx, double origin_y, double h,
                             const int32_t *__restrict__ solid,
                             uint8_t *__restrict__ near, double *__restrict__ distance) {
    const i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nx * ny) return;
    const i64 i = f / ny, j = f - i * ny, n = nx * ny;
    bool any = false;
    for (int d = 0; d < 4; ++d) {
        const int axis = d >> 1, step = (d & 1) ? 1 : -1;
        const i64 i2 = i + (axis == 0 ? step : 0), j2 = j + (axis == 1 ? step : 0);
        double out = 1.0;
        const int32_t owner = (i2 >= 0 && i2 < nx && j2 >= 0 && j2 < ny) ? solid[i2 * ny + j2] : -1;
        if (solid[f] < 0 && owner >= 0) {
            any = true;
            const double x0 = x[i], y0 = origin_y + h * (double)j;
            const double length = axis == 1 ? h : dx[step > 0 ? i : i - 1];
            const double *p = S.params + S.offset[owner];
            const int kind = S.kind[owner];
            long long code = 128, bit = 128;
            for (int k = 0; k < 8; ++k) {
                const double offset = (double)step * length * (double)code / 255.0;
                const double px = axis == 0 ? x0 + offset : x0;
                const double py = axis == 1 ? y0 + offset : y0;
                if (shape_inside(kind, p, px, py)) code -= bit;
                bit >>= 1;
                code += bit;
            }
            if (code == 0) code = 1;
            out = (double)code / 255.0;
        }
        distance[(i64)d * n + f] = out;
    }
    near[f] = any ? 1 : 0;
}

}  // namespace
}  // namespace bt

extern "C" int bt_classify_mesh(bt_ctx *ctx, const bt_shapes *shapes, int64_t nx, int64_t ny,
                                const double *x, const double *dx, double origin_y, double h,
                                int32_t *solid, uint8_t *near, double *distance) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && shapes && x && dx && solid && near && distance,
                   "classify: null argument");
        BT_REQUIRE(nx >= 2 && ny >= 2, "classify: the mesh needs 2 x 2 nodes");
        BT_REQUIRE(shapes->count == 0 || (shapes->kind && shapes->offset && shapes->params),
                   "classify: null shape arrays");
        const bt::Shapes S{shapes->count, shapes->kind, shapes->offset, shapes->params};
        const int64_t n = nx * ny;
        BT_LAUNCH(ctx, bt::node_solid, bt::blocks_for(n, 256), 256, 0, ctx->stream, S, nx, ny, x,
                  origin_y, h, solid);
        BT_LAUNCH(ctx, bt::node_bracket, bt::blocks_for(n, 256), 256, 0, ctx->stream, S, nx, ny, x,
                  dx, origin_y, h, solid, near, distance);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_subcell_table(bt_ctx *ctx, const bt_shapes *shapes, const int64_t *ci,
                                const int64_t *cj, int64_t n_cells, double origin_x,
                                double origin_y, double h, const double *x_nodes,
                                int64_t n_x_nodes, int64_t refine, int64_t *out) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && shapes && out, "subcells: null argument");
        BT_REQUIRE(n_cells >= 0 && refine >= 1 && refine <= 64, "subcells: bad sizes");
        BT_REQUIRE(shapes->count >= 0 && (shapes->count == 0 || (shapes->kind && shapes->offset &&
                                                                 shapes->params)),
                   "subcells: null shape arrays");
        BT_REQUIRE(!x_nodes || n_x_nodes >= 2, "subcells: a graded axis needs its nodes");
        if (n_cells == 0) return;
        const bt::Shapes S{shapes->count, shapes->kind, shapes->offset, shapes->params};
        const int64_t total = n_cells * refine * refine;
        BT_LAUNCH(ctx, bt::subcell_kernel, bt::blocks_for(total, 256), 256, 0, ctx->stream, S, ci,
                  cj, n_cells, origin_x, origin_y, h, x_nodes, n_x_nodes, (int)refine, out);
        BT_CHECK_LAUNCH();
    });
}
