// The sparse maps of the composite mesh of refined boxes: a potential from the composite
// nodes to a patch's nodes (and to the wider mesh of its field, whose margin interpolates
// the coarser patches), the patches' node charges to the composite nodes, and the hanging
// nodes from the nodes they hang from.  Every map is a row-compressed matrix applied in its
// stored order, so its sums are the same bits on every run (no atomics).

#include <cstdint>

#include "bt200.h"
#include "common.cuh"

namespace bt {
namespace {

// y[out(r)] = (accumulate ? y[out(r)] : c[r]) + sum_e val[e] x[col[e]], e over row r in order
__global__ void csr_apply(i64 rows, const i64 *__restrict__ out_rows, const i64 *__restrict__ ptr,
                          const i64 *__restrict__ col, const double *__restrict__ val,
                          const double *__restrict__ constant, int accumulate,
                          const double *x, double *y) {
    const i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const i64 o = out_rows ? out_rows[r] : r;
    double s = accumulate ? y[o] : (constant ? constant[r] : 0.0);
    for (i64 e = ptr[r], end = ptr[r + 1]; e < end; ++e) s += val[e] * x[col[e]];
    y[o] = s;
}

}  // namespace
}  // namespace bt

extern "C" int bt_csr_apply(bt_ctx *ctx, int64_t rows, const int64_t *out_rows,
                            const int64_t *row_ptr, const int64_t *col, const double *val,
                            const double *constant, int32_t accumulate, const double *x,
                            double *y) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && rows >= 0, "csr apply: bad argument");
        if (rows == 0) return;
        BT_REQUIRE(row_ptr && y && (x || !col), "csr apply: null array");
        BT_LAUNCH(ctx, bt::csr_apply, bt::blocks_for(rows, 256), 256, 0, ctx->stream, rows, out_rows, row_ptr,
                  col, val, constant, accumulate, x, y);
        BT_CHECK_LAUNCH();
    });
}
