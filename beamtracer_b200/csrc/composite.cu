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

// The Boltzmann species at the nodes with an equation of their own (own[k] != 0):
// e = a exp(min(-s (phi - up) / T, 50)); r += s e and reaction = e / T there, 0 elsewhere
__global__ void boltzmann_terms(i64 n, const uint8_t *__restrict__ own, const double *__restrict__ phi,
                                double amplitude, double temperature, double up, double sign,
                                double *__restrict__ r, double *__restrict__ reaction) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!own[k]) {
        reaction[k] = 0.0;
        return;
    }
    const double e = amplitude * exp(fmin(-sign * (phi[k] - up) / temperature, 50.0));
    r[k] += sign * e;
    reaction[k] = e / temperature;
}

// y = own ? base + y - reaction x : 0 (the residual of a Newton step's correction)
__global__ void newton_residual(i64 n, const uint8_t *__restrict__ own, const double *__restrict__ base,
                                const double *__restrict__ reaction, const double *__restrict__ x,
                                double *__restrict__ y) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    y[k] = own[k] ? base[k] + y[k] - reaction[k] * x[k] : 0.0;
}

}  // namespace
}  // namespace bt

extern "C" int bt_newton_residual(bt_ctx *ctx, int64_t n, const uint8_t *own, const double *base,
                                  const double *reaction, const double *x, double *y) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && n >= 0, "newton residual: bad argument");
        if (n == 0) return;
        BT_REQUIRE(own && base && reaction && x && y, "newton residual: null array");
        BT_LAUNCH(ctx, bt::newton_residual, bt::blocks_for(n, 256), 256, 0, ctx->stream, n, own, base,
                  reaction, x, y);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_boltzmann_terms(bt_ctx *ctx, int64_t n, const uint8_t *own, const double *phi,
                                  double amplitude, double temperature, double up, int32_t sign,
                                  double *r, double *reaction) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && n >= 0, "boltzmann terms: bad argument");
        BT_REQUIRE(temperature > 0.0 && (sign == 1 || sign == -1),
                   "boltzmann terms: the temperature must be positive and the sign +-1");
        if (n == 0) return;
        BT_REQUIRE(own && phi && r && reaction, "boltzmann terms: null array");
        BT_LAUNCH(ctx, bt::boltzmann_terms, bt::blocks_for(n, 256), 256, 0, ctx->stream, n, own, phi,
                  amplitude, temperature, up, (double)sign, r, reaction);
        BT_CHECK_LAUNCH();
    });
}

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
