// The per-iteration updates of the Vlasov iteration on the device: the node charges to a
// density (tracer.py:700-705: over the node volumes), the space-charge compensation
// (vlasov.py:176-184: a factor per node column), the linear mixing
// (vlasov.py:391-397: (1 - w) rho + w deposit, or the deposit itself in iteration 0), and
// the largest changes the convergence tests read (vlasov.py:362-366).
#include "common.cuh"

namespace bt {
namespace {

constexpr int kReduceThreads = 256;
constexpr int kReduceBlocks = 296;  // 2 per SM of a B200

// The larger of two values, NaN if either is NaN (fmax would drop a NaN, and a NaN
// potential or density would then read as converged; the reference's np.max keeps it).
__device__ __forceinline__ double max_nan(double m, double v) {
    return (v > m || v != v) ? v : m;
}

__device__ __forceinline__ double block_max(double v, double *part) {
    part[threadIdx.x] = v;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] = max_nan(part[threadIdx.x], part[threadIdx.x + off]);
        __syncthreads();
    }
    return part[0];
}

// rho <- mixed density; per block: max |rho_new - rho_old| and max |rho_new|
__global__ void mix(const double *__restrict__ charge, const double *__restrict__ volumes,
                    const double *__restrict__ column, i64 nx, i64 ny, double w, int first,
                    double *__restrict__ rho, double *__restrict__ partial) {
    __shared__ double part[kReduceThreads];
    const i64 n = nx * ny;
    double dmax = 0.0, rmax = 0.0;
    for (i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (i64)gridDim.x * blockDim.x) {
        double deposit = charge[f] / volumes[f];
        if (column) deposit = deposit * column[f / ny];
        const double old = rho[f];
        const double next = first ? deposit : (1.0 - w) * old + w * deposit;
        rho[f] = next;
        dmax = max_nan(dmax, fabs(next - old));
        rmax = max_nan(rmax, fabs(next));
    }
    const double a = block_max(dmax, part);
    __syncthreads();
    const double b = block_max(rmax, part);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

__global__ void diff_max(const double *__restrict__ a, const double *__restrict__ b, i64 n,
                         double *__restrict__ partial) {
    __shared__ double part[kReduceThreads];
    double m = 0.0;
    for (i64 f = (i64)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (i64)gridDim.x * blockDim.x)
        m = max_nan(m, fabs(a[f] - b[f]));
    const double r = block_max(m, part);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void finish_max(const double *__restrict__ partial, int blocks, int stride,
                           double *__restrict__ out) {
    __shared__ double part[kReduceThreads];
    for (int c = 0; c < stride; ++c) {
        double m = 0.0;
        for (int bi = threadIdx.x; bi < blocks; bi += blockDim.x) m = max_nan(m, partial[bi * stride + c]);
        const double r = block_max(m, part);
        if (threadIdx.x == 0) out[c] = r;
        __syncthreads();
    }
}

}  // namespace
}  // namespace bt

extern "C" int bt_vlasov_mix(bt_ctx *ctx, const double *charge, const double *volumes,
                             const double *column_factor, int64_t nx, int64_t ny,
                             double relaxation, int32_t first, double *rho, double *stats) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && charge && volumes && rho && stats, "vlasov mix: null argument");
        BT_REQUIRE(nx > 0 && ny > 0, "vlasov mix: empty mesh");
        double *partial = ctx->reduce_partial.as<double>(2 * bt::kReduceBlocks);
        bt::Timed timed(ctx, "vlasov_mix");
        BT_LAUNCH(ctx, bt::mix, bt::kReduceBlocks, bt::kReduceThreads, 0, ctx->stream, charge, volumes, column_factor, nx, ny, relaxation, first, rho, partial);
        BT_LAUNCH(ctx, bt::finish_max, 1, bt::kReduceThreads, 0, ctx->stream, partial, bt::kReduceBlocks, 2, stats);
        BT_CHECK_LAUNCH();
    });
}

extern "C" int bt_max_abs_diff(bt_ctx *ctx, const double *a, const double *b, int64_t n,
                               double *out) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && a && b && out, "max abs diff: null argument");
        double *partial = ctx->reduce_partial.as<double>(2 * bt::kReduceBlocks);
        BT_LAUNCH(ctx, bt::diff_max, bt::kReduceBlocks, bt::kReduceThreads, 0, ctx->stream, a, b, n, partial);
        BT_LAUNCH(ctx, bt::finish_max, 1, bt::kReduceThreads, 0, ctx->stream, partial, bt::kReduceBlocks, 1, out);
        BT_CHECK_LAUNCH();
    });
}
