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

// -- Anderson mixing (vlasov.py:127-173) ------------------------------------------------------
//
// Type II: from the last m + 1 iterates x_k and residuals f_k = G(x_k) - x_k, the m
// differences dX, dF of consecutive ones, gamma = argmin |f - dF gamma| and
// x + w f - (dX + w dF) gamma.  The least-squares problem is solved as NumPy's lstsq
// solves it, up to rounding: dF = Q R by classical Gram-Schmidt applied twice (each pass a
// grid-wide sum of fixed order: per-block partials, added in block order by the last block
// to finish), then R = U S V^T by one-sided Jacobi in one thread, the singular values below
// rcond of the largest left out, gamma = V S^+ U^T (Q^T f).  The iterates live in two ring
// buffers of depth + 1 rows on the device; only scalars are read back by nobody: the loop
// stays on the device.

constexpr int kMaxDepth = 16;
constexpr int kSums = kMaxDepth + 1;  // dots with up to kMaxDepth columns, and a norm

struct AndersonWork {
    double part[kReduceBlocks][kSums];  // per-block partial sums of a pass
    double coef[kMaxDepth];             // the last pass's projection coefficients
    double r[kMaxDepth][kMaxDepth];     // R, r[k][j] = R_kj (upper triangular)
    double qf[kMaxDepth];               // Q^T f
    double gamma[kMaxDepth];
    double scale;                       // 1 / R_jj of the column last normalised (0: none)
    unsigned int done;                  // blocks of the current pass that finished
};

struct Slots {
    int s[kMaxDepth + 1];  // ring rows of the iterates, oldest first
};

// The stored iterate and residual: x = rho, f = deposit - x (deposit = the node charges
// over the volumes -- or the density itself without volumes -- times the compensation
// factor of the node's column).
__global__ void anderson_store(const double *__restrict__ charge,
                               const double *__restrict__ volumes,
                               const double *__restrict__ column, i64 nx, i64 ny,
                               const double *__restrict__ rho, double *__restrict__ x_row,
                               double *__restrict__ f_row) {
    const i64 n = nx * ny;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        double deposit = volumes ? charge[i] / volumes[i] : charge[i];
        if (column) deposit = deposit * column[i / ny];
        const double x = rho[i];
        x_row[i] = x;
        f_row[i] = deposit - x;
    }
}

enum GsMode { kFresh = 0, kProject = 1, kRhs = 2 };

// One Gram-Schmidt pass over column j of dF (rows fa, fb: dF_j = fb - fa) held in q[j]:
// kFresh: v = fb - fa (and Q_{j-1} scaled by its 1 / R); kProject: v = q[j] - Q coef;
// kRhs: v = f (and Q_{j-1} scaled), not stored.  Sums Q_k . v (k < j) and v . v; the last
// block to finish adds the blocks' partials in block order and, per `final`, records them.
__global__ void gs_pass(i64 n, int j, int mode, int final_pass, const double *__restrict__ fa,
                        const double *__restrict__ fb, double *__restrict__ q,
                        AndersonWork *__restrict__ w) {
    __shared__ double warp_sums[kReduceThreads / 32][kSums];
    __shared__ bool last;
    double acc[kSums];
#pragma unroll
    for (int k = 0; k < kSums; ++k) acc[k] = 0.0;
    const bool scale_prev = (mode != kProject) && j > 0;
    const double prev_scale = scale_prev ? w->scale : 1.0;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        if (scale_prev) q[(i64)(j - 1) * n + i] *= prev_scale;
        double v;
        if (mode == kFresh) {
            v = fb[i] - fa[i];
        } else if (mode == kRhs) {
            v = fb[i];
        } else {
            v = q[(i64)j * n + i];
#pragma unroll
            for (int k = 0; k < kMaxDepth; ++k)
                if (k < j) v -= w->coef[k] * q[(i64)k * n + i];
        }
        if (mode != kRhs) q[(i64)j * n + i] = v;
#pragma unroll
        for (int k = 0; k < kMaxDepth; ++k)
            if (k < j) acc[k] += q[(i64)k * n + i] * v;
        acc[kMaxDepth] += v * v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kSums; ++k) {
        double a = acc[k];
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) warp_sums[warp][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < kSums) {
        double a = 0.0;
        for (int wi = 0; wi < kReduceThreads / 32; ++wi) a += warp_sums[wi][threadIdx.x];
        w->part[blockIdx.x][threadIdx.x] = a;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&w->done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int k = threadIdx.x;
    if (k < kSums) {
        double total = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) total += w->part[b][k];
        if (mode == kRhs) {
            if (k < j) w->qf[k] = total;
        } else if (k < j) {
            w->coef[k] = total;
            if (mode == kFresh) w->r[k][j] = total;
            else if (!final_pass) w->r[k][j] += total;
        } else if (k == kMaxDepth && final_pass) {
            const double norm = sqrt(total);
            w->r[j][j] = norm;
            w->scale = norm > 0.0 ? 1.0 / norm : 0.0;  // a zero column stays zero
        }
    }
    if (threadIdx.x == 0) w->done = 0;
}

// gamma = V S^+ U^T qf from R = U S V^T (one-sided Jacobi on R's m columns), singular
// values at most rcond times the largest left out.  One thread; m <= kMaxDepth.
__global__ void anderson_solve(int m, double rcond, AndersonWork *__restrict__ w) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a[kMaxDepth][kMaxDepth];  // a[c][r]: column c of the rotated R
    double v[kMaxDepth][kMaxDepth];
    for (int c = 0; c < m; ++c)
        for (int r = 0; r < m; ++r) {
            a[c][r] = r <= c ? w->r[r][c] : 0.0;
            v[c][r] = r == c ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        bool rotated = false;
        for (int p = 0; p < m - 1; ++p)
            for (int qc = p + 1; qc < m; ++qc) {
                double alpha = 0.0, beta = 0.0, g = 0.0;
                for (int r = 0; r < m; ++r) {
                    alpha += a[p][r] * a[p][r];
                    beta += a[qc][r] * a[qc][r];
                    g += a[p][r] * a[qc][r];
                }
                if (g == 0.0 || fabs(g) <= 1e-15 * sqrt(alpha * beta)) continue;
                rotated = true;
                const double zeta = (beta - alpha) / (2.0 * g);
                const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                for (int r = 0; r < m; ++r) {
                    const double ap = a[p][r], aq = a[qc][r];
                    a[p][r] = c * ap - s * aq;
                    a[qc][r] = s * ap + c * aq;
                    const double vp = v[p][r], vq = v[qc][r];
                    v[p][r] = c * vp - s * vq;
                    v[qc][r] = s * vp + c * vq;
                }
            }
        if (!rotated) break;
    }
    double sv[kMaxDepth], smax = 0.0;
    for (int c = 0; c < m; ++c) {
        double ss = 0.0;
        for (int r = 0; r < m; ++r) ss += a[c][r] * a[c][r];
        sv[c] = sqrt(ss);
        smax = fmax(smax, sv[c]);
    }
    double gamma[kMaxDepth];
    for (int r = 0; r < m; ++r) gamma[r] = 0.0;
    for (int c = 0; c < m; ++c) {
        if (!(sv[c] > rcond * smax)) continue;
        double ut_qf = 0.0;  // (U^T qf)_c with U_c = a_c / s_c
        for (int r = 0; r < m; ++r) ut_qf += a[c][r] * w->qf[r];
        const double coefficient = ut_qf / (sv[c] * sv[c]);
        for (int r = 0; r < m; ++r) gamma[r] += v[c][r] * coefficient;
    }
    for (int r = 0; r < m; ++r) w->gamma[r] = gamma[r];
}

// rho <- x + w f - sum_j gamma_j (dX_j + w dF_j); per block max |new - x| and max |new|.
__global__ void anderson_apply(i64 n, int m, Slots slots, double omega,
                               const double *__restrict__ xs, const double *__restrict__ fs,
                               const AndersonWork *__restrict__ w, double *__restrict__ rho,
                               double *__restrict__ partial) {
    __shared__ double part[kReduceThreads];
    const int newest = slots.s[m];
    double dmax = 0.0, rmax = 0.0;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (i64)gridDim.x * blockDim.x) {
        const double x = xs[(i64)newest * n + i];
        const double f = fs[(i64)newest * n + i];
        double next = x + omega * f;
        if (m > 0) {
            double corr = 0.0;
            for (int j = 0; j < m; ++j) {
                const i64 a = (i64)slots.s[j] * n + i, b = (i64)slots.s[j + 1] * n + i;
                corr += ((xs[b] - xs[a]) + omega * (fs[b] - fs[a])) * w->gamma[j];
            }
            next = next - corr;
        }
        rho[i] = next;
        dmax = max_nan(dmax, fabs(next - x));
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

}  // namespace
}  // namespace bt

extern "C" int bt_anderson_mix(bt_ctx *ctx, const double *charge, const double *volumes,
                               const double *column_factor, int64_t nx, int64_t ny,
                               int32_t depth, int32_t count, int32_t head, double relaxation,
                               double *xs, double *fs, double *q, double *rho, double *stats) {
    using namespace bt;
    return guarded([&] {
        BT_REQUIRE(ctx && charge && xs && fs && q && rho && stats, "anderson mix: null argument");
        BT_REQUIRE(nx > 0 && ny > 0, "anderson mix: empty mesh");
        BT_REQUIRE(depth >= 1 && depth <= kMaxDepth, "anderson mix: depth must be 1 to 16");
        BT_REQUIRE(count >= 1 && count <= depth + 1, "anderson mix: count must be 1 to depth + 1");
        BT_REQUIRE(head >= 0 && head <= depth, "anderson mix: head outside the ring");
        const i64 n = nx * ny;
        const int rows = depth + 1;
        const int m = count - 1;
        Slots slots{};
        for (int c = 0; c < count; ++c) slots.s[c] = (head - (count - 1) + c + rows) % rows;
        cudaStream_t st = ctx->stream;
        AndersonWork *w = ctx->anderson.as<AndersonWork>(1);
        double *partial = ctx->reduce_partial.as<double>(2 * kReduceBlocks);
        const unsigned grid = (unsigned)std::min<i64>(kReduceBlocks, std::max<i64>(1, blocks_for(n, kReduceThreads)));
        Timed timed(ctx, "anderson_mix");
        BT_LAUNCH(ctx, anderson_store, kReduceBlocks, kReduceThreads, 0, st, charge, volumes,
                  column_factor, nx, ny, rho, xs + (i64)head * n, fs + (i64)head * n);
        if (m > 0) {
            BT_CUDA(cudaMemsetAsync(&w->done, 0, sizeof(unsigned int), st));
            for (int j = 0; j < m; ++j) {
                const double *fa = fs + (i64)slots.s[j] * n, *fb = fs + (i64)slots.s[j + 1] * n;
                BT_LAUNCH(ctx, gs_pass, grid, kReduceThreads, 0, st, n, j, (int)kFresh,
                          (int)(j == 0), fa, fb, q, w);
                if (j > 0) {
                    BT_LAUNCH(ctx, gs_pass, grid, kReduceThreads, 0, st, n, j, (int)kProject, 0,
                              fa, fb, q, w);
                    BT_LAUNCH(ctx, gs_pass, grid, kReduceThreads, 0, st, n, j, (int)kProject, 1,
                              fa, fb, q, w);
                }
            }
            BT_LAUNCH(ctx, gs_pass, grid, kReduceThreads, 0, st, n, m, (int)kRhs, 0,
                      (const double *)nullptr, fs + (i64)head * n, q, w);
            BT_LAUNCH(ctx, anderson_solve, 1, 32, 0, st, m, 1e-10, w);
        }
        BT_LAUNCH(ctx, anderson_apply, kReduceBlocks, kReduceThreads, 0, st, n, m, slots,
                  relaxation, (const double *)xs, (const double *)fs, (const AndersonWork *)w,
                  rho, partial);
        BT_LAUNCH(ctx, finish_max, 1, kReduceThreads, 0, st, partial, kReduceBlocks, 2, stats);
        BT_CHECK_LAUNCH();
    });
}

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
