// The FP64 pipe's measured peak: independent chains of fused multiply-adds on every SM,
// timed with CUDA events on the context's stream -- the denominator of the tracer's FP64
// roofline (there is no tensor-core FP64 path in this workload, and no measured FP64 figure
// beside the copy bandwidth and the bf16 GEMM the pool measures).
#include "common.cuh"

namespace bt {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kPeakChains = 8;  // independent chains a thread: enough to cover the latency

__global__ void __launch_bounds__(kPeakThreads) fma_chains(int iterations, double a, double b,
                                                          double *__restrict__ out) {
    double x[kPeakChains];
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int c = 0; c < kPeakChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) s += x[c];
    out[(i64)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace bt

extern "C" int bt_measure_fp64_peak(bt_ctx *ctx, double *tflops) {
    using namespace bt;
    return guarded([&] {
        BT_REQUIRE(ctx && tflops, "fp64 peak: null argument");
        const int blocks = ctx->num_sms * 8;
        double *out = ctx->measure.as<double>((size_t)blocks * kPeakThreads);
        const int iterations = 4096;
        cudaEvent_t start, stop;
        BT_CUDA(cudaEventCreate(&start));
        BT_CUDA(cudaEventCreate(&stop));
        float best = 0.0f;
        for (int rep = 0; rep < 4; ++rep) {  // the first launch warms up; the fastest counts
            BT_CUDA(cudaEventRecord(start, ctx->stream));
            BT_LAUNCH(ctx, fma_chains, blocks, kPeakThreads, 0, ctx->stream, iterations,
                      0.999999, 1e-7, out);
            BT_CUDA(cudaEventRecord(stop, ctx->stream));
            BT_CUDA(cudaEventSynchronize(stop));
            float ms = 0.0f;
            BT_CUDA(cudaEventElapsedTime(&ms, start, stop));
            if (rep > 0 && (best == 0.0f || ms < best)) best = ms;
        }
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        BT_CHECK_LAUNCH();
        const double flops = 2.0 * (double)blocks * kPeakThreads * kPeakChains * iterations;
        *tflops = flops / (best * 1e-3) / 1e12;
    });
}
