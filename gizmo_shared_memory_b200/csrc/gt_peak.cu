// CUDA-core throughput probe: the FP32 and FP64 FMA rates the walk's roofline fraction is quoted
// against.  Each thread runs 8 independent FMA chains for `iters` steps on registers only; the
// grid is 8 resident blocks of 256 threads per SM.  No reference counterpart.
#include "gt_internal.cuh"

namespace gt {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T* out, int iters, T a, T b) {
    T v0 = (T)threadIdx.x, v1 = v0 + (T)1, v2 = v0 + (T)2, v3 = v0 + (T)3;
    T v4 = v0 + (T)4, v5 = v0 + (T)5, v6 = v0 + (T)6, v7 = v0 + (T)7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            v0 = v0 * a + b; v1 = v1 * a + b; v2 = v2 * a + b; v3 = v3 * a + b;
            v4 = v4 * a + b; v5 = v5 * a + b; v6 = v6 * a + b; v7 = v7 * a + b;
        }
    }
    const T s = v0 + v1 + v2 + v3 + v4 + v5 + v6 + v7;
    if (s == (T)-1.2345) out[0] = s;  // keeps the chains alive; never true for these inputs
}

template <typename T>
double probe(gt_context* ctx, int iters) {
    T* out = (T*)scratch(ctx, kSlotPartials, 64);
    const int blocks = ctx->num_sms * 8;
    fma_probe_kernel<T><<<blocks, 256, 0, ctx->stream>>>(out, 16, (T)0.999999, (T)1e-7);  // warm-up
    check_launch(ctx, "fma_probe_kernel");
    check_cuda(cudaEventRecord(ctx->ev0, ctx->stream), "event");
    fma_probe_kernel<T><<<blocks, 256, 0, ctx->stream>>>(out, iters, (T)0.999999, (T)1e-7);
    check_launch(ctx, "fma_probe_kernel");
    check_cuda(cudaEventRecord(ctx->ev1, ctx->stream), "event");
    check_cuda(cudaEventSynchronize(ctx->ev1), "sync");
    float ms = 0;
    check_cuda(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1), "elapsed");
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

void run_peaks(gt_context* ctx, double* fp32, double* fp64) {
    if (fp32) *fp32 = probe<float>(ctx, 4096);
    if (fp64) *fp64 = probe<double>(ctx, 1024);
}

}  // namespace gt
