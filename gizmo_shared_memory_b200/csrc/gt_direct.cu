// O(N_targets * N) direct summation: the replacement for shmem::accel_brute (shmem/tree.cc:946-971)
// and for the reference's only CUDA kernel, accel_bruteforce_kernel (shmem/grav_cuda.cu:66-141).
//
// Each block holds 256 targets in registers and streams one contiguous chunk of the sources
// through shared memory in tiles of 256; the grid's second dimension splits the sources so that a
// few thousand targets (the error sample) still fill all 148 SMs.  Per-chunk partial sums go to a
// scratch array and a second kernel adds the chunks in a fixed order, so results are deterministic.
//   FP64: every operation in double, the pair rule of tree.cc:39-53 with zeta = 0 (kernel of the
//         larger softening, self and r == 0 skipped) -- the error oracle of the walk.
//   FP32: the pair offset is differenced in double and narrowed, everything after it is float
//         (grav_cuda.cu:108-134 without zeta terms or a periodic wrap).
#include <algorithm>

#include "gt_internal.cuh"

namespace gt {
namespace {

constexpr int kDirThreads = 256;
constexpr int kDirTile = 256;

__device__ __forceinline__ void spline_d(double r, double h, double& f, double& p) {
    const double hinv = 1.0 / h;
    const double u = r * hinv;
    if (u >= 1.0) {
        f = 1.0 / (r * r * r);
        p = -1.0 / r;
        return;
    }
    const double hinv3 = hinv * hinv * hinv;
    if (u < 0.5) {
        f = hinv3 * (10.666666666666667 + u * u * (32.0 * u - 38.4));
        p = hinv * (-2.8 + u * u * (5.333333333333333 + u * u * (6.4 * u - 9.6)));
    } else {
        f = hinv3 * (21.333333333333332 - 48.0 * u + 38.4 * u * u - 10.666666666666667 * u * u * u -
                     0.06666666666666667 / (u * u * u));
        p = hinv * (-3.2 + 0.06666666666666667 / u +
                    u * u * (10.666666666666667 + u * (-16.0 + u * (9.6 - 2.1333333333333333 * u))));
    }
}

__device__ __forceinline__ void spline_f(float r, float h, float& f, float& p) {
    const float hinv = 1.0f / h;
    const float u = r * hinv;
    if (u >= 1.0f) {
        const float ri = 1.0f / r;
        f = ri * ri * ri;
        p = -ri;
        return;
    }
    const float hinv3 = hinv * hinv * hinv;
    if (u < 0.5f) {
        f = hinv3 * (10.666666666666667f + u * u * (32.0f * u - 38.4f));
        p = hinv * (-2.8f + u * u * (5.333333333333333f + u * u * (6.4f * u - 9.6f)));
    } else {
        const float u3 = u * u * u;
        f = hinv3 * (21.333333333333332f - 48.0f * u + 38.4f * u * u - 10.666666666666667f * u3 -
                     0.06666666666666667f / u3);
        p = hinv * (-3.2f + 0.06666666666666667f / u +
                    u * u * (10.666666666666667f + u * (-16.0f + u * (9.6f - 2.1333333333333333f * u))));
    }
}

template <bool FP64>
__global__ void __launch_bounds__(kDirThreads)
direct_kernel(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
              const double* __restrict__ m, const double* __restrict__ soft, int64_t n,
              const uint32_t* __restrict__ targets, int64_t nt, int64_t chunk,
              double* __restrict__ partial) {
    __shared__ double shx[kDirTile], shy[kDirTile], shz[kDirTile], shm[kDirTile], shs[kDirTile];
    const int64_t t = (int64_t)blockIdx.x * kDirThreads + threadIdx.x;
    const bool live = t < nt;
    const int64_t self = live ? (int64_t)targets[t] : -1;
    const double px = live ? x[self] : 0.0, py = live ? y[self] : 0.0, pz = live ? z[self] : 0.0;
    const double ps = (live && soft) ? soft[self] : 0.0;
    const int64_t s0 = (int64_t)blockIdx.y * chunk, s1 = min(n, s0 + chunk);
    double ax = 0, ay = 0, az = 0, ap = 0;
    float fx = 0, fy = 0, fz = 0, fp = 0;
    for (int64_t base = s0; base < s1; base += kDirTile) {
        const int64_t q = base + threadIdx.x;
        if (q < s1) {
            shx[threadIdx.x] = x[q]; shy[threadIdx.x] = y[q]; shz[threadIdx.x] = z[q];
            shm[threadIdx.x] = m[q];
            shs[threadIdx.x] = soft ? soft[q] : 0.0;
        }
        __syncthreads();
        const int nq = (int)min((int64_t)kDirTile, s1 - base);
        if (live) {
            for (int k = 0; k < nq; ++k) {
                if (base + k == self) continue;
                const double ox = shx[k] - px, oy = shy[k] - py, oz = shz[k] - pz;
                if (FP64) {
                    const double r = sqrt(ox * ox + oy * oy + oz * oz);
                    if (r <= 0) continue;
                    const double e = fmax(fmax(ps, shs[k]), 1e-300);
                    double f, p;
                    spline_d(r, e, f, p);
                    const double mf = shm[k] * f;
                    ax += ox * mf; ay += oy * mf; az += oz * mf;
                    ap += shm[k] * p;
                } else {
                    const float dx = (float)ox, dy = (float)oy, dz = (float)oz;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 <= 0.0f) continue;
                    const float r = sqrtf(r2);
                    float e = fmaxf((float)ps, (float)shs[k]);
                    if (!(e > 0.0f)) e = 1e-30f;
                    float f, p;
                    spline_f(r, e, f, p);
                    const float mf = (float)shm[k] * f;
                    fx += dx * mf; fy += dy * mf; fz += dz * mf;
                    fp += (float)shm[k] * p;
                }
            }
        }
        __syncthreads();
    }
    if (live) {
        double* P = partial + (int64_t)blockIdx.y * 4 * nt;
        P[t] = FP64 ? ax : (double)fx;
        P[nt + t] = FP64 ? ay : (double)fy;
        P[2 * nt + t] = FP64 ? az : (double)fz;
        P[3 * nt + t] = FP64 ? ap : (double)fp;
    }
}

__global__ void direct_reduce_kernel(const double* __restrict__ partial, int64_t nt, int nchunk, double G,
                                     double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
                                     double* __restrict__ phi) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nt;
         t += (int64_t)gridDim.x * blockDim.x) {
        double s[4] = {0, 0, 0, 0};
        for (int c = 0; c < nchunk; ++c)
            for (int k = 0; k < 4; ++k) s[k] += partial[((int64_t)c * 4 + k) * nt + t];
        if (ax) ax[t] = G * s[0];
        if (ay) ay[t] = G * s[1];
        if (az) az[t] = G * s[2];
        if (phi) phi[t] = G * s[3];
    }
}

}  // namespace

void run_direct(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                const double* m, const double* soft, int64_t nt, const uint32_t* targets, double G,
                int precision, double* ax, double* ay, double* az, double* phi) {
    if (nt <= 0) return;
    const int bx = div_up(nt, kDirThreads);
    int nchunk = std::max(1, div_up((int64_t)ctx->num_sms * 4, bx));
    nchunk = std::min<int64_t>(nchunk, std::max<int64_t>(1, div_up(n, 4 * kDirTile)));
    nchunk = std::min(nchunk, 65535);
    const int64_t chunk = std::max<int64_t>(1, div_up(n, nchunk));
    nchunk = std::max(1, div_up(n, chunk));
    double* partial = (double*)scratch(ctx, kSlotDirect, (size_t)nchunk * 4 * nt * 8);
    const dim3 grid(bx, nchunk);
    if (precision == GT_DIRECT_FP32)
        direct_kernel<false><<<grid, kDirThreads, 0, ctx->stream>>>(x, y, z, m, soft, n, targets, nt, chunk, partial);
    else
        direct_kernel<true><<<grid, kDirThreads, 0, ctx->stream>>>(x, y, z, m, soft, n, targets, nt, chunk, partial);
    check_launch(ctx, "direct_kernel");
    direct_reduce_kernel<<<std::max(1, std::min(div_up(nt, 256), ctx->num_sms * 4)), 256, 0, ctx->stream>>>(
        partial, nt, nchunk, G, ax, ay, az, phi);
    check_launch(ctx, "direct_reduce_kernel");
}

}  // namespace gt
