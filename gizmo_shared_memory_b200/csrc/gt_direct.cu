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
#include <cmath>
#include <mutex>

#include "gt_internal.cuh"

// Fixed scratch of the allocation-free entry point gt_direct_noalloc: the per-chunk partial sums,
// 8 MiB, present on every GPU that loads this library until the process exits.  Host code must
// never pass this name to a kernel -- on the host it is only a stand-in symbol; its device address
// comes from cudaGetSymbolAddress (see noalloc_scratch below).
static __device__ __align__(256) double g_direct_noalloc_scratch[GT_DIRECT_NOALLOC_SCRATCH_DOUBLES];

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

// dW/dr of the 3-D cubic spline of support h (shmem/hydro.h:46-54), FP64, zero from r = h.
__device__ __forceinline__ double kernel_dwdr_d(double r, double h) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = 8.0 / (M_PI * h * h * h);
    double fp;
    if (q < 0.5) {
        fp = -12.0 * q + 18.0 * q * q;
    } else {
        const double u = 1.0 - q;
        fp = -6.0 * u * u;
    }
    return norm * fp / h;
}

// GAS (FP64 only): the adaptive-softening zeta terms of gas-gas pairs (tree.cc:39-53); type
// (0 = gas; null = every particle gas) and zeta (null = none) are indexed like the particles.
template <bool FP64, bool GAS = false>
__global__ void __launch_bounds__(kDirThreads)
direct_kernel(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
              const double* __restrict__ m, const double* __restrict__ soft, int64_t n,
              const uint32_t* __restrict__ targets, int64_t nt, int64_t chunk,
              double* __restrict__ partial, const uint8_t* __restrict__ type = nullptr,
              const double* __restrict__ zeta = nullptr) {
    __shared__ double shx[kDirTile], shy[kDirTile], shz[kDirTile], shm[kDirTile], shs[kDirTile];
    __shared__ double shzeta[GAS ? kDirTile : 1];
    __shared__ unsigned char shgas[GAS ? kDirTile : 1];
    const int64_t t = (int64_t)blockIdx.x * kDirThreads + threadIdx.x;
    // a target index at or beyond n (device target arrays are not checked on the host) reads
    // nothing and sums nothing: its outputs are zero
    const bool slot = t < nt;
    const int64_t self = slot ? (int64_t)targets[t] : -1;
    const bool live = slot && self < n;
    const double px = live ? x[self] : 0.0, py = live ? y[self] : 0.0, pz = live ? z[self] : 0.0;
    const double ps = (live && soft) ? soft[self] : 0.0;
    // a gas target with mass: zeta_t / m_t and 1 / m_t of its pair terms
    double tzm = 0.0, tm = 0.0, tzeta = 0.0;
    bool tgas = false;
    if (GAS && live) {
        tgas = !type || type[self] == 0;
        tzeta = zeta ? zeta[self] : 0.0;
        tm = m[self];
        if (tm > 0) tzm = tzeta / tm;
    }
    const int64_t s0 = (int64_t)blockIdx.y * chunk, s1 = min(n, s0 + chunk);
    double ax = 0, ay = 0, az = 0, ap = 0;
    float fx = 0, fy = 0, fz = 0, fp = 0;
    for (int64_t base = s0; base < s1; base += kDirTile) {
        const int64_t q = base + threadIdx.x;
        if (q < s1) {
            shx[threadIdx.x] = x[q]; shy[threadIdx.x] = y[q]; shz[threadIdx.x] = z[q];
            shm[threadIdx.x] = m[q];
            shs[threadIdx.x] = soft ? soft[q] : 0.0;
            if (GAS) {
                shzeta[threadIdx.x] = zeta ? zeta[q] : 0.0;
                shgas[threadIdx.x] = (!type || type[q] == 0) ? 1 : 0;
            }
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
                    double mf = shm[k] * f;
                    if (GAS && tgas && shgas[k] && tm > 0.0) {
                        const double es = fmax(shs[k], 1e-300);
                        if (tzeta != 0.0 && r < e) mf -= tzm * kernel_dwdr_d(r, e) / r;
                        if (shzeta[k] != 0.0 && r < es) mf -= (shzeta[k] / tm) * kernel_dwdr_d(r, es) / r;
                    }
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
    if (slot) {
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

// Source chunking: enough chunks that (target blocks x chunks) fills the GPU, at most
// `max_chunks`.  Returns the chunk length and sets nchunk.
int64_t plan_chunks(int64_t n, int64_t nt, int num_sms, int64_t max_chunks, int& nchunk) {
    const int bx = div_up(nt, kDirThreads);
    int64_t c = std::max(1, div_up((int64_t)num_sms * 4, bx));
    c = std::min<int64_t>(c, std::max<int64_t>(1, div_up(n, 4 * kDirTile)));
    c = std::min<int64_t>(c, std::min<int64_t>(65535, std::max<int64_t>(1, max_chunks)));
    const int64_t chunk = std::max<int64_t>(1, div_up(n, c));
    nchunk = std::max(1, div_up(n, chunk));
    return chunk;
}

void launch_direct(cudaStream_t st, int num_sms, int64_t n, const double* x, const double* y,
                   const double* z, const double* m, const double* soft, int64_t nt,
                   const uint32_t* targets, double G, int precision, double* ax, double* ay,
                   double* az, double* phi, double* partial, int nchunk, int64_t chunk) {
    const dim3 grid(div_up(nt, kDirThreads), nchunk);
    if (precision == GT_DIRECT_FP32)
        direct_kernel<false><<<grid, kDirThreads, 0, st>>>(x, y, z, m, soft, n, targets, nt, chunk, partial);
    else
        direct_kernel<true><<<grid, kDirThreads, 0, st>>>(x, y, z, m, soft, n, targets, nt, chunk, partial);
    direct_reduce_kernel<<<std::max(1, std::min(div_up(nt, 256), num_sms * 4)), 256, 0, st>>>(
        partial, nt, nchunk, G, ax, ay, az, phi);
}

}  // namespace

void run_direct_gas(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z, const double* m,
                    const double* soft, const uint8_t* type, const double* zeta, int64_t nt, const uint32_t* targets,
                    double G, double* ax, double* ay, double* az) {
    if (nt <= 0) return;
    int nchunk = 1;
    const int64_t chunk = plan_chunks(n, nt, ctx->num_sms, 65535, nchunk);
    double* partial = (double*)scratch(ctx, kSlotDirect, (size_t)nchunk * 4 * nt * 8);
    const dim3 grid(div_up(nt, kDirThreads), nchunk);
    direct_kernel<true, true><<<grid, kDirThreads, 0, ctx->stream>>>(x, y, z, m, soft, n, targets, nt, chunk, partial,
                                                                     type, zeta);
    direct_reduce_kernel<<<std::max(1, std::min(div_up(nt, 256), ctx->num_sms * 4)), 256, 0, ctx->stream>>>(
        partial, nt, nchunk, G, ax, ay, az, nullptr);
    ctx->launches += 2;
    check_cuda(cudaGetLastError(), "direct_kernel");
}

void run_direct(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                const double* m, const double* soft, int64_t nt, const uint32_t* targets, double G,
                int precision, double* ax, double* ay, double* az, double* phi) {
    if (nt <= 0) return;
    int nchunk = 1;
    const int64_t chunk = plan_chunks(n, nt, ctx->num_sms, 65535, nchunk);
    double* partial = (double*)scratch(ctx, kSlotDirect, (size_t)nchunk * 4 * nt * 8);
    launch_direct(ctx->stream, ctx->num_sms, n, x, y, z, m, soft, nt, targets, G, precision, ax, ay,
                  az, phi, partial, nchunk, chunk);
    ctx->launches += 2;
    check_cuda(cudaGetLastError(), "direct_kernel");
}

}  // namespace gt

// ---------------------------------------------------------------------------------------------
// gt_direct_noalloc: the direct sum for callers that must not allocate device memory
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Device address of g_direct_noalloc_scratch on `dev` (which is current), looked up once per device.
int noalloc_scratch(int dev, double** ptr, int* sms) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_direct_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GT_ERR_CUDA;
        }
        int nsm = 0;
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || nsm <= 0) {
            cudaGetLastError();
            return GT_ERR_CUDA;
        }
        g_noalloc_sms[dev] = nsm;
        g_noalloc_ptr[dev] = (double*)p;
    }
    *ptr = g_noalloc_ptr[dev];
    *sms = g_noalloc_sms[dev];
    return GT_OK;
}

}  // namespace

extern "C" int gt_direct_noalloc(int64_t n, const double* x, const double* y, const double* z,
                                 const double* m, const double* soft, int64_t n_targets,
                                 const uint32_t* targets, double G, int precision, double* ax,
                                 double* ay, double* az, double* phi, void* stream) {
    if (n < 0 || n_targets < 0) return GT_ERR_INVALID;
    if (n > 0 && (!x || !y || !z || !m)) return GT_ERR_INVALID;
    if (n_targets > 0 && (!targets || !ax || !ay || !az)) return GT_ERR_INVALID;
    if (precision != GT_DIRECT_FP64 && precision != GT_DIRECT_FP32) return GT_ERR_INVALID;
    if (n_targets > GT_DIRECT_NOALLOC_MAX_TARGETS) return GT_ERR_OVERFLOW;
    if (n_targets == 0) return GT_OK;
    if (n == 0) return GT_ERR_INVALID;  // no particle can be a target
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        cudaGetLastError();
        return GT_ERR_DEVICE;
    }
    double* partial = nullptr;
    int sms = 0;
    const int st = noalloc_scratch(dev, &partial, &sms);
    if (st != GT_OK) return st;
    // every (chunk, target) partial the reduction reads is written by this call's first kernel,
    // so the scratch needs no clearing; the chunk count is capped so the partials fit
    const int64_t max_chunks = GT_DIRECT_NOALLOC_SCRATCH_DOUBLES / (4 * n_targets);
    int nchunk = 1;
    const int64_t chunk = gt::plan_chunks(n, n_targets, sms, max_chunks, nchunk);
    gt::launch_direct((cudaStream_t)stream, sms, n, x, y, z, m, soft, n_targets, targets, G, precision,
                      ax, ay, az, phi, partial, nchunk, chunk);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GT_OK : GT_ERR_CUDA;
}
