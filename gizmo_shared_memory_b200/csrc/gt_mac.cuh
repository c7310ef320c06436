// Learned multipole-acceptance criterion: feature definition and the small MLP, shared by the
// sampling kernel, the training kernels and the walk.
//
// The plain relative criterion (shmem/tree.h:134-135) accepts a node for a group when
//     rho = M L^2 / (r_min^4 aold_min) <= 1,
// i.e. it estimates the monopole error of the node as M L^2 / r^4.  The network predicts, from 8
// dimensionless features of the (group, node) geometry, c = log10 of how far the true worst error
// of accepting the node (measured against the exact sum over the node's particles) sits above or
// below that estimate.  The learned rule accepts when rho * 10^c <= kappa.
#pragma once
#include "gt_internal.cuh"

namespace gt {

constexpr int kMacIn = GT_MAC_FEATURES;     // 8
constexpr int kMacHidden = GT_MAC_HIDDEN;   // 32
// model layout (floats): mean[8], inv_sd[8], W1[32][8], b1[32], W2[32][32], b2[32], W3[32], b3
constexpr int kMacNorm = 2 * kMacIn;
constexpr int kMacW1 = kMacNorm;
constexpr int kMacB1 = kMacW1 + kMacHidden * kMacIn;
constexpr int kMacW2 = kMacB1 + kMacHidden;
constexpr int kMacB2 = kMacW2 + kMacHidden * kMacHidden;
constexpr int kMacW3 = kMacB2 + kMacHidden;
constexpr int kMacB3 = kMacW3 + kMacHidden;
constexpr int kMacModel = kMacB3 + 1;
static_assert(kMacModel == GT_MAC_MODEL_FLOATS, "model layout");
constexpr int kMacParams = kMacModel - kMacNorm;

// The 8 features of (group, node).  r2 is the squared nearest-point distance of the node's COM to
// the group box, rho the plain criterion's ratio, ext2 the squared diagonal of the group box.
// Ratios are formed in FP64 (they span many decades) and their logarithms taken in FP32 with the
// hardware log2: the features only need a few digits.
__device__ __forceinline__ float lg10f(double v) { return __log2f((float)v) * 0.30102999566398120f; }

__device__ __forceinline__ void mac_features(double r2, double rho, double len, double s, double mass,
                                             double q2, double nsoft, double emax, int count,
                                             double rmax2, double ext2, float* f) {
    const double l = fmax(len, 1e-300);
    const double l2 = l * l;
    f[0] = 0.5f * lg10f(r2 / l2);
    f[1] = lg10f(q2 / fmax(mass * l2, 1e-300) + 1e-12);
    f[2] = lg10f((s - len) / l + 1e-6);
    f[3] = 0.5f * lg10f(rmax2 / fmax(r2, 1e-300));
    f[4] = lg10f(fmax(rho, 1e-30));
    f[5] = lg10f((double)max(count, 1));
    const double h = fmax(emax, nsoft);
    f[6] = 0.5f * lg10f(h * h / fmax(r2, 1e-300) + 1e-24);
    f[7] = 0.5f * lg10f(ext2 / l2 + 1e-12);
}

// The node-only features of the per-node criterion (GT_MAC_NODE_FEATURES): the same definitions as
// mac_features for features 1, 2 and 5; the pair features stay 0 (the model ignores them).
__device__ __forceinline__ void mac_node_features(double len, double s, double mass, double q2, int count,
                                                  float* f) {
    const double l = fmax(len, 1e-300);
    const double l2 = l * l;
#pragma unroll
    for (int i = 0; i < kMacIn; ++i) f[i] = 0.0f;
    f[1] = lg10f(q2 / fmax(mass * l2, 1e-300) + 1e-12);
    f[2] = lg10f((s - len) / l + 1e-6);
    f[5] = lg10f((double)max(count, 1));
}

// MLP forward in FP32 on normalised features; `m` points at a model in shared or global memory.
__device__ __forceinline__ float mac_forward(const float* __restrict__ m, const float* x) {
    float xn[kMacIn];
#pragma unroll
    for (int i = 0; i < kMacIn; ++i) xn[i] = (x[i] - m[i]) * m[kMacIn + i];
    float h1[kMacHidden];
#pragma unroll
    for (int j = 0; j < kMacHidden; ++j) {
        float a = m[kMacB1 + j];
#pragma unroll
        for (int i = 0; i < kMacIn; ++i) a = fmaf(m[kMacW1 + j * kMacIn + i], xn[i], a);
        h1[j] = fmaxf(a, 0.0f);
    }
    float y = m[kMacB3];
#pragma unroll 4
    for (int k = 0; k < kMacHidden; ++k) {
        float a = m[kMacB2 + k];
#pragma unroll
        for (int j = 0; j < kMacHidden; ++j) a = fmaf(m[kMacW2 + k * kMacHidden + j], h1[j], a);
        y = fmaf(m[kMacW3 + k], fmaxf(a, 0.0f), y);
    }
    return y;
}

}  // namespace gt
