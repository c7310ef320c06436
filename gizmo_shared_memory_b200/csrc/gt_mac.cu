// Learned multipole-acceptance criterion: training data from the walk, and the MLP's training
// and inference kernels (no library GEMMs: the network is 8 -> 32 -> 32 -> 1).
//
// Sampling.  mac_sample_kernel walks the tree for a subset of target windows exactly as the plain
// relative criterion does (shmem/tree.h:109-144, leaves offered first).  Every node it tests that
// the softening-overlap and inside-node arms leave undecided and whose ratio
// rho = M L^2 / (r_min^4 aold_min) falls in a window around the plain threshold becomes a sample:
// the warp sums the node's particles exactly (FP64 offsets from the window centre, FP32 pair rule)
// for each target, compares with the node's monopole, and records the worst relative error
// across the window next to the node's 8 features.
//
// Training.  Pinball (quantile) loss, so the network predicts an upper quantile of the error
// correction (a conservative criterion); Adam.  Each step: one thread per sample for the forward
// and backward pass (activations and deltas to a buffer), then one block per parameter sums its
// gradient over the batch in a fixed order (deterministic), then the Adam update.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "gt_mac.cuh"

namespace gt {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double wmin(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ float wmaxf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ int warp_incl_scan_i(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Pair force factor of the cubic spline in FP32 (shmem/tree.h:59-67); 0 for r == 0.
__device__ __forceinline__ float pair_factor(float r2, float h, float m) {
    if (!(r2 > 0.0f)) return 0.0f;
    if (r2 >= h * h) {
        const float ri = rsqrtf(r2);
        return m * ri * ri * ri;
    }
    const float r = sqrtf(r2), hi = 1.0f / h, u = r * hi, hi3 = hi * hi * hi;
    if (u < 0.5f) return m * hi3 * (10.666666666666667f + u * u * (32.0f * u - 38.4f));
    const float u3 = u * u * u;
    return m * hi3 * (21.333333333333332f - 48.0f * u + 38.4f * u * u - 10.666666666666667f * u3 -
                      0.06666666666666667f / u3);
}

struct SampleArgs {
    const GNode* nodes;
    const SrcP* src;
    const double* ssoft;
    const float* nq2;
    const int2* groups;
    int n_groups;
    const double* amag;
    double alpha, rho_lo, rho_hi;
    int* stack;
    int stack_cap;
    unsigned* next_group;
    float* feat;
    float* label;
    float* rho;
    long long cap;
    unsigned long long* count;
    int* error;
};

__global__ void __launch_bounds__(256) mac_sample_kernel(const SampleArgs A) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int* stk = A.stack + (size_t)gw * A.stack_cap;
    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(A.next_group, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= A.n_groups) break;
        const int2 gr = A.groups[g];
        const int t0 = gr.x, nt = gr.y - gr.x;  // <= 32
        const bool tv = lane < nt;
        double px = 0, py = 0, pz = 0, ps = 0, am = 1e300;
        if (tv) {
            const SrcP s = A.src[t0 + lane];
            px = s.x; py = s.y; pz = s.z;
            ps = A.ssoft[t0 + lane];
            am = A.amag[t0 + lane];
        }
        const double lx = wmin(tv ? px : 1e300), hx = wmax(tv ? px : -1e300);
        const double ly = wmin(tv ? py : 1e300), hy = wmax(tv ? py : -1e300);
        const double lz = wmin(tv ? pz : 1e300), hz = wmax(tv ? pz : -1e300);
        const double emax = wmax(tv ? ps : 0.0);
        const double amin = wmin(am);
        const double aold = A.alpha * amin;
        const double gcx = 0.5 * (lx + hx), gcy = 0.5 * (ly + hy), gcz = 0.5 * (lz + hz);
        const double ext2 = (hx - lx) * (hx - lx) + (hy - ly) * (hy - ly) + (hz - lz) * (hz - lz);
        const float tx = (float)(px - gcx), ty = (float)(py - gcy), tz = (float)(pz - gcz);
        const float th = (float)ps;
        if (!(aold > 0)) continue;  // the relative criterion needs a previous acceleration

        int top = 1;
        if (lane == 0) stk[0] = 0;
        __syncwarp();
        while (top > 0) {
            const int npop = min(top, 32);
            top -= npop;
            const int node = lane < npop ? stk[top + lane] : -1;
            __syncwarp();
            bool push = false, sample = false;
            GNode nd;
            nd.first = -1; nd.nchild = 0; nd.plo = nd.phi = 0;
            double rho = 0;
            float f[kMacIn];
            if (node >= 0) {
                nd = A.nodes[node];
                const double len = (double)nd.len;
                const double dx = fmax(0.0, fmax(lx - nd.cx, nd.cx - hx));
                const double dy = fmax(0.0, fmax(ly - nd.cy, nd.cy - hy));
                const double dz = fmax(0.0, fmax(lz - nd.cz, nd.cz - hz));
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double rt = emax + 0.6 * len, rn = (double)nd.soft + 0.6 * len;
                const bool overlap = (r2 < rt * rt) | (r2 < rn * rn);
                const double lim = 0.6 * len;
                const bool inside = (dx < lim) & (dy < lim) & (dz < lim);
                rho = (nd.mass * len * len) / (r2 * r2 * aold);
                const bool open = overlap | inside | (nd.mass * len * len > r2 * r2 * aold);
                push = open && nd.first >= 0;
                sample = !overlap && !inside && rho >= A.rho_lo && rho <= A.rho_hi;
                if (sample) {
                    const double ax_ = fmax(fabs(nd.cx - lx), fabs(nd.cx - hx));
                    const double ay_ = fmax(fabs(nd.cy - ly), fabs(nd.cy - hy));
                    const double az_ = fmax(fabs(nd.cz - lz), fabs(nd.cz - hz));
                    mac_features(r2, rho, len, nd.s, nd.mass, (double)A.nq2[node], (double)nd.soft,
                                 emax, nd.phi - nd.plo, ax_ * ax_ + ay_ * ay_ + az_ * az_, ext2, f);
                }
            }
            // exact error of every sampled node, one at a time across the window's targets
            unsigned sm = __ballot_sync(kFull, sample);
            while (sm) {
                const int l = __ffs(sm) - 1;
                sm &= sm - 1;
                const int plo = __shfl_sync(kFull, nd.plo, l), phi = __shfl_sync(kFull, nd.phi, l);
                const double ncx = __shfl_sync(kFull, nd.cx, l), ncy = __shfl_sync(kFull, nd.cy, l);
                const double ncz = __shfl_sync(kFull, nd.cz, l), nm = __shfl_sync(kFull, nd.mass, l);
                const double nrho = __shfl_sync(kFull, rho, l);
                float ex = 0, ey = 0, ez = 0;
                for (int j = plo; j < phi; ++j) {
                    const SrcP q = A.src[j];
                    const float dx = (float)(q.x - gcx) - tx, dy = (float)(q.y - gcy) - ty,
                                dz = (float)(q.z - gcz) - tz;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    const float fac = pair_factor(r2, fmaxf(th, q.soft), q.m);
                    ex += dx * fac; ey += dy * fac; ez += dz * fac;
                }
                const float mdx = (float)(ncx - gcx) - tx, mdy = (float)(ncy - gcy) - ty,
                            mdz = (float)(ncz - gcz) - tz;
                const float mr2 = fmaxf(mdx * mdx + mdy * mdy + mdz * mdz, 1e-30f);
                const float mri = rsqrtf(mr2);
                const float mf = (float)nm * mri * mri * mri;
                const float ddx = mdx * mf - ex, ddy = mdy * mf - ey, ddz = mdz * mf - ez;
                const float e = tv ? sqrtf(ddx * ddx + ddy * ddy + ddz * ddz) / (float)am : 0.0f;
                const float emax_w = wmaxf(e);
                if (lane == l) {
                    const unsigned long long slot = atomicAdd(A.count, 1ull);
                    if ((long long)slot < A.cap) {
#pragma unroll
                        for (int k = 0; k < kMacIn; ++k) A.feat[slot * kMacIn + k] = f[k];
                        const double lbl = log10(fmax((double)emax_w, 1e-10 * A.alpha * nrho)) -
                                           log10(A.alpha * nrho);
                        A.label[slot] = (float)lbl;
                        A.rho[slot] = (float)nrho;
                    }
                }
            }
            const int nch = push ? nd.nchild : 0;
            const int incl = warp_incl_scan_i(nch);
            const int tot = __shfl_sync(kFull, incl, 31);
            if (top + tot > A.stack_cap) {
                if (lane == 0) atomicExch(A.error, 1);
                break;
            }
            for (int c = 0; c < nch; ++c) stk[top + incl - nch + c] = nd.first + c;
            top += tot;
            __syncwarp();
        }
    }
}

// ---- the exact-label criterion: what a perfect learned predictor could reach ------------------
//
// ceiling_kernel walks chosen windows of consecutive targets as the grouped walk does (nearest
// point of the window's box, largest target softening, leaves offered to the criterion first;
// shmem/tree.cc:682-702, 744-779) and sums the forces in FP64.  Its acceptance rule is either
//   mode 0: the plain relative criterion, M L^2 <= r^4 alpha min|a| (shmem/tree.h:134-135), or
//   mode 1: exact labels -- inside the band rho_lo < rho <= rho_hi the warp sums the node's
//           particles for every target of the window and accepts the node only when the monopole's
//           worst error over the window, |a_mono - a_exact|_t / |a_t|, is at most
//           eps * ((c - 1) / 7)^cost_exp, c the interactions opening it costs one step ahead (its
//           children, or a leaf's particles; c - 1 floored at 1); below the band it accepts, above
//           it it opens.  cost_exp = 0 is a constant threshold; cost_exp > 0 spends more of the
//           error budget where opening is dearer.
// Modes 2-5 keep the form of the relative criterion, X / r^4 <= alpha |a|, with one ingredient of
// the exact rule each, to show which of them carry the exact rule's savings:
//   mode 2: r = the larger of the distances to the window's box and to its enclosing sphere (about
//           the box centre): both are lower bounds of the distance to every target;
//   mode 3: per target, r_t = its own distance to the node's centre of mass and its own |a_t|;
//           the node opens if any target's ratio exceeds alpha;
//   mode 4: mode 3 with X = 4 q2, q2 the node's second mass moment about its centre of mass,
//           in place of M L^2 (4 q2 = M L^2 for a uniform cube);
//   mode 5: mode 0 (the box's nearest point, min |a|) with X = 4 q2.
// All modes share the softening-overlap and inside-node arms.  Mode 1 is the rule a learned
// criterion that predicted every (window, node) error exactly would apply, so its interactions and
// node visits at a given force error bound what any learned acceptance rule over the monopole walk
// can save.  Mode 0 reproduces the production walk's decisions (the test checks its counts).
struct CeilArgs {
    const GNode* nodes;
    const SrcP* src;
    const double* ssoft;
    const int64_t* wins;  // window indices: targets [w * window, min((w + 1) * window, n_live))
    int n_win, window;
    int64_t n_live;
    const double* amag;   // |a| per live particle in tree order
    const float* nq2;     // per node second mass moment about the centre of mass (modes 4, 5)
    double alpha, eps, cost_exp, rho_lo, rho_hi;
    int mode;
    int* stack;
    int stack_cap;
    unsigned* next;
    double *ax, *ay, *az;          // n_win * window, slot w * window + lane
    unsigned long long* counts;    // per window: visits, multipole, pairs, labelled nodes, label sum
    int* error;
};

// FP64 force factor of the cubic spline of support h (shmem/tree.h:59-67): 1/r^3 outside.
__device__ __forceinline__ double spline_force_d(double r2, double h) {
    const double r = sqrt(r2);
    if (r >= h) return 1.0 / (r2 * r);
    const double hi = 1.0 / h, u = r * hi, hi3 = hi * hi * hi;
    if (u < 0.5) return hi3 * (10.666666666666667 + u * u * (32.0 * u - 38.4));
    return hi3 * (21.333333333333332 - 48.0 * u + 38.4 * u * u - 10.666666666666667 * u * u * u -
                  0.06666666666666667 / (u * u * u));
}

__global__ void __launch_bounds__(256) ceiling_kernel(const CeilArgs A) {
    __shared__ SrcP tile[8][32];
    __shared__ double tq[8][32][4];  // the window's targets: position and 1 / |a| (modes 3, 4)
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + wi;
    int* stk = A.stack + (size_t)gw * A.stack_cap;
    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(A.next, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= A.n_win) break;
        const int64_t t0 = A.wins[g] * A.window;
        const int nt = (int)min((int64_t)A.window, A.n_live - t0);
        const bool tv = lane < nt;
        double px = 0, py = 0, pz = 0, ps = 0, am = 1e300;
        if (tv) {
            const SrcP s = A.src[t0 + lane];
            px = s.x; py = s.y; pz = s.z;
            ps = A.ssoft[t0 + lane];
            am = A.amag[t0 + lane];
        }
        const double lx = wmin(tv ? px : 1e300), hx = wmax(tv ? px : -1e300);
        const double ly = wmin(tv ? py : 1e300), hy = wmax(tv ? py : -1e300);
        const double lz = wmin(tv ? pz : 1e300), hz = wmax(tv ? pz : -1e300);
        const double emax = wmax(tv ? ps : 0.0);
        const double aold = A.alpha * wmin(am);
        const double inv_a = tv && am > 0.0 ? 1.0 / am : 0.0;  // 0: a target without |a| never accepts
        const double gcx = 0.5 * (lx + hx), gcy = 0.5 * (ly + hy), gcz = 0.5 * (lz + hz);
        // enclosing sphere about the box centre (mode 2)
        const double rsph = sqrt(wmax(tv ? (px - gcx) * (px - gcx) + (py - gcy) * (py - gcy) + (pz - gcz) * (pz - gcz) : 0.0));
        tq[wi][lane][0] = px; tq[wi][lane][1] = py; tq[wi][lane][2] = pz;
        tq[wi][lane][3] = tv ? (am > 0.0 ? 1.0 / am : 1e300) : 0.0;
        __syncwarp();
        double sx = 0, sy = 0, sz = 0;
        unsigned long long c_vis = 0, c_mul = 0, c_pair = 0, c_lab = 0, c_labsum = 0;
        unsigned c_self = 0;  // pairs at r = 0 (the target itself), which count as no interaction

        int top = 1;
        if (lane == 0) stk[0] = 0;
        __syncwarp();
        bool overflow = false;
        while (top > 0) {
            const int npop = min(top, 32);
            top -= npop;
            const int node = lane < npop ? stk[top + lane] : -1;
            __syncwarp();
            GNode nd;
            nd.first = -1; nd.nchild = 0; nd.plo = nd.phi = 0; nd.cx = nd.cy = nd.cz = nd.mass = 0.0;
            bool open = false, label = false;
            if (node >= 0) {
                nd = A.nodes[node];
                const double len = (double)nd.len;
                const double dx = fmax(0.0, fmax(lx - nd.cx, nd.cx - hx));
                const double dy = fmax(0.0, fmax(ly - nd.cy, nd.cy - hy));
                const double dz = fmax(0.0, fmax(lz - nd.cz, nd.cz - hz));
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double rt = emax + 0.6 * len, rn = (double)nd.soft + 0.6 * len;
                const double lim = 0.6 * len;
                const bool hard = (r2 < rt * rt) | (r2 < rn * rn) | ((dx < lim) & (dy < lim) & (dz < lim));
                if (hard || !(aold > 0)) {
                    open = true;
                } else {
                    const double rho = nd.mass * len * len / (r2 * r2 * aold);
                    const double X = (A.mode == 4 || A.mode == 5) ? 4.0 * (double)A.nq2[node] : nd.mass * len * len;
                    if (A.mode == 0) open = rho > 1.0;
                    else if (A.mode == 5) open = X > r2 * r2 * aold;
                    else if (A.mode == 2) {
                        const double cx = nd.cx - gcx, cy = nd.cy - gcy, cz = nd.cz - gcz;
                        const double rb = sqrt(r2), rs = sqrt(cx * cx + cy * cy + cz * cz) - rsph;
                        const double r = rs > rb ? rs : rb;
                        open = X > r * r * r * r * aold;
                    } else if (A.mode == 3 || A.mode == 4) {
                        double worst = 0.0;
                        for (int k = 0; k < nt; ++k) {
                            const double ex = nd.cx - tq[wi][k][0], ey = nd.cy - tq[wi][k][1], ez = nd.cz - tq[wi][k][2];
                            const double q = ex * ex + ey * ey + ez * ez;
                            worst = fmax(worst, X * tq[wi][k][3] / (q * q));
                        }
                        open = worst > A.alpha;
                    }
                    else if (rho <= A.rho_lo) open = false;
                    else if (rho > A.rho_hi) open = true;
                    else label = true;
                }
            }
            // exact labels, one node at a time across the window's targets; the node's particles
            // are staged 32 at a time in shared memory
            unsigned lm = __ballot_sync(kFull, label);
            while (lm) {
                const int l = __ffs(lm) - 1;
                lm &= lm - 1;
                const int plo = __shfl_sync(kFull, nd.plo, l), phi = __shfl_sync(kFull, nd.phi, l);
                const double ncx = __shfl_sync(kFull, nd.cx, l), ncy = __shfl_sync(kFull, nd.cy, l);
                const double ncz = __shfl_sync(kFull, nd.cz, l), nm = __shfl_sync(kFull, nd.mass, l);
                double ex = 0, ey = 0, ez = 0;
                for (int base = plo; base < phi; base += 32) {
                    if (base + lane < phi) tile[wi][lane] = A.src[base + lane];
                    __syncwarp();
                    const int k = min(32, phi - base);
                    for (int j = 0; j < k; ++j) {
                        const SrcP q = tile[wi][j];
                        const double dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                        const double r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 > 0.0) {
                            const double f = (double)q.m * spline_force_d(r2, fmax(ps, (double)q.soft));
                            ex += dx * f; ey += dy * f; ez += dz * f;
                        }
                    }
                    __syncwarp();
                }
                const double mdx = ncx - px, mdy = ncy - py, mdz = ncz - pz;
                const double mr2 = mdx * mdx + mdy * mdy + mdz * mdz;
                const double mf = nm / (mr2 * sqrt(mr2));
                const double ddx = mdx * mf - ex, ddy = mdy * mf - ey, ddz = mdz * mf - ez;
                const double e = tv ? (inv_a > 0.0 ? sqrt(ddx * ddx + ddy * ddy + ddz * ddz) * inv_a : 1e300) : 0.0;
                const double worst = wmax(e);
                if (lane == l) {
                    const int cost = nd.first < 0 ? nd.phi - nd.plo : nd.nchild;
                    const double thr = A.cost_exp == 0.0 ? A.eps
                                                         : A.eps * pow(fmax((double)(cost - 1), 1.0) / 7.0, A.cost_exp);
                    open = worst > thr;
                }
                if (lane == 0) { ++c_lab; c_labsum += (unsigned long long)(phi - plo); }
            }
            const bool leaf = nd.first < 0;
            const bool accept = node >= 0 && !open;
            const bool expand = node >= 0 && open && leaf;
            const bool push = node >= 0 && open && !leaf;
            if (lane == 0) c_vis += npop;
            // accepted nodes: Newtonian monopoles for every target
            unsigned am_ = __ballot_sync(kFull, accept);
            if (lane == 0) c_mul += (unsigned long long)__popc(am_) * nt;
            while (am_) {
                const int l = __ffs(am_) - 1;
                am_ &= am_ - 1;
                const double ncx = __shfl_sync(kFull, nd.cx, l), ncy = __shfl_sync(kFull, nd.cy, l);
                const double ncz = __shfl_sync(kFull, nd.cz, l), nm = __shfl_sync(kFull, nd.mass, l);
                const double dx = ncx - px, dy = ncy - py, dz = ncz - pz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (tv && r2 > 0.0) {
                    const double f = nm / (r2 * sqrt(r2));
                    sx += dx * f; sy += dy * f; sz += dz * f;
                }
            }
            // expanded leaves: their particles with the pair rule (kernel of the larger softening)
            unsigned em = __ballot_sync(kFull, expand);
            while (em) {
                const int l = __ffs(em) - 1;
                em &= em - 1;
                const int plo = __shfl_sync(kFull, nd.plo, l), phi = __shfl_sync(kFull, nd.phi, l);
                if (lane == 0) c_pair += (unsigned long long)(phi - plo) * nt;
                for (int base = plo; base < phi; base += 32) {
                    if (base + lane < phi) tile[wi][lane] = A.src[base + lane];
                    __syncwarp();
                    const int k = min(32, phi - base);
                    for (int j = 0; j < k; ++j) {
                        const SrcP q = tile[wi][j];
                        const double dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                        const double r2 = dx * dx + dy * dy + dz * dz;
                        if (tv && r2 > 0.0) {
                            const double f = (double)q.m * spline_force_d(r2, fmax(ps, (double)q.soft));
                            sx += dx * f; sy += dy * f; sz += dz * f;
                        }
                        c_self += (tv && r2 == 0.0);
                    }
                    __syncwarp();
                }
            }
            const int nch = push ? nd.nchild : 0;
            const int incl = warp_incl_scan_i(nch);
            const int tot = __shfl_sync(kFull, incl, 31);
            if (top + tot > A.stack_cap) { overflow = true; break; }
            for (int c = 0; c < nch; ++c) stk[top + incl - nch + c] = nd.first + c;
            top += tot;
            __syncwarp();
        }
        if (overflow) {
            if (lane == 0) atomicExch(A.error, 1);
            continue;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c_self += __shfl_xor_sync(kFull, c_self, o);
        const int64_t slot = (int64_t)g * A.window + lane;
        if (lane < A.window) {
            A.ax[slot] = tv ? sx : 0.0;
            A.ay[slot] = tv ? sy : 0.0;
            A.az[slot] = tv ? sz : 0.0;
        }
        if (lane == 0) {
            unsigned long long* c = A.counts + (size_t)g * 5;
            c[0] = c_vis; c[1] = c_mul; c[2] = c_pair - c_self; c[3] = c_lab; c[4] = c_labsum;
        }
    }
}

// ---- training --------------------------------------------------------------------------------
constexpr int kActStride = kMacIn + 4 * kMacHidden + 1;  // xn, h1, h2, d2, d1, dy

__global__ void feat_stats_kernel(const float* __restrict__ X, int64_t n, float* __restrict__ model) {
    const int f = blockIdx.x;
    double s = 0, s2 = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = X[i * kMacIn + f];
        s += v;
        s2 += v * v;
    }
    __shared__ double sh[2][256];
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = s2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double cnt = n > 0 ? (double)n : 1.0;
        const double mean = sh[0][0] / cnt;
        const double var = fmax(sh[1][0] / cnt - mean * mean, 0.0);
        model[f] = (float)mean;
        model[kMacIn + f] = (float)(1.0 / sqrt(var + 1e-8));
    }
}

__global__ void mlp_fwd_bwd_kernel(const float* __restrict__ m, const float* __restrict__ X,
                                   const float* __restrict__ Y, const int* __restrict__ perm,
                                   int64_t off, int B, float tau, float* __restrict__ act,
                                   double* __restrict__ loss_part) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double loss = 0;
    if (s < B) {
        const int64_t idx = perm ? perm[off + s] : off + s;
        float* a = act + (int64_t)s * kActStride;
        float xn[kMacIn];
#pragma unroll
        for (int i = 0; i < kMacIn; ++i) {
            xn[i] = (X[idx * kMacIn + i] - m[i]) * m[kMacIn + i];
            a[i] = xn[i];
        }
        float h1[kMacHidden], h2[kMacHidden];
        for (int j = 0; j < kMacHidden; ++j) {
            float v = m[kMacB1 + j];
#pragma unroll
            for (int i = 0; i < kMacIn; ++i) v = fmaf(m[kMacW1 + j * kMacIn + i], xn[i], v);
            h1[j] = fmaxf(v, 0.0f);
            a[kMacIn + j] = h1[j];
        }
        float yhat = m[kMacB3];
        for (int k = 0; k < kMacHidden; ++k) {
            float v = m[kMacB2 + k];
#pragma unroll 8
            for (int j = 0; j < kMacHidden; ++j) v = fmaf(m[kMacW2 + k * kMacHidden + j], h1[j], v);
            h2[k] = fmaxf(v, 0.0f);
            a[kMacIn + kMacHidden + k] = h2[k];
            yhat = fmaf(m[kMacW3 + k], h2[k], yhat);
        }
        const float r = Y[idx] - yhat;
        loss = r >= 0.0f ? (double)tau * r : (double)(tau - 1.0f) * r;
        const float dy = (r >= 0.0f ? -tau : 1.0f - tau) / (float)B;
        float d2[kMacHidden];
        for (int k = 0; k < kMacHidden; ++k) {
            d2[k] = h2[k] > 0.0f ? dy * m[kMacW3 + k] : 0.0f;
            a[kMacIn + 2 * kMacHidden + k] = d2[k];
        }
        for (int j = 0; j < kMacHidden; ++j) {
            float v = 0.0f;
            if (h1[j] > 0.0f) {
#pragma unroll 8
                for (int k = 0; k < kMacHidden; ++k) v = fmaf(d2[k], m[kMacW2 + k * kMacHidden + j], v);
            }
            a[kMacIn + 3 * kMacHidden + j] = v;
        }
        a[kMacIn + 4 * kMacHidden] = dy;
    }
    // deterministic block sum of the loss
    __shared__ double sh[256];
    sh[threadIdx.x] = loss;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0];
}

// One block per trainable parameter (index into the model after the normalisation).
__global__ void mlp_grad_kernel(const float* __restrict__ act, int B, float* __restrict__ grad) {
    const int p = blockIdx.x;
    int ka, kb;  // act offsets of the two factors; kb < 0: the factor is 1 (a bias)
    const int H = kMacHidden, I = kMacIn;
    const int o_h1 = I, o_h2 = I + H, o_d2 = I + 2 * H, o_d1 = I + 3 * H, o_dy = I + 4 * H;
    if (p < H * I) { ka = o_d1 + p / I; kb = p % I; }                 // W1[j][i] = sum d1[j] xn[i]
    else if (p < H * I + H) { ka = o_d1 + (p - H * I); kb = -1; }     // b1
    else if (p < H * I + H + H * H) {                                 // W2[k][j] = sum d2[k] h1[j]
        const int q = p - H * I - H;
        ka = o_d2 + q / H; kb = o_h1 + q % H;
    } else if (p < H * I + 2 * H + H * H) { ka = o_d2 + (p - H * I - H - H * H); kb = -1; }  // b2
    else if (p < H * I + 3 * H + H * H) { ka = o_dy; kb = o_h2 + (p - H * I - 2 * H - H * H); }  // W3
    else { ka = o_dy; kb = -1; }                                      // b3
    double s = 0;
    for (int i = threadIdx.x; i < B; i += blockDim.x) {
        const float* a = act + (int64_t)i * kActStride;
        s += (double)a[ka] * (kb >= 0 ? (double)a[kb] : 1.0);
    }
    __shared__ double sh[128];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) grad[p] = (float)sh[0];
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ mo,
                            float* __restrict__ ve, int n, float lr, float b1, float b2, float c1,
                            float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    mo[i] = b1 * mo[i] + (1.0f - b1) * g[i];
    ve[i] = b2 * ve[i] + (1.0f - b2) * g[i] * g[i];
    w[i] -= lr * (mo[i] / c1) / (sqrtf(ve[i] / c2) + 1e-8f);
}

__global__ void mlp_predict_kernel(const float* __restrict__ m, const float* __restrict__ X, int64_t n,
                                   float* __restrict__ out) {
    __shared__ float sm[kMacModel];
    for (int i = threadIdx.x; i < kMacModel; i += blockDim.x) sm[i] = m[i];
    __syncthreads();
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        float x[kMacIn];
#pragma unroll
        for (int i = 0; i < kMacIn; ++i) x[i] = X[s * kMacIn + i];
        out[s] = mac_forward(sm, x);
    }
}

void init_params(float* model, uint64_t seed, float bias_out) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    const float s1 = std::sqrt(2.0f / kMacIn), s2 = std::sqrt(2.0f / kMacHidden), s3 = std::sqrt(1.0f / kMacHidden);
    for (int i = 0; i < kMacHidden * kMacIn; ++i) model[kMacW1 + i] = s1 * nd(rng);
    for (int i = 0; i < kMacHidden; ++i) model[kMacB1 + i] = 0.0f;
    for (int i = 0; i < kMacHidden * kMacHidden; ++i) model[kMacW2 + i] = s2 * nd(rng);
    for (int i = 0; i < kMacHidden; ++i) model[kMacB2 + i] = 0.0f;
    for (int i = 0; i < kMacHidden; ++i) model[kMacW3 + i] = 0.1f * s3 * nd(rng);
    model[kMacB3] = bias_out;
}

}  // namespace

void run_mac_ceiling(gt_context* ctx, const gt_tree* t, const double* amag, double alpha, int window,
                     int64_t n_win, const int64_t* wins, int mode, double eps, double cost_exp, double rho_lo,
                     double rho_hi, double* ax, double* ay, double* az, unsigned long long* counts) {
    cudaStream_t st = ctx->stream;
    if (n_win <= 0) return;
    const int warps = 8;
    const int blocks = std::max(1, std::min<int>((int)((n_win + warps - 1) / warps), ctx->num_sms * 4));
    const int stack_cap = 256 * std::max(1, t->n_levels) + 32;
    CeilArgs a;
    a.nodes = t->nodes; a.src = t->src; a.ssoft = t->ssoft;
    a.wins = wins; a.n_win = (int)n_win; a.window = window; a.n_live = t->n_live;
    a.amag = amag; a.nq2 = t->nq2; a.alpha = alpha; a.eps = eps; a.cost_exp = cost_exp; a.rho_lo = rho_lo; a.rho_hi = rho_hi; a.mode = mode;
    a.stack = (int*)scratch(ctx, kSlotStack, (size_t)blocks * warps * stack_cap * 4);
    a.stack_cap = stack_cap;
    unsigned long long* ctr = (unsigned long long*)scratch(ctx, kSlotCounters, 256);
    a.next = (unsigned*)ctr;
    a.error = (int*)(ctr + 1);
    a.ax = ax; a.ay = ay; a.az = az; a.counts = counts;
    check_cuda(cudaMemsetAsync(ctr, 0, 16, st), "memset");
    ceiling_kernel<<<blocks, warps * 32, 0, st>>>(a);
    check_launch(ctx, "ceiling_kernel");
    int err = 0;
    check_cuda(cudaMemcpyAsync(ctx->pinned, ctr + 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    std::memcpy(&err, ctx->pinned, 4);
    if (err) throw Fail{GT_ERR_OVERFLOW, "exact-label walk stack overflow"};
}

void run_mac_sample(gt_context* ctx, const gt_tree* t, const double* amag, double alpha, int window,
                    int64_t stride, double rho_lo, double rho_hi, int64_t cap, float* feat,
                    float* label, float* rho, int64_t* n_samples) {
    cudaStream_t st = ctx->stream;
    const int64_t nl = t->n_live;
    const int64_t nwin = (nl + window - 1) / window;
    std::vector<int2> hg;
    for (int64_t w = 0; w < nwin; w += std::max<int64_t>(stride, 1))
        hg.push_back(make_int2((int)(w * window), (int)std::min<int64_t>((w + 1) * window, nl)));
    *n_samples = 0;
    if (hg.empty()) return;
    int2* dg = (int2*)scratch(ctx, kSlotGroupsB, hg.size() * sizeof(int2));
    check_cuda(cudaMemcpyAsync(dg, hg.data(), hg.size() * sizeof(int2), cudaMemcpyHostToDevice, st), "H2D");
    const int warps = 8;
    const int blocks = std::max(1, std::min<int>((int)((hg.size() + warps - 1) / warps), ctx->num_sms * 4));
    const int stack_cap = 256 * std::max(1, t->n_levels) + 32;
    SampleArgs a;
    a.nodes = t->nodes; a.src = t->src; a.ssoft = t->ssoft; a.nq2 = t->nq2;
    a.groups = dg; a.n_groups = (int)hg.size();
    a.amag = amag; a.alpha = alpha; a.rho_lo = rho_lo; a.rho_hi = rho_hi;
    a.stack = (int*)scratch(ctx, kSlotStack, (size_t)blocks * warps * stack_cap * 4);
    a.stack_cap = stack_cap;
    unsigned long long* ctr = (unsigned long long*)scratch(ctx, kSlotCounters, 256);
    a.count = ctr;
    a.next_group = (unsigned*)(ctr + 1);
    a.error = (int*)(ctr + 2);
    a.feat = feat; a.label = label; a.rho = rho; a.cap = cap;
    check_cuda(cudaMemsetAsync(ctr, 0, 32, st), "memset");
    mac_sample_kernel<<<blocks, warps * 32, 0, st>>>(a);
    check_launch(ctx, "mac_sample_kernel");
    unsigned long long h[3];
    check_cuda(cudaMemcpyAsync(ctx->pinned, ctr, 24, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    std::memcpy(h, ctx->pinned, 24);
    if ((int)h[2]) throw Fail{GT_ERR_OVERFLOW, "sampling walk stack overflow"};
    *n_samples = (int64_t)h[0];
}

void run_mac_grad(gt_context* ctx, const float* dmodel, const float* X, const float* Y, const int* perm,
                  int64_t off, int B, double tau, float* dgrad, double* loss) {
    cudaStream_t st = ctx->stream;
    float* act = (float*)scratch(ctx, kSlotNodeTmp0, (size_t)B * kActStride * 4);
    const int nb = div_up(B, 256);
    double* lp = (double*)scratch(ctx, kSlotPartials, (size_t)nb * 8);
    mlp_fwd_bwd_kernel<<<nb, 256, 0, st>>>(dmodel, X, Y, perm, off, B, (float)tau, act, lp);
    check_launch(ctx, "mlp_fwd_bwd_kernel");
    mlp_grad_kernel<<<kMacParams, 128, 0, st>>>(act, B, dgrad);
    check_launch(ctx, "mlp_grad_kernel");
    if (loss) {
        std::vector<double> h((size_t)nb);
        check_cuda(cudaMemcpyAsync(h.data(), lp, (size_t)nb * 8, cudaMemcpyDeviceToHost, st), "D2H");
        check_cuda(cudaStreamSynchronize(st), "sync");
        double s = 0;
        for (double v : h) s += v;
        *loss = s / std::max(B, 1);
    }
}

void run_mac_train(gt_context* ctx, int64_t n, const float* X, const float* Y,
                   const gt_mac_train_options& o, float* model_host, double* loss_out) {
    cudaStream_t st = ctx->stream;
    if (n <= 0) throw Fail{GT_ERR_INVALID, "no training samples"};
    float* dmodel = (float*)scratch(ctx, kSlotOut3, kMacModel * 4);
    float* dgrad = (float*)scratch(ctx, kSlotOut2, kMacParams * 4 * 3);
    float* dm = dgrad + kMacParams;
    float* dv = dm + kMacParams;
    // normalisation from the data, output bias from the label median
    feat_stats_kernel<<<kMacIn, 256, 0, st>>>(X, n, dmodel);
    check_launch(ctx, "feat_stats_kernel");
    std::vector<float> hy((size_t)n);
    check_cuda(cudaMemcpyAsync(hy.data(), Y, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaMemcpyAsync(model_host, dmodel, kMacNorm * 4, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    for (int i = 0; i < kMacIn; ++i)
        if (!((o.feature_mask >> i) & 1u)) { model_host[i] = 0.0f; model_host[kMacIn + i] = 0.0f; }
    std::vector<float> ys = hy;
    std::nth_element(ys.begin(), ys.begin() + (ptrdiff_t)(o.tau * (n - 1)), ys.end());
    init_params(model_host, o.seed, ys[(size_t)(o.tau * (n - 1))]);
    check_cuda(cudaMemcpyAsync(dmodel, model_host, kMacModel * 4, cudaMemcpyHostToDevice, st), "H2D");
    check_cuda(cudaMemsetAsync(dm, 0, kMacParams * 8, st), "memset");
    std::vector<int> perm((size_t)n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(o.seed * 7919 + 1);
    int* dperm = (int*)scratch(ctx, kSlotNodeTmp1, (size_t)n * 4);
    const int B = (int)std::min<int64_t>(std::max(o.batch, 32), n);
    const float b1 = 0.9f, b2 = 0.999f;
    int step = 0;
    double epoch_loss = 0;
    for (int ep = 0; ep < o.epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        check_cuda(cudaMemcpyAsync(dperm, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st), "H2D");
        const bool last = ep + 1 == o.epochs;
        double lsum = 0;
        int64_t lcount = 0;
        for (int64_t off = 0; off + B <= n; off += B) {
            ++step;
            double l = 0;
            run_mac_grad(ctx, dmodel, X, Y, dperm, off, B, o.tau, dgrad, last ? &l : nullptr);
            if (last) { lsum += l * B; lcount += B; }
            const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
            adam_kernel<<<div_up(kMacParams, 256), 256, 0, st>>>(dmodel + kMacNorm, dgrad, dm, dv, kMacParams,
                                                                 (float)o.lr, b1, b2, c1, c2);
            check_launch(ctx, "adam_kernel");
        }
        if (last) epoch_loss = lcount ? lsum / lcount : 0.0;
    }
    check_cuda(cudaMemcpyAsync(model_host, dmodel, kMacModel * 4, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    if (loss_out) *loss_out = epoch_loss;
}

void run_mac_predict(gt_context* ctx, const float* dmodel, int64_t n, const float* X, float* out) {
    if (n <= 0) return;
    mlp_predict_kernel<<<std::max(1, std::min(div_up(n, 256), ctx->num_sms * 8)), 256, 0, ctx->stream>>>(
        dmodel, X, n, out);
    check_launch(ctx, "mlp_predict_kernel");
}

// ---- per-node criterion (GT_MAC_NODE) ---------------------------------------------------------
namespace {

// l2[i] = len^2 * 10^(c(node) - log10 kappa): the relative arm's M L^2 with the node's learned
// correction folded in, so the walk tests M * l2 > r^4 aold exactly as the plain criterion does.
__global__ void mac_node_scale_kernel(const GNode* __restrict__ nodes, const float* __restrict__ nq2,
                                      int64_t n_nodes, const float* __restrict__ model, float log_kappa,
                                      float* __restrict__ l2) {
    __shared__ float m[kMacModel];
    for (int i = threadIdx.x; i < kMacModel; i += blockDim.x) m[i] = model[i];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        const GNode nd = nodes[i];
        float f[kMacIn];
        mac_node_features((double)nd.len, nd.s, nd.mass, (double)nq2[i], nd.phi - nd.plo, f);
        const float c = mac_forward(m, f);
        const double len = (double)nd.len;
        l2[i] = (float)(len * len * (double)exp10f(c - log_kappa));
    }
}

}  // namespace

void run_mac_node_scale(gt_context* ctx, const gt_tree* t, const float* dmodel, double kappa, float* l2) {
    if (t->n_nodes <= 0) return;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(t->n_nodes, 256), ctx->num_sms * 4));
    mac_node_scale_kernel<<<blocks, 256, 0, ctx->stream>>>(t->nodes, t->nq2, t->n_nodes, dmodel,
                                                           (float)std::log10(kappa), l2);
    check_launch(ctx, "mac_node_scale_kernel");
}

}  // namespace gt
