// Tree reuse between rebuilds: the incremental node moments of shmem/tree.cc:211-274 and
// tree.h:286-331 (GIZMO's force_update_tree / force_kick_node / force_drift_node), on the device.
//
// Each node keeps its build-time mass m0 and centre of mass C0.  Since the build it accumulates
// a mass change dm, a momentum change dp and a first-moment change dq, so that at time tau since
// the build
//     M(tau) = m0 + dm,    COM(tau) = (m0 C0 + (m0 vcom + dp) tau - dq) / M(tau),
// which is exact for particles moving ballistically between kicks (a kick of dp at tau_k adds
// dp (tau - tau_k) to the first moment, so dq gathers dp tau_k).  The opening radius and side of
// the walk node grow by 2 (vmax tau + xpad): every particle may have moved that far.
//
// Events arrive as arrays.  Kicks, shifts and the speed/softening bounds commute, so one thread
// per event climbs the parent chain with atomics (a call with many kicks or shifts sums them per
// leaf and carries the sums up level by level instead); mass events and displacement pads depend on the
// order of earlier events (the centre of mass they read, the pad they add to), so one thread
// applies them in array order, as the reference's serial callers do.
#include <algorithm>
#include <cstring>

#include "gt_internal.cuh"

namespace gt {
namespace {

constexpr int kBlk = 256;
constexpr int64_t kLevelSumEvents = 1 << 16;  // kicks / shifts per call from which sums go up by level

int grid_of(gt_context* ctx, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + kBlk - 1) / kBlk, (int64_t)ctx->num_sms * 8));
}

__device__ __forceinline__ double min_image(double s, double box) {
    if (box > 0) {
        if (s > 0.5 * box) s -= box;
        else if (s < -0.5 * box) s += box;
    }
    return s;
}

// atomic max of a non-negative float through its bit pattern (monotonic for x >= 0)
__device__ __forceinline__ void atomic_max_nonneg(float* slot, float v) {
    atomicMax(reinterpret_cast<unsigned int*>(slot), __float_as_uint(v));
}

__device__ __forceinline__ void atomic_max_double_nonneg(double* slot, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(slot), (unsigned long long)__double_as_longlong(v));
}

// A float at least h (rounded up), so a bound kept in float stays one-sided.
__device__ __forceinline__ float up_float(double h) {
    const float f = __double2float_rn(h);
    return ((double)f < h) ? nextafterf(f, 1e30f) : f;
}

struct Moments {
    const double *m0, *c0, *vcom;
    double *dp, *dq, *dmass;
};

__device__ __forceinline__ double node_mass(const Moments& S, int no) { return S.m0[no] + S.dmass[no]; }

__device__ void node_com(const Moments& S, int no, double tau, double* c) {
    const double M = node_mass(S, no);
    const double m0 = S.m0[no];
    if (!S.vcom || M <= 0) {
        for (int k = 0; k < 3; ++k) c[k] = S.c0[3 * no + k];
        return;
    }
    for (int k = 0; k < 3; ++k)
        c[k] = (m0 * S.c0[3 * no + k] + (m0 * S.vcom[3 * no + k] + S.dp[3 * no + k]) * tau - S.dq[3 * no + k]) / M;
}

// kick_node (tree.cc:211-226): dp and dp tau into every ancestor
__global__ void kick_kernel(const int* __restrict__ parent, const int* __restrict__ leaf, const double* __restrict__ dp,
                            int64_t n, double tau, double* __restrict__ adp, double* __restrict__ adq) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double px = dp[3 * e], py = dp[3 * e + 1], pz = dp[3 * e + 2];
        for (int no = leaf[e]; no >= 0; no = parent[no]) {
            atomicAdd(adp + 3 * no, px); atomicAdd(adp + 3 * no + 1, py); atomicAdd(adp + 3 * no + 2, pz);
            atomicAdd(adq + 3 * no, px * tau); atomicAdd(adq + 3 * no + 1, py * tau); atomicAdd(adq + 3 * no + 2, pz * tau);
        }
    }
}

// shift_node (tree.cc:248-253): a displacement dx of a particle of mass m, no velocity change
__global__ void shift_kernel(const int* __restrict__ parent, const int* __restrict__ leaf, const double* __restrict__ m,
                             const double* __restrict__ dx, int64_t n, double* __restrict__ adq) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double a = m[e] * dx[3 * e], b = m[e] * dx[3 * e + 1], c = m[e] * dx[3 * e + 2];
        for (int no = leaf[e]; no >= 0; no = parent[no]) {
            atomicAdd(adq + 3 * no, -a); atomicAdd(adq + 3 * no + 1, -b); atomicAdd(adq + 3 * no + 2, -c);
        }
    }
}

// Many kicks or shifts at once: climbing the chain per event would send every event's six
// atomics to the root and the other top nodes, where they serialise.  Instead the events are first
// summed into their leaves (a few events per leaf), the sums are carried up one level at a time
// (a node adds its contiguous children), and every node then takes its total once.  kind 0: kick
// (a = dp, 3 per event); kind 1: shift (a = m, x = dx, 3 per event).
__global__ void leaf_sum_kernel(const int* __restrict__ leaf, const double* __restrict__ a, const double* __restrict__ x,
                                int64_t n, int kind, double* __restrict__ acc) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int lf = leaf[e];
        if (lf < 0) continue;
        for (int k = 0; k < 3; ++k) {
            const double v = kind == 0 ? a[3 * e + k] : -a[e] * x[3 * e + k];
            atomicAdd(acc + 3 * lf + k, v);
        }
    }
}

__global__ void level_sum_kernel(const GNode* __restrict__ nodes, int64_t lo, int64_t hi, double* __restrict__ acc) {
    for (int64_t i = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += (int64_t)gridDim.x * blockDim.x) {
        const int f = nodes[i].first, nc = nodes[i].nchild;
        if (f < 0) continue;
        double s0 = acc[3 * i], s1 = acc[3 * i + 1], s2 = acc[3 * i + 2];
        for (int c = f; c < f + nc; ++c) {
            s0 += acc[3 * c]; s1 += acc[3 * c + 1]; s2 += acc[3 * c + 2];
        }
        acc[3 * i] = s0; acc[3 * i + 1] = s1; acc[3 * i + 2] = s2;
    }
}

// kick: dp += sum, dq += sum tau; shift: dq += sum (the sum already carries -m dx)
__global__ void apply_sum_kernel(int64_t nn, const double* __restrict__ acc, int kind, double tau,
                                 double* __restrict__ adp, double* __restrict__ adq) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * nn; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = acc[i];
        if (kind == 0) {
            adp[i] += v;
            adq[i] += v * tau;
        } else {
            adq[i] += v;
        }
    }
}

// raise_vmax (tree.cc:276-284): climb while an ancestor does not already cover the speed
__global__ void raise_vmax_kernel(const int* __restrict__ parent, const int* __restrict__ leaf,
                                  const float* __restrict__ speed, int64_t n, float* __restrict__ vmax) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float s = speed[e];
        for (int no = leaf[e]; no >= 0; no = parent[no]) {
            if (__float_as_uint(vmax[no]) >= __float_as_uint(s)) break;
            atomic_max_nonneg(vmax + no, s);
        }
    }
}

// raise_soft (tree.cc:310-319): the node's float and double softening bounds
__global__ void raise_soft_kernel(const int* __restrict__ parent, const int* __restrict__ leaf,
                                  const double* __restrict__ soft, int64_t n, GNode* __restrict__ nodes,
                                  double* __restrict__ nsoft) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double sd = soft[e];
        const float sf = up_float(sd);
        for (int no = leaf[e]; no >= 0; no = parent[no]) {
            if (nodes[no].soft >= sf) break;
            atomic_max_nonneg(&nodes[no].soft, sf);
            atomic_max_double_nonneg(nsoft + no, sd);
        }
    }
}

// mass_event (tree.cc:229-246) and raise_pad (tree.cc:322-329), in array order.  kind 0: mass
// event (dm, x, v); kind 1: pad d.
__global__ void serial_events_kernel(const int* __restrict__ parent, const int* __restrict__ leaf, int kind,
                                     const double* __restrict__ a, const double* __restrict__ x,
                                     const double* __restrict__ v, int64_t n, double tau, double box, Moments S,
                                     float* __restrict__ xpad) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int64_t e = 0; e < n; ++e) {
        const int lf = leaf[e];
        if (lf < 0) continue;
        if (kind == 0) {
            const double dm = a[e];
            if (dm == 0.0) continue;
            for (int no = lf; no >= 0; no = parent[no]) {
                double c[3];
                node_com(S, no, tau, c);
                S.dmass[no] += dm;
                for (int k = 0; k < 3; ++k) {
                    const double xr = c[k] + min_image(x[3 * e + k] - c[k], box);
                    S.dp[3 * no + k] += dm * v[3 * e + k];
                    S.dq[3 * no + k] -= dm * (xr - v[3 * e + k] * tau);
                }
            }
        } else {
            const double d = a[e];
            if (!(d > 0)) continue;
            const float pad = up_float((double)xpad[lf] + d);
            for (int no = lf; no >= 0; no = parent[no]) {
                if (xpad[no] >= pad) break;
                xpad[no] = pad;
            }
        }
    }
}

// refresh_walk_nodes (tree.cc:256-274): the walk nodes from the incremental moments; also the
// node velocity the jerk reads (tree.h:333-341)
__global__ void refresh_kernel(GNode* __restrict__ nodes, int64_t nn, Moments S, const double* __restrict__ size,
                               const double* __restrict__ delta, const float* __restrict__ vmax,
                               const float* __restrict__ xpad, double tau, int nodelta, float4* __restrict__ nvel) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const int no = (int)i;
        double c[3];
        node_com(S, no, tau, c);
        GNode& w = nodes[i];
        w.cx = c[0]; w.cy = c[1]; w.cz = c[2];
        const double M = node_mass(S, no);
        w.mass = M;
        const double grow = 2.0 * ((double)vmax[i] * tau + (double)xpad[i]);
        w.s = size[i] + (nodelta ? 0.0 : delta[i]) + grow;
        w.len = (float)(size[i] + grow);
        if (nvel && S.vcom) {
            double v[3];
            const double m0 = S.m0[no];
            for (int k = 0; k < 3; ++k)
                v[k] = M > 0 ? (m0 * S.vcom[3 * no + k] + S.dp[3 * no + k]) / M : S.vcom[3 * no + k];
            nvel[i] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.0f);
        }
    }
}

__global__ void copy_base_kernel(const GNode* __restrict__ nodes, int64_t nn, double* __restrict__ m0,
                                 double* __restrict__ c0) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        m0[i] = nodes[i].mass;
        c0[3 * i] = nodes[i].cx; c0[3 * i + 1] = nodes[i].cy; c0[3 * i + 2] = nodes[i].cz;
    }
}

__global__ void node_state_kernel(int64_t nn, Moments S, double tau, double* __restrict__ com,
                                  double* __restrict__ vel, double* __restrict__ mass) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const int no = (int)i;
        double c[3];
        node_com(S, no, tau, c);
        const double M = node_mass(S, no);
        for (int k = 0; k < 3; ++k) {
            com[3 * i + k] = c[k];
            if (S.vcom) vel[3 * i + k] = M > 0 ? (S.m0[no] * S.vcom[3 * i + k] + S.dp[3 * i + k]) / M : S.vcom[3 * i + k];
            else vel[3 * i + k] = 0.0;
        }
        mass[i] = M;
    }
}

// current particle state into tree order (positions, masses, softenings; null keeps the value)
__global__ void particles_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, const double* __restrict__ m,
                                 const double* __restrict__ soft, const uint32_t* __restrict__ order, int64_t nl,
                                 SrcP* __restrict__ src, double* __restrict__ ssoft, double* __restrict__ smass) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = order[i];
        SrcP r = src[i];
        if (x) { r.x = x[p]; r.y = y[p]; r.z = z[p]; }
        if (m) { r.m = (float)m[p]; smass[i] = m[p]; }
        if (soft) { r.soft = (float)soft[p]; ssoft[i] = soft[p]; }
        src[i] = r;
    }
}

template <typename T>
T* zeroed(size_t count, cudaStream_t st) {
    void* p = nullptr;
    const cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Fail{GT_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e)};
    }
    check_cuda(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), st), "memset");
    return (T*)p;
}

Moments moments_of(const gt_tree* t) {
    Moments S;
    S.m0 = t->m0; S.c0 = t->c0; S.vcom = t->vcom;
    S.dp = t->dp; S.dq = t->dq; S.dmass = t->dmass;
    return S;
}

}  // namespace

void reuse_begin(gt_context* ctx, gt_tree* t) {
    if (t->m0) return;
    cudaStream_t st = ctx->stream;
    const int64_t nn = std::max<int64_t>(t->n_nodes, 1);
    t->m0 = zeroed<double>((size_t)nn, st);
    t->c0 = zeroed<double>((size_t)nn * 3, st);
    t->dp = zeroed<double>((size_t)nn * 3, st);
    t->dq = zeroed<double>((size_t)nn * 3, st);
    t->dmass = zeroed<double>((size_t)nn, st);
    t->xpad = zeroed<float>((size_t)nn, st);
    if (!t->vmax) t->vmax = zeroed<float>((size_t)nn, st);
    if (t->n_nodes > 0) {
        copy_base_kernel<<<grid_of(ctx, t->n_nodes), kBlk, 0, st>>>(t->nodes, t->n_nodes, t->m0, t->c0);
        check_launch(ctx, "copy_base_kernel");
    }
}

void reuse_events(gt_context* ctx, gt_tree* t, int kind, int64_t n, const int* leaf, const double* a,
                  const double* x, const double* v, const float* f, double tau, double box) {
    reuse_begin(ctx, t);
    if (n <= 0) return;
    cudaStream_t st = ctx->stream;
    const bool have_vcom = t->vcom != nullptr;  // the momentum arrays exist only with vcom (tree.cc:212)
    switch (kind) {
        case kReuseKick:
        case kReuseShift:
            if (!have_vcom) return;
            if (n >= kLevelSumEvents) {
                const int k = kind == kReuseKick ? 0 : 1;
                const int64_t nn = t->n_nodes;
                double* acc = (double*)scratch(ctx, kSlotNodeTmp1, (size_t)std::max<int64_t>(nn, 1) * 24);
                check_cuda(cudaMemsetAsync(acc, 0, (size_t)std::max<int64_t>(nn, 1) * 24, st), "memset");
                leaf_sum_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(leaf, a, x, n, k, acc);
                check_launch(ctx, "leaf_sum_kernel");
                for (int L = t->n_levels - 1; L >= 0; --L) {
                    const int64_t lo = t->lvl_off[L], hi = t->lvl_off[L + 1];
                    level_sum_kernel<<<grid_of(ctx, hi - lo), kBlk, 0, st>>>(t->nodes, lo, hi, acc);
                    check_launch(ctx, "level_sum_kernel");
                }
                apply_sum_kernel<<<grid_of(ctx, 3 * nn), kBlk, 0, st>>>(nn, acc, k, tau, t->dp, t->dq);
                check_launch(ctx, "apply_sum_kernel");
            } else if (kind == kReuseKick) {
                kick_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(t->parent, leaf, a, n, tau, t->dp, t->dq);
                check_launch(ctx, "kick_kernel");
            } else {
                shift_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(t->parent, leaf, a, x, n, t->dq);
                check_launch(ctx, "shift_kernel");
            }
            break;
        case kReuseVmax:
            raise_vmax_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(t->parent, leaf, f, n, t->vmax);
            check_launch(ctx, "raise_vmax_kernel");
            break;
        case kReuseSoft:
            raise_soft_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(t->parent, leaf, a, n, t->nodes, t->nsoft);
            check_launch(ctx, "raise_soft_kernel");
            break;
        case kReuseMass:
            if (!have_vcom) return;
            serial_events_kernel<<<1, 1, 0, st>>>(t->parent, leaf, 0, a, x, v, n, tau, box, moments_of(t), t->xpad);
            check_launch(ctx, "serial_events_kernel");
            break;
        case kReusePad:
            serial_events_kernel<<<1, 1, 0, st>>>(t->parent, leaf, 1, a, nullptr, nullptr, n, tau, box,
                                                  moments_of(t), t->xpad);
            check_launch(ctx, "serial_events_kernel");
            break;
        default:
            throw Fail{GT_ERR_INVALID, "unknown tree event kind"};
    }
}

void reuse_refresh(gt_context* ctx, gt_tree* t, double tau) {
    reuse_begin(ctx, t);
    if (t->n_nodes <= 0) return;
    refresh_kernel<<<grid_of(ctx, t->n_nodes), kBlk, 0, ctx->stream>>>(t->nodes, t->n_nodes, moments_of(t), t->size,
                                                                       t->delta, t->vmax, t->xpad, tau, t->opt.nodelta,
                                                                       t->nvel);
    check_launch(ctx, "refresh_kernel");
}

void reuse_node_state(gt_context* ctx, gt_tree* t, double tau, double* com, double* vel, double* mass) {
    reuse_begin(ctx, t);
    if (t->n_nodes <= 0) return;
    node_state_kernel<<<grid_of(ctx, t->n_nodes), kBlk, 0, ctx->stream>>>(t->n_nodes, moments_of(t), tau, com, vel,
                                                                           mass);
    check_launch(ctx, "node_state_kernel");
}

void tree_particles(gt_context* ctx, gt_tree* t, const double* x, const double* y, const double* z,
                    const double* m, const double* soft) {
    if (t->n_live <= 0) return;
    particles_kernel<<<grid_of(ctx, t->n_live), kBlk, 0, ctx->stream>>>(x, y, z, m, soft, t->order, t->n_live,
                                                                        t->src, t->ssoft, t->smass);
    check_launch(ctx, "particles_kernel");
}

}  // namespace gt
