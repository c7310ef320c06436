// Autotuner of the all-active grouped walk (gt_autotune).
//
// The walk's speed depends on the group shape and size (fixed windows in tree order, node
// groups, leaf groups), on the warps per block and on the interaction-list capacity (longer lists
// amortise the flushes but take shared memory, hence blocks per SM).  Group size also changes the
// result: a group opens nodes for its nearest member with its smallest aold (the reference's
// conservative batch rule, shmem/tree.cc:682-702), so larger groups are more accurate and slower.
// The tuner therefore measures each candidate's device time and, given a sample with FP64
// reference accelerations, its sampled median and p99 relative error; it picks the fastest
// candidate whose p99 meets the target.  The learned criterion is tried the same way, so it is
// used only where it is accepted and faster, and the plain criterion remains the fallback.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gt_internal.cuh"

namespace gt {
namespace {

__global__ void gather_sample_kernel(const double* __restrict__ ax, const double* __restrict__ ay,
                                     const double* __restrict__ az, const uint32_t* __restrict__ rank,
                                     const uint32_t* __restrict__ sample, int64_t ns, int64_t n_live,
                                     double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = rank[sample[i]];
        const bool ok = (int64_t)p < n_live;  // massless particles have no tree position
        out[3 * i] = ok ? ax[p] : NAN;
        out[3 * i + 1] = ok ? ay[p] : NAN;
        out[3 * i + 2] = ok ? az[p] : NAN;
    }
}

// q-quantile of sorted values with linear interpolation between order statistics (numpy's default)
double quantile_sorted(const std::vector<double>& v, double q) {
    if (v.empty()) return -1.0;
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] + f * (v[i + 1] - v[i]) : v[i];
}

struct DevArr {
    void* p = nullptr;
    ~DevArr() { if (p) cudaFree(p); }
    void alloc(size_t bytes) { check_cuda(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc tuner buffer"); }
};

}  // namespace

void run_autotune(gt_context* ctx, const gt_tree* t, const double* aold, double theta, double G,
                  const TuneRequest& tr, std::vector<gt_tune_entry>& entries, gt_tune_entry& best) {
    cudaStream_t st = ctx->stream;
    const int64_t nl = t->n_live;
    if (nl <= 0) throw Fail{GT_ERR_INVALID, "the tree has no live particles"};
    DevArr bx, by, bz, samp, gath;
    bx.alloc((size_t)nl * 8); by.alloc((size_t)nl * 8); bz.alloc((size_t)nl * 8);
    const int64_t ns = tr.n_sample;
    std::vector<double> host((size_t)std::max<int64_t>(ns, 1) * 3);
    if (ns > 0) {
        samp.alloc((size_t)ns * 4);
        gath.alloc((size_t)ns * 24);
        check_cuda(cudaMemcpyAsync(samp.p, tr.sample, (size_t)ns * 4, cudaMemcpyHostToDevice, st), "h2d");
    }
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } guard{e0, e1};

    auto measure = [&](gt_tune_entry c) {
        WalkRequest rq;
        rq.aold = aold;
        rq.theta = theta;
        rq.G = G;
        rq.group_mode = c.group_mode;
        rq.group_param = c.group_size;
        rq.leaf_accept = true;
        rq.ax = (double*)bx.p; rq.ay = (double*)by.p; rq.az = (double*)bz.p;
        rq.block_warps = c.block_warps;
        rq.list_capacity = c.list_capacity;
        rq.mac = c.mac;
        if (c.mac != GT_MAC_PLAIN) {
            rq.mac_model = tr.mac_model;
            rq.mac_kappa = c.mac_kappa;
            rq.mac_band_lo = tr.mac_band[0];
            rq.mac_band_hi = tr.mac_band[1];
        }
        run_walk(ctx, t, rq);  // warm-up: group list, kernel attributes
        std::vector<float> ms;
        for (int r = 0; r < std::max(1, tr.reps); ++r) {
            check_cuda(cudaEventRecord(e0, st), "event");
            run_walk(ctx, t, rq);
            check_cuda(cudaEventRecord(e1, st), "event");
            check_cuda(cudaEventSynchronize(e1), "sync");
            float v = 0;
            check_cuda(cudaEventElapsedTime(&v, e0, e1), "elapsed");
            ms.push_back(v);
        }
        std::sort(ms.begin(), ms.end());
        c.ms = ms[ms.size() / 2];
        c.p99 = c.median = -1.0;
        c.accepted = 1;
        if (ns > 0) {
            gather_sample_kernel<<<std::max(1, std::min(div_up(ns, 256), ctx->num_sms * 4)), 256, 0, st>>>(
                (double*)bx.p, (double*)by.p, (double*)bz.p, t->rank, (const uint32_t*)samp.p, ns, nl,
                (double*)gath.p);
            check_launch(ctx, "gather_sample_kernel");
            check_cuda(cudaMemcpyAsync(host.data(), gath.p, (size_t)ns * 24, cudaMemcpyDeviceToHost, st), "d2h");
            check_cuda(cudaStreamSynchronize(st), "sync");
            std::vector<double> err;
            err.reserve((size_t)ns);
            for (int64_t i = 0; i < ns; ++i) {
                const double rx = tr.ref_ax[i], ry = tr.ref_ay[i], rz = tr.ref_az[i];
                const double dx = host[3 * i] - rx, dy = host[3 * i + 1] - ry, dz = host[3 * i + 2] - rz;
                const double nr = std::sqrt(rx * rx + ry * ry + rz * rz);
                const double e = std::sqrt(dx * dx + dy * dy + dz * dz) / (nr > 0 ? nr : 1.0);
                err.push_back(std::isfinite(e) ? e : 1e300);
            }
            std::sort(err.begin(), err.end());
            c.median = quantile_sorted(err, 0.5);
            c.p99 = quantile_sorted(err, 0.99);
            c.accepted = c.p99 <= tr.p99_max;
        }
        entries.push_back(c);
        return c;
    };
    auto better = [](const gt_tune_entry& a, const gt_tune_entry& b) {  // a preferred over b
        if (a.accepted != b.accepted) return a.accepted > b.accepted;
        if (a.accepted) return a.ms < b.ms;
        return a.p99 < b.p99;
    };
    auto candidate = [](int mode, int size, int warps, int cap) {
        gt_tune_entry c;
        std::memset(&c, 0, sizeof(c));
        c.group_mode = mode; c.group_size = size; c.block_warps = warps; c.list_capacity = cap;
        c.mac = GT_MAC_PLAIN;
        return c;
    };

    // 1. group shape and size at the default block shape
    std::vector<gt_tune_entry> shape;
    for (int b : {16, 32, 64, 128}) shape.push_back(measure(candidate(GT_GROUP_BATCH, b, 8, 256)));
    for (int gmax : {32, 64}) shape.push_back(measure(candidate(GT_GROUP_NODE, gmax, 8, 256)));
    shape.push_back(measure(candidate(GT_GROUP_LEAF, 0, 8, 256)));
    std::sort(shape.begin(), shape.end(), better);
    best = shape[0];
    // 2. block shape and list capacity for the two best shapes
    for (size_t k = 0; k < std::min<size_t>(2, shape.size()); ++k) {
        for (int warps : {4, 8})
            for (int cap : {128, 256, 512}) {
                if (warps == 8 && cap == 256) continue;  // measured in stage 1
                const gt_tune_entry c =
                    measure(candidate(shape[k].group_mode, shape[k].group_size, warps, cap));
                if (better(c, best)) best = c;
            }
    }
    // 3. the learned criterion on the best configuration (the gas pair rule takes the plain one)
    if (tr.mac_model && !(t->szeta && t->gas_zeta)) {
        for (double kap : tr.kappa) {
            gt_tune_entry c = best;
            c.mac = tr.mac_mode;
            c.mac_kappa = kap;
            c = measure(c);
            if (better(c, best)) best = c;
        }
    }
}

}  // namespace gt
