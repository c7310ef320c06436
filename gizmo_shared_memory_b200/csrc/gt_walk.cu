// Group tree walk on the device: the replacement for shmem::accel_grouped (shmem/tree.cc:626-897),
// shmem::accel (tree.cc:528-582) and shmem::potential (tree.cc:899-944).
//
// One warp walks the tree for one group of targets (a leaf's targets, a fixed window, a group
// node's particles, or a single target) and applies the result to all of them:
//
//   * Group reduction (FP64, warp shuffles): bounding box, largest target softening, smallest aold
//     -- the conservative per-group inputs of the reference's batch walk (tree.cc:682-702).
//   * Traversal: a per-warp LIFO of node indices.  Each step pops up to 32 nodes, one per lane,
//     loads each 64-byte node with four 16-byte loads and evaluates the opening test in FP64 on the
//     group box's nearest point, in the reference's order (shmem/tree.h:109-144; leaves are offered
//     to the criterion first in the grouped walk, tree.cc:751-779, and always expanded in the
//     per-target walks).  Opened interior nodes push their contiguous children (a warp prefix sum
//     gives each lane its slots).  The stack never holds more than 256 entries per tree level: the
//     blocks of entries pushed by one step have strictly increasing minimum depth from bottom to
//     top, and one step pushes at most 32*8.
//   * Interaction list (shared memory, per warp): accepted nodes as monopoles and the particles of
//     expanded leaves, each stored as its FP64 offset from the group centre cast to FP32, FP32 mass
//     and softening.  When the list fills it is evaluated against the group's targets.
//   * Evaluation (FP32): r^2, rsqrt, Newtonian force and potential; the cubic-spline branch only
//     when r < max(h_target, h_source) (shmem/tree.h:59-80).  r^2 == 0 (the target itself, or a
//     coincident particle) contributes nothing, as tree.cc:799-802 skips it.  Full groups store
//     both lists in pairs of entries and evaluate two entries per sm_100 packed FP32 instruction.
//     Groups of <= 16 targets split the list across the idle lanes (lane = slice * NT + target)
//     and reduce the slices at the end.
//   * Accumulation: each list evaluation sums into FP32 partials, which are added into FP32
//     Kahan-compensated totals (acceleration) and an FP64 total (potential); the final sums and
//     the factor G are FP64.
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "gt_internal.cuh"
#include "gt_mac.cuh"

namespace gt {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxWarps = 8;     // warps per block of the walk kernel

// The debug library (make debug: libgt_debug.so, built with -DGT_BOUNDS_CHECK) checks every index
// the walk derives before it is used -- node, particle slot, target position, list slot, output
// index -- and on a violation records error 3 and skips the access.  The ordinary library compiles
// the checks away.
#ifdef GT_BOUNDS_CHECK
#define GT_IN_BOUNDS(i, n) ((i) >= 0 && (int64_t)(i) < (int64_t)(n) ? true : (atomicExch(A.error, 3), false))
#else
#define GT_IN_BOUNDS(i, n) true
#endif
constexpr int kPnCapDefault = 256;  // monopole-list entries per warp (gt_walk_options.list_capacity)
constexpr int kPnCapMax = 1024;     // the particle list holds half as many entries

struct WalkArgs {
    const GNode* nodes;
    const SrcP* src;
    const double* ssoft;
    const uint32_t* tpos;       // target -> tree position; null: identity
    const double* aold;         // per target; null: 0 everywhere
    const int2* groups;         // [start, end) in target index space
    int n_groups;
    const uint32_t* n_groups_dev;  // non-null: the group count, on the device (overrides n_groups)
    double theta2, G;
    double *ax, *ay, *az, *phi;
    const uint32_t* out_map;    // null: write at the target index
    int* stack;
    int stack_cap;
    unsigned int* next_group;   // dynamic group counter
    unsigned long long* stats;  // [nodes, multipole, pairs_structural, zero_r2, flushes, max_stack, steps]
    int* error;                 // 1: stack overflow; 3: an index out of bounds (debug library)
    int64_t n_nodes, n_src, n_out;  // array extents, for the debug library's bounds checks
    int pn_cap, pp_cap;         // list capacities per warp (multiples of 32)
    int warp_bytes;             // shared memory per warp: header + lists
    // learned criterion
    const float* mac_model;     // GT_MAC_MODEL_FLOATS on the device
    const float* nq2;           // node second moments
    double mac_band_lo, mac_band_hi, mac_log_kappa;
    const float* mac_l2;        // GT_MAC_NODE: per-node L^2 10^(c - log10 kappa)
    // tidal tensor (6 per target: xx yy zz xy yz xz, not times G) and jerk (3 per target, times G)
    double* tidal;
    double* jerk;
    const float4* svel;         // particle velocities in tree order (jerk)
    const float4* nvel;         // node centre-of-mass velocities (jerk)
    // forest: root node of each group (its system's root); null: node 0
    const int* group_root;
    // gas and sinks (XT kernel): tree-order type and zeta, FP64 mass; null szeta: no zeta terms.
    // nsink (per node) non-null with sink_r > 0: sink-direct opening.
    const uint8_t* stype;
    const double* szeta;
    const double* smass;
    const uint32_t* nsink;
    double sink_r;
};

__device__ __forceinline__ int warp_incl_scan_i(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

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

struct NodeV {
    double cx, cy, cz, mass, s;
    float len, soft;
    int first, nchild, plo, phi;
};

__device__ __forceinline__ NodeV load_node(const GNode* __restrict__ p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    const int4 c = __ldg(reinterpret_cast<const int4*>(p) + 2);
    const int4 d = __ldg(reinterpret_cast<const int4*>(p) + 3);
    NodeV v;
    v.cx = a.x; v.cy = a.y; v.cz = b.x; v.mass = b.y;
    v.s = __hiloint2double(c.y, c.x);
    v.len = __int_as_float(c.z);
    v.soft = __int_as_float(c.w);
    v.first = d.x; v.nchild = d.y; v.plo = d.z; v.phi = d.w;
    return v;
}

__device__ __forceinline__ void load_src(const SrcP* __restrict__ p, double& x, double& y, double& z,
                                         float& m, float& h) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const int4 b = __ldg(reinterpret_cast<const int4*>(p) + 1);
    x = a.x; y = a.y;
    z = __hiloint2double(b.y, b.x);
    m = __int_as_float(b.z);
    h = __int_as_float(b.w);
}

// The opening test of shmem/tree.h:109-144 in FP64.  Every arm of the reference returns "open" as
// soon as it holds and the last arm decides otherwise, so the test is the OR of the arms: softening
// overlap, Barnes-Hut (theta > 0), relative criterion (aold > 0; with aold == 0 and no theta it
// opens), inside-node.  Evaluated without branches so the lanes of a warp do not diverge.
// ml2 is the relative arm's M L^2 (with the per-node learned correction folded in, GT_MAC_NODE).
__device__ __forceinline__ bool open_node(double r2, double len, double l_open, double ml2,
                                          double nsoft, double tsoft, double aold, double theta2,
                                          double dx, double dy, double dz) {
    const double rt = tsoft + 0.6 * len, rn = nsoft + 0.6 * len;
    const bool overlap = (r2 < rt * rt) | (r2 < rn * rn);
    const bool bh = (theta2 > 0.0) & (l_open * l_open >= theta2 * r2);
    const bool rel = (aold > 0) ? (ml2 > r2 * r2 * aold) : (theta2 <= 0.0);
    const double lim = 0.6 * len;
    const bool inside = (dx < lim) & (dy < lim) & (dz < lim);
    return overlap | bh | rel | inside;
}

// Softened pair inside the kernel (r < h): force factor and potential of the cubic spline,
// shmem/tree.h:59-80, in FP32.  r2 == 0 contributes nothing.
__device__ __noinline__ void spline_pair(float r2, float h, float m, float& f, float& p) {
    if (!(r2 > 0.0f)) { f = 0.0f; p = 0.0f; return; }
    const float r = sqrtf(r2);
    const float hinv = 1.0f / h;
    const float u = r * hinv;
    const float hinv3 = hinv * hinv * hinv;
    if (u < 0.5f) {
        f = m * hinv3 * (10.666666666666667f + u * u * (32.0f * u - 38.4f));
        p = m * hinv * (-2.8f + u * u * (5.333333333333333f + u * u * (6.4f * u - 9.6f)));
    } else {
        const float u3 = u * u * u;
        f = m * hinv3 * (21.333333333333332f - 48.0f * u + 38.4f * u * u - 10.666666666666667f * u3 -
                         0.06666666666666667f / u3);
        p = m * hinv * (-3.2f + 0.06666666666666667f / u +
                        u * u * (10.666666666666667f + u * (-16.0f + u * (9.6f - 2.1333333333333333f * u))));
    }
}

// The same pair inside the kernel plus the second-derivative (tidal) factor g2 of the cubic spline,
// shmem/tree.h:85-96 (GIZMO's kernel_gravity mode 2), in FP32.  r2 == 0 contributes nothing.
__device__ __noinline__ void spline_pair_tidal(float r2, float h, float m, float& f, float& p, float& g2) {
    spline_pair(r2, h, m, f, p);
    if (!(r2 > 0.0f)) { g2 = 0.0f; return; }
    const float hinv = 1.0f / h;
    const float u = sqrtf(r2) * hinv;
    const float hinv2 = hinv * hinv;
    const float hinv5 = hinv2 * hinv2 * hinv;
    float wk;
    if (u < 0.5f) {
        wk = 76.8f - 96.0f * u;
    } else {
        const float u2 = u * u;
        wk = -0.2f / (u2 * u2 * u) + 48.0f / u - 76.8f + 32.0f * u;
    }
    g2 = m * wk * hinv5;
}

// dW/dr / r of the 3-D cubic spline of support h at r < h (shmem/hydro.h:28-32, 46-54):
// (8 / pi) fp(q) / (q h^5), with fp(q) / q = 18 q - 12 below q = 1/2 and -6 (1-q)^2 / q above.
__device__ __forceinline__ float dwdr_over_r(float r, float h) {
    const float hinv = 1.0f / h;
    const float q = r * hinv;
    const float hinv2 = hinv * hinv;
    float g;
    if (q < 0.5f) {
        g = fmaf(18.0f, q, -12.0f);
    } else {
        const float u = 1.0f - q;
        g = -6.0f * u * u / q;
    }
    return 2.5464790894703255f * g * (hinv2 * hinv2 * hinv);
}

// The adaptive-softening terms of a gas-gas pair (shmem/tree.cc:39-53), subtracted from the pair's
// force factor: (zeta_t / m_t) dW/dr(r, h) / r inside h = max(h_t, h_s), plus (zeta_s / m_t)
// dW/dr(r, h_s) / r inside h_s.  ztm = zeta_t / m_t and itm = 1 / m_t are 0 for a target that is not
// gas or has no mass; zs is NaN for a source that is not gas.  r2 == 0 contributes nothing.
__device__ __noinline__ float zeta_pair(float r2, float h, float hs, float zs, float ztm, float itm) {
    if (!(r2 > 0.0f) || zs != zs) return 0.0f;
    const float r = sqrtf(r2);
    float c = 0.0f;
    if (ztm != 0.0f && r < h) c = ztm * dwdr_over_r(r, h);
    if (zs != 0.0f && itm != 0.0f && r < hs) c = fmaf(zs * itm, dwdr_over_r(r, hs), c);
    return c;
}

// 1/sqrt(x) by the PTX approximate reciprocal square root with flush-to-zero.  The monopole loops
// floor r^2 at 1e-30, far above the FP32 subnormal range, and the particle loops take it only for
// r^2 > 0 and r^2 >= h^2 with h the larger softening, a normal number for any h above 1.1e-19.  So
// the result equals rsqrtf's except for two particles closer than 1.1e-19 with softenings below
// that, whose force overflows FP32 either way.  The non-FTZ form only adds subnormal-range scaling
// instructions.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// max(0, |c - mid| - hw): the gap between coordinate c and the group box's interval of centre mid
// and half width hw (0 inside), the nearest-point distance of the reference's batch walk
// (shmem/tree.cc:682-702, max(0, lo - c, c - hi)) up to the rounding of mid and hw, a few ulps of
// the coordinates.  Three FP64 instructions fewer per axis than the two-sided form.  Written with
// a comparison: fmax on doubles costs more instructions (and gives 0 here for a NaN c, as fmax
// does).
__device__ __forceinline__ double box_gap(double c, double mid, double hw) {
    const double g = fabs(c - mid) - hw;
    return g > 0.0 ? g : 0.0;
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float x) {
    const float y = x - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// Per-warp shared memory: this header, then the monopole list (pn_cap float4: offset, mass) and
// the particle list (pp_cap float4 + pp_cap float softenings).  The capacities are a launch
// parameter (the autotuner trades list length against blocks per SM).
struct alignas(16) WarpHdr {
    int lo[32];   // leaf-expansion scratch
    int pre[32];
    // the group's FP64 state, read where needed instead of held in registers for the whole walk:
    // box low/high corners, centre, largest target softening, smallest aold
    double lo_x, lo_y, lo_z, hi_x, hi_y, hi_z, c_x, c_y, c_z, emax, amin;
    double w_x, w_y, w_z;  // half widths of the box
};

// ext 1 (tidal tensor / jerk): the lists also carry each entry's velocity (float4), for the jerk,
// and the particle list each source's zeta (float), for the gas pair rule; ext 2 (gas rules only):
// just the zeta.
__host__ __device__ constexpr int warp_smem_bytes(int pn_cap, int pp_cap, int ext = 0) {
    return ((int)sizeof(WarpHdr) + pn_cap * 16 + pp_cap * 20 +
            (ext == 1 ? (pn_cap + pp_cap) * 16 + pp_cap * 4 : ext == 2 ? pp_cap * 4 : 0) + 15) &
           ~15;
}

// MAC: 0 plain relative criterion, 1 network inside the walk (GT_MAC_LEARNED), 2 per-node
// learned scale (GT_MAC_NODE).  XT 1: also the tidal tensor and/or the jerk (A.tidal, A.jerk), the
// zeta terms of gas-gas pairs (A.szeta) and sink-direct opening (A.nsink); XT 2: the gas rules
// alone, with the packed monopole evaluation of the plain walk.
template <int TPL, bool LEAF_ACCEPT, bool WANT_POT, bool COUNT, int MAC, int XT = 0>
// One target per lane runs at 3 blocks of 8 warps per SM, also with the gas rules (XT 2: 13 %
// faster than at 2 blocks, no spills); the tidal tensor (XT 1) and 2 or 4 targets per lane keep 2.
__global__ void __launch_bounds__(kMaxWarps * 32, (TPL == 1 && XT != 1) ? 3 : 2)
walk_kernel(const WalkArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int gw = blockIdx.x * (blockDim.x >> 5) + w;
    int* __restrict__ stk = A.stack + (size_t)gw * A.stack_cap;
    unsigned char* wbase = smem_raw + (size_t)w * A.warp_bytes;
    WarpHdr& S = *reinterpret_cast<WarpHdr*>(wbase);
    // the learned criterion's network, one copy per block after the warps' lists
    float* __restrict__ mac_w = reinterpret_cast<float*>(smem_raw + (size_t)A.warp_bytes * (blockDim.x >> 5));
    if (MAC == 1) {
        for (int i = threadIdx.x; i < kMacModel; i += blockDim.x) mac_w[i] = A.mac_model[i];
        __syncthreads();
    }
    float4* __restrict__ pn = reinterpret_cast<float4*>(wbase + sizeof(WarpHdr));
    float4* __restrict__ pp = pn + A.pn_cap;
    float* __restrict__ ph = reinterpret_cast<float*>(pp + A.pp_cap);
    float4* __restrict__ pnv = reinterpret_cast<float4*>(ph + A.pp_cap);  // XT 1 only
    float4* __restrict__ ppv = pnv + A.pn_cap;
    // source zeta of the particle list: after the velocities (XT 1) or after the softenings (XT 2)
    float* __restrict__ pzs = XT == 1 ? reinterpret_cast<float*>(ppv + A.pp_cap) : ph + A.pp_cap;
    const bool want_tid = XT == 1 && A.tidal != nullptr;
    const bool want_jerk = XT == 1 && A.jerk != nullptr;
    const bool want_zeta = XT != 0 && A.szeta != nullptr;
    const bool sink_rule = XT != 0 && A.nsink != nullptr;

    unsigned long long c_nodes = 0, c_multi = 0, c_pairs = 0, c_zero = 0, c_flush = 0, c_steps = 0;
    int c_maxtop = 0;
    const int n_groups = A.n_groups_dev ? (int)*A.n_groups_dev : A.n_groups;

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(A.next_group, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= n_groups) break;
        const int2 gr = A.groups[g];
        const int t0 = gr.x, nt = gr.y - gr.x;
        const int nk = TPL > 1 ? min(TPL, (nt + 31) >> 5) : 1;  // targets per lane in use (warp-uniform)

        // ---- targets: lane l holds targets l and l+32 --------------------------------------
        double px[TPL], py[TPL], pz[TPL], ps[TPL];
        double lx = 1e300, ly = 1e300, lz = 1e300, hx = -1e300, hy = -1e300, hz = -1e300;
        double emax = 0.0, amin = A.aold ? 1e300 : 0.0;
#pragma unroll
        for (int k = 0; k < TPL; ++k) {
            px[k] = py[k] = pz[k] = 0.0;
            ps[k] = 0.0;
            const int i = lane + 32 * k;
            if (k < nk && i < nt) {
                int p = A.tpos ? (int)A.tpos[t0 + i] : t0 + i;
                if (!GT_IN_BOUNDS(p, A.n_src)) p = 0;
                float mf, hf;
                load_src(A.src + p, px[k], py[k], pz[k], mf, hf);
                ps[k] = A.ssoft[p];
                lx = fmin(lx, px[k]); hx = fmax(hx, px[k]);
                ly = fmin(ly, py[k]); hy = fmax(hy, py[k]);
                lz = fmin(lz, pz[k]); hz = fmax(hz, pz[k]);
                emax = fmax(emax, ps[k]);
                if (A.aold) amin = fmin(amin, A.aold[t0 + i]);
            }
        }
        lx = wmin(lx); ly = wmin(ly); lz = wmin(lz);
        hx = wmax(hx); hy = wmax(hy); hz = wmax(hz);
        emax = wmax(emax);
        if (A.aold) amin = wmin(amin);
        if (lane == 0) {
            S.lo_x = lx; S.lo_y = ly; S.lo_z = lz; S.hi_x = hx; S.hi_y = hy; S.hi_z = hz;
            S.c_x = 0.5 * (lx + hx); S.c_y = 0.5 * (ly + hy); S.c_z = 0.5 * (lz + hz);
            S.w_x = 0.5 * (hx - lx); S.w_y = 0.5 * (hy - ly); S.w_z = 0.5 * (hz - lz);
            S.emax = emax; S.amin = amin;
        }
        __syncwarp();
        const double gcx = S.c_x, gcy = S.c_y, gcz = S.c_z;

        // ---- evaluation lanes: lane = slice * NT + target ---------------------------------
        int lg = 5;
        if (nt <= 16) lg = 32 - __clz(nt - 1);  // NT = next power of two >= nt (nt >= 1)
        if (nt <= 1) lg = 0;
        const int NT = 1 << lg, NS = 32 >> lg;
        const int ti = lane & (NT - 1), slice = lane >> lg;
        float tx[TPL], ty[TPL], tz[TPL], th[TPL];
        float sx[TPL], sy[TPL], sz[TPL], cxk[TPL], cyk[TPL], czk[TPL];
        double pot[TPL];
#pragma unroll
        for (int k = 0; k < TPL; ++k) {
            const double qx = __shfl_sync(kFull, px[k], ti);
            const double qy = __shfl_sync(kFull, py[k], ti);
            const double qz = __shfl_sync(kFull, pz[k], ti);
            const double qs = __shfl_sync(kFull, ps[k], ti);
            tx[k] = (float)(qx - gcx);
            ty[k] = (float)(qy - gcy);
            tz[k] = (float)(qz - gcz);
            th[k] = (float)qs;
            sx[k] = sy[k] = sz[k] = cxk[k] = cyk[k] = czk[k] = 0.0f;
            pot[k] = 0.0;
        }
        // monopole-list entry pos (paired layout, see flush_pn)
        // The monopole list is paired (see flush_pn) for the packed evaluation of full groups
        // and one float4 per entry otherwise (warp-uniform: the group size decides).
        const bool paired = NS == 1;
        auto pn_put = [&](int pos, float x, float y, float z, float m) {
            if (paired) {
                float* q = reinterpret_cast<float*>(pn + 2 * (pos >> 1)) + (pos & 1);
                q[0] = x; q[2] = y; q[4] = z; q[6] = m;
            } else {
                pn[pos] = make_float4(x, y, z, m);
            }
        };
        // the particle list is paired the same way for full groups of the plain walk (the tidal
        // tensor, the jerk and the gas rules read it one entry at a time)
        const bool ppair = XT == 0 && paired;
        auto pp_put = [&](int pos, float x, float y, float z, float m) {
            float* q = reinterpret_cast<float*>(pp + 2 * (pos >> 1)) + (pos & 1);
            q[0] = x; q[2] = y; q[4] = z; q[6] = m;
        };
        // tidal tensor and jerk: FP64 totals (xx yy zz xy yz xz, jx jy jz) and target velocities;
        // gas targets: zeta / m and 1 / m (0 for a target that is not gas or has no mass,
        // tree.cc:46); a group holding a sink opens by the sink rule (tree.cc:691-698)
        double xt[9][TPL];
        float tvx[TPL], tvy[TPL], tvz[TPL], tzm[TPL], tim[TPL];
        bool has_sink = false;
        if (XT != 0) {
            bool sink = false;
#pragma unroll
            for (int k = 0; k < TPL; ++k) {
#pragma unroll
                for (int c = 0; c < 9; ++c) xt[c][k] = 0.0;
                tvx[k] = tvy[k] = tvz[k] = 0.0f;
                tzm[k] = tim[k] = 0.0f;
                const int i = ti + 32 * k;
                const int p = i < nt ? (A.tpos ? (int)A.tpos[t0 + i] : t0 + i) : 0;
                if (want_jerk && i < nt) {
                    const float4 v = A.svel[p];
                    tvx[k] = v.x; tvy[k] = v.y; tvz[k] = v.z;
                }
                if (want_zeta && i < nt && A.stype[p] == 0) {
                    const double mt = A.smass[p];
                    if (mt > 0.0) {
                        tzm[k] = (float)(A.szeta[p] / mt);
                        tim[k] = (float)(1.0 / mt);
                    }
                }
                if (sink_rule && i < nt) sink |= A.stype[p] == 5;
            }
            has_sink = __any_sync(kFull, sink);
        }
        // one interaction's tidal and jerk terms: T += -g1 I + g2 d d, J += g1 dv - (dv.d) g2 d
        // (shmem/tree.cc:811-837, 845-872); d = source - target, dv = v_source - v_target.  The
        // list's g2 d d and its sum of g1 (q[9]) are kept apart and the diagonal's -g1 is taken off
        // in FP64 when the list is added to the totals: 10 FP32 operations per interaction instead
        // of 15, and the diagonal's cancellation happens in FP64.
        auto xt_add = [&](float (&q)[10], float dx, float dy, float dz, float g1, float g2, float4 ev, int k) {
            if (want_tid) {
                const float gx = g2 * dx, gy = g2 * dy, gz = g2 * dz;
                q[0] = fmaf(gx, dx, q[0]);
                q[1] = fmaf(gy, dy, q[1]);
                q[2] = fmaf(gz, dz, q[2]);
                q[3] = fmaf(gx, dy, q[3]);
                q[4] = fmaf(gy, dz, q[4]);
                q[5] = fmaf(gx, dz, q[5]);
                q[9] += g1;
            }
            if (want_jerk) {
                const float dvx = ev.x - tvx[k], dvy = ev.y - tvy[k], dvz = ev.z - tvz[k];
                const float vg = fmaf(dvx, dx, fmaf(dvy, dy, dvz * dz)) * g2;
                q[6] += fmaf(g1, dvx, -vg * dx);
                q[7] += fmaf(g1, dvy, -vg * dy);
                q[8] += fmaf(g1, dvz, -vg * dz);
            }
        };

        // ---- evaluate the lists against the targets ---------------------------------------
        auto accumulate = [&](const float* ax_, const float* ay_, const float* az_, const float* ap_) {
#pragma unroll
            for (int k = 0; k < TPL; ++k) {
                kahan_add(sx[k], cxk[k], ax_[k]);
                kahan_add(sy[k], cyk[k], ay_[k]);
                kahan_add(sz[k], czk[k], az_[k]);
                if (WANT_POT) pot[k] += (double)ap_[k];
            }
            if (COUNT) c_flush += (lane == 0);
        };
        // Monopoles.  An accepted node passed the softening-overlap test, so every target of the
        // group is farther than max(h_target, h_node) from it: the interaction is Newtonian.
        // The list pairs its entries: entries 2p and 2p+1 share two float4s, {x0, x1, y0, y1} and
        // {z0, z1, m0, m1}, so two 16-byte loads put a pair straight into the register pairs of the
        // sm_100 packed FP32 instructions (FADD2 / FMUL2 / FFMA2): two interactions per
        // instruction, each with exactly the scalar rounding.  An odd list is padded with a
        // massless entry, which contributes an exact zero.  r^2 is floored at 1e-30 by starting
        // its FMA chain at 1e-30 instead of 0: no extra instruction, and below the rounding of any
        // r^2 above 1e-22, so only a point closer than FP32 resolves is affected (it then adds 0
        // along that axis instead of a NaN).
        auto flush_pn = [&](int n) {
            if (paired && (n & 1) && lane == 0) {
                pn_put(n, 0.0f, 0.0f, 0.0f, 0.0f);
                if (want_jerk) pnv[n] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // the pad's velocity
            }
            __syncwarp();
            const int np = (n + 1) >> 1;
            float ax_[TPL], ay_[TPL], az_[TPL], ap_[TPL];
            float xq[XT == 1 ? TPL : 1][10];
#pragma unroll
            for (int k = 0; k < TPL; ++k) ax_[k] = ay_[k] = az_[k] = ap_[k] = 0.0f;
            // packed for full groups; groups of <= 16 targets split the list over lane slices, where
            // the scalar loop measured faster
            if (paired) {
                float2 ax2[TPL], ay2[TPL], az2[TPL], ap2[TPL];
                float2 ntx[TPL], nty[TPL], ntz[TPL];
                // XT 1: the tidal and jerk sums of xt_add, two entries per instruction
                float2 xq2[XT == 1 ? TPL : 1][10];
                const float2 r2_floor = make_float2(1e-30f, 1e-30f);
#pragma unroll
                for (int k = 0; k < TPL; ++k) {
                    ax2[k] = ay2[k] = az2[k] = ap2[k] = make_float2(0.0f, 0.0f);
                    ntx[k] = make_float2(-tx[k], -tx[k]);
                    nty[k] = make_float2(-ty[k], -ty[k]);
                    ntz[k] = make_float2(-tz[k], -tz[k]);
                    if (XT == 1)
#pragma unroll
                        for (int c = 0; c < 10; ++c) xq2[XT == 1 ? k : 0][c] = make_float2(0.0f, 0.0f);
                }
                // 8 pairs in flight per lane (unroll 2 and 4 measured 1.9 % and 0.6 % slower); the
                // tidal and jerk body is three times longer, and unrolled it outgrows instruction fetch
#pragma unroll (XT == 1 ? 1 : 8)
                for (int jp = slice; jp < np; jp += NS) {
                    const float4 A = pn[2 * jp], B = pn[2 * jp + 1];
                    const float2 X = make_float2(A.x, A.y), Y = make_float2(A.z, A.w);
                    const float2 Z = make_float2(B.x, B.y), M = make_float2(B.z, B.w);
#pragma unroll
                    for (int k = 0; k < TPL; ++k) {
                        if (k < nk) {
                            const float2 dx = __fadd2_rn(X, ntx[k]), dy = __fadd2_rn(Y, nty[k]);
                            const float2 dz = __fadd2_rn(Z, ntz[k]);
                            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, r2_floor)));
                            const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
                            const float2 mri = __fmul2_rn(M, ri);
                            const float2 f = __fmul2_rn(mri, __fmul2_rn(ri, ri));
                            ax2[k] = __ffma2_rn(dx, f, ax2[k]);
                            ay2[k] = __ffma2_rn(dy, f, ay2[k]);
                            az2[k] = __ffma2_rn(dz, f, az2[k]);
                            if (WANT_POT) ap2[k] = __fadd2_rn(ap2[k], mri);
                            if (XT == 1) {
                                // Newtonian: g1 = f, g2 = 3 f / r^2, each element rounded as xt_add
                                float2(&q)[10] = xq2[XT == 1 ? k : 0];
                                const float2 g2 = __fmul2_rn(__fmul2_rn(make_float2(3.0f, 3.0f), f), __fmul2_rn(ri, ri));
                                if (want_tid) {
                                    const float2 gx = __fmul2_rn(g2, dx), gy = __fmul2_rn(g2, dy), gz = __fmul2_rn(g2, dz);
                                    q[0] = __ffma2_rn(gx, dx, q[0]);
                                    q[1] = __ffma2_rn(gy, dy, q[1]);
                                    q[2] = __ffma2_rn(gz, dz, q[2]);
                                    q[3] = __ffma2_rn(gx, dy, q[3]);
                                    q[4] = __ffma2_rn(gy, dz, q[4]);
                                    q[5] = __ffma2_rn(gx, dz, q[5]);
                                    q[9] = __fadd2_rn(q[9], f);
                                }
                                if (want_jerk) {
                                    const float4 v0 = pnv[2 * jp], v1 = pnv[2 * jp + 1];
                                    const float2 dvx = __fadd2_rn(make_float2(v0.x, v1.x), make_float2(-tvx[k], -tvx[k]));
                                    const float2 dvy = __fadd2_rn(make_float2(v0.y, v1.y), make_float2(-tvy[k], -tvy[k]));
                                    const float2 dvz = __fadd2_rn(make_float2(v0.z, v1.z), make_float2(-tvz[k], -tvz[k]));
                                    const float2 vg =
                                        __fmul2_rn(__ffma2_rn(dvx, dx, __ffma2_rn(dvy, dy, __fmul2_rn(dvz, dz))), g2);
                                    const float2 nvg = make_float2(-vg.x, -vg.y);
                                    q[6] = __fadd2_rn(q[6], __ffma2_rn(f, dvx, __fmul2_rn(nvg, dx)));
                                    q[7] = __fadd2_rn(q[7], __ffma2_rn(f, dvy, __fmul2_rn(nvg, dy)));
                                    q[8] = __fadd2_rn(q[8], __ffma2_rn(f, dvz, __fmul2_rn(nvg, dz)));
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < TPL; ++k) {
                    ax_[k] = ax2[k].x + ax2[k].y;
                    ay_[k] = ay2[k].x + ay2[k].y;
                    az_[k] = az2[k].x + az2[k].y;
                    ap_[k] = -(ap2[k].x + ap2[k].y);
                    if (XT == 1)
#pragma unroll
                        for (int c = 0; c < 10; ++c)
                            xq[XT == 1 ? k : 0][c] = xq2[XT == 1 ? k : 0][c].x + xq2[XT == 1 ? k : 0][c].y;
                }
            } else {
                if (XT == 1) {
#pragma unroll
                    for (int k = 0; k < TPL; ++k)
#pragma unroll
                        for (int c = 0; c < 10; ++c) xq[XT == 1 ? k : 0][c] = 0.0f;
                }
#pragma unroll 4
                for (int j = slice; j < n; j += NS) {
                    const float4 e = pn[j];
#pragma unroll
                    for (int k = 0; k < TPL; ++k) {
                        if (k < nk) {
                            const float dx = e.x - tx[k], dy = e.y - ty[k], dz = e.z - tz[k];
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 1e-30f)));
                            const float ri = rsqrt_ftz(r2);
                            const float mri = e.w * ri;
                            const float f = mri * (ri * ri);
                            ax_[k] = fmaf(dx, f, ax_[k]);
                            ay_[k] = fmaf(dy, f, ay_[k]);
                            az_[k] = fmaf(dz, f, az_[k]);
                            if (WANT_POT) ap_[k] -= mri;
                            if (XT == 1) {
                                // Newtonian: g2 = 3 m / r^5
                                const float4 ev = want_jerk ? pnv[j] : make_float4(0.f, 0.f, 0.f, 0.f);
                                xt_add(xq[XT == 1 ? k : 0], dx, dy, dz, f, 3.0f * f * (ri * ri), ev, k);
                            }
                        }
                    }
                }
            }
            accumulate(ax_, ay_, az_, ap_);
            if (XT == 1) {
#pragma unroll
                for (int k = 0; k < TPL; ++k) {
                    const double sg = (double)xq[XT == 1 ? k : 0][9];  // the diagonal's -g1 terms
#pragma unroll
                    for (int c = 0; c < 9; ++c) xt[c][k] += (double)xq[XT == 1 ? k : 0][c] - (c < 3 ? sg : 0.0);
                }
            }
            __syncwarp();
        };
        // Particles: kernel of the larger softening; r^2 == 0 (the target itself) contributes 0.
        // Full groups of the plain walk pair the list like the monopoles and evaluate two entries
        // per packed instruction while both are outside the kernel or at r = 0; a pair with an
        // entry inside the kernel takes the scalar spline for both, with the same terms, so the
        // sums do not depend on which lanes diverge.  An odd list is padded with a massless entry
        // far outside (1e18 on each axis), which adds exact zeros.
        auto flush_pp = [&](int n) {
            if (ppair && (n & 1) && lane == 0) {
                pp_put(n, 1e18f, 1e18f, 1e18f, 0.0f);
                ph[n] = 0.0f;
            }
            __syncwarp();
            float ax_[TPL], ay_[TPL], az_[TPL], ap_[TPL];
            float xq[XT == 1 ? TPL : 1][10];
#pragma unroll
            for (int k = 0; k < TPL; ++k) ax_[k] = ay_[k] = az_[k] = ap_[k] = 0.0f;
            if (XT == 1) {
#pragma unroll
                for (int k = 0; k < TPL; ++k)
#pragma unroll
                    for (int c = 0; c < 10; ++c) xq[XT == 1 ? k : 0][c] = 0.0f;
            }
            unsigned zero = 0;
            if (ppair) {
                float2 ax2[TPL], ay2[TPL], az2[TPL], np2[TPL];  // np2: minus the potential
#pragma unroll
                for (int k = 0; k < TPL; ++k) ax2[k] = ay2[k] = az2[k] = np2[k] = make_float2(0.0f, 0.0f);
                const float2* __restrict__ H = reinterpret_cast<const float2*>(ph);
                const int np = (n + 1) >> 1;
                for (int jp = slice; jp < np; jp += NS) {
                    const float4 P = pp[2 * jp], Q = pp[2 * jp + 1];
                    const float2 hj = H[jp];
                    const float2 X = make_float2(P.x, P.y), Y = make_float2(P.z, P.w);
                    const float2 Z = make_float2(Q.x, Q.y), M = make_float2(Q.z, Q.w);
#pragma unroll
                    for (int k = 0; k < TPL; ++k) {
                        if (k < nk) {
                            const float2 dx = __fadd2_rn(X, make_float2(-tx[k], -tx[k]));
                            const float2 dy = __fadd2_rn(Y, make_float2(-ty[k], -ty[k]));
                            const float2 dz = __fadd2_rn(Z, make_float2(-tz[k], -tz[k]));
                            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                            const float2 hh = make_float2(fmaxf(th[k], hj.x), fmaxf(th[k], hj.y));
                            const float2 hh2 = __fmul2_rn(hh, hh);
                            const bool z0 = r2.x == 0.0f, z1 = r2.y == 0.0f;
                            if (COUNT) zero += (unsigned)z0 + (unsigned)z1;
                            float2 f, mp;
                            if ((r2.x >= hh2.x || z0) && (r2.y >= hh2.y || z1)) {
                                const float2 ri = make_float2(z0 ? 0.0f : rsqrt_ftz(r2.x), z1 ? 0.0f : rsqrt_ftz(r2.y));
                                mp = __fmul2_rn(M, ri);
                                f = __fmul2_rn(mp, __fmul2_rn(ri, ri));
                            } else {
                                // the same terms one entry at a time, the spline where r < h
                                const float r2s[2] = {r2.x, r2.y}, hs[2] = {hh.x, hh.y}, ms[2] = {M.x, M.y};
                                float fs[2], ps[2];
#pragma unroll
                                for (int e = 0; e < 2; ++e) {
                                    if (r2s[e] >= hs[e] * hs[e] && r2s[e] > 0.0f) {
                                        const float ri = rsqrt_ftz(r2s[e]);
                                        const float mri = ms[e] * ri;
                                        fs[e] = mri * (ri * ri);
                                        ps[e] = -mri;
                                    } else {
                                        spline_pair(r2s[e], hs[e], ms[e], fs[e], ps[e]);
                                    }
                                }
                                f = make_float2(fs[0], fs[1]);
                                mp = make_float2(-ps[0], -ps[1]);
                            }
                            ax2[k] = __ffma2_rn(dx, f, ax2[k]);
                            ay2[k] = __ffma2_rn(dy, f, ay2[k]);
                            az2[k] = __ffma2_rn(dz, f, az2[k]);
                            if (WANT_POT) np2[k] = __fadd2_rn(np2[k], mp);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < TPL; ++k) {
                    ax_[k] = ax2[k].x + ax2[k].y;
                    ay_[k] = ay2[k].x + ay2[k].y;
                    az_[k] = az2[k].x + az2[k].y;
                    ap_[k] = -(np2[k].x + np2[k].y);
                }
            } else {
                for (int j = slice; j < n; j += NS) {
                    const float4 e = pp[j];
                    const float hj = ph[j];
#pragma unroll
                    for (int k = 0; k < TPL; ++k) {
                        if (k < nk) {
                            const float dx = e.x - tx[k], dy = e.y - ty[k], dz = e.z - tz[k];
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float hh = fmaxf(th[k], hj);
                            float f, p, g2 = 0.0f;
                            float fa;  // the acceleration's factor: f less the gas pair's zeta terms
                            // r = 0 (the target itself) takes this branch with 1/r = 0: every term
                            // is then 0, as the spline branch gives it, without the call
                            if (r2 >= hh * hh || r2 == 0.0f) {
                                const float ri = r2 > 0.0f ? rsqrt_ftz(r2) : 0.0f;
                                const float mri = e.w * ri;
                                f = mri * ri * ri;
                                p = -mri;
                                if (XT == 1) g2 = 3.0f * f * (ri * ri);
                                fa = f;
                            } else if (XT == 1) {
                                spline_pair_tidal(r2, hh, e.w, f, p, g2);
                                fa = want_zeta ? f - zeta_pair(r2, hh, hj, pzs[j], tzm[k], tim[k]) : f;
                            } else {
                                spline_pair(r2, hh, e.w, f, p);
                                fa = (XT == 2 && want_zeta) ? f - zeta_pair(r2, hh, hj, pzs[j], tzm[k], tim[k]) : f;
                            }
                            if (COUNT) zero += (r2 == 0.0f);
                            ax_[k] = fmaf(dx, fa, ax_[k]);
                            ay_[k] = fmaf(dy, fa, ay_[k]);
                            az_[k] = fmaf(dz, fa, az_[k]);
                            if (WANT_POT) ap_[k] += p;
                            if (XT == 1) {
                                const float4 ev = want_jerk ? ppv[j] : make_float4(0.f, 0.f, 0.f, 0.f);
                                xt_add(xq[XT == 1 ? k : 0], dx, dy, dz, f, g2, ev, k);
                            }
                        }
                    }
                }
            }
            accumulate(ax_, ay_, az_, ap_);
            if (XT == 1) {
#pragma unroll
                for (int k = 0; k < TPL; ++k) {
                    const double sg = (double)xq[XT == 1 ? k : 0][9];  // the diagonal's -g1 terms
#pragma unroll
                    for (int c = 0; c < 9; ++c) xt[c][k] += (double)xq[XT == 1 ? k : 0][c] - (c < 3 ? sg : 0.0);
                }
            }
            if (COUNT) c_zero += zero;
            __syncwarp();
        };

        // ---- traversal ----------------------------------------------------------------------
        int top = 1;
        if (lane == 0) stk[0] = A.group_root ? A.group_root[g] : 0;
        __syncwarp();
        int npn = 0, npp = 0;
        bool overflow = false;
        while (top > 0) {
            const int npop = min(top, 32);
            top -= npop;
            int node = lane < npop ? stk[top + lane] : -1;
            if (node >= 0 && !GT_IN_BOUNDS(node, A.n_nodes)) node = -1;
            __syncwarp();
            bool accept = false, expand = false, push = false;
            // idle lanes read node 0 and decide nothing (cheaper than defaulting every field)
            const NodeV nd = load_node(A.nodes + (node >= 0 ? node : 0));
            if (node >= 0) {
                const bool leaf = nd.first < 0;
                const double dx = box_gap(nd.cx, S.c_x, S.w_x);
                const double dy = box_gap(nd.cy, S.c_y, S.w_y);
                const double dz = box_gap(nd.cz, S.c_z, S.w_z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                bool open = true;
                if (MAC != 1) {
                    if (LEAF_ACCEPT || !leaf) {
                        const double len = (double)nd.len;
                        const double ml2 = MAC == 2 ? nd.mass * (double)__ldg(A.mac_l2 + node) : nd.mass * len * len;
                        open = open_node(r2, len, nd.s, ml2, (double)nd.soft, S.emax, S.amin, A.theta2, dx, dy, dz);
                    }
                } else if (LEAF_ACCEPT || !leaf) {
                    // learned criterion: the softening-overlap, inside-node and Barnes-Hut arms
                    // stay; the relative arm's estimate M L^2 / r^4 is corrected by the network
                    // inside the band of rho where it may change the decision
                    const double len = (double)nd.len;
                    const double rt = S.emax + 0.6 * len, rn = (double)nd.soft + 0.6 * len;
                    const double lim = 0.6 * len;
                    const bool hard = (r2 < rt * rt) | (r2 < rn * rn) |
                                      ((A.theta2 > 0.0) & (nd.s * nd.s >= A.theta2 * r2)) |
                                      ((dx < lim) & (dy < lim) & (dz < lim));
                    const double aold = S.amin;
                    if (hard) {
                        open = true;
                    } else if (!(aold > 0)) {
                        open = A.theta2 <= 0.0;
                    } else {
                        const double rho = nd.mass * len * len / (r2 * r2 * aold);
                        if (rho <= A.mac_band_lo) {
                            open = false;
                        } else if (rho > A.mac_band_hi) {
                            open = true;
                        } else {
                            const double ex = fmax(fabs(nd.cx - S.lo_x), fabs(nd.cx - S.hi_x));
                            const double ey = fmax(fabs(nd.cy - S.lo_y), fabs(nd.cy - S.hi_y));
                            const double ez = fmax(fabs(nd.cz - S.lo_z), fabs(nd.cz - S.hi_z));
                            const double gx = S.hi_x - S.lo_x, gy = S.hi_y - S.lo_y, gz = S.hi_z - S.lo_z;
                            float f[kMacIn];
                            mac_features(r2, rho, len, nd.s, nd.mass, (double)A.nq2[node], (double)nd.soft,
                                         S.emax, nd.phi - nd.plo, ex * ex + ey * ey + ez * ez,
                                         gx * gx + gy * gy + gz * gz, f);
                            const float c = mac_forward(mac_w, f);
                            open = f[4] + c > (float)A.mac_log_kappa;  // f[4] = log10(rho)
                        }
                    }
                }
                // sink-direct opening (tree.cc:772-778): only ever adds opening
                if (sink_rule && has_sink && !open && __ldg(A.nsink + node) > 0u) {
                    const double reach = A.sink_r + 0.6 * (double)nd.len;
                    if (r2 < reach * reach) open = true;
                }
                if (!open) accept = true;
                else if (leaf) expand = true;
                else push = true;
            }
            if (COUNT && lane == 0) { c_nodes += npop; ++c_steps; }

            // children of opened interior nodes
            // One scan gives both the children's stack slots and the expanded leaves' particle
            // slots, packed as nch + (cnt << 10): nch <= 8, so the children's total stays below
            // 1024, and the particles' total fits the upper 21 bits while every leaf holds fewer
            // than 2^16 particles (else two scans).
            const int nch = push ? nd.nchild : 0;
            const int cnt = expand ? nd.phi - nd.plo : 0;
            int incl, inc2;
            if (!__any_sync(kFull, cnt >= (1 << 16))) {
                const int both = warp_incl_scan_i(nch | (cnt << 10));
                incl = both & 1023;
                inc2 = both >> 10;
            } else {
                incl = warp_incl_scan_i(nch);
                inc2 = warp_incl_scan_i(cnt);
            }
            const int tot = __shfl_sync(kFull, incl, 31);
            if (top + tot > A.stack_cap) { overflow = true; break; }
            {
                // an octree node has at most 8 children: a fixed, predicated loop
                int* dst = stk + (top + incl - nch);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (c < nch) dst[c] = nd.first + c;
            }
            top += tot;
            __syncwarp();  // pushes are visible to the lanes that pop them
            if (COUNT) c_maxtop = max(c_maxtop, top);

            // accepted nodes: monopoles
            const unsigned am = __ballot_sync(kFull, accept);
            if (am) {
                const int na = __popc(am);
                if (npn + na > A.pn_cap) { flush_pn(npn); npn = 0; }
                if (accept && GT_IN_BOUNDS(npn + __popc(am & lt_mask), A.pn_cap)) {
                    const int pos = npn + __popc(am & lt_mask);
                    pn_put(pos, (float)(nd.cx - S.c_x), (float)(nd.cy - S.c_y), (float)(nd.cz - S.c_z),
                           (float)nd.mass);
                    if (want_jerk) pnv[pos] = A.nvel[node];  // the node's centre-of-mass velocity
                }
                npn += na;
                if (COUNT && lane == 0) c_multi += (unsigned long long)na * nt;
            }

            // expanded leaves: their particles
            const unsigned em = __ballot_sync(kFull, expand);
            if (em) {
                const int tot2 = __shfl_sync(kFull, inc2, 31);
                S.lo[lane] = nd.plo;
                S.pre[lane] = inc2 - cnt;
                __syncwarp();
                if (COUNT && lane == 0) c_pairs += (unsigned long long)tot2 * nt;
                // 32 particles at a time, one per lane.  A particle farther from the group box
                // than max(largest target softening, its own) is Newtonian for every target
                // (the reference's spline is exactly 1/r^3 for r >= h): it joins the monopole
                // list.  The rest -- the group's own particles among them -- need the softened
                // pair rule and go to the particle list.
                for (int base = 0; base < tot2; base += 32) {
                    const int q = base + lane;
                    const bool live = q < tot2;
                    double qx = 0, qy = 0, qz = 0;
                    float qm = 0.0f, qh = 0.0f;
                    bool far = false;
                    int qpos = 0;
                    if (live) {
                        // owner: the last lane whose exclusive prefix is <= q
                        int l = 0;
#pragma unroll
                        for (int step = 16; step > 0; step >>= 1)
                            if (S.pre[l + step] <= q) l += step;
                        qpos = S.lo[l] + (q - S.pre[l]);
                        if (!GT_IN_BOUNDS(qpos, A.n_src)) qpos = 0;
                        load_src(A.src + qpos, qx, qy, qz, qm, qh);
                        const double ex = box_gap(qx, S.c_x, S.w_x);
                        const double ey = box_gap(qy, S.c_y, S.w_y);
                        const double ez = box_gap(qz, S.c_z, S.w_z);
                        const double qhd = (double)qh;
                        const double reach = S.emax > qhd ? S.emax : qhd;
                        far = ex * ex + ey * ey + ez * ez > reach * reach;
                    }
                    const unsigned fm = __ballot_sync(kFull, live && far);
                    const unsigned nm = __ballot_sync(kFull, live && !far);
                    const int nf = __popc(fm), nn = __popc(nm);
                    if (npn + nf > A.pn_cap) { flush_pn(npn); npn = 0; }
                    if (npp + nn > A.pp_cap) { flush_pp(npp); npp = 0; }
                    const float4 e = make_float4((float)(qx - S.c_x), (float)(qy - S.c_y), (float)(qz - S.c_z), qm);
                    if (live && far && GT_IN_BOUNDS(npn + __popc(fm & lt_mask), A.pn_cap)) {
                        pn_put(npn + __popc(fm & lt_mask), e.x, e.y, e.z, e.w);
                        if (want_jerk) pnv[npn + __popc(fm & lt_mask)] = A.svel[qpos];
                    } else if (live && GT_IN_BOUNDS(npp + __popc(nm & lt_mask), A.pp_cap)) {
                        const int pos = npp + __popc(nm & lt_mask);
                        if (ppair) pp_put(pos, e.x, e.y, e.z, e.w);
                        else pp[pos] = e;
                        ph[pos] = qh;
                        if (want_jerk) ppv[pos] = A.svel[qpos];
                        if (want_zeta) pzs[pos] = A.stype[qpos] == 0 ? (float)A.szeta[qpos] : __int_as_float(0x7fc00000);
                    }
                    npn += nf;
                    npp += nn;
                    __syncwarp();
                }
            }
        }
        if (overflow) {
            if (lane == 0) atomicExch(A.error, 1);
            continue;
        }
        if (npn > 0) flush_pn(npn);
        if (npp > 0) flush_pp(npp);

        // ---- combine slices and write -------------------------------------------------------
#pragma unroll
        for (int k = 0; k < TPL; ++k) {
            double vx = (double)sx[k] - (double)cxk[k];
            double vy = (double)sy[k] - (double)cyk[k];
            double vz = (double)sz[k] - (double)czk[k];
            double vp = pot[k];
            for (int o = NT; o < 32; o <<= 1) {
                vx += __shfl_xor_sync(kFull, vx, o);
                vy += __shfl_xor_sync(kFull, vy, o);
                vz += __shfl_xor_sync(kFull, vz, o);
                if (WANT_POT) vp += __shfl_xor_sync(kFull, vp, o);
            }
            if (XT == 1) {
#pragma unroll
                for (int c = 0; c < 9; ++c)
                    for (int o = NT; o < 32; o <<= 1) xt[c][k] += __shfl_xor_sync(kFull, xt[c][k], o);
            }
            const int i = ti + 32 * k;
            if (slice == 0 && k < nk && i < nt) {
                const int idx = t0 + i;
                const int o = A.out_map ? (int)A.out_map[idx] : idx;
                if (!GT_IN_BOUNDS(o, A.n_out)) continue;
                if (A.ax) {
                    A.ax[o] = A.G * vx;
                    A.ay[o] = A.G * vy;
                    A.az[o] = A.G * vz;
                }
                if (WANT_POT && A.phi) A.phi[o] = A.G * vp;
                if (want_tid)
#pragma unroll
                    for (int c = 0; c < 6; ++c) A.tidal[6 * (size_t)o + c] = xt[c][k];
                if (want_jerk)
#pragma unroll
                    for (int c = 0; c < 3; ++c) A.jerk[3 * (size_t)o + c] = A.G * xt[6 + c][k];
            }
        }
    }
    if (COUNT) {
        if (lane == 0) {
            atomicAdd(&A.stats[0], c_nodes);
            atomicAdd(&A.stats[1], c_multi);
            atomicAdd(&A.stats[2], c_pairs);
            atomicAdd(&A.stats[4], c_flush);
            atomicMax(&A.stats[5], (unsigned long long)c_maxtop);
            atomicAdd(&A.stats[6], c_steps);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c_zero += __shfl_xor_sync(kFull, c_zero, o);
        if (lane == 0) atomicAdd(&A.stats[3], c_zero);
    }
}

// ---------------------------------------------------------------------------------------------
// Paired windows
// ---------------------------------------------------------------------------------------------
// Two consecutive windows of a batch walk (groups 2p and 2p+1 of the list, up to 32 targets each)
// share one traversal.  Each stack entry carries, in its two low bits, the windows for which its
// parent was opened, and a popped node is tested against the boxes of those windows only.  So each
// window tests exactly the nodes its own walk tests, makes the same decisions and collects the
// same monopoles and particles, into its own lists.  The pop, the node load, the child pushes and
// the expanded leaves' particle loads are shared: windows adjacent in Peano-Hilbert order open
// mostly the same nodes.  Lane l holds target l of each window; the lists are evaluated window by
// window with walk_kernel's packed monopole loop.  A window's nodes can join its list in another
// order than in its own walk (the other window's nodes interleave on the stack), so the sums agree
// with walk_kernel's to FP32 rounding, not bit for bit.  One target per lane, the grouped walk,
// the plain or per-node learned criterion; in a forest the two windows may start from two roots.

struct alignas(16) PairHdr {
    int lo[32];   // leaf-expansion scratch: first slot, exclusive prefix and windows of each leaf
    int pre[32];
    int msk[32];
    // per window, in one 64-byte record: box centre and half width per axis side by side (one
    // 16-byte shared-memory load per axis of a box gap), largest target softening, smallest aold
    struct alignas(16) Win { double c_x, w_x, c_y, w_y, c_z, w_z, emax, amin; } wb[2];
};

__host__ __device__ constexpr int pair_list_bytes(int pn_cap, int pp_cap) { return pn_cap * 16 + pp_cap * 20; }
__host__ __device__ constexpr int pair_smem_bytes(int pn_cap, int pp_cap) {
    return ((int)sizeof(PairHdr) + 2 * pair_list_bytes(pn_cap, pp_cap) + 15) & ~15;
}

template <bool WANT_POT, bool COUNT, int MAC>
__global__ void __launch_bounds__(kMaxWarps * 32, 3) walk_pair_kernel(const WalkArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int gw = blockIdx.x * (blockDim.x >> 5) + w;
    int* __restrict__ stk = A.stack + (size_t)gw * A.stack_cap;
    unsigned char* wbase = smem_raw + (size_t)w * A.warp_bytes;
    PairHdr& S = *reinterpret_cast<PairHdr*>(wbase);
    const int list_bytes = pair_list_bytes(A.pn_cap, A.pp_cap);
    // window v's lists: monopoles (pn_cap float4, paired layout), particles (pp_cap float4) and
    // their softenings (pp_cap float)
    auto pn_of = [&](int v) { return reinterpret_cast<float4*>(wbase + sizeof(PairHdr) + (size_t)v * list_bytes); };
    auto pp_of = [&](int v) { return pn_of(v) + A.pn_cap; };
    auto ph_of = [&](int v) { return reinterpret_cast<float*>(pp_of(v) + A.pp_cap); };
    const int n_groups = A.n_groups_dev ? (int)*A.n_groups_dev : A.n_groups;
    const int n_pairs = (n_groups + 1) >> 1;
    // SHMEM_COUNT_WALK: per window, as walk_kernel counts them (node tests, monopoles and
    // particles times the window's targets, r = 0 pairs), so a paired walk counts what the two
    // one-window walks count
    unsigned long long c_nodes = 0, c_multi = 0, c_pairs = 0, c_zero = 0, c_flush = 0, c_steps = 0;
    int c_maxtop = 0;

    for (;;) {
        int pr = 0;
        if (lane == 0) pr = (int)atomicAdd(A.next_group, 1u);
        pr = __shfl_sync(kFull, pr, 0);
        if (pr >= n_pairs) break;
        int t0[2], nt[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int g = 2 * pr + v;
            const int2 gr = g < n_groups ? A.groups[g] : make_int2(0, 0);
            t0[v] = gr.x;
            nt[v] = gr.y - gr.x;
        }

        // ---- targets: lane l holds target l of each window ---------------------------------
        float tx[2], ty[2], tz[2], th[2];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            double px = 0.0, py = 0.0, pz = 0.0, ps = 0.0;
            double lx = 1e300, ly = 1e300, lz = 1e300, hx = -1e300, hy = -1e300, hz = -1e300;
            double amin = A.aold ? 1e300 : 0.0;
            if (lane < nt[v]) {
                int p = A.tpos ? (int)A.tpos[t0[v] + lane] : t0[v] + lane;
                if (!GT_IN_BOUNDS(p, A.n_src)) p = 0;
                float mf, hf;
                load_src(A.src + p, px, py, pz, mf, hf);
                ps = A.ssoft[p];
                lx = hx = px;
                ly = hy = py;
                lz = hz = pz;
                if (A.aold) amin = A.aold[t0[v] + lane];
            }
            lx = wmin(lx); ly = wmin(ly); lz = wmin(lz);
            hx = wmax(hx); hy = wmax(hy); hz = wmax(hz);
            const double emax = wmax(ps);
            if (A.aold) amin = wmin(amin);
            const double cx = 0.5 * (lx + hx), cy = 0.5 * (ly + hy), cz = 0.5 * (lz + hz);
            if (lane == 0) {
                S.wb[v].c_x = cx; S.wb[v].c_y = cy; S.wb[v].c_z = cz;
                S.wb[v].w_x = 0.5 * (hx - lx); S.wb[v].w_y = 0.5 * (hy - ly); S.wb[v].w_z = 0.5 * (hz - lz);
                S.wb[v].emax = emax; S.wb[v].amin = amin;
            }
            tx[v] = (float)(px - cx);
            ty[v] = (float)(py - cy);
            tz[v] = (float)(pz - cz);
            th[v] = (float)ps;
        }
        __syncwarp();
        float sx0 = 0.0f, sy0 = 0.0f, sz0 = 0.0f, cx0 = 0.0f, cy0 = 0.0f, cz0 = 0.0f;
        float sx1 = 0.0f, sy1 = 0.0f, sz1 = 0.0f, cx1 = 0.0f, cy1 = 0.0f, cz1 = 0.0f;
        double pot0 = 0.0, pot1 = 0.0;
        // one window's partial sums into its Kahan-compensated totals (v at run time: the
        // evaluation loops below exist once in the code, for both windows)
        auto add_partial = [&](int v, float ax, float ay, float az, float ap) {
            if (v == 0) {
                kahan_add(sx0, cx0, ax); kahan_add(sy0, cy0, ay); kahan_add(sz0, cz0, az);
                if (WANT_POT) pot0 += (double)ap;
            } else {
                kahan_add(sx1, cx1, ax); kahan_add(sy1, cy1, ay); kahan_add(sz1, cz1, az);
                if (WANT_POT) pot1 += (double)ap;
            }
        };
        // monopole-list entry pos of window v, in walk_kernel's paired layout (see flush_pn there)
        auto pn_put = [&](int v, int pos, float x, float y, float z, float m) {
            float* q = reinterpret_cast<float*>(pn_of(v) + 2 * (pos >> 1)) + (pos & 1);
            q[0] = x; q[2] = y; q[4] = z; q[6] = m;
        };
        // particle-list entry pos of window v, in the same paired layout
        auto pp_put = [&](int v, int pos, float x, float y, float z, float m) {
            float* q = reinterpret_cast<float*>(pp_of(v) + 2 * (pos >> 1)) + (pos & 1);
            q[0] = x; q[2] = y; q[4] = z; q[6] = m;
        };
        // window v's monopoles against its targets: walk_kernel's packed loop
        auto flush_pn = [&](int v, int n) {
            if ((n & 1) && lane == 0) pn_put(v, n, 0.0f, 0.0f, 0.0f, 0.0f);
            __syncwarp();
            const int np = (n + 1) >> 1;
            float2 ax2 = make_float2(0.0f, 0.0f), ay2 = ax2, az2 = ax2, ap2 = ax2;
            const float qx = v ? tx[1] : tx[0], qy = v ? ty[1] : ty[0], qz = v ? tz[1] : tz[0];
            const float2 ntx = make_float2(-qx, -qx), nty = make_float2(-qy, -qy), ntz = make_float2(-qz, -qz);
            const float2 r2_floor = make_float2(1e-30f, 1e-30f);
            const float4* __restrict__ L = pn_of(v);
#pragma unroll 8
            for (int jp = 0; jp < np; ++jp) {
                const float4 P = L[2 * jp], Q = L[2 * jp + 1];
                const float2 X = make_float2(P.x, P.y), Y = make_float2(P.z, P.w);
                const float2 Z = make_float2(Q.x, Q.y), M = make_float2(Q.z, Q.w);
                const float2 dx = __fadd2_rn(X, ntx), dy = __fadd2_rn(Y, nty), dz = __fadd2_rn(Z, ntz);
                const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, r2_floor)));
                const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
                const float2 mri = __fmul2_rn(M, ri);
                const float2 f = __fmul2_rn(mri, __fmul2_rn(ri, ri));
                ax2 = __ffma2_rn(dx, f, ax2);
                ay2 = __ffma2_rn(dy, f, ay2);
                az2 = __ffma2_rn(dz, f, az2);
                if (WANT_POT) ap2 = __fadd2_rn(ap2, mri);
            }
            add_partial(v, ax2.x + ax2.y, ay2.x + ay2.y, az2.x + az2.y, -(ap2.x + ap2.y));
            if (COUNT) c_flush += (lane == 0);
            __syncwarp();
        };
        // window v's particles: the kernel of the larger softening; r^2 == 0 contributes 0.  The
        // list is paired like the monopoles (pp_put), softenings side by side, and evaluated two
        // entries per packed instruction while both are outside the kernel or at r = 0 (the
        // window's own particles); a pair with an entry inside the kernel takes the scalar spline
        // for both.  Each entry's terms are the same on either path, so the sums do not depend on
        // which lanes diverge.  An odd list is padded with a massless entry far outside (1e18 on
        // each axis, r^2 ~ 3e36 below the FP32 range's end), which adds exact zeros.
        auto flush_pp = [&](int v, int n) {
            if ((n & 1) && lane == 0) {
                pp_put(v, n, 1e18f, 1e18f, 1e18f, 0.0f);
                ph_of(v)[n] = 0.0f;
            }
            __syncwarp();
            const int np = (n + 1) >> 1;
            float2 ax2 = make_float2(0.0f, 0.0f), ay2 = ax2, az2 = ax2, np2 = ax2;  // np2: minus the potential
            const float qx = v ? tx[1] : tx[0], qy = v ? ty[1] : ty[0], qz = v ? tz[1] : tz[0];
            const float qh = v ? th[1] : th[0];
            const float2 ntx = make_float2(-qx, -qx), nty = make_float2(-qy, -qy), ntz = make_float2(-qz, -qz);
            const float4* __restrict__ L = pp_of(v);
            const float2* __restrict__ H = reinterpret_cast<const float2*>(ph_of(v));
            for (int jp = 0; jp < np; ++jp) {
                const float4 P = L[2 * jp], Q = L[2 * jp + 1];
                const float2 hj = H[jp];
                const float2 X = make_float2(P.x, P.y), Y = make_float2(P.z, P.w);
                const float2 Z = make_float2(Q.x, Q.y), M = make_float2(Q.z, Q.w);
                const float2 dx = __fadd2_rn(X, ntx), dy = __fadd2_rn(Y, nty), dz = __fadd2_rn(Z, ntz);
                const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                const float2 hh = make_float2(fmaxf(qh, hj.x), fmaxf(qh, hj.y));
                const float2 hh2 = __fmul2_rn(hh, hh);
                const bool z0 = r2.x == 0.0f, z1 = r2.y == 0.0f;
                if (COUNT) c_zero += (unsigned long long)z0 + (unsigned long long)z1;
                if ((r2.x >= hh2.x || z0) && (r2.y >= hh2.y || z1)) {
                    const float2 ri = make_float2(z0 ? 0.0f : rsqrt_ftz(r2.x), z1 ? 0.0f : rsqrt_ftz(r2.y));
                    const float2 mri = __fmul2_rn(M, ri);
                    const float2 f = __fmul2_rn(mri, __fmul2_rn(ri, ri));
                    ax2 = __ffma2_rn(dx, f, ax2);
                    ay2 = __ffma2_rn(dy, f, ay2);
                    az2 = __ffma2_rn(dz, f, az2);
                    if (WANT_POT) np2 = __fadd2_rn(np2, mri);
                } else {
                    // the same terms one entry at a time, the spline where r < h
                    const float r2s[2] = {r2.x, r2.y}, hs[2] = {hh.x, hh.y}, ms[2] = {M.x, M.y};
                    float fs[2], ps[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        if (r2s[e] >= hs[e] * hs[e] && r2s[e] > 0.0f) {
                            const float ri = rsqrt_ftz(r2s[e]);
                            const float mri = ms[e] * ri;
                            fs[e] = mri * (ri * ri);
                            ps[e] = -mri;
                        } else {
                            spline_pair(r2s[e], hs[e], ms[e], fs[e], ps[e]);
                        }
                    }
                    const float2 f = make_float2(fs[0], fs[1]);
                    ax2 = __ffma2_rn(dx, f, ax2);
                    ay2 = __ffma2_rn(dy, f, ay2);
                    az2 = __ffma2_rn(dz, f, az2);
                    if (WANT_POT) np2 = __fadd2_rn(np2, make_float2(-ps[0], -ps[1]));
                }
            }
            add_partial(v, ax2.x + ax2.y, ay2.x + ay2.y, az2.x + az2.y, -(np2.x + np2.y));
            if (COUNT) c_flush += (lane == 0);
            __syncwarp();
        };

        // ---- traversal ----------------------------------------------------------------------
        // One loop: each pass either walks one traversal step or places the next 32 particles of
        // the leaves the last step expanded.  A pass adds at most 32 entries to each list, so the
        // lists are flushed at the top of the loop, when the next pass could overflow them, and at
        // the end: one flush site per list kind, which keeps the kernel's code small (instruction
        // fetch, not arithmetic, limited the first version with a flush at every append site).
        // the root of each window: node 0, or in a forest its system's root; windows of one
        // system share a root entry, windows of two systems start from one entry each
        int top = 1;
        {
            const int ra = A.group_root ? A.group_root[2 * pr] : 0;
            const int rb = (A.group_root && nt[1] > 0) ? A.group_root[2 * pr + 1] : ra;
            if (ra == rb) {
                if (lane == 0) stk[0] = (ra << 2) | 1 | (nt[1] > 0 ? 2 : 0);
            } else {
                if (lane == 0) { stk[0] = (ra << 2) | 1; stk[1] = (rb << 2) | 2; }
                top = 2;
            }
        }
        __syncwarp();
        int npn0 = 0, npn1 = 0, npp0 = 0, npp1 = 0;
        int base = 0, tot2 = 0;  // the expanded leaves' particles still to place: [base, tot2)
        bool overflow = false;
        for (;;) {
            const bool done = top == 0 && base >= tot2;
#pragma unroll 1
            for (int v = 0; v < 2; ++v) {
                const int n1 = v ? npn1 : npn0, n2 = v ? npp1 : npp0;
                if (n1 > 0 && (done || n1 > A.pn_cap - 32)) {
                    flush_pn(v, n1);
                    if (v) npn1 = 0; else npn0 = 0;
                }
                if (n2 > 0 && (done || n2 > A.pp_cap - 32)) {
                    flush_pp(v, n2);
                    if (v) npp1 = 0; else npp0 = 0;
                }
            }
            if (done) break;

            if (base < tot2) {
                // 32 expanded-leaf particles, one per lane, to the windows that opened their leaf:
                // a particle farther from a window's box than max(its largest target softening,
                // the particle's) is a monopole for that window, the rest need the softened pair
                const int q = base + lane;
                const bool live = q < tot2;
                double qx = 0, qy = 0, qz = 0;
                float qm = 0.0f, qh = 0.0f;
                int wm = 0;
                if (live) {
                    int l = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1)
                        if (S.pre[l + step] <= q) l += step;
                    int qpos = S.lo[l] + (q - S.pre[l]);
                    if (!GT_IN_BOUNDS(qpos, A.n_src)) qpos = 0;
                    load_src(A.src + qpos, qx, qy, qz, qm, qh);
                    wm = S.msk[l];
                }
#pragma unroll
                for (int v = 0; v < 2; ++v) {
                    const bool in = (wm >> v) & 1;
                    bool far = false;
                    if (in) {
                        const double ex = box_gap(qx, S.wb[v].c_x, S.wb[v].w_x);
                        const double ey = box_gap(qy, S.wb[v].c_y, S.wb[v].w_y);
                        const double ez = box_gap(qz, S.wb[v].c_z, S.wb[v].w_z);
                        const double qhd = (double)qh;
                        const double reach = S.wb[v].emax > qhd ? S.wb[v].emax : qhd;
                        far = ex * ex + ey * ey + ez * ez > reach * reach;
                    }
                    const unsigned fm = __ballot_sync(kFull, in && far);
                    const unsigned nm = __ballot_sync(kFull, in && !far);
                    int& npn = v ? npn1 : npn0;
                    int& npp = v ? npp1 : npp0;
                    if (COUNT && lane == 0) c_pairs += (unsigned long long)__popc(fm | nm) * nt[v];
                    const float ex = (float)(qx - S.wb[v].c_x), ey = (float)(qy - S.wb[v].c_y), ez = (float)(qz - S.wb[v].c_z);
                    if (in && far && GT_IN_BOUNDS(npn + __popc(fm & lt_mask), A.pn_cap)) {
                        pn_put(v, npn + __popc(fm & lt_mask), ex, ey, ez, qm);
                    } else if (in && GT_IN_BOUNDS(npp + __popc(nm & lt_mask), A.pp_cap)) {
                        const int pos = npp + __popc(nm & lt_mask);
                        pp_put(v, pos, ex, ey, ez, qm);
                        ph_of(v)[pos] = qh;
                    }
                    npn += __popc(fm);
                    npp += __popc(nm);
                }
                base += 32;
                __syncwarp();
                continue;
            }

            // one traversal step: pop up to 32 nodes, test each against its windows
            const int npop = min(top, 32);
            top -= npop;
            const int ent = lane < npop ? stk[top + lane] : -1;
            int node = ent >= 0 ? (ent >> 2) : -1;
            if (node >= 0 && !GT_IN_BOUNDS(node, A.n_nodes)) node = -1;
            const int mk = node >= 0 ? (ent & 3) : 0;
            __syncwarp();
            const NodeV nd = load_node(A.nodes + (node >= 0 ? node : 0));
            const bool leaf = nd.first < 0;
            if (COUNT) {
                const unsigned tests = __reduce_add_sync(kFull, (unsigned)__popc(mk));
                if (lane == 0) { c_nodes += tests; ++c_steps; }
            }
            bool acc[2], opn[2];
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                acc[v] = false;
                opn[v] = false;
                if ((mk >> v) & 1) {
                    const double dx = box_gap(nd.cx, S.wb[v].c_x, S.wb[v].w_x);
                    const double dy = box_gap(nd.cy, S.wb[v].c_y, S.wb[v].w_y);
                    const double dz = box_gap(nd.cz, S.wb[v].c_z, S.wb[v].w_z);
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    const double len = (double)nd.len;
                    const double ml2 = MAC == 2 ? nd.mass * (double)__ldg(A.mac_l2 + node) : nd.mass * len * len;
                    const bool o = open_node(r2, len, nd.s, ml2, (double)nd.soft, S.wb[v].emax, S.wb[v].amin, A.theta2,
                                             dx, dy, dz);
                    acc[v] = !o;
                    opn[v] = o;
                }
            }
            const int pm = (opn[0] ? 1 : 0) | (opn[1] ? 2 : 0);  // the windows that open this node
            const bool push = pm != 0 && !leaf, expand = pm != 0 && leaf;

            // children of opened interior nodes, with the windows that opened them; one scan for
            // the children's stack slots and the expanded leaves' particle slots (walk_kernel)
            const int nch = push ? nd.nchild : 0;
            const int cnt = expand ? nd.phi - nd.plo : 0;
            int incl, inc2;
            if (!__any_sync(kFull, cnt >= (1 << 16))) {
                const int both = warp_incl_scan_i(nch | (cnt << 10));
                incl = both & 1023;
                inc2 = both >> 10;
            } else {
                incl = warp_incl_scan_i(nch);
                inc2 = warp_incl_scan_i(cnt);
            }
            const int tot = __shfl_sync(kFull, incl, 31);
            if (top + tot > A.stack_cap) { overflow = true; break; }
            {
                int* dst = stk + (top + incl - nch);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (c < nch) dst[c] = ((nd.first + c) << 2) | pm;
            }
            top += tot;
            if (COUNT) c_maxtop = max(c_maxtop, top);

            // accepted nodes: monopoles of the windows that accept them
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const unsigned am = __ballot_sync(kFull, acc[v]);
                int& npn = v ? npn1 : npn0;
                if (COUNT && lane == 0) c_multi += (unsigned long long)__popc(am) * nt[v];
                if (acc[v] && GT_IN_BOUNDS(npn + __popc(am & lt_mask), A.pn_cap))
                    pn_put(v, npn + __popc(am & lt_mask), (float)(nd.cx - S.wb[v].c_x), (float)(nd.cy - S.wb[v].c_y),
                           (float)(nd.cz - S.wb[v].c_z), (float)nd.mass);
                npn += __popc(am);
            }

            // expanded leaves: their particles are placed by the next passes
            tot2 = __shfl_sync(kFull, inc2, 31);
            base = 0;
            if (tot2 > 0) {
                S.lo[lane] = nd.plo;
                S.pre[lane] = inc2 - cnt;
                S.msk[lane] = pm;
            }
            __syncwarp();
        }
        if (overflow) {
            if (lane == 0) atomicExch(A.error, 1);
            continue;
        }

        // ---- write --------------------------------------------------------------------------
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            if (lane < nt[v]) {
                const int idx = t0[v] + lane;
                const int o = A.out_map ? (int)A.out_map[idx] : idx;
                if (!GT_IN_BOUNDS(o, A.n_out)) continue;
                const float sx = v ? sx1 : sx0, sy = v ? sy1 : sy0, sz = v ? sz1 : sz0;
                const float cx = v ? cx1 : cx0, cy = v ? cy1 : cy0, cz = v ? cz1 : cz0;
                if (A.ax) {
                    A.ax[o] = A.G * ((double)sx - (double)cx);
                    A.ay[o] = A.G * ((double)sy - (double)cy);
                    A.az[o] = A.G * ((double)sz - (double)cz);
                }
                if (WANT_POT && A.phi) A.phi[o] = A.G * (v ? pot1 : pot0);
            }
        }
    }
    if (COUNT) {
        if (lane == 0) {
            atomicAdd(&A.stats[0], c_nodes);
            atomicAdd(&A.stats[1], c_multi);
            atomicAdd(&A.stats[2], c_pairs);
            atomicAdd(&A.stats[4], c_flush);
            atomicMax(&A.stats[5], (unsigned long long)c_maxtop);
            atomicAdd(&A.stats[6], c_steps);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c_zero += __shfl_xor_sync(kFull, c_zero, o);
        if (lane == 0) atomicAdd(&A.stats[3], c_zero);
    }
}

// ---------------------------------------------------------------------------------------------
// Groups
// ---------------------------------------------------------------------------------------------

// Mark the first tree position of every leaf (mode 0) or group node (mode 1).
__global__ void mark_group_nodes_kernel(const GNode* __restrict__ nodes, const int* __restrict__ parent,
                                        int64_t n_nodes, int mode, int gmax, uint32_t* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        const GNode& nd = nodes[i];
        const int cnt = nd.phi - nd.plo;
        if (cnt <= 0) continue;
        bool mark;
        if (mode == 0) {
            mark = nd.first < 0;
        } else {
            const int pa = parent[i];
            const bool parent_big = pa < 0 || (nodes[pa].phi - nodes[pa].plo) > gmax;
            mark = (cnt <= gmax && parent_big) || (nd.first < 0 && cnt > gmax);
        }
        if (mark) flag[nd.plo] = 1u;
    }
}

// Per-tree-position group node id (mode 1), for explicit target lists.
__global__ void fill_group_id_kernel(const GNode* __restrict__ nodes, const int* __restrict__ parent,
                                     int64_t n_nodes, int gmax, int* __restrict__ gid) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        const GNode& nd = nodes[i];
        const int cnt = nd.phi - nd.plo;
        if (cnt <= 0) continue;
        const int pa = parent[i];
        const bool parent_big = pa < 0 || (nodes[pa].phi - nodes[pa].plo) > gmax;
        if ((cnt <= gmax && parent_big) || (nd.first < 0 && cnt > gmax))
            for (int p = nd.plo; p < nd.phi; ++p) gid[p] = (int)i;
    }
}

// A target index as the grouping reads it: an index at or beyond the particle count sets *bad
// (the call then fails with GT_ERR_INVALID) and reads particle 0 instead, so nothing is read out of
// bounds; the check costs nothing on the host, which does not walk the target list.
__device__ __forceinline__ uint32_t checked_target(const uint32_t* __restrict__ targets, int64_t k, int64_t n,
                                                   unsigned* __restrict__ bad) {
    const uint32_t p = targets[k];
    if ((int64_t)p < n) return p;
    if (bad) atomicOr(bad, 1u);
    return 0u;
}

// Whether target k starts a group (a new group where the key changes or is negative); also
// records its tree position.  In a forest a target's system comes from its particle index
// (in_off): massless particles sit after every live one in tree order, outside sys_off's ranges.
__device__ __forceinline__ bool target_starts(const uint32_t* __restrict__ targets, int64_t k, int mode,
                                              int param, const uint32_t* __restrict__ rank,
                                              const int* __restrict__ leaf_of, const int* __restrict__ gid,
                                              uint32_t* __restrict__ tpos, const int* __restrict__ sys_off,
                                              const int64_t* __restrict__ in_off, int n_systems, int all_live,
                                              int64_t n, unsigned* __restrict__ bad) {
    const uint32_t p = checked_target(targets, k, n, bad);
    const uint32_t pos = rank[p];
    tpos[k] = pos;
    if (k == 0) return true;
    const uint32_t q = checked_target(targets, k - 1, n, nullptr);  // reported at its own k
    if (mode == GT_GROUP_LEAF) {
        const int a = leaf_of[p], b = leaf_of[q];
        return a != b || a < 0;
    }
    if (mode == GT_GROUP_NODE) {
        const int a = gid[pos], b = gid[rank[q]];
        return a != b || a < 0;
    }
    if (mode == GT_GROUP_BATCH) {
        if (n_systems > 1) {
            // a window never spans two systems of a forest; over all live targets the windows of
            // each system start at its first particle, as in its own tree
            const int s = system_of(in_off, n_systems, p);
            return s != system_of(in_off, n_systems, q) ||
                   (all_live ? ((int64_t)pos - sys_off[s]) % param == 0 : (k % param) == 0);
        }
        return (k % param) == 0;
    }
    return true;
}

__global__ void target_flags_kernel(const uint32_t* __restrict__ targets, int64_t nt, int mode,
                                    int param, const uint32_t* __restrict__ rank,
                                    const int* __restrict__ leaf_of, const int* __restrict__ gid,
                                    uint32_t* __restrict__ tpos, uint32_t* __restrict__ flag,
                                    const int* __restrict__ sys_off, const int64_t* __restrict__ in_off,
                                    int n_systems, int all_live, int64_t n = INT64_MAX,
                                    unsigned* __restrict__ bad = nullptr) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nt;
         k += (int64_t)gridDim.x * blockDim.x)
        flag[k] = target_starts(targets, k, mode, param, rank, leaf_of, gid, tpos, sys_off, in_off, n_systems,
                                all_live, n, bad) ? 1u : 0u;
}

// Small explicit target lists (the sparse active sets of deep time bins) form their groups in one
// block, in one launch: flags, an ordered compaction of the group starts into shared memory, then
// the chunking of groups longer than kmax.  count[0] = groups, count[1] = chunks, as
// finish_groups_dev leaves them; the walk reads count[1].
constexpr int kSmallTargets = 8192;
constexpr int kSmallThreads = 1024;

// Exclusive scan of one value per thread over the 1024-thread block; *total gets the sum.
__device__ __forceinline__ int block_excl_scan_1024(int v, int* wsum, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        const int x = wsum[lane];
        int y = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, y, o);
            if (lane >= o) y += t;
        }
        wsum[lane] = y - x;
        if (lane == 31) *total = y;
    }
    __syncthreads();
    const int r = inc - v + wsum[w];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kSmallThreads)
small_groups_kernel(const uint32_t* __restrict__ targets, int nt, int mode, int param,
                    const uint32_t* __restrict__ rank, const int* __restrict__ leaf_of,
                    const int* __restrict__ gid, uint32_t* __restrict__ tpos,
                    const int* __restrict__ sys_off, const int64_t* __restrict__ in_off, int n_systems,
                    int kmax, int2* __restrict__ groups, uint32_t* __restrict__ count, int64_t n,
                    unsigned* __restrict__ bad) {
    __shared__ int starts[kSmallTargets + 1];
    __shared__ int wsum[32];
    __shared__ int total;
    int ng = 0;
    for (int base = 0; base < nt; base += kSmallThreads) {
        const int k = base + (int)threadIdx.x;
        const bool st = k < nt && target_starts(targets, k, mode, param, rank, leaf_of, gid, tpos, sys_off,
                                                in_off, n_systems, 0, n, bad);
        const int at = block_excl_scan_1024(st ? 1 : 0, wsum, &total);
        if (st) starts[ng + at] = k;
        ng += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) starts[ng] = nt;
    __syncthreads();
    int nc = 0;
    for (int base = 0; base < ng; base += kSmallThreads) {
        const int gi = base + (int)threadIdx.x;
        const int s = gi < ng ? starts[gi] : 0, e = gi < ng ? starts[gi + 1] : 0;
        const int c = gi < ng ? (e - s + kmax - 1) / kmax : 0;
        int o = nc + block_excl_scan_1024(c, wsum, &total);
        for (int a = s; a < e; a += kmax, ++o) groups[o] = make_int2(a, min(a + kmax, e));
        nc += total;
    }
    if (threadIdx.x == 0) { count[0] = (uint32_t)ng; count[1] = (uint32_t)nc; }
}

__global__ void compact_starts_kernel(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                                      int64_t n, int64_t* __restrict__ starts) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (flag[i]) starts[pos[i]] = i;
}

// Fixed windows of `w` consecutive targets over all n live particles of one system.
__global__ void window_groups_kernel(int2* __restrict__ groups, int64_t ng, int64_t n, int w) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng;
         g += (int64_t)gridDim.x * blockDim.x)
        groups[g] = make_int2((int)(g * w), (int)std::min<int64_t>((g + 1) * w, n));
}

// Split groups longer than kmax into consecutive chunks (each walks with its own, tighter box).
__global__ void chunk_count_kernel(const int64_t* __restrict__ starts, int64_t ng, int64_t n_end,
                                   int kmax, uint32_t* __restrict__ nchunk) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = starts[g], e = (g + 1 < ng) ? starts[g + 1] : n_end;
        nchunk[g] = (uint32_t)((e - s + kmax - 1) / kmax);
    }
}

__global__ void chunk_emit_kernel(const int64_t* __restrict__ starts, int64_t ng, int64_t n_end, int kmax,
                                  const uint32_t* __restrict__ coff, int2* __restrict__ groups) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = starts[g], e = (g + 1 < ng) ? starts[g + 1] : n_end;
        int64_t o = coff[g];
        for (int64_t a = s; a < e; a += kmax, ++o) groups[o] = make_int2((int)a, (int)std::min<int64_t>(a + kmax, e));
    }
}

// Forest: the root of each group is the root of the system of its first target (roots are
// nodes 0 .. n_systems-1, groups never span two systems).  All live targets: group members are
// live tree positions (sys_off); explicit targets: particle indices (in_off), below n as the
// grouping has checked (an index beyond it has failed the call and reads system 0 here).
__global__ void group_root_kernel(const int2* __restrict__ groups, int64_t ng, const uint32_t* __restrict__ targets,
                                  int64_t n, const int* __restrict__ sys_off, const int64_t* __restrict__ in_off,
                                  int n_systems, int* __restrict__ root, const uint32_t* __restrict__ ng_dev = nullptr) {
    if (ng_dev) ng = min(ng, (int64_t)*ng_dev);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int t0 = groups[g].x;
        if (targets) {
            const int64_t p = (int64_t)targets[t0];
            root[g] = p < n ? system_of(in_off, n_systems, p) : 0;
        } else {
            root[g] = system_of(sys_off, n_systems, (int64_t)t0);
        }
    }
}

int grid1d(gt_context* ctx, int64_t n) {
    const int64_t want = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->num_sms * 8));
}

uint32_t read_u32(gt_context* ctx, const uint32_t* dev) {
    check_cuda(cudaMemcpyAsync(ctx->pinned, dev, 4, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
    check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
    uint32_t v;
    std::memcpy(&v, ctx->pinned, 4);
    return v;
}

// Turn group starts (flag array over n items) into chunked [start, end) pairs in `out`.
// Returns the number of chunks.  `out` is allocated with cudaMalloc when own_out is set.
int64_t finish_groups(gt_context* ctx, const uint32_t* flag, int64_t n, int kmax, int2** out, bool own_out) {
    uint32_t* pos = (uint32_t*)scratch(ctx, kSlotScanA, (size_t)n * 4);
    uint32_t* total = (uint32_t*)scratch(ctx, kSlotCounters, 64);
    scan_exclusive_u32(ctx, flag, pos, n, total);
    const int64_t ng = read_u32(ctx, total);
    int64_t* starts = (int64_t*)scratch(ctx, kSlotGroupsA, (size_t)(ng + 1) * 8);
    compact_starts_kernel<<<grid1d(ctx, n), 256, 0, ctx->stream>>>(flag, pos, n, starts);
    check_launch(ctx, "compact_starts_kernel");
    uint32_t* nchunk = (uint32_t*)scratch(ctx, kSlotNodeTmp1, (size_t)std::max<int64_t>(ng, 1) * 4);
    uint32_t* coff = (uint32_t*)scratch(ctx, kSlotNodeTmp2, (size_t)std::max<int64_t>(ng, 1) * 4);
    chunk_count_kernel<<<grid1d(ctx, ng), 256, 0, ctx->stream>>>(starts, ng, n, kmax, nchunk);
    check_launch(ctx, "chunk_count_kernel");
    scan_exclusive_u32(ctx, nchunk, coff, ng, total);
    const int64_t nc = read_u32(ctx, total);
    int2* groups;
    if (own_out) {
        void* p = nullptr;
        if (cudaMalloc(&p, (size_t)std::max<int64_t>(nc, 1) * sizeof(int2)) != cudaSuccess) {
            cudaGetLastError();
            throw Fail{GT_ERR_NOMEM, "cudaMalloc for the group list failed"};
        }
        groups = (int2*)p;
    } else {
        groups = (int2*)scratch(ctx, kSlotGroupsB, (size_t)std::max<int64_t>(nc, 1) * sizeof(int2));
    }
    chunk_emit_kernel<<<grid1d(ctx, ng), 256, 0, ctx->stream>>>(starts, ng, n, kmax, coff, groups);
    check_launch(ctx, "chunk_emit_kernel");
    *out = groups;
    return nc;
}

// The same chunking with the group count on the device (gc[0]): no host read-back.  Threads past
// the count write no chunks.
__global__ void chunk_count_dev_kernel(const int64_t* __restrict__ starts, const uint32_t* __restrict__ gc,
                                       int64_t cap, int64_t n_end, int kmax, uint32_t* __restrict__ nchunk) {
    const int64_t ng = min(cap, (int64_t)gc[0]);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < cap;
         g += (int64_t)gridDim.x * blockDim.x) {
        if (g >= ng) { nchunk[g] = 0; continue; }
        const int64_t s = starts[g], e = (g + 1 < ng) ? starts[g + 1] : n_end;
        nchunk[g] = (uint32_t)((e - s + kmax - 1) / kmax);
    }
}

__global__ void chunk_emit_dev_kernel(const int64_t* __restrict__ starts, const uint32_t* __restrict__ gc,
                                      int64_t cap, int64_t n_end, int kmax, const uint32_t* __restrict__ coff,
                                      int2* __restrict__ groups) {
    const int64_t ng = min(cap, (int64_t)gc[0]);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = starts[g], e = (g + 1 < ng) ? starts[g + 1] : n_end;
        int64_t o = coff[g];
        for (int64_t a = s; a < e; a += kmax, ++o) groups[o] = make_int2((int)a, (int)std::min<int64_t>(a + kmax, e));
    }
}

// Group starts (flag over n items) to chunked [start, end) pairs without a host read-back: the
// number of chunks stays on the device (*count_dev), at most n.  For explicit target lists, where
// a read-back per call is most of the cost of a small walk.
int2* finish_groups_dev(gt_context* ctx, const uint32_t* flag, int64_t n, int kmax, const uint32_t** count_dev) {
    cudaStream_t st = ctx->stream;
    uint32_t* gc = (uint32_t*)scratch(ctx, kSlotGroupCount, 64);  // [0] groups, [1] chunks
    uint32_t* pos = (uint32_t*)scratch(ctx, kSlotScanA, (size_t)n * 4);
    scan_exclusive_u32(ctx, flag, pos, n, gc);
    int64_t* starts = (int64_t*)scratch(ctx, kSlotGroupsA, (size_t)(n + 1) * 8);
    compact_starts_kernel<<<grid1d(ctx, n), 256, 0, st>>>(flag, pos, n, starts);
    check_launch(ctx, "compact_starts_kernel");
    uint32_t* nchunk = (uint32_t*)scratch(ctx, kSlotNodeTmp1, (size_t)n * 4);
    uint32_t* coff = (uint32_t*)scratch(ctx, kSlotNodeTmp2, (size_t)n * 4);
    chunk_count_dev_kernel<<<grid1d(ctx, n), 256, 0, st>>>(starts, gc, n, n, kmax, nchunk);
    check_launch(ctx, "chunk_count_dev_kernel");
    scan_exclusive_u32(ctx, nchunk, coff, n, gc + 1);
    int2* groups = (int2*)scratch(ctx, kSlotGroupsB, (size_t)n * sizeof(int2));
    chunk_emit_dev_kernel<<<grid1d(ctx, n), 256, 0, st>>>(starts, gc, n, n, kmax, coff, groups);
    check_launch(ctx, "chunk_emit_dev_kernel");
    *count_dev = gc + 1;
    return groups;
}

size_t walk_smem(int warps, bool mac, int pn_cap, int ext = 0) {
    return (size_t)warps * warp_smem_bytes(pn_cap, pn_cap / 2, ext) + (mac ? kMacModel * sizeof(float) : 0);
}

// Dynamic shared memory above 48 KB needs a per-kernel opt-in, done once per instantiation.
template <int TPL, bool LA, bool POT, bool CNT, int MAC, int XT = 0>
void prepare_walk() {
    static bool done = false;
    if (done) return;
    // the largest request of this instantiation: 8 warps at the largest list capacity (XT 1 lists
    // carry velocities too, so XT 1 stops at half the capacity)
    check_cuda(cudaFuncSetAttribute(walk_kernel<TPL, LA, POT, CNT, MAC, XT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)walk_smem(kMaxWarps, MAC == 1, XT == 1 ? kPnCapMax / 2 : kPnCapMax, XT)),
               "cudaFuncSetAttribute");
    // the lists need 3 blocks x 55 KB per SM: ask for the largest shared-memory carveout
    check_cuda(cudaFuncSetAttribute(walk_kernel<TPL, LA, POT, CNT, MAC, XT>,
                                    cudaFuncAttributePreferredSharedMemoryCarveout, 100),
               "cudaFuncSetAttribute");
    done = true;
}

template <int TPL, bool LA, bool POT, bool CNT, int MAC, int XT = 0>
void launch_walk(gt_context* ctx, const WalkArgs& a, int blocks, int warps) {
    prepare_walk<TPL, LA, POT, CNT, MAC, XT>();
    walk_kernel<TPL, LA, POT, CNT, MAC, XT><<<blocks, warps * 32, walk_smem(warps, MAC == 1, a.pn_cap, XT),
                                              ctx->stream>>>(a);
    check_launch(ctx, "walk_kernel");
}

template <int TPL, bool LA, bool POT, int MAC>
void dispatch_count(gt_context* ctx, const WalkArgs& a, int blocks, int warps, bool cnt) {
    if (cnt) launch_walk<TPL, LA, POT, true, MAC>(ctx, a, blocks, warps);
    else launch_walk<TPL, LA, POT, false, MAC>(ctx, a, blocks, warps);
}

// Tidal tensor / jerk / gas rules: plain criterion, groups of at most 32 targets.  The per-target
// walk (no leaf acceptance) only for the gas rules of accelerations.
template <int EXT>
void dispatch_ext_level(gt_context* ctx, const WalkArgs& a, int blocks, int warps, bool la, bool pot, bool cnt) {
    if (!la) {
        if (cnt) launch_walk<1, false, false, true, 0, EXT>(ctx, a, blocks, warps);
        else launch_walk<1, false, false, false, 0, EXT>(ctx, a, blocks, warps);
    } else if (pot) {
        if (cnt) launch_walk<1, true, true, true, 0, EXT>(ctx, a, blocks, warps);
        else launch_walk<1, true, true, false, 0, EXT>(ctx, a, blocks, warps);
    } else {
        if (cnt) launch_walk<1, true, false, true, 0, EXT>(ctx, a, blocks, warps);
        else launch_walk<1, true, false, false, 0, EXT>(ctx, a, blocks, warps);
    }
}

// ext 1: the tidal-tensor / jerk kernel (the gas rules too); ext 2: the gas rules alone
void dispatch_xt(gt_context* ctx, const WalkArgs& a, int blocks, int warps, int ext, bool la, bool pot, bool cnt) {
    if (ext == 1) dispatch_ext_level<1>(ctx, a, blocks, warps, la, pot, cnt);
    else dispatch_ext_level<2>(ctx, a, blocks, warps, la, pot, cnt);
}

// The learned criteria are grouped-walk options (leaves offered to the criterion).
template <int TPL>
void dispatch(gt_context* ctx, const WalkArgs& a, int blocks, int warps, bool la, bool pot, bool cnt,
              int mac) {
    if (mac == GT_MAC_LEARNED) {
        if (pot) dispatch_count<TPL, true, true, 1>(ctx, a, blocks, warps, cnt);
        else dispatch_count<TPL, true, false, 1>(ctx, a, blocks, warps, cnt);
    } else if (mac == GT_MAC_NODE) {
        if (pot) dispatch_count<TPL, true, true, 2>(ctx, a, blocks, warps, cnt);
        else dispatch_count<TPL, true, false, 2>(ctx, a, blocks, warps, cnt);
    } else if (la) {
        if (pot) dispatch_count<TPL, true, true, 0>(ctx, a, blocks, warps, cnt);
        else dispatch_count<TPL, true, false, 0>(ctx, a, blocks, warps, cnt);
    } else {
        if (pot) dispatch_count<TPL, false, true, 0>(ctx, a, blocks, warps, cnt);
        else dispatch_count<TPL, false, false, 0>(ctx, a, blocks, warps, cnt);
    }
}

// The paired-window walk: at most 512 list entries per window (two windows' lists of 8 warps fit
// the 227 KB of shared memory).
constexpr int kPairCapMax = 512;
constexpr int kPairCapDefault = 160;

size_t pair_smem(int warps, int pn_cap) { return (size_t)warps * pair_smem_bytes(pn_cap, pn_cap / 2); }

template <bool POT, bool CNT, int MAC>
void prepare_pair() {
    static bool done = false;
    if (done) return;
    check_cuda(cudaFuncSetAttribute(walk_pair_kernel<POT, CNT, MAC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)pair_smem(kMaxWarps, kPairCapMax)),
               "cudaFuncSetAttribute");
    check_cuda(cudaFuncSetAttribute(walk_pair_kernel<POT, CNT, MAC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    100),
               "cudaFuncSetAttribute");
    done = true;
}

template <bool POT, bool CNT, int MAC>
int pair_occupancy(int warps, int pn_cap) {
    prepare_pair<POT, CNT, MAC>();
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_pair_kernel<POT, CNT, MAC>, warps * 32,
                                                  pair_smem(warps, pn_cap));
    return std::max(1, nb);
}

template <bool POT, bool CNT, int MAC>
void launch_pair(gt_context* ctx, const WalkArgs& a, int blocks, int warps) {
    prepare_pair<POT, CNT, MAC>();
    walk_pair_kernel<POT, CNT, MAC><<<blocks, warps * 32, pair_smem(warps, a.pn_cap), ctx->stream>>>(a);
    check_launch(ctx, "walk_pair_kernel");
}

template <bool POT, bool CNT>
void dispatch_pair_mac(gt_context* ctx, const WalkArgs& a, int blocks, int warps, int mac) {
    if (mac == GT_MAC_NODE) launch_pair<POT, CNT, 2>(ctx, a, blocks, warps);
    else launch_pair<POT, CNT, 0>(ctx, a, blocks, warps);
}

void dispatch_pair(gt_context* ctx, const WalkArgs& a, int blocks, int warps, bool pot, bool cnt, int mac) {
    if (pot) {
        if (cnt) dispatch_pair_mac<true, true>(ctx, a, blocks, warps, mac);
        else dispatch_pair_mac<true, false>(ctx, a, blocks, warps, mac);
    } else {
        if (cnt) dispatch_pair_mac<false, true>(ctx, a, blocks, warps, mac);
        else dispatch_pair_mac<false, false>(ctx, a, blocks, warps, mac);
    }
}

// Chunks of the copy-overlapped walk, as cumulative percentages of the targets.  The first chunk is
// small, so the walk starts once a tenth of the host aold is across, and so is the last, so that
// little of the results' download is left when the last kernel ends; the chunks between are large
// enough that each one's download hides under the next one's walk.
constexpr int kChunks = 5;
struct ChunkEdges {
    int pct[kChunks + 1];
};
constexpr ChunkEdges kChunkEdge{{0, 10, 45, 80, 93, 100}};

// Chunk boundaries of a group list for the copy-overlapped walk: chunk c starts at the first group
// whose first target is at or after nt * edges.pct[c] / 100 (rounded down to an even group when
// the walk pairs windows, so that no pair straddles two chunks).  out: kChunks+1 pairs (group
// index, first target).
__global__ void chunk_bounds_kernel(const int2* __restrict__ groups, int ng, int nt, ChunkEdges edges,
                                    int2* __restrict__ out, const uint32_t* __restrict__ ng_dev, int even) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (ng_dev) ng = min(ng, (int)*ng_dev);
    for (int c = 0; c <= kChunks; ++c) {
        const int64_t want = (int64_t)nt * edges.pct[c] / 100;
        int lo = 0, hi = ng;  // first g with groups[g].x >= want
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (groups[mid].x < want) lo = mid + 1; else hi = mid;
        }
        if (even && c > 0 && c < kChunks) lo &= ~1;
        out[c] = make_int2(lo, lo < ng ? groups[lo].x : nt);
    }
}

template <int TPL, bool LA, bool POT, bool CNT, int MAC, int XT = 0>
int occupancy_blocks(int warps, int pn_cap) {
    prepare_walk<TPL, LA, POT, CNT, MAC, XT>();
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, walk_kernel<TPL, LA, POT, CNT, MAC, XT>, warps * 32,
                                                  walk_smem(warps, MAC == 1, pn_cap, XT));
    return std::max(1, nb);
}

struct OutputCopy {
    const double* dev;
    double* host;
    int stride;
};

}  // namespace

bool run_walk(gt_context* ctx, const gt_tree* tc, const WalkRequest& rq) {
    gt_tree* t = const_cast<gt_tree*>(tc);  // only the group cache is mutated
    cudaStream_t st = ctx->stream;
    const bool all = rq.targets == nullptr;
    const int64_t nt = all ? t->n_live : rq.n_targets;
    ctx->stats = gt_walk_stats{};
    ctx->stats.targets = nt;
    if (nt <= 0) return false;
    if (nt > (int64_t)INT32_MAX) throw Fail{GT_ERR_INVALID, "too many targets for one walk"};

    int mode = rq.group_mode;
    int param = rq.group_param;
    if (mode == GT_GROUP_NODE && param <= 0) param = 32;
    if (mode == GT_GROUP_BATCH && param <= 0) mode = GT_GROUP_LEAF;
    // a warp holds up to 32, 64 or 128 targets (1, 2 or 4 per lane); longer groups are chunked.
    // The tidal tensor, the jerk and the gas rules run on the XT kernel.
    const bool zeta_on = t->szeta && t->gas_zeta && rq.want_acc && rq.ax;
    const bool sink_on = t->nsink && rq.sink_radius > 0.0 && rq.leaf_accept;
    // ext 1: the tidal tensor or the jerk (with the gas rules if the tree has them); ext 2: the gas
    // rules alone.  Both walk groups of at most 32 targets.
    const int ext = (rq.tidal != nullptr || rq.jerk != nullptr) ? 1 : ((zeta_on || sink_on) ? 2 : 0);
    const bool xt = ext != 0;
    int kmax = 32;
    if (!xt && (mode == GT_GROUP_NODE || mode == GT_GROUP_BATCH) && param > 32) kmax = param > 64 ? 128 : 64;
    const int tpl = kmax / 32;

    // ---- groups -------------------------------------------------------------------------------
    int2* groups = nullptr;
    int* roots = nullptr;
    int64_t ng = 0;
    const uint32_t* tpos = nullptr;
    const uint32_t* ng_dev = nullptr;  // explicit targets: the group count stays on the device
    if (all) {
        // the cache is shared by every context that walks this tree: look up and fill it under
        // the tree's lock, and publish a new list only once it is complete on the device
        std::lock_guard<std::mutex> lk(t->lazy_mu);
        for (auto& c : t->group_cache)
            if (c.mode == mode && c.param == param && c.kmax == kmax) {
                groups = c.groups; roots = c.roots; ng = c.n_groups;
            }
        if (!groups && !rq.capture && mode == GT_GROUP_BATCH && t->n_systems == 1 && param <= kmax &&
            t->n_live > 0) {
            // fixed windows over the tree order of one system: [param*g, param*(g+1)), the same
            // list the flags below give, without their scans and read-backs
            const int64_t n = t->n_live;
            ng = (n + param - 1) / param;
            void* p = nullptr;
            if (cudaMallocAsync(&p, (size_t)ng * sizeof(int2), st) != cudaSuccess) {
                cudaGetLastError();
                throw Fail{GT_ERR_NOMEM, "cudaMallocAsync for the group list failed"};
            }
            groups = (int2*)p;
            window_groups_kernel<<<grid1d(ctx, ng), 256, 0, st>>>(groups, ng, n, param);
            check_launch(ctx, "window_groups_kernel");
            check_cuda(cudaStreamSynchronize(st), "sync");  // complete before other contexts see it
            gt_tree::GroupCache c;
            c.mode = mode; c.param = param; c.kmax = kmax; c.groups = groups; c.n_groups = ng; c.pooled = true;
            t->group_cache.push_back(c);
        }
        if (!groups) {
            const int64_t n = t->n_live;
            uint32_t* flag = (uint32_t*)scratch(ctx, kSlotTargets, (size_t)n * 4);
            check_cuda(cudaMemsetAsync(flag, 0, (size_t)n * 4, st), "memset");
            if (mode == GT_GROUP_LEAF || mode == GT_GROUP_NODE) {
                mark_group_nodes_kernel<<<grid1d(ctx, t->n_nodes), 256, 0, st>>>(
                    t->nodes, t->parent, t->n_nodes, mode == GT_GROUP_LEAF ? 0 : 1, param, flag);
                check_launch(ctx, "mark_group_nodes_kernel");
            } else {
                // fixed windows (or one group per target) over the tree order
                target_flags_kernel<<<grid1d(ctx, n), 256, 0, st>>>(
                    t->order, n, mode == GT_GROUP_BATCH ? GT_GROUP_BATCH : GT_GROUP_SINGLE, param,
                    t->rank, t->leaf_of, nullptr, (uint32_t*)scratch(ctx, kSlotGroupKey, (size_t)n * 4),
                    flag, t->sys_off_dev, t->in_off_dev, t->n_systems, 1);
                check_launch(ctx, "target_flags_kernel");
            }
            ng = finish_groups(ctx, flag, n, kmax, &groups, true);
            if (t->n_systems > 1 && ng > 0) {
                void* p = nullptr;
                if (cudaMalloc(&p, (size_t)ng * sizeof(int)) != cudaSuccess) {
                    cudaGetLastError();
                    cudaFree(groups);
                    throw Fail{GT_ERR_NOMEM, "cudaMalloc for the group roots failed"};
                }
                roots = (int*)p;
                group_root_kernel<<<grid1d(ctx, ng), 256, 0, st>>>(groups, ng, nullptr, 0, t->sys_off_dev,
                                                                   t->in_off_dev, t->n_systems, roots);
                check_launch(ctx, "group_root_kernel");
            }
            if (!rq.capture) check_cuda(cudaStreamSynchronize(st), "sync");
            gt_tree::GroupCache c;
            c.mode = mode; c.param = param; c.kmax = kmax; c.groups = groups; c.roots = roots; c.n_groups = ng;
            t->group_cache.push_back(c);
        }
    } else {
        uint32_t* tp = (uint32_t*)scratch(ctx, kSlotGroupKey, (size_t)nt * 4);
        uint32_t* flag = (uint32_t*)scratch(ctx, kSlotTargets, (size_t)nt * 4);
        int* gid = nullptr;
        if (mode == GT_GROUP_NODE) {
            gid = (int*)scratch(ctx, kSlotNodeTmp0, (size_t)std::max<int64_t>(t->n, 1) * 4);
            check_cuda(cudaMemsetAsync(gid, 0xff, (size_t)std::max<int64_t>(t->n, 1) * 4, st), "memset");
            fill_group_id_kernel<<<grid1d(ctx, t->n_nodes), 256, 0, st>>>(t->nodes, t->parent, t->n_nodes,
                                                                          param, gid);
            check_launch(ctx, "fill_group_id_kernel");
        }
        // every chunk holds at least one target: nt bounds the count, which the walk reads on the
        // device, so the call needs no read-back before the walk
        // gc[2]: set when a target index is out of range (read by the caller after the walk)
        uint32_t* gc = (uint32_t*)scratch(ctx, kSlotGroupCount, 64);
        check_cuda(cudaMemsetAsync(gc + 2, 0, 4, st), "memset");
        unsigned* bad = gc + 2;
        if (nt <= kSmallTargets) {
            groups = (int2*)scratch(ctx, kSlotGroupsB, (size_t)nt * sizeof(int2));
            small_groups_kernel<<<1, kSmallThreads, 0, st>>>(rq.targets, (int)nt, mode, param, t->rank, t->leaf_of,
                                                             gid, tp, t->sys_off_dev, t->in_off_dev, t->n_systems,
                                                             kmax, groups, gc, t->n, bad);
            check_launch(ctx, "small_groups_kernel");
            ng_dev = gc + 1;
        } else {
            target_flags_kernel<<<grid1d(ctx, nt), 256, 0, st>>>(rq.targets, nt, mode, param, t->rank,
                                                                 t->leaf_of, gid, tp, flag, t->sys_off_dev,
                                                                 t->in_off_dev, t->n_systems, 0, t->n, bad);
            check_launch(ctx, "target_flags_kernel");
            groups = finish_groups_dev(ctx, flag, nt, kmax, &ng_dev);
        }
        ng = nt;
        tpos = tp;
        if (t->n_systems > 1) {
            roots = (int*)scratch(ctx, kSlotGroupRoot, (size_t)ng * sizeof(int));
            group_root_kernel<<<grid1d(ctx, ng), 256, 0, st>>>(groups, ng, rq.targets, t->n, t->sys_off_dev,
                                                               t->in_off_dev, t->n_systems, roots, ng_dev);
            check_launch(ctx, "group_root_kernel");
        }
    }
    ctx->stats.groups = ng;
    if (ng <= 0) return false;

    // ---- launch -------------------------------------------------------------------------------
    const int warps = (rq.block_warps > 0 && rq.block_warps <= kMaxWarps) ? rq.block_warps : kMaxWarps;
    const bool mac = rq.mac == GT_MAC_LEARNED;
    const bool macn = rq.mac == GT_MAC_NODE;
    int pn_cap = kPnCapDefault;
    if (rq.list_capacity != 0) {
        if (rq.list_capacity < 64 || rq.list_capacity > kPnCapMax || (rq.list_capacity & 31))
            throw Fail{GT_ERR_INVALID, "list_capacity must be a multiple of 32 in [64, 1024]"};
        pn_cap = rq.list_capacity;
    }
    if (ext == 1 && pn_cap > kPnCapMax / 2)
        throw Fail{GT_ERR_INVALID, "list_capacity must be at most 512 with the tidal tensor or the jerk"};
    // two consecutive windows per warp (walk_pair_kernel) where it applies; its default lists hold
    // 128 entries per window, so that three blocks of eight warps fit an SM
    const bool paired = rq.pair_windows && !xt && tpl == 1 && mode == GT_GROUP_BATCH && param > 16 &&
                        rq.leaf_accept && !mac && t->n_nodes < (1 << 29) && pn_cap <= kPairCapMax;
    if (paired && rq.list_capacity == 0) pn_cap = kPairCapDefault;
    int per_sm;
    if (paired)
        per_sm = macn ? pair_occupancy<false, false, 2>(warps, pn_cap) : pair_occupancy<false, false, 0>(warps, pn_cap);
    else if (ext == 1)
        per_sm = occupancy_blocks<1, true, false, false, 0, 1>(warps, pn_cap);
    else if (ext == 2)
        per_sm = occupancy_blocks<1, true, false, false, 0, 2>(warps, pn_cap);
    else if (tpl == 1)
        per_sm = mac ? occupancy_blocks<1, true, false, false, 1>(warps, pn_cap)
               : macn ? occupancy_blocks<1, true, false, false, 2>(warps, pn_cap)
                      : (rq.leaf_accept ? occupancy_blocks<1, true, false, false, 0>(warps, pn_cap)
                                        : occupancy_blocks<1, false, false, false, 0>(warps, pn_cap));
    else if (tpl == 2)
        per_sm = mac ? occupancy_blocks<2, true, false, false, 1>(warps, pn_cap)
               : macn ? occupancy_blocks<2, true, false, false, 2>(warps, pn_cap)
                      : occupancy_blocks<2, true, false, false, 0>(warps, pn_cap);
    else
        per_sm = mac ? occupancy_blocks<4, true, false, false, 1>(warps, pn_cap)
               : macn ? occupancy_blocks<4, true, false, false, 2>(warps, pn_cap)
                      : occupancy_blocks<4, true, false, false, 0>(warps, pn_cap);
    const int64_t want_blocks = ((paired ? (ng + 1) / 2 : ng) + warps - 1) / warps;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want_blocks, (int64_t)per_sm * ctx->num_sms));
    int stack_cap = rq.stack_capacity > 0 ? rq.stack_capacity : 256 * std::max(1, t->n_levels) + 32;
    stack_cap = (stack_cap + 31) & ~31;

    WalkArgs a;
    a.nodes = t->nodes;
    a.src = t->src;
    a.ssoft = t->ssoft;
    a.tpos = tpos;
    a.aold = rq.aold;
    a.n_nodes = t->n_nodes;
    a.n_src = t->n;
    a.n_out = (all && rq.out_original) ? t->n : nt;
    a.groups = groups;
    a.n_groups = (int)ng;
    a.n_groups_dev = ng_dev;
    a.theta2 = rq.theta * rq.theta;
    a.G = rq.G;
    a.ax = rq.want_acc ? rq.ax : nullptr;
    a.ay = rq.want_acc ? rq.ay : nullptr;
    a.az = rq.want_acc ? rq.az : nullptr;
    a.phi = rq.phi;
    a.out_map = (all && rq.out_original) ? t->order : nullptr;
    const int total_warps = blocks * warps;
    a.pn_cap = pn_cap;
    a.pp_cap = pn_cap / 2;
    a.warp_bytes = paired ? pair_smem_bytes(a.pn_cap, a.pp_cap) : warp_smem_bytes(a.pn_cap, a.pp_cap, ext);
    a.tidal = rq.tidal;
    a.jerk = rq.jerk;
    a.svel = t->svel;
    a.nvel = t->nvel;
    if (xt && rq.mac != GT_MAC_PLAIN)
        throw Fail{GT_ERR_UNSUPPORTED, "the tidal tensor, the jerk and the gas rules take the plain criterion"};
    if (xt && !rq.leaf_accept && (rq.tidal || rq.jerk || (rq.want_phi && rq.phi)))
        throw Fail{GT_ERR_UNSUPPORTED, "the tidal tensor and the jerk come from the grouped walk"};
    a.stype = t->stype;
    a.szeta = zeta_on ? t->szeta : nullptr;
    a.smass = t->smass;
    a.nsink = sink_on ? t->nsink : nullptr;
    a.sink_r = rq.sink_radius;
    if (rq.jerk && !t->svel) throw Fail{GT_ERR_INVALID, "the jerk needs velocities (gt_tree_velocities)"};
    // a captured graph keeps its pointers: it runs on buffers its plan owns, not on the workspace
    WalkBuffers* wb = rq.bufs;
    auto own = [&](void** p, size_t& have, size_t need) {
        if (have >= need) return;
        if (rq.capture) throw Fail{GT_ERR_INVALID, "walk plan buffers changed size during capture"};
        if (*p) { check_cuda(cudaStreamSynchronize(st), "sync"); cudaFree(*p); *p = nullptr; have = 0; }
        check_cuda(cudaMalloc(p, need), "cudaMalloc walk plan buffer");
        have = need;
    };
    unsigned long long* ctr;
    if (wb) {
        own((void**)&wb->ctr, wb->ctr_bytes, 256);
        ctr = wb->ctr;
    } else {
        ctr = (unsigned long long*)scratch(ctx, kSlotCounters, 256);
    }
    a.next_group = (unsigned int*)(ctr + 8);
    a.stats = ctr;
    a.error = (int*)(ctr + 9);
    const bool want_pot = rq.want_phi && rq.phi;
    a.mac_model = rq.mac_model;
    a.nq2 = t->nq2;
    a.group_root = roots;
    a.mac_band_lo = rq.mac_band_lo;
    a.mac_band_hi = rq.mac_band_hi;
    a.mac_log_kappa = rq.mac_kappa > 0 ? std::log10(rq.mac_kappa) : -300.0;
    if ((mac || macn) && (!rq.mac_model || !rq.leaf_accept))
        throw Fail{GT_ERR_INVALID, "the learned criterion needs a model and a grouped walk"};
    a.mac_l2 = nullptr;
    if (macn) {
        // the per-node correction is part of the walk: computed on the stream before it (and
        // captured with it in a plan)
        float* l2;
        const size_t need = (size_t)std::max<int64_t>(t->n_nodes, 1) * sizeof(float);
        if (wb) {
            own((void**)&wb->mac_l2, wb->mac_l2_bytes, need);
            l2 = wb->mac_l2;
        } else {
            l2 = (float*)scratch(ctx, kSlotMacL2, need);
        }
        run_mac_node_scale(ctx, t, rq.mac_model, rq.mac_kappa > 0 ? rq.mac_kappa : 1.0, l2);
        a.mac_l2 = l2;
    }

    // Host outputs of a large walk: split the groups into chunks (kChunkEdge), and copy each chunk's
    // results to the host on a second stream while the next chunk runs.
    const bool chunked = rq.host.any() && !rq.count && rq.stack_capacity == 0 && !rq.capture &&
                         ng >= 64 * kChunks && nt >= (1 << 18);
    if (rq.host_aold && !chunked)
        check_cuda(cudaMemcpyAsync((void*)rq.aold, rq.host_aold, (size_t)nt * sizeof(double), cudaMemcpyHostToDevice, st),
                   "aold h2d");
    if (chunked) {
        ensure_copy_stream(ctx);
        int2* bounds = (int2*)(ctr + 16);  // K+1 int2 after the counters
        check_cuda(cudaMemsetAsync(ctr, 0, 256, st), "memset counters");
        chunk_bounds_kernel<<<1, 1, 0, st>>>(groups, (int)ng, (int)nt, kChunkEdge, bounds, ng_dev, paired ? 1 : 0);
        check_launch(ctx, "chunk_bounds_kernel");
        int2 hb[kChunks + 1];
        check_cuda(cudaMemcpyAsync(ctx->pinned, bounds, sizeof(hb), cudaMemcpyDeviceToHost, st), "d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(hb, ctx->pinned, sizeof(hb));
        const size_t stack_bytes = (size_t)total_warps * stack_cap * 4;
        if (wb) {
            own((void**)&wb->stack, wb->stack_bytes, stack_bytes);
            a.stack = wb->stack;
        } else {
            a.stack = (int*)scratch(ctx, kSlotStack, stack_bytes);
        }
        a.stack_cap = stack_cap;
        const OutputCopy outs[6] = {{rq.ax, rq.host.ax, 1},  {rq.ay, rq.host.ay, 1},       {rq.az, rq.host.az, 1},
                                    {rq.phi, rq.host.phi, 1}, {rq.tidal, rq.host.tidal, 6}, {rq.jerk, rq.host.jerk, 3}};
        // pageable host outputs (std::vector, numpy) are copied into the context's pinned staging
        // buffer and from there, chunk by chunk, into the caller's arrays while later chunks run:
        // a device-to-host copy into pageable memory would block this thread until its chunk is
        // done, and so hold back the launch of the next one
        size_t stage_off[6] = {0, 0, 0, 0, 0, 0};
        bool staged[6] = {false, false, false, false, false, false};
        size_t stage_need = 0;
        for (int i = 0; i < 6; ++i) {
            if (!outs[i].dev || !outs[i].host) continue;
            cudaPointerAttributes at;
            const bool pageable = cudaPointerGetAttributes(&at, outs[i].host) != cudaSuccess ||
                                  at.type == cudaMemoryTypeUnregistered;
            cudaGetLastError();
            if (!pageable) continue;
            staged[i] = true;
            stage_off[i] = stage_need;
            stage_need += (size_t)nt * outs[i].stride * sizeof(double);
        }
        char* stage = stage_need ? static_cast<char*>(host_stage(ctx, stage_need)) : nullptr;
        if (rq.host_aold) {
            // every chunk's aold ahead of the results on the copy stream, after the work queued
            // before this walk (which may still read the buffer); chunk c reads only the aold of
            // its own targets [hb[c].y, hb[c+1].y), so it waits for that piece alone
            check_cuda(cudaEventRecord(ctx->main_ev, st), "event");
            check_cuda(cudaStreamWaitEvent(ctx->copy_stream, ctx->main_ev, 0), "wait");
            for (int c = 0; c < kChunks; ++c) {
                const int64_t t0 = hb[c].y, t1 = hb[c + 1].y;
                if (t1 > t0)
                    check_cuda(cudaMemcpyAsync((void*)(rq.aold + t0), rq.host_aold + t0, (size_t)(t1 - t0) * sizeof(double),
                                               cudaMemcpyHostToDevice, ctx->copy_stream), "aold h2d chunk");
                check_cuda(cudaEventRecord(ctx->up_ev[c], ctx->copy_stream), "event");
            }
        }
        // The chunks alternate between the context stream and a second compute stream, so a chunk
        // fills the SMs that the previous one's last groups leave idle.  The warps of two chunks in
        // flight need their own traversal stacks; a plan's own buffers keep one stream.
        const bool two = wb == nullptr;
        cudaStream_t cs[2] = {st, two ? ctx->walk2 : st};
        int* stacks[2] = {a.stack, two ? (int*)scratch(ctx, kSlotStack2, stack_bytes) : a.stack};
        check_cuda(cudaEventRecord(ctx->ev0, st), "event");
        if (two) {
            check_cuda(cudaEventRecord(ctx->walk2_start, st), "event");
            check_cuda(cudaStreamWaitEvent(ctx->walk2, ctx->walk2_start, 0), "wait");
        }
        for (int c = 0; c < kChunks; ++c) {
            const int g0 = hb[c].x, g1 = hb[c + 1].x;
            cudaStream_t s = cs[c & 1];
            if (rq.host_aold) check_cuda(cudaStreamWaitEvent(s, ctx->up_ev[c], 0), "wait");
            if (g1 > g0) {
                // the dispatch launches on ctx->stream: point it at this chunk's stream meanwhile
                struct OnStream {
                    gt_context* c;
                    cudaStream_t old;
                    ~OnStream() { c->stream = old; }
                } on{ctx, ctx->stream};
                ctx->stream = s;
                WalkArgs ac = a;
                ac.stack = stacks[c & 1];
                ac.groups = groups + g0;
                ac.n_groups = g1 - g0;
                ac.n_groups_dev = nullptr;
                ac.group_root = roots ? roots + g0 : nullptr;
                ac.next_group = (unsigned int*)(ctr + 10) + c;
                const int64_t units = paired ? ((int64_t)(g1 - g0) + 1) / 2 : (int64_t)(g1 - g0);
                const int cb = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (units + warps - 1) / warps));
                if (paired) dispatch_pair(ctx, ac, cb, warps, want_pot, false, rq.mac);
                else if (xt) dispatch_xt(ctx, ac, cb, warps, ext, rq.leaf_accept, want_pot, false);
                else if (tpl == 1) dispatch<1>(ctx, ac, cb, warps, rq.leaf_accept, want_pot, false, rq.mac);
                else if (tpl == 2) dispatch<2>(ctx, ac, cb, warps, rq.leaf_accept, want_pot, false, rq.mac);
                else dispatch<4>(ctx, ac, cb, warps, rq.leaf_accept, want_pot, false, rq.mac);
            }
            // this chunk's targets [hb[c].y, hb[c+1].y) go back while the next chunk runs
            check_cuda(cudaEventRecord(ctx->chunk_ev[c], s), "event");
            check_cuda(cudaStreamWaitEvent(ctx->copy_stream, ctx->chunk_ev[c], 0), "wait");
            const int64_t t0 = hb[c].y, t1 = hb[c + 1].y;
            for (int i = 0; i < 6; ++i) {
                const OutputCopy& o = outs[i];
                if (!o.dev || !o.host || t1 <= t0) continue;
                double* dst = staged[i] ? reinterpret_cast<double*>(stage + stage_off[i]) + t0 * o.stride
                                        : o.host + t0 * o.stride;
                check_cuda(cudaMemcpyAsync(dst, o.dev + t0 * o.stride, (size_t)(t1 - t0) * o.stride * sizeof(double),
                                           cudaMemcpyDeviceToHost, ctx->copy_stream), "d2h chunk");
            }
            check_cuda(cudaEventRecord(ctx->down_ev[c], ctx->copy_stream), "event");
        }
        if (stage) {
            // every chunk is queued: move each one's results into the caller's arrays as they land
            for (int c = 0; c < kChunks; ++c) {
                const int64_t t0 = hb[c].y, t1 = hb[c + 1].y;
                if (t1 <= t0) continue;
                check_cuda(cudaEventSynchronize(ctx->down_ev[c]), "sync");
                for (int i = 0; i < 6; ++i)
                    if (staged[i])
                        std::memcpy(outs[i].host + t0 * outs[i].stride,
                                    reinterpret_cast<const double*>(stage + stage_off[i]) + t0 * outs[i].stride,
                                    (size_t)(t1 - t0) * outs[i].stride * sizeof(double));
            }
        }
        if (two) {
            check_cuda(cudaEventRecord(ctx->walk2_done, ctx->walk2), "event");
            check_cuda(cudaStreamWaitEvent(st, ctx->walk2_done, 0), "wait");
        }
        check_cuda(cudaEventRecord(ctx->ev1, st), "event");
        check_cuda(cudaEventRecord(ctx->copy_done, ctx->copy_stream), "event");
        check_cuda(cudaStreamWaitEvent(st, ctx->copy_done, 0), "wait");
        return true;
    }

    for (int attempt = 0; attempt < 3; ++attempt) {
        const size_t stack_bytes = (size_t)total_warps * stack_cap * 4;
        if (wb) {
            own((void**)&wb->stack, wb->stack_bytes, stack_bytes);
            a.stack = wb->stack;
        } else {
            a.stack = (int*)scratch(ctx, kSlotStack, stack_bytes);
        }
        a.stack_cap = stack_cap;
        check_cuda(cudaMemsetAsync(ctr, 0, 96, st), "memset counters");
        if (!rq.capture) check_cuda(cudaEventRecord(ctx->ev0, st), "event");
        if (paired) dispatch_pair(ctx, a, blocks, warps, want_pot, rq.count, rq.mac);
        else if (xt) dispatch_xt(ctx, a, blocks, warps, ext, rq.leaf_accept, want_pot, rq.count);
        else if (tpl == 1) dispatch<1>(ctx, a, blocks, warps, rq.leaf_accept, want_pot, rq.count, rq.mac);
        else if (tpl == 2) dispatch<2>(ctx, a, blocks, warps, rq.leaf_accept, want_pot, rq.count, rq.mac);
        else dispatch<4>(ctx, a, blocks, warps, rq.leaf_accept, want_pot, rq.count, rq.mac);
        if (rq.capture) break;  // the default stack capacity is a proven bound
        check_cuda(cudaEventRecord(ctx->ev1, st), "event");
#ifndef GT_BOUNDS_CHECK
        if (!rq.count && attempt == 0 && rq.stack_capacity == 0) {
            // the default capacity is a proven bound: no read-back needed on the fast path
            break;
        }
#endif
        check_cuda(cudaMemcpyAsync(ctx->pinned, ctr, 80, cudaMemcpyDeviceToHost, st), "stats d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        unsigned long long h[10];
        std::memcpy(h, ctx->pinned, 80);
        if ((int)h[9] == 3) throw Fail{GT_ERR_INVALID, "walk: an index failed its bounds check"};
        if ((int)h[9] == 0) {
            if (ng_dev) {
                uint32_t hg = 0;
                check_cuda(cudaMemcpy(&hg, ng_dev, 4, cudaMemcpyDeviceToHost), "group count d2h");
                ctx->stats.groups = hg;
            }
            ctx->stats.nodes_visited = (int64_t)h[0];
            ctx->stats.multipole = (int64_t)h[1];
            ctx->stats.pairs = (int64_t)h[2] - (int64_t)h[3];
            ctx->stats.list_flushes = (int64_t)h[4];
            ctx->stats.max_stack = (int64_t)h[5];
            ctx->stats.traversal_steps = (int64_t)h[6];
            break;
        }
        if (attempt == 2) throw Fail{GT_ERR_OVERFLOW, "walk stack overflow"};
        stack_cap *= 2;
    }
    return false;
}

}  // namespace gt
