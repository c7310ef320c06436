// Tree build on the device: the replacement for shmem::build (shmem/tree.cc:350-526).
//
// Stages (each a handful of kernels on the context stream):
//   1. bbox       grid-stride min/max over live particles, one block finishes the root cell
//                 exactly as tree.cc:361-417 does (centre, side*1.0000001, optional randomised or
//                 shifted root, 20-bit scale).
//   2. keys       20-bit-per-axis quantisation of tree.cc:409-417, then a Peano-Hilbert key
//                 (system/peano.cc:297-313 state machine) or the shmem Morton key (tree.h:161-173).
//                 Massless particles get a key above every live key and sort last.
//   3. sort       stable LSD radix sort of (key, particle index) (gt_scan.cu).
//   4. gather     particles into tree order: 32-byte SrcP records (FP64 position, FP32 mass and
//                 softening) plus FP64 mass/softening for the moments and the opening test.
//   5. structure  level-synchronous split: one thread per node binary-searches its key range for
//                 the 8 digit boundaries of the next level (a leaf at <= leaf_max particles or at
//                 max_level, tree.cc:89); a scan over child counts places every node's children
//                 contiguously in the next level (BFS order).  Child centres are parent +-
//                 side/4 by the child's octant bits, as tree.cc:116-118.
//   6. moments    deepest level first, eight lanes per node: a leaf reduces its particles, an
//                 interior node its children, with shuffles (mass, mass-weighted position,
//                 max softening), then COM, delta = |COM - centre| and the packed walk node
//                 (tree.cc:145-196, 507-523).
// The next/first threading of the reference (tree.cc:340-348) is produced alongside for the host
// download; the GPU walk itself only uses the contiguous child ranges.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "gt_internal.cuh"
#include "gt_ph_table.cuh"

namespace gt {
namespace {

constexpr int kBlk = 256;

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---- 1. bbox ---------------------------------------------------------------------------------
__global__ void bbox_partial_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                    const double* __restrict__ z, const double* __restrict__ m,
                                    const double* __restrict__ soft, int64_t n,
                                    double* __restrict__ part, unsigned long long* __restrict__ cnt) {
    double lo0 = 1e300, lo1 = 1e300, lo2 = 1e300, hi0 = -1e300, hi1 = -1e300, hi2 = -1e300;
    unsigned long long live = 0, bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double xi = x[i], yi = y[i], zi = z[i], mi = m[i];
        const double si = soft ? soft[i] : 0.0;
        if (!isfinite(xi) || !isfinite(yi) || !isfinite(zi) || !isfinite(mi) || !isfinite(si)) ++bad;
        if (!(mi > 0)) continue;
        ++live;
        lo0 = fmin(lo0, xi); hi0 = fmax(hi0, xi);
        lo1 = fmin(lo1, yi); hi1 = fmax(hi1, yi);
        lo2 = fmin(lo2, zi); hi2 = fmax(hi2, zi);
    }
    lo0 = warp_min_d(lo0); lo1 = warp_min_d(lo1); lo2 = warp_min_d(lo2);
    hi0 = warp_max_d(hi0); hi1 = warp_max_d(hi1); hi2 = warp_max_d(hi2);
    __shared__ double sh[8][6];
    __shared__ unsigned long long sc[8][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        live += __shfl_xor_sync(0xffffffffu, live, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        sh[w][0] = lo0; sh[w][1] = lo1; sh[w][2] = lo2; sh[w][3] = hi0; sh[w][4] = hi1; sh[w][5] = hi2;
        sc[w][0] = live; sc[w][1] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            for (int c = 0; c < 3; ++c) sh[0][c] = fmin(sh[0][c], sh[k][c]);
            for (int c = 3; c < 6; ++c) sh[0][c] = fmax(sh[0][c], sh[k][c]);
            sc[0][0] += sc[k][0]; sc[0][1] += sc[k][1];
        }
        for (int c = 0; c < 6; ++c) part[blockIdx.x * 6 + c] = sh[0][c];
        cnt[blockIdx.x * 2 + 0] = sc[0][0];
        cnt[blockIdx.x * 2 + 1] = sc[0][1];
    }
}

// Root cell from the live bounding box, tree.cc:361-417.  A handful of flops, one thread.
__device__ void finish_root(const double* lo, const double* hi, unsigned long long live, RootGeom* __restrict__ g,
                            long long seed, double fx, double fy, double fz, int max_level) {
    double cx = 0.5 * (lo[0] + hi[0]), cy = 0.5 * (lo[1] + hi[1]), cz = 0.5 * (lo[2] + hi[2]);
    double side = fmax(hi[0] - lo[0], fmax(hi[1] - lo[1], hi[2] - lo[2])) * 1.0000001;
    if (side <= 0) side = 1.0;
    if (seed >= 0) {  // RANDOMIZE_GRAVTREE, splitmix64 draws of tree.cc:381-393
        uint64_t s = (uint64_t)seed * 0x9E3779B97F4A7C15ull;
        double d[3];
        for (int k = 0; k < 3; ++k) {
            s += 0x9E3779B97F4A7C15ull;
            uint64_t v = s;
            v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
            v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
            d[k] = (double)((v ^ (v >> 31)) >> 11) * (1.0 / 9007199254740992.0);
        }
        // the reference's compiler fuses these into FMAs (checked on its x86 build); so do we
        cx = fma(side, d[0] - 0.5, cx);
        cy = fma(side, d[1] - 0.5, cy);
        cz = fma(side, d[2] - 0.5, cz);
        side *= 2.0;
    }
    if (fx != 0.0 || fy != 0.0 || fz != 0.0) {  // SHMEM_TREE_SHIFT, tree.cc:400-407
        cx = fma(fx, side, cx); cy = fma(fy, side, cy); cz = fma(fz, side, cz);
        side *= 1.0 + 2.0 * (fabs(fx) + fabs(fy) + fabs(fz));
    }
    g->cx = cx; g->cy = cy; g->cz = cz; g->side = side;
    g->scale = (double)((1u << max_level) - 1) / side;
    g->corner_x = fma(-0.5, side, cx);  // 0.5*side is exact: fused or not, the same bits
    g->corner_y = fma(-0.5, side, cy);
    g->corner_z = fma(-0.5, side, cz);
    g->n_live = (long long)live;
}

// One block combines the partial boxes and counts (minimum, maximum and integer sums are exact in
// any order, so the root cell does not depend on the block shape), then thread 0 finishes the root.
constexpr int kRootThreads = 256;
__global__ void __launch_bounds__(kRootThreads)
root_geom_kernel(const double* __restrict__ part, const unsigned long long* __restrict__ cnt,
                 int nb, RootGeom* __restrict__ g, unsigned long long* __restrict__ bad_out,
                 long long seed, double fx, double fy, double fz, int max_level) {
    __shared__ double sh[6][kRootThreads];
    __shared__ unsigned long long sc[2][kRootThreads];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    unsigned long long live = 0, bad = 0;
    for (int b = threadIdx.x; b < nb; b += kRootThreads) {
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], part[b * 6 + c]);
            hi[c] = fmax(hi[c], part[b * 6 + 3 + c]);
        }
        live += cnt[b * 2];
        bad += cnt[b * 2 + 1];
    }
    for (int c = 0; c < 3; ++c) { sh[c][threadIdx.x] = lo[c]; sh[3 + c][threadIdx.x] = hi[c]; }
    sc[0][threadIdx.x] = live;
    sc[1][threadIdx.x] = bad;
    __syncthreads();
    for (int o = kRootThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            for (int c = 0; c < 3; ++c) {
                sh[c][threadIdx.x] = fmin(sh[c][threadIdx.x], sh[c][threadIdx.x + o]);
                sh[3 + c][threadIdx.x] = fmax(sh[3 + c][threadIdx.x], sh[3 + c][threadIdx.x + o]);
            }
            sc[0][threadIdx.x] += sc[0][threadIdx.x + o];
            sc[1][threadIdx.x] += sc[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int c = 0; c < 3; ++c) { lo[c] = sh[c][0]; hi[c] = sh[3 + c][0]; }
        finish_root(lo, hi, sc[0][0], g, seed, fx, fy, fz, max_level);
        *bad_out = sc[1][0];
    }
}

// Forest: `chunks` blocks per system each reduce a slice of that system's input range into a
// partial box (6 doubles) and counts (live, non-finite); root_systems_kernel combines them.
__global__ void bbox_systems_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                    const double* __restrict__ z, const double* __restrict__ m,
                                    const double* __restrict__ soft, const int64_t* __restrict__ off,
                                    int chunks, double* __restrict__ part, unsigned long long* __restrict__ cnt) {
    const int s = blockIdx.x / chunks, c0 = blockIdx.x % chunks;
    const int64_t a = off[s], len = off[s + 1] - off[s];
    const int64_t lo_i = a + len * c0 / chunks, hi_i = a + len * (c0 + 1) / chunks;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    unsigned long long live = 0, bad = 0;
    for (int64_t i = lo_i + threadIdx.x; i < hi_i; i += blockDim.x) {
        const double xi = x[i], yi = y[i], zi = z[i], mi = m[i];
        const double si = soft ? soft[i] : 0.0;
        if (!isfinite(xi) || !isfinite(yi) || !isfinite(zi) || !isfinite(mi) || !isfinite(si)) ++bad;
        if (!(mi > 0)) continue;
        ++live;
        lo[0] = fmin(lo[0], xi); hi[0] = fmax(hi[0], xi);
        lo[1] = fmin(lo[1], yi); hi[1] = fmax(hi[1], yi);
        lo[2] = fmin(lo[2], zi); hi[2] = fmax(hi[2], zi);
    }
    for (int c = 0; c < 3; ++c) { lo[c] = warp_min_d(lo[c]); hi[c] = warp_max_d(hi[c]); }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        live += __shfl_xor_sync(0xffffffffu, live, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    __shared__ double sh[8][6];
    __shared__ unsigned long long sc[8][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        for (int c = 0; c < 3; ++c) { sh[w][c] = lo[c]; sh[w][3 + c] = hi[c]; }
        sc[w][0] = live; sc[w][1] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            for (int c = 0; c < 3; ++c) {
                lo[c] = fmin(lo[c], sh[k][c]);
                hi[c] = fmax(hi[c], sh[k][3 + c]);
            }
            live += sc[k][0]; bad += sc[k][1];
        }
        for (int c = 0; c < 3; ++c) { part[6 * blockIdx.x + c] = lo[c]; part[6 * blockIdx.x + 3 + c] = hi[c]; }
        cnt[2 * blockIdx.x] = live;
        cnt[2 * blockIdx.x + 1] = bad;
    }
}

// One thread per system: combine its chunks and finish its root cell; the non-finite counts add
// up into bad_out.
__global__ void root_systems_kernel(const double* __restrict__ part, const unsigned long long* __restrict__ cnt,
                                    int n_systems, int chunks, RootGeom* __restrict__ geoms,
                                    unsigned long long* __restrict__ bad_out, long long seed, double fx, double fy,
                                    double fz, int max_level) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_systems) return;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    unsigned long long live = 0, bad = 0;
    for (int k = s * chunks; k < (s + 1) * chunks; ++k) {
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], part[6 * k + c]);
            hi[c] = fmax(hi[c], part[6 * k + 3 + c]);
        }
        live += cnt[2 * k];
        bad += cnt[2 * k + 1];
    }
    finish_root(lo, hi, live, geoms + s, seed, fx, fy, fz, max_level);
    if (bad) atomicAdd(bad_out, bad);
}

// ---- 2. keys ---------------------------------------------------------------------------------
__device__ __forceinline__ void quantise(const RootGeom& g, double x, double y, double z,
                                         uint32_t& a, uint32_t& b, uint32_t& c) {
    a = (uint32_t)((x - g.corner_x) * g.scale);
    b = (uint32_t)((y - g.corner_y) * g.scale);
    c = (uint32_t)((z - g.corner_z) * g.scale);
}

__device__ __forceinline__ uint64_t spread3_21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | v << 32) & 0x1F00000000FFFFull;
    v = (v | v << 16) & 0x1F0000FF0000FFull;
    v = (v | v << 8) & 0x100F00F00F00F00Full;
    v = (v | v << 4) & 0x10C30C30C30C30C3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__global__ void keys_kernel(const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ m, int64_t n,
                            const RootGeom* __restrict__ gp, int key_mode, int levels,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ idx,
                            const int64_t* __restrict__ sys_in, int n_systems, uint64_t* __restrict__ sys_key,
                            double2* __restrict__ pk) {
    __shared__ uint16_t tab[48 * 8];
    for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x) tab[k] = kPhStep[k];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        idx[i] = (uint32_t)i;
        // x, y, z, m packed in one 32-byte sector per particle: the gather into tree order then
        // reads one sector per particle through the permutation instead of four
        pk[2 * i] = make_double2(x[i], y[i]);
        pk[2 * i + 1] = make_double2(z[i], m[i]);
        // forest: the particle's own system's root cell; the second sort key is the system
        // (massless particles of every system go last)
        const int s = n_systems > 1 ? system_of(sys_in, n_systems, i) : 0;
        const bool live = m[i] > 0;
        if (n_systems > 1) sys_key[i] = live ? (uint64_t)s : (uint64_t)n_systems;
        if (!live) { keys[i] = kDeadKey; continue; }
        const RootGeom& g = gp[s];
        uint32_t a, b, c;
        quantise(g, x[i], y[i], z[i], a, b, c);
        uint64_t key;
        if (key_mode == GT_KEY_MORTON) {
            key = spread3_21(a) | (spread3_21(b) << 1) | (spread3_21(c) << 2);
        } else {
            key = 0;
            unsigned state = 0;
            for (int l = levels - 1; l >= 0; --l) {
                const unsigned pix = ((a >> l) & 1u) << 2 | ((b >> l) & 1u) << 1 | ((c >> l) & 1u);
                const unsigned step = tab[state * 8 + pix];
                key = (key << 3) | (step & 7u);
                state = step >> 3;
            }
        }
        keys[i] = key;
    }
}

// ---- 4. gather into tree order ---------------------------------------------------------------
// Tree order: x, y, z, m from the packed copy the keys pass wrote (pk), the softening from its own
// array.  leaf_of is preset to -1 by a memset (the moments pass sets the live particles' leaves).
__global__ void gather_kernel(const double2* __restrict__ pk, const double* __restrict__ soft,
                              const uint32_t* __restrict__ idx, int64_t n, SrcP* __restrict__ src,
                              double* __restrict__ ssoft, double* __restrict__ smass, uint32_t* __restrict__ order,
                              uint32_t* __restrict__ rank, int* __restrict__ sleaf,
                              unsigned long long* __restrict__ bad_soft) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = idx[i];
        const double2 a = __ldg(pk + 2 * (int64_t)p), b = __ldg(pk + 2 * (int64_t)p + 1);
        SrcP r;
        r.x = a.x; r.y = a.y; r.z = b.x;
        const double sp = soft ? soft[p] : 0.0;
        // softenings that arrived after the bounding-box pass are checked here
        if (bad_soft && !isfinite(sp)) atomicAdd(bad_soft, 1ull);
        r.m = (float)b.y;
        r.soft = (float)sp;
        src[i] = r;
        ssoft[i] = sp;
        smass[i] = b.y;
        order[i] = p;
        rank[p] = (uint32_t)i;
        sleaf[i] = -1;
    }
}

// ---- 5. structure ----------------------------------------------------------------------------
__device__ __forceinline__ int lower_bound_digit(const uint64_t* __restrict__ key, int lo, int hi,
                                                 int shift, unsigned v) {
    // first index in [lo, hi) whose digit is >= v (digits are non-decreasing over the range)
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if ((unsigned)((key[mid] >> shift) & 7ull) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// The level array of the structure stage on the device: level starts lv[L], level counts
// lv[kLvCount + L], and the overflow flag lv[2 * kLvCount].
constexpr int kLvCount = 32;

// Deepest level at which the build splits a cell, from the sorted keys alone: particles i and
// i + leaf_max share their top d digits exactly when they share a level-d cell, which then holds
// more than leaf_max particles and splits (below max_level).  So the deepest split level is the
// largest such d over i, capped at max_level - 1; -1 when nothing splits.  A forest's keys are
// compared across system boundaries too, which can only deepen the estimate (the extra levels are
// then empty).
__global__ void split_depth_kernel(const uint64_t* __restrict__ skey, int64_t n_live, int leaf_max,
                                   int max_level, int* __restrict__ depth) {
    int d = -1;
    const int pad = 64 - 3 * max_level;  // key bits above the 3 * max_level used ones
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i + leaf_max < n_live;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t x = skey[i] ^ skey[i + leaf_max];
        const int common = x == 0 ? max_level : (__clzll((long long)x) - pad) / 3;
        d = max(d, min(common, max_level - 1));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0 && d >= 0) atomicMax(depth, d);
}

// Child boundaries of a level's nodes, eight lanes per node: lane v finds where digit v starts in
// the node's sorted keys (one binary search each, in parallel, where a single thread would run
// seven in sequence), the eight lanes count the non-empty octants.  bnd holds nine boundaries per
// node (the octant ranges [B[v], B[v+1])), nchild the count (0 for a node that stays a leaf).  The
// level's range comes from lv when given (device-side levels), else from [a, b).
__global__ void split_kernel(const GNode* __restrict__ nodes, const uint64_t* __restrict__ skey,
                             int64_t a, int64_t b, int level, int max_level, int leaf_max,
                             int* __restrict__ bnd, uint32_t* __restrict__ nchild,
                             const int64_t* __restrict__ lv = nullptr) {
    if (lv) { a = lv[level]; b = a + lv[kLvCount + level]; }
    const int lane = threadIdx.x & 31, sub = lane & 7;
    const int64_t cnt = b - a;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4; base < cnt;
         base += warps * 4) {
        const int64_t t = base + (lane >> 3);
        const bool live = t < cnt;
        int lo = 0, hi = 0;
        if (live) { lo = nodes[a + t].plo; hi = nodes[a + t].phi; }
        const bool split = live && !(hi - lo <= leaf_max || level >= max_level);
        int bv = lo;
        if (split && sub > 0) bv = lower_bound_digit(skey, lo, hi, 3 * (max_level - level - 1), (unsigned)sub);
        int nx = __shfl_down_sync(0xffffffffu, bv, 1, 8);
        if (sub == 7) nx = hi;
        int c = (split && nx > bv) ? 1 : 0;
        c += __shfl_xor_sync(0xffffffffu, c, 1, 8);
        c += __shfl_xor_sync(0xffffffffu, c, 2, 8);
        c += __shfl_xor_sync(0xffffffffu, c, 4, 8);
        if (split) {
            int* B = bnd + t * 9;
            B[sub] = bv;
            if (sub == 7) B[8] = hi;
        }
        if (live && sub == 0) nchild[t] = (uint32_t)c;
    }
}

// After the scan of level L's child counts: level L+1 starts where L ends and holds `total` nodes,
// unless that overruns the node arrays; then the overflow flag is set, nothing more is emitted and
// the host redoes the stage one level at a time, growing the arrays.
__global__ void advance_level_kernel(int64_t* __restrict__ lv, int level, const uint32_t* __restrict__ total,
                                     int64_t node_cap) {
    int64_t* cnt = lv + kLvCount;
    int64_t* ovf = lv + 2 * kLvCount;
    const int64_t b = lv[level] + cnt[level];
    int64_t tot = *ovf ? 0 : (int64_t)*total;
    if (b + tot > node_cap) { *ovf = 1; tot = 0; }
    lv[level + 1] = b;
    cnt[level + 1] = tot;
}

__global__ void init_levels_kernel(int64_t* __restrict__ lv, int64_t n_roots) {
    for (int i = 0; i <= 2 * kLvCount; ++i) lv[i] = 0;
    lv[kLvCount] = n_roots;  // level 0: the roots [0, n_roots)
}

__global__ void emit_kernel(GNode* __restrict__ nodes, const SrcP* __restrict__ src,
                            const RootGeom* __restrict__ gp, int64_t a, int64_t b, int level,
                            int max_level, const int* __restrict__ bnd,
                            const uint32_t* __restrict__ nchild, const uint32_t* __restrict__ coff,
                            int* __restrict__ parent, int* __restrict__ next, int* __restrict__ lvl,
                            double* __restrict__ size, double* __restrict__ gc,
                            const int* __restrict__ sys_off, int n_systems,
                            const int64_t* __restrict__ lv = nullptr) {
    if (lv) {
        if (lv[2 * kLvCount] != 0) return;  // the node arrays overflowed: the host redoes the stage
        a = lv[level];
        b = a + lv[kLvCount + level];
    }
    const int bit = max_level - 1 - level;  // coordinate bit that selects the octant at this level
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < b - a;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = a + t;
        const int nc = (int)nchild[t];
        if (nc == 0) {
            nodes[i].first = -1;
            nodes[i].nchild = 0;
            continue;
        }
        const RootGeom g = gp[n_systems > 1 ? system_of(sys_off, n_systems, nodes[i].plo) : 0];
        const int first = (int)(b + coff[t]);
        nodes[i].first = first;
        nodes[i].nchild = nc;
        const int* B = bnd + t * 9;
        const double sz = size[i], half = sz * 0.5, quarter = sz * 0.25;
        const double pcx = gc[3 * i], pcy = gc[3 * i + 1], pcz = gc[3 * i + 2];
        const int pnext = next[i];
        int k = 0;
        for (int v = 0; v < 8; ++v) {
            if (B[v + 1] <= B[v]) continue;
            const int c = first + k;
            const SrcP& s0 = src[B[v]];
            uint32_t qa, qb, qc;
            quantise(g, s0.x, s0.y, s0.z, qa, qb, qc);
            const int oct = (int)((qa >> bit) & 1u) | (int)(((qb >> bit) & 1u) << 1) | (int)(((qc >> bit) & 1u) << 2);
            GNode& ch = nodes[c];
            ch.plo = B[v];
            ch.phi = B[v + 1];
            ch.first = -1;
            ch.nchild = 0;
            parent[c] = (int)i;
            lvl[c] = level + 1;
            size[c] = half;
            gc[3 * c] = pcx + ((oct & 1) ? quarter : -quarter);
            gc[3 * c + 1] = pcy + ((oct & 2) ? quarter : -quarter);
            gc[3 * c + 2] = pcz + ((oct & 4) ? quarter : -quarter);
            next[c] = (k + 1 < nc) ? c + 1 : pnext;
            ++k;
        }
    }
}

// ---- 6. moments, eight lanes per node, deepest level first ------------------------------------
// An interior node has at most 8 children and a leaf usually at most leaf_max (16) particles, so
// a node gets 8 lanes of a warp (4 nodes per warp) and 3-level shuffle reductions.
constexpr int kMomLanes = 8;
constexpr int kMomNodesPerBlock = kBlk / kMomLanes;

__device__ __forceinline__ double group_sum_d(double v) {
#pragma unroll
    for (int o = kMomLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double group_max_d(double v) {
#pragma unroll
    for (int o = kMomLanes / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void moments_kernel(GNode* __restrict__ nodes, const SrcP* __restrict__ src,
                               const double* __restrict__ smass, const double* __restrict__ ssoft,
                               const uint32_t* __restrict__ order, int64_t a, int64_t b,
                               const double* __restrict__ size, const double* __restrict__ gc,
                               double* __restrict__ delta, double* __restrict__ nsoft,
                               float* __restrict__ nq2, int* __restrict__ leaf_of,
                               int* __restrict__ sleaf, int nodelta) {
    const int sub = threadIdx.x & (kMomLanes - 1);
    const int64_t i = a + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kMomLanes;
    // every lane takes part in the group shuffles; lanes past the level's last node add nothing
    const bool valid = i < b;
    int first = 0, nc = 0, lo = 0, hi = 0;
    if (valid) {
        first = nodes[i].first; nc = nodes[i].nchild;
        lo = nodes[i].plo; hi = nodes[i].phi;
    }
    const bool leaf = valid && first < 0;
    double M = 0, mx = 0, my = 0, mz = 0, smax = 0;
    if (leaf) {
        for (int j = lo + sub; j < hi; j += kMomLanes) {
            const double mj = smass[j];
            const SrcP s = src[j];
            M += mj; mx += mj * s.x; my += mj * s.y; mz += mj * s.z;
            smax = fmax(smax, ssoft[j]);
            leaf_of[order[j]] = (int)i;
            sleaf[j] = (int)i;
        }
    } else if (valid && sub < nc) {
        const GNode& ch = nodes[first + sub];
        M = ch.mass; mx = M * ch.cx; my = M * ch.cy; mz = M * ch.cz;
        smax = nsoft[first + sub];
    }
    M = group_sum_d(M); mx = group_sum_d(mx); my = group_sum_d(my); mz = group_sum_d(mz);
    smax = group_max_d(smax);
    // Second mass moment about the COM, sum m |x - com|^2: from the particles in a leaf, from the
    // children by the parallel-axis rule otherwise.  Not used by the plain criterion; it is an input
    // of the learned one (the quadrupole error a monopole makes scales with it).
    {
        const double ox = M > 0 ? mx / M : 0.0, oy = M > 0 ? my / M : 0.0, oz = M > 0 ? mz / M : 0.0;
        double q = 0;
        if (leaf) {
            for (int j = lo + sub; j < hi; j += kMomLanes) {
                const SrcP s = src[j];
                const double ex = s.x - ox, ey = s.y - oy, ez = s.z - oz;
                q += smass[j] * (ex * ex + ey * ey + ez * ez);
            }
        } else if (valid && sub < nc) {
            const GNode& ch = nodes[first + sub];
            const double ex = ch.cx - ox, ey = ch.cy - oy, ez = ch.cz - oz;
            q = (double)nq2[first + sub] + ch.mass * (ex * ex + ey * ey + ez * ez);
        }
        q = group_sum_d(q);
        if (valid && sub == 0) nq2[i] = (float)q;
    }
    if (valid && sub == 0) {
        if (M > 0) { mx /= M; my /= M; mz /= M; }
        const double dx = mx - gc[3 * i], dy = my - gc[3 * i + 1], dz = mz - gc[3 * i + 2];
        const double dl = sqrt(dx * dx + dy * dy + dz * dz);
        GNode& nd = nodes[i];
        nd.cx = mx; nd.cy = my; nd.cz = mz; nd.mass = M;
        nd.s = size[i] + (nodelta ? 0.0 : dl);
        nd.len = (float)size[i];
        nd.soft = (float)smax;
        delta[i] = dl;
        nsoft[i] = smax;
    }
}

// Roots: node s is system s's root, covering its live tree positions [sys_off[s], sys_off[s+1]).
// Each root stands alone in the reference threading (next = -1).
__global__ void root_init_kernel(GNode* __restrict__ nodes, const RootGeom* __restrict__ gp,
                                 const int* __restrict__ sys_off, int n_systems,
                                 int* parent, int* next, int* lvl, double* size, double* gc) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_systems; s += gridDim.x * blockDim.x) {
        const RootGeom& g = gp[s];
        GNode& r = nodes[s];
        r.plo = sys_off[s];
        r.phi = sys_off[s + 1];
        r.first = -1;
        r.nchild = 0;
        parent[s] = -1;
        next[s] = -1;
        lvl[s] = 0;
        size[s] = g.side;
        gc[3 * s] = g.cx; gc[3 * s + 1] = g.cy; gc[3 * s + 2] = g.cz;
    }
}

// Second key of the forest sort: system of each key-sorted particle.
__global__ void gather_sys_key_kernel(const uint64_t* __restrict__ sys_key, const uint32_t* __restrict__ idx,
                                      int64_t n, uint64_t* __restrict__ out, uint32_t* __restrict__ pos) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        out[i] = sys_key[idx[i]];
        pos[i] = (uint32_t)i;
    }
}

__global__ void permute_pairs_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ val,
                                     const uint32_t* __restrict__ pos, int64_t n, uint64_t* __restrict__ key_out,
                                     uint32_t* __restrict__ val_out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pos[i];
        key_out[i] = key[p];
        val_out[i] = val[p];
    }
}

// ---- MPI-code keys (domain.cc:2682-2702, peano.cc:297-355) -------------------------------------
__device__ __forceinline__ uint64_t mantissa_bits(double d, int bits) {
    const uint64_t u = (uint64_t)__double_as_longlong(d);
    return (u & 0xFFFFFFFFFFFFFull) >> (52 - bits);
}

__global__ void peano_keys_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                  const double* __restrict__ z, int64_t n, double c0, double c1,
                                  double c2, double len, int bits, uint64_t* ph_hi, uint64_t* ph_lo,
                                  uint64_t* mo_hi, uint64_t* mo_lo) {
    __shared__ uint16_t tab[48 * 8];
    for (int k = threadIdx.x; k < 48 * 8; k += blockDim.x) tab[k] = kPhStep[k];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t xb = mantissa_bits((x[i] - c0) / len + 1.0, bits);
        const uint64_t yb = mantissa_bits((y[i] - c1) / len + 1.0, bits);
        const uint64_t zb = mantissa_bits((z[i] - c2) / len + 1.0, bits);
        uint64_t hh = 0, hl = 0, mh = 0, ml = 0;
        unsigned state = 0;
        for (int l = bits - 1; l >= 0; --l) {
            const unsigned bx = (unsigned)((xb >> l) & 1u), by = (unsigned)((yb >> l) & 1u),
                           bz = (unsigned)((zb >> l) & 1u);
            const unsigned step = tab[state * 8 + (bx << 2 | by << 1 | bz)];
            state = step >> 3;
            hh = (hh << 3) | (hl >> 61);
            hl = (hl << 3) | (step & 7u);
            mh = (mh << 3) | (ml >> 61);
            ml = (ml << 3) | (bz << 2 | by << 1 | bx);
        }
        if (ph_hi) ph_hi[i] = hh;
        if (ph_lo) ph_lo[i] = hl;
        if (mo_hi) mo_hi[i] = mh;
        if (mo_lo) mo_lo[i] = ml;
    }
}

// ---- velocities: particle velocities in tree order, node centre-of-mass velocity and speed bound
// (tree.cc:149-190: leaves from their particles, interior nodes from their children) -------------
__global__ void gather_vel_kernel(const double* __restrict__ vx, const double* __restrict__ vy,
                                  const double* __restrict__ vz, const uint32_t* __restrict__ order,
                                  int64_t n_live, float4* __restrict__ svel) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_live;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = order[i];
        svel[i] = make_float4((float)vx[p], (float)vy[p], (float)vz[p], 0.0f);
    }
}

// ---- gas and sinks: particle types and adaptive-softening zeta in tree order, sinks per node ----
// (shmem::Particles::type / ::zeta, tree.h:38-49; the per-node sink count of tree.cc:155-187)
__global__ void gather_gas_kernel(const uint8_t* __restrict__ type, const double* __restrict__ zeta,
                                  const uint32_t* __restrict__ order, int64_t n, uint8_t* __restrict__ stype,
                                  double* __restrict__ szeta) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = order[i];
        stype[i] = type ? type[p] : (uint8_t)0;
        szeta[i] = zeta ? zeta[p] : 0.0;
    }
}

// Each live sink adds one to its leaf and every ancestor.  Integer atomics: the counts do not
// depend on the order of the additions.
__global__ void count_sinks_kernel(const uint8_t* __restrict__ stype, const int* __restrict__ sleaf,
                                   const int* __restrict__ parent, int64_t n_live, uint32_t* __restrict__ nsink) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_live;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (stype[i] != 5) continue;
        for (int no = sleaf[i]; no >= 0; no = parent[no]) atomicAdd(nsink + no, 1u);
    }
}

__global__ void vel_moments_kernel(const GNode* __restrict__ nodes, const double* __restrict__ smass,
                                   const uint32_t* __restrict__ order, const double* __restrict__ vx,
                                   const double* __restrict__ vy, const double* __restrict__ vz, int64_t a,
                                   int64_t b, double* __restrict__ vcom, float4* __restrict__ nvel,
                                   float* __restrict__ vmax) {
    const int sub = threadIdx.x & (kMomLanes - 1);
    const int64_t i = a + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kMomLanes;
    const bool valid = i < b;  // all lanes take part in the group shuffles
    GNode nd{};
    if (valid) nd = nodes[i];
    double px = 0, py = 0, pz = 0, vm = 0;
    if (valid && nd.first < 0) {
        for (int j = nd.plo + sub; j < nd.phi; j += kMomLanes) {
            const uint32_t p = order[j];
            const double m = smass[j], ux = vx[p], uy = vy[p], uz = vz[p];
            px += m * ux; py += m * uy; pz += m * uz;
            vm = fmax(vm, sqrt(ux * ux + uy * uy + uz * uz));
        }
    } else if (valid && sub < nd.nchild) {
        const int c = nd.first + sub;
        const double m = nodes[c].mass;
        px = m * vcom[3 * c]; py = m * vcom[3 * c + 1]; pz = m * vcom[3 * c + 2];
        vm = (double)vmax[c];
    }
    px = group_sum_d(px); py = group_sum_d(py); pz = group_sum_d(pz);
    vm = group_max_d(vm);
    if (valid && sub == 0) {
        const double M = nd.mass;
        const double ux = M > 0 ? px / M : 0.0, uy = M > 0 ? py / M : 0.0, uz = M > 0 ? pz / M : 0.0;
        vcom[3 * i] = ux; vcom[3 * i + 1] = uy; vcom[3 * i + 2] = uz;
        nvel[i] = make_float4((float)ux, (float)uy, (float)uz, 0.0f);
        vmax[i] = (float)vm;
    }
}

__global__ void form_aold_kernel(const double* __restrict__ ax, const double* __restrict__ ay,
                                 const double* __restrict__ az, int64_t n, double alpha, double G,
                                 double* __restrict__ aold) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        aold[i] = alpha * sqrt(ax[i] * ax[i] + ay[i] * ay[i] + az[i] * az[i]) / G;
}

// Tree arrays come from the device's stream-ordered pool (the context keeps freed memory in the
// pool), so rebuilding a tree every step does not pay cudaMalloc/cudaFree and their device syncs.
template <typename T>
T* dalloc(size_t count, cudaStream_t stream) {
    void* p = nullptr;
    const cudaError_t e = cudaMallocAsync(&p, count * sizeof(T) + 16, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Fail{GT_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e)};
    }
    return (T*)p;
}

int grid_for(gt_context* ctx, int64_t n, int per_block = kBlk) {
    const int64_t want = (n + per_block - 1) / per_block;
    const int64_t cap = (int64_t)ctx->num_sms * 8;
    return (int)std::max<int64_t>(1, std::min(want, cap));
}

void grow_nodes(gt_tree* t, int64_t need, cudaStream_t stream) {
    if (need <= t->node_cap) return;
    const int64_t cap = std::max<int64_t>(need, t->node_cap * 2);
    auto grow = [&](auto*& p, size_t per) {
        using T = std::remove_reference_t<decltype(*p)>;
        T* q = dalloc<T>((size_t)cap * per, stream);
        if (p) {
            check_cuda(cudaMemcpyAsync(q, p, (size_t)t->node_cap * per * sizeof(T), cudaMemcpyDeviceToDevice,
                                       stream), "grow nodes");
            check_cuda(cudaFreeAsync(p, stream), "cudaFreeAsync");
        }
        p = q;
    };
    grow(t->nodes, 1); grow(t->parent, 1); grow(t->next, 1); grow(t->level, 1);
    grow(t->size, 1); grow(t->delta, 1); grow(t->nsoft, 1); grow(t->gc, 3); grow(t->nq2, 1);
    t->node_cap = cap;
}

}  // namespace

void build_tree(gt_context* ctx, gt_tree* t, const double* x, const double* y, const double* z,
                const double* m, const double* soft, int n_systems, const int64_t* in_off,
                cudaEvent_t soft_ready) {
    // with the softenings still on their way, the bounding-box pass checks x, y, z, m alone
    const double* bbox_soft = soft_ready ? nullptr : soft;
    cudaStream_t st = ctx->stream;
    const int64_t n = t->n;
    const gt_build_options& o = t->opt;
    const int S = std::max(1, n_systems);
    t->n_systems = S;
    cudaEvent_t ev[7];
    for (auto& e : ev) check_cuda(cudaEventCreate(&e), "event");
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() { for (int k = 0; k < 7; ++k) cudaEventDestroy(e[k]); }
    } guard{ev};
    check_cuda(cudaEventRecord(ev[0], st), "event");

    // 1. bbox: per-system root cells (geom_dev), live counts, the non-finite count
    t->geom_dev = dalloc<RootGeom>((size_t)S, st);
    t->sys_off_dev = dalloc<int>((size_t)S + 1, st);
    RootGeom* gdev = t->geom_dev;
    unsigned long long* bad_dev = (unsigned long long*)scratch(ctx, kSlotCounters, 64);
    int64_t* in_off_dev = nullptr;
    if (S == 1) {
        const int nbb = std::max(1, std::min(ctx->num_sms * 2, div_up(std::max<int64_t>(n, 1), kBlk)));
        double* part = (double*)scratch(ctx, kSlotPartials, (size_t)nbb * 6 * 8 + (size_t)nbb * 16 + 256);
        unsigned long long* cnt = (unsigned long long*)(part + (size_t)nbb * 6);
        bbox_partial_kernel<<<nbb, kBlk, 0, st>>>(x, y, z, m, bbox_soft, n, part, cnt);
        check_launch(ctx, "bbox_partial_kernel");
        root_geom_kernel<<<1, kRootThreads, 0, st>>>(part, cnt, nbb, gdev, bad_dev, o.randomize_seed, o.shift[0],
                                          o.shift[1], o.shift[2], o.max_level);
        check_launch(ctx, "root_geom_kernel");
    } else {
        // chunks per system: enough blocks that the largest system is not one block's serial work
        int64_t nmax = 0;
        for (int s = 0; s < S; ++s) nmax = std::max<int64_t>(nmax, in_off[s + 1] - in_off[s]);
        const int chunks = (int)std::min<int64_t>(64, std::max<int64_t>(1, (nmax + 8191) / 8192));
        const size_t nparts = (size_t)S * chunks;
        double* part = (double*)scratch(ctx, kSlotPartials, nparts * 64 + 256);
        unsigned long long* cnt = (unsigned long long*)(part + nparts * 6);
        // kept with the tree: the neighbour search, the density solve and explicit-target walks
        // find a particle's system from its index.  Pageable source: the copy is staged before
        // the call returns, in_off may go away after
        t->in_off.assign(in_off, in_off + S + 1);
        t->in_off_dev = dalloc<int64_t>((size_t)S + 1, st);
        in_off_dev = t->in_off_dev;
        check_cuda(cudaMemcpyAsync(in_off_dev, in_off, (size_t)(S + 1) * 8, cudaMemcpyHostToDevice, st),
                   "offsets h2d");
        check_cuda(cudaMemsetAsync(bad_dev, 0, 8, st), "memset");
        bbox_systems_kernel<<<(int)nparts, kBlk, 0, st>>>(x, y, z, m, bbox_soft, in_off_dev, chunks, part, cnt);
        check_launch(ctx, "bbox_systems_kernel");
        root_systems_kernel<<<div_up(S, 128), 128, 0, st>>>(part, cnt, S, chunks, gdev, bad_dev, o.randomize_seed,
                                                            o.shift[0], o.shift[1], o.shift[2], o.max_level);
        check_launch(ctx, "root_systems_kernel");
    }
    {
        t->sys_geom.resize(S);
        unsigned long long bad = 0;
        check_cuda(cudaMemcpyAsync(t->sys_geom.data(), gdev, sizeof(RootGeom) * S, cudaMemcpyDeviceToHost, st),
                   "geom d2h");
        check_cuda(cudaMemcpyAsync(ctx->pinned, bad_dev, 8, cudaMemcpyDeviceToHost, st), "d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(&bad, ctx->pinned, 8);
        if (o.validate && bad > 0)
            throw Fail{GT_ERR_NONFINITE, "gt_build: " + std::to_string(bad) + " particle(s) with non-finite input"};
    }
    t->geom = t->sys_geom[0];
    t->sys_off.assign(1, 0);
    for (int s = 0; s < S; ++s) t->sys_off.push_back(t->sys_off.back() + t->sys_geom[s].n_live);
    t->n_live = t->sys_off.back();
    {
        std::vector<int> off32(t->sys_off.begin(), t->sys_off.end());
        check_cuda(cudaMemcpyAsync(t->sys_off_dev, off32.data(), off32.size() * sizeof(int), cudaMemcpyHostToDevice, st),
                   "offsets h2d");
        check_cuda(cudaStreamSynchronize(st), "sync");  // off32 is pageable and goes out of scope
    }
    check_cuda(cudaEventRecord(ev[1], st), "event");

    // 2. keys (and, in a forest, each particle's system as the second sort key)
    uint64_t* keys = (uint64_t*)scratch(ctx, kSlotKeysA, (size_t)std::max<int64_t>(n, 1) * 8);
    uint32_t* idx = (uint32_t*)scratch(ctx, kSlotValsA, (size_t)std::max<int64_t>(n, 1) * 4);
    uint64_t* sys_key = nullptr;
    if (S > 1) sys_key = dalloc<uint64_t>((size_t)std::max<int64_t>(n, 1), st);
    // the packed x, y, z, m (32 bytes per particle) until the gather; the structure stage reuses
    // the slot afterwards
    double2* pk = (double2*)scratch(ctx, kSlotNodeTmp0, (size_t)std::max<int64_t>(n, 1) * 32);
    if (n > 0) {
        keys_kernel<<<grid_for(ctx, n), kBlk, 0, st>>>(x, y, z, m, n, gdev, o.key_mode, o.max_level, keys, idx,
                                                       in_off_dev, S, sys_key, pk);
        check_launch(ctx, "keys_kernel");
    }
    check_cuda(cudaEventRecord(ev[2], st), "event");

    // 3. sort: live keys < 2^(3*max_level), the massless sentinel is 2^60.  A forest then sorts
    // stably by system (LSD order: key first, system last), which keeps each system's key order
    // and puts every massless particle after all live ones.
    radix_sort_pairs(ctx, keys, idx, n, 61);
    if (S > 1 && n > 1) {
        uint64_t* k2 = dalloc<uint64_t>((size_t)n, st);
        uint32_t* pos = dalloc<uint32_t>((size_t)n, st);
        gather_sys_key_kernel<<<grid_for(ctx, n), kBlk, 0, st>>>(sys_key, idx, n, k2, pos);
        check_launch(ctx, "gather_sys_key_kernel");
        int bits = 1;
        while ((1ll << bits) <= (long long)S) ++bits;
        radix_sort_pairs(ctx, k2, pos, n, bits);
        // permute (keys, idx) by pos through the sys_key buffer and k2's value array
        uint32_t* idx2 = (uint32_t*)k2;  // k2 is no longer needed once pos is sorted: reuse as idx
        permute_pairs_kernel<<<grid_for(ctx, n), kBlk, 0, st>>>(keys, idx, pos, n, sys_key, idx2);
        check_launch(ctx, "permute_pairs_kernel");
        check_cuda(cudaMemcpyAsync(keys, sys_key, (size_t)n * 8, cudaMemcpyDeviceToDevice, st), "copy keys");
        check_cuda(cudaMemcpyAsync(idx, idx2, (size_t)n * 4, cudaMemcpyDeviceToDevice, st), "copy idx");
        check_cuda(cudaFreeAsync(k2, st), "cudaFreeAsync");
        check_cuda(cudaFreeAsync(pos, st), "cudaFreeAsync");
    }
    if (sys_key) check_cuda(cudaFreeAsync(sys_key, st), "cudaFreeAsync");
    check_cuda(cudaEventRecord(ev[3], st), "event");

    // 4. particle arrays in tree order
    const int64_t nalloc = std::max<int64_t>(n, 1);
    t->src = dalloc<SrcP>(nalloc, st);
    t->ssoft = dalloc<double>(nalloc, st);
    t->smass = dalloc<double>(nalloc, st);
    t->order = dalloc<uint32_t>(nalloc, st);
    t->rank = dalloc<uint32_t>(nalloc, st);
    t->leaf_of = dalloc<int>(nalloc, st);
    t->sleaf = dalloc<int>(nalloc, st);
    t->skey = dalloc<uint64_t>(nalloc, st);
    if (n > 0) {
        unsigned long long* bad_soft = nullptr;
        if (soft_ready) {
            check_cuda(cudaStreamWaitEvent(st, soft_ready, 0), "wait");
            if (o.validate) {
                bad_soft = bad_dev + 1;
                check_cuda(cudaMemsetAsync(bad_soft, 0, 8, st), "memset");
            }
        }
        check_cuda(cudaMemsetAsync(t->leaf_of, 0xff, (size_t)n * sizeof(int), st), "memset");
        gather_kernel<<<grid_for(ctx, n), kBlk, 0, st>>>(pk, soft, idx, n, t->src, t->ssoft, t->smass, t->order,
                                                         t->rank, t->sleaf, bad_soft);
        check_launch(ctx, "gather_kernel");
        if (bad_soft) {
            unsigned long long bad = 0;
            check_cuda(cudaMemcpyAsync(ctx->pinned, bad_soft, 8, cudaMemcpyDeviceToHost, st), "d2h");
            check_cuda(cudaStreamSynchronize(st), "sync");
            std::memcpy(&bad, ctx->pinned, 8);
            if (bad > 0)
                throw Fail{GT_ERR_NONFINITE, "gt_build: " + std::to_string(bad) + " particle(s) with non-finite input"};
        }
        check_cuda(cudaMemcpyAsync(t->skey, keys, (size_t)n * 8, cudaMemcpyDeviceToDevice, st), "skey");
    }

    // 5. structure, level by level
    const int64_t nl = t->n_live;
    grow_nodes(t, std::max<int64_t>(1024, (2 * nl) / std::max(1, o.leaf_max) * 3 + 1024) + S, st);
    root_init_kernel<<<div_up(S, kBlk), kBlk, 0, st>>>(t->nodes, gdev, t->sys_off_dev, S, t->parent, t->next,
                                                       t->level, t->size, t->gc);
    check_launch(ctx, "root_init_kernel");
    t->lvl_off.assign(1, 0);
    t->lvl_off.push_back(S);
    uint32_t* total_dev = (uint32_t*)(bad_dev + 2);
    // The tree's depth comes from the sorted keys (one read-back); then every level runs on the
    // device with its offsets and counts in a small device array, each kernel reading its level's
    // range from it and sized for the widest level the node arrays hold, and one read-back at the
    // end.  If the levels outgrow the node arrays the kernels stop emitting and the stage is redone
    // below one level at a time, growing the arrays as it goes.
    bool structured = false;
    if (nl > 0 && o.max_level + 2 < kLvCount) {
        int* depth = (int*)(bad_dev + 3);
        check_cuda(cudaMemsetAsync(depth, 0xff, 4, st), "memset");  // -1: nothing splits
        split_depth_kernel<<<grid_for(ctx, nl), kBlk, 0, st>>>(t->skey, nl, o.leaf_max, o.max_level, depth);
        check_launch(ctx, "split_depth_kernel");
        int dmax = -1;
        check_cuda(cudaMemcpyAsync(ctx->pinned, depth, 4, cudaMemcpyDeviceToHost, st), "depth d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(&dmax, ctx->pinned, 4);
        const int64_t cap = t->node_cap;
        int64_t* lv = (int64_t*)scratch(ctx, kSlotLevels, (2 * kLvCount + 1) * sizeof(int64_t));
        int* bnd = (int*)scratch(ctx, kSlotNodeTmp0, (size_t)cap * 9 * 4);
        uint32_t* nch = (uint32_t*)scratch(ctx, kSlotNodeTmp1, (size_t)cap * 4);
        uint32_t* coff = (uint32_t*)scratch(ctx, kSlotNodeTmp2, (size_t)cap * 4);
        init_levels_kernel<<<1, 1, 0, st>>>(lv, S);
        check_launch(ctx, "init_levels_kernel");
        const int g_split = grid_for(ctx, cap * 8), g_emit = grid_for(ctx, cap);
        for (int L = 0; L <= dmax; ++L) {
            split_kernel<<<g_split, kBlk, 0, st>>>(t->nodes, t->skey, 0, 0, L, o.max_level, o.leaf_max, bnd, nch, lv);
            check_launch(ctx, "split_kernel");
            scan_exclusive_u32(ctx, nch, coff, cap, total_dev, lv + kLvCount + L);
            advance_level_kernel<<<1, 1, 0, st>>>(lv, L, total_dev, cap);
            check_launch(ctx, "advance_level_kernel");
            emit_kernel<<<g_emit, kBlk, 0, st>>>(t->nodes, t->src, gdev, 0, 0, L, o.max_level, bnd, nch, coff,
                                                 t->parent, t->next, t->level, t->size, t->gc, t->sys_off_dev, S, lv);
            check_launch(ctx, "emit_kernel");
        }
        // the deepest level's nodes are all leaves: mark them (emit writes first/nchild of its level)
        const int Lz = dmax + 1;
        if (Lz + 1 < kLvCount) {
            split_kernel<<<g_split, kBlk, 0, st>>>(t->nodes, t->skey, 0, 0, Lz, o.max_level, o.leaf_max, bnd, nch, lv);
            check_launch(ctx, "split_kernel");
            scan_exclusive_u32(ctx, nch, coff, cap, total_dev, lv + kLvCount + Lz);
            advance_level_kernel<<<1, 1, 0, st>>>(lv, Lz, total_dev, cap);
            check_launch(ctx, "advance_level_kernel");
            emit_kernel<<<g_emit, kBlk, 0, st>>>(t->nodes, t->src, gdev, 0, 0, Lz, o.max_level, bnd, nch, coff,
                                                 t->parent, t->next, t->level, t->size, t->gc, t->sys_off_dev, S, lv);
            check_launch(ctx, "emit_kernel");
        }
        int64_t h[2 * kLvCount + 1];
        check_cuda(cudaMemcpyAsync(ctx->pinned, lv, sizeof(h), cudaMemcpyDeviceToHost, st), "levels d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(h, ctx->pinned, sizeof(h));
        // sound only if nothing overflowed and the level after the last one run is empty
        if (h[2 * kLvCount] == 0 && (Lz + 1 >= kLvCount || h[kLvCount + Lz + 1] == 0)) {
            for (int L = 1; L < kLvCount && h[kLvCount + L] > 0; ++L) t->lvl_off.push_back(h[L] + h[kLvCount + L]);
            structured = true;
        }
    }
    for (int L = 0; !structured; ++L) {
        const int64_t a = t->lvl_off[L], b = t->lvl_off[L + 1];
        const int64_t cnt_l = b - a;
        if (cnt_l <= 0) break;
        // sized for the widest level possible (node_cap), so the workspace never regrows mid-build
        const int64_t wmax = std::max<int64_t>(cnt_l, t->node_cap);
        int* bnd = (int*)scratch(ctx, kSlotNodeTmp0, (size_t)wmax * 9 * 4);
        uint32_t* nch = (uint32_t*)scratch(ctx, kSlotNodeTmp1, (size_t)wmax * 4);
        uint32_t* coff = (uint32_t*)scratch(ctx, kSlotNodeTmp2, (size_t)wmax * 4);
        split_kernel<<<div_up(cnt_l * 8, kBlk), kBlk, 0, st>>>(t->nodes, t->skey, a, b, L, o.max_level,
                                                               o.leaf_max, bnd, nch);
        check_launch(ctx, "split_kernel");
        scan_exclusive_u32(ctx, nch, coff, cnt_l, total_dev);
        uint32_t total = 0;
        check_cuda(cudaMemcpyAsync(ctx->pinned, total_dev, 4, cudaMemcpyDeviceToHost, st), "count d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(&total, ctx->pinned, 4);
        grow_nodes(t, b + (int64_t)total, st);
        emit_kernel<<<div_up(cnt_l, kBlk), kBlk, 0, st>>>(t->nodes, t->src, gdev, a, b, L, o.max_level,
                                                          bnd, nch, coff, t->parent, t->next, t->level,
                                                          t->size, t->gc, t->sys_off_dev, S);
        check_launch(ctx, "emit_kernel");
        if (total == 0) break;
        t->lvl_off.push_back(b + (int64_t)total);
    }
    t->n_levels = (int)t->lvl_off.size() - 1;
    t->n_nodes = t->lvl_off.back();
    check_cuda(cudaEventRecord(ev[4], st), "event");

    // 6. moments, deepest level first
    for (int L = t->n_levels - 1; L >= 0; --L) {
        const int64_t a = t->lvl_off[L], b = t->lvl_off[L + 1];
        const int64_t warps = b - a;
        moments_kernel<<<div_up(warps, kMomNodesPerBlock), kBlk, 0, st>>>(
            t->nodes, t->src, t->smass, t->ssoft, t->order, a, b, t->size, t->gc, t->delta,
            t->nsoft, t->nq2, t->leaf_of, t->sleaf, o.nodelta);
        check_launch(ctx, "moments_kernel");
    }
    check_cuda(cudaEventRecord(ev[5], st), "event");
    check_cuda(cudaEventRecord(ev[6], st), "event");
    check_cuda(cudaEventSynchronize(ev[6]), "sync");
    float ms;
    for (int k = 0; k < 6; ++k) {
        check_cuda(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
        t->build_ms[k] = ms;
    }
    check_cuda(cudaEventElapsedTime(&ms, ev[0], ev[6]), "elapsed");
    t->build_ms[6] = ms;
}

void run_peano_keys(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                    const double corner[3], double len, int bits, uint64_t* ph_hi, uint64_t* ph_lo,
                    uint64_t* mo_hi, uint64_t* mo_lo) {
    if (n <= 0) return;
    peano_keys_kernel<<<grid_for(ctx, n), kBlk, 0, ctx->stream>>>(x, y, z, n, corner[0], corner[1],
                                                                  corner[2], len, bits, ph_hi, ph_lo,
                                                                  mo_hi, mo_lo);
    check_launch(ctx, "peano_keys_kernel");
}

void tree_velocities(gt_context* ctx, gt_tree* t, const double* vx, const double* vy, const double* vz,
                     bool particles_only) {
    cudaStream_t st = ctx->stream;
    const int64_t nl = std::max<int64_t>(t->n_live, 1), nn = std::max<int64_t>(t->n_nodes, 1);
    if (!t->svel) {
        t->svel = dalloc<float4>((size_t)nl, st);
        t->nvel = dalloc<float4>((size_t)nn, st);
        t->vcom = dalloc<double>((size_t)nn * 3, st);
        if (!t->vmax) t->vmax = dalloc<float>((size_t)nn, st);  // tree reuse may have made it
    }
    if (t->n_live > 0) {
        gather_vel_kernel<<<grid_for(ctx, t->n_live), kBlk, 0, st>>>(vx, vy, vz, t->order, t->n_live, t->svel);
        check_launch(ctx, "gather_vel_kernel");
    }
    for (int L = t->n_levels - 1; L >= 0 && !particles_only; --L) {
        const int64_t a = t->lvl_off[L], b = t->lvl_off[L + 1];
        vel_moments_kernel<<<div_up(b - a, kMomNodesPerBlock), kBlk, 0, st>>>(t->nodes, t->smass, t->order, vx, vy, vz, a,
                                                                       b, t->vcom, t->nvel, t->vmax);
        check_launch(ctx, "vel_moments_kernel");
    }
}

void tree_gas(gt_context* ctx, gt_tree* t, const uint8_t* type, const double* zeta) {
    cudaStream_t st = ctx->stream;
    const int64_t n = std::max<int64_t>(t->n, 1), nn = std::max<int64_t>(t->n_nodes, 1);
    // allocated once: a plan captured after the first call keeps pointing at them
    if (!t->stype) {
        t->stype = dalloc<uint8_t>((size_t)n, st);
        t->szeta = dalloc<double>((size_t)n, st);
        t->nsink = dalloc<uint32_t>((size_t)nn, st);
    }
    if (t->n > 0) {
        gather_gas_kernel<<<grid_for(ctx, t->n), kBlk, 0, st>>>(type, zeta, t->order, t->n, t->stype, t->szeta);
        check_launch(ctx, "gather_gas_kernel");
    }
    check_cuda(cudaMemsetAsync(t->nsink, 0, (size_t)nn * sizeof(uint32_t), st), "memset");
    if (t->n_live > 0 && type) {
        count_sinks_kernel<<<grid_for(ctx, t->n_live), kBlk, 0, st>>>(t->stype, t->sleaf, t->parent, t->n_live,
                                                                      t->nsink);
        check_launch(ctx, "count_sinks_kernel");
    }
    t->gas_zeta = zeta != nullptr;
}

void run_form_aold(gt_context* ctx, int64_t n, const double* ax, const double* ay,
                   const double* az, double alpha, double G, double* aold) {
    if (n <= 0) return;
    form_aold_kernel<<<grid_for(ctx, n), kBlk, 0, ctx->stream>>>(ax, ay, az, n, alpha, G, aold);
    check_launch(ctx, "form_aold_kernel");
}

}  // namespace gt
