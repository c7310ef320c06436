// Neighbour search and the density solve on the gravity tree: shmem::ngb_search,
// ngb_search_reverse and density (shmem/hydro.h:65-117, hydro.cc:37-327), with the per-node hmax
// of Tree::init_hmax / raise_hmax (tree.cc:287-338).
//
// The search prunes against each node's BOX, not its centre of mass: a 32-byte search node holds
// the float geometric centre and a conservative half side (the build's half side plus 1e-6 of the
// root side plus four float ulps of the largest centre coordinate, tree.cc:490-505), with the
// reference's threading (first child / next).  One thread follows the threading for one centre,
// as the reference's loop does, so every list comes out in tree order -- the reference's order --
// and the density sums accumulate in the reference's order too.  Neighbouring centres (tree-ordered
// targets) follow nearly the same path, so a warp's threads mostly read the same nodes.
//
// Lists are CSR: a counting pass, an exclusive scan, and a filling pass over the same traversal.
//
// Forests (gt_build_systems): roots 0 .. n_systems-1 each stand alone in the threading.  A centre
// searches every system in turn, or the one system its caller names; a density target searches the
// system that owns its particle index.  Each system's search nodes are padded by its own root side,
// so a system searched in a forest finds what it finds in a tree of its own.
//
// SHMEM_NGB_COUNT (hydro.cc:7-35): a context with counting on tallies, per gather search, the nodes
// visited, the particles examined, the neighbours kept and the nodes admitted only by the staleness
// pad, and per density target the iterations it took; the counting variants of the kernels are
// separate instantiations, so the plain ones keep their code.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "gt_internal.cuh"

namespace gt {
namespace {

constexpr int kBlk = 128;

int grid_of(gt_context* ctx, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + kBlk - 1) / kBlk, (int64_t)ctx->num_sms * 16));
}

__device__ __forceinline__ double min_image(double s, double box) {
    if (box > 0) {
        if (s > 0.5 * box) s -= box;
        else if (s < -0.5 * box) s += box;
    }
    return s;
}

__device__ __forceinline__ float up_float(double h) {  // rounded up to float (tree.cc:288-291)
    const float f = (float)h;
    return (double)f < h ? nextafterf(f, 1e30f) : f;
}

// The pad 1e-6 of the root side is that of the node's own system: root s is node s, and a deeper
// node belongs to the system whose live tree positions hold its first particle.
__global__ void pack_snode_kernel(const GNode* __restrict__ nodes, const int* __restrict__ next,
                                  const double* __restrict__ gc, const double* __restrict__ size, int64_t nn,
                                  const int* __restrict__ sys_off, int n_systems, SNodeG* __restrict__ sn) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = gc[3 * i], y = gc[3 * i + 1], z = gc[3 * i + 2];
        const double cm = fmax(fabs(x), fmax(fabs(y), fabs(z)));
        const int sys = n_systems > 1 ? (i < n_systems ? (int)i : system_of(sys_off, n_systems, nodes[i].plo)) : 0;
        const double eps = 1e-6 * size[sys];
        SNodeG s;
        s.cx = (float)x; s.cy = (float)y; s.cz = (float)z;
        s.half = (float)(0.5 * size[i] + eps + 4.0 * (double)FLT_EPSILON * cm);
        s.first = nodes[i].first;
        s.next = next[i];
        s.plo = nodes[i].plo;
        s.phi = nodes[i].phi;
        sn[i] = s;
    }
}

// Tree::init_hmax: every gas particle i < n_gas with h > 0 raises its leaf and ancestors to h
// rounded up to float; the climb stops at the first ancestor already covering it.  A float max
// through its bit pattern (non-negative), so the result does not depend on the order.
__global__ void hmax_kernel(const double* __restrict__ h, const int* __restrict__ leaf, int64_t n,
                            const int* __restrict__ parent, bool by_particle, float* __restrict__ hmax) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double hi = h[i];
        const int lf = leaf[i];
        if ((by_particle && !(hi > 0)) || lf < 0) continue;
        const unsigned int want = __float_as_uint(up_float(hi));
        for (int no = lf; no >= 0; no = parent[no]) {
            unsigned int* slot = reinterpret_cast<unsigned int*>(hmax + no);
            if (*reinterpret_cast<volatile unsigned int*>(slot) >= want) break;
            atomicMax(slot, want);
        }
    }
}

struct SearchGeom {
    int n_roots;         // roots 0 .. n_roots-1: 1, n_systems in a forest, 0 for a tree without nodes
    int n_systems;
    const int64_t* in_off;  // forest: system s owns the particle indices [in_off[s], in_off[s+1])
    const SNodeG* sn;
    const SrcP* src;
    const uint32_t* order;
    const float* xpad;   // null: 0
    const float* vmax;   // null: 0
    const float* hmax;   // reverse search
    double elapsed, box;
};

// What a gather search tallies under SHMEM_NGB_COUNT (hydro.cc:51-106): nodes visited, particles
// examined in the leaves opened, nodes admitted only by the vmax * elapsed and xpad pads.
struct NgbTally {
    unsigned long long nodes = 0, examined = 0, pad = 0;
};

// One traversal for one centre in the reference's node order, from roots r0 .. r1-1 in turn.
// REVERSE: gas particles j < n_gas with radius <= r < h[j] (ngb_search_reverse); otherwise
// r < radius (ngb_search).  emit(j, s) receives the particle index and its tree position.  COUNT
// (gather only, as the reference counts): the tally.
template <bool REVERSE, bool COUNT = false, typename F>
__device__ __forceinline__ void search(const SearchGeom& g, int r0, int r1, double px, double py, double pz,
                                       double radius, const double* __restrict__ h, int64_t n_gas, F&& emit,
                                       NgbTally* tally = nullptr) {
    const double r2max = radius * radius;
    for (int root = r0; root < r1; ++root)
    for (int node = root; node >= 0;) {
        if (COUNT) ++tally->nodes;
        const float4 a = __ldg(reinterpret_cast<const float4*>(g.sn + node));
        const int4 b = __ldg(reinterpret_cast<const int4*>(g.sn + node) + 1);
        const double half = (double)a.w;
        double dist;
        if (REVERSE) {
            const double hm = (double)__ldg(g.hmax + node);
            if (hm <= radius) { node = b.y; continue; }
            dist = hm + half;
        } else {
            dist = radius + half;
        }
        if (g.xpad) dist += (double)__ldg(g.xpad + node);
        if (g.elapsed > 0 && g.vmax) dist += (double)__ldg(g.vmax + node) * g.elapsed;
        const double dx = min_image((double)a.x - px, g.box);
        if (dx > dist || -dx > dist) { node = b.y; continue; }
        const double dy = min_image((double)a.y - py, g.box);
        if (dy > dist || -dy > dist) { node = b.y; continue; }
        const double dz = min_image((double)a.z - pz, g.box);
        if (dz > dist || -dz > dist) { node = b.y; continue; }
        dist += 0.7320508075688772 * half;
        if (dx * dx + dy * dy + dz * dz > dist * dist) { node = b.y; continue; }
        if (COUNT && g.elapsed > 0) {
            const double nopad = radius + 1.7320508075688772 * half;
            if (dx * dx + dy * dy + dz * dz > nopad * nopad) ++tally->pad;
        }
        if (b.x < 0) {
            if (COUNT) tally->examined += (unsigned long long)(b.w - b.z);
            for (int s = b.z; s < b.w; ++s) {
                const uint32_t j = __ldg(g.order + s);
                if (REVERSE && (int64_t)j >= n_gas) continue;
                const double2 xy = __ldg(reinterpret_cast<const double2*>(g.src + s));
                const double zz = __ldg(reinterpret_cast<const double*>(g.src + s) + 2);
                const double ox = min_image(xy.x - px, g.box), oy = min_image(xy.y - py, g.box),
                             oz = min_image(zz - pz, g.box);
                // |d|^2 as x*x + y*y + z*z without contraction (Vec3d::norm_sq)
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(oz, oz));
                bool keep;
                if (REVERSE) {
                    const double hj = __ldg(h + j);
                    keep = r2 >= r2max && r2 < hj * hj;
                } else {
                    keep = r2 < r2max;
                }
                if (keep) emit(j, s);
            }
            node = b.y;
        } else {
            node = b.x;
        }
    }
}

struct NgbArgs {
    SearchGeom g;
    const double *cx, *cy, *cz, *radius;
    const int* systems;           // per centre, the one system searched; null: every system
    int64_t n;
    int mode;
    const double* h;
    int64_t n_gas;
    uint32_t* count;              // counting pass
    unsigned long long* total;    // counting pass: [0] sum of the counts, [1] centres naming no
                                  // system, [2] centres with more than kcache entries
    const int64_t* start;         // filling pass
    uint32_t* found;
    unsigned long long* tally;    // SHMEM_NGB_COUNT totals (calls, nodes, examined, kept, pad)
    // The counting pass keeps each centre's first kcache entries (entry k of centre c at
    // cache[k * n + c]); the lists of centres with at most kcache entries are then copied from
    // there, and only the others are searched again.  kcache 0: no cache.
    uint32_t* cache;
    int kcache;
};

// Sums v over the warp and adds it to *dst from lane 0; every lane of the warp calls it.
__device__ __forceinline__ void warp_flush(unsigned long long v, unsigned long long* dst) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// The roots a centre searches: every system's, or those of the system it names (checked: a
// system outside [0, n_systems) searches nothing and is counted in *bad).
__device__ __forceinline__ void roots_of(const SearchGeom& g, const int* systems, int64_t c, int& r0, int& r1,
                                         unsigned long long* bad) {
    r0 = 0;
    r1 = g.n_roots;
    if (!systems) return;
    const int s = systems[c];
    if (s < 0 || s >= g.n_systems) {
        if (bad) atomicAdd(bad, 1ull);
        r1 = 0;
        return;
    }
    r0 = s;
    r1 = min(s + 1, g.n_roots);
}

template <bool FILL, bool COUNT>
__global__ void __launch_bounds__(kBlk) ngb_kernel(const NgbArgs a) {
    unsigned long long mine = 0, calls = 0, kept = 0, over = 0;
    NgbTally tl;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < a.n; c += (int64_t)gridDim.x * blockDim.x) {
        const double px = a.cx[c], py = a.cy[c], pz = a.cz[c], r = a.radius[c];
        int r0, r1;
        roots_of(a.g, a.systems, c, r0, r1, FILL ? nullptr : a.total + 1);
        if (FILL && a.kcache > 0 && a.count[c] <= (uint32_t)a.kcache) continue;  // copied from the cache
        int64_t k = FILL ? a.start[c] : 0;
        auto emit = [&](uint32_t j, int) {
            if (FILL) a.found[k] = j;
            else if (k < a.kcache) a.cache[k * a.n + c] = j;
            ++k;
        };
        if (a.mode != GT_NGB_REVERSE) {
            search<false, COUNT>(a.g, r0, r1, px, py, pz, r, nullptr, 0, emit, &tl);
            if (COUNT) {
                ++calls;
                kept += (unsigned long long)k;
            }
        }
        if (a.mode != GT_NGB_GATHER) search<true>(a.g, r0, r1, px, py, pz, r, a.h, a.n_gas, emit);
        if (!FILL) {
            a.count[c] = (uint32_t)k;
            mine += (unsigned long long)k;
            over += k > a.kcache ? 1ull : 0ull;
        }
    }
    if (!FILL) {
        warp_flush(mine, a.total);
        warp_flush(over, a.total + 2);
    }
    if (COUNT) {
        warp_flush(calls, a.tally + 0);
        warp_flush(tl.nodes, a.tally + 1);
        warp_flush(tl.examined, a.tally + 2);
        warp_flush(kept, a.tally + 3);
        warp_flush(tl.pad, a.tally + 4);
    }
}

// The lists of the centres the counting pass kept whole in the cache, into their CSR slots.
__global__ void ngb_copy_kernel(const uint32_t* __restrict__ cache, int kcache, const uint32_t* __restrict__ cnt,
                                const int64_t* __restrict__ start, int64_t n, uint32_t* __restrict__ found) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t m = cnt[c];
        if (m > (uint32_t)kcache) continue;
        const int64_t s0 = start[c];
        for (uint32_t k = 0; k < m; ++k) found[s0 + k] = cache[(int64_t)k * n + c];
    }
}

__global__ void widen_kernel(const uint32_t* __restrict__ ex, const uint32_t* __restrict__ cnt, int64_t n,
                             int64_t* __restrict__ start) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        start[i] = (int64_t)ex[i];
        if (i == n - 1) start[n] = (int64_t)ex[i] + (int64_t)cnt[i];
    }
}

// ---- the density solve ------------------------------------------------------------------------
// The cubic spline of support h in n_dims dimensions (shmem/hydro.h:25-63).
__device__ __forceinline__ double kernel_norm(double h, int dim) {
    if (dim == 1) return (4.0 / 3.0) / h;
    if (dim == 2) return 40.0 / (7.0 * M_PI * h * h);
    return 8.0 / (M_PI * h * h * h);
}
__device__ __forceinline__ double ball_vol(double h, int dim) {
    if (dim == 1) return 2.0 * h;
    if (dim == 2) return M_PI * h * h;
    return 4.0 * M_PI / 3.0 * h * h * h;
}

struct DensSums {
    double wsum, dwdh, rho, mom[6], face[3];
    int inside;
};

struct DensArgs {
    SearchGeom g;
    const double* smass;
    const uint8_t* stype;  // tree order; null: every particle gas
    const uint32_t* rank;
    const uint32_t* targets;
    int64_t nt;
    double des_ngb, ngb_tol, h_default;
    const double* h_default_sys;  // forest without h_start: the default h of each system
    const double* h_start;
    const double* cond_prev;  // per particle index
    int n_dims, face_corr;
    double *h, *rho;
    int *nngb, *iters;
    unsigned long long* tally;  // SHMEM_NGB_COUNT: calls, nodes, examined, kept, pad, iterations [8]
    // candidate cache: per thread of the grid, cand_cap tree positions, interleaved (entry k of
    // thread i at cand[k * n_threads + i])
    uint32_t* cand;
    int cand_cap;
    int64_t n_threads;
};

__device__ __forceinline__ void dens_zero(DensSums& s) {
    s.wsum = s.dwdh = s.rho = 0.0;
    for (int c = 0; c < 6; ++c) s.mom[c] = 0.0;
    s.face[0] = s.face[1] = s.face[2] = 0.0;
    s.inside = 0;
}

// One gas neighbour at offset (dx, dy, dz) from the target, inside h: its kernel weight and the
// sums the solve reads (hydro.cc:209-222).
__device__ __forceinline__ void dens_add(double dx, double dy, double dz, double m, double h, double norm, int dim,
                                         DensSums& s) {
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double q = r / h;
    double w = 0.0, dh = 0.0;
    if (q < 1.0) {
        double f, fp;
        if (q < 0.5) {
            f = 1.0 - 6.0 * q * q + 6.0 * q * q * q;
            fp = -12.0 * q + 18.0 * q * q;
        } else {
            const double u = 1.0 - q;
            f = 2.0 * u * u * u;
            fp = -6.0 * u * u;
        }
        w = norm * f;
        dh = -((double)dim / h) * norm * f - (q / h) * norm * fp;
    }
    s.wsum += w;
    s.dwdh += dh;
    s.rho += m * w;
    s.mom[0] += dx * dx * w; s.mom[1] += dy * dy * w; s.mom[2] += dz * dz * w;
    s.mom[3] += dx * dy * w; s.mom[4] += dy * dz * w; s.mom[5] += dx * dz * w;
    s.face[0] += dx * w; s.face[1] += dy * w; s.face[2] += dz * w;
    if (r < h) ++s.inside;
}

// One evaluation at h: the sums over the GAS neighbours inside h, in tree order (hydro.cc:205-222).
// The neighbours found are buffered and their kernel sums evaluated in runs, in the order found:
// interleaving the FP64 sums with the traversal made the lanes of a warp that were still walking
// wait on every neighbour another lane had found.
constexpr int kDensBuf = 64;
// The candidate cache (below): capacity per thread, and the radius of a refill relative to the h
// that outgrew the cache.
constexpr int kCandCap = 160;
constexpr double kCacheFirst = 1.1;
constexpr double kCacheGrow = 1.4;

template <bool COUNT>
__device__ void dens_eval(const DensArgs& a, int r0, int r1, double px, double py, double pz, double h, DensSums& s,
                          NgbTally& tl, unsigned long long& kept) {
    dens_zero(s);
    const int dim = a.n_dims;
    const double norm = kernel_norm(h, dim);
    int buf[kDensBuf];
    int nb = 0;
    auto drain = [&]() {
        for (int i = 0; i < nb; ++i) {
            const int sp = buf[i];
            if (a.stype && __ldg(a.stype + sp) != 0) continue;
            const double2 xy = __ldg(reinterpret_cast<const double2*>(a.g.src + sp));
            const double zz = __ldg(reinterpret_cast<const double*>(a.g.src + sp) + 2);
            dens_add(min_image(xy.x - px, a.g.box), min_image(xy.y - py, a.g.box), min_image(zz - pz, a.g.box),
                     __ldg(a.smass + sp), h, norm, dim, s);
        }
        nb = 0;
    };
    search<false, COUNT>(a.g, r0, r1, px, py, pz, h, nullptr, 0, [&](uint32_t, int sp) {
        if (COUNT) ++kept;
        if (nb == kDensBuf) drain();
        buf[nb++] = sp;
    }, &tl);
    drain();
}

// The candidate cache of the Newton iterations.  One search at radius R stores the GAS particles it
// finds (their tree positions, in the search's order) in the thread's slice of a global array; an
// evaluation at any h <= R then scans them and keeps those with r^2 < h^2, with the search's own
// r^2 expression.  That is the set a search at h would keep, in the same order (a larger radius
// only adds particles between them: the order is the threading's), so the sums are bit-identical,
// and an iteration that shrinks h costs a scan of a few dozen candidates instead of a traversal.
// A search that finds more than cand_cap gas particles leaves the cache empty.
__device__ __forceinline__ int cache_fill(const DensArgs& a, int r0, int r1, double px, double py, double pz,
                                          double R, uint32_t* __restrict__ slot, int64_t stride) {
    int k = 0;
    const int cap = a.cand_cap;
    NgbTally none;
    search<false>(a.g, r0, r1, px, py, pz, R, nullptr, 0, [&](uint32_t, int sp) {
        if (a.stype && __ldg(a.stype + sp) != 0) return;
        if (k < cap) slot[(int64_t)k * stride] = (uint32_t)sp;
        ++k;
    }, &none);
    return k <= cap ? k : -1;
}

__device__ void cache_eval(const DensArgs& a, const uint32_t* __restrict__ slot, int64_t stride, int n, double px,
                           double py, double pz, double h, DensSums& s) {
    dens_zero(s);
    const int dim = a.n_dims;
    const double norm = kernel_norm(h, dim);
    const double r2max = h * h;
    for (int k = 0; k < n; ++k) {
        const int sp = (int)slot[(int64_t)k * stride];
        const double2 xy = __ldg(reinterpret_cast<const double2*>(a.g.src + sp));
        const double zz = __ldg(reinterpret_cast<const double*>(a.g.src + sp) + 2);
        const double ox = min_image(xy.x - px, a.g.box), oy = min_image(xy.y - py, a.g.box),
                     oz = min_image(zz - pz, a.g.box);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(oz, oz));
        if (r2 < r2max) dens_add(ox, oy, oz, __ldg(a.smass + sp), h, norm, dim, s);
    }
}

// Rank-d inverse of the symmetric moments (xx yy zz xy yz xz), row-major, zero when degenerate
// (shmem/vec.h:43-66; 3-D: cofactors over the determinant).
__device__ bool invert_moments(const double* m, double* B, int n_dims) {
    for (int i = 0; i < 9; ++i) B[i] = 0.0;
    if (n_dims == 1) {
        if (fabs(m[0]) < 1e-300) return false;
        B[0] = 1.0 / m[0];
        return true;
    }
    if (n_dims == 2) {
        const double det = m[0] * m[1] - m[3] * m[3];
        if (fabs(det) < 1e-300) return false;
        B[0] = m[1] / det; B[1] = -m[3] / det;
        B[3] = -m[3] / det; B[4] = m[0] / det;
        return true;
    }
    const double a00 = m[0], a01 = m[3], a02 = m[5], a11 = m[1], a12 = m[4], a22 = m[2];
    const double a10 = a01, a20 = a02, a21 = a12;
    const double d = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
    if (d == 0.0 || d != d) return false;
    const double id = 1.0 / d;
    B[0] = (a11 * a22 - a12 * a21) * id; B[1] = (a02 * a21 - a01 * a22) * id; B[2] = (a01 * a12 - a02 * a11) * id;
    B[3] = (a12 * a20 - a10 * a22) * id; B[4] = (a00 * a22 - a02 * a20) * id; B[5] = (a02 * a10 - a00 * a12) * id;
    B[6] = (a10 * a21 - a11 * a20) * id; B[7] = (a01 * a20 - a00 * a21) * id; B[8] = (a00 * a11 - a01 * a10) * id;
    return true;
}

// The convergence test and the bisection-guarded Newton step of one iteration with the
// face-closure and condition-number corrections and the growing tolerance (hydro.cc:224-272) for
// particle p after an evaluation at h: true when converged (h kept), else h moves.
struct NewtonParams {
    double des_ngb, ngb_tol;
    const double* cond_prev;
    int n_dims, face_corr;
};

__device__ __forceinline__ bool dens_newton(const NewtonParams a, uint32_t p, const DensSums& s, int iter, double& h,
                                         double& h_lo, double& h_hi) {
    const int dim = a.n_dims;
    const double n_eff = ball_vol(h, dim) * s.wsum;
    double ncorr = 1.0;
    if (a.cond_prev) {
        const double cn = a.cond_prev[p];
        if (cn > 100.0) ncorr = fmin(sqrt(1.0 + (cn - 100.0) / 1000.0), 2.0);
    }
    double des_eff = a.des_ngb * ncorr, tol_eff = a.ngb_tol * ncorr;
    if (a.face_corr && s.wsum > 0) {
        double B[9];
        if (invert_moments(s.mom, B, dim)) {
            const double vol = 1.0 / s.wsum;
            const double dx_i = sqrt(vol * (s.mom[0] + s.mom[1] + s.mom[2]));
            double sum_abs = 0.0;
            for (int r = 0; r < 3; ++r) {
                const double leak =
                    (B[3 * r] * s.face[0] + B[3 * r + 1] * s.face[1] + B[3 * r + 2] * s.face[2]) * (2.0 * vol);
                sum_abs += fabs(leak) / dim;
            }
            const double denom = 2.0 * dim * pow(dx_i, dim - 1);
            if (denom > 0) {
                const double fce = sum_abs / denom;
                if (fce > 0.35) ncorr = fmax(ncorr, fmin(fce / 0.35, 2.0));
                des_eff = a.des_ngb * ncorr;
                tol_eff = a.ngb_tol * ncorr;
            }
        }
    }
    if (iter > 1) tol_eff = fmin(0.25 * des_eff, tol_eff * exp(0.1 * log(des_eff / (16.0 * tol_eff)) * iter));
    const double res = n_eff - des_eff;
    if (fabs(res) < tol_eff) return true;
    if (res > 0) h_hi = h; else h_lo = h;
    const double dn = ball_vol(h, dim) * ((double)dim / h * s.wsum + s.dwdh);
    double hn = dn > 0 ? h - res / dn : 0.0;
    if (hn <= h_lo || (h_hi > 0 && hn >= h_hi) || hn <= 0) {
        if (h_hi > 0) hn = h_lo > 0 ? sqrt(h_lo * h_hi) : 0.5 * h_hi;
        else hn = h * (res > 0 ? 0.7 : 1.6);
    }
    h = hn;
    return false;
}

__device__ __forceinline__ NewtonParams newton_params(const DensArgs& a) {
    return NewtonParams{a.des_ngb, a.ngb_tol, a.cond_prev, a.n_dims, a.face_corr};
}

// One thread per target: up to 100 iterations of evaluation and Newton step, then, when the solve
// did not converge, one more evaluation at the final h (hydro.cc:189-297).  In a forest the target
// searches the system that owns its particle index.  COUNT: every evaluation is one gather search
// of the tally, and the target's iterations go to the histogram (hydro.cc:293-296).  ONE_ROOT: a
// single-system tree with nodes, whose one root (node 0) the compiler then knows, which keeps the
// traversal's registers those of a plain tree walk.
template <bool COUNT, bool ONE_ROOT>
__global__ void __launch_bounds__(kBlk, 6) density_kernel(const DensArgs a) {
    NgbTally tl;
    unsigned long long calls = 0, kept = 0, hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nt; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p = a.targets[t];
        const uint32_t sp = a.rank[p];
        const double px = a.g.src[sp].x, py = a.g.src[sp].y, pz = a.g.src[sp].z;
        int r0 = 0, r1 = ONE_ROOT ? 1 : a.g.n_roots;
        if (!ONE_ROOT && a.g.in_off) {
            r0 = system_of(a.g.in_off, a.g.n_systems, (int64_t)p);
            r1 = r0 + 1;
        }
        double h = a.h_start ? a.h_start[t] : (a.h_default_sys ? a.h_default_sys[r0] : a.h_default);
        double h_lo = 0.0, h_hi = 0.0;
        int iter = 0;
        bool converged = false;
        DensSums s;
        // the candidate cache (not for the counting variant, whose tallies are per search):
        // filled at the first h, refilled at kCacheGrow times h when h outgrows it
        uint32_t* slot = a.cand ? a.cand + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) : nullptr;
        double R = -1.0;   // radius of the cached search; < 0: nothing cached
        int ncand = 0;
        bool cache_ok = !COUNT && a.cand != nullptr;
        auto evaluate = [&](double hh) {
            if (cache_ok && !(R >= hh)) {
                const double rad = (R < 0 ? kCacheFirst : kCacheGrow) * hh;
                ncand = cache_fill(a, r0, r1, px, py, pz, rad, slot, a.n_threads);
                if (ncand < 0) cache_ok = false;  // too many candidates: search directly from now on
                else R = rad;
            }
            if (cache_ok) cache_eval(a, slot, a.n_threads, ncand, px, py, pz, hh, s);
            else dens_eval<COUNT>(a, r0, r1, px, py, pz, hh, s, tl, kept);
        };
        for (; iter < 100; ++iter) {
            evaluate(h);
            if (COUNT) ++calls;
            if (dens_newton(newton_params(a), p, s, iter, h, h_lo, h_hi)) { converged = true; break; }
        }
        if (!converged) {  // rho of the final h (hydro.cc:281-293)
            evaluate(h);
            if (COUNT) ++calls;
        }
        if (COUNT) ++hist[min(converged ? iter + 1 : 100, 8) - 1];
        a.h[t] = h;
        a.rho[t] = s.rho;
        a.nngb[t] = s.inside;
        a.iters[t] = iter;
    }
    if (COUNT) {
        warp_flush(calls, a.tally + 0);
        warp_flush(tl.nodes, a.tally + 1);
        warp_flush(tl.examined, a.tally + 2);
        warp_flush(kept, a.tally + 3);
        warp_flush(tl.pad, a.tally + 4);
        for (int k = 0; k < 8; ++k) warp_flush(hist[k], a.tally + 5 + k);
    }
}

// Per system of a forest, the bounding box of all its particles (massless too) for its default h:
// block b reduces chunk b % chunks of system b / chunks, through the particles' tree positions.
__global__ void density_bbox_kernel(const SrcP* __restrict__ src, const uint32_t* __restrict__ rank,
                                    const int64_t* __restrict__ in_off, int chunks, double* __restrict__ part) {
    const int s = blockIdx.x / chunks, c = blockIdx.x % chunks;
    const int64_t lo0 = in_off[s], len = in_off[s + 1] - lo0;
    const int64_t b = lo0 + len * c / chunks, e = lo0 + len * (c + 1) / chunks;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
        const SrcP q = src[rank[i]];
        const double v[3] = {q.x, q.y, q.z};
        for (int k = 0; k < 3; ++k) { lo[k] = fmin(lo[k], v[k]); hi[k] = fmax(hi[k], v[k]); }
    }
    __shared__ double sh[6][kBlk];
    for (int k = 0; k < 3; ++k) { sh[k][threadIdx.x] = lo[k]; sh[3 + k][threadIdx.x] = hi[k]; }
    __syncthreads();
    for (int o = kBlk / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 3; ++k) {
                sh[k][threadIdx.x] = fmin(sh[k][threadIdx.x], sh[k][threadIdx.x + o]);
                sh[3 + k][threadIdx.x] = fmax(sh[3 + k][threadIdx.x], sh[3 + k][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) part[6 * (int64_t)blockIdx.x + k] = sh[k][0];
}

// bounding box of every particle (massless too), for the density solve's default h
__global__ void bbox_all_kernel(const SrcP* __restrict__ src, int64_t n, double* __restrict__ part) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v[3] = {src[i].x, src[i].y, src[i].z};
        for (int k = 0; k < 3; ++k) { lo[k] = fmin(lo[k], v[k]); hi[k] = fmax(hi[k], v[k]); }
    }
    __shared__ double sh[6][kBlk];
    for (int k = 0; k < 3; ++k) { sh[k][threadIdx.x] = lo[k]; sh[3 + k][threadIdx.x] = hi[k]; }
    __syncthreads();
    for (int o = kBlk / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 3; ++k) {
                sh[k][threadIdx.x] = fmin(sh[k][threadIdx.x], sh[k][threadIdx.x + o]);
                sh[3 + k][threadIdx.x] = fmax(sh[3 + k][threadIdx.x], sh[3 + k][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) part[6 * blockIdx.x + k] = sh[k][0];
}

SearchGeom geom_of(gt_context* ctx, gt_tree* t, double elapsed, double box) {
    ensure_snodes(ctx, t);
    SearchGeom g;
    g.n_roots = t->n_nodes > 0 ? t->n_systems : 0;
    g.n_systems = t->n_systems;
    g.in_off = t->n_systems > 1 ? t->in_off_dev : nullptr;
    g.sn = t->snode;
    g.src = t->src;
    g.order = t->order;
    g.xpad = t->xpad;
    g.vmax = t->vmax;
    g.hmax = t->hmax;
    g.elapsed = elapsed;
    g.box = box;
    return g;
}

}  // namespace

// Made once per tree, under the tree's lock: contexts on other threads and streams may search the
// same tree, so the nodes are complete on the device before the pointer is published.
void ensure_snodes(gt_context* ctx, gt_tree* t) {
    if (t->n_nodes <= 0) return;
    std::lock_guard<std::mutex> lk(t->lazy_mu);
    if (t->snode) return;
    SNodeG* p = nullptr;
    check_cuda(cudaMallocAsync((void**)&p, (size_t)t->n_nodes * sizeof(SNodeG), ctx->stream), "cudaMallocAsync");
    pack_snode_kernel<<<grid_of(ctx, t->n_nodes), kBlk, 0, ctx->stream>>>(t->nodes, t->next, t->gc, t->size,
                                                                          t->n_nodes, t->sys_off_dev, t->n_systems, p);
    check_launch(ctx, "pack_snode_kernel");
    check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
    t->snode = p;
}

namespace {
// The context's device tally, zeroed for one call (allocated on first use).
unsigned long long* fresh_tally(gt_context* ctx) {
    if (!ctx->tally_dev) {
        unsigned long long* p = nullptr;
        check_cuda(cudaMalloc((void**)&p, GT_NGB_COUNTERS * sizeof(unsigned long long)), "cudaMalloc");
        ctx->tally_dev = p;
    }
    check_cuda(cudaMemsetAsync(ctx->tally_dev, 0, GT_NGB_COUNTERS * sizeof(unsigned long long), ctx->stream),
               "memset");
    return ctx->tally_dev;
}
}  // namespace

void tree_hmax(gt_context* ctx, gt_tree* t, const double* h, int64_t n_gas) {
    const int64_t nn = std::max<int64_t>(t->n_nodes, 1);
    if (!t->hmax) check_cuda(cudaMallocAsync((void**)&t->hmax, (size_t)nn * 4, ctx->stream), "cudaMallocAsync");
    check_cuda(cudaMemsetAsync(t->hmax, 0, (size_t)nn * 4, ctx->stream), "memset");
    const int64_t n = std::min<int64_t>(n_gas, t->n);
    if (n > 0) {
        hmax_kernel<<<grid_of(ctx, n), kBlk, 0, ctx->stream>>>(h, t->leaf_of, n, t->parent, true, t->hmax);
        check_launch(ctx, "hmax_kernel");
    }
}

void raise_hmax(gt_context* ctx, gt_tree* t, int64_t n, const int* leaf, const double* h) {
    if (!t->hmax || n <= 0) return;  // Tree::raise_hmax is a no-op before init_hmax
    hmax_kernel<<<grid_of(ctx, n), kBlk, 0, ctx->stream>>>(h, leaf, n, t->parent, false, t->hmax);
    check_launch(ctx, "hmax_kernel");
}

int64_t run_ngb(gt_context* ctx, gt_tree* t, int64_t n, const double* cx, const double* cy, const double* cz,
                const double* radius, const int* systems, int mode, const double* h, int64_t n_gas, double box,
                double elapsed, int64_t* start, uint32_t* found, int64_t capacity, int64_t* tally,
                uint32_t** list_out) {
    if (mode != GT_NGB_GATHER && !t->hmax) throw Fail{GT_ERR_INVALID, "the reverse search needs gt_tree_hmax first"};
    cudaStream_t st = ctx->stream;
    NgbArgs a;
    a.g = geom_of(ctx, t, elapsed, box);
    a.cx = cx; a.cy = cy; a.cz = cz; a.radius = radius;
    a.systems = systems;
    a.tally = tally ? fresh_tally(ctx) : nullptr;
    a.n = n;
    a.mode = mode;
    a.h = h;
    a.n_gas = n_gas;
    uint32_t* cnt = (uint32_t*)scratch(ctx, kSlotNgb0, (size_t)std::max<int64_t>(n, 1) * 4);
    uint32_t* ex = (uint32_t*)scratch(ctx, kSlotNgb1, (size_t)std::max<int64_t>(n, 1) * 4);
    unsigned long long* tot = (unsigned long long*)scratch(ctx, kSlotNgb2, 24);
    check_cuda(cudaMemsetAsync(tot, 0, 24, st), "memset");
    a.count = cnt;
    a.total = tot;
    a.start = nullptr;
    a.found = nullptr;
    // the first entries of every centre, kept by the counting pass when the lists are wanted: up
    // to 64 per centre within 2 GiB (none below 8)
    const bool want = (found && capacity > 0) || list_out;
    a.kcache = want ? (int)std::min<int64_t>(64, ((int64_t)1 << 31) / (4 * std::max<int64_t>(n, 1))) : 0;
    if (a.kcache < 8) a.kcache = 0;
    a.cache = a.kcache ? (uint32_t*)scratch(ctx, kSlotNgb3, (size_t)n * a.kcache * 4) : nullptr;
    if (a.tally) ngb_kernel<false, true><<<grid_of(ctx, n), kBlk, 0, st>>>(a);
    else ngb_kernel<false, false><<<grid_of(ctx, n), kBlk, 0, st>>>(a);
    check_launch(ctx, "ngb_kernel");
    unsigned long long total[3] = {0, 0, 0};
    check_cuda(cudaMemcpyAsync(ctx->pinned, tot, 24, cudaMemcpyDeviceToHost, st), "d2h");
    if (a.tally)
        check_cuda(cudaMemcpyAsync((char*)ctx->pinned + 64, a.tally, 5 * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check_cuda(cudaStreamSynchronize(st), "sync");
    std::memcpy(total, ctx->pinned, 24);
    if (a.tally) std::memcpy(tally, (char*)ctx->pinned + 64, 5 * 8);
    if (total[1] > 0) throw Fail{GT_ERR_INVALID, "a centre names a system outside [0, n_systems)"};
    if (total[0] >= (1ull << 32)) throw Fail{GT_ERR_OVERFLOW, "more than 2^32 neighbours in one call"};
    scan_exclusive_u32(ctx, cnt, ex, n, nullptr);
    widen_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(ex, cnt, n, start);
    check_launch(ctx, "widen_kernel");
    uint32_t* dst = nullptr;
    if ((int64_t)total[0] <= capacity && total[0] > 0) {
        if (found) dst = found;
        else if (list_out) dst = (uint32_t*)scratch(ctx, kSlotOut1, (size_t)total[0] * 4);
    }
    if (dst) {
        if (a.kcache) {
            ngb_copy_kernel<<<grid_of(ctx, n), kBlk, 0, st>>>(a.cache, a.kcache, cnt, start, n, dst);
            check_launch(ctx, "ngb_copy_kernel");
        }
        if (!a.kcache || total[2] > 0) {  // the centres the cache did not hold whole
            a.start = start;
            a.found = dst;
            a.tally = nullptr;
            ngb_kernel<true, false><<<grid_of(ctx, n), kBlk, 0, st>>>(a);
            check_launch(ctx, "ngb_kernel");
        }
    }
    if (list_out) *list_out = dst;
    return (int64_t)total[0];
}

// The default h of a particle set: des_ngb particles at the mean number density of its bounding
// box (lo, hi) over n particles (hydro.cc:169-183).
double default_h(const double* lo, const double* hi, double n, double des_ngb, int n_dims) {
    const double vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
    double hd = std::cbrt(3.0 * des_ngb * vol / (4.0 * M_PI * n));
    if (n_dims == 1) hd = 0.5 * des_ngb * (hi[0] - lo[0]) / n;
    if (n_dims == 2) hd = std::sqrt(des_ngb * (hi[0] - lo[0]) * (hi[1] - lo[1]) / (M_PI * n));
    return hd;
}

void run_density(gt_context* ctx, gt_tree* t, int64_t nt, const uint32_t* targets, double des_ngb, double ngb_tol,
                 const double* h_start, double box, int n_dims, const double* cond_prev, int face_corr,
                 double elapsed, double* h, double* rho, int* nngb, int* iters, int64_t* tally) {
    cudaStream_t st = ctx->stream;
    DensArgs a;
    a.g = geom_of(ctx, t, elapsed, box);
    a.smass = t->smass;
    a.stype = t->stype;
    a.rank = t->rank;
    a.targets = targets;
    a.nt = nt;
    a.des_ngb = des_ngb;
    a.ngb_tol = ngb_tol;
    a.h_start = h_start;
    a.cond_prev = cond_prev;
    a.n_dims = n_dims;
    a.face_corr = face_corr;
    a.h = h; a.rho = rho; a.nngb = nngb; a.iters = iters;
    a.tally = tally && nt > 0 ? fresh_tally(ctx) : nullptr;
    a.cand = nullptr;
    a.cand_cap = kCandCap;
    a.n_threads = 0;
    if (!a.tally && nt > 0) {
        a.n_threads = (int64_t)grid_of(ctx, nt) * kBlk;
        a.cand = (uint32_t*)scratch(ctx, kSlotNgb0, (size_t)a.n_threads * kCandCap * sizeof(uint32_t));
    }
    a.h_default = 0.0;
    a.h_default_sys = nullptr;
    if (!h_start && t->n_systems > 1) {
        // each system's own default, from its own particles (all of them, massless too)
        const int S = t->n_systems;
        int64_t nmax = 0;
        for (int s = 0; s < S; ++s) nmax = std::max<int64_t>(nmax, t->in_off[s + 1] - t->in_off[s]);
        const int chunks = (int)std::min<int64_t>(64, std::max<int64_t>(1, (nmax + 8191) / 8192));
        const size_t nparts = (size_t)S * chunks;
        double* part = (double*)scratch(ctx, kSlotNgb2, nparts * 6 * 8);
        density_bbox_kernel<<<(int)nparts, kBlk, 0, st>>>(t->src, t->rank, t->in_off_dev, chunks, part);
        check_launch(ctx, "density_bbox_kernel");
        std::vector<double> hp(nparts * 6), hd(S, 0.0);
        check_cuda(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, st), "d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        for (int s = 0; s < S; ++s) {
            const int64_t ns = t->in_off[s + 1] - t->in_off[s];
            if (ns == 0) continue;  // an empty system owns no target
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int c = 0; c < chunks; ++c)
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], hp[6 * ((size_t)s * chunks + c) + k]);
                    hi[k] = std::max(hi[k], hp[6 * ((size_t)s * chunks + c) + 3 + k]);
                }
            hd[s] = default_h(lo, hi, (double)ns, des_ngb, n_dims);
        }
        double* dhd = (double*)scratch(ctx, kSlotNgb1, (size_t)S * 8);
        check_cuda(cudaMemcpyAsync(dhd, hd.data(), (size_t)S * 8, cudaMemcpyHostToDevice, st), "h2d");
        check_cuda(cudaStreamSynchronize(st), "sync");  // hd is pageable and goes out of scope
        a.h_default_sys = dhd;
    } else if (!h_start) {
        // des_ngb particles at the mean number density of the bounding box of all particles
        const int nb = std::max(1, std::min(grid_of(ctx, t->n), ctx->num_sms * 2));
        double* part = (double*)scratch(ctx, kSlotNgb2, (size_t)nb * 6 * 8);
        bbox_all_kernel<<<nb, kBlk, 0, st>>>(t->src, t->n, part);
        check_launch(ctx, "bbox_all_kernel");
        std::vector<double> hp((size_t)nb * 6);
        check_cuda(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, st), "d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int b = 0; b < nb; ++b)
            for (int k = 0; k < 3; ++k) {
                lo[k] = std::min(lo[k], hp[6 * b + k]);
                hi[k] = std::max(hi[k], hp[6 * b + 3 + k]);
            }
        a.h_default = default_h(lo, hi, (double)t->n, des_ngb, n_dims);
    }
    if (nt <= 0) return;
    const bool one = a.g.n_roots == 1;
    if (a.tally) density_kernel<true, false><<<grid_of(ctx, nt), kBlk, 0, st>>>(a);
    else if (one) density_kernel<false, true><<<grid_of(ctx, nt), kBlk, 0, st>>>(a);
    else density_kernel<false, false><<<grid_of(ctx, nt), kBlk, 0, st>>>(a);
    check_launch(ctx, "density_kernel");
    if (a.tally) {
        check_cuda(cudaMemcpyAsync(ctx->pinned, a.tally, GT_NGB_COUNTERS * 8, cudaMemcpyDeviceToHost, st), "d2h");
        check_cuda(cudaStreamSynchronize(st), "sync");
        std::memcpy(tally, ctx->pinned, GT_NGB_COUNTERS * 8);
    }
}

}  // namespace gt
