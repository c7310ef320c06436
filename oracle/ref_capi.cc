// ORACLE — test infrastructure only; never linked into the product library.
//
// Plain C-ABI wrapper around the reference's own shared-memory tree (shmem/tree.h, shmem/tree.cc)
// and its Peano-Hilbert key functions (system/peano.cc:192-355, domain/domain.cc:2693-2702).
// The reference sources are NOT copied here: oracle/Makefile.ref compiles them where they lie and
// links this file against them into oracle/_ref/libgizmo_ref.so.  Only tests/, bench.py's CPU
// baseline / reference arm and __graft_entry__.smoke() load that library, and only as the checker
// or the timed CPU baseline.
#include "tree.h"

#include <cstdint>
#include <cstring>
#include <omp.h>

using namespace shmem;

// Extracted at build time from system/peano.cc (typedefs supplied by the recipe's prelude).
typedef __int128 peanokey;
typedef unsigned long long peano1D;
peanokey peano_hilbert_key(peano1D x, peano1D y, peano1D z, int bits);
peanokey morton_key(peano1D x, peano1D y, peano1D z, int bits);
peanokey peano_and_morton_key(peano1D x, peano1D y, peano1D z, int bits, peanokey* morton);
// Extracted at build time from domain/domain.cc (BITS_PER_DIMENSION 42).
peano1D domain_double_to_int(double d);

namespace {
struct RefHandle {
    Particles P;
    Tree T;
    std::vector<double> v[3];  // velocities, when the tree was built with them
    const double* vel[3] = {nullptr, nullptr, nullptr};
};
void split128(peanokey k, uint64_t* hi, uint64_t* lo) {
    const unsigned __int128 u = (unsigned __int128)k;
    *hi = (uint64_t)(u >> 64);
    *lo = (uint64_t)u;
}
}  // namespace

static_assert(sizeof(SymTensor3d) == 6 * sizeof(double), "SymTensor3d is six doubles");

extern "C" {

int ref_max_threads() { return omp_get_max_threads(); }
void ref_set_threads(int n) { omp_set_num_threads(n); }

// shmem::build (tree.cc:350-526).  bt_out, when non-null, receives the 7 BuildTimes fields (ms).
void* ref_build(int64_t n, const double* x, const double* y, const double* z, const double* m,
                const double* soft, long long randomize_seed, double* bt_out) {
    RefHandle* h = new RefHandle();
    h->P.x.assign(x, x + n); h->P.y.assign(y, y + n); h->P.z.assign(z, z + n);
    h->P.m.assign(m, m + n);
    if (soft) h->P.soft.assign(soft, soft + n);
    BuildTimes bt;
    h->T = build(h->P, &bt, nullptr, false, randomize_seed);
    if (bt_out) {
        bt_out[0] = bt.bbox; bt_out[1] = bt.keys; bt_out[2] = bt.sort; bt_out[3] = bt.recurse;
        bt_out[4] = bt.links; bt_out[5] = bt.pack; bt_out[6] = bt.total;
    }
    return h;
}

// shmem::build with velocities and want_vcom (tree.cc:350, 149-190): adds the per-node
// centre-of-mass velocity (Tree::vcom) and speed bound (Tree::vmax) the jerk needs.
void* ref_build_vel(int64_t n, const double* x, const double* y, const double* z, const double* m,
                    const double* soft, const double* vx, const double* vy, const double* vz,
                    long long randomize_seed) {
    RefHandle* h = new RefHandle();
    h->P.x.assign(x, x + n); h->P.y.assign(y, y + n); h->P.z.assign(z, z + n);
    h->P.m.assign(m, m + n);
    if (soft) h->P.soft.assign(soft, soft + n);
    h->v[0].assign(vx, vx + n); h->v[1].assign(vy, vy + n); h->v[2].assign(vz, vz + n);
    for (int k = 0; k < 3; ++k) h->vel[k] = h->v[k].data();
    h->T = build(h->P, nullptr, h->vel, true, randomize_seed);
    return h;
}

// shmem::build of particles with types and adaptive-softening zeta (Particles::type, ::zeta,
// tree.h:38-49): the build counts sinks (type 5) per node for sink-direct opening (tree.cc:155-187).
void* ref_build_gas(int64_t n, const double* x, const double* y, const double* z, const double* m,
                    const double* soft, const double* zeta, const uint8_t* type) {
    RefHandle* h = new RefHandle();
    h->P.x.assign(x, x + n); h->P.y.assign(y, y + n); h->P.z.assign(z, z + n);
    h->P.m.assign(m, m + n);
    if (soft) h->P.soft.assign(soft, soft + n);
    if (zeta) h->P.zeta.assign(zeta, zeta + n);
    if (type) h->P.type.assign(type, type + n);
    h->T = build(h->P, nullptr, nullptr, false, -1);
    return h;
}

// shmem::accel_grouped with the gas pair rule (zeta terms for gas-gas pairs, tree.cc:39-53) and
// sink-direct opening within sink_direct_radius (tree.cc:773-778).
void ref_accel_grouped_gas(void* p, int64_t nt, const uint32_t* targets, double theta, double G, int batch,
                           const double* aold, double sink_direct_radius, double* ax, double* ay, double* az) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> vx, vy, vz;
    accel_grouped(h->T, h->P, tg, theta, G, batch, vx, vy, vz, nullptr, aold, nullptr, nullptr, nullptr,
                  sink_direct_radius);
    std::memcpy(ax, vx.data(), nt * 8); std::memcpy(ay, vy.data(), nt * 8);
    std::memcpy(az, vz.data(), nt * 8);
}

void ref_tree_nsink(void* p, uint32_t* nsink) {
    const Tree& T = static_cast<RefHandle*>(p)->T;
    if (!T.nsink.empty()) std::memcpy(nsink, T.nsink.data(), T.nnodes() * 4);
}

// Per-node centre-of-mass velocity and speed bound (nnodes each; any pointer may be null).
void ref_tree_vel(void* p, double* vcx, double* vcy, double* vcz, float* vmax) {
    const Tree& T = static_cast<RefHandle*>(p)->T;
    const size_t nn = T.nnodes();
    if (vcx && !T.vcom_x.empty()) std::memcpy(vcx, T.vcom_x.data(), nn * 8);
    if (vcy && !T.vcom_y.empty()) std::memcpy(vcy, T.vcom_y.data(), nn * 8);
    if (vcz && !T.vcom_z.empty()) std::memcpy(vcz, T.vcom_z.data(), nn * 8);
    if (vmax) std::memcpy(vmax, T.vmax.data(), nn * 4);
}

// shmem::accel_grouped with the tidal tensor (6 per target: xx yy zz xy yz xz, not multiplied by
// G, tree.cc:876-880) and the jerk (3 per target, times G; needs ref_build_vel).  Either output
// may be null.
void ref_accel_grouped_ext(void* p, int64_t nt, const uint32_t* targets, double theta, double G,
                           int batch, const double* aold, double* ax, double* ay, double* az,
                           double* tidal, double* jerk) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> vx, vy, vz;
    std::vector<SymTensor3d> tt;
    std::vector<Vec3d> jj;
    accel_grouped(h->T, h->P, tg, theta, G, batch, vx, vy, vz, tidal ? &tt : nullptr, aold, nullptr,
                  jerk ? &jj : nullptr, jerk ? h->vel : nullptr);
    std::memcpy(ax, vx.data(), nt * 8); std::memcpy(ay, vy.data(), nt * 8);
    std::memcpy(az, vz.data(), nt * 8);
    if (tidal) std::memcpy(tidal, tt.data(), nt * 6 * 8);
    for (int64_t i = 0; jerk && i < nt; ++i)
        for (int k = 0; k < 3; ++k) jerk[3 * i + k] = jj[i][k];
}

// Tree reuse (tree.cc:211-274, tree.h:286-331): the incremental-moment events on leaf nodes of the
// reference's own numbering, then refresh_walk_nodes.  The incremental arrays are allocated the
// way the engine's rebuild does (mfm.cc:1408-1414): dp/dq/dmass sized to the nodes, zeroed.
void ref_reuse_begin(void* p) {
    Tree& T = static_cast<RefHandle*>(p)->T;
    const size_t nn = T.nnodes();
    for (auto* v : {&T.dp_x, &T.dp_y, &T.dp_z, &T.dq_x, &T.dq_y, &T.dq_z, &T.dmass}) v->assign(nn, 0.0);
}
void ref_kick_node(void* p, int leaf, const double* dp, double tau) {
    static_cast<RefHandle*>(p)->T.kick_node(leaf, Vec3d{dp[0], dp[1], dp[2]}, tau);
}
void ref_mass_event(void* p, int leaf, double dm, const double* x, const double* v, double tau, double box) {
    static_cast<RefHandle*>(p)->T.mass_event(leaf, dm, Vec3d{x[0], x[1], x[2]}, Vec3d{v[0], v[1], v[2]}, tau, box);
}
void ref_shift_node(void* p, int leaf, double m, const double* dx) {
    static_cast<RefHandle*>(p)->T.shift_node(leaf, m, Vec3d{dx[0], dx[1], dx[2]});
}
void ref_raise_vmax(void* p, int leaf, float speed) { static_cast<RefHandle*>(p)->T.raise_vmax(leaf, speed); }
void ref_raise_pad(void* p, int leaf, double d) { static_cast<RefHandle*>(p)->T.raise_pad(leaf, d); }
void ref_raise_soft(void* p, int leaf, double s) { static_cast<RefHandle*>(p)->T.raise_soft(leaf, s); }
void ref_refresh_walk_nodes(void* p, double tau) { static_cast<RefHandle*>(p)->T.refresh_walk_nodes(tau); }
// Node state after the events: node_com(tau), node_vel, node_mass, vmax, xpad, and the packed walk
// node's s and len (nnodes each, com/vel 3 per node; any pointer may be null).
void ref_node_state(void* p, double tau, double* com, double* vel, double* mass, float* vmax, float* xpad,
                    double* w_s, float* w_len, float* w_soft) {
    const Tree& T = static_cast<RefHandle*>(p)->T;
    for (size_t i = 0; i < T.nnodes(); ++i) {
        const Vec3d c = T.node_com((int)i, tau);
        if (com) for (int k = 0; k < 3; ++k) com[3 * i + k] = c[k];
        if (vel && !T.vcom_x.empty()) {
            const Vec3d v = T.node_vel((int)i);
            for (int k = 0; k < 3; ++k) vel[3 * i + k] = v[k];
        }
        if (mass) mass[i] = T.node_mass((int)i);
        if (vmax) vmax[i] = T.vmax[i];
        if (xpad) xpad[i] = T.xpad[i];
        if (w_s) w_s[i] = T.wn[i].s;
        if (w_len) w_len[i] = T.wn[i].len;
        if (w_soft) w_soft[i] = T.wn[i].soft;
    }
}
// Replace the particles' positions (the walk reads P.x; a reused tree keeps its structure).
void ref_set_positions(void* p, const double* x, const double* y, const double* z) {
    RefHandle* h = static_cast<RefHandle*>(p);
    const size_t n = h->P.x.size();
    std::memcpy(h->P.x.data(), x, n * 8); std::memcpy(h->P.y.data(), y, n * 8); std::memcpy(h->P.z.data(), z, n * 8);
}

void ref_free(void* p) { delete static_cast<RefHandle*>(p); }

int64_t ref_tree_nnodes(void* p) { return (int64_t)static_cast<RefHandle*>(p)->T.nnodes(); }
int ref_tree_root(void* p) { return static_cast<RefHandle*>(p)->T.root; }
int64_t ref_tree_nlive(void* p) { return (int64_t)static_cast<RefHandle*>(p)->T.orderbuf.size(); }

// Node arrays, each nnodes long (any pointer may be null).
void ref_tree_nodes(void* p, double* cx, double* cy, double* cz, double* mass, double* size,
                    double* delta, double* soft, double* gcx, double* gcy, double* gcz,
                    int* first, int* next, int* plo, int* phi, int* parent,
                    double* w_s, float* w_len, float* w_soft) {
    const Tree& T = static_cast<RefHandle*>(p)->T;
    const size_t nn = T.nnodes();
    auto cpd = [nn](double* dst, const std::vector<double>& src) { if (dst) std::memcpy(dst, src.data(), nn * 8); };
    auto cpi = [nn](int* dst, const std::vector<int>& src) { if (dst) std::memcpy(dst, src.data(), nn * 4); };
    cpd(cx, T.cx); cpd(cy, T.cy); cpd(cz, T.cz); cpd(mass, T.mass); cpd(size, T.size);
    cpd(delta, T.delta); cpd(soft, T.soft); cpd(gcx, T.gcx); cpd(gcy, T.gcy); cpd(gcz, T.gcz);
    cpi(first, T.first); cpi(next, T.next); cpi(plo, T.plo); cpi(phi, T.phi); cpi(parent, T.parent);
    for (size_t i = 0; i < nn; ++i) {
        if (w_s) w_s[i] = T.wn[i].s;
        if (w_len) w_len[i] = T.wn[i].len;
        if (w_soft) w_soft[i] = T.wn[i].soft;
    }
}

// orderbuf (nlive), rank (n), leaf_of (n).
void ref_tree_order(void* p, uint32_t* orderbuf, uint32_t* rank, int* leaf_of) {
    const Tree& T = static_cast<RefHandle*>(p)->T;
    if (orderbuf) std::memcpy(orderbuf, T.orderbuf.data(), T.orderbuf.size() * 4);
    if (rank) std::memcpy(rank, T.rank.data(), T.rank.size() * 4);
    if (leaf_of) std::memcpy(leaf_of, T.leaf_of.data(), T.leaf_of.size() * 4);
}

// shmem::accel_grouped (tree.cc:626-897), gravity only (no tidal/jerk/lazy/sinks).
void ref_accel_grouped(void* p, int64_t nt, const uint32_t* targets, double theta, double G,
                       int batch, const double* aold, double* ax, double* ay, double* az) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> vx, vy, vz;
    accel_grouped(h->T, h->P, tg, theta, G, batch, vx, vy, vz, nullptr, aold);
    std::memcpy(ax, vx.data(), nt * 8); std::memcpy(ay, vy.data(), nt * 8);
    std::memcpy(az, vz.data(), nt * 8);
}

// shmem::accel (tree.cc:528-582): one walk per target, leaves always direct-summed.
void ref_accel(void* p, int64_t nt, const uint32_t* targets, double theta, double G,
               const double* aold, double* ax, double* ay, double* az) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> vx, vy, vz;
    accel(h->T, h->P, tg, theta, G, vx, vy, vz, aold);
    std::memcpy(ax, vx.data(), nt * 8); std::memcpy(ay, vy.data(), nt * 8);
    std::memcpy(az, vz.data(), nt * 8);
}

// shmem::potential (tree.cc:899-944).
void ref_potential(void* p, int64_t nt, const uint32_t* targets, double theta, double G,
                   const double* aold, double* phi) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> out;
    potential(h->T, h->P, tg, theta, G, out, aold);
    std::memcpy(phi, out.data(), nt * 8);
}

// shmem::accel_brute (tree.cc:946-971), FP64 direct sum over every particle of the handle.
void ref_accel_brute(void* p, int64_t nt, const uint32_t* targets, double G,
                     double* ax, double* ay, double* az) {
    RefHandle* h = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> vx, vy, vz;
    accel_brute(h->P, tg, G, vx, vy, vz);
    std::memcpy(ax, vx.data(), nt * 8); std::memcpy(ay, vy.data(), nt * 8);
    std::memcpy(az, vz.data(), nt * 8);
}

// Keys.  morton20: shmem::morton (tree.h:161-173).  The 128-bit keys come back as (hi, lo).
uint64_t ref_morton20(uint32_t a, uint32_t b, uint32_t c) { return morton(a, b, c); }
void ref_peano_hilbert_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo) {
    split128(peano_hilbert_key(x, y, z, bits), hi, lo);
}
void ref_morton_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo) {
    split128(morton_key(x, y, z, bits), hi, lo);
}
void ref_peano_and_morton_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* phi_hi,
                              uint64_t* phi_lo, uint64_t* mo_hi, uint64_t* mo_lo) {
    peanokey mk = 0;
    split128(peano_and_morton_key(x, y, z, bits, &mk), phi_hi, phi_lo);
    split128(mk, mo_hi, mo_lo);
}
uint64_t ref_domain_double_to_int(double d) { return domain_double_to_int(d); }

// Scalar kernels of tree.h, for known-answer checks.
double ref_spline_force_over_r(double r, double h) { return spline_force_over_r(r, h); }
double ref_spline_potential(double r, double h) { return spline_potential(r, h); }
int ref_open_node(double r_sq, double len, double l_open, double node_mass, double node_maxsoft,
                  double soft_target, double aold, double theta_sq, double adx, double ady,
                  double adz) {
    return open_node(r_sq, len, l_open, node_mass, node_maxsoft, soft_target, aold, theta_sq,
                     adx, ady, adz) ? 1 : 0;
}

}  // extern "C"

// ---- neighbour search and the density solve (shmem/hydro.h:65-117, hydro.cc:37-327) --------------
#include "hydro.h"

namespace {
void to_csr(const std::vector<std::vector<uint32_t>>& lists, int64_t* start, uint32_t* found, int64_t cap) {
    int64_t tot = 0;
    start[0] = 0;
    for (size_t c = 0; c < lists.size(); ++c) start[c + 1] = (tot += (int64_t)lists[c].size());
    if (found && tot <= cap)
        for (size_t c = 0; c < lists.size(); ++c)
            if (!lists[c].empty()) std::memcpy(found + start[c], lists[c].data(), lists[c].size() * 4);
}
}  // namespace

extern "C" {

// Tree::t_since_build (the staleness pad of the search prune).
void ref_set_elapsed(void* p, double elapsed) { static_cast<RefHandle*>(p)->T.t_since_build = elapsed; }

// The SHMEM_NGB_COUNT totals (hydro.cc:20-35): calls, nodes, examined, kept, pad nodes, then the
// iteration histogram (8).  Zero unless SHMEM_NGB_COUNT was in the environment at the first search.
void ref_ngb_counters(int64_t* out, int reset) {
    long long c[5], h[8];
    ngb_counters(c[0], c[1], c[2], c[3], c[4], reset != 0);
    hiter_counters(h, reset != 0);
    for (int k = 0; k < 5; ++k) out[k] = c[k];
    for (int k = 0; k < 8; ++k) out[5 + k] = h[k];
}

// Tree::init_hmax (tree.cc:332-338) and a copy of the result (nnodes floats; may be null).
void ref_init_hmax(void* p, const double* h, int64_t n_gas, float* hmax_out) {
    RefHandle* H = static_cast<RefHandle*>(p);
    std::vector<double> hv(h, h + n_gas);
    H->T.init_hmax(hv, (size_t)n_gas);
    if (hmax_out) std::memcpy(hmax_out, H->T.hmax.data(), H->T.nnodes() * 4);
}

// Tree::raise_hmax (tree.cc:293-302) for a list of (leaf, h).
void ref_raise_hmax(void* p, int64_t n, const int* leaf, const double* h) {
    RefHandle* H = static_cast<RefHandle*>(p);
    for (int64_t e = 0; e < n; ++e) H->T.raise_hmax(leaf[e], h[e]);
}

// ngb_search for each centre (hydro.cc:37-108); the lists as CSR (start: n+1, found: start[n]
// entries when cap suffices).  mode 0: gather (r < radius); 1: reverse, ngb_search_reverse
// (hydro.cc:110-148) with h_i = radius and the particles' h (n_gas); 2: both, gather first.
void ref_ngb_search(void* p, int64_t n, const double* cx, const double* cy, const double* cz, const double* radius,
                    int mode, const double* h, int64_t n_gas, double box, int64_t* start, uint32_t* found,
                    int64_t cap) {
    RefHandle* H = static_cast<RefHandle*>(p);
    std::vector<std::vector<uint32_t>> lists((size_t)n);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t c = 0; c < n; ++c) {
        const Vec3d ce{cx[c], cy[c], cz[c]};
        if (mode == 0 || mode == 2) ngb_search(H->T, H->P, ce, radius[c], lists[(size_t)c], box);
        if (mode == 1 || mode == 2) ngb_search_reverse(H->T, H->P, h, (size_t)n_gas, ce, radius[c], lists[(size_t)c], box);
    }
    to_csr(lists, start, found, cap);
}

// density (hydro.cc:150-327) with its neighbour cache as CSR (cache_start may be null).
void ref_density(void* p, int64_t nt, const uint32_t* targets, double des_ngb, double ngb_tol, const double* h_start,
                 double box, int n_dims, const double* cond_prev, double* h, double* rho, int32_t* nngb,
                 int32_t* iters, int64_t* cache_start, uint32_t* cache_flat, int64_t cache_cap) {
    RefHandle* H = static_cast<RefHandle*>(p);
    std::vector<uint32_t> tg(targets, targets + nt);
    std::vector<double> hs;
    if (h_start) hs.assign(h_start, h_start + nt);
    NeighborCache cache;
    DensityResult R = density(H->T, H->P, tg, des_ngb, ngb_tol, hs, box, n_dims, cache_start ? &cache : nullptr,
                              nullptr, cond_prev);
    std::memcpy(h, R.h.data(), nt * 8);
    std::memcpy(rho, R.rho.data(), nt * 8);
    for (int64_t t = 0; t < nt; ++t) { nngb[t] = R.nngb[(size_t)t]; iters[t] = R.iters[(size_t)t]; }
    if (cache_start) {
        for (int64_t t = 0; t <= nt; ++t) cache_start[t] = (int64_t)cache.start[(size_t)t];
        if (cache_flat && (int64_t)cache.flat.size() <= cache_cap)
            std::memcpy(cache_flat, cache.flat.data(), cache.flat.size() * 4);
    }
}

}  // extern "C"
