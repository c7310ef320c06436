// shmem:: tree surface on the B200 library.
//
// Same declarations as the reference's shmem/tree.h (Particles, WNode, SNode, Tree, build,
// accel, accel_grouped, potential, accel_brute, audit_tree, LEAF_MAX, MAX_LEVEL and the
// scalar kernels), so callers written against that header -- shmem/test_tree.cc,
// shmem/bench_treeforce.cc -- compile unchanged with this directory on the include path and link
// against libshmem_gt.so + libgt.so.  Every force call goes to the GPU through the C ABI of gt.h;
// there is no CPU walk behind these functions.
//
// Differences a caller can observe:
//   * Node numbering is breadth-first (root 0, children contiguous) instead of the reference's
//     depth-first allocation order; first/next threading, plo/phi, parent and leaf_of are
//     consistent with it.
//   * Equal keys keep particle-index order (the reference's parallel sort leaves them unordered).
//   * Options the GPU path does not implement throw std::runtime_error naming the option:
//     build_node and setup_walk (the device build makes the whole tree in one call).
//   * Lazy drift catches up every particle behind the target before the walk (the device walk
//     reads all of them), not only those the walk reaches.
//   * After the first tree event or refresh, each walk uploads the particles' current positions,
//     masses and softenings; types and zeta are uploaded before every walk that has them.
#pragma once
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <numeric>
#include <vector>

#include "vec.h"

struct gt_tree;

namespace shmem {

struct Particles {
    std::vector<double> x, y, z, m, soft;
    std::vector<double> zeta;    // adaptive-softening corrections (gas-gas pairs); empty = none
    std::vector<uint8_t> type;   // GIZMO particle type (0 = gas); empty = all gas
    size_t size() const { return m.size(); }
    Vec3d pos(size_t i) const { return Vec3d{x[i], y[i], z[i]}; }
    bool is_gas(size_t i) const { return type.empty() || type[i] == 0; }
};

// Cubic-spline kernels of GIZMO's kernel_gravity (modes 1, -1, 2, 0).
static inline double spline_force_over_r(double r, double h) {
    const double hi = 1.0 / h, u = r * hi;
    if (u >= 1.0) return 1.0 / (r * r * r);
    const double hi3 = hi * hi * hi;
    if (u < 0.5) return hi3 * (10.666666666666667 + u * u * (32.0 * u - 38.4));
    return hi3 * (21.333333333333332 - 48.0 * u + 38.4 * u * u - 10.666666666666667 * u * u * u -
                  0.06666666666666667 / (u * u * u));
}
static inline double spline_potential(double r, double h) {
    const double hi = 1.0 / h, u = r * hi;
    if (u >= 1.0) return -1.0 / r;
    if (u < 0.5) return hi * (-2.8 + u * u * (5.333333333333333 + u * u * (6.4 * u - 9.6)));
    return hi * (-3.2 + 0.06666666666666667 / u +
                 u * u * (10.666666666666667 + u * (-16.0 + u * (9.6 - 2.1333333333333333 * u))));
}
static inline double grav_tidal_factor(double r, double h) {
    const double hi = 1.0 / h, u = r * hi;
    if (u >= 1.0) return 3.0 / (r * r * r * r * r);
    const double hi5 = hi * hi * hi * hi * hi;
    const double wk = (u < 0.5) ? 76.8 - 96.0 * u : -0.2 / (u * u * u * u * u) + 48.0 / u - 76.8 + 32.0 * u;
    return wk * hi5;
}
static inline double grav_dphi_dh(double r, double h) {
    const double hi = 1.0 / h, u = r * hi;
    if (u >= 1.0) return 0.0;
    const double wk = (u < 0.5) ? 2.8 + 16.0 * u * u * (-1.0 + 3.0 * u * u * (1.0 - 0.8 * u))
                                : 3.2 + 32.0 * u * u * (-1.0 + u * (2.0 - 1.5 * u + 0.4 * u * u));
    return wk * hi * hi;
}
// Opening test: softening overlap, Barnes-Hut (theta_sq > 0), relative criterion (aold > 0; with
// aold == 0 and no theta it opens), inside-node.
static inline bool open_node(double r_sq, double len, double l_open, double node_mass,
                             double node_maxsoft, double soft_target, double aold, double theta_sq,
                             double adx, double ady, double adz) {
    const double gt_ = soft_target + 0.6 * len, gn = node_maxsoft + 0.6 * len;
    if (r_sq < gt_ * gt_ || r_sq < gn * gn) return true;
    if (theta_sq > 0.0 && l_open * l_open >= theta_sq * r_sq) return true;
    if (aold > 0) {
        if (node_mass * len * len > r_sq * r_sq * aold) return true;
    } else if (theta_sq <= 0.0) {
        return true;
    }
    return adx < 0.6 * len && ady < 0.6 * len && adz < 0.6 * len;
}
// Morton key of three 21-bit coordinates (x lowest).
static inline uint64_t spread3(uint64_t v) {
    uint64_t out = 0;
    for (int b = 0; b < 21; ++b) out |= ((v >> b) & 1ull) << (3 * b);
    return out;
}
static inline uint64_t morton(uint32_t a, uint32_t b, uint32_t c) {
    return spread3(a) | (spread3(b) << 1) | (spread3(c) << 2);
}

struct LazyDrift {
    const long long* last = nullptr;
    long long target = 0;
    void (*catch_up)(void*, uint32_t) = nullptr;
    void* ctx = nullptr;
};

struct alignas(64) WNode {
    double cx, cy, cz;
    double s;
    double mass;
    float soft;
    float len;
    int first;
    int next;
    int plo, phi;
};

struct SNode {
    float cx, cy, cz;
    float half;
    int first;
    int next;
    int plo, phi;
};

struct Tree {
    std::vector<double> cx, cy, cz, mass, size, delta, gcx, gcy, gcz, soft;
    std::vector<int> first, next, plo, phi;
    std::vector<uint32_t> orderbuf;
    std::vector<uint32_t> rank;
    std::vector<WNode> wn;
    std::vector<SNode> sn;
    int root = 0;
    int nalloc = 0;
    std::vector<int> parent;
    std::vector<int> leaf_of;
    std::vector<float> vmax, hmax, xpad;
    std::vector<uint32_t> nsink;
    std::vector<double> vcom_x, vcom_y, vcom_z;
    std::vector<double> dp_x, dp_y, dp_z;
    std::vector<double> dq_x, dq_y, dq_z, dmass;
    double t_since_build = 0.0;
    // the device tree behind this host copy (shared by copies of the Tree)
    std::shared_ptr<gt_tree> gpu;
    // tree reuse: events queued for the device tree (shared by copies of the Tree)
    std::shared_ptr<struct ReuseQueue> reuse;

    size_t nnodes() const { return mass.size(); }
    // Incremental moments (tree reuse across steps, tree.cc:211-329).  The events are queued and
    // applied on the device before the next walk, refresh or node query (gt_tree_events); the host
    // copies kept current are vmax (the engine reads vmax[root]) and xpad.  The incremental arrays
    // dp/dq/dmass are allocated like the reference's (their emptiness says whether the build had
    // node velocities) but their values live on the device: read node state through node_mass,
    // node_com and node_vel.  raise_hmax / init_hmax belong to the neighbour search and throw.
    void raise_vmax(int leaf_node, float speed);
    void raise_hmax(int leaf_node, double h);
    void init_hmax(const std::vector<double>& h, size_t n_gas);
    void raise_soft(int leaf_node, double soft);
    void raise_pad(int leaf_node, double d);
    void kick_node(int leaf_node, const Vec3d& dp, double tau);
    void mass_event(int leaf_node, double dm, const Vec3d& x, const Vec3d& v, double tau, double box);
    void shift_node(int leaf_node, double m, const Vec3d& dx);
    double node_mass(int no) const;
    Vec3d node_com(int no, double tau) const;
    void refresh_walk_nodes(double tau);
    Vec3d node_vel(int node_id) const;
};

long long audit_tree(const Tree& T, const Particles& P, const double* h, size_t n_gas,
                     const double* vx, const double* vy, const double* vz, double box,
                     const double* dt_behind, char* msg, size_t msglen);

static const int LEAF_MAX = 16;
static const int MAX_LEVEL = 20;

// The recursive per-node build of the reference has no GPU counterpart (the device build is
// level-synchronous); these throw std::runtime_error.
int build_node(Tree& T, const Particles& P, const std::vector<uint32_t>& order,
               const std::vector<uint64_t>& key, int lo, int hi, int level, double cxi, double cyi,
               double czi, double sz, const double* const* vel = nullptr);
void setup_walk(Tree& T, int node, int next_sibling);

struct BuildTimes { double bbox = 0, keys = 0, sort = 0, recurse = 0, links = 0, pack = 0, total = 0; };

Tree build(const Particles& P, BuildTimes* bt = nullptr, const double* const* vel = nullptr,
           bool want_vcom = false, long long randomize_seed = -1);

void accel(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets, double theta,
           double G, std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az,
           const double* aold = nullptr);

void accel_soa(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
               double theta, double G, std::vector<double>& ax, std::vector<double>& ay,
               std::vector<double>& az);

void accel_grouped(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
                   double theta, double G, int batch, std::vector<double>& ax,
                   std::vector<double>& ay, std::vector<double>& az,
                   std::vector<SymTensor3d>* tidal = nullptr, const double* aold = nullptr,
                   const LazyDrift* lazy = nullptr, std::vector<Vec3d>* jerk = nullptr,
                   const double* const* vel = nullptr, double sink_direct_radius = 0.0);

void potential(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
               double theta, double G, std::vector<double>& phi, const double* aold = nullptr);

void accel_brute(const Particles& P, const std::vector<uint32_t>& targets, double G,
                 std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az);

}  // namespace shmem
