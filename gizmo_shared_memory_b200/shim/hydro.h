// shmem:: neighbour search and density solve on the B200 library.
//
// Same declarations as the reference's shmem/hydro.h (the cubic-spline kernel functions,
// ngb_search, ngb_search_reverse, NeighborCache, DensityResult, density and the diagnostic
// counters), so callers written against that header -- shmem/bench_density.cc -- compile
// unchanged against this directory and link against libshmem_gt.so + libgt.so.  density() runs
// on the GPU (gt_density) for all targets in one launch; the neighbour lists of its cache come from
// one batched search (gt_ngb_search) at the converged h.
//
// Differences a caller can observe:
//   * ngb_search / ngb_search_reverse answer one centre per call, as the reference's do; each
//     call is a device launch.  Batch through gt_ngb_search where the caller can.
//   * The per-centre searches read the particle positions the device holds: those of the build,
//     or, once the tree has seen an event or a refresh, those uploaded by the first search or walk
//     after it.  Lazy drift catches up every particle behind the target first.
//   * ngb_counters / hiter_counters (SHMEM_NGB_COUNT) total every host thread's library context;
//     read them between searches, as the reference's callers do.
#pragma once
#include <cmath>

#include "tree.h"

namespace shmem {

// ---- cubic spline, support radius h, dimension-aware (the reference's kernel conventions) ----
static inline double kernel_norm(double h, int dim) {
    if (dim == 1) return (4.0 / 3.0) / h;
    if (dim == 2) return 40.0 / (7.0 * M_PI * h * h);
    return 8.0 / (M_PI * h * h * h);
}
static inline double ball_vol(double h, int dim) {
    if (dim == 1) return 2.0 * h;
    if (dim == 2) return M_PI * h * h;
    return 4.0 * M_PI / 3.0 * h * h * h;
}
static inline double kernel_w(double r, double h, int dim = 3) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = kernel_norm(h, dim);
    if (q < 0.5) return norm * (1.0 - 6.0 * q * q + 6.0 * q * q * q);
    const double u = 1.0 - q;
    return norm * 2.0 * u * u * u;
}
static inline double kernel_dwdr(double r, double h, int dim = 3) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = kernel_norm(h, dim);
    double fp;
    if (q < 0.5) {
        fp = -12.0 * q + 18.0 * q * q;
    } else {
        const double u = 1.0 - q;
        fp = -6.0 * u * u;
    }
    return norm * fp / h;
}
static inline double kernel_dwdh(double r, double h, int dim = 3) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = kernel_norm(h, dim);
    double f, fp;
    if (q < 0.5) {
        f = 1.0 - 6.0 * q * q + 6.0 * q * q * q;
        fp = -12.0 * q + 18.0 * q * q;
    } else {
        const double u = 1.0 - q;
        f = 2.0 * u * u * u;
        fp = -6.0 * u * u;
    }
    return -((double)dim / h) * norm * f - (q / h) * norm * fp;
}

void ngb_counters(long long& calls, long long& nodes, long long& examined, long long& kept,
                  long long& pad_nodes, bool reset);
void hiter_counters(long long out[8], bool reset);

// All particles within `radius` of `centre`; APPENDS indices to `found`, in tree order.
void ngb_search(const Tree& tree, const Particles& particles, const Vec3d& centre,
                double radius, std::vector<uint32_t>& found, double box = 0.0,
                const LazyDrift* lazy = nullptr);

// Gas particles j < n_gas with h_i <= r < h[j]; APPENDS to `found`.  Needs tree.hmax (init_hmax).
void ngb_search_reverse(const Tree& tree, const Particles& particles, const double* h,
                        size_t n_gas, const Vec3d& centre, double h_i,
                        std::vector<uint32_t>& found, double box = 0.0,
                        const LazyDrift* lazy = nullptr);

struct DensityResult {
    std::vector<double> h;
    std::vector<double> rho;
    std::vector<int> nngb;
    std::vector<int> iters;
};

// Flat CSR of each target's neighbour list at the converged h, indexed by position in the target
// list.
struct NeighborCache {
    std::vector<uint32_t> flat;
    std::vector<size_t> start;
    bool valid = false;

    void clear() { flat.clear(); start.clear(); valid = false; }
};

DensityResult density(const Tree& tree, const Particles& particles,
                      const std::vector<uint32_t>& targets, double des_ngb, double ngb_tol,
                      const std::vector<double>& h_start, double box = 0.0, int n_dims = 3,
                      NeighborCache* cache = nullptr, const LazyDrift* lazy = nullptr,
                      const double* cond_prev = nullptr);

}  // namespace shmem
