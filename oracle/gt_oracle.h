/* ORACLE — test infrastructure only.
 *
 * CPU restatement (plain C, OpenMP over groups) of the reference's shared-memory tree-gravity path:
 * the shmem build (shmem/tree.cc:350-526), its leaf/batch-grouped walk (shmem/tree.cc:626-897), the
 * per-target walk and potential (shmem/tree.cc:528-582, 899-944), the FP64 direct sum
 * (shmem/tree.cc:946-971) and the key functions (shmem/tree.h:161-173, system/peano.cc:192-355,
 * domain/domain.cc:2693-2702).  Only tests/, bench.py's CPU baseline leg and
 * __graft_entry__.smoke() may load it, and only as the checker.  It is pinned against the
 * reference itself (oracle/_ref, compiled from the reference sources) and against the committed
 * fixtures under tests/golden/.
 */
#ifndef GT_ORACLE_H
#define GT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_tree or_tree;

/* Scalar kernels (shmem/tree.h:59-80) and the opening test (shmem/tree.h:109-144). */
double or_spline_force_over_r(double r, double h);
double or_spline_potential(double r, double h);
double or_spline_tidal_factor(double r, double h); /* shmem/tree.h:85-96 */
int or_open_node(double r_sq, double len, double l_open, double node_mass, double node_maxsoft,
                 double soft_target, double aold, double theta_sq, double adx, double ady, double adz);

/* Keys. */
uint64_t or_morton20(uint32_t a, uint32_t b, uint32_t c);                 /* shmem/tree.h:161-173 */
void or_peano_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo);
void or_morton_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo);
uint64_t or_double_to_int(double d, int bits);                             /* domain.cc:2693-2702 */
/* 20-bit-per-axis keys of every particle exactly as shmem::build quantises (tree.cc:361-418);
 * key_mode 0 = Morton (shmem), 1 = Peano-Hilbert over the same integer cells.  Massless particles
 * get key (1<<60).  geom_out (may be null) receives {cx, cy, cz, side, scale}. */
void or_keys20(int64_t n, const double* x, const double* y, const double* z, const double* m,
               int key_mode, long long randomize_seed, uint64_t* keys, double* geom_out);

/* Tree (Morton order, as shmem::build). */
or_tree* or_build(int64_t n, const double* x, const double* y, const double* z, const double* m,
                  const double* soft, long long randomize_seed, int nodelta);
void or_free(or_tree* t);
int64_t or_nnodes(const or_tree* t);
int64_t or_nlive(const or_tree* t);
int or_root(const or_tree* t);
void or_nodes(const or_tree* t, double* cx, double* cy, double* cz, double* mass, double* size,
              double* delta, double* soft, double* gcx, double* gcy, double* gcz, int* first,
              int* next, int* plo, int* phi, int* parent, int* level, double* w_s, float* w_len,
              float* w_soft);
void or_order(const or_tree* t, uint32_t* orderbuf, uint32_t* rank, int* leaf_of);

/* Grouping.  Leaf groups (batch <= 0, tree.cc:656-667) or fixed windows (batch > 0).  Returns the
 * number of groups; starts must hold nt+1 entries. */
int64_t or_groups(const or_tree* t, int64_t nt, const uint32_t* targets, int batch, int64_t* starts);

/* Walk over explicit groups of `targets` (group g = targets[starts[g] .. starts[g+1])).
 * leaf_accept = 1: leaves are offered to the criterion first (accel_grouped, tree.cc:751-779);
 * leaf_accept = 0: leaves are always direct-summed (accel / potential, tree.cc:554-575).
 * Any of ax/ay/az/phi may be null.  counters (may be null) receives
 * {nodes_visited, multipole, pairs} as SHMEM_COUNT_WALK counts them (tree.cc:671-677, 746, 803, 841). */
void or_walk_groups(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                    const int64_t* starts, double theta, double G, const double* aold,
                    int leaf_accept, double* ax, double* ay, double* az, double* phi,
                    int64_t* counters);
/* Node centre-of-mass velocity and speed bound (tree.cc:149-190); arrays of nnodes. */
void or_velocity_moments(const or_tree* t, const double* vx, const double* vy, const double* vz,
                         double* vcx, double* vcy, double* vcz, float* vmax);
/* Grouped walk with the tidal tensor (6 per target, xx yy zz xy yz xz, not times G) and the jerk
 * (3 per target, times G; needs particle velocities and node vcom); either may be null.
 * tree.cc:811-837, 845-880. */
void or_walk_groups_ext(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                        const int64_t* starts, double theta, double G, const double* aold,
                        const double* vx, const double* vy, const double* vz, const double* vcx,
                        const double* vcy, const double* vcz, double* ax, double* ay, double* az,
                        double* tidal, double* jerk);
/* dW/dr of the 3-D cubic spline at fixed h (shmem/hydro.h:46-54). */
double or_kernel_dwdr(double r, double h);
/* Walk of explicit groups with the adaptive-softening pair rule (zeta terms for gas-gas pairs,
 * tree.cc:39-53) and, with leaf_accept = 1, sink-direct opening within sink_radius
 * (tree.cc:691-698, 772-778).  type (0 = gas, 5 = sink; null = all gas) and zeta (null = 0) are
 * indexed like the build's particles.  leaf_accept = 0 is the per-target accel (tree.cc:528-582). */
void or_walk_groups_gas(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                        const int64_t* starts, double theta, double G, const double* aold,
                        const uint8_t* type, const double* zeta, double sink_radius, int leaf_accept,
                        double* ax, double* ay, double* az);
/* accel_brute with the gas pair rule (tree.cc:946-971, 39-53). */
void or_direct_gas(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   const double* soft, const uint8_t* type, const double* zeta, int64_t nt,
                   const uint32_t* targets, double G, double* ax, double* ay, double* az);
/* Sinks below each node (tree.cc:155-187); nnodes entries. */
void or_node_sinks(const or_tree* t, const uint8_t* type, uint32_t* nsink);
/* Neighbour search (shmem/hydro.cc:37-148) for n centres as CSR, in tree order: mode 0 gather
 * (r < radius), 1 reverse (gas j < n_gas with radius <= r < h[j]), 2 gather then reverse.  start
 * has n+1 entries; found (may be null) receives start[n] entries when cap suffices. */
void or_ngb_search(const or_tree* t, int64_t n, const double* cx, const double* cy, const double* cz,
                   const double* radius, int mode, const double* h, int64_t n_gas, double box, int64_t* start,
                   uint32_t* found, int64_t cap);
/* Tree::init_hmax (tree.cc:332-338); hmax has nnodes entries. */
void or_init_hmax(const or_tree* t, const double* h, int64_t n_gas, float* hmax);
/* density (hydro.cc:150-327).  h_start (per target), cond_prev (per particle) and type (per
 * particle, 0 = gas) may be null. */
void or_density(const or_tree* t, int64_t nt, const uint32_t* targets, double des_ngb, double ngb_tol,
                const double* h_start, double box, int n_dims, const double* cond_prev, const uint8_t* type,
                int face_corr, double* h_out, double* rho_out, int32_t* nngb_out, int32_t* iters_out);
/* Tree reuse: overwrite the walk's node fields (COM, mass, opening radius, side, softening) and
 * re-point the particle positions (the caller keeps the arrays alive). */
void or_set_walk_nodes(or_tree* t, const double* cx, const double* cy, const double* cz, const double* mass,
                       const double* w_s, const float* w_len, const float* w_soft);
void or_set_positions(or_tree* t, const double* x, const double* y, const double* z);
/* accel_grouped (tree.cc:626-897), gravity only. */
void or_accel_grouped(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
                      int batch, const double* aold, double* ax, double* ay, double* az,
                      int64_t* counters);
/* accel (tree.cc:528-582) and potential (tree.cc:899-944): one walk per target. */
void or_accel(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
              const double* aold, double* ax, double* ay, double* az);
void or_potential(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
                  const double* aold, double* phi);
/* accel_brute (tree.cc:946-971): FP64 direct sum over all n particles.  phi may be null. */
void or_direct(int64_t n, const double* x, const double* y, const double* z, const double* m,
               const double* soft, int64_t nt, const uint32_t* targets, double G, double* ax,
               double* ay, double* az, double* phi);

#ifdef __cplusplus
}
#endif
#endif
