/*
 * gt.h — C ABI of the B200-native tree-gravity library (libgt.so).
 *
 * This is the drop-in boundary for GIZMO's shared-memory tree-gravity path.  Each entry point
 * replaces one function of the reference's call surface, shmem/tree.h:359-451 (cited per entry),
 * or the reference's only existing C-ABI, shmem_cuda_accel_bruteforce (shmem/grav_cuda.cu:188-192).
 * The C++ shim in gizmo_shared_memory_b200/shim/ wraps these in the exact shmem:: signatures so
 * shmem/bench_treeforce.cc and shmem/test_tree.cc compile against it unchanged.
 *
 * Conventions
 *  - Plain pointers and sizes only.  `mem` says where every array argument of a call lives:
 *    GT_MEM_HOST (ordinary or pinned host memory; the call copies in and out and returns when the
 *    results are on the host) or GT_MEM_DEVICE (device pointers on the context's device; the call
 *    enqueues on the context's stream and returns when the work is complete unless
 *    gt_walk_options.async is set).
 *  - Every entry point returns a gt_status; nothing calls exit().  A failing call leaves the
 *    context usable and records a message for gt_last_error().
 *  - Outputs are indexed parallel to `targets` and multiplied by G, as in the reference
 *    (shmem/tree.h:389-394).  targets == NULL means "every live particle in tree order", i.e.
 *    targets = orderbuf (what shmem/bench_treeforce.cc:41 passes).
 *  - One context per host thread; one CUDA stream per context.  Trees may be used by any context
 *    on the same device, and walks and searches of one tree may run from several contexts at
 *    once (what a tree builds on first use is made under a lock).  Calls that change a tree
 *    (gt_tree_events, _refresh, _particles, _velocities, _gas, _hmax) must not overlap other calls
 *    on that tree: the caller orders them.
 *  - Options the GPU path does not implement (lazy drift inside the walk, periodic boxes) are
 *    rejected with GT_ERR_UNSUPPORTED; there is no CPU fallback.
 */
#ifndef GT_H
#define GT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GT_VERSION 1

#if defined(__GNUC__)
#define GT_API __attribute__((visibility("default")))
#else
#define GT_API
#endif

typedef enum {
    GT_OK = 0,
    GT_ERR_INVALID = 1,     /* bad argument (null pointer, negative size, unknown option) */
    GT_ERR_CUDA = 2,        /* CUDA runtime error; see gt_last_error() */
    GT_ERR_NOMEM = 3,       /* device allocation failed */
    GT_ERR_UNSUPPORTED = 4, /* option of the reference not implemented on the GPU path */
    GT_ERR_OVERFLOW = 5,    /* a walk stack or list capacity was exceeded and could not be grown */
    GT_ERR_TIMEOUT = 6,     /* a bounded device-side wait gave up */
    GT_ERR_NONFINITE = 7,   /* input validation found a NaN or Inf */
    GT_ERR_DEVICE = 8       /* no usable CUDA device, or the tree belongs to another device */
} gt_status;

enum { GT_MEM_HOST = 0, GT_MEM_DEVICE = 1 };
/* Sort keys.  Both quantise each axis to 20 bits exactly as shmem::build (shmem/tree.cc:409-417),
 * so both give the same cells and the same tree; only the order of children differs. */
enum { GT_KEY_PEANO = 0, GT_KEY_MORTON = 1 };
/* Target grouping of the walk. */
enum {
    GT_GROUP_LEAF = 0,  /* consecutive targets sharing a leaf: accel_grouped batch <= 0 (tree.cc:656-667) */
    GT_GROUP_BATCH = 1, /* fixed windows of `batch` consecutive targets: accel_grouped batch > 0 */
    GT_GROUP_NODE = 2,  /* consecutive targets sharing the deepest ancestor holding <= group_max particles */
    GT_GROUP_SINGLE = 3 /* one walk per target (accel / potential, tree.cc:528, 899) */
};
/* Opening criterion used inside the walk.
 * GT_MAC_LEARNED: the network runs inside the walk for every (group, node) pair in the band.
 * GT_MAC_NODE: the network sees only the node's own features (GT_MAC_NODE_FEATURES; every other
 * feature must have inv_sd = 0 in the model, as gt_mac_train gives with that feature mask), so
 * its correction is evaluated once per node before the walk and the walk itself costs what the
 * plain one does: accept when M L^2 10^c(node) / kappa <= r^4 aold. */
enum { GT_MAC_PLAIN = 0, GT_MAC_LEARNED = 1, GT_MAC_NODE = 2 };
/* Features that depend on the node alone: second moment, COM offset, particle count. */
#define GT_MAC_NODE_FEATURES ((1u << 1) | (1u << 2) | (1u << 5))
/* Precision of gt_direct. */
enum { GT_DIRECT_FP64 = 0, GT_DIRECT_FP32 = 1 };
/* Output order of a walk over targets == NULL. */
enum { GT_OUT_TARGETS = 0, GT_OUT_ORIGINAL = 1 };

typedef struct gt_context gt_context;
typedef struct gt_tree gt_tree;
typedef struct gt_plan gt_plan;

/* Learned multipole-acceptance criterion: an MLP of 8 geometric features, 2 hidden layers of 32
 * (ReLU), one output, FP32.  A model is a flat host array of GT_MAC_MODEL_FLOATS floats:
 * feature mean[8], 1/std[8], W1[32][8], b1[32], W2[32][32], b2[32], W3[32], b3. */
#define GT_MAC_FEATURES 8
#define GT_MAC_HIDDEN 32
#define GT_MAC_MODEL_FLOATS (2 * 8 + 32 * 8 + 32 + 32 * 32 + 32 + 32 + 1)
#define GT_MAC_PARAM_FLOATS (GT_MAC_MODEL_FLOATS - 2 * 8)

typedef struct {
    int key_mode;             /* GT_KEY_PEANO (default) or GT_KEY_MORTON */
    int leaf_max;             /* particles per leaf, default 16 (shmem/tree.h:357) */
    int max_level;            /* deepest level, default 20 (shmem/tree.h:358) */
    long long randomize_seed; /* >= 0: RANDOMIZE_GRAVTREE root shift and doubling (tree.cc:381-393) */
    int nodelta;              /* 1: opening radius = side only (SHMEM_TREE_NODELTA, tree.cc:512-519) */
    int validate;             /* 1: reject non-finite positions/masses/softenings (default 1) */
    double shift[3];          /* SHMEM_TREE_SHIFT fractions of a side (tree.cc:400-407); 0 = none */
} gt_build_options;

typedef struct {
    int group_mode;      /* GT_GROUP_* ; default GT_GROUP_LEAF */
    int group_max;       /* GT_GROUP_NODE: most particles per group node (default 32) */
    int mac;             /* GT_MAC_PLAIN (default) or GT_MAC_LEARNED */
    int out_order;       /* GT_OUT_TARGETS (default) or GT_OUT_ORIGINAL (targets == NULL only) */
    int async;           /* GT_MEM_DEVICE only: 1 = return without synchronising the stream */
    int count;           /* 1 = collect interaction counts (gt_walk_stats); slightly slower */
    int block_warps;     /* warps per block of the walk kernel; 0 = autotuned default */
    int list_capacity;   /* interaction-list entries per warp; 0 = default */
    int stack_capacity;  /* node-stack entries per warp; 0 = default (always sufficient) */
    int dtype_out_f32;   /* reserved, must be 0 */
    /* GT_MAC_LEARNED / GT_MAC_NODE: the model (host array of GT_MAC_MODEL_FLOATS), the acceptance threshold
     * kappa (accept when rho * 10^prediction <= kappa, rho = M L^2 / (r^4 aold)), and the band of
     * rho outside which the network is not consulted: rho <= mac_band[0] accepts, rho >
     * mac_band[1] opens.  The softening-overlap and inside-node arms always apply. */
    const float* mac_model;
    double mac_kappa;
    double mac_band[2];
    /* SINGLE_STAR_DIRECT_GRAVITY_RADIUS: > 0 turns on sink-direct opening in the grouped walks of a
     * tree with particle types (gt_tree_gas): a group holding a sink opens every node the criterion
     * accepted that holds a sink and comes within this radius + 0.6 side of the group's box
     * (accel_grouped's sink_direct_radius, tree.h:435-440, tree.cc:691-698, 772-778).  Default 0. */
    double sink_direct_radius;
    /* Grouped windows of 17-32 targets (GT_GROUP_BATCH) are walked two per warp by default: two
     * consecutive windows share one traversal, each testing exactly its own nodes, so every
     * window gets its own walk's decisions and interactions (sums equal to FP32 rounding, not bit
     * for bit: the list order can differ).  Forests and counting walks included; not for
     * GT_MAC_LEARNED, the tidal tensor, the jerk or the gas rules.  1: one window per warp. */
    int no_window_pairs;
} gt_walk_options;

typedef struct {
    int epochs;      /* passes over the samples (default 30) */
    int batch;       /* samples per step (default 4096) */
    double lr;       /* Adam step size (default 2e-3) */
    double tau;      /* quantile of the pinball loss (default 0.9: a conservative upper quantile) */
    uint64_t seed;   /* initialisation and shuffling (default 1) */
    uint32_t feature_mask; /* features the network may read (bit i = feature i; default all 8).
                              Masked features get mean 0 and inv_sd 0 in the model. */
} gt_mac_train_options;

typedef struct {
    int64_t n;          /* particles passed to gt_build */
    int64_t n_live;     /* particles with m > 0 (the tree's) */
    int64_t n_nodes;
    int32_t n_levels;
    int32_t root;       /* always 0 */
    double center[3];   /* root cell centre */
    double side;        /* root cell side */
    double build_ms[7]; /* bbox, keys, sort, structure, moments, pack, total (device time) */
    int64_t n_systems;  /* 1, or the number of systems of a forest (gt_build_systems) */
} gt_tree_info;

typedef struct {
    int64_t groups, nodes_visited, multipole, pairs, targets;
    int64_t max_stack, list_flushes;
    int64_t traversal_steps; /* warp steps of the traversal (each pops up to 32 nodes) */
    double walk_ms;    /* device time of the walk kernel(s) of the last walk call */
} gt_walk_stats;

/* Node arrays of gt_tree_download, in the reference's conventions (shmem/tree.h:228-247):
 * first/next threading, plo/phi index orderbuf, root = 0.  Any pointer may be null. */
typedef struct {
    double *cx, *cy, *cz, *mass, *size, *delta, *soft, *gcx, *gcy, *gcz;
    int32_t *first, *next, *plo, *phi, *parent, *level;
    double* w_s;   /* WNode::s = size + delta (tree.h:197) */
    float* w_len;  /* WNode::len */
    float* w_soft; /* WNode::soft */
} gt_node_arrays;

/* ---- library / context ------------------------------------------------------------------- */
GT_API int gt_version(void);
GT_API const char* gt_status_string(int status);
GT_API void gt_build_options_default(gt_build_options* opt);
GT_API void gt_walk_options_default(gt_walk_options* opt);

/* Create a context on `device` with its own non-blocking stream.  No reference counterpart: the
 * reference's state lives in process globals (grav_cuda.cu:143-153). */
GT_API int gt_context_create(int device, gt_context** out);
GT_API int gt_context_destroy(gt_context* ctx);
/* Message of the last failed call on this context ("" if none). */
GT_API const char* gt_last_error(const gt_context* ctx);
/* The context's cudaStream_t (as void*), and a way to replace it (the caller keeps ownership). */
GT_API int gt_context_get_stream(gt_context* ctx, void** stream);
GT_API int gt_context_set_stream(gt_context* ctx, void* stream);
GT_API int gt_synchronize(gt_context* ctx);
/* Number of kernels this library launched on the context so far. */
GT_API int gt_launch_count(const gt_context* ctx, uint64_t* count);

/* ---- tree ---------------------------------------------------------------------------------- */
/* Build the tree of n particles.  Replaces shmem::build (shmem/tree.h:384-385, tree.cc:350-526):
 * bbox, 20-bit quantisation, key sort, octree with LEAF_MAX / MAX_LEVEL, monopole moments,
 * next/first threading, rank, leaf_of.  Massless particles (m <= 0) are left out of the tree
 * (tree.cc:355-359).  soft may be null (all zero).  The tree keeps its own device copy of the
 * particles, so the input arrays may be freed after the call. */
GT_API int gt_build(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
             const double* m, const double* soft, int mem, const gt_build_options* opt,
             gt_tree** out);
/* Forest: n_systems independent systems built in one pass.  System s owns the input particles
 * [offsets[s], offsets[s+1]) (host array of n_systems + 1; offsets[0] = 0, offsets[n_systems] = n,
 * non-decreasing).  Each system gets its own root cell and tree exactly as gt_build would give it
 * alone (same keys, order and cells); its root is node s and its live particles are the tree
 * positions gt_tree_systems reports.  Walks on a forest keep every group inside one system and
 * start it at that system's root, so all systems share one persistent walk launch.  No reference
 * counterpart: shmem::build makes one tree per call (tree.cc:350). */
GT_API int gt_build_systems(gt_context* ctx, int64_t n, int32_t n_systems, const int64_t* offsets,
                     const double* x, const double* y, const double* z, const double* m,
                     const double* soft, int mem, const gt_build_options* opt, gt_tree** out);
/* Per-system live tree-position offsets (n_systems + 1) and root cells (4 doubles per system:
 * centre x, y, z, side).  Either pointer may be null. */
GT_API int gt_tree_systems(const gt_tree* tree, int64_t* live_offsets, double* roots);
GT_API int gt_tree_free(gt_tree* tree);
GT_API int gt_tree_info_get(const gt_tree* tree, gt_tree_info* info);
/* Copy the tree to host arrays in the reference's layout: orderbuf (n_live), rank (n; UINT32_MAX
 * for massless particles), leaf_of (n; -1 for massless), nodes (n_nodes each).  Fills the fields
 * of shmem::Tree that the engine and the benches read (tree.h:228-247).  Any pointer may be null. */
GT_API int gt_tree_download(gt_context* ctx, const gt_tree* tree, uint32_t* orderbuf, uint32_t* rank,
                     int32_t* leaf_of, const gt_node_arrays* nodes);
/* Sorted keys (n_live, u64) of the tree: PH or Morton per the build's key_mode. */
GT_API int gt_tree_keys(gt_context* ctx, const gt_tree* tree, uint64_t* keys);
/* Attach particle velocities (indexed like the build's input) to the tree: the per-node
 * centre-of-mass velocity and speed bound of shmem::build with vel and want_vcom
 * (tree.cc:149-190, Tree::vcom and Tree::vmax), which the jerk needs.  particles_only = 1
 * refreshes only the particles' velocities and keeps the node moments of the earlier call, as the
 * reference's jerk reads the current particle velocities but the build-time node velocities
 * (tree.cc:793-797, 862-866). */
GT_API int gt_tree_velocities(gt_context* ctx, gt_tree* tree, const double* vx, const double* vy,
                       const double* vz, int particles_only, int mem);
/* ---- tree reuse between rebuilds (shmem/tree.cc:211-274, tree.h:286-341) -----------------
 * Events of one kind on leaf nodes (the tree's own numbering, e.g. leaf_of of gt_tree_download),
 * applied in array order where the result depends on it:
 *   GT_EVENT_KICK   kick_node(leaf, dp = a[3e..3e+2], tau)         tree.cc:211-226 (no-op without node vcom)
 *   GT_EVENT_SHIFT  shift_node(leaf, m = a[e], dx = x[3e..3e+2])   tree.cc:248-253 (no-op without node vcom)
 *   GT_EVENT_VMAX   raise_vmax(leaf, speed = f[e])                 tree.cc:276-284
 *   GT_EVENT_SOFT   raise_soft(leaf, soft = a[e])                  tree.cc:310-319
 *   GT_EVENT_MASS   mass_event(leaf, dm = a[e], x[3e..], v[3e..], tau, box)  tree.cc:229-246 (serial; no-op without vcom)
 *   GT_EVENT_PAD    raise_pad(leaf, d = a[e])                      tree.cc:322-329 (serial)
 *   GT_EVENT_HMAX   raise_hmax(leaf, h = a[e])                     tree.cc:293-302 (no-op before gt_tree_hmax)
 * Node vcom comes from gt_tree_velocities. */
enum { GT_EVENT_KICK = 0, GT_EVENT_SHIFT = 1, GT_EVENT_VMAX = 2, GT_EVENT_SOFT = 3, GT_EVENT_MASS = 4,
       GT_EVENT_PAD = 5, GT_EVENT_HMAX = 6 };
GT_API int gt_tree_events(gt_context* ctx, gt_tree* tree, int kind, int64_t n, const int32_t* leaf,
                   const double* a, const double* x, const double* v, const float* f, double tau,
                   double box, int mem);
/* refresh_walk_nodes(tau) (tree.cc:256-274): the walk nodes' centre of mass, mass, opening radius
 * and side from the incremental moments (radius and side grow by 2 (vmax tau + xpad)).  Call
 * before a walk on a reused tree. */
GT_API int gt_tree_refresh(gt_context* ctx, gt_tree* tree, double tau);
/* node_com(tau), node_vel and node_mass of every node (tree.h:326-341), with the speed and
 * displacement bounds; host arrays (com, vel: 3 per node), any may be null. */
GT_API int gt_tree_node_state(gt_context* ctx, gt_tree* tree, double tau, double* com, double* vel,
                       double* mass, float* vmax, float* xpad);
/* The particles' current positions, masses and softenings (indexed like the build input; a NULL
 * group keeps its values) for walks on a reused tree: the reference walk reads the particles'
 * current state (tree.cc:786-789), the structure stays the build's. */
GT_API int gt_tree_particles(gt_context* ctx, gt_tree* tree, const double* x, const double* y,
                      const double* z, const double* m, const double* soft, int mem);
/* Gas and sinks.  Attach particle types (GIZMO numbering: 0 gas, 5 sink; NULL = every particle
 * gas) and the adaptive-softening zeta (NULL = none), indexed like the build's input, as
 * shmem::Particles::type and ::zeta (tree.h:38-49); the tree counts the sinks below every node
 * (tree.cc:155-187).  From then on every walk of the tree that returns accelerations applies the
 * zeta terms of gas-gas pairs inside the kernel (pair_force_over_r, tree.cc:39-53) -- the
 * potential, the tidal tensor and the jerk keep the zeta-free pair factor, as the reference's do --
 * and gt_walk_options.sink_direct_radius > 0 turns on sink-direct opening.  Call again to update
 * zeta between steps: the tree keeps the same buffers, so a plan created after the first call
 * sees the new values.  A plan created before the first call does not apply the gas rules. */
GT_API int gt_tree_gas(gt_context* ctx, gt_tree* tree, const uint8_t* type, const double* zeta, int mem);
/* Per-node centre-of-mass velocity (n_nodes each) and speed bound; any pointer may be null. */
GT_API int gt_tree_velocity_moments(gt_context* ctx, const gt_tree* tree, double* vcx, double* vcy,
                             double* vcz, float* vmax);

/* Audit of the tree's invariants on the device: the replacement for shmem::audit_tree
 * (shmem/tree.cc:973-1119).  Checks the structure (particle ranges, children contiguous and
 * partitioning their parent's range, parent, level, side, the reference's next threading, leaf
 * size), re-derives every node's mass and centre of mass from its particles (FP64; mass to 1e-10,
 * centre of mass to 1e-6 of the node's reach), checks every particle lies in each ancestor's cell
 * (plus 1e-6 of the root side and the node's displacement pad) and under its softening, and checks
 * the maps (leaf_of, rank, order) and the live/massless split.  *n_bad receives the number of
 * violations (0: the tree is sound); msg (may be NULL) the first one found.  On a reused tree call
 * it after gt_tree_refresh: the moments compared are the walk nodes'. */
GT_API int gt_tree_audit(gt_context* ctx, const gt_tree* tree, int64_t* n_bad, char* msg, size_t msglen);

/* ---- walks --------------------------------------------------------------------------------- *//* ---- walks --------------------------------------------------------------------------------- */
/* Grouped walk.  Replaces shmem::accel_grouped (shmem/tree.h:428-440, tree.cc:626-897) without
 * the tidal tensor and the jerk (gt_accel_grouped_ext) and without lazy drift; the gas rules and
 * sink-direct opening come from gt_tree_gas and gt_walk_options.sink_direct_radius.  batch <= 0 groups
 * targets by leaf, batch > 0 in fixed windows, unless opt->group_mode overrides it.
 * aold (may be NULL) is ErrTolForceAcc*|a_prev|/G per target (tree.h:389-391); theta > 0 adds the
 * Barnes-Hut test.  phi (may be NULL) receives the potential from the same walk.  Every targets[k]
 * must be < n: the walk checks the indices on the device as it groups them and never reads past
 * the particles; a call that synchronises (host arrays, or gt_walk_options.async = 0) then fails with
 * GT_ERR_INVALID, while an asynchronous call cannot report it and leaves that target's outputs
 * undefined. */
GT_API int gt_accel_grouped(gt_context* ctx, const gt_tree* tree, int64_t n_targets,
                     const uint32_t* targets, const double* aold, double theta, double G, int batch,
                     const gt_walk_options* opt, int mem, double* ax, double* ay, double* az,
                     double* phi);
/* The grouped walk with the tidal tensor and the jerk: shmem::accel_grouped's `tidal` and `jerk`
 * arguments (tree.cc:811-837, 845-880).  tidal (may be NULL) receives 6 values per target in
 * SymTensor3d storage order xx yy zz xy yz xz, NOT multiplied by G (as the reference stores it);
 * jerk (may be NULL) receives 3 values per target, multiplied by G, from the source velocities:
 * particles' own and nodes' centre-of-mass velocities (gt_tree_velocities must have been
 * called).  Plain criterion only; groups hold at most 32 targets (longer windows are split). */
GT_API int gt_accel_grouped_ext(gt_context* ctx, const gt_tree* tree, int64_t n_targets,
                     const uint32_t* targets, const double* aold, double theta, double G, int batch,
                     const gt_walk_options* opt, int mem, double* ax, double* ay, double* az,
                     double* phi, double* tidal, double* jerk);
/* Walk plan: the all-active grouped walk of gt_accel_grouped (targets = NULL) captured once as a
 * CUDA graph and replayed by gt_plan_launch on the context stream, asynchronously.  aold and the
 * outputs are DEVICE arrays whose addresses are fixed at creation (update their contents between
 * launches); the plan owns its stack and counters, so other calls on the context cannot move
 * them.  The tree, the arrays and the context must outlive the plan.  On a forest
 * (gt_build_systems) one replay walks every system in one persistent launch.  opt->count and
 * opt->stack_capacity are not allowed.  No reference counterpart (the engine calls
 * shmem::accel_grouped once per step, mfm.cc:782). */
GT_API int gt_plan_create(gt_context* ctx, const gt_tree* tree, const double* aold, double theta,
                   double G, int batch, const gt_walk_options* opt, double* ax, double* ay,
                   double* az, double* phi, gt_plan** out);
GT_API int gt_plan_launch(gt_plan* plan);
GT_API int gt_plan_destroy(gt_plan* plan);
/* Per-target walk (leaves always direct-summed).  Replaces shmem::accel (tree.h:392-394,
 * tree.cc:528-582). */
GT_API int gt_accel(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
             double theta, double G, const double* aold, int mem, double* ax, double* ay,
             double* az);
/* Per-target potential walk.  Replaces shmem::potential (tree.h:446-447, tree.cc:899-944). */
GT_API int gt_potential(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
                 double theta, double G, const double* aold, int mem, double* phi);
/* Counts and device time of the last walk on this context (SHMEM_COUNT_WALK, tree.cc:671-677). */
GT_API int gt_walk_stats_get(const gt_context* ctx, gt_walk_stats* stats);

/* ---- neighbour search and the density solve (shmem/hydro.h:65-117, hydro.cc:37-327) --------
 * On the gravity tree, through search nodes that hold each node's box (shmem::SNode,
 * tree.h:206-226), made on first use.  Lists are in tree order, which is the reference's order for
 * a tree built with GT_KEY_MORTON.  On a forest (gt_build_systems) a centre searches every system
 * in turn (system 0's tree order first), or the one system gt_ngb_options.systems names for it; a
 * density target searches the system that owns its particle index, with that system's own default
 * h.  Each system then finds exactly what it finds as a tree of its own (particle indices shifted
 * by its offset).  No reference counterpart for forests: shmem::build makes one tree per call. */
enum {
    GT_NGB_GATHER = 0,  /* ngb_search (hydro.cc:37-108): particles with r < radius */
    GT_NGB_REVERSE = 1, /* ngb_search_reverse (hydro.cc:110-148): gas particles j < n_gas with radius <= r < h[j] */
    GT_NGB_PAIRS = 2    /* the gather list followed by the reverse list: every pair with r < max(h_i, h_j) */
};
typedef struct {
    int mode;          /* GT_NGB_* (default GT_NGB_GATHER) */
    double box;        /* periodic box side, minimum-image separations (vec.h:25-31); 0 = open */
    double elapsed;    /* Tree::t_since_build: node boxes widen by vmax * elapsed (and always by xpad) */
    int64_t n_gas;     /* reverse: particles [0, n_gas) are gas */
    const double* h;   /* reverse: support radius of each gas particle (n_gas), located like the other arrays */
    const int32_t* systems; /* per centre, the one system searched (n_centres, in [0, n_systems), located
                            * like the other arrays; GT_ERR_INVALID otherwise); NULL: every system */
} gt_ngb_options;
GT_API void gt_ngb_options_default(gt_ngb_options* opt);
/* Tree::init_hmax (tree.cc:332-338): per node the largest h, rounded up to float, of the gas
 * particles [0, n_gas) below it.  The reverse search needs it; GT_EVENT_HMAX raises it later. */
GT_API int gt_tree_hmax(gt_context* ctx, gt_tree* tree, const double* h, int64_t n_gas, int mem);
/* Neighbour lists of n_centres centres (cx, cy, cz, radius: n_centres each) as CSR: start
 * (n_centres + 1 int64) always; found (particle indices) when it is not NULL and the total fits
 * `capacity`, else GT_ERR_OVERFLOW with start and *total filled (call again with room).  *total
 * (may be NULL) receives the number of entries.  A call with room traverses the tree once: its
 * counting pass keeps each centre's first entries and copies them into place. */
GT_API int gt_ngb_search(gt_context* ctx, const gt_tree* tree, int64_t n_centres, const double* cx,
                  const double* cy, const double* cz, const double* radius, const gt_ngb_options* opt,
                  int mem, int64_t* start, uint32_t* found, int64_t capacity, int64_t* total);
typedef struct {
    double des_ngb;        /* DesNumNgb (default 32) */
    double ngb_tol;        /* tolerance on N_eff (default 0.05, as shmem/bench_density.cc) */
    double box;            /* periodic box side; 0 = open */
    double elapsed;        /* Tree::t_since_build (search prune pad) */
    int n_dims;            /* 1, 2 or 3 (default 3) */
    int face_correction;   /* 1 (default): the face-closure correction; 0: SHMEM_NO_FACECORR */
    const double* h_start; /* per target initial h; NULL: DesNumNgb at the mean density of the box */
    const double* cond_prev; /* per particle condition number of the last evaluation, or NULL */
} gt_density_options;
GT_API void gt_density_options_default(gt_density_options* opt);
/* shmem::density (hydro.cc:150-327): per target, bisection-guarded Newton on the effective
 * neighbour number N_eff(h) = DesNumNgb over GAS neighbours (types of gt_tree_gas; all gas without
 * them), with the face-closure and condition-number corrections.  Outputs per target: the
 * converged support radius h, rho = sum m_j W(r_ij, h), the neighbours inside h and the
 * iterations (100 = not converged).  One thread per target follows the tree in the reference's
 * order, so the sums accumulate in its order.  Any output pointer may be NULL. */
GT_API int gt_density(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
               const gt_density_options* opt, int mem, double* h, double* rho, int32_t* nngb,
               int32_t* iters);
/* SHMEM_NGB_COUNT diagnostics (hydro.cc:7-35, 51-106, 293-296; shmem::ngb_counters and
 * hiter_counters).  While counting is on, this context's gather searches add to its totals:
 *   [0] calls: gather searches, one per centre and per density evaluation;
 *   [1] nodes visited;  [2] particles examined in the leaves opened;  [3] neighbours kept;
 *   [4] nodes admitted only by the vmax * elapsed and xpad pads (elapsed > 0 only);
 *   [5 + i] density targets that took i + 1 iterations (i = 7: 8 or more, the 100 of a solve that
 *   did not converge included).
 * gt_ngb_search counts the centres of the gather and pairs modes once the call has delivered its
 * lists: a count-only call (found NULL) or one that overflows counts nothing, so counting and then
 * filling counts each search once.  gt_density counts every evaluation.  Off by default; the
 * counting variants of the kernels are separate instantiations, so the plain ones are unchanged.
 * gt_ngb_counters_get copies the totals (GT_NGB_COUNTERS int64) and zeroes them when reset is
 * non-zero. */
#define GT_NGB_COUNTERS 13
GT_API int gt_ngb_count(gt_context* ctx, int enable);
GT_API int gt_ngb_counters_get(gt_context* ctx, int64_t* counts, int reset);

/* ---- autotuner ----------------------------------------------------------------------------- */
/* One candidate launch configuration of the all-active grouped walk and what it measured. */
typedef struct {
    int group_mode;     /* GT_GROUP_BATCH, GT_GROUP_NODE or GT_GROUP_LEAF */
    int group_size;     /* window (batch) or group_max (node groups); 0 for leaf groups */
    int block_warps;    /* warps per block */
    int list_capacity;  /* monopole-list entries per warp (the particle list holds half) */
    int mac;            /* GT_MAC_PLAIN or GT_MAC_LEARNED */
    double mac_kappa;   /* learned threshold (GT_MAC_LEARNED) */
    double ms;          /* median device time of the timed walks */
    double p99;         /* sampled p99 relative force error; -1 without a sample */
    double median;      /* sampled median relative force error; -1 without a sample */
    int accepted;       /* p99 <= p99_max (1 without a sample) */
} gt_tune_entry;

typedef struct {
    int reps;                 /* timed walks per candidate (default 3) */
    double p99_max;           /* sampled-error target (default 5e-3) */
    int64_t n_sample;         /* sampled targets; 0 = no error check */
    const uint32_t* sample;   /* host, particle indices of the sample */
    const double* ref_ax;     /* host, FP64 reference accelerations of the sample (gt_direct) */
    const double* ref_ay;
    const double* ref_az;
    const float* mac_model;   /* optional learned criterion to try (host, GT_MAC_MODEL_FLOATS) */
    int n_kappa;              /* thresholds of the learned criterion to try */
    const double* kappa;      /* host, n_kappa */
    double mac_band[2];       /* band of the learned criterion (gt_walk_options.mac_band) */
    int mac_mode;             /* GT_MAC_LEARNED (0 = default) or GT_MAC_NODE */
} gt_tune_options;

GT_API void gt_tune_options_default(gt_tune_options* opt);
/* Pick the launch configuration of the all-active grouped walk of `tree` by measurement: group
 * shape and size (windows 16-128, node groups, leaf groups), then warps per block and interaction-
 * list capacity for the two fastest shapes, then -- when a model is given -- the learned criterion
 * at each kappa on the fastest configuration.  With a sample, a candidate is accepted only if its
 * sampled p99 error is at most p99_max, so the learned criterion replaces the plain one only
 * where it is both accepted and faster; the plain criterion stays the fallback.  `best` receives
 * the fastest accepted candidate as walk options (with *best_batch the window for
 * gt_accel_grouped), or the most accurate one if none is accepted.  aold is in tree order (as the
 * all-active walk takes it).  entries (may be NULL) receive up to max_entries measured candidates.
 * No reference counterpart. */
GT_API int gt_autotune(gt_context* ctx, const gt_tree* tree, const double* aold, int mem, double theta,
                double G, const gt_tune_options* opt, gt_walk_options* best, int* best_batch,
                gt_tune_entry* entries, int max_entries, int* n_entries);

/* aold[i] = alpha * |a_i| / G, the relative-criterion input the engine forms from the previous
 * force (shmem/mfm.cc:743-751). */
GT_API int gt_form_aold(gt_context* ctx, int64_t n, const double* ax, const double* ay, const double* az,
                 double alpha, double G, int mem, double* aold);

/* ---- direct sum ---------------------------------------------------------------------------- */
/* O(n_targets * n) direct summation with the walk's pair rule (kernel of the larger softening,
 * self and r == 0 skipped).  GT_DIRECT_FP64 replaces shmem::accel_brute (tree.h:450-451,
 * tree.cc:946-971); GT_DIRECT_FP32 (FP64 pair offset, FP32 arithmetic) replaces
 * shmem_cuda_accel_bruteforce (grav_cuda.cu:188-247) without zeta terms or periodic wrap.
 * targets index the n sources; phi may be NULL.  Results include the factor G. */
GT_API int gt_direct(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
              const double* m, const double* soft, int64_t n_targets, const uint32_t* targets,
              double G, int precision, int mem, double* ax, double* ay, double* az, double* phi);

/* The FP64 direct sum with the adaptive-softening zeta terms of gas-gas pairs: shmem::accel_brute
 * (tree.h:450-451, tree.cc:946-971) on particles with types and zeta (Particles::type, ::zeta;
 * pair_force_over_r, tree.cc:39-53).  type (0 = gas; NULL = every particle gas) and zeta (NULL =
 * none) are indexed like the particles.  Accelerations only, times G. */
GT_API int gt_direct_gas(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                  const double* m, const double* soft, const uint8_t* type, const double* zeta,
                  int64_t n_targets, const uint32_t* targets, double G, int mem, double* ax, double* ay,
                  double* az);

/* Allocation-free direct sum.  No counterpart in the reference: it exists for callers that cannot
 * allocate device memory at the point of the call -- an application whose pool allocator already
 * owns all free device memory, or one that must not trigger the implicit device-wide
 * synchronisation that cudaMalloc/cudaFree can cause in the middle of an asynchronous step.
 * Same computation as gt_direct, but every array is a device pointer on the current device, no
 * context is used, and the per-chunk partial sums live in one fixed 8 MiB device array inside the
 * library (GT_DIRECT_NOALLOC_SCRATCH_DOUBLES doubles, held on every GPU that loads the library
 * until the process exits).  The call never calls cudaMalloc or cudaFree.  It enqueues its two
 * kernels on `stream` (NULL: the default stream) and returns without synchronising.
 *  - n_targets above GT_DIRECT_NOALLOC_MAX_TARGETS is rejected with GT_ERR_OVERFLOW, before
 *    anything is launched; n == 0 with n_targets > 0 is rejected with GT_ERR_INVALID.
 *  - Every targets[k] must be < n.  The device array is not read on the host, so an index at or
 *    beyond n is not reported: the kernel reads nothing for it and its outputs are zero.
 *  - The first call on a device looks up the array's device address with cudaGetSymbolAddress
 *    (once per device, with that device current); make that first call before any stream capture.
 *    The address is kept for the life of the process: do not call this entry point after
 *    cudaDeviceReset on that device (the reset unloads the module and the kept address is stale).
 *  - Every call shares the one array, which keeps the last call's contents (each call overwrites
 *    every partial it reads, so nothing needs clearing).  Calls that overlap on the GPU -- on
 *    different streams, or from different host threads -- race on it and give wrong results;
 *    serialise them. */
#define GT_DIRECT_NOALLOC_SCRATCH_DOUBLES (1 << 20)
#define GT_DIRECT_NOALLOC_MAX_TARGETS (GT_DIRECT_NOALLOC_SCRATCH_DOUBLES / 4)
GT_API int gt_direct_noalloc(int64_t n, const double* x, const double* y, const double* z,
                             const double* m, const double* soft, int64_t n_targets,
                             const uint32_t* targets, double G, int precision, double* ax,
                             double* ay, double* az, double* phi, void* stream);

/* ---- keys ---------------------------------------------------------------------------------- */
/* Peano-Hilbert (and Morton) keys of the MPI code's domain decomposition: each coordinate mapped
 * to [1,2) as (pos - corner)/len + 1 and its top `bits` mantissa bits taken
 * (domain/domain.cc:2682-2702), then keyed by the table-driven Hilbert curve
 * (system/peano.cc:297-355).  bits <= 42; the 126-bit keys come back as hi/lo halves (any output
 * may be NULL). */
GT_API int gt_peano_keys(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                  const double corner[3], double len, int bits, int mem, uint64_t* ph_hi,
                  uint64_t* ph_lo, uint64_t* morton_hi, uint64_t* morton_lo);

/* ---- learned opening criterion ------------------------------------------------------------- */
/* No reference counterpart: the learned criterion is new.  Training data come from the walk and
 * an exact per-node sum; the network is trained and evaluated by this library's own kernels. */
GT_API void gt_mac_train_options_default(gt_mac_train_options* opt);
/* Walk the tree with the plain relative criterion (aold = alpha * amag, amag = |a| per live
 * particle in tree order) over every `group_stride`-th window of `window` consecutive targets;
 * for each node the walk tests that is not opened by the softening or inside-node arms and whose
 * ratio rho lies in [rho_lo, rho_hi], record its 8 features, rho, and the label
 * log10(worst over the window of |a_monopole - a_exact| / |a_target|) - log10(alpha * rho),
 * the exact value summing the node's particles with the walk's pair rule.  At most `capacity`
 * samples are written; *n_samples receives how many were found (possibly more). */
GT_API int gt_mac_sample(gt_context* ctx, const gt_tree* tree, const double* amag, double alpha,
                         int window, int64_t group_stride, double rho_lo, double rho_hi,
                         int64_t capacity, int mem, float* features, float* labels, float* rho,
                         int64_t* n_samples);
/* The exact-label walk: what a perfect learned criterion could reach.  Walks the windows
 * windows[k] (targets [w * window, min((w + 1) * window, n_live)) in tree order, window <= 32) as
 * the grouped walk does -- nearest point of the window's box, largest target softening, leaves
 * offered to the criterion (shmem/tree.cc:682-779) -- with FP64 sums.  mode 0 accepts by the plain
 * relative criterion M L^2 <= r^4 alpha min|a| (shmem/tree.h:134-135) and reproduces the grouped
 * walk's decisions; mode 1 sums, for every node whose rho = M L^2 / (r^4 alpha min|a|) lies in
 * (rho_lo, rho_hi], the node's particles for every target of the window and accepts the node only
 * if the monopole's worst error over the window, |a_mono - a_exact| / |a_t|, is at most
 * eps * ((c - 1) / 7)^cost_exp, c the interactions opening the node costs one step ahead (its
 * children, or a leaf's particles; c - 1 floored at 1; cost_exp in [0, 4], 0 = a constant
 * threshold).  Below the band it accepts, above it it opens.  Modes 2-5 keep the plain form
 * X / r^4 <= alpha |a| with one ingredient of the exact rule each: 2 = r from the larger of the
 * window box's and its enclosing sphere's distances; 3 = each target's own r_t and |a_t| (the node
 * opens if any target's ratio exceeds alpha); 4 = mode 3 with X = 4 q2 (the node's second mass
 * moment about its centre of mass) in place of M L^2; 5 = mode 0 with X = 4 q2.  amag = |a| per live particle in tree order.
 * Outputs: ax/ay/az (n_windows * window; slot k * window + i is target i of window k, 0 past
 * n_live) and counts (n_windows * 5: node visits, monopole and pair interactions counted as
 * SHMEM_COUNT_WALK counts them, labelled nodes, particles summed for labels).  No reference
 * counterpart: measurement of the learned criterion's ceiling. */
GT_API int gt_mac_ceiling(gt_context* ctx, const gt_tree* tree, const double* amag, double alpha, int window,
                          int64_t n_windows, const int64_t* windows, int mode, double eps, double cost_exp,
                          double rho_lo, double rho_hi, int mem, double* ax, double* ay, double* az,
                          int64_t* counts);
/* Train a model on (features, labels) with the pinball loss at quantile tau, Adam, on the GPU.
 * model (host, GT_MAC_MODEL_FLOATS) receives the trained network; loss the final epoch's mean. */
GT_API int gt_mac_train(gt_context* ctx, int64_t n, const float* features, const float* labels,
                        const gt_mac_train_options* opt, int mem, float* model, double* loss);
/* Network output for n feature rows. */
GT_API int gt_mac_predict(gt_context* ctx, const float* model, int64_t n, const float* features,
                          int mem, float* out);
/* Mean pinball loss at quantile tau and its gradient with respect to the GT_MAC_PARAM_FLOATS
 * trainable parameters (model without the normalisation), for checking the training kernels. */
GT_API int gt_mac_gradient(gt_context* ctx, const float* model, int64_t n, const float* features,
                           const float* labels, double tau, int mem, float* grad, double* loss);

/* ---- measurement --------------------------------------------------------------------------- */
/* FP32 and FP64 FMA throughput of this device's CUDA cores in TFLOP/s (independent FMA chains on
 * every SM), the denominators of the walk's roofline fraction.  No reference counterpart. */
GT_API int gt_measure_peaks(gt_context* ctx, double* fp32_tflops, double* fp64_tflops);

#ifdef __cplusplus
}
#endif
#endif /* GT_H */
