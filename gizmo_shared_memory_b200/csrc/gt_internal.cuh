// Internal declarations of libgt: device layouts, context/tree structs, launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "gt.h"

namespace gt {

constexpr int kWarp = 32;
constexpr uint64_t kDeadKey = 1ull << 60;  // massless particles sort after every live key

// ---------------------------------------------------------------------------------------------
// Device layouts
// ---------------------------------------------------------------------------------------------

// Walk node, 64 bytes = two 32-byte sectors, read with four 16-byte loads.  Holds what the
// opening test and a monopole interaction need (the reference's WNode, shmem/tree.h:195-204)
// plus the BFS child range: children of a node are contiguous, first .. first+nchild-1.
struct alignas(16) GNode {
    double cx, cy;      // centre of mass
    double cz, mass;
    double s;           // size + delta: conservative opening radius (size only with nodelta)
    float len;          // side length (float, as WNode::len)
    float soft;         // max softening in the node (float, as WNode::soft)
    int first;          // first child, -1 for a leaf
    int nchild;         // number of children (0 for a leaf)
    int plo, phi;       // particle range in tree order
};
static_assert(sizeof(GNode) == 64, "GNode must be one 64-byte record");

// Source particle in tree order, 32 bytes: FP64 position (offsets are formed in FP64), FP32 mass
// and softening (the interaction arithmetic is FP32).
struct alignas(16) SrcP {
    double x, y;
    double z;
    float m, soft;
};
static_assert(sizeof(SrcP) == 32, "SrcP must be 32 bytes");

// Search node of the neighbour search, 32 bytes: float geometric centre and conservative half side
// (the reference's SNode, shmem/tree.h:206-226), first child / next in the reference's threading,
// particle range.
struct alignas(16) SNodeG {
    float cx, cy, cz, half;
    int first, next, plo, phi;
};
static_assert(sizeof(SNodeG) == 32, "SNodeG must be 32 bytes");

// Root cell geometry computed on the device (bbox -> centre, side, scale).
struct RootGeom {
    double cx, cy, cz, side, scale;
    double corner_x, corner_y, corner_z;
    long long n_live;
};

// System of an index in a forest: the last s with off[s] <= i (off has n_systems + 1 entries,
// non-decreasing; empty systems are skipped because off[s] == off[s+1]).
template <typename T>
__device__ __forceinline__ int system_of(const T* __restrict__ off, int n_systems, int64_t i) {
    int lo = 0, hi = n_systems;  // invariant: off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((int64_t)off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------------------------
// Host-side structs behind the opaque C handles
// ---------------------------------------------------------------------------------------------

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace gt

struct gt_context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    uint64_t launches = 0;
    gt_walk_stats stats{};
    std::vector<gt::DevBuf> scratch;  // grow-only workspace slots, indexed by gt::Slot
    void* pinned = nullptr;           // small pinned host buffer for scalar read-backs (4096 B)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host copies overlapped with the main stream's work (made on first use): a walk split into
    // chunks uploads each chunk's aold and copies its results back there; a build from host
    // arrays uploads the softenings there while the bounding box, keys and sort run
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t chunk_ev[8] = {};
    cudaEvent_t up_ev[8] = {};
    cudaEvent_t down_ev[8] = {};      // a chunk's results are in the pinned staging buffer
    // pinned staging for pageable host outputs of a chunked walk (grow-only, made on first use):
    // a copy to pageable memory blocks the host thread until it is done, which would serialise
    // the chunks with their copies
    void* stage = nullptr;
    size_t stage_bytes = 0;
    cudaEvent_t copy_done = nullptr;
    cudaEvent_t main_ev = nullptr;
    // second compute stream: the chunks of a chunked walk alternate between it and `stream`
    cudaStream_t walk2 = nullptr;
    cudaEvent_t walk2_start = nullptr, walk2_done = nullptr;
    // SHMEM_NGB_COUNT (gt_ngb_count): while ngb_count is set, a counted call tallies on the
    // device into tally_dev (GT_NGB_COUNTERS, made on first use, zeroed per call) and adds the
    // tally to the host totals ngb_totals once the call has delivered its results
    bool ngb_count = false;
    unsigned long long* tally_dev = nullptr;
    int64_t ngb_totals[GT_NGB_COUNTERS] = {};
};

struct gt_tree {
    int device = 0;
    int64_t n = 0, n_live = 0, n_nodes = 0, node_cap = 0;
    int n_levels = 0;
    gt_build_options opt{};
    gt::RootGeom geom{};           // root cell (of system 0 in a forest)
    // A forest holds n_systems independent trees built in one pass: system s has root node s and
    // the live tree positions [sys_off[s], sys_off[s+1]).
    int n_systems = 1;
    std::vector<gt::RootGeom> sys_geom;  // per-system root cells
    std::vector<int64_t> sys_off;        // n_systems + 1
    int* sys_off_dev = nullptr;          // device copy (int32), n_systems + 1
    // forest: device copy of the input offsets (n_systems + 1): system s owns the particle indices
    // [in_off_dev[s], in_off_dev[s+1]), massless ones included (null for one system)
    int64_t* in_off_dev = nullptr;
    std::vector<int64_t> in_off;         // host copy (forest only)
    gt::RootGeom* geom_dev = nullptr;    // device copy of sys_geom
    std::vector<int64_t> lvl_off;  // node index range of each level: [lvl_off[L], lvl_off[L+1])
    double build_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    // device arrays (owned)
    gt::SrcP* src = nullptr;     // n (live first, in tree order; massless after)
    double* ssoft = nullptr;     // n, FP64 softening in tree order (targets' opening inputs)
    double* smass = nullptr;     // n, FP64 mass in tree order
    uint32_t* order = nullptr;   // n, tree position -> particle index
    uint32_t* rank = nullptr;    // n, particle index -> tree position (UINT32_MAX: massless)
    int* leaf_of = nullptr;      // n, particle index -> leaf (-1: massless)
    int* sleaf = nullptr;        // n, tree position -> leaf (-1: massless)
    uint64_t* skey = nullptr;    // n, sorted keys
    gt::GNode* nodes = nullptr;  // node_cap
    int* parent = nullptr;       // node_cap
    int* next = nullptr;         // node_cap, reference threading (shmem/tree.cc:340-348)
    int* level = nullptr;        // node_cap
    double* size = nullptr;      // node_cap
    double* delta = nullptr;     // node_cap
    double* nsoft = nullptr;     // node_cap, FP64 max softening
    float* nq2 = nullptr;        // node_cap, second mass moment about the COM (learned criterion)
    double* gc = nullptr;        // node_cap * 3, geometric centres
    // velocities (gt_tree_velocities): per particle in tree order, per-node centre-of-mass
    // velocity (FP64 for download, float4 for the walk's jerk) and speed bound
    float4* svel = nullptr;      // n_live
    float4* nvel = nullptr;      // n_nodes
    double* vcom = nullptr;      // 3 * n_nodes
    float* vmax = nullptr;       // n_nodes
    // tree reuse (gt_tree_refresh and the event calls): build-time node mass and centre of mass,
    // mass / momentum / first-moment changes since the build, non-ballistic displacement pads
    double* m0 = nullptr;        // n_nodes
    double* c0 = nullptr;        // 3 * n_nodes
    double* dp = nullptr;        // 3 * n_nodes
    double* dq = nullptr;        // 3 * n_nodes
    double* dmass = nullptr;     // n_nodes
    float* xpad = nullptr;       // n_nodes
    // gas and sinks (gt_tree_gas): particle type (GIZMO numbering) and adaptive-softening zeta in
    // tree order, sinks (type 5) below each node; gas_zeta: zeta was given (the pair rule applies)
    uint8_t* stype = nullptr;    // n
    double* szeta = nullptr;     // n
    uint32_t* nsink = nullptr;   // n_nodes
    bool gas_zeta = false;
    // neighbour search (gt_ngb_search, gt_density): search nodes made on first use, and the
    // per-node largest gas support radius of the reverse search (gt_tree_hmax)
    gt::SNodeG* snode = nullptr; // n_nodes
    float* hmax = nullptr;       // n_nodes
    // cached all-active group lists, keyed by (mode, param)
    struct GroupCache {
        int mode = -1, param = 0, kmax = 0;
        int2* groups = nullptr;
        int* roots = nullptr;  // forest: root node of each group
        int64_t n_groups = 0;
        bool pooled = false;   // groups came from the stream-ordered pool (cudaMallocAsync)
    };
    std::vector<GroupCache> group_cache;
    // guards the state made on first use (the group cache, the search nodes): trees may be used by
    // contexts on several threads
    std::mutex lazy_mu;
};

namespace gt {

// Byte offset in gt_context::pinned of the out-of-range-target flag a walk reads back; the other
// read-backs use the start of the buffer.
constexpr size_t kPinnedTargetCheck = 4000;

// Scratch slots of the context workspace.
enum Slot {
    kSlotIn0 = 0, kSlotIn1, kSlotIn2, kSlotIn3, kSlotIn4,  // staged host inputs
    kSlotKeysA, kSlotKeysB, kSlotValsA, kSlotValsB,
    kSlotHist, kSlotScanA, kSlotScanB, kSlotPartials,
    kSlotNodeTmp0, kSlotNodeTmp1, kSlotNodeTmp2,
    kSlotTargets, kSlotAold, kSlotGroupKey, kSlotGroupsA, kSlotGroupsB,
    kSlotOut0, kSlotOut1, kSlotOut2, kSlotOut3, kSlotOut4, kSlotOut5,
    kSlotStack, kSlotCounters, kSlotDirect, kSlotGroupRoot, kSlotMacL2,
    kSlotNgb0, kSlotNgb1, kSlotNgb2, kSlotNgb3,
    kSlotStack2,  // traversal stacks of the second compute stream (chunked walks)
    kSlotGroupCount,  // device-side group and chunk counts of an explicit-target walk
    kSlotLevels,      // device-side level offsets and counts of the build's structure stage
    kSlotIn5,         // a sixth staged input (the neighbour search's per-centre systems)
    kSlotCount
};

// Error plumbing: every entry point funnels CUDA failures into a gt_status and a message.
struct Fail {
    int status;
    std::string msg;
};

void set_error(gt_context* ctx, int status, const std::string& msg);
void* scratch(gt_context* ctx, Slot s, size_t bytes);  // throws Fail on allocation failure
void check_cuda(cudaError_t e, const char* what);       // throws Fail
void check_launch(gt_context* ctx, const char* what);   // counts the launch, throws on error

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Device-wide helpers (gt_scan.cu).
// Exclusive scan of n uint32 values into out (may alias in); returns nothing, total written to
// total_dev[0] when total_dev is non-null.
// n_dev (optional): the number of items, on the device, at most n; the launch is sized by n, so
// the host needs no read-back of the count.
void scan_exclusive_u32(gt_context* ctx, const uint32_t* in, uint32_t* out, int64_t n,
                        uint32_t* total_dev, const int64_t* n_dev = nullptr);
// Stable LSD radix sort of (key, value) pairs over the low `bits` bits of the key.
void radix_sort_pairs(gt_context* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int bits);

// Build (gt_build.cu)
// n_systems > 1 builds a forest: particles of system s are the input range [in_off[s], in_off[s+1])
// (host array of n_systems + 1), each system gets its own root cell and tree.
// soft_ready (may be null): an event that the softenings' upload records; the build reads them
// first in the gather stage and waits for it there, and it then checks them for non-finite values
// in that stage instead of in the bounding-box pass.
void build_tree(gt_context* ctx, gt_tree* t, const double* x, const double* y, const double* z,
                const double* m, const double* soft, int n_systems = 1, const int64_t* in_off = nullptr,
                cudaEvent_t soft_ready = nullptr);
// The context's second stream (and its events), made on first use: host copies that overlap work
// on the main stream.
void ensure_copy_stream(gt_context* ctx);
// The context's pinned staging buffer of at least `bytes` (grow-only; throws Fail).
void* host_stage(gt_context* ctx, size_t bytes);

// Walk (gt_walk.cu)
// Stack and counters owned by a walk plan (a captured graph must not point into the workspace).
struct WalkBuffers {
    int* stack = nullptr;
    size_t stack_bytes = 0;
    unsigned long long* ctr = nullptr;
    size_t ctr_bytes = 0;
    float* model = nullptr;  // device copy of the learned criterion's network
    float* mac_l2 = nullptr; // GT_MAC_NODE per-node scale
    size_t mac_l2_bytes = 0;
};
struct WalkRequest {
    const uint32_t* targets = nullptr;  // device, original indices; null = all live in tree order
    int64_t n_targets = 0;
    const double* aold = nullptr;       // device, parallel to targets
    double theta = 0, G = 1;
    int group_mode = GT_GROUP_LEAF;
    int group_param = 0;                // batch or group_max
    bool leaf_accept = true;
    bool want_acc = true, want_phi = false;
    bool out_original = false;
    int mac = GT_MAC_PLAIN;
    const float* mac_model = nullptr;   // device copy of the network (GT_MAC_LEARNED)
    double mac_kappa = 1.0, mac_band_lo = 0.0, mac_band_hi = 0.0;
    bool count = false;
    int block_warps = 0, list_capacity = 0, stack_capacity = 0;
    bool pair_windows = true;     // windows of 17-32 targets: two per warp (walk_pair_kernel)
    WalkBuffers* bufs = nullptr;  // plan-owned buffers; null: the context workspace
    bool capture = false;         // being captured into a graph: no events, no read-back
    double *ax = nullptr, *ay = nullptr, *az = nullptr, *phi = nullptr;  // device outputs
    double* tidal = nullptr;  // 6 per target (xx yy zz xy yz xz), not times G
    double* jerk = nullptr;   // 3 per target, times G
    double sink_radius = 0;   // > 0: sink-direct opening (grouped walks of a tree with types)
    // host destinations of the outputs (indexed like the device outputs): the walk copies each
    // chunk's results while the next chunk runs; null: the caller copies
    struct HostOut {
        double *ax = nullptr, *ay = nullptr, *az = nullptr, *phi = nullptr, *tidal = nullptr, *jerk = nullptr;
        bool any() const { return ax || ay || az || phi || tidal || jerk; }
    } host;
    // host source of aold not yet copied into the device buffer `aold`: the walk uploads it, per
    // chunk ahead of each chunk when it splits the groups, else whole before its first kernel
    const double* host_aold = nullptr;
};
// true when the walk copied the outputs to rq.host itself (chunked, overlapped with the walk)
bool run_walk(gt_context* ctx, const gt_tree* t, const WalkRequest& rq);

// Autotuner (gt_tune.cu); aold and mac_model are device pointers, the sample arrays host ones
// except `sample`, which is copied to the device by the tuner.
struct TuneRequest {
    int reps = 3;
    double p99_max = 5e-3;
    int64_t n_sample = 0;
    const uint32_t* sample = nullptr;
    const double *ref_ax = nullptr, *ref_ay = nullptr, *ref_az = nullptr;
    const float* mac_model = nullptr;
    std::vector<double> kappa;
    double mac_band[2] = {0, 0};
    int mac_mode = GT_MAC_LEARNED;
};
void run_autotune(gt_context* ctx, const gt_tree* t, const double* aold, double theta, double G,
                  const TuneRequest& tr, std::vector<gt_tune_entry>& entries, gt_tune_entry& best);

// Direct sum (gt_direct.cu)
void run_direct(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                const double* m, const double* soft, int64_t nt, const uint32_t* targets, double G,
                int precision, double* ax, double* ay, double* az, double* phi);

// The FP64 direct sum with the zeta terms of gas-gas pairs; type / zeta may be null.
void run_direct_gas(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z, const double* m,
                    const double* soft, const uint8_t* type, const double* zeta, int64_t nt, const uint32_t* targets,
                    double G, double* ax, double* ay, double* az);

// Keys (gt_build.cu)
void run_peano_keys(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                    const double corner[3], double len, int bits, uint64_t* ph_hi, uint64_t* ph_lo,
                    uint64_t* mo_hi, uint64_t* mo_lo);
// Learned criterion (gt_mac.cu); all arrays are device pointers.
void run_mac_sample(gt_context* ctx, const gt_tree* t, const double* amag, double alpha, int window,
                    int64_t stride, double rho_lo, double rho_hi, int64_t cap, float* feat,
                    float* label, float* rho, int64_t* n_samples);
void run_tree_audit(gt_context* ctx, const gt_tree* t, int64_t* n_bad, char* msg, size_t msglen);
void run_mac_ceiling(gt_context* ctx, const gt_tree* t, const double* amag, double alpha, int window,
                     int64_t n_win, const int64_t* wins, int mode, double eps, double cost_exp, double rho_lo,
                     double rho_hi, double* ax, double* ay, double* az, unsigned long long* counts);
void run_mac_train(gt_context* ctx, int64_t n, const float* X, const float* Y,
                   const gt_mac_train_options& o, float* model_host, double* loss);
void run_mac_grad(gt_context* ctx, const float* dmodel, const float* X, const float* Y, const int* perm,
                  int64_t off, int B, double tau, float* dgrad, double* loss);
void run_mac_predict(gt_context* ctx, const float* dmodel, int64_t n, const float* X, float* out);
// GT_MAC_NODE: per-node l2 = len^2 10^(c - log10 kappa) (n_nodes floats).
void run_mac_node_scale(gt_context* ctx, const gt_tree* t, const float* dmodel, double kappa, float* l2);

// Peak probe (gt_peak.cu)
void run_peaks(gt_context* ctx, double* fp32_tflops, double* fp64_tflops);
// Tree reuse (gt_reuse.cu).  Event kinds, applied to leaf nodes (device arrays): kick (a = dp, 3
// per event, at tau), shift (a = m, x = dx 3 per event), speed bound (f), softening bound (a),
// mass event (a = dm, x, v 3 per event, at tau, box), displacement pad (a = d).
enum { kReuseKick = 0, kReuseShift, kReuseVmax, kReuseSoft, kReuseMass, kReusePad };
void reuse_begin(gt_context* ctx, gt_tree* t);
void reuse_events(gt_context* ctx, gt_tree* t, int kind, int64_t n, const int* leaf, const double* a,
                  const double* x, const double* v, const float* f, double tau, double box);
void reuse_refresh(gt_context* ctx, gt_tree* t, double tau);
void reuse_node_state(gt_context* ctx, gt_tree* t, double tau, double* com, double* vel, double* mass);
void tree_particles(gt_context* ctx, gt_tree* t, const double* x, const double* y, const double* z,
                    const double* m, const double* soft);
// Per-particle velocities in tree order and the per-node centre-of-mass velocity and speed bound
// (gt_tree_velocities); vx, vy, vz are device arrays over the tree's input particles.
void tree_velocities(gt_context* ctx, gt_tree* t, const double* vx, const double* vy, const double* vz,
                     bool particles_only = false);
// Particle types (null: every particle gas) and zeta (null: none), device arrays over the tree's
// input particles, gathered into tree order; the per-node sink count (gt_tree_gas).
void tree_gas(gt_context* ctx, gt_tree* t, const uint8_t* type, const double* zeta);
// Neighbour search and the density solve (gt_ngb.cu); array arguments are device pointers.
void ensure_snodes(gt_context* ctx, gt_tree* t);
void tree_hmax(gt_context* ctx, gt_tree* t, const double* h, int64_t n_gas);
void raise_hmax(gt_context* ctx, gt_tree* t, int64_t n, const int* leaf, const double* h);
// Counts into start (n+1, exclusive prefix sums) and, when found is given and the total fits
// capacity, the lists; returns the total.
// systems: per centre, the one system searched (null: every system).  tally (host, 5 values, or
// null): the SHMEM_NGB_COUNT tally of the gather searches of the counting pass.  list_out (with
// found null): when the lists fit capacity, they are made in a workspace buffer whose device
// pointer is returned there (null otherwise).
int64_t run_ngb(gt_context* ctx, gt_tree* t, int64_t n, const double* cx, const double* cy, const double* cz,
                const double* radius, const int* systems, int mode, const double* h, int64_t n_gas, double box,
                double elapsed, int64_t* start, uint32_t* found, int64_t capacity, int64_t* tally,
                uint32_t** list_out = nullptr);
// tally (host, GT_NGB_COUNTERS values, or null): the solve's SHMEM_NGB_COUNT tally (synchronises).
void run_density(gt_context* ctx, gt_tree* t, int64_t nt, const uint32_t* targets, double des_ngb, double ngb_tol,
                 const double* h_start, double box, int n_dims, const double* cond_prev, int face_corr,
                 double elapsed, double* h, double* rho, int* nngb, int* iters, int64_t* tally);
void run_form_aold(gt_context* ctx, int64_t n, const double* ax, const double* ay,
                   const double* az, double alpha, double G, double* aold);

}  // namespace gt

// A captured all-active walk (gt_plan_create): the graph and the buffers it points at.
struct gt_plan {
    gt_context* ctx = nullptr;
    const gt_tree* tree = nullptr;
    gt::WalkBuffers bufs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;  // kernel launches one replay makes
};
