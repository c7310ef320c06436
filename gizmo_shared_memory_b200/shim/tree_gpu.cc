// shmem:: tree functions implemented on libgt (include/gt.h).  See tree.h in this directory for
// the differences a caller can observe.
#include "tree.h"
#include "hydro.h"

#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "gt.h"

namespace shmem {
namespace {

// SHMEM_NGB_COUNT (hydro.cc:24-27): every context counts its searches from creation.
bool ngb_counting() {
    static const bool v = getenv("SHMEM_NGB_COUNT") != nullptr;
    return v;
}

// Every context of the process, for the process-wide counter totals the reference keeps.
std::mutex g_contexts_mu;
std::vector<gt_context*> g_contexts;

// One library context per host thread, on device $GT_DEVICE (default 0), created on first use.
// It is deliberately never destroyed: a destructor running at thread or process exit could call
// into the CUDA runtime after the runtime has begun its own teardown; process exit releases the
// context's device memory and stream anyway.
gt_context* context() {
    thread_local gt_context* ctx = nullptr;
    if (!ctx) {
        const char* d = getenv("GT_DEVICE");
        gt_context* c = nullptr;
        const int st = gt_context_create(d ? atoi(d) : 0, &c);
        if (st != GT_OK) throw std::runtime_error(std::string("gt_context_create: ") + gt_status_string(st));
        if (ngb_counting() && gt_ngb_count(c, 1) != GT_OK)
            throw std::runtime_error(std::string("gt_ngb_count: ") + gt_last_error(c));
        std::lock_guard<std::mutex> lk(g_contexts_mu);
        g_contexts.push_back(c);
        ctx = c;
    }
    return ctx;
}

void check(int st, const char* what) {
    if (st != GT_OK)
        throw std::runtime_error(std::string(what) + ": " + gt_last_error(context()));
}

[[noreturn]] void unsupported(const char* what) {
    throw std::runtime_error(std::string("shmem (GPU): ") + what + " is not implemented on the GPU path");
}


const double* soft_or_null(const Particles& P) { return P.soft.empty() ? nullptr : P.soft.data(); }

}  // namespace

Tree build(const Particles& P, BuildTimes* bt, const double* const* vel, bool want_vcom,
           long long randomize_seed) {
    if (!vel) want_vcom = false;  // no velocities, no centre-of-mass velocity (tree.cc:352)
    const int64_t n = (int64_t)P.size();
    gt_build_options o;
    gt_build_options_default(&o);
    o.key_mode = GT_KEY_MORTON;  // the reference's child order
    o.randomize_seed = randomize_seed;
    // the reference's build-time switches (shmem/tree.cc:17-20, 400-407)
    o.nodelta = getenv("SHMEM_TREE_NODELTA") != nullptr;
    if (const char* s = getenv("SHMEM_TREE_SHIFT")) {
        double fx = 0, fy = 0, fz = 0;
        if (sscanf(s, "%lf,%lf,%lf", &fx, &fy, &fz) == 3) {
            o.shift[0] = fx; o.shift[1] = fy; o.shift[2] = fz;
        }
    }
    gt_context* ctx = context();
    gt_tree* h = nullptr;
    check(gt_build(ctx, n, P.x.data(), P.y.data(), P.z.data(), P.m.data(), soft_or_null(P),
                   GT_MEM_HOST, &o, &h), "gt_build");
    Tree T;
    T.gpu = std::shared_ptr<gt_tree>(h, [](gt_tree* p) { gt_tree_free(p); });
    gt_tree_info info;
    check(gt_tree_info_get(h, &info), "gt_tree_info_get");
    const size_t nn = (size_t)info.n_nodes, nl = (size_t)info.n_live;
    for (auto* v : {&T.cx, &T.cy, &T.cz, &T.mass, &T.size, &T.delta, &T.gcx, &T.gcy, &T.gcz, &T.soft})
        v->resize(nn);
    for (auto* v : {&T.first, &T.next, &T.plo, &T.phi, &T.parent}) v->resize(nn);
    std::vector<int> level(nn);
    std::vector<double> ws(nn);
    std::vector<float> wlen(nn), wsoft(nn);
    T.orderbuf.resize(nl);
    T.rank.resize((size_t)n);
    T.leaf_of.resize((size_t)n);
    gt_node_arrays na{T.cx.data(), T.cy.data(), T.cz.data(), T.mass.data(), T.size.data(),
                      T.delta.data(), T.soft.data(), T.gcx.data(), T.gcy.data(), T.gcz.data(),
                      T.first.data(), T.next.data(), T.plo.data(), T.phi.data(), T.parent.data(),
                      level.data(), ws.data(), wlen.data(), wsoft.data()};
    check(gt_tree_download(ctx, h, T.orderbuf.data(), T.rank.data(), T.leaf_of.data(), &na),
          "gt_tree_download");
    T.root = 0;
    T.nalloc = (int)nn;
    T.vmax.assign(nn, 0.0f);
    T.xpad.assign(nn, 0.0f);
    T.reuse = std::make_shared<ReuseQueue>();
    if (vel) {
        // per-node speed bound, and with want_vcom the centre-of-mass velocity the jerk reads
        check(gt_tree_velocities(ctx, h, vel[0], vel[1], vel[2], 0, GT_MEM_HOST), "gt_tree_velocities");
        if (want_vcom) {
            T.vcom_x.resize(nn); T.vcom_y.resize(nn); T.vcom_z.resize(nn);
        }
        check(gt_tree_velocity_moments(ctx, h, want_vcom ? T.vcom_x.data() : nullptr,
                                       want_vcom ? T.vcom_y.data() : nullptr,
                                       want_vcom ? T.vcom_z.data() : nullptr, T.vmax.data()),
              "gt_tree_velocity_moments");
        if (want_vcom)  // the reference allocates the incremental arrays with vcom (tree.cc:449-452)
            for (auto* v : {&T.dp_x, &T.dp_y, &T.dp_z, &T.dq_x, &T.dq_y, &T.dq_z, &T.dmass}) v->assign(nn, 0.0);
    }
    if (!P.type.empty()) {
        // sinks (type 5) under each node, for the engine's sink bookkeeping (tree.cc:168, 178)
        T.nsink.assign(nn, 0u);
        for (size_t i = 0; i < (size_t)n; ++i)
            if (P.type[i] == 5)
                for (int no = T.leaf_of[i]; no >= 0; no = T.parent[no]) ++T.nsink[no];
    }
    T.wn.resize(nn);
    for (size_t i = 0; i < nn; ++i) {
        WNode& w = T.wn[i];
        w.cx = T.cx[i]; w.cy = T.cy[i]; w.cz = T.cz[i];
        w.s = ws[i]; w.mass = T.mass[i]; w.soft = wsoft[i]; w.len = wlen[i];
        w.first = T.first[i]; w.next = T.next[i]; w.plo = T.plo[i]; w.phi = T.phi[i];
    }
    // search nodes: geometric centre and half side widened to stay one-sided in float
    const double eps = 1e-6 * (nn ? T.size[0] : 1.0);
    T.sn.resize(nn);
    for (size_t i = 0; i < nn; ++i) {
        SNode& s = T.sn[i];
        s.cx = (float)T.gcx[i]; s.cy = (float)T.gcy[i]; s.cz = (float)T.gcz[i];
        const double cm = std::max(std::fabs(T.gcx[i]), std::max(std::fabs(T.gcy[i]), std::fabs(T.gcz[i])));
        s.half = (float)(0.5 * T.size[i] + eps + 4.0 * FLT_EPSILON * cm);
        s.first = T.first[i]; s.next = T.next[i]; s.plo = T.plo[i]; s.phi = T.phi[i];
    }
    if (bt) {
        bt->bbox = info.build_ms[0]; bt->keys = info.build_ms[1]; bt->sort = info.build_ms[2];
        bt->recurse = info.build_ms[3] + info.build_ms[4]; bt->links = 0; bt->pack = info.build_ms[5];
        bt->total = info.build_ms[6];
    }
    return T;
}

// ---- tree reuse ----------------------------------------------------------------------------
// Events are queued per host thread (the engine feeds kicks and speed bounds from OpenMP loops)
// and applied on the device in one gt_tree_events call per kind.  Kicks, shifts and the speed and
// softening bounds commute, so their per-thread queues merge in any order; mass events and pads
// depend on order and the reference's callers are serial, so they flush the queues and go
// straight to the device.
struct ReuseQueue {
    struct Buf {
        std::vector<int32_t> kick_leaf, vmax_leaf, soft_leaf, shift_leaf, hmax_leaf;
        std::vector<double> kick_dp, soft_val, shift_m, shift_dx, hmax_val;
        std::vector<float> vmax_val;
        double kick_tau = 0.0;
    };
    std::vector<Buf> bufs;
    std::mutex mu;
    bool moved = false;  // events or a refresh since the build: the walk needs current particles
    // the per-centre neighbour search uploads the particles once per change of the tree
    uint64_t gen = 0, search_gen = 0;
    std::mutex search_mu;
    ReuseQueue() : bufs((size_t)std::max(1, omp_get_max_threads())) {}
    Buf& mine() {
        const size_t t = (size_t)omp_get_thread_num();
        if (t >= bufs.size()) throw std::runtime_error("shmem (GPU): more threads than at tree build");
        return bufs[t];
    }
};

namespace {

ReuseQueue& queue_of(const Tree& T) {
    if (!T.reuse) throw std::runtime_error("shmem (GPU): the Tree was not built by shmem::build");
    return *T.reuse;
}

// Apply every queued commutative event on the device (kick runs grouped by their tau).
void flush(const Tree& T) {
    ReuseQueue& Q = queue_of(T);
    std::lock_guard<std::mutex> lk(Q.mu);
    gt_tree* h = T.gpu.get();
    for (auto& b : Q.bufs) {
        if (!b.kick_leaf.empty())
            check(gt_tree_events(context(), h, GT_EVENT_KICK, (int64_t)b.kick_leaf.size(), b.kick_leaf.data(),
                                 b.kick_dp.data(), nullptr, nullptr, nullptr, b.kick_tau, 0.0, GT_MEM_HOST),
                  "gt_tree_events");
        if (!b.vmax_leaf.empty())
            check(gt_tree_events(context(), h, GT_EVENT_VMAX, (int64_t)b.vmax_leaf.size(), b.vmax_leaf.data(),
                                 nullptr, nullptr, nullptr, b.vmax_val.data(), 0.0, 0.0, GT_MEM_HOST),
                  "gt_tree_events");
        if (!b.soft_leaf.empty())
            check(gt_tree_events(context(), h, GT_EVENT_SOFT, (int64_t)b.soft_leaf.size(), b.soft_leaf.data(),
                                 b.soft_val.data(), nullptr, nullptr, nullptr, 0.0, 0.0, GT_MEM_HOST),
                  "gt_tree_events");
        if (!b.shift_leaf.empty())
            check(gt_tree_events(context(), h, GT_EVENT_SHIFT, (int64_t)b.shift_leaf.size(), b.shift_leaf.data(),
                                 b.shift_m.data(), b.shift_dx.data(), nullptr, nullptr, 0.0, 0.0, GT_MEM_HOST),
                  "gt_tree_events");
        if (!b.hmax_leaf.empty())
            check(gt_tree_events(context(), h, GT_EVENT_HMAX, (int64_t)b.hmax_leaf.size(), b.hmax_leaf.data(),
                                 b.hmax_val.data(), nullptr, nullptr, nullptr, 0.0, 0.0, GT_MEM_HOST),
                  "gt_tree_events");
        b = ReuseQueue::Buf{};
    }
}

struct NodeState {
    std::vector<double> com, vel, mass;
};
NodeState node_state(const Tree& T, double tau) {
    flush(T);
    const size_t nn = T.nnodes();
    NodeState s;
    s.com.resize(3 * nn); s.vel.resize(3 * nn); s.mass.resize(nn);
    check(gt_tree_node_state(context(), T.gpu.get(), tau, s.com.data(), s.vel.data(), s.mass.data(), nullptr,
                             nullptr), "gt_tree_node_state");
    return s;
}

// climb with a float max that stops at the first ancestor already covering the value
// (tree.cc:276-284); the host copy the engine reads
void climb_max(std::vector<float>& arr, const std::vector<int>& parent, int leaf, float v) {
    uint32_t want;
    std::memcpy(&want, &v, 4);
    for (int no = leaf; no >= 0; no = parent[no]) {
        uint32_t* bits = reinterpret_cast<uint32_t*>(&arr[no]);
        uint32_t seen = __atomic_load_n(bits, __ATOMIC_RELAXED);
        if (seen >= want) return;
        while (seen < want && !__atomic_compare_exchange_n(bits, &seen, want, true, __ATOMIC_RELAXED,
                                                            __ATOMIC_RELAXED)) {
        }
    }
}

}  // namespace

static void touch(const Tree& T) {
    ReuseQueue& Q = queue_of(T);
    Q.moved = true;
    ++Q.gen;
}

static void need_gpu(const Tree& T) {
    if (!T.gpu) throw std::runtime_error("shmem (GPU): the Tree was not built by shmem::build");
}

// Before a walk: queued tree events go to the device, and on a reused tree the device gets the
// particles' current state, which the reference walk reads (tree.cc:786-789).  Lazy drift
// (tree.cc:783-785) catches a particle up when the walk reaches it; the device walk reads all of
// them, so every particle behind the target is caught up first.
static void prepare_walk(const Tree& T, const Particles& P, const LazyDrift* lazy) {
    flush(T);
    const bool drift = lazy && lazy->catch_up && lazy->last;
    if (drift)
        for (uint32_t q : T.orderbuf)
            if (lazy->last[q] < lazy->target) lazy->catch_up(lazy->ctx, q);
    ReuseQueue& Q = queue_of(T);
    if (Q.moved || drift) {
        check(gt_tree_particles(context(), T.gpu.get(), P.x.data(), P.y.data(), P.z.data(), P.m.data(),
                                soft_or_null(P), GT_MEM_HOST), "gt_tree_particles");
        Q.search_gen = Q.gen;
    }
    // types and zeta as the walk reads them now (the engine updates zeta between steps): the gas
    // pair rule and the per-node sink counts of sink-direct opening
    if (!P.type.empty() || !P.zeta.empty()) {
        if ((!P.type.empty() && P.type.size() != P.size()) || (!P.zeta.empty() && P.zeta.size() != P.size()))
            throw std::runtime_error("shmem (GPU): Particles::type / ::zeta sizes differ from the particle count");
        check(gt_tree_gas(context(), T.gpu.get(), P.type.empty() ? nullptr : P.type.data(),
                          P.zeta.empty() ? nullptr : P.zeta.data(), GT_MEM_HOST), "gt_tree_gas");
    }
}

void accel(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets, double theta,
           double G, std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az,
           const double* aold) {
    need_gpu(T);
    prepare_walk(T, P, nullptr);
    const size_t nt = targets.size();
    ax.resize(nt); ay.resize(nt); az.resize(nt);  // every target's outputs are written
    if (!nt) return;
    check(gt_accel(context(), T.gpu.get(), (int64_t)nt, targets.data(), theta, G, aold, GT_MEM_HOST,
                   ax.data(), ay.data(), az.data()), "gt_accel");
}

void accel_soa(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
               double theta, double G, std::vector<double>& ax, std::vector<double>& ay,
               std::vector<double>& az) {
    // The reference keeps this SoA-layout walk only as a timing control; on the GPU there is one
    // node layout, so it is the per-target walk.
    accel(T, P, targets, theta, G, ax, ay, az, nullptr);
}

void accel_grouped(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
                   double theta, double G, int batch, std::vector<double>& ax,
                   std::vector<double>& ay, std::vector<double>& az,
                   std::vector<SymTensor3d>* tidal, const double* aold, const LazyDrift* lazy,
                   std::vector<Vec3d>* jerk, const double* const* vel, double sink_direct_radius) {
    need_gpu(T);
    prepare_walk(T, P, lazy);
    // the jerk needs source velocities: the walk's `vel` for particles and the build's node
    // centre-of-mass velocities (tree.cc:638-640); without them it stays zero
    const bool want_jerk = jerk && vel && !T.vcom_x.empty();
    const size_t nt = targets.size();
    // every target's outputs are written by the walk: size the vectors without clearing them
    // (a jerk without velocities stays zero)
    ax.resize(nt); ay.resize(nt); az.resize(nt);
    if (tidal) tidal->resize(nt);
    if (jerk) {
        if (want_jerk) jerk->resize(nt);
        else jerk->assign(nt, Vec3d{0, 0, 0});
    }
    if (!nt) return;
    gt_walk_options o;
    gt_walk_options_default(&o);
    // live only with types (tree.cc:634-635): without them the tree counted no sinks
    o.sink_direct_radius = (P.type.empty() || !(sink_direct_radius > 0.0)) ? 0.0 : sink_direct_radius;
    if (!tidal && !want_jerk) {
        check(gt_accel_grouped(context(), T.gpu.get(), (int64_t)nt, targets.data(), aold, theta, G, batch,
                               &o, GT_MEM_HOST, ax.data(), ay.data(), az.data(), nullptr), "gt_accel_grouped");
        return;
    }
    if (want_jerk)  // the particles' current velocities, the build's node velocities
        check(gt_tree_velocities(context(), T.gpu.get(), vel[0], vel[1], vel[2], 1, GT_MEM_HOST),
              "gt_tree_velocities");
    static_assert(sizeof(SymTensor3d) == 6 * sizeof(double), "SymTensor3d is six doubles");
    static_assert(sizeof(Vec3d) == 3 * sizeof(double), "Vec3d is three doubles");
    check(gt_accel_grouped_ext(context(), T.gpu.get(), (int64_t)nt, targets.data(), aold, theta, G, batch,
                               &o, GT_MEM_HOST, ax.data(), ay.data(), az.data(), nullptr,
                               tidal ? reinterpret_cast<double*>(tidal->data()) : nullptr,
                               want_jerk ? reinterpret_cast<double*>(jerk->data()) : nullptr),
          "gt_accel_grouped_ext");
}

void potential(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets,
               double theta, double G, std::vector<double>& phi, const double* aold) {
    need_gpu(T);
    prepare_walk(T, P, nullptr);
    const size_t nt = targets.size();
    phi.assign(nt, 0.0);
    if (!nt) return;
    check(gt_potential(context(), T.gpu.get(), (int64_t)nt, targets.data(), theta, G, aold,
                       GT_MEM_HOST, phi.data()), "gt_potential");
}

void accel_brute(const Particles& P, const std::vector<uint32_t>& targets, double G,
                 std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az) {
    const size_t nt = targets.size();
    ax.assign(nt, 0.0); ay.assign(nt, 0.0); az.assign(nt, 0.0);
    if (!nt) return;
    if (!P.zeta.empty()) {
        // gas particles with zeta: the pair rule's correction terms (tree.cc:39-53)
        check(gt_direct_gas(context(), (int64_t)P.size(), P.x.data(), P.y.data(), P.z.data(), P.m.data(),
                            soft_or_null(P), P.type.empty() ? nullptr : P.type.data(), P.zeta.data(),
                            (int64_t)nt, targets.data(), G, GT_MEM_HOST, ax.data(), ay.data(), az.data()),
              "gt_direct_gas");
        return;
    }
    check(gt_direct(context(), (int64_t)P.size(), P.x.data(), P.y.data(), P.z.data(), P.m.data(),
                    soft_or_null(P), (int64_t)nt, targets.data(), G, GT_DIRECT_FP64, GT_MEM_HOST,
                    ax.data(), ay.data(), az.data(), nullptr), "gt_direct");
}

int build_node(Tree&, const Particles&, const std::vector<uint32_t>&, const std::vector<uint64_t>&,
               int, int, int, double, double, double, double, const double* const*) {
    unsupported("build_node (the device build is level-synchronous)");
}
void setup_walk(Tree&, int, int) { unsupported("setup_walk (threading is produced by the device build)"); }


void Tree::raise_vmax(int leaf_node, float speed) {
    if (leaf_node < 0) return;
    climb_max(vmax, parent, leaf_node, speed);
    auto& b = queue_of(*this).mine();
    b.vmax_leaf.push_back(leaf_node);
    b.vmax_val.push_back(speed);
}
// rounded up to float, so the prune stays one-sided (tree.cc:288-291)
static float up_float(double h) {
    const float f = (float)h;
    return ((double)f < h) ? std::nextafter(f, 1e30f) : f;
}
void Tree::raise_hmax(int leaf_node, double h) {
    if (hmax.empty() || leaf_node < 0) return;  // before init_hmax: nothing to raise (tree.cc:294)
    climb_max(hmax, parent, leaf_node, up_float(h));
    auto& b = queue_of(*this).mine();
    b.hmax_leaf.push_back(leaf_node);
    b.hmax_val.push_back(h);
}
void Tree::init_hmax(const std::vector<double>& h, size_t n_gas) {
    flush(*this);
    const size_t n = std::min(std::min(n_gas, h.size()), leaf_of.size());
    hmax.assign(nnodes(), 0.0f);
    for (size_t i = 0; i < n; ++i)
        if (h[i] > 0 && leaf_of[i] >= 0) climb_max(hmax, parent, leaf_of[i], up_float(h[i]));
    check(gt_tree_hmax(context(), gpu.get(), h.data(), (int64_t)n, GT_MEM_HOST), "gt_tree_hmax");
}
void Tree::raise_soft(int leaf_node, double s) {
    if (leaf_node < 0) return;
    auto& b = queue_of(*this).mine();
    b.soft_leaf.push_back(leaf_node);
    b.soft_val.push_back(s);
}
void Tree::raise_pad(int leaf_node, double d) {
    if (leaf_node < 0 || !(d > 0)) return;
    flush(*this);
    const int32_t lf = leaf_node;
    check(gt_tree_events(context(), gpu.get(), GT_EVENT_PAD, 1, &lf, &d, nullptr, nullptr, nullptr, 0.0, 0.0,
                         GT_MEM_HOST), "gt_tree_events");
    // the host copy (the neighbour search reads it): the same serial climb (tree.cc:322-329)
    float leaf_pad = (float)((double)xpad[leaf_node] + d);
    if ((double)leaf_pad < (double)xpad[leaf_node] + d) leaf_pad = std::nextafter(leaf_pad, 1e30f);
    for (int no = leaf_node; no >= 0 && xpad[no] < leaf_pad; no = parent[no]) xpad[no] = leaf_pad;
    touch(*this);
}
void Tree::kick_node(int leaf_node, const Vec3d& dp, double tau) {
    if (dp_x.empty() || leaf_node < 0) return;  // no vcom, nothing to keep current (tree.cc:212)
    auto& b = queue_of(*this).mine();
    if (!b.kick_leaf.empty() && b.kick_tau != tau) flush(*this);
    b.kick_tau = tau;
    b.kick_leaf.push_back(leaf_node);
    for (int k = 0; k < 3; ++k) b.kick_dp.push_back(dp[k]);
    touch(*this);
}
void Tree::mass_event(int leaf_node, double dm, const Vec3d& x, const Vec3d& v, double tau, double box) {
    if (dp_x.empty() || leaf_node < 0 || dm == 0.0) return;
    flush(*this);
    const int32_t lf = leaf_node;
    const double xx[3] = {x[0], x[1], x[2]}, vv[3] = {v[0], v[1], v[2]};
    check(gt_tree_events(context(), gpu.get(), GT_EVENT_MASS, 1, &lf, &dm, xx, vv, nullptr, tau, box, GT_MEM_HOST),
          "gt_tree_events");
    touch(*this);
}
void Tree::shift_node(int leaf_node, double m, const Vec3d& dx) {
    if (dp_x.empty() || leaf_node < 0) return;
    auto& b = queue_of(*this).mine();
    b.shift_leaf.push_back(leaf_node);
    b.shift_m.push_back(m);
    for (int k = 0; k < 3; ++k) b.shift_dx.push_back(dx[k]);
    touch(*this);
}
double Tree::node_mass(int no) const { return node_state(*this, 0.0).mass[no]; }
Vec3d Tree::node_com(int no, double tau) const {
    const NodeState s = node_state(*this, tau);
    return Vec3d{s.com[3 * no], s.com[3 * no + 1], s.com[3 * no + 2]};
}
Vec3d Tree::node_vel(int no) const {
    const NodeState s = node_state(*this, 0.0);
    return Vec3d{s.vel[3 * no], s.vel[3 * no + 1], s.vel[3 * no + 2]};
}
void Tree::refresh_walk_nodes(double tau) {
    flush(*this);
    check(gt_tree_refresh(context(), gpu.get(), tau), "gt_tree_refresh");
    if (tau != 0.0) touch(*this);
}

// Structural audit of the downloaded tree (the topology and coverage parts of the reference's
// audit_tree, shmem/tree.cc:986-1056): every child chain closes on next[X], parent[] agrees with
// the threading, every massive particle is reached exactly once, leaf_of agrees, and node masses
// equal the sums of their particles.
long long audit_tree(const Tree& T, const Particles& P, const double*, size_t, const double*,
                     const double*, const double*, double, const double*, char* msg, size_t msglen) {
    long long bad = 0;
    auto fail = [&](const char* what, long long a, long long b) {
        if (bad++ == 0 && msg) snprintf(msg, msglen, "%s (%lld, %lld)", what, a, b);
    };
    const size_t N = P.size(), nn = T.nnodes();
    if (T.parent.size() != nn || T.leaf_of.size() != N || T.wn.size() != nn) {
        fail("array sizes", (long long)nn, (long long)N);
        return bad;
    }
    std::vector<uint8_t> seen_node(nn, 0), seen_part(N, 0);
    std::vector<int> stack{T.root};
    if (T.parent[T.root] != -1) fail("root has a parent", T.root, T.parent[T.root]);
    while (!stack.empty()) {
        const int X = stack.back();
        stack.pop_back();
        if (X < 0 || (size_t)X >= nn) { fail("node index out of range", X, (long long)nn); continue; }
        if (seen_node[X]++) { fail("node reached twice", X, 0); continue; }
        if (T.first[X] < 0) {
            double msum = 0;
            for (int s = T.plo[X]; s < T.phi[X]; ++s) {
                const uint32_t p = T.orderbuf[s];
                if (p >= N) { fail("leaf holds a bad index", X, p); continue; }
                if (seen_part[p]++) fail("particle reached twice", p, X);
                if (T.leaf_of[p] != X) fail("leaf_of disagrees with the threading", p, X);
                msum += P.m[p];
            }
            if (std::fabs(msum - T.mass[X]) > 1e-10 * std::max(msum, std::fabs(T.mass[X])) + 1e-300)
                fail("leaf mass differs from its particles", X, 0);
            continue;
        }
        size_t steps = 0;
        for (int c = T.first[X]; c != T.next[X]; c = T.next[c]) {
            if (c < 0 || (size_t)c >= nn || ++steps > 8) { fail("child chain never reaches next[X]", X, c); break; }
            if (T.parent[c] != X) fail("parent disagrees with the threading", c, X);
            stack.push_back(c);
        }
    }
    for (size_t p = 0; p < N; ++p)
        if (!seen_part[p] && P.m[p] > 0) { fail("particle unreachable from the root", (long long)p, 0); break; }
    return bad;
}

// ---- neighbour search and the density solve (hydro.h) ------------------------------------------

// The counters (hydro.cc:28-35, 20-23) summed over every context: each read moves the contexts'
// device totals into these host totals, which the two readers reset separately, as the
// reference's do.  Read them where the reference does, between searches.
static long long g_tally[GT_NGB_COUNTERS] = {};

static void gather_tallies() {
    std::lock_guard<std::mutex> lk(g_contexts_mu);
    for (gt_context* c : g_contexts) {
        int64_t v[GT_NGB_COUNTERS];
        if (gt_ngb_counters_get(c, v, 1) != GT_OK)
            throw std::runtime_error(std::string("gt_ngb_counters_get: ") + gt_last_error(c));
        for (int k = 0; k < GT_NGB_COUNTERS; ++k) g_tally[k] += (long long)v[k];
    }
}

void ngb_counters(long long& calls, long long& nodes, long long& examined, long long& kept, long long& pad_nodes,
                  bool reset) {
    gather_tallies();
    calls = g_tally[0]; nodes = g_tally[1]; examined = g_tally[2]; kept = g_tally[3]; pad_nodes = g_tally[4];
    if (reset)
        for (int k = 0; k < 5; ++k) g_tally[k] = 0;
}
void hiter_counters(long long out[8], bool reset) {
    gather_tallies();
    for (int i = 0; i < 8; ++i) {
        out[i] = g_tally[5 + i];
        if (reset) g_tally[5 + i] = 0;
    }
}

// Before a per-centre search: queued events to the device, lazy catch-up of every particle behind
// the target, and the particles' current state on the device once per change of the tree.
static void prepare_search(const Tree& T, const Particles& P, const LazyDrift* lazy) {
    flush(T);
    ReuseQueue& Q = queue_of(T);
    std::lock_guard<std::mutex> lk(Q.search_mu);
    bool behind = false;
    if (lazy && lazy->catch_up && lazy->last)
        for (uint32_t q : T.orderbuf)
            if (lazy->last[q] < lazy->target) {
                lazy->catch_up(lazy->ctx, q);
                behind = true;
            }
    if (behind || (Q.moved && Q.search_gen != Q.gen)) {
        check(gt_tree_particles(context(), T.gpu.get(), P.x.data(), P.y.data(), P.z.data(), P.m.data(),
                                soft_or_null(P), GT_MEM_HOST), "gt_tree_particles");
        Q.search_gen = Q.gen;
    }
}

// One centre through the batched search: a first call with the thread's buffer, a second with
// room for the total when the first overflowed.
static void search_one(const Tree& T, const gt_ngb_options& o, const Vec3d& c, double radius,
                       std::vector<uint32_t>& found) {
    thread_local std::vector<uint32_t> buf(512);
    const double cx = c[0], cy = c[1], cz = c[2];
    int64_t start[2] = {0, 0}, tot = 0;
    int st = gt_ngb_search(context(), T.gpu.get(), 1, &cx, &cy, &cz, &radius, &o, GT_MEM_HOST, start, buf.data(),
                           (int64_t)buf.size(), &tot);
    if (st == GT_ERR_OVERFLOW) {  // (an overflowed call counts nothing under SHMEM_NGB_COUNT)
        buf.resize((size_t)tot * 2);
        st = gt_ngb_search(context(), T.gpu.get(), 1, &cx, &cy, &cz, &radius, &o, GT_MEM_HOST, start, buf.data(),
                           (int64_t)buf.size(), &tot);
    }
    check(st, "gt_ngb_search");
    found.insert(found.end(), buf.begin(), buf.begin() + tot);
}

void ngb_search(const Tree& T, const Particles& P, const Vec3d& centre, double radius, std::vector<uint32_t>& found,
                double box, const LazyDrift* lazy) {
    need_gpu(T);
    prepare_search(T, P, lazy);
    gt_ngb_options o;
    gt_ngb_options_default(&o);
    o.box = box;
    o.elapsed = T.t_since_build;
    search_one(T, o, centre, radius, found);
}

void ngb_search_reverse(const Tree& T, const Particles& P, const double* h, size_t n_gas, const Vec3d& centre,
                        double h_i, std::vector<uint32_t>& found, double box, const LazyDrift* lazy) {
    need_gpu(T);
    if (T.hmax.empty()) throw std::runtime_error("shmem (GPU): ngb_search_reverse needs Tree::init_hmax first");
    prepare_search(T, P, lazy);
    gt_ngb_options o;
    gt_ngb_options_default(&o);
    o.mode = GT_NGB_REVERSE;
    o.box = box;
    o.elapsed = T.t_since_build;
    o.n_gas = (int64_t)n_gas;
    o.h = h;
    search_one(T, o, centre, h_i, found);
}

DensityResult density(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets, double des_ngb,
                      double ngb_tol, const std::vector<double>& h_start, double box, int n_dims, NeighborCache* cache,
                      const LazyDrift* lazy, const double* cond_prev) {
    need_gpu(T);
    prepare_walk(T, P, lazy);  // current particles and types (the solve counts gas neighbours only)
    const size_t nt = targets.size();
    DensityResult R;
    R.h.assign(nt, 0.0); R.rho.assign(nt, 0.0); R.nngb.assign(nt, 0); R.iters.assign(nt, 0);
    if (cache) { cache->clear(); cache->start.assign(nt + 1, 0); }
    if (!h_start.empty() && h_start.size() < nt)
        throw std::runtime_error("shmem (GPU): density h_start has fewer entries than targets");
    if (nt) {
        gt_density_options o;
        gt_density_options_default(&o);
        o.des_ngb = des_ngb;
        o.ngb_tol = ngb_tol;
        o.box = box;
        o.elapsed = T.t_since_build;
        o.n_dims = n_dims;
        o.face_correction = getenv("SHMEM_NO_FACECORR") ? 0 : 1;  // the reference's A/B switch
        o.h_start = h_start.empty() ? nullptr : h_start.data();
        o.cond_prev = cond_prev;
        std::vector<int32_t> nngb(nt), iters(nt);
        check(gt_density(context(), T.gpu.get(), (int64_t)nt, targets.data(), &o, GT_MEM_HOST, R.h.data(),
                         R.rho.data(), nngb.data(), iters.data()), "gt_density");
        for (size_t t = 0; t < nt; ++t) { R.nngb[t] = nngb[t]; R.iters[t] = iters[t]; }
    }
    if (cache) {
        // every target's list at its final h: one batched search
        if (nt) {
            std::vector<double> cx(nt), cy(nt), cz(nt);
            for (size_t t = 0; t < nt; ++t) { cx[t] = P.x[targets[t]]; cy[t] = P.y[targets[t]]; cz[t] = P.z[targets[t]]; }
            gt_ngb_options o;
            gt_ngb_options_default(&o);
            o.box = box;
            o.elapsed = T.t_since_build;
            std::vector<int64_t> start(nt + 1);
            int64_t tot = 0;
            // the reference's cache holds the solve's own lists: these searches are not counted.
            // One call with room for 64 neighbours per target, a sized second one if that overflows.
            if (ngb_counting()) check(gt_ngb_count(context(), 0), "gt_ngb_count");
            cache->flat.resize(nt * 64);
            int st = gt_ngb_search(context(), T.gpu.get(), (int64_t)nt, cx.data(), cy.data(), cz.data(), R.h.data(),
                                   &o, GT_MEM_HOST, start.data(), cache->flat.data(), (int64_t)cache->flat.size(), &tot);
            if (st == GT_ERR_OVERFLOW) {
                cache->flat.resize((size_t)tot);
                st = gt_ngb_search(context(), T.gpu.get(), (int64_t)nt, cx.data(), cy.data(), cz.data(), R.h.data(),
                                   &o, GT_MEM_HOST, start.data(), cache->flat.data(), tot, &tot);
            }
            if (ngb_counting()) check(gt_ngb_count(context(), 1), "gt_ngb_count");
            check(st, "gt_ngb_search");
            cache->flat.resize((size_t)tot);
            for (size_t t = 0; t <= nt; ++t) cache->start[t] = (size_t)start[t];
        }
        cache->valid = true;
    }
    return R;
}

}  // namespace shmem
