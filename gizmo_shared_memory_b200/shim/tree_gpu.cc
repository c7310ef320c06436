// shmem:: tree functions implemented on libgt (include/gt.h).  See tree.h in this directory for
// the differences a caller can observe.
#include "tree.h"

#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "gt.h"

namespace shmem {
namespace {

// One library context per host thread, on device $GT_DEVICE (default 0), created on first use.
// It is deliberately never destroyed: a destructor running at thread or process exit could call
// into the CUDA runtime after the runtime has begun its own teardown; process exit releases the
// context's device memory and stream anyway.
gt_context* context() {
    thread_local gt_context* ctx = nullptr;
    if (!ctx) {
        const char* d = getenv("GT_DEVICE");
        const int st = gt_context_create(d ? atoi(d) : 0, &ctx);
        if (st != GT_OK) {
            ctx = nullptr;
            throw std::runtime_error(std::string("gt_context_create: ") + gt_status_string(st));
        }
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

void require_gravity_only(const Particles& P) {
    for (double z : P.zeta)
        if (z != 0.0) unsupported("the adaptive-softening zeta pair terms");
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

static void need_gpu(const Tree& T) {
    if (!T.gpu) throw std::runtime_error("shmem (GPU): the Tree was not built by shmem::build");
}

void accel(const Tree& T, const Particles& P, const std::vector<uint32_t>& targets, double theta,
           double G, std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az,
           const double* aold) {
    need_gpu(T);
    require_gravity_only(P);
    const size_t nt = targets.size();
    ax.assign(nt, 0.0); ay.assign(nt, 0.0); az.assign(nt, 0.0);
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
    require_gravity_only(P);
    if (lazy) unsupported("lazy drift");
    if (sink_direct_radius > 0 && !P.type.empty()) unsupported("sink-direct opening");
    // the jerk needs source velocities: the walk's `vel` for particles and the build's node
    // centre-of-mass velocities (tree.cc:638-640); without them it stays zero
    const bool want_jerk = jerk && vel && !T.vcom_x.empty();
    const size_t nt = targets.size();
    ax.assign(nt, 0.0); ay.assign(nt, 0.0); az.assign(nt, 0.0);
    if (tidal) tidal->assign(nt, SymTensor3d{0, 0, 0, 0, 0, 0});
    if (jerk) jerk->assign(nt, Vec3d{0, 0, 0});
    if (!nt) return;
    gt_walk_options o;
    gt_walk_options_default(&o);
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
    (void)P;
    const size_t nt = targets.size();
    phi.assign(nt, 0.0);
    if (!nt) return;
    check(gt_potential(context(), T.gpu.get(), (int64_t)nt, targets.data(), theta, G, aold,
                       GT_MEM_HOST, phi.data()), "gt_potential");
}

void accel_brute(const Particles& P, const std::vector<uint32_t>& targets, double G,
                 std::vector<double>& ax, std::vector<double>& ay, std::vector<double>& az) {
    require_gravity_only(P);
    const size_t nt = targets.size();
    ax.assign(nt, 0.0); ay.assign(nt, 0.0); az.assign(nt, 0.0);
    if (!nt) return;
    check(gt_direct(context(), (int64_t)P.size(), P.x.data(), P.y.data(), P.z.data(), P.m.data(),
                    soft_or_null(P), (int64_t)nt, targets.data(), G, GT_DIRECT_FP64, GT_MEM_HOST,
                    ax.data(), ay.data(), az.data(), nullptr), "gt_direct");
}

int build_node(Tree&, const Particles&, const std::vector<uint32_t>&, const std::vector<uint64_t>&,
               int, int, int, double, double, double, double, const double* const*) {
    unsupported("build_node (the device build is level-synchronous)");
}
void setup_walk(Tree&, int, int) { unsupported("setup_walk (threading is produced by the device build)"); }

void Tree::raise_vmax(int, float) { unsupported("Tree::raise_vmax (tree reuse)"); }
void Tree::raise_hmax(int, double) { unsupported("Tree::raise_hmax (tree reuse)"); }
void Tree::init_hmax(const std::vector<double>&, size_t) { unsupported("Tree::init_hmax (tree reuse)"); }
void Tree::raise_soft(int, double) { unsupported("Tree::raise_soft (tree reuse)"); }
void Tree::raise_pad(int, double) { unsupported("Tree::raise_pad (tree reuse)"); }
void Tree::kick_node(int, const Vec3d&, double) { unsupported("Tree::kick_node (tree reuse)"); }
void Tree::mass_event(int, double, const Vec3d&, const Vec3d&, double, double) {
    unsupported("Tree::mass_event (tree reuse)");
}
void Tree::shift_node(int, double, const Vec3d&) { unsupported("Tree::shift_node (tree reuse)"); }
Vec3d Tree::node_com(int no, double) const { return Vec3d{cx[no], cy[no], cz[no]}; }
void Tree::refresh_walk_nodes(double tau) {
    if (tau != 0.0) unsupported("Tree::refresh_walk_nodes with tau != 0 (tree reuse)");
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

}  // namespace shmem
