// Device-side audit of a tree's invariants: the replacement for shmem::audit_tree
// (shmem/tree.cc:973-1119), which walks the tree on the host.
//
// One warp per node.  Lane 0 checks the node's place in the structure: particle range inside the
// live range, children contiguous and partitioning the node's range in order, each child's parent,
// level and side, the reference's `next` threading, leaf size.  All lanes then stride over the
// node's particles (a node holds the contiguous tree-order range [plo, phi)) and
//   * re-derive its mass and centre of mass in FP64 and compare with the walk node's (the build's
//     moments, or refresh_walk_nodes' after reuse events);
//   * check every particle lies inside the node's cell (geometric centre +- half side, plus 1e-6
//     of the root side as the reference's search boxes carry, tree.cc:490-505, and any
//     displacement pad): the 20-bit quantisation maps the root side onto 2^20 - 1 steps, so its
//     cells sit up to 9.5e-7 root sides off the geometric ones) and its softening is covered by
//     the node's;
//   * on a leaf, check the maps: leaf of each particle, tree position <-> particle index.
// Every node visits its particles, so the audit costs N x depth particle reads (a few ms at 16M).
// Violations are counted; the first one found records a code and its indices for the message.
#include <cstdio>
#include <cstring>

#include "gt_internal.cuh"

namespace gt {
namespace {

constexpr unsigned kFull = 0xffffffffu;

enum AuditCode : int {
    kAuditNone = 0,
    kAuditRange,        // node particle range outside [0, n_live] or reversed
    kAuditRoot,         // a root has a parent
    kAuditParent,       // parent[X] does not list X among its children
    kAuditChildren,     // child block out of range or more than 8 children
    kAuditPartition,    // children do not partition the node's range in order (or one is empty)
    kAuditChildGeom,    // child level or side inconsistent with the parent
    kAuditNext,         // `next` threading differs from the reference's convention
    kAuditLeafSize,     // leaf above leaf_max particles below max_level
    kAuditLeafMap,      // sleaf / leaf_of of a leaf's particle is not that leaf
    kAuditRankMap,      // rank[order[s]] != s
    kAuditMass,         // node mass differs from the sum over its particles
    kAuditCom,          // node centre of mass off the particles'
    kAuditBox,          // a particle outside its node's cell
    kAuditSoft,         // a particle's softening above its node's
    kAuditDead          // a massless particle in the live range, or a live one after it
};

struct AuditArgs {
    const GNode* nodes;
    const int* parent;
    const int* next;
    const int* level;
    const double* size;
    const double* gc;
    const double* nsoft;
    const float* xpad;  // may be null
    const SrcP* src;
    const double* smass;
    const double* ssoft;
    const uint32_t* order;
    const uint32_t* rank;
    const int* leaf_of;
    const int* sleaf;
    const int* sys_off;       // forest: live tree-position offsets of the systems
    int64_t n, n_live, n_nodes;
    int n_systems, leaf_max, max_level;
    unsigned long long* bad;  // [0] count, [1] first-record flag
    long long* rec;           // code, node, slot, then two values as bit patterns
};

__device__ void report(const AuditArgs& A, int code, long long node, long long slot, double v1, double v2) {
    atomicAdd(A.bad, 1ull);
    if (atomicCAS(A.bad + 1, 0ull, 1ull) == 0ull) {
        A.rec[0] = code;
        A.rec[1] = node;
        A.rec[2] = slot;
        A.rec[3] = __double_as_longlong(v1);
        A.rec[4] = __double_as_longlong(v2);
    }
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__global__ void __launch_bounds__(256) audit_nodes_kernel(const AuditArgs A) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t X = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); X < A.n_nodes; X += warps) {
        const GNode nd = A.nodes[X];
        if (nd.plo < 0 || nd.phi < nd.plo || nd.phi > A.n_live) {
            if (lane == 0) report(A, kAuditRange, X, -1, nd.plo, nd.phi);
            continue;
        }
        if (lane == 0) {
            // place in the structure
            const int pa = A.parent[X];
            if (X < A.n_systems) {
                if (pa != -1) report(A, kAuditRoot, X, -1, pa, 0);
            } else if (pa < 0 || pa >= A.n_nodes || X < A.nodes[pa].first ||
                       X >= A.nodes[pa].first + A.nodes[pa].nchild) {
                report(A, kAuditParent, X, -1, pa, 0);
            } else {
                // the reference's threading: the next sibling, or the parent's next after the last
                const GNode& pn = A.nodes[pa];
                const int want = X + 1 < pn.first + pn.nchild ? (int)X + 1 : A.next[pa];
                if (A.next[X] != want) report(A, kAuditNext, X, -1, A.next[X], want);
            }
            if (nd.first >= 0) {
                if (nd.nchild < 1 || nd.nchild > 8 || nd.first <= X || nd.first + nd.nchild > A.n_nodes) {
                    report(A, kAuditChildren, X, -1, nd.first, nd.nchild);
                } else {
                    int at = nd.plo;
                    for (int c = nd.first; c < nd.first + nd.nchild; ++c) {
                        const GNode& ch = A.nodes[c];
                        if (ch.plo != at || ch.phi <= ch.plo) { report(A, kAuditPartition, X, c, ch.plo, at); break; }
                        at = ch.phi;
                        if (A.parent[c] != (int)X) report(A, kAuditParent, c, -1, A.parent[c], (double)X);
                        if (A.level[c] != A.level[X] + 1 || A.size[c] != 0.5 * A.size[X])
                            report(A, kAuditChildGeom, c, -1, A.level[c], A.size[c]);
                    }
                    if (at != nd.phi) report(A, kAuditPartition, X, -1, at, nd.phi);
                }
            } else {
                if (nd.nchild != 0) report(A, kAuditChildren, X, -1, nd.first, nd.nchild);
                if (nd.phi - nd.plo > A.leaf_max && A.level[X] < A.max_level)
                    report(A, kAuditLeafSize, X, -1, nd.phi - nd.plo, A.level[X]);
            }
        }
        // the node's particles: moments, cell and softening coverage, leaf maps
        const int sys = A.n_systems > 1 ? system_of(A.sys_off, A.n_systems, nd.plo) : 0;
        const double hx = 0.5 * A.size[X] + 1e-6 * A.size[sys] + (A.xpad ? (double)A.xpad[X] : 0.0);
        const double gx = A.gc[3 * X], gy = A.gc[3 * X + 1], gz = A.gc[3 * X + 2];
        const double ns = A.nsoft[X] * (1.0 + 1e-6);
        double m = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
        for (int s = nd.plo + lane; s < nd.phi; s += 32) {
            const SrcP p = A.src[s];
            const double pm = A.smass[s];
            m += pm;
            mx += pm * (p.x - nd.cx); my += pm * (p.y - nd.cy); mz += pm * (p.z - nd.cz);
            const double dx = fabs(p.x - gx), dy = fabs(p.y - gy), dz = fabs(p.z - gz);
            if (!(dx <= hx && dy <= hx && dz <= hx)) report(A, kAuditBox, X, s, fmax(dx, fmax(dy, dz)), hx);
            if (!(A.ssoft[s] <= ns)) report(A, kAuditSoft, X, s, A.ssoft[s], A.nsoft[X]);
            if (nd.first < 0) {
                const uint32_t pi = A.order[s];
                if (pi >= A.n || A.rank[pi] != (uint32_t)s) report(A, kAuditRankMap, X, s, pi, 0);
                else if (A.leaf_of[pi] != (int)X || A.sleaf[s] != (int)X)
                    report(A, kAuditLeafMap, X, s, A.leaf_of[pi], A.sleaf[s]);
                if (!(pm > 0.0)) report(A, kAuditDead, X, s, pm, 0);
            }
        }
        m = wsum(m); mx = wsum(mx); my = wsum(my); mz = wsum(mz);
        if (lane == 0 && nd.phi > nd.plo) {
            if (fabs(m - nd.mass) > 1e-10 * fmax(m, fabs(nd.mass)) + 1e-300) report(A, kAuditMass, X, -1, nd.mass, m);
            if (m > 0.0) {
                const double off = sqrt(mx * mx + my * my + mz * mz) / m;
                const double reach = A.size[X] + 2.0 * (A.xpad ? (double)A.xpad[X] : 0.0);
                if (off > 1e-6 * reach) report(A, kAuditCom, X, -1, off, reach);
            }
        }
    }
}

// Tree positions past the live range hold the massless particles, in no leaf (the device keeps
// their tree positions in rank; gt_tree_download marks them UINT32_MAX as the reference does).
__global__ void audit_dead_kernel(const AuditArgs A) {
    for (int64_t s = A.n_live + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < A.n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t pi = A.order[s];
        if (A.smass[s] > 0.0 || pi >= A.n || A.leaf_of[pi] != -1 || A.rank[pi] != (uint32_t)s || A.sleaf[s] != -1)
            report(A, kAuditDead, -1, s, A.smass[s], pi < A.n ? (double)A.leaf_of[pi] : -2.0);
    }
}

const char* audit_text(int code) {
    switch (code) {
        case kAuditRange: return "particle range outside the live range (plo, phi)";
        case kAuditRoot: return "a root has a parent (parent)";
        case kAuditParent: return "parent does not list the node among its children (parent, -)";
        case kAuditChildren: return "bad child block (first, nchild)";
        case kAuditPartition: return "children do not partition the node's particle range (position, expected)";
        case kAuditChildGeom: return "child level or side inconsistent with its parent (level, side)";
        case kAuditNext: return "next threading differs from the reference's (next, expected)";
        case kAuditLeafSize: return "leaf above leaf_max below max_level (count, level)";
        case kAuditLeafMap: return "leaf map of a leaf's particle is not that leaf (leaf_of, sleaf)";
        case kAuditRankMap: return "rank[order[s]] != s (particle, -)";
        case kAuditMass: return "node mass differs from its particles' sum (node, particles)";
        case kAuditCom: return "node centre of mass off its particles' (offset, reach)";
        case kAuditBox: return "particle outside its node's cell (offset, half side)";
        case kAuditSoft: return "particle softening above its node's (particle, node)";
        case kAuditDead: return "live/massless split of the tree order broken (mass, leaf)";
        default: return "unknown";
    }
}

}  // namespace

void run_tree_audit(gt_context* ctx, const gt_tree* t, int64_t* n_bad, char* msg, size_t msglen) {
    cudaStream_t st = ctx->stream;
    unsigned long long* ctr = (unsigned long long*)scratch(ctx, kSlotCounters, 256);
    AuditArgs a;
    a.nodes = t->nodes; a.parent = t->parent; a.next = t->next; a.level = t->level; a.size = t->size;
    a.gc = t->gc; a.nsoft = t->nsoft; a.xpad = t->xpad; a.src = t->src; a.smass = t->smass;
    a.ssoft = t->ssoft; a.order = t->order; a.rank = t->rank; a.leaf_of = t->leaf_of; a.sleaf = t->sleaf;
    a.sys_off = t->sys_off_dev;
    a.n = t->n; a.n_live = t->n_live; a.n_nodes = t->n_nodes; a.n_systems = t->n_systems;
    a.leaf_max = t->opt.leaf_max; a.max_level = t->opt.max_level;
    a.bad = ctr;
    a.rec = (long long*)(ctr + 2);
    check_cuda(cudaMemsetAsync(ctr, 0, 7 * 8, st), "memset");
    if (t->n_nodes > 0) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((t->n_nodes + 7) / 8, (int64_t)ctx->num_sms * 16));
        audit_nodes_kernel<<<blocks, 256, 0, st>>>(a);
        check_launch(ctx, "audit_nodes_kernel");
    }
    if (t->n > t->n_live) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((t->n - t->n_live + 255) / 256, (int64_t)ctx->num_sms * 8));
        audit_dead_kernel<<<blocks, 256, 0, st>>>(a);
        check_launch(ctx, "audit_dead_kernel");
    }
    unsigned long long h[7];
    check_cuda(cudaMemcpyAsync(ctx->pinned, ctr, sizeof(h), cudaMemcpyDeviceToHost, st), "d2h");
    check_cuda(cudaStreamSynchronize(st), "sync");
    std::memcpy(h, ctx->pinned, sizeof(h));
    *n_bad = (int64_t)h[0];
    if (msg && msglen > 0) {
        if (h[0] == 0) {
            msg[0] = '\0';
        } else {
            double v1, v2;
            std::memcpy(&v1, &h[5], 8);
            std::memcpy(&v2, &h[6], 8);
            std::snprintf(msg, msglen, "%s: node %lld, tree position %lld, values %.17g, %.17g",
                          audit_text((int)h[2]), (long long)h[3], (long long)h[4], v1, v2);
        }
    }
}

}  // namespace gt
