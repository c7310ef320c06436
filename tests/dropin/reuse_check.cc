// Tree reuse through the shmem:: API, compiled unchanged against the reference's shmem/tree.h (CPU,
// oracle/_ref/reuse_check) and against the GPU shim (gizmo_shared_memory_b200/shim/_build/
// reuse_check); tests/test_dropin.py compares what the two write.
//
//   reuse_check STATE OUT
//
// STATE is the bench_treeforce state format (N, then x y z m h vx vy vz as float64).  The program
// builds the tree with velocities, walks once for aold, then feeds a fixed sequence of
// incremental-moment events (kicks, speed bounds, shifts, mass events, pads), refreshes the walk
// nodes at tau, drifts the particles ballistically by tau, and walks the reused tree for the
// acceleration, tidal tensor and jerk.  OUT receives ax, ay, az (N each), tidal (6N) and jerk
// (3N) for the targets in orderbuf order, as float64, then the node masses and centres of mass
// of the root.
#include "tree.h"

#include <cmath>
#include <cstdio>
#include <vector>

using namespace shmem;

int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s STATE OUT\n", argv[0]); return 2; }
    FILE* fh = fopen(argv[1], "rb");
    if (!fh) { fprintf(stderr, "cannot open %s\n", argv[1]); return 1; }
    uint64_t N = 0;
    if (fread(&N, 8, 1, fh) != 1) return 1;
    Particles P;
    P.x.resize(N); P.y.resize(N); P.z.resize(N); P.m.resize(N); P.soft.resize(N);
    std::vector<double> vx(N), vy(N), vz(N);
    for (auto* a : {&P.x, &P.y, &P.z, &P.m, &P.soft, &vx, &vy, &vz})
        if (fread(a->data(), 8, N, fh) != N) return 1;
    fclose(fh);
    const double* vel[3] = {vx.data(), vy.data(), vz.data()};
    Tree T = build(P, nullptr, vel, true);
    std::vector<uint32_t> targets(T.orderbuf.begin(), T.orderbuf.end());
    std::vector<double> ax, ay, az;
    accel_grouped(T, P, targets, 0.7, 1.0, 0, ax, ay, az);
    std::vector<double> aold(targets.size());
    for (size_t k = 0; k < targets.size(); ++k)
        aold[k] = 0.005 * std::sqrt(ax[k] * ax[k] + ay[k] * ay[k] + az[k] * az[k]);

    // events, in a fixed order (the serial ones in particle order)
    const double tau = 0.02;
    for (size_t i = 0; i < N; i += 7) {
        const int leaf = T.leaf_of[i];
        if (leaf < 0) continue;
        const double s = 1e-3 * (double)((i * 2654435761ull) % 1000) / 1000.0;
        T.kick_node(leaf, Vec3d{P.m[i] * s, -P.m[i] * s, 0.5 * P.m[i] * s}, 0.01);
    }
    for (size_t i = 0; i < N; i += 5) {
        const int leaf = T.leaf_of[i];
        if (leaf < 0) continue;
        T.raise_vmax(leaf, (float)(1.2 * std::sqrt(vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i])));
    }
    std::vector<double> shift_x(N, 0.0);
    for (size_t i = 0; i < N; i += 97) {
        const int leaf = T.leaf_of[i];
        if (leaf < 0) continue;
        shift_x[i] = 1e-4;
        T.shift_node(leaf, P.m[i], Vec3d{1e-4, 0.0, 0.0});
    }
    for (size_t i = 0; i < N; i += 1013) {
        const int leaf = T.leaf_of[i];
        if (leaf < 0) continue;
        T.mass_event(leaf, 0.1 * P.m[i], Vec3d{P.x[i], P.y[i], P.z[i]}, Vec3d{vx[i], vy[i], vz[i]}, tau, 0.0);
        T.raise_pad(leaf, 1e-4);
    }
    T.refresh_walk_nodes(tau);
    T.t_since_build = tau;
    for (size_t i = 0; i < N; ++i) {
        P.x[i] += vx[i] * tau + shift_x[i];
        P.y[i] += vy[i] * tau;
        P.z[i] += vz[i] * tau;
    }
    std::vector<SymTensor3d> tt;
    std::vector<Vec3d> jj;
    accel_grouped(T, P, targets, 0.0, 1.0, 0, ax, ay, az, &tt, aold.data(), nullptr, &jj, vel);

    FILE* out = fopen(argv[2], "wb");
    if (!out) return 1;
    fwrite(ax.data(), 8, ax.size(), out);
    fwrite(ay.data(), 8, ay.size(), out);
    fwrite(az.data(), 8, az.size(), out);
    for (auto& t : tt) fwrite(&t, 8, 6, out);
    for (auto& j : jj) fwrite(&j, 8, 3, out);
    const Vec3d c = T.node_com(T.root, tau);
    const double root[4] = {T.node_mass(T.root), c[0], c[1], c[2]};
    fwrite(root, 8, 4, out);
    fclose(out);
    printf("reuse_check: N=%llu nodes=%zu root mass %.17g vmax %.9g\n", (unsigned long long)N, T.nnodes(),
           root[0], (double)T.vmax[T.root]);
    return 0;
}
