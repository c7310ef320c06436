// Gas, stars and sinks through the shmem:: API, compiled unchanged against the reference's
// shmem/tree.h (CPU, oracle/_ref/gas_check) and against the GPU shim (gizmo_shared_memory_b200/
// shim/_build/gas_check); tests/test_dropin.py compares what the two write.
//
//   gas_check STATE OUT
//
// STATE is the bench_treeforce state format (N, then x y z m h vx vy vz as float64).  Particles get
// fixed types (7 in 10 gas, every 37th a sink, the rest stars), gas particles a softening of 0.1 to
// 0.15 (a kernel holding tens of neighbours) and a zeta of the size that makes its pair terms a
// percent-level correction.  The program walks the tree three times: accel_grouped by leaf at
// theta 0.7 without and with sink-direct opening (radius 0.2), and the per-target accel at theta
// 0.5 for every 5th target.  OUT receives the three accelerations (ax, ay, az per walk) as float64.
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
    P.type.resize(N);
    P.zeta.assign(N, 0.0);
    for (size_t i = 0; i < N; ++i) {
        const double u = (double)((i * 2654435761ull) % 1000) / 1000.0;  // fixed, in [0, 1)
        P.type[i] = (i % 37 == 0) ? 5 : ((i % 10 < 7) ? 0 : 4);
        if (P.type[i] == 0) {
            P.soft[i] = 0.1 * (1.0 + 0.5 * u);
            P.zeta[i] = 0.1 * P.m[i] * P.m[i] * P.soft[i] * P.soft[i] * (2.0 * u - 1.0);
        }
    }
    Tree T = build(P);
    std::vector<uint32_t> targets(T.orderbuf.begin(), T.orderbuf.end());
    std::vector<double> out;
    std::vector<double> ax, ay, az;
    for (double rs : {0.0, 0.2}) {
        accel_grouped(T, P, targets, 0.7, 1.0, 0, ax, ay, az, nullptr, nullptr, nullptr, nullptr, nullptr, rs);
        for (auto* a : {&ax, &ay, &az}) out.insert(out.end(), a->begin(), a->end());
    }
    std::vector<uint32_t> sub;
    for (size_t k = 0; k < targets.size(); k += 5) sub.push_back(targets[k]);
    accel(T, P, sub, 0.5, 1.0, ax, ay, az);
    for (auto* a : {&ax, &ay, &az}) out.insert(out.end(), a->begin(), a->end());
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) return 1;
    fwrite(out.data(), 8, out.size(), fo);
    fclose(fo);
    printf("gas_check: %zu targets, %zu values\n", targets.size(), out.size());
    return 0;
}
