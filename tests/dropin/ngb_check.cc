// The neighbour search and the density solve through the shmem:: API, compiled unchanged against
// the reference's shmem/hydro.h (CPU, oracle/_ref/ngb_check) and against the GPU shim
// (gizmo_shared_memory_b200/shim/_build/ngb_check); tests/test_dropin.py compares what the two write.
//
//   ngb_check STATE OUT
//
// STATE is the bench_treeforce state format (N, then x y z m h vx vy vz as float64).  The first
// 70 % of the particles are gas (type 0), the rest stars (type 4).  The program solves the density
// of every gas particle with the neighbour cache, sets the tree's hmax from the converged h, and
// then searches, for every 50th gas particle, both ways: ngb_search at its h and
// ngb_search_reverse (gas neighbours whose own kernel reaches it).  OUT receives, as int64 and
// float64 blocks: the counts, the iteration numbers and the h and rho of the solve, the cache
// (offsets and indices), the gather and reverse lists (offsets and indices), and the
// SHMEM_NGB_COUNT totals of all of it (ngb_counters then hiter_counters; zeros unless the
// variable is set).
#include "hydro.h"

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
    const size_t n_gas = N * 7 / 10;
    P.type.assign(N, 4);
    for (size_t i = 0; i < n_gas; ++i) P.type[i] = 0;
    Tree T = build(P);
    std::vector<uint32_t> targets;
    for (uint32_t q : T.orderbuf)
        if (q < n_gas) targets.push_back(q);
    NeighborCache cache;
    DensityResult R = density(T, P, targets, 32.0, 0.05, {}, 0.0, 3, &cache);
    std::vector<double> h(n_gas, 0.0);
    for (size_t t = 0; t < targets.size(); ++t) h[targets[t]] = R.h[t];
    T.init_hmax(h, n_gas);
    std::vector<int64_t> gstart{0}, rstart{0};
    std::vector<uint32_t> gather, reverse;
    for (size_t t = 0; t < targets.size(); t += 50) {
        const uint32_t p = targets[t];
        const Vec3d c{P.x[p], P.y[p], P.z[p]};
        ngb_search(T, P, c, h[p], gather);
        gstart.push_back((int64_t)gather.size());
        ngb_search_reverse(T, P, h.data(), n_gas, c, h[p], reverse);
        rstart.push_back((int64_t)reverse.size());
    }
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) return 1;
    auto put64 = [&](const std::vector<int64_t>& v) {
        const int64_t k = (int64_t)v.size();
        fwrite(&k, 8, 1, fo);
        fwrite(v.data(), 8, v.size(), fo);
    };
    auto putd = [&](const std::vector<double>& v) {
        const int64_t k = (int64_t)v.size();
        fwrite(&k, 8, 1, fo);
        fwrite(v.data(), 8, v.size(), fo);
    };
    auto putu = [&](const std::vector<uint32_t>& v) {
        std::vector<int64_t> w(v.begin(), v.end());
        put64(w);
    };
    std::vector<int64_t> nngb(R.nngb.begin(), R.nngb.end()), iters(R.iters.begin(), R.iters.end());
    std::vector<int64_t> cstart(cache.start.begin(), cache.start.end());
    put64(nngb); put64(iters); putd(R.h); putd(R.rho);
    put64(cstart); putu(cache.flat);
    put64(gstart); putu(gather);
    put64(rstart); putu(reverse);
    long long c[5], hh[8];
    ngb_counters(c[0], c[1], c[2], c[3], c[4], true);
    hiter_counters(hh, true);
    std::vector<int64_t> counts(c, c + 5);
    counts.insert(counts.end(), hh, hh + 8);
    put64(counts);
    fclose(fo);
    printf("ngb_check: %zu targets, %zu gather, %zu reverse\n", targets.size(), gather.size(), reverse.size());
    return 0;
}
