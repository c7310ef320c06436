/* ORACLE — test infrastructure only (see gt_oracle.h).
 *
 * A CPU restatement of the reference's shared-memory tree-gravity path, written in plain C so it
 * builds anywhere gcc does and can be loaded by the tests on a GPU box where the reference tree is
 * absent.  It is NOT part of the product: the CUDA library never links it, and no product code
 * path calls it.  Every function cites the reference file:line it restates.
 */
#define _GNU_SOURCE
#include "gt_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_LEAF_MAX 16 /* shmem/tree.h:357 */
#define OR_MAX_LEVEL 20 /* shmem/tree.h:358 */

/* ------------------------------------------------------------------------------------------- */
/* Scalar kernels                                                                               */
/* ------------------------------------------------------------------------------------------- */

/* (1/r) dphi/dr of the cubic spline, Newtonian for r >= h.  shmem/tree.h:59-67. */
double or_spline_force_over_r(double r, double h) {
    const double hinv = 1.0 / h;
    const double u = r * hinv;
    if (u >= 1.0) return 1.0 / (r * r * r);
    const double hinv3 = hinv * hinv * hinv;
    if (u < 0.5) return hinv3 * (10.666666666666667 + u * u * (32.0 * u - 38.4));
    return hinv3 * (21.333333333333332 - 48.0 * u + 38.4 * u * u - 10.666666666666667 * u * u * u -
                    0.06666666666666667 / (u * u * u));
}

/* phi(r) of the same spline, -1/r for r >= h.  shmem/tree.h:72-80. */
double or_spline_potential(double r, double h) {
    const double hinv = 1.0 / h;
    const double u = r * hinv;
    if (u >= 1.0) return -1.0 / r;
    if (u < 0.5) return hinv * (-2.8 + u * u * (5.333333333333333 + u * u * (6.4 * u - 9.6)));
    return hinv * (-3.2 + 0.06666666666666667 / u +
                   u * u * (10.666666666666667 + u * (-16.0 + u * (9.6 - 2.1333333333333333 * u))));
}

/* Second-derivative (tidal) factor of the same spline: 3/r^5 for r >= h.  shmem/tree.h:85-96. */
double or_spline_tidal_factor(double r, double h) {
    const double hinv = 1.0 / h;
    const double u = r * hinv;
    if (u >= 1.0) return 3.0 / (r * r * r * r * r);
    const double hinv5 = hinv * hinv * hinv * hinv * hinv;
    const double wk = u < 0.5 ? 76.8 - 96.0 * u : -0.2 / (u * u * u * u * u) + 48.0 / u - 76.8 + 32.0 * u;
    return wk * hinv5;
}

/* Node-opening decision, in the reference's order: softening overlap, Barnes-Hut (theta > 0),
 * relative criterion M L^2 > r^4 aold (aold > 0; with aold == 0 and no theta: open), then the
 * inside-node test.  shmem/tree.h:109-144. */
int or_open_node(double r_sq, double len, double l_open, double node_mass, double node_maxsoft,
                 double soft_target, double aold, double theta_sq, double adx, double ady, double adz) {
    const double reach_t = soft_target + 0.6 * len;
    const double reach_n = node_maxsoft + 0.6 * len;
    if (r_sq < reach_t * reach_t || r_sq < reach_n * reach_n) return 1;
    if (theta_sq > 0.0 && l_open * l_open >= theta_sq * r_sq) return 1;
    if (aold > 0) {
        if (node_mass * len * len > r_sq * r_sq * aold) return 1;
    } else if (theta_sq <= 0.0) {
        return 1;
    }
    const double lim = 0.6 * len;
    return (adx < lim && ady < lim && adz < lim) ? 1 : 0;
}

/* ------------------------------------------------------------------------------------------- */
/* Keys                                                                                         */
/* ------------------------------------------------------------------------------------------- */

/* Morton key of three 21-bit coordinates, x in the lowest bit of each triple.  shmem/tree.h:161-173. */
static uint64_t spread_bits3(uint64_t v) {
    uint64_t out = 0;
    for (int b = 0; b < 21; ++b) out |= ((v >> b) & 1ull) << (3 * b);
    return out;
}
uint64_t or_morton20(uint32_t a, uint32_t b, uint32_t c) {
    return spread_bits3(a) | (spread_bits3(b) << 1) | (spread_bits3(c) << 2);
}

/* Peano-Hilbert state machine of system/peano.cc:192-292 (rottable3 / subpix3), stored as one
 * table: entry = (next_state << 3) | key_digit, indexed [state][pix], pix = 4x + 2y + z. */
static const uint16_t PH_STEP[48][8] = {
    {0x120, 0x0e7, 0x0c9, 0x0de, 0x053, 0x054, 0x0ca, 0x0dd},
    {0x0ef, 0x05c, 0x0c6, 0x0c5, 0x128, 0x05b, 0x0d1, 0x0d2},
    {0x044, 0x043, 0x0cd, 0x0da, 0x0f7, 0x130, 0x0ce, 0x0d9},
    {0x04b, 0x138, 0x0c2, 0x0c1, 0x04c, 0x0ff, 0x0d5, 0x0d6},
    {0x141, 0x0c0, 0x166, 0x107, 0x142, 0x033, 0x165, 0x034},
    {0x0c8, 0x03b, 0x10f, 0x03c, 0x149, 0x14a, 0x16e, 0x16d},
    {0x023, 0x152, 0x024, 0x175, 0x0d0, 0x151, 0x117, 0x176},
    {0x15a, 0x159, 0x17d, 0x17e, 0x02b, 0x0d8, 0x02c, 0x11f},
    {0x10e, 0x119, 0x127, 0x0e0, 0x10d, 0x11a, 0x014, 0x013},
    {0x101, 0x102, 0x0e8, 0x01b, 0x116, 0x115, 0x12f, 0x01c},
    {0x10a, 0x11d, 0x003, 0x004, 0x109, 0x11e, 0x0f0, 0x137},
    {0x105, 0x106, 0x00c, 0x13f, 0x112, 0x111, 0x00b, 0x0f8},
    {0x0c7, 0x156, 0x100, 0x171, 0x074, 0x155, 0x073, 0x172},
    {0x15e, 0x15d, 0x179, 0x17a, 0x0cf, 0x07c, 0x108, 0x07b},
    {0x145, 0x064, 0x162, 0x063, 0x146, 0x0d7, 0x161, 0x110},
    {0x06c, 0x0df, 0x06b, 0x118, 0x14d, 0x14e, 0x16a, 0x169},
    {0x0e6, 0x14f, 0x0e5, 0x0b4, 0x131, 0x158, 0x132, 0x0b3},
    {0x157, 0x140, 0x0bc, 0x0bb, 0x0ee, 0x139, 0x0ed, 0x13a},
    {0x148, 0x121, 0x0a3, 0x122, 0x15f, 0x0f6, 0x0a4, 0x0f5},
    {0x129, 0x0fe, 0x12a, 0x0fd, 0x150, 0x147, 0x0ab, 0x0ac},
    {0x0e2, 0x093, 0x0e1, 0x168, 0x135, 0x094, 0x136, 0x17f},
    {0x09b, 0x09c, 0x170, 0x167, 0x0ea, 0x13d, 0x0e9, 0x13e},
    {0x084, 0x125, 0x16f, 0x126, 0x083, 0x0f2, 0x178, 0x0f1},
    {0x12d, 0x0fa, 0x12e, 0x0f9, 0x08c, 0x08b, 0x177, 0x160},
    {0x067, 0x020, 0x00e, 0x019, 0x114, 0x113, 0x00d, 0x01a},
    {0x028, 0x11b, 0x001, 0x002, 0x06f, 0x11c, 0x016, 0x015},
    {0x103, 0x104, 0x00a, 0x01d, 0x030, 0x077, 0x009, 0x01e},
    {0x10c, 0x07f, 0x005, 0x006, 0x10b, 0x038, 0x012, 0x011},
    {0x086, 0x007, 0x0a1, 0x040, 0x085, 0x0f4, 0x0a2, 0x0f3},
    {0x00f, 0x0fc, 0x048, 0x0fb, 0x08e, 0x08d, 0x0a9, 0x0aa},
    {0x0e4, 0x095, 0x0e3, 0x0b2, 0x017, 0x096, 0x050, 0x0b1},
    {0x09d, 0x09e, 0x0ba, 0x0b9, 0x0ec, 0x01f, 0x0eb, 0x058},
    {0x049, 0x05e, 0x060, 0x027, 0x04a, 0x05d, 0x0d3, 0x0d4},
    {0x046, 0x045, 0x02f, 0x0dc, 0x051, 0x052, 0x068, 0x0db},
    {0x04d, 0x05a, 0x0c4, 0x0c3, 0x04e, 0x059, 0x037, 0x070},
    {0x042, 0x041, 0x0cb, 0x078, 0x055, 0x056, 0x0cc, 0x03f},
    {0x000, 0x091, 0x047, 0x0b6, 0x133, 0x092, 0x134, 0x0b5},
    {0x099, 0x09a, 0x0be, 0x0bd, 0x008, 0x13b, 0x04f, 0x13c},
    {0x082, 0x123, 0x0a5, 0x124, 0x081, 0x010, 0x0a6, 0x057},
    {0x12b, 0x018, 0x12c, 0x05f, 0x08a, 0x089, 0x0ad, 0x0ae},
    {0x021, 0x088, 0x022, 0x173, 0x076, 0x09f, 0x075, 0x174},
    {0x090, 0x087, 0x17b, 0x17c, 0x029, 0x07e, 0x02a, 0x07d},
    {0x08f, 0x066, 0x164, 0x065, 0x098, 0x031, 0x163, 0x032},
    {0x06e, 0x039, 0x06d, 0x03a, 0x097, 0x080, 0x16c, 0x16b},
    {0x025, 0x154, 0x026, 0x0af, 0x072, 0x153, 0x071, 0x0b8},
    {0x15c, 0x15b, 0x0b7, 0x0a0, 0x02d, 0x07a, 0x02e, 0x079},
    {0x143, 0x062, 0x0a8, 0x061, 0x144, 0x035, 0x0bf, 0x036},
    {0x06a, 0x03d, 0x069, 0x03e, 0x14b, 0x14c, 0x0b0, 0x0a7},
};

/* Table-driven Hilbert key, most significant level first.  system/peano.cc:297-313. */
void or_peano_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo) {
    unsigned __int128 key = 0;
    unsigned state = 0;
    for (int b = bits - 1; b >= 0; --b) {
        const unsigned pix = (unsigned)(((x >> b) & 1) << 2 | ((y >> b) & 1) << 1 | ((z >> b) & 1));
        const unsigned step = PH_STEP[state][pix];
        key = (key << 3) | (step & 7u);
        state = step >> 3;
    }
    *hi = (uint64_t)(key >> 64);
    *lo = (uint64_t)key;
}

/* Morton key of the MPI code: z in the top bit of each triple.  system/peano.cc:317-329. */
void or_morton_key(uint64_t x, uint64_t y, uint64_t z, int bits, uint64_t* hi, uint64_t* lo) {
    unsigned __int128 key = 0;
    for (int b = bits - 1; b >= 0; --b)
        key = (key << 3) | (((z >> b) & 1) << 2 | ((y >> b) & 1) << 1 | ((x >> b) & 1));
    *hi = (uint64_t)(key >> 64);
    *lo = (uint64_t)key;
}

/* Mantissa extraction of d in [1,2): the top `bits` fraction bits.  domain/domain.cc:2693-2702. */
uint64_t or_double_to_int(double d, int bits) {
    uint64_t u;
    memcpy(&u, &d, 8);
    return (u & 0xFFFFFFFFFFFFFull) >> (52 - bits);
}

/* Root cell of shmem::build: bbox of live particles, centre, side * 1.0000001, optional
 * randomised root (splitmix64 draw, box doubled).  shmem/tree.cc:355-393. */
typedef struct {
    double cx, cy, cz, side, scale;
} or_geom;

static or_geom root_geometry(int64_t n, const double* x, const double* y, const double* z,
                             const double* m, long long randomize_seed) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < n; ++i) {
        if (!(m[i] > 0)) continue;
        if (x[i] < lo[0]) lo[0] = x[i];
        if (x[i] > hi[0]) hi[0] = x[i];
        if (y[i] < lo[1]) lo[1] = y[i];
        if (y[i] > hi[1]) hi[1] = y[i];
        if (z[i] < lo[2]) lo[2] = z[i];
        if (z[i] > hi[2]) hi[2] = z[i];
    }
    or_geom g;
    g.cx = 0.5 * (lo[0] + hi[0]);
    g.cy = 0.5 * (lo[1] + hi[1]);
    g.cz = 0.5 * (lo[2] + hi[2]);
    double ext = hi[0] - lo[0];
    if (hi[1] - lo[1] > ext) ext = hi[1] - lo[1];
    if (hi[2] - lo[2] > ext) ext = hi[2] - lo[2];
    g.side = ext * 1.0000001;
    if (g.side <= 0) g.side = 1.0;
    if (randomize_seed >= 0) {
        uint64_t s = (uint64_t)randomize_seed * 0x9E3779B97F4A7C15ull;
        double draw[3];
        for (int k = 0; k < 3; ++k) {
            s += 0x9E3779B97F4A7C15ull;
            uint64_t v = s;
            v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
            v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
            draw[k] = (double)((v ^ (v >> 31)) >> 11) * (1.0 / 9007199254740992.0);
        }
        g.cx += g.side * (draw[0] - 0.5);
        g.cy += g.side * (draw[1] - 0.5);
        g.cz += g.side * (draw[2] - 0.5);
        g.side *= 2.0;
    }
    g.scale = (double)((1u << OR_MAX_LEVEL) - 1) / g.side;
    return g;
}

/* 20-bit quantisation of shmem/tree.cc:409-418. */
static void quantise20(const or_geom* g, double x, double y, double z, uint32_t* a, uint32_t* b,
                       uint32_t* c) {
    *a = (uint32_t)((x - (g->cx - 0.5 * g->side)) * g->scale);
    *b = (uint32_t)((y - (g->cy - 0.5 * g->side)) * g->scale);
    *c = (uint32_t)((z - (g->cz - 0.5 * g->side)) * g->scale);
}

void or_keys20(int64_t n, const double* x, const double* y, const double* z, const double* m,
               int key_mode, long long randomize_seed, uint64_t* keys, double* geom_out) {
    const or_geom g = root_geometry(n, x, y, z, m, randomize_seed);
    if (geom_out) {
        geom_out[0] = g.cx; geom_out[1] = g.cy; geom_out[2] = g.cz;
        geom_out[3] = g.side; geom_out[4] = g.scale;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (!(m[i] > 0)) { keys[i] = 1ull << 60; continue; }
        uint32_t a, b, c;
        quantise20(&g, x[i], y[i], z[i], &a, &b, &c);
        if (key_mode == 0) {
            keys[i] = or_morton20(a, b, c);
        } else {
            uint64_t hi, lo;
            or_peano_key(a, b, c, OR_MAX_LEVEL, &hi, &lo);
            keys[i] = lo;
        }
    }
}

/* ------------------------------------------------------------------------------------------- */
/* Tree                                                                                         */
/* ------------------------------------------------------------------------------------------- */

struct or_tree {
    int64_t n, nlive, nnodes, cap;
    int root;
    const double *x, *y, *z, *m, *soft; /* borrowed: the caller keeps them alive */
    double *cx, *cy, *cz, *mass, *size, *delta, *nsoft, *gcx, *gcy, *gcz, *w_s;
    float *w_len, *w_soft;
    int *first, *next, *plo, *phi, *parent, *level;
    uint32_t* order;
    uint32_t* rank;
    int* leaf_of;
    uint64_t* skey;
};

typedef struct {
    uint64_t key;
    uint32_t idx;
} key_idx;

static int cmp_key_idx(const void* a, const void* b) {
    const key_idx* p = (const key_idx*)a;
    const key_idx* q = (const key_idx*)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

static int claim_node(or_tree* t) {
    if (t->nnodes >= t->cap) {
        t->cap = t->cap * 2 + 1024;
#define GROW(a, T) t->a = (T*)realloc(t->a, (size_t)t->cap * sizeof(T))
        GROW(cx, double); GROW(cy, double); GROW(cz, double); GROW(mass, double);
        GROW(size, double); GROW(delta, double); GROW(nsoft, double); GROW(gcx, double);
        GROW(gcy, double); GROW(gcz, double); GROW(w_s, double); GROW(w_len, float);
        GROW(w_soft, float); GROW(first, int); GROW(next, int); GROW(plo, int); GROW(phi, int);
        GROW(parent, int); GROW(level, int);
#undef GROW
    }
    return (int)t->nnodes++;
}

/* Recursive octant split of a key-sorted range: leaf at <= LEAF_MAX particles or level 20;
 * children in octant order; moments from particles (leaf) or from children (interior).
 * shmem/tree.cc:70-197.  Serial, so node numbering is the preorder the reference produces when
 * it runs without tasks. */
static int build_cell(or_tree* t, int lo, int hi, int lvl, double ccx, double ccy, double ccz,
                      double sz) {
    const int me = claim_node(t);
    t->size[me] = sz; t->first[me] = -1; t->next[me] = -1; t->plo[me] = lo; t->phi[me] = hi;
    t->parent[me] = -1; t->level[me] = lvl;
    t->gcx[me] = ccx; t->gcy[me] = ccy; t->gcz[me] = ccz;
    int kids[8], nk = 0;
    if (!(hi - lo <= OR_LEAF_MAX || lvl >= OR_MAX_LEVEL)) {
        const int shift = 3 * (OR_MAX_LEVEL - lvl - 1);
        const double half = sz * 0.5, quarter = sz * 0.25;
        int at = lo;
        for (int oct = 0; oct < 8; ++oct) {
            const int a = at;
            while (at < hi && (int)((t->skey[at] >> shift) & 7ull) == oct) ++at;
            if (at == a) continue;
            const double ox = ccx + ((oct & 1) ? quarter : -quarter);
            const double oy = ccy + ((oct & 2) ? quarter : -quarter);
            const double oz = ccz + ((oct & 4) ? quarter : -quarter);
            kids[nk++] = build_cell(t, a, at, lvl + 1, ox, oy, oz, half);
        }
        for (int k = 0; k < nk; ++k) {
            t->parent[kids[k]] = me;
            t->next[kids[k]] = (k + 1 < nk) ? kids[k + 1] : -1;
        }
        if (nk > 0) t->first[me] = kids[0];
    }
    double M = 0, sx = 0, sy = 0, sz_ = 0, smax = 0;
    if (nk == 0) {
        for (int i = lo; i < hi; ++i) {
            const uint32_t p = t->order[i];
            const double mp = t->m[p];
            M += mp; sx += mp * t->x[p]; sy += mp * t->y[p]; sz_ += mp * t->z[p];
            if (t->soft && t->soft[p] > smax) smax = t->soft[p];
            t->leaf_of[p] = me;
        }
    } else {
        for (int k = 0; k < nk; ++k) {
            const int c = kids[k];
            const double mc = t->mass[c];
            M += mc; sx += mc * t->cx[c]; sy += mc * t->cy[c]; sz_ += mc * t->cz[c];
            if (t->nsoft[c] > smax) smax = t->nsoft[c];
        }
    }
    if (M > 0) { sx /= M; sy /= M; sz_ /= M; }
    t->mass[me] = M; t->cx[me] = sx; t->cy[me] = sy; t->cz[me] = sz_; t->nsoft[me] = smax;
    const double dx = sx - ccx, dy = sy - ccy, dz = sz_ - ccz;
    t->delta[me] = sqrt(dx * dx + dy * dy + dz * dz);
    return me;
}

/* next[] threading: a node's last child falls through to the node's own next.  shmem/tree.cc:340-348. */
static void thread_walk(or_tree* t, int node, int next_sib) {
    t->next[node] = next_sib;
    for (int c = t->first[node]; c >= 0;) {
        const int sib = t->next[c];
        thread_walk(t, c, sib >= 0 ? sib : next_sib);
        c = sib;
    }
}

or_tree* or_build(int64_t n, const double* x, const double* y, const double* z, const double* m,
                  const double* soft, long long randomize_seed, int nodelta) {
    or_tree* t = (or_tree*)calloc(1, sizeof(or_tree));
    t->n = n; t->x = x; t->y = y; t->z = z; t->m = m; t->soft = soft;
    uint64_t* keys = (uint64_t*)malloc((size_t)(n > 0 ? n : 1) * 8);
    or_keys20(n, x, y, z, m, 0, randomize_seed, keys, NULL);
    const or_geom g = root_geometry(n, x, y, z, m, randomize_seed);
    /* live particles (m > 0), sorted by key; ties keep index order */
    key_idx* ki = (key_idx*)malloc((size_t)(n > 0 ? n : 1) * sizeof(key_idx));
    int64_t nl = 0;
    for (int64_t i = 0; i < n; ++i)
        if (m[i] > 0) { ki[nl].key = keys[i]; ki[nl].idx = (uint32_t)i; ++nl; }
    qsort(ki, (size_t)nl, sizeof(key_idx), cmp_key_idx);
    t->nlive = nl;
    t->order = (uint32_t*)malloc((size_t)(nl > 0 ? nl : 1) * 4);
    t->skey = (uint64_t*)malloc((size_t)(nl > 0 ? nl : 1) * 8);
    for (int64_t r = 0; r < nl; ++r) { t->order[r] = ki[r].idx; t->skey[r] = ki[r].key; }
    free(ki);
    free(keys);
    t->leaf_of = (int*)malloc((size_t)(n > 0 ? n : 1) * 4);
    for (int64_t i = 0; i < n; ++i) t->leaf_of[i] = -1;
    t->rank = (uint32_t*)malloc((size_t)(n > 0 ? n : 1) * 4);
    for (int64_t i = 0; i < n; ++i) t->rank[i] = UINT32_MAX;
    for (int64_t r = 0; r < nl; ++r) t->rank[t->order[r]] = (uint32_t)r;
    t->cap = 0; t->nnodes = 0;
    t->root = build_cell(t, 0, (int)nl, 0, g.cx, g.cy, g.cz, g.side);
    thread_walk(t, t->root, -1);
    for (int64_t i = 0; i < t->nnodes; ++i) {
        /* packed walk node, shmem/tree.cc:507-523 (nodelta: SHMEM_TREE_NODELTA, tree.cc:512-519) */
        t->w_s[i] = t->size[i] + (nodelta ? 0.0 : t->delta[i]);
        t->w_len[i] = (float)t->size[i];
        t->w_soft[i] = (float)t->nsoft[i];
    }
    return t;
}

void or_free(or_tree* t) {
    if (!t) return;
    free(t->cx); free(t->cy); free(t->cz); free(t->mass); free(t->size); free(t->delta);
    free(t->nsoft); free(t->gcx); free(t->gcy); free(t->gcz); free(t->w_s); free(t->w_len);
    free(t->w_soft); free(t->first); free(t->next); free(t->plo); free(t->phi); free(t->parent);
    free(t->level); free(t->order); free(t->rank); free(t->leaf_of); free(t->skey);
    free(t);
}

int64_t or_nnodes(const or_tree* t) { return t->nnodes; }
int64_t or_nlive(const or_tree* t) { return t->nlive; }
int or_root(const or_tree* t) { return t->root; }

void or_nodes(const or_tree* t, double* cx, double* cy, double* cz, double* mass, double* size,
              double* delta, double* soft, double* gcx, double* gcy, double* gcz, int* first,
              int* next, int* plo, int* phi, int* parent, int* level, double* w_s, float* w_len,
              float* w_soft) {
    const size_t nn = (size_t)t->nnodes;
#define CP(dst, src, sz) if (dst) memcpy(dst, t->src, nn * sz)
    CP(cx, cx, 8); CP(cy, cy, 8); CP(cz, cz, 8); CP(mass, mass, 8); CP(size, size, 8);
    CP(delta, delta, 8); CP(soft, nsoft, 8); CP(gcx, gcx, 8); CP(gcy, gcy, 8); CP(gcz, gcz, 8);
    CP(first, first, 4); CP(next, next, 4); CP(plo, plo, 4); CP(phi, phi, 4);
    CP(parent, parent, 4); CP(level, level, 4); CP(w_s, w_s, 8); CP(w_len, w_len, 4);
    CP(w_soft, w_soft, 4);
#undef CP
}

void or_order(const or_tree* t, uint32_t* orderbuf, uint32_t* rank, int* leaf_of) {
    if (orderbuf) memcpy(orderbuf, t->order, (size_t)t->nlive * 4);
    if (rank) memcpy(rank, t->rank, (size_t)t->n * 4);
    if (leaf_of) memcpy(leaf_of, t->leaf_of, (size_t)t->n * 4);
}

/* ------------------------------------------------------------------------------------------- */
/* Walks                                                                                        */
/* ------------------------------------------------------------------------------------------- */

/* Leaf groups: a new group wherever leaf_of changes or is -1 (tree.cc:656-667); fixed windows of
 * `batch` consecutive targets otherwise (tree.cc:668-681). */
int64_t or_groups(const or_tree* t, int64_t nt, const uint32_t* targets, int batch, int64_t* starts) {
    int64_t ng = 0;
    if (nt <= 0) { starts[0] = 0; return 0; }
    if (batch <= 0) {
        starts[ng++] = 0;
        for (int64_t i = 1; i < nt; ++i) {
            const int li = t->leaf_of[targets[i]], lp = t->leaf_of[targets[i - 1]];
            if (li != lp || li < 0) starts[ng++] = i;
        }
    } else {
        for (int64_t i = 0; i < nt; i += batch) starts[ng++] = i;
    }
    starts[ng] = nt;
    return ng;
}

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

/* One walk per group over the threaded tree: bbox-nearest-point opening with the group's
 * largest softening and smallest aold, P-P sums over opened leaves (self and r == 0 skipped,
 * kernel of the larger softening), P-N monopoles otherwise.  shmem/tree.cc:678-888 (grouped),
 * tree.cc:538-581 and 905-943 (leaf_accept = 0, the per-target walks). */
void or_walk_groups(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                    const int64_t* starts, double theta, double G, const double* aold,
                    int leaf_accept, double* ax, double* ay, double* az, double* phi,
                    int64_t* counters) {
    const double theta2 = theta * theta;
    long long c_nodes = 0, c_multi = 0, c_pairs = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : c_nodes, c_multi, c_pairs)
    for (int64_t g = 0; g < ngroups; ++g) {
        const int64_t lo = starts[g], hi = starts[g + 1];
        const int nb = (int)(hi - lo);
        double b0[3] = {1e300, 1e300, 1e300}, b1[3] = {-1e300, -1e300, -1e300}, emax = 0;
        double amin = aold ? 1e300 : 0.0;
        double* tx = (double*)malloc((size_t)nb * 8 * 8);
        double *ty = tx + nb, *tz = tx + 2 * nb, *te = tx + 3 * nb;
        double *oax = tx + 4 * nb, *oay = tx + 5 * nb, *oaz = tx + 6 * nb, *oph = tx + 7 * nb;
        for (int i = 0; i < nb; ++i) {
            const uint32_t p = targets[lo + i];
            tx[i] = t->x[p]; ty[i] = t->y[p]; tz[i] = t->z[p];
            te[i] = t->soft ? t->soft[p] : 0.0;
            b0[0] = dmin(b0[0], tx[i]); b1[0] = dmax(b1[0], tx[i]);
            b0[1] = dmin(b0[1], ty[i]); b1[1] = dmax(b1[1], ty[i]);
            b0[2] = dmin(b0[2], tz[i]); b1[2] = dmax(b1[2], tz[i]);
            emax = dmax(emax, te[i]);
            if (aold) amin = dmin(amin, aold[lo + i]);
            oax[i] = oay[i] = oaz[i] = oph[i] = 0.0;
        }
        int node = t->root;
        while (node >= 0) {
            ++c_nodes;
            const double ncx = t->cx[node], ncy = t->cy[node], ncz = t->cz[node];
            const double dx = dmax(0.0, dmax(b0[0] - ncx, ncx - b1[0]));
            const double dy = dmax(0.0, dmax(b0[1] - ncy, ncy - b1[1]));
            const double dz = dmax(0.0, dmax(b0[2] - ncz, ncz - b1[2]));
            const double rmin2 = dx * dx + dy * dy + dz * dz;
            const int is_leaf = t->first[node] < 0;
            int accept;
            if (leaf_accept || !is_leaf)
                accept = !or_open_node(rmin2, (double)t->w_len[node], t->w_s[node], t->mass[node],
                                       (double)t->w_soft[node], emax, amin, theta2, dx, dy, dz);
            else
                accept = 0;
            if (accept) {
                /* monopole with the softening max(target, node) */
                c_multi += nb;
                const double nm = t->mass[node];
                for (int i = 0; i < nb; ++i) {
                    const double ox = ncx - tx[i], oy = ncy - ty[i], oz = ncz - tz[i];
                    const double r2 = ox * ox + oy * oy + oz * oz;
                    if (r2 <= 0) continue;
                    const double r = sqrt(r2);
                    const double e = dmax(dmax(te[i], (double)t->w_soft[node]), 1e-300);
                    const double f = nm * or_spline_force_over_r(r, e);
                    oax[i] += ox * f; oay[i] += oy * f; oaz[i] += oz * f;
                    oph[i] += nm * or_spline_potential(r, e);
                }
                node = t->next[node];
            } else if (is_leaf) {
                for (int k = t->plo[node]; k < t->phi[node]; ++k) {
                    const uint32_t q = t->order[k];
                    const double qx = t->x[q], qy = t->y[q], qz = t->z[q], qm = t->m[q];
                    const double qs = t->soft ? t->soft[q] : 0.0;
                    for (int i = 0; i < nb; ++i) {
                        if (targets[lo + i] == q) continue;
                        const double ox = qx - tx[i], oy = qy - ty[i], oz = qz - tz[i];
                        const double r2 = ox * ox + oy * oy + oz * oz;
                        if (r2 <= 0) continue;
                        ++c_pairs;
                        const double r = sqrt(r2);
                        const double e = dmax(dmax(te[i], qs), 1e-300);
                        const double f = qm * or_spline_force_over_r(r, e);
                        oax[i] += ox * f; oay[i] += oy * f; oaz[i] += oz * f;
                        oph[i] += qm * or_spline_potential(r, e);
                    }
                }
                node = t->next[node];
            } else {
                node = t->first[node];
            }
        }
        for (int i = 0; i < nb; ++i) {
            if (ax) ax[lo + i] = G * oax[i];
            if (ay) ay[lo + i] = G * oay[i];
            if (az) az[lo + i] = G * oaz[i];
            if (phi) phi[lo + i] = G * oph[i];
        }
        free(tx);
    }
    if (counters) { counters[0] = c_nodes; counters[1] = c_multi; counters[2] = c_pairs; }
}

void or_accel_grouped(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
                      int batch, const double* aold, double* ax, double* ay, double* az,
                      int64_t* counters) {
    int64_t* starts = (int64_t*)malloc((size_t)(nt + 1) * 8);
    const int64_t ng = or_groups(t, nt, targets, batch, starts);
    or_walk_groups(t, nt, targets, ng, starts, theta, G, aold, 1, ax, ay, az, NULL, counters);
    free(starts);
}

static int64_t* singleton_groups(int64_t nt) {
    int64_t* s = (int64_t*)malloc((size_t)(nt + 1) * 8);
    for (int64_t i = 0; i <= nt; ++i) s[i] = i;
    return s;
}

void or_accel(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
              const double* aold, double* ax, double* ay, double* az) {
    int64_t* s = singleton_groups(nt);
    or_walk_groups(t, nt, targets, nt, s, theta, G, aold, 0, ax, ay, az, NULL, NULL);
    free(s);
}

void or_potential(const or_tree* t, int64_t nt, const uint32_t* targets, double theta, double G,
                  const double* aold, double* phi) {
    int64_t* s = singleton_groups(nt);
    or_walk_groups(t, nt, targets, nt, s, theta, G, aold, 0, NULL, NULL, NULL, phi, NULL);
    free(s);
}

/* FP64 direct sum with the walk's pair rule (kernel of max(eps_i, eps_j), self and r == 0
 * skipped).  shmem/tree.cc:946-971. */
void or_direct(int64_t n, const double* x, const double* y, const double* z, const double* m,
               const double* soft, int64_t nt, const uint32_t* targets, double G, double* ax,
               double* ay, double* az, double* phi) {
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nt; ++k) {
        const uint32_t p = targets[k];
        const double px = x[p], py = y[p], pz = z[p], ep = soft ? soft[p] : 0.0;
        double sx = 0, sy = 0, sz = 0, sp = 0;
        for (int64_t q = 0; q < n; ++q) {
            if (q == (int64_t)p) continue;
            const double ox = x[q] - px, oy = y[q] - py, oz = z[q] - pz;
            const double r = sqrt(ox * ox + oy * oy + oz * oz);
            if (r <= 0) continue;
            const double e = dmax(dmax(ep, soft ? soft[q] : 0.0), 1e-300);
            const double f = m[q] * or_spline_force_over_r(r, e);
            sx += ox * f; sy += oy * f; sz += oz * f;
            sp += m[q] * or_spline_potential(r, e);
        }
        if (ax) ax[k] = G * sx;
        if (ay) ay[k] = G * sy;
        if (az) az[k] = G * sz;
        if (phi) phi[k] = G * sp;
    }
}

/* Per-node centre-of-mass velocity and speed bound, from the particles of a leaf and from the
 * children of an interior node (shmem/tree.cc:149-190, built when velocities are supplied).
 * Nodes are numbered in preorder, so every child comes after its parent: one reverse sweep. */
void or_velocity_moments(const or_tree* t, const double* vx, const double* vy, const double* vz,
                         double* vcx, double* vcy, double* vcz, float* vmax) {
    for (int64_t i = t->nnodes - 1; i >= 0; --i) {
        double M = 0, px = 0, py = 0, pz = 0, vm = 0;
        if (t->first[i] < 0) {
            for (int k = t->plo[i]; k < t->phi[i]; ++k) {
                const uint32_t p = t->order[k];
                const double m = t->m[p];
                const double v = sqrt(vx[p] * vx[p] + vy[p] * vy[p] + vz[p] * vz[p]);
                if (v > vm) vm = v;
                M += m; px += m * vx[p]; py += m * vy[p]; pz += m * vz[p];
            }
        } else {
            for (int c = t->first[i]; c >= 0 && t->parent[c] == i; c = t->next[c]) {
                const double m = t->mass[c];
                if ((double)vmax[c] > vm) vm = (double)vmax[c];
                M += m; px += m * vcx[c]; py += m * vcy[c]; pz += m * vcz[c];
            }
        }
        vmax[i] = (float)vm;
        vcx[i] = M > 0 ? px / M : 0.0;
        vcy[i] = M > 0 ? py / M : 0.0;
        vcz[i] = M > 0 ? pz / M : 0.0;
    }
}

/* The grouped walk of or_walk_groups (leaf_accept = 1) with the tidal tensor and the jerk:
 * every P-P and P-N interaction adds T += -g1 I + g2 d d and J += g1 dv - (dv.d) g2 d, with g1
 * the zeta-free force factor and g2 the tidal factor of the same softening, d = source - target
 * and dv = v_source - v_target (particles' own velocities, nodes' centre-of-mass velocities).
 * tidal (6 per target, xx yy zz xy yz xz) is not multiplied by G, jerk (3 per target) is.
 * shmem/tree.cc:811-837, 845-880. */
void or_walk_groups_ext(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                        const int64_t* starts, double theta, double G, const double* aold,
                        const double* vx, const double* vy, const double* vz, const double* vcx,
                        const double* vcy, const double* vcz, double* ax, double* ay, double* az,
                        double* tidal, double* jerk) {
    const double theta2 = theta * theta;
    const int wj = jerk != NULL;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < ngroups; ++g) {
        const int64_t lo = starts[g], hi = starts[g + 1];
        const int nb = (int)(hi - lo);
        double b0[3] = {1e300, 1e300, 1e300}, b1[3] = {-1e300, -1e300, -1e300}, emax = 0;
        double amin = aold ? 1e300 : 0.0;
        double* buf = (double*)calloc((size_t)nb * 19, 8);
        double *tx = buf, *ty = buf + nb, *tz = buf + 2 * nb, *te = buf + 3 * nb;
        double *tvx = buf + 4 * nb, *tvy = buf + 5 * nb, *tvz = buf + 6 * nb;
        double *oax = buf + 7 * nb, *oay = buf + 8 * nb, *oaz = buf + 9 * nb;
        double* ot = buf + 10 * nb; /* 6 * nb */
        double* oj = buf + 16 * nb; /* 3 * nb */
        for (int i = 0; i < nb; ++i) {
            const uint32_t p = targets[lo + i];
            tx[i] = t->x[p]; ty[i] = t->y[p]; tz[i] = t->z[p];
            te[i] = t->soft ? t->soft[p] : 0.0;
            if (wj) { tvx[i] = vx[p]; tvy[i] = vy[p]; tvz[i] = vz[p]; }
            b0[0] = dmin(b0[0], tx[i]); b1[0] = dmax(b1[0], tx[i]);
            b0[1] = dmin(b0[1], ty[i]); b1[1] = dmax(b1[1], ty[i]);
            b0[2] = dmin(b0[2], tz[i]); b1[2] = dmax(b1[2], tz[i]);
            emax = dmax(emax, te[i]);
            if (aold) amin = dmin(amin, aold[lo + i]);
        }
        int node = t->root;
        while (node >= 0) {
            const double ncx = t->cx[node], ncy = t->cy[node], ncz = t->cz[node];
            const double dx = dmax(0.0, dmax(b0[0] - ncx, ncx - b1[0]));
            const double dy = dmax(0.0, dmax(b0[1] - ncy, ncy - b1[1]));
            const double dz = dmax(0.0, dmax(b0[2] - ncz, ncz - b1[2]));
            const int is_leaf = t->first[node] < 0;
            const int accept = !or_open_node(dx * dx + dy * dy + dz * dz, (double)t->w_len[node], t->w_s[node],
                                             t->mass[node], (double)t->w_soft[node], emax, amin, theta2, dx, dy, dz);
            if (accept || is_leaf) {
                const int kb = accept ? -1 : t->plo[node], ke = accept ? 0 : t->phi[node];
                for (int k = kb; k < ke; ++k) {
                    /* k == -1: the node as a monopole; otherwise the leaf's particle k */
                    uint32_t q = 0;
                    double qx, qy, qz, qm, qs, qvx = 0, qvy = 0, qvz = 0;
                    if (k < 0) {
                        qx = ncx; qy = ncy; qz = ncz; qm = t->mass[node]; qs = (double)t->w_soft[node];
                        if (wj) { qvx = vcx[node]; qvy = vcy[node]; qvz = vcz[node]; }
                    } else {
                        q = t->order[k];
                        qx = t->x[q]; qy = t->y[q]; qz = t->z[q]; qm = t->m[q];
                        qs = t->soft ? t->soft[q] : 0.0;
                        if (wj) { qvx = vx[q]; qvy = vy[q]; qvz = vz[q]; }
                    }
                    for (int i = 0; i < nb; ++i) {
                        if (k >= 0 && targets[lo + i] == q) continue;
                        const double ox = qx - tx[i], oy = qy - ty[i], oz = qz - tz[i];
                        const double r2 = ox * ox + oy * oy + oz * oz;
                        if (r2 <= 0) continue;
                        const double r = sqrt(r2);
                        const double e = dmax(dmax(te[i], qs), 1e-300);
                        const double g1 = qm * or_spline_force_over_r(r, e);
                        const double g2 = qm * or_spline_tidal_factor(r, e);
                        oax[i] += ox * g1; oay[i] += oy * g1; oaz[i] += oz * g1;
                        if (tidal) {
                            ot[6 * i + 0] += -g1 + ox * ox * g2;
                            ot[6 * i + 1] += -g1 + oy * oy * g2;
                            ot[6 * i + 2] += -g1 + oz * oz * g2;
                            ot[6 * i + 3] += ox * oy * g2;
                            ot[6 * i + 4] += oy * oz * g2;
                            ot[6 * i + 5] += ox * oz * g2;
                        }
                        if (wj) {
                            const double dvx = qvx - tvx[i], dvy = qvy - tvy[i], dvz = qvz - tvz[i];
                            const double vdr = dvx * ox + dvy * oy + dvz * oz;
                            oj[3 * i + 0] += g1 * dvx - vdr * g2 * ox;
                            oj[3 * i + 1] += g1 * dvy - vdr * g2 * oy;
                            oj[3 * i + 2] += g1 * dvz - vdr * g2 * oz;
                        }
                    }
                }
                node = t->next[node];
            } else {
                node = t->first[node];
            }
        }
        for (int i = 0; i < nb; ++i) {
            if (ax) { ax[lo + i] = G * oax[i]; ay[lo + i] = G * oay[i]; az[lo + i] = G * oaz[i]; }
            if (tidal) for (int c = 0; c < 6; ++c) tidal[6 * (lo + i) + c] = ot[6 * i + c];
            if (wj) for (int c = 0; c < 3; ++c) jerk[3 * (lo + i) + c] = G * oj[3 * i + c];
        }
        free(buf);
    }
}

/* dW/dr of the 3-D cubic-spline kernel at fixed h (shmem/hydro.h:28-32, 46-54): norm 8/(pi h^3),
 * fp(q) = -12 q + 18 q^2 below q = 1/2 and -6 (1-q)^2 above, zero from q = 1. */
double or_kernel_dwdr(double r, double h) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = 8.0 / (M_PI * h * h * h);
    double fp;
    if (q < 0.5) {
        fp = -12.0 * q + 18.0 * q * q;
    } else {
        const double u = 1.0 - q;
        fp = -6.0 * u * u;
    }
    return norm * fp / h;
}

/* Particle-particle force factor under adaptive gas softening (shmem/tree.cc:39-53): the spline
 * of the larger softening, and for a gas-gas pair with a massive target the two zeta terms (the
 * target's on the pair softening, the source's on its own), each only inside its kernel and
 * divided by the target's mass. */
static double or_pair_fac(double r, double qm, double te, double qs, double zt, double zq, double mt,
                          int gas_gas) {
    const double e = dmax(dmax(te, qs), 1e-300);
    double fac = qm * or_spline_force_over_r(r, e);
    if (!gas_gas || mt <= 0) return fac;
    const double es = dmax(qs, 1e-300);
    if (zt != 0.0 && r < e) fac -= (zt / mt) * or_kernel_dwdr(r, e) / r;
    if (zq != 0.0 && r < es) fac -= (zq / mt) * or_kernel_dwdr(r, es) / r;
    return fac;
}

/* Walk of explicit groups with the gas pair rule and sink-direct opening.  type (GIZMO numbering,
 * 0 = gas, 5 = sink; null = every particle gas) and zeta (null = 0) are indexed like the build's
 * particles.  leaf_accept = 1 is accel_grouped (tree.cc:626-897): a group holding a sink opens
 * every node the criterion accepted that holds a sink and whose box comes within
 * sink_radius + 0.6 len of the group's box (tree.cc:691-698, 772-778); leaf_accept = 0 is the
 * per-target accel (tree.cc:528-582), with no sink rule. */
void or_walk_groups_gas(const or_tree* t, int64_t nt, const uint32_t* targets, int64_t ngroups,
                        const int64_t* starts, double theta, double G, const double* aold,
                        const uint8_t* type, const double* zeta, double sink_radius, int leaf_accept,
                        double* ax, double* ay, double* az) {
    const double theta2 = theta * theta;
    (void)nt;
    /* sinks below each node: a prefix count over the tree order (a node owns [plo, phi)) */
    int64_t* pre = (int64_t*)calloc((size_t)t->nlive + 1, sizeof(int64_t));
    for (int64_t k = 0; k < t->nlive; ++k) pre[k + 1] = pre[k] + (type && type[t->order[k]] == 5);
    const int sink_direct = sink_radius > 0.0 && type != NULL && leaf_accept;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < ngroups; ++g) {
        const int64_t lo = starts[g], hi = starts[g + 1];
        const int nb = (int)(hi - lo);
        double b0[3] = {1e300, 1e300, 1e300}, b1[3] = {-1e300, -1e300, -1e300}, emax = 0;
        double amin = aold ? 1e300 : 0.0;
        int has_sink = 0;
        double* buf = (double*)calloc((size_t)nb * 9, 8);
        double *tx = buf, *ty = buf + nb, *tz = buf + 2 * nb, *te = buf + 3 * nb;
        double *tm = buf + 4 * nb, *tzeta = buf + 5 * nb;
        double *oax = buf + 6 * nb, *oay = buf + 7 * nb, *oaz = buf + 8 * nb;
        char* tgas = (char*)calloc((size_t)nb, 1);
        for (int i = 0; i < nb; ++i) {
            const uint32_t p = targets[lo + i];
            tx[i] = t->x[p]; ty[i] = t->y[p]; tz[i] = t->z[p];
            te[i] = t->soft ? t->soft[p] : 0.0;
            tm[i] = t->m[p];
            tzeta[i] = zeta ? zeta[p] : 0.0;
            tgas[i] = type == NULL || type[p] == 0;
            if (sink_direct && type[p] == 5) has_sink = 1;
            b0[0] = dmin(b0[0], tx[i]); b1[0] = dmax(b1[0], tx[i]);
            b0[1] = dmin(b0[1], ty[i]); b1[1] = dmax(b1[1], ty[i]);
            b0[2] = dmin(b0[2], tz[i]); b1[2] = dmax(b1[2], tz[i]);
            emax = dmax(emax, te[i]);
            if (aold) amin = dmin(amin, aold[lo + i]);
        }
        int node = t->root;
        while (node >= 0) {
            const double ncx = t->cx[node], ncy = t->cy[node], ncz = t->cz[node];
            const double dx = dmax(0.0, dmax(b0[0] - ncx, ncx - b1[0]));
            const double dy = dmax(0.0, dmax(b0[1] - ncy, ncy - b1[1]));
            const double dz = dmax(0.0, dmax(b0[2] - ncz, ncz - b1[2]));
            const double r2n = dx * dx + dy * dy + dz * dz;
            const int is_leaf = t->first[node] < 0;
            int accept = 0;
            if (leaf_accept || !is_leaf)
                accept = !or_open_node(r2n, (double)t->w_len[node], t->w_s[node], t->mass[node],
                                       (double)t->w_soft[node], emax, amin, theta2, dx, dy, dz);
            if (accept && has_sink && pre[t->phi[node]] > pre[t->plo[node]]) {
                const double reach = sink_radius + 0.6 * (double)t->w_len[node];
                if (r2n < reach * reach) accept = 0;
            }
            if (accept || is_leaf) {
                if (accept) {
                    for (int i = 0; i < nb; ++i) {
                        const double ox = ncx - tx[i], oy = ncy - ty[i], oz = ncz - tz[i];
                        const double r2 = ox * ox + oy * oy + oz * oz;
                        if (r2 <= 0) continue;
                        const double f = t->mass[node] *
                                         or_spline_force_over_r(sqrt(r2), dmax(dmax(te[i], (double)t->w_soft[node]), 1e-300));
                        oax[i] += ox * f; oay[i] += oy * f; oaz[i] += oz * f;
                    }
                } else {
                    for (int k = t->plo[node]; k < t->phi[node]; ++k) {
                        const uint32_t q = t->order[k];
                        const double qx = t->x[q], qy = t->y[q], qz = t->z[q], qm = t->m[q];
                        const double qs = t->soft ? t->soft[q] : 0.0;
                        const double zq = zeta ? zeta[q] : 0.0;
                        const int qgas = type == NULL || type[q] == 0;
                        for (int i = 0; i < nb; ++i) {
                            if (targets[lo + i] == q) continue;
                            const double ox = qx - tx[i], oy = qy - ty[i], oz = qz - tz[i];
                            const double r2 = ox * ox + oy * oy + oz * oz;
                            if (r2 <= 0) continue;
                            const double f = or_pair_fac(sqrt(r2), qm, te[i], qs, tzeta[i], zq, tm[i], tgas[i] && qgas);
                            oax[i] += ox * f; oay[i] += oy * f; oaz[i] += oz * f;
                        }
                    }
                }
                node = t->next[node];
            } else {
                node = t->first[node];
            }
        }
        for (int i = 0; i < nb; ++i) {
            ax[lo + i] = G * oax[i]; ay[lo + i] = G * oay[i]; az[lo + i] = G * oaz[i];
        }
        free(tgas);
        free(buf);
    }
    free(pre);
}

/* accel_brute with the gas pair rule (tree.cc:946-971, 39-53): FP64 direct sum over all n
 * particles; type (null = all gas) and zeta (null = 0) indexed like the particles. */
void or_direct_gas(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   const double* soft, const uint8_t* type, const double* zeta, int64_t nt,
                   const uint32_t* targets, double G, double* ax, double* ay, double* az) {
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; ++t) {
        const uint32_t p = targets[t];
        const double te = soft ? soft[p] : 0.0, zt = zeta ? zeta[p] : 0.0;
        const int tg = type == NULL || type[p] == 0;
        double sx = 0, sy = 0, sz = 0;
        for (int64_t q = 0; q < n; ++q) {
            if (q == (int64_t)p) continue;
            const double ox = x[q] - x[p], oy = y[q] - y[p], oz = z[q] - z[p];
            const double r = sqrt(ox * ox + oy * oy + oz * oz);
            if (r <= 0) continue;
            const double f = or_pair_fac(r, m[q], te, soft ? soft[q] : 0.0, zt, zeta ? zeta[q] : 0.0, m[p],
                                         tg && (type == NULL || type[q] == 0));
            sx += ox * f; sy += oy * f; sz += oz * f;
        }
        ax[t] = G * sx; ay[t] = G * sy; az[t] = G * sz;
    }
}

/* Sinks (type 5) below every node (tree.cc:155-187); nsink has nnodes entries. */
void or_node_sinks(const or_tree* t, const uint8_t* type, uint32_t* nsink) {
    for (int64_t i = 0; i < t->nnodes; ++i) {
        uint32_t c = 0;
        for (int k = t->plo[i]; k < t->phi[i]; ++k) c += type[t->order[k]] == 5;
        nsink[i] = c;
    }
}

/* Tree reuse: replace the walk's node fields with refreshed ones (refresh_walk_nodes writes the
 * packed walk nodes, tree.cc:256-274) and point the tree at the particles' current positions (the
 * walk reads them, tree.cc:786-789). */
void or_set_walk_nodes(or_tree* t, const double* cx, const double* cy, const double* cz, const double* mass,
                       const double* w_s, const float* w_len, const float* w_soft) {
    const size_t nn = (size_t)t->nnodes;
    memcpy(t->cx, cx, nn * 8); memcpy(t->cy, cy, nn * 8); memcpy(t->cz, cz, nn * 8);
    memcpy(t->mass, mass, nn * 8); memcpy(t->w_s, w_s, nn * 8);
    memcpy(t->w_len, w_len, nn * 4); memcpy(t->w_soft, w_soft, nn * 4);
}

void or_set_positions(or_tree* t, const double* x, const double* y, const double* z) {
    t->x = x; t->y = y; t->z = z;
}

/* ---- neighbour search and the density solve (shmem/hydro.h:25-117, hydro.cc:37-327) ---------- */

/* Minimum-image separation, box <= 0 = open (shmem/vec.h:25-31). */
static inline double or_min_image(double s, double box) {
    if (box > 0) {
        if (s > 0.5 * box) s -= box;
        else if (s < -0.5 * box) s += box;
    }
    return s;
}

/* The search node's conservative half side: float centre, so widened by 1e-6 of the root side plus
 * four float ulps of the centre's largest coordinate (tree.cc:490-505).  Only the prune uses it. */
static float or_snode_half(const or_tree* t, int i) {
    const double eps = 1e-6 * (t->nnodes ? t->size[t->root] : 1.0);
    const double cm = dmax(fabs(t->gcx[i]), dmax(fabs(t->gcy[i]), fabs(t->gcz[i])));
    return (float)(0.5 * t->size[i] + eps + 4.0 * (double)FLT_EPSILON * cm);
}

/* Tree::init_hmax (tree.cc:287-302, 332-338): per node the largest h, rounded up to float, of the
 * gas particles [0, n_gas) below it with h > 0. */
void or_init_hmax(const or_tree* t, const double* h, int64_t n_gas, float* hmax) {
    for (int64_t i = 0; i < t->nnodes; ++i) hmax[i] = 0.0f;
    const int64_t n = n_gas < t->n ? n_gas : t->n;
    for (int64_t i = 0; i < n; ++i) {
        if (!(h[i] > 0) || t->leaf_of[i] < 0) continue;
        float f = (float)h[i];
        if ((double)f < h[i]) f = nextafterf(f, 1e30f);
        for (int no = t->leaf_of[i]; no >= 0; no = t->parent[no]) {
            if (hmax[no] >= f) break;
            hmax[no] = f;
        }
    }
}

/* One centre's search, appending particle indices to out (capacity cap; returns the count, which
 * may exceed cap).  mode 0: ngb_search, r < radius (hydro.cc:37-108); mode 1: ngb_search_reverse,
 * gas j < n_gas with radius <= r < h[j] (hydro.cc:110-148), pruned by hmax.  Nodes in the
 * reference's threading order, so the lists come out in tree order. */
static int64_t or_ngb_one(const or_tree* t, const float* half, const float* hmax, double cx, double cy, double cz,
                          double radius, int mode, const double* h, int64_t n_gas, double box, uint32_t* out,
                          int64_t cap) {
    int64_t k = 0;
    const double r2max = radius * radius;
    int node = t->root;
    while (node >= 0) {
        const double hn = (double)half[node];
        double dist;
        if (mode == 0) {
            dist = radius + hn;
        } else {
            const double hm = (double)hmax[node];
            if (hm <= radius) { node = t->next[node]; continue; }
            dist = hm + hn;
        }
        const double dx = or_min_image((double)(float)t->gcx[node] - cx, box);
        if (dx > dist || -dx > dist) { node = t->next[node]; continue; }
        const double dy = or_min_image((double)(float)t->gcy[node] - cy, box);
        if (dy > dist || -dy > dist) { node = t->next[node]; continue; }
        const double dz = or_min_image((double)(float)t->gcz[node] - cz, box);
        if (dz > dist || -dz > dist) { node = t->next[node]; continue; }
        dist += 0.7320508075688772 * hn;
        if (dx * dx + dy * dy + dz * dz > dist * dist) { node = t->next[node]; continue; }
        if (t->first[node] < 0) {
            for (int s = t->plo[node]; s < t->phi[node]; ++s) {
                const uint32_t j = t->order[s];
                if (mode == 1 && (int64_t)j >= n_gas) continue;
                const double ox = or_min_image(t->x[j] - cx, box), oy = or_min_image(t->y[j] - cy, box),
                             oz = or_min_image(t->z[j] - cz, box);
                const double r2 = ox * ox + oy * oy + oz * oz;
                const int keep = mode == 0 ? r2 < r2max : (r2 >= r2max && r2 < h[j] * h[j]);
                if (keep) {
                    if (k < cap) out[k] = j;
                    ++k;
                }
            }
            node = t->next[node];
        } else {
            node = t->first[node];
        }
    }
    return k;
}

/* Searches for n centres as CSR: mode 0 gather, 1 reverse (h, n_gas), 2 gather then reverse.
 * start has n+1 entries; found (may be null) receives start[n] entries if cap suffices. */
void or_ngb_search(const or_tree* t, int64_t n, const double* cx, const double* cy, const double* cz,
                   const double* radius, int mode, const double* h, int64_t n_gas, double box, int64_t* start,
                   uint32_t* found, int64_t cap) {
    float* half = (float*)malloc((size_t)(t->nnodes > 0 ? t->nnodes : 1) * 4);
    float* hmax = (float*)calloc((size_t)(t->nnodes > 0 ? t->nnodes : 1), 4);
    for (int64_t i = 0; i < t->nnodes; ++i) half[i] = or_snode_half(t, (int)i);
    if (mode != 0) or_init_hmax(t, h, n_gas, hmax);
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, 8);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t c = 0; c < n; ++c) {
        int64_t k = 0;
        if (mode != 1) k += or_ngb_one(t, half, hmax, cx[c], cy[c], cz[c], radius[c], 0, h, n_gas, box, NULL, 0);
        if (mode != 0) k += or_ngb_one(t, half, hmax, cx[c], cy[c], cz[c], radius[c], 1, h, n_gas, box, NULL, 0);
        cnt[c] = k;
    }
    start[0] = 0;
    for (int64_t c = 0; c < n; ++c) start[c + 1] = start[c] + cnt[c];
    if (found && start[n] <= cap) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t c = 0; c < n; ++c) {
            int64_t k = 0;
            uint32_t* o = found + start[c];
            if (mode != 1) k += or_ngb_one(t, half, hmax, cx[c], cy[c], cz[c], radius[c], 0, h, n_gas, box, o, cnt[c]);
            if (mode != 0)
                or_ngb_one(t, half, hmax, cx[c], cy[c], cz[c], radius[c], 1, h, n_gas, box, o + k, cnt[c] - k);
        }
    }
    free(cnt);
    free(hmax);
    free(half);
}

/* The cubic spline of support h in n_dims dimensions (shmem/hydro.h:25-63): norm, W, dW/dh and the
 * unit ball volume. */
static double or_kernel_norm(double h, int dim) {
    if (dim == 1) return (4.0 / 3.0) / h;
    if (dim == 2) return 40.0 / (7.0 * M_PI * h * h);
    return 8.0 / (M_PI * h * h * h);
}
static double or_ball_vol(double h, int dim) {
    if (dim == 1) return 2.0 * h;
    if (dim == 2) return M_PI * h * h;
    return 4.0 * M_PI / 3.0 * h * h * h;
}
static double or_kernel_w(double r, double h, int dim) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = or_kernel_norm(h, dim);
    if (q < 0.5) return norm * (1.0 - 6.0 * q * q + 6.0 * q * q * q);
    const double u = 1.0 - q;
    return norm * 2.0 * u * u * u;
}
static double or_kernel_dwdh(double r, double h, int dim) {
    const double q = r / h;
    if (q >= 1.0) return 0.0;
    const double norm = or_kernel_norm(h, dim);
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

/* Rank-d inverse of the symmetric moments (xx yy zz xy yz xz) into a row-major 3x3, zero when
 * degenerate (shmem/vec.h:43-66; the 3-D case is the cofactor inverse of math_types/mat3.h:41-67). */
static int or_invert_moments(const double* m, double* B, int n_dims) {
    for (int i = 0; i < 9; ++i) B[i] = 0.0;
    if (n_dims == 1) {
        if (fabs(m[0]) < 1e-300) return 0;
        B[0] = 1.0 / m[0];
        return 1;
    }
    if (n_dims == 2) {
        const double det = m[0] * m[1] - m[3] * m[3];
        if (fabs(det) < 1e-300) return 0;
        B[0] = m[1] / det; B[1] = -m[3] / det;
        B[3] = -m[3] / det; B[4] = m[0] / det;
        return 1;
    }
    const double a00 = m[0], a01 = m[3], a02 = m[5], a10 = m[3], a11 = m[1], a12 = m[4], a20 = m[5], a21 = m[4],
                 a22 = m[2];
    const double d = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
    if (d == 0.0 || d != d) return 0;
    const double id = 1.0 / d;
    B[0] = (a11 * a22 - a12 * a21) * id; B[1] = (a02 * a21 - a01 * a22) * id; B[2] = (a01 * a12 - a02 * a11) * id;
    B[3] = (a12 * a20 - a10 * a22) * id; B[4] = (a00 * a22 - a02 * a20) * id; B[5] = (a02 * a10 - a00 * a12) * id;
    B[6] = (a10 * a21 - a11 * a20) * id; B[7] = (a01 * a20 - a00 * a21) * id; B[8] = (a00 * a11 - a01 * a10) * id;
    return 1;
}

/* One density evaluation at h over the gather list of the target at (px,py,pz): the sums the
 * solve reads (hydro.cc:205-222). */
typedef struct {
    double wsum, dwdh, rho, mom[6], face[3];
    int inside;
} or_dens_sums;
static void or_dens_eval(const or_tree* t, const uint8_t* type, const uint32_t* ngb, int64_t nn, double px, double py,
                         double pz, double h, double box, int n_dims, or_dens_sums* s) {
    memset(s, 0, sizeof(*s));
    for (int64_t k = 0; k < nn; ++k) {
        const uint32_t j = ngb[k];
        if (type && type[j] != 0) continue;
        const double dx = or_min_image(t->x[j] - px, box), dy = or_min_image(t->y[j] - py, box),
                     dz = or_min_image(t->z[j] - pz, box);
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double w = or_kernel_w(r, h, n_dims);
        s->wsum += w;
        s->dwdh += or_kernel_dwdh(r, h, n_dims);
        s->rho += t->m[j] * w;
        s->mom[0] += dx * dx * w; s->mom[1] += dy * dy * w; s->mom[2] += dz * dz * w;
        s->mom[3] += dx * dy * w; s->mom[4] += dy * dz * w; s->mom[5] += dx * dz * w;
        s->face[0] += dx * w; s->face[1] += dy * w; s->face[2] += dz * w;
        if (r < h) ++s->inside;
    }
}

/* density (hydro.cc:150-327) for nt targets: bisection-guarded Newton on N_eff(h) = des_ngb with
 * the face-closure and condition-number corrections.  h_start (per target) and cond_prev (per
 * particle) may be null; type (per particle, 0 = gas) may be null (all gas).  face_corr = 0 is
 * SHMEM_NO_FACECORR. */
void or_density(const or_tree* t, int64_t nt, const uint32_t* targets, double des_ngb, double ngb_tol,
                const double* h_start, double box, int n_dims, const double* cond_prev, const uint8_t* type,
                int face_corr, double* h_out, double* rho_out, int32_t* nngb_out, int32_t* iters_out) {
    double h_default = 0.0;
    if (!h_start) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int64_t i = 0; i < t->n; ++i) {
            lo[0] = dmin(lo[0], t->x[i]); hi[0] = dmax(hi[0], t->x[i]);
            lo[1] = dmin(lo[1], t->y[i]); hi[1] = dmax(hi[1], t->y[i]);
            lo[2] = dmin(lo[2], t->z[i]); hi[2] = dmax(hi[2], t->z[i]);
        }
        const double vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
        h_default = cbrt(3.0 * des_ngb * vol / (4.0 * M_PI * (double)t->n));
        if (n_dims == 1) h_default = 0.5 * des_ngb * (hi[0] - lo[0]) / (double)t->n;
        if (n_dims == 2) h_default = sqrt(des_ngb * (hi[0] - lo[0]) * (hi[1] - lo[1]) / (M_PI * (double)t->n));
    }
    float* half = (float*)malloc((size_t)(t->nnodes > 0 ? t->nnodes : 1) * 4);
    for (int64_t i = 0; i < t->nnodes; ++i) half[i] = or_snode_half(t, (int)i);
#pragma omp parallel
    {
        int64_t cap = 256;
        uint32_t* ngb = (uint32_t*)malloc((size_t)cap * 4);
#pragma omp for schedule(dynamic, 16)
        for (int64_t c = 0; c < nt; ++c) {
            const uint32_t p = targets[c];
            const double px = t->x[p], py = t->y[p], pz = t->z[p];
            double h = h_start ? h_start[c] : h_default, h_lo = 0.0, h_hi = 0.0;
            int iter = 0, converged = 0;
            or_dens_sums s;
            memset(&s, 0, sizeof(s));
            for (; iter < 100; ++iter) {
                int64_t nn = or_ngb_one(t, half, NULL, px, py, pz, h, 0, NULL, 0, box, ngb, cap);
                if (nn > cap) {
                    cap = nn * 2;
                    ngb = (uint32_t*)realloc(ngb, (size_t)cap * 4);
                    nn = or_ngb_one(t, half, NULL, px, py, pz, h, 0, NULL, 0, box, ngb, cap);
                }
                or_dens_eval(t, type, ngb, nn, px, py, pz, h, box, n_dims, &s);
                const double n_eff = or_ball_vol(h, n_dims) * s.wsum;
                double ncorr = 1.0;
                if (cond_prev) {
                    const double cn = cond_prev[p];
                    if (cn > 100.0) ncorr = dmin(sqrt(1.0 + (cn - 100.0) / 1000.0), 2.0);
                }
                double des_eff = des_ngb * ncorr, tol_eff = ngb_tol * ncorr;
                if (face_corr && s.wsum > 0) {
                    double B[9];
                    if (or_invert_moments(s.mom, B, n_dims)) {
                        const double vol = 1.0 / s.wsum;
                        const double dx_i = sqrt(vol * (s.mom[0] + s.mom[1] + s.mom[2]));
                        double sum_abs = 0.0;
                        for (int r = 0; r < 3; ++r) {
                            const double leak = (B[3 * r] * s.face[0] + B[3 * r + 1] * s.face[1] + B[3 * r + 2] * s.face[2]) *
                                                (2.0 * vol);
                            sum_abs += fabs(leak) / n_dims;
                        }
                        const double denom = 2.0 * n_dims * pow(dx_i, n_dims - 1);
                        if (denom > 0) {
                            const double fce = sum_abs / denom;
                            if (fce > 0.35) ncorr = dmax(ncorr, dmin(fce / 0.35, 2.0));
                            des_eff = des_ngb * ncorr;
                            tol_eff = ngb_tol * ncorr;
                        }
                    }
                }
                if (iter > 1)
                    tol_eff = dmin(0.25 * des_eff, tol_eff * exp(0.1 * log(des_eff / (16.0 * tol_eff)) * iter));
                const double res = n_eff - des_eff;
                if (fabs(res) < tol_eff) { converged = 1; break; }
                if (res > 0) h_hi = h; else h_lo = h;
                const double dn = or_ball_vol(h, n_dims) * ((double)n_dims / h * s.wsum + s.dwdh);
                double hn = dn > 0 ? h - res / dn : 0.0;
                if (hn <= h_lo || (h_hi > 0 && hn >= h_hi) || hn <= 0) {
                    if (h_hi > 0) hn = h_lo > 0 ? sqrt(h_lo * h_hi) : 0.5 * h_hi;
                    else hn = h * (res > 0 ? 0.7 : 1.6);
                }
                h = hn;
            }
            if (!converged) {
                int64_t nn = or_ngb_one(t, half, NULL, px, py, pz, h, 0, NULL, 0, box, ngb, cap);
                if (nn > cap) {
                    cap = nn * 2;
                    ngb = (uint32_t*)realloc(ngb, (size_t)cap * 4);
                    nn = or_ngb_one(t, half, NULL, px, py, pz, h, 0, NULL, 0, box, ngb, cap);
                }
                or_dens_eval(t, type, ngb, nn, px, py, pz, h, box, n_dims, &s);
            }
            h_out[c] = h;
            rho_out[c] = s.rho;
            nngb_out[c] = s.inside;
            iters_out[c] = iter;
        }
        free(ngb);
    }
    free(half);
}
