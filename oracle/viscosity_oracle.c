/*
 * viscosity_oracle.c -- CPU restatement of the reference's variational
 * viscosity UAAMG-PCG (SIMD_UAAMG/simd_viscosity3d.cpp, volume_fractions.cpp)
 * on flattened 8^3 leaves.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
 * baseline.  Parity is UNPINNED except for volume_fraction (the solver needs
 * OpenVDB, TBB and Eigen, none of which exist here, and ships no golden
 * vectors; its volume_fractions.cpp is plain C++, and
 * tests/test_oracle_ref_pin.py checks this file's tetrahedron and cube
 * fractions against it bit for bit).
 *
 * Float arithmetic follows the reference operation by operation; compile with
 * -ffp-contract=off.  Deliberate, documented deviations:
 *  - grid-to-grid position transforms are done in index space (voxel centre i
 *    at world i*dx for every input grid), which equals OpenVDB's world-space
 *    round trip exactly when dx is a power of two;
 *  - BoxSampler restates OpenVDB 7+'s trilinearInterpolation (float
 *    difference, double weight product rounded to float, float add);
 *  - dot products sum per-leaf float partials in leaf order and the
 *    solid-velocity rhs contributions of one DOF are summed in a fixed gather
 *    order; the reference's tbb::parallel_reduce fixes neither order;
 *  - coefficient values at voxels outside the DOF pattern but inside pattern
 *    leaves are computed as if inside; no operator, coarsening or trimming
 *    step reads them (each read lies within distance 2 of a DOF).
 */
#include "uaamg_oracle.h"
#include "oracle_common.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VNA ORC_VA_COUNT

static void* vcalloc(size_t n, size_t s) {
    void* p = calloc(n ? n : 1, s ? s : 1);
    if (!p) { fprintf(stderr, "viscosity oracle: out of memory\n"); abort(); }
    return p;
}
static inline int floordiv8(int v) { return (v >= 0) ? (v / 8) : -((-v + 7) / 8); }
static inline int leaf_of(int v) { return floordiv8(v) * 8; }

/* ------------------------------------------------------------------------ */
/* leaf sets */
typedef struct { int n; int32_t* org; } leafset;

static int cmp_org_vdb(const void* a, const void* b) {
    leafkey ka, kb;
    make_key(&ka, (const int32_t*)a, 0);
    make_key(&kb, (const int32_t*)b, 0);
    return cmp_key(&ka, &kb);
}
/* sort in OpenVDB tree order and drop duplicates */
static void leafset_finish(leafset* s) {
    if (s->n == 0) return;
    qsort(s->org, (size_t)s->n, 3 * sizeof(int32_t), cmp_org_vdb);
    int m = 1;
    for (int i = 1; i < s->n; ++i) {
        const int32_t* p = s->org + 3 * (m - 1);
        const int32_t* q = s->org + 3 * i;
        if (p[0] != q[0] || p[1] != q[1] || p[2] != q[2]) {
            memmove(s->org + 3 * m, q, 3 * sizeof(int32_t));
            m++;
        }
    }
    s->n = m;
}

/* Leaves of dilateActiveValues(tree, r, NN_FACE_EDGE_VERTEX or NN_FACE) of a
 * tree with the given leaves and active masks (masks NULL = all active): the
 * input leaves plus every neighbour leaf that a dilated active voxel enters.
 * activity(i, off) tests voxel off of leaf i. */
typedef int (*active_fn)(const void* ctx, int64_t leaf, int off);
static void leafset_dilate(int64_t n, const int32_t* org, const void* ctx, active_fn act, int r,
                           int face_only, leafset* out) {
    out->org = (int32_t*)vcalloc((size_t)n * 27 * 3, sizeof(int32_t));
    out->n = 0;
    for (int64_t i = 0; i < n; ++i) {
        int touched[27] = {0};
        touched[13] = 1;
        for (int off = 0; off < LSZ; ++off) {
            if (!act(ctx, i, off)) continue;
            int lc[3] = {off >> 6, (off >> 3) & 7, off & 7};
            int ok[3][3];
            for (int a = 0; a < 3; ++a) {
                ok[a][0] = lc[a] <= r - 1;
                ok[a][1] = 1;
                ok[a][2] = lc[a] >= 8 - r;
            }
            for (int dx = 0; dx < 3; ++dx)
                for (int dy = 0; dy < 3; ++dy)
                    for (int dz = 0; dz < 3; ++dz) {
                        int nz = (dx != 1) + (dy != 1) + (dz != 1);
                        if (nz == 0) continue;
                        if (face_only && nz != 1) continue;
                        if (ok[0][dx] && ok[1][dy] && ok[2][dz]) touched[dx * 9 + dy * 3 + dz] = 1;
                    }
        }
        for (int d = 0; d < 27; ++d) {
            if (!touched[d]) continue;
            int32_t* o = out->org + 3 * out->n;
            o[0] = org[3 * i] + 8 * (d / 9 - 1);
            o[1] = org[3 * i + 1] + 8 * ((d / 3) % 3 - 1);
            o[2] = org[3 * i + 2] + 8 * (d % 3 - 1);
            out->n++;
        }
    }
    leafset_finish(out);
}

typedef struct { const uint64_t* masks; } mask_ctx;
static int act_masks(const void* ctx, int64_t leaf, int off) {
    const mask_ctx* m = (const mask_ctx*)ctx;
    if (!m->masks) return 1;
    return mbit(m->masks + 8 * leaf, off);
}

/* ------------------------------------------------------------------------ */
/* ------------------------------------------------------------------------ */
/* volume_fractions.cpp:82-120 */
static inline void swapf(float* a, float* b) { float t = *a; *a = *b; *b = t; }
/* util.h sort(a,b,c,d): ascending */
static inline void sort4(float* a, float* b, float* c, float* d) {
    if (*a > *b) swapf(a, b);
    if (*c > *d) swapf(c, d);
    if (*a > *c) swapf(a, c);
    if (*b > *d) swapf(b, d);
    if (*b > *c) swapf(b, c);
}
static inline float sorted_tet_fraction(float p0, float p1, float p2, float p3) {
    return p0 * p0 * p0 / ((p0 - p1) * (p0 - p2) * (p0 - p3));
}
static inline float sorted_prism_fraction(float p0, float p1, float p2, float p3) {
    float a = p0 / (p0 - p2), b = p0 / (p0 - p3), c = p1 / (p1 - p3), d = p1 / (p1 - p2);
    return a * b * (1 - d) + b * (1 - c) * d + c * d;
}
static float tet_fraction(float p0, float p1, float p2, float p3) {
    sort4(&p0, &p1, &p2, &p3);
    if (p3 <= 0) return 1;
    else if (p2 <= 0) return 1 - sorted_tet_fraction(p3, p2, p1, p0);
    else if (p1 <= 0) return sorted_prism_fraction(p0, p1, p2, p3);
    else if (p0 <= 0) return sorted_tet_fraction(p0, p1, p2, p3);
    else return 0;
}
static float cube_fraction(float p000, float p100, float p010, float p110, float p001, float p101,
                           float p011, float p111) {
    if (p000 < 0.f && p100 < 0.f && p010 < 0.f && p110 < 0.f && p001 < 0.f && p101 < 0.f &&
        p011 < 0.f && p111 < 0.f)
        return 1.0f;
    return (tet_fraction(p000, p001, p101, p011) + tet_fraction(p000, p101, p100, p110) +
            tet_fraction(p000, p010, p011, p110) + tet_fraction(p101, p011, p111, p110) +
            2 * tet_fraction(p000, p011, p101, p110) + tet_fraction(p100, p101, p001, p111) +
            tet_fraction(p100, p001, p000, p010) + tet_fraction(p100, p110, p111, p010) +
            tet_fraction(p001, p111, p011, p010) + 2 * tet_fraction(p100, p111, p001, p010)) /
           12;
}
float orc_tet_fraction(float p0, float p1, float p2, float p3) { return tet_fraction(p0, p1, p2, p3); }
float orc_cube_fraction(float p000, float p100, float p010, float p110, float p001, float p101, float p011,
                        float p111) {
    return cube_fraction(p000, p100, p010, p110, p001, p101, p011, p111);
}

/* ------------------------------------------------------------------------ */
/* a float field over a leaf set with getValue semantics */
typedef struct {
    leafset s;
    leafmap map;
    float* v;   /* [n][512] */
    float bg;
} field;
static void field_init(field* f, leafset s, float bg) {
    f->s = s;
    leafmap_init(&f->map, s.n, s.org);
    f->v = (float*)vcalloc((size_t)s.n * LSZ, sizeof(float));
    f->bg = bg;
}
static void field_free(field* f) {
    leafmap_free(&f->map);
    free(f->v);
    free(f->s.org);
    memset(f, 0, sizeof(*f));
}
static inline float field_get(const field* f, int x, int y, int z) {
    int32_t li = leafmap_find(&f->map, x, y, z);
    if (li < 0) return f->bg;
    return f->v[(size_t)li * LSZ + voff(x, y, z)];
}

/* ------------------------------------------------------------------------ */
typedef struct {
    int nl;
    int32_t* org;
    leafmap map;
    uint64_t* dof;      /* [3][nl][8] */
    int32_t* dof_base;  /* [3][nl] */
    int ndof_c[3];
    int ndof;
    float* coef;        /* [3][VNA][nl][512] */
    uint32_t* trim;     /* [nl] */
    float def[3][VNA];  /* tree backgrounds (getValue of a missing leaf) */
    float app[3][VNA];  /* light_weight_applier defaults for a missing leaf */
    int32_t* child;     /* [nl][8] fine leaf per octant (x<<2|y<<1|z), -1 if absent */
    float *lhs, *rhs, *tmp; /* [3][nl][512] mu-cycle scratch */
} vlevel;

struct orc_visc {
    int nlev;
    vlevel lv[32];
    float dt, rho, dx, factor, def_off, def_diag;
    /* viscosity grid (owned copy) and level-0 construction fields kept for the rhs */
    int32_t* mu_org;
    float* mu_val;
    ogrid mu;
    field face_vol[3], voxel_vol, edge_vol[3];
    leafset solid_leaves;   /* leaves of the is_solid grids */
    leafmap solid_map;
    uint64_t* is_solid;     /* [3][n][8] */
    /* coarsest explicit matrix (CSR, columns ascending like a RowMajor
     * Eigen matrix after setFromTriplets) */
    int c_n;
    int32_t *c_rowptr, *c_col, *c_row_ch, *c_row_leaf, *c_row_off;
    float *c_val, *c_invdiag, *c_b, *c_x, *c_r, *c_p, *c_z, *c_t;
    int c_order;            /* summation order of the coarsest CG (ORC_CG_ORDER_*) */
};

static inline size_t vidx(const vlevel* L, int c, int32_t leaf, int off) {
    return ((size_t)c * L->nl + leaf) * LSZ + off;
}
static inline size_t cidx(const vlevel* L, int c, int a, int32_t leaf, int off) {
    return (((size_t)c * VNA + a) * L->nl + leaf) * LSZ + off;
}
static inline int dof_at(const vlevel* L, int c, int x, int y, int z) {
    int32_t li = leafmap_find(&L->map, x, y, z);
    if (li < 0) return 0;
    return mbit(L->dof + ((size_t)c * L->nl + li) * 8, voff(x, y, z));
}
static inline float coef_at(const vlevel* L, int c, int a, int x, int y, int z) {
    int32_t li = leafmap_find(&L->map, x, y, z);
    if (li < 0) return L->def[c][a];
    return L->coef[cidx(L, c, a, li, voff(x, y, z))];
}
static int32_t dof_number(const vlevel* L, int c, int x, int y, int z) {
    int32_t li = leafmap_find(&L->map, x, y, z);
    if (li < 0) return -1;
    const uint64_t* m = L->dof + ((size_t)c * L->nl + li) * 8;
    int off = voff(x, y, z);
    if (!mbit(m, off)) return -1;
    int32_t d = L->dof_base[(size_t)c * L->nl + li];
    for (int w = 0; w < (off >> 6); ++w) d += __builtin_popcountll(m[w]);
    uint64_t below = (off & 63) ? (m[off >> 6] & ((1ull << (off & 63)) - 1ull)) : 0ull;
    return d + __builtin_popcountll(below);
}

/* 27-leaf neighbourhood of a leaf: nb[(dx+1)*9+(dy+1)*3+(dz+1)] */
static void nb27(const vlevel* L, int32_t leaf, int32_t* nb) {
    const int32_t* o = L->org + 3 * leaf;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz)
                nb[(dx + 1) * 9 + (dy + 1) * 3 + dz + 1] =
                    leafmap_find(&L->map, o[0] + 8 * dx, o[1] + 8 * dy, o[2] + 8 * dz);
}
/* local coordinates in [-8, 15] -> (leaf, offset) through the neighbourhood */
static inline int32_t nb_locate(const int32_t* nb, int x, int y, int z, int* off) {
    int dx = (x < 0) ? -1 : (x > 7 ? 1 : 0);
    int dy = (y < 0) ? -1 : (y > 7 ? 1 : 0);
    int dz = (z < 0) ? -1 : (z > 7 ? 1 : 0);
    *off = voff(x, y, z);
    return nb[(dx + 1) * 9 + (dy + 1) * 3 + dz + 1];
}

static void level_alloc(vlevel* L, leafset s) {
    L->nl = s.n;
    L->org = s.org;
    leafmap_init(&L->map, s.n, s.org);
    L->dof = (uint64_t*)vcalloc((size_t)3 * s.n * 8, sizeof(uint64_t));
    L->dof_base = (int32_t*)vcalloc((size_t)3 * s.n, sizeof(int32_t));
    L->coef = (float*)vcalloc((size_t)3 * VNA * s.n * LSZ, sizeof(float));
    L->trim = (uint32_t*)vcalloc((size_t)s.n, sizeof(uint32_t));
    L->child = NULL;
    L->lhs = (float*)vcalloc((size_t)3 * s.n * LSZ, sizeof(float));
    L->rhs = (float*)vcalloc((size_t)3 * s.n * LSZ, sizeof(float));
    L->tmp = (float*)vcalloc((size_t)3 * s.n * LSZ, sizeof(float));
}

/* set_dof (:500-538): global numbering channel by channel, leaves in tree
 * order, voxels in offset order; numbering continues across channels. */
static void level_number_dofs(vlevel* L, int* running) {
    for (int c = 0; c < 3; ++c) {
        int start = *running;
        for (int i = 0; i < L->nl; ++i) {
            L->dof_base[(size_t)c * L->nl + i] = *running;
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int w = 0; w < 8; ++w) *running += __builtin_popcountll(m[w]);
        }
        L->ndof_c[c] = *running - start;
    }
}

/* union of the channel DOF masks, dilated: the coefficient pattern leaves */
typedef struct { const uint64_t* dof; int nl; } union_ctx;
static int act_union(const void* ctx, int64_t leaf, int off) {
    const union_ctx* u = (const union_ctx*)ctx;
    for (int c = 0; c < 3; ++c)
        if (mbit(u->dof + ((size_t)c * u->nl + leaf) * 8, off)) return 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Level 0: calculate_subcell_sdf_volume (:258-330),
 * calculate_matrix_coefficients_volume (:332-406), mark_dof (:408-498),
 * calculate_matrix_coefficients (:881-963). */
static void build_level0(orc_visc* h, const ogrid* liq, const uint64_t* liq_masks,
                         const ogrid* sol, const ogrid* mu) {
    const float dx = h->dx;
    const int64_t nliq = liq->n;
    mask_ctx mc = {liq_masks};

    /* subcell SDF / volume leaves: 2*O + {0,8}^3 for the liquid leaves dilated by 1 */
    leafset a1;
    leafset_dilate(nliq, liq->org, &mc, act_masks, 1, 0, &a1);
    leafset sub = {a1.n * 8, (int32_t*)vcalloc((size_t)a1.n * 8 * 3, sizeof(int32_t))};
    for (int i = 0; i < a1.n; ++i)
        for (int q = 0; q < 8; ++q) {
            int32_t* o = sub.org + 3 * (8 * i + q);
            o[0] = 2 * a1.org[3 * i] + 8 * (q >> 2);
            o[1] = 2 * a1.org[3 * i + 1] + 8 * ((q >> 1) & 1);
            o[2] = 2 * a1.org[3 * i + 2] + 8 * (q & 1);
        }
    free(a1.org);
    leafset sub2 = {sub.n, (int32_t*)vcalloc((size_t)sub.n * 3, sizeof(int32_t))};
    memcpy(sub2.org, sub.org, (size_t)sub.n * 3 * sizeof(int32_t));

    const float sub_bg = 1.5f * dx;
    field sdf, svol;
    field_init(&sdf, sub, sub_bg);
    field_init(&svol, sub2, 0.f);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < sdf.s.n; ++i) {
        const int32_t* o = sdf.s.org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int s0 = o[0] + (off >> 6), s1 = o[1] + ((off >> 3) & 7), s2 = o[2] + (off & 7);
            /* subcell corner s sits at liquid index s/2 - 1/2 */
            float v = box_sample(liq, 0.5 * s0 - 0.5, 0.5 * s1 - 0.5, 0.5 * s2 - 0.5);
            sdf.v[(size_t)i * LSZ + off] = (v < sub_bg) ? v : sub_bg;
        }
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < svol.s.n; ++i) {
        const int32_t* o = svol.s.org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int s0 = o[0] + (off >> 6), s1 = o[1] + ((off >> 3) & 7), s2 = o[2] + (off & 7);
            float p[2][2][2];
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b)
                    for (int c = 0; c < 2; ++c) p[a][b][c] = field_get(&sdf, s0 + a, s1 + b, s2 + c);
            float f = cube_fraction(p[0][0][0], p[1][0][0], p[0][1][0], p[1][1][0], p[0][0][1], p[1][0][1],
                                    p[0][1][1], p[1][1][1]);
            svol.v[(size_t)i * LSZ + off] = (f > 0) ? f : 0.f;
        }
    }
    field_free(&sdf);

    /* control volumes over the liquid leaves dilated by 2 */
    leafset a2;
    leafset_dilate(nliq, liq->org, &mc, act_masks, 2, 0, &a2);
    {
        leafset cp[7];
        for (int k = 0; k < 7; ++k) {
            cp[k].n = a2.n;
            cp[k].org = (int32_t*)vcalloc((size_t)a2.n * 3, sizeof(int32_t));
            memcpy(cp[k].org, a2.org, (size_t)a2.n * 3 * sizeof(int32_t));
        }
        field_init(&h->voxel_vol, cp[0], 0.f);
        for (int c = 0; c < 3; ++c) {
            field_init(&h->face_vol[c], cp[1 + c], 0.f);
            field_init(&h->edge_vol[c], cp[4 + c], 0.f);
        }
        free(a2.org);
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < h->voxel_vol.s.n; ++i) {
        const int32_t* o = h->voxel_vol.s.org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            float vol_c = 0, vol_f[3] = {0, 0, 0}, vol_e[3] = {0, 0, 0};
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b)
                    for (int cc = 0; cc < 2; ++cc) {
                        int s[3] = {2 * g[0] + a, 2 * g[1] + b, 2 * g[2] + cc};
                        vol_c += field_get(&svol, s[0], s[1], s[2]);
                        for (int c = 0; c < 3; ++c) {
                            int f[3] = {s[0], s[1], s[2]};
                            f[c]--;
                            vol_f[c] += field_get(&svol, f[0], f[1], f[2]);
                            int e[3] = {s[0] - 1, s[1] - 1, s[2] - 1};
                            e[c]++;
                            vol_e[c] += field_get(&svol, e[0], e[1], e[2]);
                        }
                    }
            size_t at = (size_t)i * LSZ + off;
            h->voxel_vol.v[at] = (vol_c > 0) ? vol_c * 0.125f : 0.f;
            for (int c = 0; c < 3; ++c) {
                h->face_vol[c].v[at] = (vol_f[c] > 0) ? vol_f[c] * 0.125f : 0.f;
                h->edge_vol[c].v[at] = (vol_e[c] > 0) ? vol_e[c] * 0.125f : 0.f;
            }
        }
    }
    field_free(&svol);

    /* is_solid and DOF marking over the liquid leaves face-dilated by 1 */
    leafset a1f;
    leafset_dilate(nliq, liq->org, &mc, act_masks, 1, 1, &a1f);
    h->solid_leaves = a1f;
    leafmap_init(&h->solid_map, a1f.n, a1f.org);
    h->is_solid = (uint64_t*)vcalloc((size_t)3 * a1f.n * 8, sizeof(uint64_t));
    uint64_t* dofm = (uint64_t*)vcalloc((size_t)3 * a1f.n * 8, sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < a1f.n; ++i) {
        const int32_t* o = a1f.org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            for (int c = 0; c < 3; ++c) {
                double p[3] = {g[0], g[1], g[2]};
                p[c] -= 0.5;
                float s = box_sample(sol, p[0], p[1], p[2]);
                uint64_t bit = 1ull << (off & 63);
                if (s < 0) {
                    h->is_solid[((size_t)c * a1f.n + i) * 8 + (off >> 6)] |= bit;
                    continue;
                }
                int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
                int on = 0;
                if (field_get(&h->face_vol[c], g[0], g[1], g[2]) > 0) on = 1;
                else {
                    int m[3] = {g[0], g[1], g[2]};
                    m[c]--;
                    if (field_get(&h->voxel_vol, g[0], g[1], g[2]) > 0 ||
                        field_get(&h->voxel_vol, m[0], m[1], m[2]) > 0)
                        on = 1;
                    else {
                        int q2[3] = {g[0], g[1], g[2]};
                        q2[d2]++;
                        int q1[3] = {g[0], g[1], g[2]};
                        q1[d1]++;
                        float e1n = field_get(&h->edge_vol[d1], g[0], g[1], g[2]);
                        float e1p = field_get(&h->edge_vol[d1], q2[0], q2[1], q2[2]);
                        float e2n = field_get(&h->edge_vol[d2], g[0], g[1], g[2]);
                        float e2p = field_get(&h->edge_vol[d2], q1[0], q1[1], q1[2]);
                        if (e1n > 0 || e1p > 0 || e2n > 0 || e2p > 0) on = 1;
                    }
                }
                if (on) dofm[((size_t)c * a1f.n + i) * 8 + (off >> 6)] |= bit;
            }
        }
    }

    /* DOF leaves (pruned) -> pattern leaves: union dilated by 2 */
    int ndl = 0;
    int32_t* dl = (int32_t*)vcalloc((size_t)a1f.n * 3, sizeof(int32_t));
    uint64_t* dlm = (uint64_t*)vcalloc((size_t)3 * a1f.n * 8, sizeof(uint64_t));
    for (int i = 0; i < a1f.n; ++i) {
        int any = 0;
        for (int c = 0; c < 3 && !any; ++c)
            for (int w = 0; w < 8; ++w)
                if (dofm[((size_t)c * a1f.n + i) * 8 + w]) { any = 1; break; }
        if (!any) continue;
        memcpy(dl + 3 * ndl, a1f.org + 3 * i, 3 * sizeof(int32_t));
        for (int c = 0; c < 3; ++c)
            memcpy(dlm + ((size_t)c * a1f.n + ndl) * 8, dofm + ((size_t)c * a1f.n + i) * 8, 8 * sizeof(uint64_t));
        ndl++;
    }
    /* compact the channel-major masks to stride ndl */
    uint64_t* dlm2 = (uint64_t*)vcalloc((size_t)3 * (ndl ? ndl : 1) * 8, sizeof(uint64_t));
    for (int c = 0; c < 3; ++c)
        memcpy(dlm2 + (size_t)c * ndl * 8, dlm + (size_t)c * a1f.n * 8, (size_t)ndl * 8 * sizeof(uint64_t));
    free(dlm);
    union_ctx uc = {dlm2, ndl};
    leafset pat;
    leafset_dilate(ndl, dl, &uc, act_union, 2, 0, &pat);

    vlevel* L = &h->lv[0];
    level_alloc(L, pat);
    leafmap dmap;
    leafmap_init(&dmap, ndl, dl);
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        int32_t j = leafmap_find(&dmap, o[0], o[1], o[2]);
        if (j < 0) continue;
        for (int c = 0; c < 3; ++c)
            memcpy(L->dof + ((size_t)c * L->nl + i) * 8, dlm2 + ((size_t)c * ndl + j) * 8, 8 * sizeof(uint64_t));
    }
    leafmap_free(&dmap);
    free(dl);
    free(dlm2);
    free(dofm);
    int running = 0;
    level_number_dofs(L, &running);
    L->ndof = running;

    /* defaults (:911-914) */
    const float factor = h->factor;
    const float doff = h->def_off, ddiag = h->def_diag;
    for (int c = 0; c < 3; ++c) {
        L->def[c][ORC_VA_DIAG] = ddiag;
        L->def[c][ORC_VA_INVDIAG] = 0.f;
        for (int ax = 0; ax < 3; ++ax) L->def[c][ORC_VA_NEGX + ax] = (ax == c) ? -2.0f * doff : -doff;
        L->def[c][ORC_VA_T00] = doff;
        L->def[c][ORC_VA_T01] = -doff;
        L->def[c][ORC_VA_T10] = -doff;
        L->def[c][ORC_VA_T11] = doff;
        memcpy(L->app[c], L->def[c], sizeof(L->def[c]));
        L->app[c][ORC_VA_INVDIAG] = 1.0f / ddiag;
    }

    /* finest_level_matrix_setter::channel_op (:617-844) */
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        for (int c = 0; c < 3; ++c) {
            const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
            for (int off = 0; off < LSZ; ++off) {
                int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                float* cf[VNA];
                for (int a = 0; a < VNA; ++a) cf[a] = L->coef + cidx(L, c, a, i, off);
#define GP(v, ax, s) int v[3] = {g[0], g[1], g[2]}; v[ax] += (s)
                if (mbit(L->dof + ((size_t)c * L->nl + i) * 8, off)) {
                    float temp_diag = 0;
                    float face_vol = field_get(&h->face_vol[d0], g[0], g[1], g[2]);
                    if (face_vol < 1e-1f) face_vol = 1e-1f;
                    temp_diag += face_vol;
                    {
                        float term = 2 * factor * field_get(&h->voxel_vol, g[0], g[1], g[2]) *
                                     ogrid_get(mu, g[0], g[1], g[2], 0);
                        temp_diag += term;
                    }
                    {
                        GP(m, d0, -1);
                        float term = 2 * factor * field_get(&h->voxel_vol, m[0], m[1], m[2]) *
                                     ogrid_get(mu, m[0], m[1], m[2], 0);
                        temp_diag += term;
                        *cf[ORC_VA_NEGX + d0] = dof_at(L, c, m[0], m[1], m[2]) ? -term : 0.f;
                    }
                    float fc[3] = {(float)g[0], (float)g[1], (float)g[2]};
                    fc[d0] -= 0.5f;
                    {
                        GP(q, d1, 1);
                        float ev = field_get(&h->edge_vol[d2], q[0], q[1], q[2]);
                        float p[3] = {fc[0], fc[1], fc[2]};
                        p[d1] += 0.5f;
                        float sv = box_sample(mu, p[0], p[1], p[2]);
                        float term = factor * ev * sv;
                        temp_diag += term;
                    }
                    {
                        float ev = field_get(&h->edge_vol[d2], g[0], g[1], g[2]);
                        float p[3] = {fc[0], fc[1], fc[2]};
                        p[d1] -= 0.5f;
                        float sv = box_sample(mu, p[0], p[1], p[2]);
                        float term = factor * ev * sv;
                        temp_diag += term;
                        GP(m, d1, -1);
                        *cf[ORC_VA_NEGX + d1] = dof_at(L, c, m[0], m[1], m[2]) ? -term : 0.f;
                    }
                    {
                        GP(q, d2, 1);
                        float ev = field_get(&h->edge_vol[d1], q[0], q[1], q[2]);
                        float p[3] = {fc[0], fc[1], fc[2]};
                        p[d2] += 0.5f;
                        float sv = box_sample(mu, p[0], p[1], p[2]);
                        float term = factor * ev * sv;
                        temp_diag += term;
                    }
                    {
                        float ev = field_get(&h->edge_vol[d1], g[0], g[1], g[2]);
                        float p[3] = {fc[0], fc[1], fc[2]};
                        p[d2] -= 0.5f;
                        float sv = box_sample(mu, p[0], p[1], p[2]);
                        float term = factor * ev * sv;
                        temp_diag += term;
                        GP(m, d2, -1);
                        *cf[ORC_VA_NEGX + d2] = dof_at(L, c, m[0], m[1], m[2]) ? -term : 0.f;
                    }
                    *cf[ORC_VA_DIAG] = temp_diag;
                    *cf[ORC_VA_INVDIAG] = (temp_diag != 0) ? 1.0f / temp_diag : 0.f;
                } else {
                    *cf[ORC_VA_DIAG] = ddiag; /* setValueOff keeps the default */
                    *cf[ORC_VA_INVDIAG] = 0.f;
                    *cf[ORC_VA_NEGX] = 0.f;
                    *cf[ORC_VA_NEGY] = 0.f;
                    *cf[ORC_VA_NEGZ] = 0.f;
                }
                GP(p1, d1, 1);
                GP(p2, d2, 1);
                int dof1n = dof_at(L, d1, g[0], g[1], g[2]);
                int dof1p = dof_at(L, d1, p1[0], p1[1], p1[2]);
                int dof2n = dof_at(L, d2, g[0], g[1], g[2]);
                int dof2p = dof_at(L, d2, p2[0], p2[1], p2[2]);
                float gf[3] = {(float)g[0], (float)g[1], (float)g[2]};
                for (int jk = 0; jk < 4; ++jk) {
                    int j = jk >> 1, k = jk & 1;
                    int ok = (j ? dof1p : dof1n) && (k ? dof2p : dof2n);
                    if (!ok) {
                        *cf[ORC_VA_T00 + jk] = 0.f;
                        continue;
                    }
                    int e[3] = {g[0], g[1], g[2]};
                    e[d1] += j;
                    e[d2] += k;
                    float ev = field_get(&h->edge_vol[d0], e[0], e[1], e[2]);
                    float p[3] = {gf[0], gf[1], gf[2]};
                    p[d1] += j ? 0.5f : -0.5f;
                    p[d2] += k ? 0.5f : -0.5f;
                    float sv = box_sample(mu, p[0], p[1], p[2]);
                    float f = (j == k) ? factor : -factor;
                    *cf[ORC_VA_T00 + jk] = f * ev * sv;
                }
#undef GP
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Coarse level: mark_dof_from_child (:1017-1065),
 * calculate_matrix_coefficients_from_child (:1353-1451),
 * coarse_matrix_coef_setter (:1068-1350). */
static void build_coarse(orc_visc* h, int fl) {
    const vlevel* F = &h->lv[fl];
    vlevel* C = &h->lv[fl + 1];
    /* coarse DOF leaves: the parent leaf of every fine leaf with DOFs */
    leafset dl = {0, (int32_t*)vcalloc((size_t)(F->nl ? F->nl : 1) * 3, sizeof(int32_t))};
    for (int i = 0; i < F->nl; ++i) {
        int any = 0;
        for (int c = 0; c < 3 && !any; ++c)
            for (int w = 0; w < 8; ++w)
                if (F->dof[((size_t)c * F->nl + i) * 8 + w]) { any = 1; break; }
        if (!any) continue;
        const int32_t* o = F->org + 3 * i;
        int32_t* q = dl.org + 3 * dl.n++;
        for (int a = 0; a < 3; ++a) q[a] = leaf_of(floordiv8(o[a]) * 4);
    }
    leafset_finish(&dl);
    uint64_t* dm = (uint64_t*)vcalloc((size_t)3 * (dl.n ? dl.n : 1) * 8, sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < dl.n; ++i) {
        const int32_t* o = dl.org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int G[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            for (int c = 0; c < 3; ++c) {
                int on = 0;
                for (int a = 0; a < 2 && !on; ++a)
                    for (int b = 0; b < 2 && !on; ++b)
                        for (int k = 0; k < 2 && !on; ++k)
                            if (dof_at(F, c, 2 * G[0] + a, 2 * G[1] + b, 2 * G[2] + k)) on = 1;
                if (on) dm[((size_t)c * dl.n + i) * 8 + (off >> 6)] |= 1ull << (off & 63);
            }
        }
    }
    union_ctx uc = {dm, dl.n};
    leafset pat;
    leafset_dilate(dl.n, dl.org, &uc, act_union, 3, 0, &pat);
    level_alloc(C, pat);
    leafmap dmap;
    leafmap_init(&dmap, dl.n, dl.org);
    for (int i = 0; i < C->nl; ++i) {
        const int32_t* o = C->org + 3 * i;
        int32_t j = leafmap_find(&dmap, o[0], o[1], o[2]);
        if (j < 0) continue;
        for (int c = 0; c < 3; ++c)
            memcpy(C->dof + ((size_t)c * C->nl + i) * 8, dm + ((size_t)c * dl.n + j) * 8, 8 * sizeof(uint64_t));
    }
    leafmap_free(&dmap);
    free(dl.org);
    free(dm);
    int running = 0;
    level_number_dofs(C, &running);
    C->ndof = running;
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < VNA; ++a) {
            C->def[c][a] = 0.f;
            C->app[c][a] = (a == ORC_VA_DIAG || a == ORC_VA_INVDIAG) ? 1.0f : 1.0f;
        }
    for (int c = 0; c < 3; ++c) {
        /* applier defaults of a coarse level: m_default_diag = m_default_off_diag = 1 */
        for (int ax = 0; ax < 3; ++ax) C->app[c][ORC_VA_NEGX + ax] = (ax == c) ? -2.0f : -1.0f;
        C->app[c][ORC_VA_T01] = -1.0f;
        C->app[c][ORC_VA_T10] = -1.0f;
    }
    C->child = (int32_t*)vcalloc((size_t)C->nl * 8, sizeof(int32_t));
    for (int i = 0; i < C->nl; ++i)
        for (int q = 0; q < 8; ++q) {
            const int32_t* o = C->org + 3 * i;
            C->child[8 * i + q] = leafmap_find(&F->map, 2 * o[0] + 8 * (q >> 2), 2 * o[1] + 8 * ((q >> 1) & 1),
                                               2 * o[2] + 8 * (q & 1));
        }

    const float rap = 0.125f;
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < C->nl; ++i) {
        const int32_t* o = C->org + 3 * i;
        for (int c = 0; c < 3; ++c) {
            const int d[3] = {c, (c + 1) % 3, (c + 2) % 3};
            for (int off = 0; off < LSZ; ++off) {
                int G[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                float* cf[VNA];
                for (int a = 0; a < VNA; ++a) cf[a] = C->coef + cidx(C, c, a, i, off);
                if (mbit(C->dof + ((size_t)c * C->nl + i) * 8, off)) {
                    float nd = 0.f, nn[3] = {0.f, 0.f, 0.f};
                    for (int ii = 0; ii < 2; ++ii)
                        for (int jj = 0; jj < 2; ++jj)
                            for (int kk = 0; kk < 2; ++kk) {
                                int f[3] = {2 * G[0], 2 * G[1], 2 * G[2]};
                                f[d[0]] += ii;
                                f[d[1]] += jj;
                                f[d[2]] += kk;
                                if (!dof_at(F, c, f[0], f[1], f[2])) continue;
                                nd += coef_at(F, c, ORC_VA_DIAG, f[0], f[1], f[2]);
                                const int idx[3] = {ii, jj, kk};
                                for (int k = 0; k < 3; ++k) {
                                    float nt = coef_at(F, c, ORC_VA_NEGX + d[k], f[0], f[1], f[2]);
                                    int nb[3] = {f[0], f[1], f[2]};
                                    nb[d[k]]--;
                                    if (!dof_at(F, c, nb[0], nb[1], nb[2])) continue;
                                    if (idx[k] == 0) nn[k] += nt;
                                    else nd += nt * 2.0f;
                                }
                            }
                    *cf[ORC_VA_DIAG] = rap * nd;
                    *cf[ORC_VA_INVDIAG] = (nd != 0) ? 1.0f / (rap * nd) : 0.f;
                    for (int k = 0; k < 3; ++k) {
                        int nb[3] = {G[0], G[1], G[2]};
                        nb[d[k]]--;
                        *cf[ORC_VA_NEGX + d[k]] = dof_at(C, c, nb[0], nb[1], nb[2]) ? rap * nn[k] : 0.f;
                    }
                } else {
                    *cf[ORC_VA_DIAG] = 0.f;
                    *cf[ORC_VA_INVDIAG] = 0.f;
                    *cf[ORC_VA_NEGX] = 0.f;
                    *cf[ORC_VA_NEGY] = 0.f;
                    *cf[ORC_VA_NEGZ] = 0.f;
                }
                for (int t = 0; t < 4; ++t) {
                    float s = 0.f;
                    for (int ii = 0; ii < 2; ++ii)
                        for (int jj = 0; jj < 2; ++jj)
                            for (int kk = 0; kk < 2; ++kk) {
                                int f[3] = {2 * G[0], 2 * G[1], 2 * G[2]};
                                f[d[0]] += ii;
                                f[d[1]] += jj;
                                f[d[2]] += kk;
#define FT(a) coef_at(F, c, ORC_VA_T00 + (a), f[0], f[1], f[2])
                                switch (t) {
                                case 0:
                                    s += FT(0);
                                    if (kk == 0) s += FT(1);
                                    if (jj == 0) s += FT(2);
                                    if (kk == 0 && jj == 0) s += FT(3);
                                    break;
                                case 1:
                                    if (kk == 1) s += FT(1);
                                    if (jj == 0 && kk == 1) s += FT(3);
                                    break;
                                case 2:
                                    if (jj == 1) s += FT(2);
                                    if (jj == 1 && kk == 0) s += FT(3);
                                    break;
                                default:
                                    if (jj == 1 && kk == 1) s += FT(3);
                                }
#undef FT
                            }
                    int a1[3] = {G[0], G[1], G[2]}, a2[3] = {G[0], G[1], G[2]};
                    if (t & 2) a1[d[1]]++;
                    if (t & 1) a2[d[2]]++;
                    int ok = dof_at(C, d[1], a1[0], a1[1], a1[2]) && dof_at(C, d[2], a2[0], a2[1], a2[2]);
                    *cf[ORC_VA_T00 + t] = ok ? rap * s : 0.f;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* active-value predicate of each coefficient array (what setValueOn marked) */
static int coef_active(const vlevel* L, int c, int a, const int* g) {
    const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    switch (a) {
    case ORC_VA_DIAG:
    case ORC_VA_INVDIAG:
        return dof_at(L, c, g[0], g[1], g[2]);
    case ORC_VA_NEGX:
    case ORC_VA_NEGY:
    case ORC_VA_NEGZ: {
        int m[3] = {g[0], g[1], g[2]};
        m[a - ORC_VA_NEGX]--;
        return dof_at(L, c, g[0], g[1], g[2]) && dof_at(L, c, m[0], m[1], m[2]);
    }
    default: {
        int t = a - ORC_VA_T00;
        int p1[3] = {g[0], g[1], g[2]}, p2[3] = {g[0], g[1], g[2]};
        if (t & 2) p1[d1]++;
        if (t & 1) p2[d2]++;
        return dof_at(L, d1, p1[0], p1[1], p1[2]) && dof_at(L, d2, p2[0], p2[1], p2[2]);
    }
    }
}

/* trim_default_nodes (:1692-1721) with LaplacianWithLevel::trimDefaultNodes
 * (simd_vdb_poisson.cpp:1772-1811), level 0 only, eps 1e-3 */
static void trim_level0(orc_visc* h) {
    vlevel* L = &h->lv[0];
    const float eps = 1e-3f;
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        uint32_t bits = 0;
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < VNA; ++a) {
                float def = (a == ORC_VA_INVDIAG) ? 1.0f / h->def_diag : L->def[c][a];
                float tol = fabsf(def * eps);
                float maxerr = 0;
                float* v = L->coef + cidx(L, c, a, i, 0);
                for (int off = 0; off < LSZ; ++off) {
                    int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                    if (!coef_active(L, c, a, g)) continue;
                    float e = fabsf(v[off] - def);
                    if (e > maxerr) maxerr = e;
                }
                if (maxerr <= tol) {
                    for (int off = 0; off < LSZ; ++off) v[off] = def;
                    bits |= 1u << (c * VNA + a);
                }
            }
        L->trim[i] = bits;
    }
    /* a trimmed invdiag leaf reads back the trim default */
    for (int c = 0; c < 3; ++c) L->def[c][ORC_VA_INVDIAG] = 1.0f / h->def_diag;
}

/* ------------------------------------------------------------------------ */
/* explicit_matrix_reducer (:2415-2605): row entries in the reference's push
 * order; rows sorted by column afterwards for the CSR. */
static int row_entries(const vlevel* L, int c, const int* g, int32_t* cols, float* vals) {
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    int n = 0;
    cols[n] = dof_number(L, c, g[0], g[1], g[2]);
    vals[n++] = coef_at(L, c, ORC_VA_DIAG, g[0], g[1], g[2]);
    for (int f = 0; f < 6; ++f) {
        int ax = f / 2;
        int nb[3] = {g[0], g[1], g[2]};
        nb[ax] += (f % 2 == 0) ? 1 : -1;
        int32_t nd = dof_number(L, c, nb[0], nb[1], nb[2]);
        if (nd < 0) continue;
        float term = (f % 2 == 0) ? coef_at(L, c, ORC_VA_NEGX + ax, nb[0], nb[1], nb[2])
                                  : coef_at(L, c, ORC_VA_NEGX + ax, g[0], g[1], g[2]);
        cols[n] = nd;
        vals[n++] = term;
    }
    int m0[3] = {g[0], g[1], g[2]};
    m0[d0]--;
    /* Td2: channel d1 */
    struct { int ch; int dpos[3]; int arr_ch; int arr; int at_m0; } q[8];
    int p1[3] = {g[0], g[1], g[2]}; p1[d1]++;
    int m0p1[3] = {m0[0], m0[1], m0[2]}; m0p1[d1]++;
    int p2[3] = {g[0], g[1], g[2]}; p2[d2]++;
    int m0p2[3] = {m0[0], m0[1], m0[2]}; m0p2[d2]++;
    const int* pos[8] = {g, p1, m0, m0p1, g, m0, p2, m0p2};
    const int ch[8] = {d1, d1, d1, d1, d2, d2, d2, d2};
    const int ach[8] = {d2, d2, d2, d2, d1, d1, d1, d1};
    const int arr[8] = {ORC_VA_T00, ORC_VA_T01, ORC_VA_T10, ORC_VA_T11, ORC_VA_T00, ORC_VA_T01, ORC_VA_T10, ORC_VA_T11};
    const int atm0[8] = {0, 0, 1, 1, 0, 1, 0, 1};
    (void)q;
    for (int k = 0; k < 8; ++k) {
        int32_t nd = dof_number(L, ch[k], pos[k][0], pos[k][1], pos[k][2]);
        if (nd < 0) continue;
        const int* at = atm0[k] ? m0 : g;
        cols[n] = nd;
        vals[n++] = coef_at(L, ach[k], arr[k], at[0], at[1], at[2]);
    }
    return n;
}

int64_t orc_visc_triplets(const orc_visc* h, int level, int32_t* rows, int32_t* cols, float* vals) {
    const vlevel* L = &h->lv[level];
    int64_t n = 0;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < L->nl; ++i) {
            const int32_t* o = L->org + 3 * i;
            for (int off = 0; off < LSZ; ++off) {
                if (!mbit(L->dof + ((size_t)c * L->nl + i) * 8, off)) continue;
                int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                int32_t cc[16];
                float vv[16];
                int k = row_entries(L, c, g, cc, vv);
                int32_t row = cc[0];
                for (int e = 0; e < k; ++e) {
                    if (rows) {
                        rows[n] = row;
                        cols[n] = cc[e];
                        vals[n] = vv[e];
                    }
                    n++;
                }
            }
        }
    return n;
}

static void build_coarsest(orc_visc* h) {
    const vlevel* L = &h->lv[h->nlev - 1];
    int n = L->ndof;
    h->c_n = n;
    h->c_rowptr = (int32_t*)vcalloc((size_t)n + 1, sizeof(int32_t));
    h->c_col = (int32_t*)vcalloc((size_t)n * 15 + 1, sizeof(int32_t));
    h->c_val = (float*)vcalloc((size_t)n * 15 + 1, sizeof(float));
    h->c_row_ch = (int32_t*)vcalloc((size_t)n + 1, sizeof(int32_t));
    h->c_row_leaf = (int32_t*)vcalloc((size_t)n + 1, sizeof(int32_t));
    h->c_row_off = (int32_t*)vcalloc((size_t)n + 1, sizeof(int32_t));
    h->c_invdiag = (float*)vcalloc((size_t)n + 1, sizeof(float));
    int nnz = 0;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < L->nl; ++i) {
            const int32_t* o = L->org + 3 * i;
            for (int off = 0; off < LSZ; ++off) {
                if (!mbit(L->dof + ((size_t)c * L->nl + i) * 8, off)) continue;
                int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                int32_t cc[16];
                float vv[16];
                int k = row_entries(L, c, g, cc, vv);
                int row = cc[0];
                /* insertion sort by column */
                for (int a = 1; a < k; ++a) {
                    int32_t kc = cc[a];
                    float kv = vv[a];
                    int b = a - 1;
                    while (b >= 0 && cc[b] > kc) { cc[b + 1] = cc[b]; vv[b + 1] = vv[b]; b--; }
                    cc[b + 1] = kc;
                    vv[b + 1] = kv;
                }
                h->c_rowptr[row] = nnz;
                float dg = 0.f;
                int has = 0;
                for (int e = 0; e < k; ++e) {
                    h->c_col[nnz] = cc[e];
                    h->c_val[nnz] = vv[e];
                    if (cc[e] == row) { dg = vv[e]; has = 1; }
                    nnz++;
                }
                h->c_invdiag[row] = (has && dg != 0.f) ? 1.0f / dg : 1.0f;
                h->c_row_ch[row] = c;
                h->c_row_leaf[row] = i;
                h->c_row_off[row] = off;
            }
        }
    h->c_rowptr[n] = nnz;
    h->c_b = (float*)vcalloc((size_t)n + 1, sizeof(float));
    h->c_x = (float*)vcalloc((size_t)n + 1, sizeof(float));
    h->c_r = (float*)vcalloc((size_t)n + 1, sizeof(float));
    h->c_p = (float*)vcalloc((size_t)n + 1, sizeof(float));
    h->c_z = (float*)vcalloc((size_t)n + 1, sizeof(float));
    h->c_t = (float*)vcalloc((size_t)n + 1, sizeof(float));
}

static float cdot(int n, const float* a, const float* b) {
    float s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
/* Eigen::ConjugateGradient<RowMajor, Upper|Lower> with DiagonalPreconditioner,
 * tolerance FLT_EPSILON, maxIterations 10, zero guess (:2645-2657) */
static void coarsest_cg(orc_visc* h) {
    int n = h->c_n;
    float *x = h->c_x, *b = h->c_b, *r = h->c_r, *p = h->c_p, *z = h->c_z, *t = h->c_t;
    for (int i = 0; i < n; ++i) { x[i] = 0.f; r[i] = b[i]; }
    float rhsNorm2 = cdot(n, b, b);
    if (rhsNorm2 == 0.f) return;
    const float tol = FLT_EPSILON;
    float threshold = tol * tol * rhsNorm2;
    if (threshold < FLT_MIN) threshold = FLT_MIN;
    float rn2 = cdot(n, r, r);
    if (rn2 < threshold) return;
    for (int i = 0; i < n; ++i) p[i] = h->c_invdiag[i] * r[i];
    float absNew = cdot(n, r, p);
    for (int it = 0; it < 10; ++it) {
        for (int i = 0; i < n; ++i) {
            float s = 0;
            for (int k = h->c_rowptr[i]; k < h->c_rowptr[i + 1]; ++k) s += h->c_val[k] * p[h->c_col[k]];
            t[i] = s;
        }
        float alpha = absNew / cdot(n, p, t);
        for (int i = 0; i < n; ++i) x[i] += alpha * p[i];
        for (int i = 0; i < n; ++i) r[i] -= alpha * t[i];
        rn2 = cdot(n, r, r);
        if (rn2 < threshold) break;
        for (int i = 0; i < n; ++i) z[i] = h->c_invdiag[i] * r[i];
        float absOld = absNew;
        absNew = cdot(n, r, z);
        float beta = absNew / absOld;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
}

/* The same CG with the operation order of the CUDA coarsest kernel
 * (uaamg_b200/csrc/viscosity_kernels.cuh, k_vcoarsest_cg<ROWS>): row i belongs
 * to thread tid = i % 256 (the k-th row of a thread is tid + 256 k, ROWS rows
 * per thread by system size); a dot product is every thread's fused
 * multiply-add chain over its rows, then a shuffle-down tree inside each
 * 32-lane warp, then ((w0+w1)+(w2+w3)) + ((w4+w5)+(w6+w7)) over the 8 warp
 * sums; a row of A p is a fused multiply-add chain over its 15 ELL entries in
 * column order, the padding entries adding 0 * 0; the vector updates are fused
 * multiply-adds (x += alpha p, r -= alpha A p, p = z + beta p).  Eigen's own summation order
 * depends on its vectorisation (and its version is not pinned), so either
 * order restates the reference's coarsest solve; this one makes the oracle's
 * whole viscosity PCG reproducible bit for bit on the GPU. */
#define VCG_NT 256
static float warp_tree32(const float* lane_in) {
    /* lane 0 of v += __shfl_down_sync(v, o), o = 16, 8, 4, 2, 1 (a lane
     * whose source lane is out of range reads its own value) */
    float a[32], b[32];
    memcpy(a, lane_in, sizeof(a));
    for (int o = 16; o > 0; o >>= 1) {
        for (int l = 0; l < 32; ++l) b[l] = a[l] + (l + o < 32 ? a[l + o] : a[l]);
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}
static float block_tree256(const float* part) {
    float w[8];
    for (int k = 0; k < 8; ++k) w[k] = warp_tree32(part + 32 * k);
    return ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7]));
}
#define VCG_ELL 15 /* entries per row of the kernel's ELL matrix */
static int vcg_rows(int n) {
    return n <= 2 * VCG_NT ? 2 : (n <= 4 * VCG_NT ? 4 : (n <= 8 * VCG_NT ? 8 : 16));
}
static void coarsest_cg_kernel_order(orc_visc* h) {
    const int n = h->c_n, R = vcg_rows(n), N = R * VCG_NT;
    /* per row slot j = tid + k * 256 (j >= n: padding, zero) */
    float* x = (float*)vcalloc((size_t)N, sizeof(float));
    float* r = (float*)vcalloc((size_t)N, sizeof(float));
    float* p = (float*)vcalloc((size_t)N, sizeof(float));
    float* z = (float*)vcalloc((size_t)N, sizeof(float));
    float* t = (float*)vcalloc((size_t)N, sizeof(float));
    float* iv = (float*)vcalloc((size_t)N, sizeof(float));
    float part[VCG_NT], part2[VCG_NT];
    for (int j = 0; j < n; ++j) { r[j] = h->c_b[j]; iv[j] = h->c_invdiag[j]; }
#define THREAD_SUM(dst, ea, eb)                                 \
    for (int tid = 0; tid < VCG_NT; ++tid) {                    \
        float v_ = 0.f;                                         \
        for (int k = 0; k < R; ++k) {                           \
            const int j = tid + k * VCG_NT;                     \
            v_ = fmaf((ea), (eb), v_);                          \
        }                                                       \
        dst[tid] = v_;                                          \
    }
    THREAD_SUM(part, r[j], r[j]);
    const float rhsNorm2 = block_tree256(part);
    const float threshold = fmaxf((FLT_EPSILON * FLT_EPSILON) * rhsNorm2, FLT_MIN);
    if (rhsNorm2 != 0.f && !(rhsNorm2 < threshold)) {
        for (int j = 0; j < N; ++j) p[j] = iv[j] * r[j];
        THREAD_SUM(part, r[j], p[j]);
        float absNew = block_tree256(part);
        for (int it = 0; it < 10; ++it) {
            for (int j = 0; j < N; ++j) {
                float sacc = 0.f;
                if (j < n) {
                    const int len = h->c_rowptr[j + 1] - h->c_rowptr[j];
                    for (int k = h->c_rowptr[j]; k < h->c_rowptr[j + 1]; ++k) sacc = fmaf(h->c_val[k], p[h->c_col[k]], sacc);
                    for (int e = len; e < VCG_ELL; ++e) sacc = fmaf(0.f, 0.f, sacc);
                }
                t[j] = sacc;
            }
            THREAD_SUM(part, p[j], t[j]);
            const float alpha = absNew / block_tree256(part);
            for (int j = 0; j < N; ++j) {
                x[j] = fmaf(alpha, p[j], x[j]);
                r[j] = fmaf(-alpha, t[j], r[j]);
                z[j] = iv[j] * r[j];
            }
            THREAD_SUM(part, r[j], r[j]);
            THREAD_SUM(part2, r[j], z[j]);
            const float rr = block_tree256(part), rz = block_tree256(part2);
            if (rr < threshold) break;
            const float absOld = absNew;
            absNew = rz;
            const float beta = absNew / absOld;
            for (int j = 0; j < N; ++j) p[j] = fmaf(beta, p[j], z[j]);
        }
    }
#undef THREAD_SUM
    for (int j = 0; j < n; ++j) h->c_x[j] = x[j];
    free(x); free(r); free(p); free(z); free(t); free(iv);
}

void orc_visc_set_coarsest_order(orc_visc* h, int order) { h->c_order = order; }

void orc_visc_coarsest_solve(orc_visc* h, const float* rhs, float* out) {
    const vlevel* L = &h->lv[h->nlev - 1];
    for (int i = 0; i < h->c_n; ++i) h->c_b[i] = rhs[vidx(L, h->c_row_ch[i], h->c_row_leaf[i], h->c_row_off[i])];
    if (h->c_order == ORC_CG_ORDER_SEQUENTIAL) coarsest_cg(h);
    else coarsest_cg_kernel_order(h);
    for (int i = 0; i < h->c_n; ++i) out[vidx(L, h->c_row_ch[i], h->c_row_leaf[i], h->c_row_off[i])] = h->c_x[i];
}

/* ------------------------------------------------------------------------ */
/* light_weight_applier::component_operator<c> (:2849-3603) for one channel.
 * color: -1 all DOFs, 0 red ((x+y+z) even), 1 black. */
static void apply_channel(const vlevel* L, int c, int mode, const float* lhs, const float* rhs, float* out) {
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int is_gs = (mode == ORC_VMODE_RED_GS || mode == ORC_VMODE_BLACK_GS);
    const float w = 1.0f, one_minus_w = 1.0f - w; /* m_damped_jacobi_coef = 10/10 */
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < L->nl; ++i) {
        const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
        int any = 0;
        for (int q = 0; q < 8; ++q) any |= (m[q] != 0);
        if (!any) {
            if (!is_gs) memset(out + vidx(L, c, i, 0), 0, LSZ * sizeof(float));
            continue;
        }
        int32_t nb[27];
        nb27(L, i, nb);
        const int32_t* o = L->org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            int lx = off >> 6, ly = (off >> 3) & 7, lz = off & 7;
            if (!mbit(m, off)) {
                if (!is_gs) out[vidx(L, c, i, off)] = 0.f;
                continue;
            }
            if (is_gs) {
                int red = ((o[0] + lx + o[1] + ly + o[2] + lz) & 1) == 0;
                if ((mode == ORC_VMODE_RED_GS) != red) continue;
            }
#define VEC(ch, X, Y, Z) ({ int _o; int32_t _l = nb_locate(nb, X, Y, Z, &_o); \
                            _l < 0 ? 0.f : lhs[vidx(L, ch, _l, _o)]; })
#define COEF(ch, a, X, Y, Z) ({ int _o; int32_t _l = nb_locate(nb, X, Y, Z, &_o); \
                                _l < 0 ? L->app[ch][a] : L->coef[cidx(L, ch, a, _l, _o)]; })
            int l[3] = {lx, ly, lz};
            /* same channel, absolute axes */
            float fr[7];
            for (int ax = 0; ax < 3; ++ax) {
                int p[3] = {l[0], l[1], l[2]};
                p[ax]++;
                int q[3] = {l[0], l[1], l[2]};
                q[ax]--;
                float up = VEC(c, p[0], p[1], p[2]);
                float wp = COEF(c, ORC_VA_NEGX + ax, p[0], p[1], p[2]);
                float um = VEC(c, q[0], q[1], q[2]);
                float wm = COEF(c, ORC_VA_NEGX + ax, l[0], l[1], l[2]);
                fr[1 + 2 * ax] = up * wp;
                fr[2 + 2 * ax] = um * wm;
            }
            float off_sum = ((fr[1] + fr[2]) + (fr[3] + fr[4])) + (fr[5] + fr[6]);
            int m0[3] = {l[0], l[1], l[2]};
            m0[d0]--;
            int p1[3] = {l[0], l[1], l[2]};
            p1[d1]++;
            int m0p1[3] = {m0[0], m0[1], m0[2]};
            m0p1[d1]++;
            int p2[3] = {l[0], l[1], l[2]};
            p2[d2]++;
            int m0p2[3] = {m0[0], m0[1], m0[2]};
            m0p2[d2]++;
            float R0 = VEC(d1, l[0], l[1], l[2]) * COEF(d2, ORC_VA_T00, l[0], l[1], l[2]);
            float R1 = COEF(d2, ORC_VA_T01, l[0], l[1], l[2]) * VEC(d1, p1[0], p1[1], p1[2]);
            float R2 = COEF(d2, ORC_VA_T10, m0[0], m0[1], m0[2]) * VEC(d1, m0[0], m0[1], m0[2]);
            float R3 = COEF(d2, ORC_VA_T11, m0[0], m0[1], m0[2]) * VEC(d1, m0p1[0], m0p1[1], m0p1[2]);
            float Q0 = COEF(d1, ORC_VA_T00, l[0], l[1], l[2]) * VEC(d2, l[0], l[1], l[2]);
            float Q1 = COEF(d1, ORC_VA_T01, m0[0], m0[1], m0[2]) * VEC(d2, m0[0], m0[1], m0[2]);
            float Q2 = COEF(d1, ORC_VA_T10, l[0], l[1], l[2]) * VEC(d2, p2[0], p2[1], p2[2]);
            float Q3 = COEF(d1, ORC_VA_T11, m0[0], m0[1], m0[2]) * VEC(d2, m0p2[0], m0p2[1], m0p2[2]);
            float td2 = (R0 + R1) + (R2 + R3);
            float td1 = (Q0 + Q1) + (Q2 + Q3);
            off_sum = off_sum + td2;
            off_sum = off_sum + td1;
            float u = lhs[vidx(L, c, i, off)];
            float dg = COEF(c, ORC_VA_DIAG, l[0], l[1], l[2]);
            float res;
            switch (mode) {
            case ORC_VMODE_RED_GS:
            case ORC_VMODE_BLACK_GS: {
                float r = rhs[vidx(L, c, i, off)] - off_sum;
                r = r * COEF(c, ORC_VA_INVDIAG, l[0], l[1], l[2]);
                r = r * w;
                res = fmaf(u, one_minus_w, r);
                break;
            }
            case ORC_VMODE_JACOBI: {
                float a = fmaf(u, dg, off_sum);
                float r = rhs[vidx(L, c, i, off)] - a;
                r = r * COEF(c, ORC_VA_INVDIAG, l[0], l[1], l[2]);
                res = fmaf(w, r, u);
                break;
            }
            case ORC_VMODE_RESIDUAL:
                res = rhs[vidx(L, c, i, off)] - fmaf(u, dg, off_sum);
                break;
            default:
                res = fmaf(u, dg, off_sum);
            }
#undef VEC
#undef COEF
            out[vidx(L, c, i, off)] = res;
        }
    }
}

void orc_visc_apply(orc_visc* h, int level, int mode, int channel, const float* lhs, const float* rhs,
                    float* out) {
    const vlevel* L = &h->lv[level];
    if (mode == ORC_VMODE_RED_GS || mode == ORC_VMODE_BLACK_GS) {
        apply_channel(L, channel, mode, out, rhs, out);
        return;
    }
    for (int c = 0; c < 3; ++c) apply_channel(L, c, mode, lhs, rhs, out);
}

/* XYZ_RBGS_apply (:2238-2269) / ZYX_RBGS_apply (:2271-2302) */
void orc_visc_rbgs(orc_visc* h, int level, int order, float* lhs, const float* rhs) {
    const vlevel* L = &h->lv[level];
    if (order == 0) {
        for (int c = 0; c < 3; ++c) {
            apply_channel(L, c, ORC_VMODE_RED_GS, lhs, rhs, lhs);
            apply_channel(L, c, ORC_VMODE_BLACK_GS, lhs, rhs, lhs);
        }
    } else {
        for (int c = 2; c >= 0; --c) {
            apply_channel(L, c, ORC_VMODE_BLACK_GS, lhs, rhs, lhs);
            apply_channel(L, c, ORC_VMODE_RED_GS, lhs, rhs, lhs);
        }
    }
}

/* restriction (:2353-2413): coarse = (sum of active fine) * 0.125 * 0.5 * 2 */
void orc_visc_restrict(const orc_visc* h, int fine_level, const float* fine, float* coarse) {
    const vlevel* F = &h->lv[fine_level];
    const vlevel* C = &h->lv[fine_level + 1];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C->nl; ++i)
        for (int c = 0; c < 3; ++c) {
            const uint64_t* m = C->dof + ((size_t)c * C->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off) {
                size_t at = vidx(C, c, i, off);
                if (!mbit(m, off)) { coarse[at] = 0.f; continue; }
                int lx = off >> 6, ly = (off >> 3) & 7, lz = off & 7;
                int q = ((lx >= 4) << 2) | ((ly >= 4) << 1) | (lz >= 4);
                int32_t fl = C->child[8 * i + q];
                if (fl < 0) continue;
                const uint64_t* fm = F->dof + ((size_t)c * F->nl + fl) * 8;
                int base = voff(2 * lx, 2 * ly, 2 * lz);
                float s = 0;
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int k = 0; k < 2; ++k) {
                            int fo = base + 64 * a + 8 * b + k;
                            if (mbit(fm, fo)) s += fine[vidx(F, c, fl, fo)];
                        }
                coarse[at] = s * 0.125f * 0.5f * 2.0f;
            }
        }
}

/* prolongation<true> (:2659-2729) */
void orc_visc_prolongate(const orc_visc* h, int fine_level, const float* coarse, float* fine) {
    const vlevel* F = &h->lv[fine_level];
    const vlevel* C = &h->lv[fine_level + 1];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C->nl; ++i)
        for (int c = 0; c < 3; ++c) {
            const uint64_t* m = C->dof + ((size_t)c * C->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off) {
                if (!mbit(m, off)) continue;
                int lx = off >> 6, ly = (off >> 3) & 7, lz = off & 7;
                int q = ((lx >= 4) << 2) | ((ly >= 4) << 1) | (lz >= 4);
                int32_t fl = C->child[8 * i + q];
                if (fl < 0) continue;
                float v = coarse[vidx(C, c, i, off)];
                const uint64_t* fm = F->dof + ((size_t)c * F->nl + fl) * 8;
                int base = voff(2 * lx, 2 * ly, 2 * lz);
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int k = 0; k < 2; ++k) {
                            int fo = base + 64 * a + 8 * b + k;
                            if (mbit(fm, fo)) fine[vidx(F, c, fl, fo)] += v;
                        }
            }
        }
}

/* mucycle (:3837-3884), mu = 2, n = 2.  The second visit of the coarsest
 * level solves the same rhs from the same zero guess, so it is skipped. */
static void mucycle(orc_visc* h, float* lhs, const float* rhs, int for_precon, int level) {
    vlevel* L = &h->lv[level];
    if (level == h->nlev - 1) {
        orc_visc_coarsest_solve(h, rhs, lhs);
        return;
    }
    if (for_precon) memset(lhs, 0, (size_t)3 * L->nl * LSZ * sizeof(float));
    for (int it = 0; it < 2; ++it) orc_visc_rbgs(h, level, 0, lhs, rhs);
    for (int c = 0; c < 3; ++c) apply_channel(L, c, ORC_VMODE_RESIDUAL, lhs, rhs, L->tmp);
    vlevel* P = &h->lv[level + 1];
    orc_visc_restrict(h, level, L->tmp, P->rhs);
    mucycle(h, P->lhs, P->rhs, 1, level + 1);
    if (level + 1 != h->nlev - 1) mucycle(h, P->lhs, P->rhs, 0, level + 1);
    orc_visc_prolongate(h, level, P->lhs, lhs);
    for (int it = 0; it < 2; ++it) orc_visc_rbgs(h, level, 1, lhs, rhs);
}

void orc_visc_precondition(orc_visc* h, const float* r, float* out) {
    mucycle(h, out, r, 1, 0);
}

/* ------------------------------------------------------------------------ */
/* lv_abs_max / lv_dot / lv_axpy / lv_xpay (:3756-3820) */
float orc_visc_abs_max(const orc_visc* h, int level, const float* v) {
    const vlevel* L = &h->lv[level];
    float result = 0;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < L->nl; ++i) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off)
                if (mbit(m, off)) {
                    float a = fabsf(v[vidx(L, c, i, off)]);
                    if (a > result) result = a;
                }
        }
    return result;
}
float orc_visc_dot(const orc_visc* h, int level, const float* a, const float* b) {
    const vlevel* L = &h->lv[level];
    float result = 0;
    float* part = (float*)vcalloc((size_t)(L->nl ? L->nl : 1), sizeof(float));
    for (int c = 0; c < 3; ++c) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L->nl; ++i) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            float s = 0;
            for (int off = 0; off < LSZ; ++off)
                if (mbit(m, off)) s += a[vidx(L, c, i, off)] * b[vidx(L, c, i, off)];
            part[i] = s;
        }
        float cs = 0;
        for (int i = 0; i < L->nl; ++i) cs += part[i];
        result += cs;
    }
    free(part);
    return result;
}
static void vaxpy(const vlevel* L, float alpha, const float* x, float* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int c = 0; c < 3; ++c) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off)
                if (mbit(m, off)) y[vidx(L, c, i, off)] += alpha * x[vidx(L, c, i, off)];
        }
}
static void vxpay(const vlevel* L, float alpha, const float* x, float* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int c = 0; c < 3; ++c) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off)
                if (mbit(m, off)) {
                    size_t at = vidx(L, c, i, off);
                    y[at] = x[at] + alpha * y[at];
                }
        }
}

/* simd_viscosity3d::pcg_solve (:3691-3754) */
int orc_visc_pcg(orc_visc* h, float* x, const float* b, float tol, int max_iter, int* iterations,
                 float* final_abs_res) {
    vlevel* L = &h->lv[0];
    size_t n = (size_t)3 * L->nl * LSZ;
    float* r = (float*)vcalloc(n, sizeof(float));
    float* p = (float*)vcalloc(n, sizeof(float));
    float* z = (float*)vcalloc(n, sizeof(float));
    int status = 0, it = 0;
    for (int c = 0; c < 3; ++c) apply_channel(L, c, ORC_VMODE_RESIDUAL, x, b, r);
    float nu = orc_visc_abs_max(h, 0, r);
    float numax = tol * nu;
    if (!(nu <= numax)) {
        mucycle(h, p, r, 1, 0);
        float rho = orc_visc_dot(h, 0, p, r);
        status = 1;
        for (it = 0; it < max_iter; ++it) {
            for (int c = 0; c < 3; ++c) apply_channel(L, c, ORC_VMODE_NORMAL, p, NULL, z);
            float sigma = orc_visc_dot(h, 0, p, z);
            float alpha = rho / sigma;
            vaxpy(L, -alpha, z, r);
            nu = orc_visc_abs_max(h, 0, r);
            if (nu <= numax || it == max_iter - 1) {
                vaxpy(L, alpha, p, x);
                status = (nu <= numax) ? 0 : 1;
                break;
            }
            mucycle(h, z, r, 1, 0);
            float rho_new = orc_visc_dot(h, 0, z, r);
            float beta = rho_new / rho;
            rho = rho_new;
            vaxpy(L, alpha, p, x);
            vxpay(L, beta, z, p);
        }
        if (max_iter <= 0) it = 0;
    }
    if (iterations) *iterations = it;
    if (final_abs_res) *final_abs_res = nu;
    free(r);
    free(p);
    free(z);
    return status;
}

/* ------------------------------------------------------------------------ */
static inline int solid_at(const orc_visc* h, int c, const int* g) {
    int32_t li = leafmap_find(&h->solid_map, g[0], g[1], g[2]);
    if (li < 0) return 0;
    return mbit(h->is_solid + ((size_t)c * h->solid_leaves.n + li) * 8, voff(g[0], g[1], g[2]));
}
/* one cross term of channel cp at voxel p (rhs_reducer :1889-1972):
 * jk = 0..3 for 00, 01, 10, 11 */
static float cross_term(const orc_visc* h, int cp, const int* p, int jk) {
    const int d1 = (cp + 1) % 3, d2 = (cp + 2) % 3;
    int j = jk >> 1, k = jk & 1;
    int e[3] = {p[0], p[1], p[2]};
    e[d1] += j;
    e[d2] += k;
    float ev = field_get(&h->edge_vol[cp], e[0], e[1], e[2]);
    float q[3] = {(float)p[0], (float)p[1], (float)p[2]};
    q[d1] += j ? 0.5f : -0.5f;
    q[d2] += k ? 0.5f : -0.5f;
    float sv = box_sample(&h->mu, q[0], q[1], q[2]);
    float f = (j == k) ? h->factor : -h->factor;
    return f * ev * sv;
}

/* Solid-velocity part of build_rhs (:2039-2084): rhs_reducer's scattered
 * contributions gathered per DOF.  The same-channel sum comes first, then the
 * cross terms of channel c+1 (c as its second face) and of channel c+2 (c as
 * its first face), each in 00, 01, 10, 11 order. */
static void rhs_solid(const orc_visc* h, const ogrid* sv, float* rhs_out) {
    const vlevel* L = &h->lv[0];
    const float factor = h->factor;
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        for (int c = 0; c < 3; ++c) {
            const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off) {
                if (!mbit(m, off)) continue;
                int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                float acc = 0.f;
                int have = 0;
#define ADD(v) do { float _v = (v); if (have) acc += _v; else { acc = _v; have = 1; } } while (0)
                /* same channel (:1776-1868) */
                float temp_rhs = 0;
                {
                    int q[3] = {g[0], g[1], g[2]};
                    q[d0]++;
                    float term = 2 * factor * field_get(&h->voxel_vol, g[0], g[1], g[2]) *
                                 ogrid_get(&h->mu, g[0], g[1], g[2], 0);
                    if (!dof_at(L, c, q[0], q[1], q[2]) && solid_at(h, c, q))
                        temp_rhs += term * ogrid_get(sv, q[0], q[1], q[2], d0);
                }
                {
                    int q[3] = {g[0], g[1], g[2]};
                    q[d0]--;
                    float term = 2 * factor * field_get(&h->voxel_vol, q[0], q[1], q[2]) *
                                 ogrid_get(&h->mu, q[0], q[1], q[2], 0);
                    if (!dof_at(L, c, q[0], q[1], q[2]) && solid_at(h, c, q))
                        temp_rhs += term * ogrid_get(sv, q[0], q[1], q[2], d0);
                }
                float fc[3] = {(float)g[0], (float)g[1], (float)g[2]};
                fc[d0] -= 0.5f;
                for (int s = 0; s < 4; ++s) {
                    /* s: +d1, -d1, +d2, -d2 */
                    int ax = (s < 2) ? d1 : d2;
                    int eax = (s < 2) ? d2 : d1; /* edge channel */
                    int pos = (s % 2 == 0);
                    int e[3] = {g[0], g[1], g[2]};
                    if (pos) e[ax]++;
                    float ev = field_get(&h->edge_vol[eax], e[0], e[1], e[2]);
                    float p[3] = {fc[0], fc[1], fc[2]};
                    p[ax] += pos ? 0.5f : -0.5f;
                    float smu = box_sample(&h->mu, p[0], p[1], p[2]);
                    float term = factor * ev * smu;
                    int q[3] = {g[0], g[1], g[2]};
                    q[ax] += pos ? 1 : -1;
                    if (!dof_at(L, c, q[0], q[1], q[2]) && solid_at(h, c, q))
                        temp_rhs += term * ogrid_get(sv, q[0], q[1], q[2], d0);
                }
                if (temp_rhs != 0) ADD(temp_rhs);
                /* channel c+1 = cp, with c as its second face (d2' = c), d1' = c+2 */
                {
                    const int cp = (c + 1) % 3, a1 = (cp + 1) % 3;
                    int gm[3] = {g[0], g[1], g[2]};
                    gm[c]--;
                    int q[3];
                    /* 00 at g */
                    if (!dof_at(L, a1, g[0], g[1], g[2]) && solid_at(h, a1, g))
                        ADD(-cross_term(h, cp, g, 0) * ogrid_get(sv, g[0], g[1], g[2], a1));
                    /* 01 at g - e_c */
                    if (!dof_at(L, a1, gm[0], gm[1], gm[2]) && solid_at(h, a1, gm))
                        ADD(-cross_term(h, cp, gm, 1) * ogrid_get(sv, gm[0], gm[1], gm[2], a1));
                    /* 10 at g: face a1 at g + e_a1 */
                    q[0] = g[0]; q[1] = g[1]; q[2] = g[2];
                    q[a1]++;
                    if (!dof_at(L, a1, q[0], q[1], q[2]) && solid_at(h, a1, q))
                        ADD(-cross_term(h, cp, g, 2) * ogrid_get(sv, q[0], q[1], q[2], a1));
                    /* 11 at g - e_c: face a1 at g - e_c + e_a1 */
                    q[0] = gm[0]; q[1] = gm[1]; q[2] = gm[2];
                    q[a1]++;
                    if (!dof_at(L, a1, q[0], q[1], q[2]) && solid_at(h, a1, q))
                        ADD(-cross_term(h, cp, gm, 3) * ogrid_get(sv, q[0], q[1], q[2], a1));
                }
                /* channel c+2 = cp, with c as its first face (d1' = c), d2' = c+1 */
                {
                    const int cp = (c + 2) % 3, a2 = (cp + 2) % 3;
                    int gm[3] = {g[0], g[1], g[2]};
                    gm[c]--;
                    int q[3];
                    /* 00 at g */
                    if (!dof_at(L, a2, g[0], g[1], g[2]) && solid_at(h, a2, g))
                        ADD(-cross_term(h, cp, g, 0) * ogrid_get(sv, g[0], g[1], g[2], a2));
                    /* 01 at g: face a2 at g + e_a2 */
                    q[0] = g[0]; q[1] = g[1]; q[2] = g[2];
                    q[a2]++;
                    if (!dof_at(L, a2, q[0], q[1], q[2]) && solid_at(h, a2, q))
                        ADD(-cross_term(h, cp, g, 1) * ogrid_get(sv, q[0], q[1], q[2], a2));
                    /* 10 at g - e_c */
                    if (!dof_at(L, a2, gm[0], gm[1], gm[2]) && solid_at(h, a2, gm))
                        ADD(-cross_term(h, cp, gm, 2) * ogrid_get(sv, gm[0], gm[1], gm[2], a2));
                    /* 11 at g - e_c: face a2 at g - e_c + e_a2 */
                    q[0] = gm[0]; q[1] = gm[1]; q[2] = gm[2];
                    q[a2]++;
                    if (!dof_at(L, a2, q[0], q[1], q[2]) && solid_at(h, a2, q))
                        ADD(-cross_term(h, cp, gm, 3) * ogrid_get(sv, q[0], q[1], q[2], a2));
                }
#undef ADD
                if (have) {
                    size_t at = vidx(L, c, i, off);
                    rhs_out[at] = rhs_out[at] + acc;
                }
            }
        }
    }
}

/* build_rhs (:2005-2087) */
void orc_visc_build_rhs(const orc_visc* h,
    int64_t u_n, const int32_t* u_origins, const float* u_values, float u_bg,
    int64_t v_n, const int32_t* v_origins, const float* v_values, float v_bg,
    int64_t w_n, const int32_t* w_origins, const float* w_values, float w_bg,
    int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
    float* rhs_out) {
    const vlevel* L = &h->lv[0];
    ogrid vel[3], sv;
    float bgs[3] = {u_bg, v_bg, w_bg};
    ogrid_init(&vel[0], u_n, u_origins, NULL, u_values, 1, &bgs[0]);
    ogrid_init(&vel[1], v_n, v_origins, NULL, v_values, 1, &bgs[1]);
    ogrid_init(&vel[2], w_n, w_origins, NULL, w_values, 1, &bgs[2]);
    float zero3[3] = {0, 0, 0};
    ogrid_init(&sv, sv_n, sv_origins, NULL, sv_values, 3, sv_bg3 ? sv_bg3 : zero3);
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        for (int c = 0; c < 3; ++c) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            for (int off = 0; off < LSZ; ++off) {
                size_t at = vidx(L, c, i, off);
                if (!mbit(m, off)) { rhs_out[at] = 0.f; continue; }
                int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                float fv = field_get(&h->face_vol[c], g[0], g[1], g[2]);
                if (fv < 1e-1f) fv = 1e-1f;
                rhs_out[at] = ogrid_get(&vel[c], g[0], g[1], g[2], 0) * fv;
            }
        }
    }
    int any_solid = 0;
    for (size_t q = 0; q < (size_t)3 * h->solid_leaves.n * 8 && !any_solid; ++q) any_solid = h->is_solid[q] != 0;
    if (any_solid) rhs_solid(h, &sv, rhs_out);
    for (int c = 0; c < 3; ++c) leafmap_free(&vel[c].map);
    leafmap_free(&sv.map);
}

/* ------------------------------------------------------------------------ */
static int32_t* dup_i32(const int32_t* p, size_t n) {
    int32_t* q = (int32_t*)vcalloc(n ? n : 1, sizeof(int32_t));
    if (n) memcpy(q, p, n * sizeof(int32_t));
    return q;
}
static float* dup_f32(const float* p, size_t n) {
    float* q = (float*)vcalloc(n ? n : 1, sizeof(float));
    if (n) memcpy(q, p, n * sizeof(float));
    return q;
}

orc_visc* orc_visc_create(
    int64_t liq_n, const int32_t* liq_origins, const uint64_t* liq_masks,
    const float* liq_values, float liq_background,
    int64_t sol_n, const int32_t* sol_origins, const float* sol_values, float sol_background,
    int64_t mu_n, const int32_t* mu_origins, const float* mu_values, float mu_background,
    float dt, float rho, float dx, int build_hierarchy) {
    orc_visc* h = (orc_visc*)vcalloc(1, sizeof(orc_visc));
    h->dt = dt;
    h->rho = rho;
    h->dx = dx;
    h->factor = dt / (rho * dx * dx);
    h->def_off = h->factor * mu_background;
    h->def_diag = 1.0f + 8.0f * h->def_off;
    h->mu_org = dup_i32(mu_origins, (size_t)mu_n * 3);
    h->mu_val = dup_f32(mu_values, (size_t)mu_n * LSZ);
    ogrid_init(&h->mu, mu_n, h->mu_org, NULL, h->mu_val, 1, &mu_background);
    ogrid liq, sol;
    ogrid_init(&liq, liq_n, liq_origins, liq_masks, liq_values, 1, &liq_background);
    ogrid_init(&sol, sol_n, sol_origins, NULL, sol_values, 1, &sol_background);
    build_level0(h, &liq, liq_masks, &sol, &h->mu);
    leafmap_free(&liq.map);
    leafmap_free(&sol.map);
    h->nlev = 1;
    if (build_hierarchy) {
        while (h->lv[h->nlev - 1].ndof > 4000 && h->nlev < 32) {
            build_coarse(h, h->nlev - 1);
            h->nlev++;
        }
    }
    trim_level0(h);
    build_coarsest(h);
    return h;
}

void orc_visc_free(orc_visc* h) {
    if (!h) return;
    for (int l = 0; l < h->nlev; ++l) {
        vlevel* L = &h->lv[l];
        leafmap_free(&L->map);
        free(L->org); free(L->dof); free(L->dof_base); free(L->coef); free(L->trim);
        free(L->child); free(L->lhs); free(L->rhs); free(L->tmp);
    }
    field_free(&h->voxel_vol);
    for (int c = 0; c < 3; ++c) { field_free(&h->face_vol[c]); field_free(&h->edge_vol[c]); }
    leafmap_free(&h->solid_map);
    free(h->solid_leaves.org);
    free(h->is_solid);
    leafmap_free(&h->mu.map);
    free(h->mu_org); free(h->mu_val);
    free(h->c_rowptr); free(h->c_col); free(h->c_val); free(h->c_row_ch); free(h->c_row_leaf);
    free(h->c_row_off); free(h->c_invdiag); free(h->c_b); free(h->c_x); free(h->c_r); free(h->c_p);
    free(h->c_z); free(h->c_t);
    free(h);
}

int orc_visc_num_levels(const orc_visc* h) { return h->nlev; }
int orc_visc_leaf_count(const orc_visc* h, int level) { return h->lv[level].nl; }
int orc_visc_ndof(const orc_visc* h, int level) { return h->lv[level].ndof; }
void orc_visc_topology(const orc_visc* h, int level, int32_t* origins, uint64_t* dof_masks) {
    const vlevel* L = &h->lv[level];
    if (origins) memcpy(origins, L->org, (size_t)L->nl * 3 * sizeof(int32_t));
    if (dof_masks) memcpy(dof_masks, L->dof, (size_t)3 * L->nl * 8 * sizeof(uint64_t));
}
void orc_visc_coefficients(const orc_visc* h, int level, float* coef, uint32_t* trim) {
    const vlevel* L = &h->lv[level];
    if (coef) memcpy(coef, L->coef, (size_t)3 * VNA * L->nl * LSZ * sizeof(float));
    if (trim) memcpy(trim, L->trim, (size_t)L->nl * sizeof(uint32_t));
}
void orc_visc_defaults(const orc_visc* h, int level, float* out27) {
    const vlevel* L = &h->lv[level];
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < VNA; ++a) out27[c * VNA + a] = L->app[c][a];
}
void orc_visc_dof_index(const orc_visc* h, int level, int32_t* out) {
    const vlevel* L = &h->lv[level];
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < L->nl; ++i) {
            const uint64_t* m = L->dof + ((size_t)c * L->nl + i) * 8;
            int32_t d = L->dof_base[(size_t)c * L->nl + i];
            for (int off = 0; off < LSZ; ++off)
                out[vidx(L, c, i, off)] = mbit(m, off) ? d++ : -1;
        }
}
