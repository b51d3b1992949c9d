/*
 * poisson_oracle.c -- CPU restatement of the reference's SIMD UAAMG-PCG
 * Poisson solver (SIMD_UAAMG/simd_vdb_poisson.cpp) on flattened 8^3 leaves.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
 * baseline.  Parity is UNPINNED except for fraction_inside (the solver cannot
 * be built here: it needs OpenVDB, TBB and Eigen, and it ships no golden
 * vectors; its levelset_util.cpp is plain C++, and tests/test_oracle_ref_pin.py
 * checks this file's fraction_inside against it bit for bit).
 *
 * Float arithmetic follows the reference operation by operation (the AVX
 * intrinsics in LightWeightApplier are mul/add/fmadd/sub in a fixed order);
 * this file must be compiled with -ffp-contract=off so that the compiler
 * does not fuse what the reference keeps separate.
 *
 * OpenMP over leaves stands in for TBB's LeafManager::foreach.  Reductions
 * are per-leaf float partials summed in leaf order, which is one of the
 * schedules the reference's tbb::parallel_reduce can produce, and is
 * deterministic for any thread count.
 */
#include "uaamg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_common.h"

/* ------------------------------------------------------------------------ */
typedef struct {
    int nl;
    int32_t* org;      /* [nl][3] */
    uint64_t* mask;    /* [nl][8] DOF mask */
    int32_t* nbr;      /* [nl][6]  -x +x -y +y -z +z, -1 if absent */
    int32_t* child;    /* [nl][8]  fine leaves (coarse levels), -1 if absent */
    int32_t* dof_base; /* [nl] */
    int ndof;
    float *diag, *cx, *cy, *cz, *invdiag, *spai0; /* [nl][512], effective values */
    uint8_t* flags;    /* trimmed: bit0 diag, bit1 x, bit2 y, bit3 z, bit4 spai0 */
    int spai0_ready;
    float dt, dx, t;
    float def_diag, def_face, def_invdiag, def_spai0;
    float w_sor;
    leafmap map;
    float *lhs, *rhs, *tmp; /* mu-cycle scratch ([nl][512]) */
} olevel;

struct orc_poisson {
    int nlev;
    olevel lv[32];
    /* coarsest CSR */
    int c_n;
    int32_t* c_rowptr; int32_t* c_col; float* c_val; float* c_invdiag;
    int32_t* c_dof_leaf; int32_t* c_dof_off;
    float *c_b, *c_x, *c_r, *c_p, *c_z, *c_t;
};

static void* xcalloc(size_t n, size_t s) {
    void* p = calloc(n ? n : 1, s);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* neighbour voxel: returns leaf index (or -1) and writes the offset */
static inline int32_t nbv(const olevel* L, int32_t li, int off, int dir, int* noff) {
    int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
    switch (dir) {
    case 0: if (x > 0) { *noff = off - 64; return li; } *noff = off + 448; return L->nbr[6 * li + 0];
    case 1: if (x < 7) { *noff = off + 64; return li; } *noff = off - 448; return L->nbr[6 * li + 1];
    case 2: if (y > 0) { *noff = off - 8; return li; } *noff = off + 56; return L->nbr[6 * li + 2];
    case 3: if (y < 7) { *noff = off + 8; return li; } *noff = off - 56; return L->nbr[6 * li + 3];
    case 4: if (z > 0) { *noff = off - 1; return li; } *noff = off + 7; return L->nbr[6 * li + 4];
    default: if (z < 7) { *noff = off + 1; return li; } *noff = off - 7; return L->nbr[6 * li + 5];
    }
}

static void level_set_defaults(olevel* L) {
    /* LaplacianApplySIMD ctor (simd_vdb_poisson.cpp:1045-1065) with
     * in_default_term = dt/(dx*dx) (:1333-1344) */
    L->t = L->dt / (L->dx * L->dx);
    L->def_face = -L->t;
    L->def_diag = 6.f * L->t;
    L->def_invdiag = 1.0f / (6.f * L->t);
    L->def_spai0 = 1.0f / (7.f * L->t);
    L->w_sor = 1.2f;
}

/* sort leaves in tree order, build lookup, neighbour table and DOF bases */
static void level_finalize_topology(olevel* L) {
    leafmap_init(&L->map, L->nl, L->org);
    L->nbr = (int32_t*)xcalloc((size_t)L->nl * 6, sizeof(int32_t));
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        for (int d = 0; d < 6; ++d) {
            int c = d >> 1, s = (d & 1) ? 8 : -8;
            int32_t p[3] = {o[0], o[1], o[2]};
            p[c] += s;
            L->nbr[6 * i + d] = leafmap_find(&L->map, p[0], p[1], p[2]);
        }
    }
    /* setDofIndex (simd_vdb_poisson.cpp:637-671) */
    L->dof_base = (int32_t*)xcalloc((size_t)L->nl, sizeof(int32_t));
    int acc = 0;
    for (int i = 0; i < L->nl; ++i) {
        L->dof_base[i] = acc;
        for (int w = 0; w < 8; ++w) acc += __builtin_popcountll(L->mask[8 * i + w]);
    }
    L->ndof = acc;
}

/* LaplacianWithLevel::trimDefaultNodes(grid, default, eps) (simd_vdb_poisson.cpp:1772-1811):
 * a leaf whose active values are all within eps of the default is replaced by
 * the default.  Returns 1 if trimmed. */
static int trim_leaf(const uint64_t* mask, float* v, float def, float eps) {
    eps = fabsf(eps);
    float maxerr = 0.f;
    for (int off = 0; off < LSZ; ++off) {
        if (!mbit(mask, off)) continue;
        float e = fabsf(v[off] - def);
        if (e > maxerr) maxerr = e;
    }
    if (maxerr <= eps) {
        for (int off = 0; off < LSZ; ++off) v[off] = def;
        return 1;
    }
    return 0;
}

/* LaplacianWithLevel::trimDefaultNodes() (:1756-1770) + initInvDiagonal (:1081-1111) */
static void level_trim_and_invdiag(olevel* L) {
    float term = -L->dt / (L->dx * L->dx);
    float diagonalTerm = -6.0f * term;
    float epsilon = 1e-5f;
    L->flags = (uint8_t*)xcalloc((size_t)L->nl, 1);
    L->invdiag = (float*)xcalloc((size_t)L->nl * LSZ, sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        const uint64_t* m = L->mask + 8 * i;
        uint8_t f = 0;
        f |= trim_leaf(m, L->diag + (size_t)i * LSZ, diagonalTerm, diagonalTerm * epsilon) ? 1 : 0;
        f |= trim_leaf(m, L->cx + (size_t)i * LSZ, term, term * epsilon) ? 2 : 0;
        f |= trim_leaf(m, L->cy + (size_t)i * LSZ, term, term * epsilon) ? 4 : 0;
        f |= trim_leaf(m, L->cz + (size_t)i * LSZ, term, term * epsilon) ? 8 : 0;
        L->flags[i] = f;
        float* inv = L->invdiag + (size_t)i * LSZ;
        const float* d = L->diag + (size_t)i * LSZ;
        for (int off = 0; off < LSZ; ++off) {
            if (f & 1) { inv[off] = L->def_invdiag; continue; }
            if (!mbit(m, off)) { inv[off] = 1.0f / L->def_diag; continue; }
            inv[off] = (d[off] == 0.f) ? 0.f : 1.0f / d[off];
        }
    }
}

static void level_alloc_scratch(olevel* L) {
    L->lhs = (float*)xcalloc((size_t)L->nl * LSZ, sizeof(float));
    L->rhs = (float*)xcalloc((size_t)L->nl * LSZ, sizeof(float));
    L->tmp = (float*)xcalloc((size_t)L->nl * LSZ, sizeof(float));
}

static inline float fraction_inside1(float l, float r) {
    /* levelset_util.cpp:4-13 */
    if (l < 0 && r < 0) return 1;
    if (l < 0 && r >= 0) return l / (l - r);
    if (l >= 0 && r < 0) return r / (r - l);
    return 0;
}
float orc_fraction_inside2(float l, float r) { return fraction_inside1(l, r); }

/* ------------------------------------------------------------------------ */
/* Level 0: BuildFinestMatrix (simd_vdb_poisson.cpp:474-597) + initializeFinest (:600-635) */
static void build_finest(orc_poisson* h, const ogrid* phi, const ogrid* fw, float dt, float dx) {
    olevel* L = &h->lv[0];
    memset(L, 0, sizeof(*L));
    L->dt = dt; L->dx = dx;
    level_set_defaults(L);
    int64_t n = phi->n;
    float* diag = (float*)xcalloc((size_t)n * LSZ, sizeof(float));
    float* cx = (float*)xcalloc((size_t)n * LSZ, sizeof(float));
    float* cy = (float*)xcalloc((size_t)n * LSZ, sizeof(float));
    float* cz = (float*)xcalloc((size_t)n * LSZ, sizeof(float));
    uint64_t* mask = (uint64_t*)xcalloc((size_t)n * 8, sizeof(uint64_t));
    float dtOverDxSqr = dt / (dx * dx);
    float term6 = 6 * dtOverDxSqr;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t li = 0; li < n; ++li) {
        const int32_t* o = phi->org + 3 * li;
        for (int off = 0; off < LSZ; ++off) {
            diag[li * LSZ + off] = term6;
            cx[li * LSZ + off] = -dtOverDxSqr;
            cy[li * LSZ + off] = -dtOverDxSqr;
            cz[li * LSZ + off] = -dtOverDxSqr;
            if (phi->mask && !mbit(phi->mask + 8 * li, off)) continue;
            float phic = phi->val[li * LSZ + off];
            if (!(phic < 0.f)) continue;
            int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            float dg = 0.f, xyz[3] = {0.f, 0.f, 0.f};
            for (int f = 0; f < 6; ++f) {
                int comp = f / 2, pos = (f % 2 == 0);
                int wc[3] = {g[0], g[1], g[2]}, pc[3] = {g[0], g[1], g[2]};
                float weight, phiOther;
                if (pos) {
                    wc[comp]++;
                    weight = ogrid_get(fw, wc[0], wc[1], wc[2], comp);
                    pc[comp]++;
                    phiOther = ogrid_get(phi, pc[0], pc[1], pc[2], 0);
                } else {
                    weight = ogrid_get(fw, wc[0], wc[1], wc[2], comp);
                    pc[comp]--;
                    phiOther = ogrid_get(phi, pc[0], pc[1], pc[2], 0);
                }
                float term = weight * dtOverDxSqr;
                if (phiOther < 0) {
                    dg += term;
                    if (!pos) xyz[comp] = -term;
                } else {
                    float theta = fraction_inside1(phic, phiOther);
                    if (theta < 0.02f) theta = 0.02f;
                    dg += term / theta;
                }
            }
            if (dg != 0.f) {
                diag[li * LSZ + off] = dg;
                cx[li * LSZ + off] = xyz[0];
                cy[li * LSZ + off] = xyz[1];
                cz[li * LSZ + off] = xyz[2];
                mask[li * 8 + (off >> 6)] |= (1ull << (off & 63));
            }
        }
    }
    /* keep non-empty leaves in tree order */
    leafkey* keys = (leafkey*)xcalloc((size_t)n, sizeof(leafkey));
    int nk = 0;
    for (int64_t li = 0; li < n; ++li) {
        uint64_t any = 0;
        for (int w = 0; w < 8; ++w) any |= mask[li * 8 + w];
        if (any) make_key(&keys[nk++], phi->org + 3 * li, (int32_t)li);
    }
    qsort(keys, (size_t)nk, sizeof(leafkey), cmp_key);
    L->nl = nk;
    L->org = (int32_t*)xcalloc((size_t)nk * 3, sizeof(int32_t));
    L->mask = (uint64_t*)xcalloc((size_t)nk * 8, sizeof(uint64_t));
    L->diag = (float*)xcalloc((size_t)nk * LSZ, sizeof(float));
    L->cx = (float*)xcalloc((size_t)nk * LSZ, sizeof(float));
    L->cy = (float*)xcalloc((size_t)nk * LSZ, sizeof(float));
    L->cz = (float*)xcalloc((size_t)nk * LSZ, sizeof(float));
    for (int i = 0; i < nk; ++i) {
        int32_t s = keys[i].i;
        memcpy(L->org + 3 * i, phi->org + 3 * s, 3 * sizeof(int32_t));
        memcpy(L->mask + 8 * i, mask + 8 * (int64_t)s, 8 * sizeof(uint64_t));
        memcpy(L->diag + (size_t)i * LSZ, diag + (size_t)s * LSZ, LSZ * sizeof(float));
        memcpy(L->cx + (size_t)i * LSZ, cx + (size_t)s * LSZ, LSZ * sizeof(float));
        memcpy(L->cy + (size_t)i * LSZ, cy + (size_t)s * LSZ, LSZ * sizeof(float));
        memcpy(L->cz + (size_t)i * LSZ, cz + (size_t)s * LSZ, LSZ * sizeof(float));
    }
    free(keys); free(diag); free(cx); free(cy); free(cz); free(mask);
    level_finalize_topology(L);
    level_trim_and_invdiag(L);
    level_alloc_scratch(L);
}

/* ------------------------------------------------------------------------ */
/* Coarse level: initializeFromFineLevel (simd_vdb_poisson.cpp:255-471) and
 * TouchCoarseLeafReducer (SIMD_UAAMG_Ops.h:4-38). */
static void build_coarse(orc_poisson* h, int lvl) {
    const olevel* F = &h->lv[lvl - 1];
    olevel* C = &h->lv[lvl];
    memset(C, 0, sizeof(*C));
    C->dt = F->dt;
    C->dx = 2.0f * F->dx;
    level_set_defaults(C);
    /* coarse leaf origins: leaf containing fine_origin/2 */
    leafkey* keys = (leafkey*)xcalloc((size_t)F->nl, sizeof(leafkey));
    int32_t* corg = (int32_t*)xcalloc((size_t)F->nl * 3, sizeof(int32_t));
    for (int i = 0; i < F->nl; ++i) {
        for (int c = 0; c < 3; ++c) corg[3 * i + c] = (F->org[3 * i + c] / 2) & ~7;
        make_key(&keys[i], corg + 3 * i, i);
    }
    qsort(keys, (size_t)F->nl, sizeof(leafkey), cmp_key);
    int nu = 0;
    int32_t* uorg = (int32_t*)xcalloc((size_t)F->nl * 3, sizeof(int32_t));
    for (int i = 0; i < F->nl; ++i) {
        if (i > 0 && cmp_key(&keys[i], &keys[i - 1]) == 0) continue;
        memcpy(uorg + 3 * nu, corg + 3 * keys[i].i, 3 * sizeof(int32_t));
        nu++;
    }
    free(keys); free(corg);
    C->nl = nu;
    C->org = uorg;
    C->mask = (uint64_t*)xcalloc((size_t)nu * 8, sizeof(uint64_t));
    C->child = (int32_t*)xcalloc((size_t)nu * 8, sizeof(int32_t));
    for (int i = 0; i < nu; ++i)
        for (int a = 0; a < 8; ++a) {
            int32_t fo[3] = {2 * uorg[3 * i] + ((a >> 2) & 1) * 8, 2 * uorg[3 * i + 1] + ((a >> 1) & 1) * 8,
                             2 * uorg[3 * i + 2] + (a & 1) * 8};
            C->child[8 * i + a] = leafmap_find(&F->map, fo[0], fo[1], fo[2]);
        }
    /* coarse DOF mask: any of the 8 fine voxels is a DOF */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nu; ++i) {
        for (int off = 0; off < LSZ; ++off) {
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            int a = ((x >= 4) << 2) | ((y >= 4) << 1) | (z >= 4);
            int32_t fl = C->child[8 * i + a];
            if (fl < 0) continue;
            int on = 0;
            for (int ii = 0; ii < 2 && !on; ++ii)
                for (int jj = 0; jj < 2 && !on; ++jj)
                    for (int kk = 0; kk < 2 && !on; ++kk) {
                        int fo = voff(2 * x + ii, 2 * y + jj, 2 * z + kk);
                        if (mbit(F->mask + 8 * fl, fo)) on = 1;
                    }
            if (on) C->mask[8 * i + (off >> 6)] |= 1ull << (off & 63);
        }
    }
    /* drop empty leaves (they carry no DOF) */
    int w = 0;
    for (int i = 0; i < nu; ++i) {
        uint64_t any = 0;
        for (int k = 0; k < 8; ++k) any |= C->mask[8 * i + k];
        if (!any) continue;
        if (w != i) {
            memcpy(C->org + 3 * w, C->org + 3 * i, 3 * sizeof(int32_t));
            memcpy(C->mask + 8 * w, C->mask + 8 * i, 8 * sizeof(uint64_t));
            memcpy(C->child + 8 * w, C->child + 8 * i, 8 * sizeof(int32_t));
        }
        w++;
    }
    C->nl = w;
    level_finalize_topology(C);
    float dtOverDxSqr = C->dt / (C->dx * C->dx);
    C->diag = (float*)xcalloc((size_t)w * LSZ, sizeof(float));
    C->cx = (float*)xcalloc((size_t)w * LSZ, sizeof(float));
    C->cy = (float*)xcalloc((size_t)w * LSZ, sizeof(float));
    C->cz = (float*)xcalloc((size_t)w * LSZ, sizeof(float));
    const float factor = 0.5f * (1.0f / 8.0f);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < w; ++i) {
        for (int off = 0; off < LSZ; ++off) {
            size_t o = (size_t)i * LSZ + off;
            C->diag[o] = 6.0f * dtOverDxSqr;
            C->cx[o] = -dtOverDxSqr; C->cy[o] = -dtOverDxSqr; C->cz[o] = -dtOverDxSqr;
            if (!mbit(C->mask + 8 * i, off)) continue;
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            int a = ((x >= 4) << 2) | ((y >= 4) << 1) | (z >= 4);
            int32_t fl = C->child[8 * i + a];
            float dg = 0, tx = 0, ty = 0, tz = 0;
            for (int ii = 0; ii < 2; ++ii)
                for (int jj = 0; jj < 2; ++jj)
                    for (int kk = 0; kk < 2; ++kk) {
                        int fo = voff(2 * x + ii, 2 * y + jj, 2 * z + kk);
                        if (!mbit(F->mask + 8 * fl, fo)) continue;
                        size_t fi = (size_t)fl * LSZ + fo;
                        dg += F->diag[fi];
                        int no; int32_t nl;
                        nl = nbv(F, fl, fo, 0, &no);
                        if (nl >= 0 && mbit(F->mask + 8 * nl, no)) {
                            if (ii == 0) tx += F->cx[fi]; else dg += 2 * F->cx[fi];
                        }
                        nl = nbv(F, fl, fo, 2, &no);
                        if (nl >= 0 && mbit(F->mask + 8 * nl, no)) {
                            if (jj == 0) ty += F->cy[fi]; else dg += 2 * F->cy[fi];
                        }
                        nl = nbv(F, fl, fo, 4, &no);
                        if (nl >= 0 && mbit(F->mask + 8 * nl, no)) {
                            if (kk == 0) tz += F->cz[fi]; else dg += 2 * F->cz[fi];
                        }
                    }
            C->diag[o] = dg * factor;
            C->cx[o] = tx * factor;
            C->cy[o] = ty * factor;
            C->cz[o] = tz * factor;
        }
    }
    level_trim_and_invdiag(C);
    level_alloc_scratch(C);
}

/* ------------------------------------------------------------------------ */
/* init_SPAI0 (simd_vdb_poisson.cpp:1113-1190) */
static void level_init_spai0(olevel* L) {
    if (L->spai0_ready) return;
    float bg = L->def_diag; /* mDiagonal->background() */
    float defaultSPAI0Val = 6.0f / (7.f * bg);
    L->spai0 = (float*)xcalloc((size_t)L->nl * LSZ, sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        const uint64_t* m = L->mask + 8 * i;
        float* s = L->spai0 + (size_t)i * LSZ;
        for (int off = 0; off < LSZ; ++off) {
            s[off] = defaultSPAI0Val;
            if (!mbit(m, off)) continue;
            float rowNormSqr = 0;
            int no; int32_t nl; size_t me = (size_t)i * LSZ + off;
            const float* arr[3] = {L->cx, L->cy, L->cz};
            for (int c = 0; c < 3; ++c) {
                nl = nbv(L, i, off, 2 * c + 1, &no); /* + neighbour: its own minus-face entry */
                if (nl >= 0 && mbit(L->mask + 8 * nl, no)) {
                    float v = arr[c][(size_t)nl * LSZ + no];
                    rowNormSqr += v * v;
                }
                nl = nbv(L, i, off, 2 * c, &no); /* - neighbour: this voxel's minus-face entry */
                if (nl >= 0 && mbit(L->mask + 8 * nl, no)) {
                    float v = arr[c][me];
                    rowNormSqr += v * v;
                }
            }
            float d = L->diag[me];
            s[off] = (d == 0) ? 0.f : d / (d * d + rowNormSqr);
        }
        if (trim_leaf(m, s, defaultSPAI0Val, defaultSPAI0Val * 1e-5f)) {
            for (int off = 0; off < LSZ; ++off) s[off] = L->def_spai0;
            L->flags[i] |= 16;
        }
    }
    L->spai0_ready = 1;
}

/* ------------------------------------------------------------------------ */
/* LaplacianApplySIMD::LightWeightApplier::operator() (simd_vdb_poisson.cpp:755-1031)
 * in the reference's lane layout: one __m256 per (x, y) row of a leaf holds its
 * 8 z voxels; the +-x / +-y rows come from the leaf or its neighbour leaf, the
 * +-z values are the row shifted by one lane with the neighbour leaf's boundary
 * voxel blended into the end lane (vdb_SIMD_IO.h:25-191); inactive lanes are
 * written as 0.  Every lane performs the scalar path's operations in the same
 * order (products, the three pair sums, two more sums, then the mode's
 * fused multiply-adds), so both paths give the same bits. */
#include <immintrin.h>
static int g_orc_simd = 1;
void orc_set_simd(int on) { g_orc_simd = on; }

static void apply_level_avx2(olevel* L, int mode, float weight, float w_sor, const float* lhs,
                             const float* rhs, float* out) {
    const __m256i up = _mm256_setr_epi32(1, 2, 3, 4, 5, 6, 7, 7);
    const __m256i dn = _mm256_setr_epi32(0, 0, 1, 2, 3, 4, 5, 6);
    const __m256i bitsel = _mm256_setr_epi32(1, 2, 4, 8, 16, 32, 64, 128);
    const __m256 zero = _mm256_setzero_ps();
    const __m256 dface = _mm256_set1_ps(L->def_face);
    const __m256 vw = _mm256_set1_ps(weight), vsor = _mm256_set1_ps(w_sor), v1m = _mm256_set1_ps(1.0f - w_sor);
    const __m256 even = _mm256_castsi256_ps(_mm256_setr_epi32(-1, 0, -1, 0, -1, 0, -1, 0));
    const __m256 odd = _mm256_castsi256_ps(_mm256_setr_epi32(0, -1, 0, -1, 0, -1, 0, -1));
    const float* cx = L->cx;
    const float* cy = L->cy;
    const float* cz = L->cz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* nb = L->nbr + 6 * i;
        const uint64_t* m = L->mask + 8 * i;
        for (int X = 0; X < 8; ++X)
            for (int Y = 0; Y < 8; ++Y) {
                const size_t row = (size_t)i * LSZ + (size_t)X * 64 + (size_t)Y * 8;
                const unsigned bits = (unsigned)((m[X] >> (Y * 8)) & 0xFFu);
                if (!bits) { _mm256_storeu_ps(out + row, zero); continue; }
                const __m256 xc = _mm256_loadu_ps(lhs + row);
                __m256 xp, cxp, xm, yp, cyp, ym;
                if (X < 7) { xp = _mm256_loadu_ps(lhs + row + 64); cxp = _mm256_loadu_ps(cx + row + 64); }
                else if (nb[1] >= 0) {
                    const size_t r = (size_t)nb[1] * LSZ + (size_t)Y * 8;
                    xp = _mm256_loadu_ps(lhs + r); cxp = _mm256_loadu_ps(cx + r);
                } else { xp = zero; cxp = dface; }
                if (X > 0) xm = _mm256_loadu_ps(lhs + row - 64);
                else xm = nb[0] >= 0 ? _mm256_loadu_ps(lhs + (size_t)nb[0] * LSZ + 448 + (size_t)Y * 8) : zero;
                if (Y < 7) { yp = _mm256_loadu_ps(lhs + row + 8); cyp = _mm256_loadu_ps(cy + row + 8); }
                else if (nb[3] >= 0) {
                    const size_t r = (size_t)nb[3] * LSZ + (size_t)X * 64;
                    yp = _mm256_loadu_ps(lhs + r); cyp = _mm256_loadu_ps(cy + r);
                } else { yp = zero; cyp = dface; }
                if (Y > 0) ym = _mm256_loadu_ps(lhs + row - 8);
                else ym = nb[2] >= 0 ? _mm256_loadu_ps(lhs + (size_t)nb[2] * LSZ + (size_t)X * 64 + 56) : zero;
                float zp7 = 0.f, czp7 = L->def_face, zm0 = 0.f;
                if (nb[5] >= 0) {
                    const size_t r = (size_t)nb[5] * LSZ + (size_t)X * 64 + (size_t)Y * 8;
                    zp7 = lhs[r];
                    czp7 = cz[r];
                }
                if (nb[4] >= 0) zm0 = lhs[(size_t)nb[4] * LSZ + (size_t)X * 64 + (size_t)Y * 8 + 7];
                const __m256 czo = _mm256_loadu_ps(cz + row);
                const __m256 zp = _mm256_blend_ps(_mm256_permutevar8x32_ps(xc, up), _mm256_set1_ps(zp7), 0x80);
                const __m256 czp = _mm256_blend_ps(_mm256_permutevar8x32_ps(czo, up), _mm256_set1_ps(czp7), 0x80);
                const __m256 zm = _mm256_blend_ps(_mm256_permutevar8x32_ps(xc, dn), _mm256_set1_ps(zm0), 0x01);
                __m256 f1 = _mm256_mul_ps(xp, cxp), f2 = _mm256_mul_ps(xm, _mm256_loadu_ps(cx + row));
                __m256 f3 = _mm256_mul_ps(yp, cyp), f4 = _mm256_mul_ps(ym, _mm256_loadu_ps(cy + row));
                __m256 f5 = _mm256_mul_ps(zp, czp), f6 = _mm256_mul_ps(zm, czo);
                f1 = _mm256_add_ps(f1, f2);
                f3 = _mm256_add_ps(f3, f4);
                f5 = _mm256_add_ps(f5, f6);
                f1 = _mm256_add_ps(f1, f3);
                f1 = _mm256_add_ps(f1, f5);
                __m256 r;
                switch (mode) {
                case ORC_MODE_JACOBI: {
                    __m256 res = _mm256_sub_ps(_mm256_loadu_ps(rhs + row),
                                               _mm256_fmadd_ps(xc, _mm256_loadu_ps(L->diag + row), f1));
                    res = _mm256_mul_ps(res, _mm256_loadu_ps(L->invdiag + row));
                    r = _mm256_fmadd_ps(vw, res, xc);
                    break;
                }
                case ORC_MODE_RESIDUAL:
                    r = _mm256_sub_ps(_mm256_loadu_ps(rhs + row), _mm256_fmadd_ps(xc, _mm256_loadu_ps(L->diag + row), f1));
                    break;
                case ORC_MODE_RED_GS:
                case ORC_MODE_BLACK_GS: {
                    __m256 res = _mm256_sub_ps(_mm256_loadu_ps(rhs + row), f1);
                    res = _mm256_mul_ps(res, _mm256_loadu_ps(L->invdiag + row));
                    res = _mm256_mul_ps(res, vsor);
                    const __m256 v = _mm256_fmadd_ps(xc, v1m, res);
                    /* red: (x + y + z) even */
                    const int xy_even = ((X + Y) & 1) == 0;
                    const __m256 red = xy_even ? even : odd;
                    const __m256 upd = mode == ORC_MODE_RED_GS ? red : (xy_even ? odd : even);
                    r = _mm256_blendv_ps(xc, v, upd);
                    break;
                }
                case ORC_MODE_SPAI0: {
                    const __m256 res = _mm256_sub_ps(_mm256_loadu_ps(rhs + row),
                                                     _mm256_fmadd_ps(xc, _mm256_loadu_ps(L->diag + row), f1));
                    r = _mm256_fmadd_ps(_mm256_loadu_ps(L->spai0 + row), res, xc);
                    break;
                }
                default:
                    r = _mm256_fmadd_ps(xc, _mm256_loadu_ps(L->diag + row), f1);
                    break;
                }
                const __m256 act = _mm256_castsi256_ps(
                    _mm256_cmpeq_epi32(_mm256_and_si256(_mm256_set1_epi32((int)bits), bitsel), bitsel));
                _mm256_storeu_ps(out + row, _mm256_blendv_ps(zero, r, act));
            }
    }
}

static void apply_level(olevel* L, int mode, float weight, float w_sor, const float* lhs,
                        const float* rhs, float* out) {
    if (mode == ORC_MODE_SPAI0) level_init_spai0(L);
    if (g_orc_simd) {
        apply_level_avx2(L, mode, weight, w_sor, lhs, rhs, out);
        return;
    }
    const float one_minus_sor = 1.0f - w_sor;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        const uint64_t* m = L->mask + 8 * i;
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            if (!mbit(m, off)) { out[me] = 0.f; continue; }
            int no; int32_t nl;
            float xp, xm, yp, ym, zp, zm, cxp, cyp, czp;
            nl = nbv(L, i, off, 1, &no);
            xp = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            cxp = nl >= 0 ? L->cx[(size_t)nl * LSZ + no] : L->def_face;
            nl = nbv(L, i, off, 0, &no);
            xm = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            nl = nbv(L, i, off, 3, &no);
            yp = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            cyp = nl >= 0 ? L->cy[(size_t)nl * LSZ + no] : L->def_face;
            nl = nbv(L, i, off, 2, &no);
            ym = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            nl = nbv(L, i, off, 5, &no);
            zp = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            czp = nl >= 0 ? L->cz[(size_t)nl * LSZ + no] : L->def_face;
            nl = nbv(L, i, off, 4, &no);
            zm = nl >= 0 ? lhs[(size_t)nl * LSZ + no] : 0.f;
            float f1 = xp * cxp, f2 = xm * L->cx[me];
            float f3 = yp * cyp, f4 = ym * L->cy[me];
            float f5 = zp * czp, f6 = zm * L->cz[me];
            f1 = f1 + f2; f3 = f3 + f4; f5 = f5 + f6;
            f1 = f1 + f3; f1 = f1 + f5;
            float x = lhs[me], res;
            switch (mode) {
            case ORC_MODE_JACOBI:
                res = rhs[me] - fmaf(x, L->diag[me], f1);
                res = res * L->invdiag[me];
                out[me] = fmaf(weight, res, x);
                break;
            case ORC_MODE_RESIDUAL:
                out[me] = rhs[me] - fmaf(x, L->diag[me], f1);
                break;
            case ORC_MODE_RED_GS:
            case ORC_MODE_BLACK_GS: {
                int red = (((off >> 6) + (off >> 3) + off) & 1) == 0;
                int upd = (mode == ORC_MODE_RED_GS) ? red : !red;
                if (upd) {
                    res = rhs[me] - f1;
                    res = res * L->invdiag[me];
                    res = res * w_sor;
                    out[me] = fmaf(x, one_minus_sor, res);
                } else {
                    out[me] = x;
                }
                break;
            }
            case ORC_MODE_SPAI0:
                res = rhs[me] - fmaf(x, L->diag[me], f1);
                out[me] = fmaf(L->spai0[me], res, x);
                break;
            default: /* Laplacian */
                out[me] = fmaf(x, L->diag[me], f1);
                break;
            }
        }
    }
}

/* 8 activity bits of a row as a lane mask */
static inline __m256 row_mask(unsigned bits) {
    const __m256i bitsel = _mm256_setr_epi32(1, 2, 4, 8, 16, 32, 64, 128);
    return _mm256_castsi256_ps(_mm256_cmpeq_epi32(_mm256_and_si256(_mm256_set1_epi32((int)bits), bitsel), bitsel));
}

/* setGridToResultAfterFirstJacobi (:1435-1479): AVX lanes as in the reference
 * (:1472-1473), or the scalar loop */
static void first_jacobi(olevel* L, float weight, const float* rhs, float* out) {
    if (g_orc_simd) {
        const __m256 w = _mm256_set1_ps(weight), zero = _mm256_setzero_ps();
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L->nl; ++i)
            for (int xy = 0; xy < 64; ++xy) {
                const size_t row = (size_t)i * LSZ + (size_t)xy * 8;
                const unsigned bits = (unsigned)((L->mask[8 * i + (xy >> 3)] >> ((xy & 7) * 8)) & 0xFFu);
                __m256 r = _mm256_mul_ps(_mm256_loadu_ps(L->invdiag + row), _mm256_loadu_ps(rhs + row));
                r = _mm256_mul_ps(w, r);
                _mm256_storeu_ps(out + row, _mm256_blendv_ps(zero, r, row_mask(bits)));
            }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            if (!mbit(L->mask + 8 * i, off)) { out[me] = 0.f; continue; }
            float r = L->invdiag[me] * rhs[me];
            out[me] = weight * r;
        }
}
/* setGridToResultAfterFirstSPAI0 (:1481-1517).  It reads mSPAI0 without
 * calling init_SPAI0, so before the level's first spai0Apply the SPAI0 grid has
 * no leaves and every voxel uses the default 1/(7 dt/dx^2). */
static void first_spai0(olevel* L, const float* rhs, float* out) {
    const int ready = L->spai0_ready;
    if (g_orc_simd) {
        const __m256 zero = _mm256_setzero_ps(), def = _mm256_set1_ps(L->def_spai0);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L->nl; ++i)
            for (int xy = 0; xy < 64; ++xy) {
                const size_t row = (size_t)i * LSZ + (size_t)xy * 8;
                const unsigned bits = (unsigned)((L->mask[8 * i + (xy >> 3)] >> ((xy & 7) * 8)) & 0xFFu);
                const __m256 sp = ready ? _mm256_loadu_ps(L->spai0 + row) : def;
                const __m256 r = _mm256_mul_ps(sp, _mm256_loadu_ps(rhs + row));
                _mm256_storeu_ps(out + row, _mm256_blendv_ps(zero, r, row_mask(bits)));
            }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            float s = ready ? L->spai0[me] : L->def_spai0;
            out[me] = mbit(L->mask + 8 * i, off) ? s * rhs[me] : 0.f;
        }
}
/* setGridToResultAfterFirstRBGS<redFirst> (:1519-1582) */
static void first_rbgs(olevel* L, int red_first, float w_sor, const float* rhs, float* out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            int red = (((off >> 6) + (off >> 3) + off) & 1) == 0;
            int upd = red_first ? red : !red;
            if (!mbit(L->mask + 8 * i, off) || !upd) { out[me] = 0.f; continue; }
            float r = L->invdiag[me] * rhs[me];
            out[me] = w_sor * r;
        }
    apply_level(L, red_first ? ORC_MODE_BLACK_GS : ORC_MODE_RED_GS, 0.f, w_sor, out, rhs, out);
}

/* restriction (:1624-1684): coarse = 1/8 * sum of the active fine values */
static void restrict_level(const orc_poisson* h, int fl, const float* fine, float* coarse) {
    const olevel* F = &h->lv[fl];
    const olevel* C = &h->lv[fl + 1];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            if (!mbit(C->mask + 8 * i, off)) { coarse[me] = 0.f; continue; }
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            int a = ((x >= 4) << 2) | ((y >= 4) << 1) | (z >= 4);
            int32_t f = C->child[8 * i + a];
            float s = 0;
            for (int ii = 0; ii < 2; ++ii)
                for (int jj = 0; jj < 2; ++jj)
                    for (int kk = 0; kk < 2; ++kk) {
                        int fo = voff(2 * x + ii, 2 * y + jj, 2 * z + kk);
                        if (mbit(F->mask + 8 * f, fo)) s += fine[(size_t)f * LSZ + fo];
                    }
            coarse[me] = s * 0.125f;
        }
}

/* prolongation<inplace_add=true> (:1686-1754): fine += alpha * coarse */
static void prolongate_level(const orc_poisson* h, int fl, const float* coarse, float* fine,
                             float alpha) {
    const olevel* F = &h->lv[fl];
    const olevel* C = &h->lv[fl + 1];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            if (!mbit(C->mask + 8 * i, off)) continue;
            int x = off >> 6, y = (off >> 3) & 7, z = off & 7;
            int a = ((x >= 4) << 2) | ((y >= 4) << 1) | (z >= 4);
            int32_t f = C->child[8 * i + a];
            if (f < 0) continue;
            float cv = alpha * coarse[(size_t)i * LSZ + off];
            for (int ii = 0; ii < 2; ++ii)
                for (int jj = 0; jj < 2; ++jj)
                    for (int kk = 0; kk < 2; ++kk) {
                        int fo = voff(2 * x + ii, 2 * y + jj, 2 * z + kk);
                        if (mbit(F->mask + 8 * f, fo)) fine[(size_t)f * LSZ + fo] += cv;
                    }
        }
}

/* ------------------------------------------------------------------------ */
/* coarsest level: explicit matrix (getTriplets :129-206) and a restatement of
 * Eigen::ConjugateGradient<SparseMatrix<float>> with DiagonalPreconditioner,
 * tolerance NumTraits<float>::epsilon(), maxIterations 10, zero initial guess
 * (constructCoarsestLevelExactSolver :2114-2126). */
static void build_coarsest(orc_poisson* h) {
    const olevel* L = &h->lv[h->nlev - 1];
    int n = L->ndof;
    h->c_n = n;
    h->c_rowptr = (int32_t*)xcalloc((size_t)n + 1, sizeof(int32_t));
    h->c_col = (int32_t*)xcalloc((size_t)n * 7, sizeof(int32_t));
    h->c_val = (float*)xcalloc((size_t)n * 7, sizeof(float));
    h->c_invdiag = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_dof_leaf = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
    h->c_dof_off = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
    int nnz = 0, row = 0;
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            if (!mbit(L->mask + 8 * i, off)) continue;
            size_t me = (size_t)i * LSZ + off;
            h->c_rowptr[row] = nnz;
            h->c_dof_leaf[row] = i; h->c_dof_off[row] = off;
            h->c_col[nnz] = row; h->c_val[nnz] = L->diag[me]; nnz++;
            const float* arr[3] = {L->cx, L->cy, L->cz};
            for (int c = 0; c < 3; ++c) {
                int no; int32_t nl = nbv(L, i, off, 2 * c, &no);
                if (nl >= 0 && mbit(L->mask + 8 * nl, no)) {
                    int d = L->dof_base[nl];
                    for (int q = 0; q < no; ++q) d += mbit(L->mask + 8 * nl, q);
                    h->c_col[nnz] = d; h->c_val[nnz] = arr[c][me]; nnz++;
                }
                nl = nbv(L, i, off, 2 * c + 1, &no);
                if (nl >= 0 && mbit(L->mask + 8 * nl, no)) {
                    int d = L->dof_base[nl];
                    for (int q = 0; q < no; ++q) d += mbit(L->mask + 8 * nl, q);
                    h->c_col[nnz] = d; h->c_val[nnz] = arr[c][(size_t)nl * LSZ + no]; nnz++;
                }
            }
            float dg = L->diag[me];
            h->c_invdiag[row] = (dg != 0.f) ? 1.0f / dg : 1.0f;
            row++;
        }
    h->c_rowptr[n] = nnz;
    h->c_b = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_x = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_r = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_p = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_z = (float*)xcalloc((size_t)n, sizeof(float));
    h->c_t = (float*)xcalloc((size_t)n, sizeof(float));
}

static void csr_mv(const orc_poisson* h, const float* x, float* y) {
    for (int i = 0; i < h->c_n; ++i) {
        float s = 0;
        for (int k = h->c_rowptr[i]; k < h->c_rowptr[i + 1]; ++k) s += h->c_val[k] * x[h->c_col[k]];
        y[i] = s;
    }
}
static float vdot(int n, const float* a, const float* b) {
    float s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static void coarsest_cg(orc_poisson* h) {
    int n = h->c_n;
    float *x = h->c_x, *b = h->c_b, *r = h->c_r, *p = h->c_p, *z = h->c_z, *t = h->c_t;
    const float tol = FLT_EPSILON;
    const int maxIters = 10;
    for (int i = 0; i < n; ++i) { x[i] = 0.f; r[i] = b[i]; }
    float rhsNorm2 = vdot(n, b, b);
    if (rhsNorm2 == 0.f) return;
    float threshold = tol * tol * rhsNorm2;
    if (threshold < FLT_MIN) threshold = FLT_MIN;
    float residualNorm2 = vdot(n, r, r);
    if (residualNorm2 < threshold) return;
    for (int i = 0; i < n; ++i) p[i] = h->c_invdiag[i] * r[i];
    float absNew = vdot(n, r, p);
    int it = 0;
    while (it < maxIters) {
        csr_mv(h, p, t);
        float alpha = absNew / vdot(n, p, t);
        for (int i = 0; i < n; ++i) x[i] += alpha * p[i];
        for (int i = 0; i < n; ++i) r[i] -= alpha * t[i];
        residualNorm2 = vdot(n, r, r);
        if (residualNorm2 < threshold) break;
        for (int i = 0; i < n; ++i) z[i] = h->c_invdiag[i] * r[i];
        float absOld = absNew;
        absNew = vdot(n, r, z);
        float beta = absNew / absOld;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        it++;
    }
}

static void coarsest_solve(orc_poisson* h, const float* rhs, float* out) {
    for (int i = 0; i < h->c_n; ++i) h->c_b[i] = rhs[(size_t)h->c_dof_leaf[i] * LSZ + h->c_dof_off[i]];
    coarsest_cg(h);
    for (int i = 0; i < h->c_n; ++i) out[(size_t)h->c_dof_leaf[i] * LSZ + h->c_dof_off[i]] = h->c_x[i];
}

/* ------------------------------------------------------------------------ */
/* muCyclePreconditioner<mu=2, skip_first> (simd_vdb_poisson.cpp:1844-1977) */
static float sched_weight_precond(int n, int it) {
    if (it >= n) return 6.0f / 7.0f;
    if (n == 1) return 6.0f / 7.0f;
    if (n == 2) { const float w[2] = {1.7319f, 0.5695f}; return w[it]; }
    const float w[3] = {2.2473f, 0.8571f, 0.5296f};
    return w[it];
}
/* muCycleIterative (:1979-2110) */
static float sched_weight_iter(int n, int it) {
    if (it >= n) return 6.0f / 7.0f;
    if (n == 2) { const float w[2] = {1.7319f, 0.5695f}; return w[it]; }
    if (n >= 3) { const float w[3] = {2.2473f, 0.8571f, 0.5296f}; return w[it]; }
    return 6.0f / 7.0f;
}

typedef struct { float* cur; float* other; } pp; /* ping-pong pair (lhs slot, temp slot) */

static void smooth_step(olevel* L, int smoother, float w, int red_first, pp* s, const float* rhs) {
    switch (smoother) {
    case ORC_SMOOTH_RBGS:
        apply_level(L, red_first ? ORC_MODE_RED_GS : ORC_MODE_BLACK_GS, 0, L->w_sor, s->cur, rhs, s->cur);
        apply_level(L, red_first ? ORC_MODE_BLACK_GS : ORC_MODE_RED_GS, 0, L->w_sor, s->cur, rhs, s->cur);
        break;
    case ORC_SMOOTH_SPAI0:
        apply_level(L, ORC_MODE_SPAI0, 0, L->w_sor, s->cur, rhs, s->other);
        { float* t = s->cur; s->cur = s->other; s->other = t; }
        break;
    default:
        apply_level(L, ORC_MODE_JACOBI, w, L->w_sor, s->cur, rhs, s->other);
        { float* t = s->cur; s->cur = s->other; s->other = t; }
        break;
    }
}

static void mucycle_precond(orc_poisson* h, int smoother, float* lhs, const float* rhs, int level,
                            int skip_first, int n) {
    olevel* L = &h->lv[level];
    if (level == h->nlev - 1) {
        coarsest_solve(h, rhs, lhs);
        return;
    }
    pp s = {lhs, L->tmp};
    if (skip_first) {
        switch (smoother) {
        case ORC_SMOOTH_WEIGHTED_JACOBI:
            first_jacobi(L, 6.0f / 7.0f, rhs, s.other);
            { float* t = s.cur; s.cur = s.other; s.other = t; }
            break;
        case ORC_SMOOTH_RBGS:
            first_rbgs(L, 1, L->w_sor, rhs, s.cur);
            break;
        case ORC_SMOOTH_SPAI0:
            first_spai0(L, rhs, s.other);
            { float* t = s.cur; s.cur = s.other; s.other = t; }
            break;
        default:
            first_jacobi(L, sched_weight_precond(n, 0), rhs, s.other);
            { float* t = s.cur; s.cur = s.other; s.other = t; }
            break;
        }
    }
    for (int i = skip_first ? 1 : 0; i < n; ++i) {
        float w = (smoother == ORC_SMOOTH_WEIGHTED_JACOBI) ? 6.0f / 7.0f : sched_weight_precond(n, i);
        smooth_step(L, smoother, w, 1, &s, rhs);
    }
    apply_level(L, ORC_MODE_RESIDUAL, 0, L->w_sor, s.cur, rhs, s.other);
    olevel* P = &h->lv[level + 1];
    restrict_level(h, level, s.other, P->rhs);
    mucycle_precond(h, smoother, P->lhs, P->rhs, level + 1, 1, n);
    /* the second visit of the coarsest level solves the same system again */
    mucycle_precond(h, smoother, P->lhs, P->rhs, level + 1, 0, n);
    prolongate_level(h, level, P->lhs, s.cur, 1.0f);
    for (int i = 0; i < n; ++i) {
        float w = (smoother == ORC_SMOOTH_WEIGHTED_JACOBI) ? 6.0f / 7.0f : sched_weight_precond(n, n - 1 - i);
        smooth_step(L, smoother, w, 0, &s, rhs);
    }
    if (s.cur != lhs) memcpy(lhs, s.cur, sizeof(float) * (size_t)L->nl * LSZ);
}

static void mucycle_iter(orc_poisson* h, int smoother, float* lhs, const float* rhs, int level, int n) {
    olevel* L = &h->lv[level];
    if (level == h->nlev - 1) {
        pp s = {lhs, L->tmp};
        int large = 10 * n;
        for (int i = 0; i < large; ++i) {
            float w = (smoother == ORC_SMOOTH_WEIGHTED_JACOBI) ? 6.0f / 7.0f : sched_weight_iter(n, i);
            if (smoother == ORC_SMOOTH_RBGS) L->w_sor = 1.0f;
            smooth_step(L, smoother, w, 1, &s, rhs);
        }
        if (s.cur != lhs) memcpy(lhs, s.cur, sizeof(float) * (size_t)L->nl * LSZ);
        return;
    }
    pp s = {lhs, L->tmp};
    for (int i = 0; i < n; ++i) {
        float w = (smoother == ORC_SMOOTH_WEIGHTED_JACOBI) ? 6.0f / 7.0f : sched_weight_iter(n, i);
        if (smoother == ORC_SMOOTH_RBGS) L->w_sor = 1.0f;
        smooth_step(L, smoother, w, 1, &s, rhs);
    }
    apply_level(L, ORC_MODE_RESIDUAL, 0, L->w_sor, s.cur, rhs, s.other);
    olevel* P = &h->lv[level + 1];
    restrict_level(h, level, s.other, P->rhs);
    for (int mu = 0; mu < 2; ++mu) mucycle_iter(h, smoother, P->lhs, P->rhs, level + 1, n);
    prolongate_level(h, level, P->lhs, s.cur, 0.5f);
    for (int i = 0; i < n; ++i) {
        float w = (smoother == ORC_SMOOTH_WEIGHTED_JACOBI) ? 6.0f / 7.0f : sched_weight_iter(n, n - 1 - i);
        if (smoother == ORC_SMOOTH_RBGS) L->w_sor = 1.0f;
        smooth_step(L, smoother, w, 0, &s, rhs);
    }
    if (s.cur != lhs) memcpy(lhs, s.cur, sizeof(float) * (size_t)L->nl * LSZ);
}

/* ------------------------------------------------------------------------ */
/* BLAS-1 (simd_vdb_poisson.cpp:2270-2320, openvdb_grid_math_op.h:4-74) */
float orc_abs_max(const orc_poisson* h, int level, const float* v) {
    const olevel* L = &h->lv[level];
    float* part = (float*)xcalloc((size_t)L->nl + 1, sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        float m = 0;
        for (int off = 0; off < LSZ; ++off) {
            if (!mbit(L->mask + 8 * i, off)) continue;
            float x = v[(size_t)i * LSZ + off];
            if (!isfinite(x)) { m = x; break; }
            float a = fabsf(x);
            if (a > m) m = a;
        }
        part[i] = m;
    }
    float m = 0;
    for (int i = 0; i < L->nl; ++i) {
        if (!isfinite(part[i])) { m = part[i]; break; }
        if (part[i] > m) m = part[i];
    }
    free(part);
    return m;
}

float orc_dot(const orc_poisson* h, int level, const float* a, const float* b) {
    const olevel* L = &h->lv[level];
    float* part = (float*)xcalloc((size_t)L->nl + 1, sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        float s = 0;
        for (int off = 0; off < LSZ; ++off) {
            if (!mbit(L->mask + 8 * i, off)) continue;
            size_t me = (size_t)i * LSZ + off;
            float pr = a[me] * b[me];
            s = s + pr;
        }
        part[i] = s;
    }
    float s = 0;
    for (int i = 0; i < L->nl; ++i) s += part[i];
    free(part);
    return s;
}

static void axpy(const olevel* L, float alpha, const float* x, float* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off)
            if (mbit(L->mask + 8 * i, off)) {
                size_t me = (size_t)i * LSZ + off;
                y[me] = fmaf(alpha, x[me], y[me]);
            }
}
static void xpay(const olevel* L, float alpha, const float* x, float* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off)
            if (mbit(L->mask + 8 * i, off)) {
                size_t me = (size_t)i * LSZ + off;
                y[me] = fmaf(alpha, y[me], x[me]);
            }
}

/* PoissonSolver::solveMultigridPCG (simd_vdb_poisson.cpp:2155-2226) */
int orc_solve_pcg(orc_poisson* h, float* x, const float* b, float rel_tol, int max_iter,
                  int smoother, int* iterations, float* final_abs_res) {
    olevel* L = &h->lv[0];
    size_t nv = (size_t)L->nl * LSZ;
    int it = 0;
    if (L->ndof == 0) { *iterations = 0; if (final_abs_res) *final_abs_res = 0; return 0; }
    float* r = (float*)xcalloc(nv, sizeof(float));
    float* p = (float*)xcalloc(nv, sizeof(float));
    float* z = (float*)xcalloc(nv, sizeof(float));
    apply_level(L, ORC_MODE_RESIDUAL, 0, L->w_sor, x, b, r);
    float nu = orc_abs_max(h, 0, r);
    float numax = rel_tol * nu;
    int status = 1;
    if (nu <= numax) { status = 0; goto done; }
    mucycle_precond(h, smoother, p, r, 0, 1, 3);
    float rho = orc_dot(h, 0, p, r);
    float nu_old = nu;
    for (; it < max_iter; ++it) {
        apply_level(L, ORC_MODE_LAPLACIAN, 0, L->w_sor, p, NULL, z);
        float sigma = orc_dot(h, 0, p, z);
        float alpha = rho / sigma;
        axpy(L, -alpha, z, r);
        nu_old = nu;
        nu = orc_abs_max(h, 0, r);
        if (nu <= numax) { axpy(L, alpha, p, x); status = 0; goto done; }
        if (nu > nu_old && it > 3) { status = 1; goto done; }
        memset(z, 0, nv * sizeof(float));
        mucycle_precond(h, smoother, z, r, 0, 1, 3);
        float rho_new = orc_dot(h, 0, z, r);
        float beta = rho_new / rho;
        rho = rho_new;
        axpy(L, alpha, p, x);
        xpay(L, beta, z, p);
    }
    status = 1;
done:
    *iterations = it;
    if (final_abs_res) *final_abs_res = nu;
    free(r); free(p); free(z);
    return status;
}

/* PoissonSolver::solvePureMultigrid (simd_vdb_poisson.cpp:2228-2267) */
int orc_solve_mg(orc_poisson* h, float* x, const float* b, float rel_tol, int max_iter,
                 int smoother, int* iterations, float* final_abs_res) {
    olevel* L = &h->lv[0];
    size_t nv = (size_t)L->nl * LSZ;
    int it = 0, status = 1;
    if (L->ndof == 0) { *iterations = 0; if (final_abs_res) *final_abs_res = 0; return 0; }
    float* r = (float*)xcalloc(nv, sizeof(float));
    apply_level(L, ORC_MODE_RESIDUAL, 0, L->w_sor, x, b, r);
    float nu = orc_abs_max(h, 0, r);
    float numax = rel_tol * nu;
    if (nu <= numax) { status = 0; goto done; }
    float nu_old = nu;
    for (; it < max_iter; ++it) {
        mucycle_iter(h, smoother, x, b, 0, 3);
        apply_level(L, ORC_MODE_RESIDUAL, 0, L->w_sor, x, b, r);
        nu_old = nu;
        nu = orc_abs_max(h, 0, r);
        if (nu <= numax) { status = 0; goto done; }
        if (nu > nu_old && it > 8) { status = 1; goto done; }
    }
    status = 1;
done:
    *iterations = it;
    if (final_abs_res) *final_abs_res = nu;
    free(r);
    return status;
}

/* ------------------------------------------------------------------------ */
orc_poisson* orc_poisson_create(int64_t phi_n, const int32_t* phi_origins, const uint64_t* phi_masks,
                                const float* phi_values, float phi_background, int64_t fw_n,
                                const int32_t* fw_origins, const float* fw_values,
                                const float* fw_background3, float dt, float dx, int build_hierarchy) {
    orc_poisson* h = (orc_poisson*)xcalloc(1, sizeof(orc_poisson));
    ogrid phi, fw;
    float pb[3] = {phi_background, 0, 0};
    ogrid_init(&phi, phi_n, phi_origins, phi_masks, phi_values, 1, pb);
    ogrid_init(&fw, fw_n, fw_origins, NULL, fw_values, 3, fw_background3);
    build_finest(h, &phi, &fw, dt, dx);
    leafmap_free(&phi.map);
    leafmap_free(&fw.map);
    h->nlev = 1;
    if (build_hierarchy) {
        /* constructMultigridHierarchy (:1813-1842): coarsen while ndof > 4000 */
        while (h->lv[h->nlev - 1].ndof > 4000 && h->nlev < 32) {
            build_coarse(h, h->nlev);
            h->nlev++;
        }
        build_coarsest(h);
    }
    return h;
}

void orc_poisson_free(orc_poisson* h) {
    if (!h) return;
    for (int l = 0; l < h->nlev; ++l) {
        olevel* L = &h->lv[l];
        free(L->org); free(L->mask); free(L->nbr); free(L->child); free(L->dof_base);
        free(L->diag); free(L->cx); free(L->cy); free(L->cz); free(L->invdiag); free(L->spai0);
        free(L->flags); free(L->lhs); free(L->rhs); free(L->tmp);
        leafmap_free(&L->map);
    }
    free(h->c_rowptr); free(h->c_col); free(h->c_val); free(h->c_invdiag);
    free(h->c_dof_leaf); free(h->c_dof_off);
    free(h->c_b); free(h->c_x); free(h->c_r); free(h->c_p); free(h->c_z); free(h->c_t);
    free(h);
}

int orc_num_levels(const orc_poisson* h) { return h->nlev; }
int orc_level_leaf_count(const orc_poisson* h, int level) { return h->lv[level].nl; }
int orc_level_ndof(const orc_poisson* h, int level) { return h->lv[level].ndof; }
void orc_level_topology(const orc_poisson* h, int level, int32_t* origins, uint64_t* masks) {
    const olevel* L = &h->lv[level];
    if (origins) memcpy(origins, L->org, sizeof(int32_t) * 3 * (size_t)L->nl);
    if (masks) memcpy(masks, L->mask, sizeof(uint64_t) * 8 * (size_t)L->nl);
}
void orc_level_coefficients(const orc_poisson* h, int level, float* diag, float* cx, float* cy,
                            float* cz, uint8_t* flags) {
    const olevel* L = &h->lv[level];
    size_t nv = (size_t)L->nl * LSZ;
    if (diag) memcpy(diag, L->diag, nv * sizeof(float));
    if (cx) memcpy(cx, L->cx, nv * sizeof(float));
    if (cy) memcpy(cy, L->cy, nv * sizeof(float));
    if (cz) memcpy(cz, L->cz, nv * sizeof(float));
    if (flags) memcpy(flags, L->flags, (size_t)L->nl);
}
void orc_level_defaults(const orc_poisson* h, int level, float* out4) {
    const olevel* L = &h->lv[level];
    out4[0] = L->def_diag; out4[1] = L->def_face; out4[2] = L->def_invdiag; out4[3] = L->def_spai0;
}

void orc_build_rhs(const orc_poisson* h, int64_t fw_n, const int32_t* fw_origins, const float* fw_values,
                   const float* fw_bg3, int64_t vx_n, const int32_t* vx_origins, const float* vx_values,
                   float vx_bg, int64_t vy_n, const int32_t* vy_origins, const float* vy_values, float vy_bg,
                   int64_t vz_n, const int32_t* vz_origins, const float* vz_values, float vz_bg,
                   int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
                   float* rhs_out) {
    const olevel* L = &h->lv[0];
    ogrid fw, v[3], sv;
    float b0[3] = {vx_bg, 0, 0}, b1[3] = {vy_bg, 0, 0}, b2[3] = {vz_bg, 0, 0};
    ogrid_init(&fw, fw_n, fw_origins, NULL, fw_values, 3, fw_bg3);
    ogrid_init(&v[0], vx_n, vx_origins, NULL, vx_values, 1, b0);
    ogrid_init(&v[1], vy_n, vy_origins, NULL, vy_values, 1, b1);
    ogrid_init(&v[2], vz_n, vz_origins, NULL, vz_values, 1, b2);
    ogrid_init(&sv, sv_n, sv_origins, NULL, sv_values, 3, sv_bg3);
    float invdx = 1.0f / L->dx;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L->nl; ++i) {
        const int32_t* o = L->org + 3 * i;
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            if (!mbit(L->mask + 8 * i, off)) { rhs_out[me] = 0.f; continue; }
            int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            float rhs = 0;
            int nonzero = 0;
            for (int f = 0; f < 6; ++f) {
                int ch = f / 2, pos = (f % 2) == 0;
                int c[3] = {g[0], g[1], g[2]};
                c[ch] += pos;
                float weight = ogrid_get(&fw, c[0], c[1], c[2], ch);
                if (weight != 0.f) nonzero = 1;
                float vel = ogrid_get(&v[ch], c[0], c[1], c[2], 0);
                float svel = ogrid_get(&sv, c[0], c[1], c[2], ch);
                float a = weight * vel;
                float bb = (1.0f - weight) * svel;
                float flux = invdx * (a + bb);
                if (pos) rhs -= flux; else rhs += flux;
            }
            rhs_out[me] = nonzero ? rhs : 0.f;
        }
    }
    leafmap_free(&fw.map); leafmap_free(&v[0].map); leafmap_free(&v[1].map); leafmap_free(&v[2].map);
    leafmap_free(&sv.map);
}

void orc_apply(orc_poisson* h, int level, int mode, float weight, float w_sor, const float* lhs,
               const float* rhs, float* out) {
    apply_level(&h->lv[level], mode, weight, w_sor, lhs, rhs, out);
}
void orc_first_jacobi(orc_poisson* h, int level, float weight, const float* rhs, float* out) {
    first_jacobi(&h->lv[level], weight, rhs, out);
}
void orc_first_spai0(orc_poisson* h, int level, const float* rhs, float* out) {
    first_spai0(&h->lv[level], rhs, out);
}
void orc_first_rbgs(orc_poisson* h, int level, int red_first, float w_sor, const float* rhs, float* out) {
    first_rbgs(&h->lv[level], red_first, w_sor, rhs, out);
}
void orc_restrict(const orc_poisson* h, int fine_level, const float* fine, float* coarse) {
    restrict_level(h, fine_level, fine, coarse);
}
void orc_prolongate(const orc_poisson* h, int fine_level, const float* coarse, float* fine, float alpha) {
    prolongate_level(h, fine_level, coarse, fine, alpha);
}
void orc_coarsest_solve(orc_poisson* h, const float* rhs, float* out) { coarsest_solve(h, rhs, out); }
void orc_precondition(orc_poisson* h, int smoother, const float* r, float* z) {
    mucycle_precond(h, smoother, z, r, 0, 1, 3);
}

int64_t orc_triplets(const orc_poisson* h, int level, int32_t* rows, int32_t* cols, float* vals) {
    const olevel* L = &h->lv[level];
    int64_t k = 0;
    for (int i = 0; i < L->nl; ++i)
        for (int off = 0; off < LSZ; ++off) {
            if (!mbit(L->mask + 8 * i, off)) continue;
            size_t me = (size_t)i * LSZ + off;
            int row = L->dof_base[i];
            for (int q = 0; q < off; ++q) row += mbit(L->mask + 8 * i, q);
            if (rows) { rows[k] = row; cols[k] = row; vals[k] = L->diag[me]; }
            k++;
            const float* arr[3] = {L->cx, L->cy, L->cz};
            for (int c = 0; c < 3; ++c) {
                for (int s = 0; s < 2; ++s) {
                    int no; int32_t nl = nbv(L, i, off, 2 * c + s, &no);
                    if (nl >= 0 && mbit(L->mask + 8 * nl, no)) {
                        if (rows) {
                            int d = L->dof_base[nl];
                            for (int q = 0; q < no; ++q) d += mbit(L->mask + 8 * nl, q);
                            rows[k] = row; cols[k] = d;
                            vals[k] = s == 0 ? arr[c][me] : arr[c][(size_t)nl * LSZ + no];
                        }
                        k++;
                    }
                }
            }
        }
    return k;
}

void orc_dof_index(const orc_poisson* h, int level, int32_t* out) {
    const olevel* L = &h->lv[level];
    for (int i = 0; i < L->nl; ++i) {
        int d = L->dof_base[i];
        for (int off = 0; off < LSZ; ++off) {
            size_t me = (size_t)i * LSZ + off;
            if (mbit(L->mask + 8 * i, off)) out[me] = d++; else out[me] = -1;
        }
    }
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
