/*
 * oracle_common.h -- helpers shared by the CPU oracle's translation units
 * (leaf lookup, OpenVDB voxel/mask conventions, flattened input grids, OpenVDB
 * tree order of leaves).  TEST INFRASTRUCTURE ONLY.
 */
#ifndef UAAMG_ORACLE_COMMON_H
#define UAAMG_ORACLE_COMMON_H
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LSZ 512

/* ------------------------------------------------------------------------ */
/* leaf lookup: dense index volume over the bounding box of leaf coordinates */
typedef struct {
    int32_t lo[3], dim[3];
    int32_t* idx;
} leafmap;

static void leafmap_init(leafmap* m, int64_t n, const int32_t* org) {
    memset(m, 0, sizeof(*m));
    if (n <= 0) return;
    int32_t mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            int32_t v = org[3 * i + c] >> 3;
            if (v < mn[c]) mn[c] = v;
            if (v > mx[c]) mx[c] = v;
        }
    int64_t tot = 1;
    for (int c = 0; c < 3; ++c) {
        m->lo[c] = mn[c];
        m->dim[c] = mx[c] - mn[c] + 1;
        tot *= m->dim[c];
    }
    m->idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)tot);
    for (int64_t i = 0; i < tot; ++i) m->idx[i] = -1;
    for (int64_t i = 0; i < n; ++i) {
        int32_t a = (org[3 * i] >> 3) - m->lo[0], b = (org[3 * i + 1] >> 3) - m->lo[1],
                c = (org[3 * i + 2] >> 3) - m->lo[2];
        m->idx[((int64_t)a * m->dim[1] + b) * m->dim[2] + c] = (int32_t)i;
    }
}
static void leafmap_free(leafmap* m) { free(m->idx); m->idx = NULL; }

/* leaf index of the leaf containing voxel (x,y,z), -1 if none */
static inline int32_t leafmap_find(const leafmap* m, int x, int y, int z) {
    if (!m->idx) return -1;
    int32_t a = (x >> 3) - m->lo[0], b = (y >> 3) - m->lo[1], c = (z >> 3) - m->lo[2];
    if ((unsigned)a >= (unsigned)m->dim[0] || (unsigned)b >= (unsigned)m->dim[1] ||
        (unsigned)c >= (unsigned)m->dim[2])
        return -1;
    return m->idx[((int64_t)a * m->dim[1] + b) * m->dim[2] + c];
}

static inline int voff(int x, int y, int z) { return ((x & 7) << 6) | ((y & 7) << 3) | (z & 7); }
static inline int mbit(const uint64_t* m, int off) { return (int)((m[off >> 6] >> (off & 63)) & 1u); }

/* a flattened input grid with ConstAccessor::getValue semantics */
typedef struct {
    int64_t n;
    const int32_t* org;
    const uint64_t* mask;
    const float* val;
    int comps;
    float bg[3];
    leafmap map;
} ogrid;

static void ogrid_init(ogrid* g, int64_t n, const int32_t* org, const uint64_t* mask,
                       const float* val, int comps, const float* bg) {
    g->n = n; g->org = org; g->mask = mask; g->val = val; g->comps = comps;
    for (int c = 0; c < 3; ++c) g->bg[c] = (c < comps) ? bg[c] : 0.f;
    leafmap_init(&g->map, n, org);
}
static inline float ogrid_get(const ogrid* g, int x, int y, int z, int c) {
    int32_t li = leafmap_find(&g->map, x, y, z);
    if (li < 0) return g->bg[c];
    return g->val[((int64_t)li * LSZ + voff(x, y, z)) * g->comps + c];
}

/* OpenVDB BoxSampler::sample over a getValue accessor (tools/Interpolation.h):
 * floor, fractional weights in double, three levels of
 *   a + float((double)(b - a) * w). */
static inline float vdb_lerp(float a, float b, double w) {
    float d = b - a;
    double t = (double)d * w;
    return a + (float)t;
}
static inline float box_sample(const ogrid* g, double px, double py, double pz) {
    double fx = floor(px), fy = floor(py), fz = floor(pz);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    double u = px - fx, v = py - fy, w = pz - fz;
    float d[2][2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) d[i][j][k] = ogrid_get(g, ix + i, iy + j, iz + k, 0);
    float a0 = vdb_lerp(vdb_lerp(d[0][0][0], d[0][0][1], w), vdb_lerp(d[0][1][0], d[0][1][1], w), v);
    float a1 = vdb_lerp(vdb_lerp(d[1][0][0], d[1][0][1], w), vdb_lerp(d[1][1][0], d[1][1][1], w), v);
    return vdb_lerp(a0, a1, u);
}

/* ------------------------------------------------------------------------ */
/* OpenVDB tree order of leaves (RootNode std::map by Coord, then InternalNode
 * child offsets for the 5-4-3 tree). */
typedef struct { int32_t k[5]; int32_t i; } leafkey;
static void make_key(leafkey* key, const int32_t* o, int32_t i) {
    key->k[0] = o[0] & ~4095; key->k[1] = o[1] & ~4095; key->k[2] = o[2] & ~4095;
    key->k[3] = (((o[0] & 4095) >> 7) << 10) | (((o[1] & 4095) >> 7) << 5) | ((o[2] & 4095) >> 7);
    key->k[4] = (((o[0] & 127) >> 3) << 8) | (((o[1] & 127) >> 3) << 4) | ((o[2] & 127) >> 3);
    key->i = i;
}
static int cmp_key(const void* a, const void* b) {
    const leafkey* x = (const leafkey*)a; const leafkey* y = (const leafkey*)b;
    for (int c = 0; c < 5; ++c) {
        if (x->k[c] < y->k[c]) return -1;
        if (x->k[c] > y->k[c]) return 1;
    }
    return 0;
}

#endif
