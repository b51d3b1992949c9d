// poisson_bottom.cuh -- the bottom of the Poisson W-cycle in one launch.
//
// In muCyclePreconditioner<2> (SIMD_UAAMG/simd_vdb_poisson.cpp:1844-1977) the
// level next to the coarsest (level lb) is visited twice per visit of the
// level above it, and each visit is seven smoothing / transfer passes over a
// few dozen leaves plus the coarsest CG: fourteen small launches that are
// bound by launch latency, not by their bytes.  k_bottom runs both visits in
// one launch of one thread-block cluster.  Level lb and the coarsest level
// stay resident in the cluster's shared memory for the whole launch: every
// leaf of level lb, with its vectors and coefficients, lives in the shared
// memory of one CTA (leaf i in CTA i / P, slot i % P), the coarsest level's
// vectors in CTA 0.  A stencil reads a neighbour leaf that another CTA holds
// through distributed shared memory; passes are separated by cluster
// barriers.  The per-voxel arithmetic is that of the unfused kernels
// (sweep_value_s, restrict_leaf, k_materialize with SrcFirstJacobi /
// SrcProlong, coarsest_cg_body with the same rows-per-thread shape), so the
// results are bit-identical to the launch sequence it replaces.
#pragma once
#include <cooperative_groups.h>

#include "poisson_kernels.cuh"

namespace uaamg {

namespace cgx = cooperative_groups;

constexpr int BOT_THREADS = 512;     // four 128-thread leaf groups; the coarsest CG's block shape
constexpr int BOT_MAX_CLUSTER = 16;  // non-portable cluster size limit
constexpr int BOT_NT = 512;          // threads of the coarsest CG (coarsest_class 0 and 1)

// One leaf of level lb in shared memory.
struct __align__(16) SLeaf {
    float x[UAAMG_LEAF], b[UAAMG_LEAF], t[UAAMG_LEAF];
    float dg[UAAMG_LEAF], iv[UAAMG_LEAF], cx[UAAMG_LEAF], cy[UAAMG_LEAF], cz[UAAMG_LEAF];
    float fxp[64], fyp[64], fzp[64];  // c_x of the +x neighbour's x = 0 face [y][z], c_y of +y's [x][z], c_z of +z's [x][y]
    uint64_t mask[8];
    const SLeaf* nb[6];               // neighbour leaves (-x,+x,-y,+y,-z,+z) as cluster-shared addresses, or null
    int par, oct;                     // parent leaf on the coarsest level, octant in it
};
constexpr int SLEAF_X = 0, SLEAF_T = 2 * UAAMG_LEAF;  // float offsets of the x and t arrays

struct BottomArgs {
    DLevel L;              // level lb
    const float* rhs;      // level lb rhs (written by the restriction of level lb - 1)
    float* lhs;            // level lb lhs (read by the prolongation into level lb - 1)
    DCoarsest C;           // coarsest level (lb + 1) system
    int nlc;               // coarsest level leaves (held by CTA 0)
    int P;                 // level-lb leaves per CTA
    float w[3];            // pre-smoothing weights (post-smoothing uses them reversed)
};

__device__ __forceinline__ float4 lds4(const float* p, int i) { return reinterpret_cast<const float4*>(p)[i]; }
__device__ __forceinline__ void sts4(float* p, int i, float4 v) { reinterpret_cast<float4*>(p)[i] = v; }
__device__ __forceinline__ float4 mask_out(float4 v, unsigned m) {
    if (!(m & 1)) v.x = 0.f;
    if (!(m & 2)) v.y = 0.f;
    if (!(m & 4)) v.z = 0.f;
    if (!(m & 8)) v.w = 0.f;
    return v;
}
__device__ __forceinline__ unsigned smask4(const SLeaf* s, int t) {
    return (unsigned)((s->mask[t >> 4] >> ((t & 15) * 4)) & 0xFull);
}

// stencil_dyn over shared-memory leaves: the 6-neighbour sum of the float4 of
// thread t, source array at float offset `so` of every leaf
__device__ __forceinline__ void bot_stencil(const SLeaf* me, int so, int t, float4& xc, float4& off) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const float* src = reinterpret_cast<const float*>(me) + so;
    xc = lds4(src, t);
    float4 xp, xm, yp, ym;
    if (X < 7) xp = lds4(src, t + 16);
    else xp = me->nb[1] ? lds4(reinterpret_cast<const float*>(me->nb[1]) + so, t - 112) : f4zero();
    if (X > 0) xm = lds4(src, t - 16);
    else xm = me->nb[0] ? lds4(reinterpret_cast<const float*>(me->nb[0]) + so, t + 112) : f4zero();
    if (Y < 7) yp = lds4(src, t + 2);
    else yp = me->nb[3] ? lds4(reinterpret_cast<const float*>(me->nb[3]) + so, t - 14) : f4zero();
    if (Y > 0) ym = lds4(src, t - 2);
    else ym = me->nb[2] ? lds4(reinterpret_cast<const float*>(me->nb[2]) + so, t + 14) : f4zero();
    const float4 cxp = X < 7 ? lds4(me->cx, t + 16) : lds4(me->fxp, Y * 2 + zh);
    const float4 cyp = Y < 7 ? lds4(me->cy, t + 2) : lds4(me->fyp, X * 2 + zh);
    const float4 cxm = lds4(me->cx, t), cym = lds4(me->cy, t), czo = lds4(me->cz, t);
    const float px = __shfl_xor_sync(FULLMASK, xc.x, 1);
    const float pw = __shfl_xor_sync(FULLMASK, xc.w, 1);
    const float pcz = __shfl_xor_sync(FULLMASK, czo.x, 1);
    const int base = 4 * t;
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = px;
        czp3 = pcz;
        zm0 = me->nb[4] ? reinterpret_cast<const float*>(me->nb[4])[so + base + 7] : 0.f;
    } else {
        zm0 = pw;
        zp3 = me->nb[5] ? reinterpret_cast<const float*>(me->nb[5])[so + base - 4] : 0.f;
        czp3 = me->fzp[X * 8 + Y];
    }
    const float zp[4] = {xc.y, xc.z, xc.w, zp3};
    const float zm[4] = {zm0, xc.x, xc.y, xc.z};
    const float czp[4] = {czo.y, czo.z, czo.w, czp3};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float f1 = __fmul_rn(f4get(xp, j), f4get(cxp, j));
        float f2 = __fmul_rn(f4get(xm, j), f4get(cxm, j));
        float f3 = __fmul_rn(f4get(yp, j), f4get(cyp, j));
        float f4 = __fmul_rn(f4get(ym, j), f4get(cym, j));
        float f5 = __fmul_rn(zp[j], czp[j]);
        float f6 = __fmul_rn(zm[j], f4get(czo, j));
        f1 = __fadd_rn(f1, f2);
        f3 = __fadd_rn(f3, f4);
        f5 = __fadd_rn(f5, f6);
        f1 = __fadd_rn(f1, f3);
        f1 = __fadd_rn(f1, f5);
        f4set(off, j, f1);
    }
}

// weighted Jacobi (sweep_value_s<M_JACOBI>): out = x + w invdiag (b - A x)
__device__ __forceinline__ void bot_jacobi(SLeaf* me, int so, int dst, int t, float w) {
    float4 xc, off;
    bot_stencil(me, so, t, xc, off);
    const float4 bb = lds4(me->b, t), dg = lds4(me->dg, t), iv = lds4(me->iv, t);
    float4 res;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        r = __fmul_rn(r, f4get(iv, j));
        f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
    }
    sts4(reinterpret_cast<float*>(me) + dst, t, mask_out(res, smask4(me, t)));
}

// residual of T restricted into the coarsest rhs held by CTA 0 (restrict_leaf<true>)
__device__ __forceinline__ void bot_restrict(SLeaf* me, int t, float* rs, float* bc0, int group) {
    float4 xc, off;
    bot_stencil(me, SLEAF_T, t, xc, off);
    const float4 bb = lds4(me->b, t), dg = lds4(me->dg, t);
    float4 res;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
    sts4(rs, t, mask_out(res, smask4(me, t)));
    asm volatile("bar.sync %0, 128;" ::"r"(1 + group) : "memory");
    if (t < 64) {
        const int i = t >> 4, j = (t >> 2) & 3, k = t & 3;
        float s = 0.f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    int fo = ((2 * i + ii) << 6) | ((2 * j + jj) << 3) | (2 * k + kk);
                    if ((me->mask[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                }
        const int o = me->oct;
        const int coff = ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + j) << 3) | ((o & 1) * 4 + k);
        bc0[(long long)me->par * UAAMG_LEAF + coff] = __fmul_rn(s, 0.125f);
    }
    asm volatile("bar.sync %0, 128;" ::"r"(1 + group) : "memory");
}

// T = w invdiag b (the first sweep from zero, SrcFirstJacobi, materialised)
__device__ __forceinline__ void bot_first(SLeaf* me, int t, float w) {
    const float4 bb = lds4(me->b, t), iv = lds4(me->iv, t);
    const float4 v = make_float4(__fmul_rn(w, __fmul_rn(iv.x, bb.x)), __fmul_rn(w, __fmul_rn(iv.y, bb.y)),
                                 __fmul_rn(w, __fmul_rn(iv.z, bb.z)), __fmul_rn(w, __fmul_rn(iv.w, bb.w)));
    sts4(me->t, t, mask_out(v, smask4(me, t)));
}

// T += x_c(parent voxel) on the DOF (SrcProlong with alpha 1, materialised)
__device__ __forceinline__ void bot_prolong(SLeaf* me, int t, const float* xc0) {
    float4 v = lds4(me->t, t);
    const unsigned m = smask4(me, t);
    if (m) {
        const int o = me->oct;
        const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
        const int coff =
            (((o >> 2) & 1) * 4 + (X >> 1)) * 64 + (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4 + 2 * zh;
        const float* cp = xc0 + (long long)me->par * UAAMG_LEAF + coff;
        const float c0 = __fmul_rn(1.0f, cp[0]), c1 = __fmul_rn(1.0f, cp[1]);
        if (m & 1) v.x = __fadd_rn(v.x, c0);
        if (m & 2) v.y = __fadd_rn(v.y, c0);
        if (m & 4) v.z = __fadd_rn(v.z, c1);
        if (m & 8) v.w = __fadd_rn(v.w, c1);
    }
    sts4(me->t, t, mask_out(v, m));
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Dynamic shared memory of one CTA: P leaves, then (used by CTA 0 only) the
// coarsest level's lhs and rhs, the CG's vector, one restriction scratch per
// leaf group.
__host__ __device__ inline size_t bottom_smem_bytes(int P, int nlc, int rows) {
    return (size_t)P * sizeof(SLeaf) + (size_t)nlc * UAAMG_LEAF * 4 * 2 + (size_t)(BOT_NT * rows + 4) * 4 +
           (size_t)(BOT_THREADS / 128) * UAAMG_LEAF * 4;
}

template <int ROWS>
__global__ void __launch_bounds__(BOT_THREADS, 1) k_bottom(BottomArgs A) {
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ __align__(16) float red[3][64];
    cgx::cluster_group cl = cgx::this_cluster();
    const unsigned rank = cl.block_rank();
    const int group = threadIdx.x >> 7, t = threadIdx.x & 127;
    constexpr int NG = BOT_THREADS / 128;
    const int P = A.P;
    SLeaf* sl = reinterpret_cast<SLeaf*>(bsm);
    float* xc0 = reinterpret_cast<float*>(bsm + (size_t)P * sizeof(SLeaf));  // coarsest lhs (CTA 0)
    float* bc0 = xc0 + (size_t)A.nlc * UAAMG_LEAF;                            // coarsest rhs (CTA 0)
    float* ps = bc0 + (size_t)A.nlc * UAAMG_LEAF;
    float* rs = ps + BOT_NT * ROWS + 4 + group * UAAMG_LEAF;
    // the coarsest vectors of CTA 0 as every CTA addresses them
    float* xc0c = cl.map_shared_rank(xc0, 0);
    float* bc0c = cl.map_shared_rank(bc0, 0);
    const DLevel& L = A.L;
    const int nl = L.nl;

    // ---- static data (does not change during a solve): before the wait
    for (int j = group; j < P; j += NG) {
        SLeaf* me = sl + j;
        const int leaf = (int)rank * P + j;
        if (leaf >= nl) continue;
        const unsigned fl = L.flags[leaf];
        const float4 dfv = f4splat(L.def_face);
        sts4(me->dg, t, (fl & TRIM_DIAG) ? f4splat(L.def_diag) : ld4(L.diag, leaf, t));
        sts4(me->iv, t, (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : ld4(L.invdiag, leaf, t));
        sts4(me->cx, t, (fl & TRIM_X) ? dfv : ld4(L.cx, leaf, t));
        sts4(me->cy, t, (fl & TRIM_Y) ? dfv : ld4(L.cy, leaf, t));
        sts4(me->cz, t, (fl & TRIM_Z) ? dfv : ld4(L.cz, leaf, t));
        const int* nb = L.nbr + (long long)leaf * 6;
        if (t < 64) {
            // + faces: (y,z) / (x,z) / (x,y) = (t >> 3, t & 7)
            const int a = t >> 3, c = t & 7;
            const int n1 = nb[1], n3 = nb[3], n5 = nb[5];
            me->fxp[t] = n1 >= 0 ? ((L.flags[n1] & TRIM_X) ? L.def_face : L.cx[(long long)n1 * UAAMG_LEAF + a * 8 + c])
                                 : L.def_face;
            me->fyp[t] = n3 >= 0 ? ((L.flags[n3] & TRIM_Y) ? L.def_face : L.cy[(long long)n3 * UAAMG_LEAF + a * 64 + c])
                                 : L.def_face;
            me->fzp[t] = n5 >= 0 ? ((L.flags[n5] & TRIM_Z) ? L.def_face : L.cz[(long long)n5 * UAAMG_LEAF + a * 64 + c * 8])
                                 : L.def_face;
        } else if (t < 72) {
            me->mask[t - 64] = L.mask[(long long)leaf * 8 + (t - 64)];
        } else if (t < 78) {
            const int n = nb[t - 72];
            me->nb[t - 72] = n >= 0 ? cl.map_shared_rank(sl + (n % P), (unsigned)(n / P)) : nullptr;
        } else if (t == 78) {
            me->par = L.parent[leaf];
            me->oct = L.octant[leaf];
        }
    }
    griddep_wait();
    griddep_launch();
    for (int j = group; j < P; j += NG) {
        const int leaf = (int)rank * P + j;
        if (leaf < nl) sts4(sl[j].b, t, ld4(A.rhs, leaf, t));
    }
    cluster_sync_all();  // every CTA has started and filled its leaves

    const float w0 = A.w[0], w1 = A.w[1], w2 = A.w[2];
#define BOT_EACH(body)                                      \
    for (int j = group; j < P; j += NG) {                   \
        SLeaf* me = sl + j;                                 \
        if ((int)rank * P + j < nl) { body; }               \
    }                                                       \
    cluster_sync_all();
    for (int visit = 0; visit < 2; ++visit) {
        // pre-smoothing, ends in T
        if (visit == 0) {
            BOT_EACH(bot_first(me, t, w0));                  // T = first sweep from zero
            BOT_EACH(bot_jacobi(me, SLEAF_T, SLEAF_X, t, w1));  // x = J(T)
            BOT_EACH(bot_jacobi(me, SLEAF_X, SLEAF_T, t, w2));  // T = J(x)
        } else {
            BOT_EACH(bot_jacobi(me, SLEAF_X, SLEAF_T, t, w0));
            BOT_EACH(bot_jacobi(me, SLEAF_T, SLEAF_X, t, w1));
            BOT_EACH(bot_jacobi(me, SLEAF_X, SLEAF_T, t, w2));
        }
        // residual of T restricted into the coarsest rhs
        BOT_EACH(bot_restrict(me, t, rs, bc0c, group));
        // coarsest solve (its second visit in the W-cycle re-solves the same system: skipped).  The rows
        // are loaded from L2 for each solve: holding them in registers across the whole kernel measured
        // three times slower (31 against 11 us per solve on the 1916-DOF level)
        if (rank == 0) coarsest_cg_body<ROWS, BOT_NT, false>(A.C, bc0, xc0, ps, red);
        cluster_sync_all();
        // post-smoothing with reversed weights: T += P x_c, x = J(T), T = J(x), x = J(T)
        BOT_EACH(bot_prolong(me, t, xc0c));
        BOT_EACH(bot_jacobi(me, SLEAF_T, SLEAF_X, t, w2));
        BOT_EACH(bot_jacobi(me, SLEAF_X, SLEAF_T, t, w1));
        BOT_EACH(bot_jacobi(me, SLEAF_T, SLEAF_X, t, w0));
    }
#undef BOT_EACH
    for (int j = group; j < P; j += NG) {
        const int leaf = (int)rank * P + j;
        if (leaf < nl) st4(A.lhs, leaf, t, lds4(sl[j].x, t));
    }
    // (the last pass ended with a cluster barrier, so no CTA still reads another's shared memory)
}

}  // namespace uaamg
