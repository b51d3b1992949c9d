// staged_pipe.cuh -- persistent, double-buffered staged sweeps of the 7-point
// operator over the leaves of one level, for FP32 and 16-bit storage.
//
// A CTA of 128 threads walks the leaves blockIdx.x, blockIdx.x + gridDim.x, ...
// (grid = resident CTAs on the GPU, at most one per leaf).  Its shared memory
// holds two stages of a leaf's arrays (x, b, diag, 1/diag or SPAI0, c_x, c_y,
// c_z); thread 0 issues the bulk copies of the NEXT leaf into the idle stage
// before the CTA computes the current one, so the copy latency overlaps the
// compute and the halo loads instead of adding to every leaf.  The first
// leaf's coefficient copies and neighbour data, which do not change during a
// solve, are issued before the wait for the previous kernel (programmatic
// dependent launch).  Each thread computes 4 z-consecutive voxels with the
// operation sequence of stencil4 / staged_value (simd_vdb_poisson.cpp
// LightWeightApplier, :1190-1470), so the results equal those of the one-leaf
// kernels; a dot product keeps one partial per leaf (reduce_sum over the
// level's leaves), so reductions match too.
#pragma once
#include "poisson_kernels.cuh"

namespace uaamg {

// storage element traits: ARR bytes per leaf array, shared and global access
template <typename E> struct PipeE;
template <> struct PipeE<float> {
    static constexpr unsigned ARR = UAAMG_LEAF * 4;
    static __device__ __forceinline__ float4 s4(const unsigned char* a, int t) {
        return reinterpret_cast<const float4*>(a)[t];
    }
    static __device__ __forceinline__ float s1(const unsigned char* a, int i) {
        return reinterpret_cast<const float*>(a)[i];
    }
    static __device__ __forceinline__ float4 g4(const float* p, long long leaf, int t) { return ld4(p, leaf, t); }
    static __device__ __forceinline__ float g1(const float* p, long long i) { return p[i]; }
    static __device__ __forceinline__ void st(float* p, long long leaf, int t, float4 v) { st4(p, leaf, t, v); }
    static __device__ __forceinline__ void st1(float* p, long long i, float v) { p[i] = v; }
};

// level traits: the FP32 level reads unscaled values; the 16-bit level
// (poisson_mixed.cuh) scales coefficients and rhs by cs and 1/diag by ics
template <class LV> struct PipeLv;
template <> struct PipeLv<DLevel> {
    using E = float;
    static constexpr bool SCALED = false;
    static __device__ __forceinline__ float cs(const DLevel&) { return 1.0f; }
    static __device__ __forceinline__ float ics(const DLevel&) { return 1.0f; }
};

template <class LV>
__device__ __forceinline__ float4 pscale4(const LV& L, float4 v) {
    if constexpr (PipeLv<LV>::SCALED)
        return make_float4(__fmul_rn(v.x, PipeLv<LV>::cs(L)), __fmul_rn(v.y, PipeLv<LV>::cs(L)),
                           __fmul_rn(v.z, PipeLv<LV>::cs(L)), __fmul_rn(v.w, PipeLv<LV>::cs(L)));
    else
        return v;
}
template <class LV>
__device__ __forceinline__ float pscale1(const LV& L, float v) {
    if constexpr (PipeLv<LV>::SCALED) return __fmul_rn(v, PipeLv<LV>::cs(L));
    else return v;
}
template <class LV>
__device__ __forceinline__ float4 piscale4(const LV& L, float4 v) {
    if constexpr (PipeLv<LV>::SCALED)
        return make_float4(__fmul_rn(v.x, PipeLv<LV>::ics(L)), __fmul_rn(v.y, PipeLv<LV>::ics(L)),
                           __fmul_rn(v.z, PipeLv<LV>::ics(L)), __fmul_rn(v.w, PipeLv<LV>::ics(L)));
    else
        return v;
}

// offsets of the arrays inside a stage
enum { PS_X = 0, PS_B = 1, PS_D = 2, PS_I = 3, PS_CX = 4, PS_CY = 5, PS_CZ = 6, PS_N = 7 };

// which arrays a leaf stages in a mode (trimmed leaves use the defaults)
template <int MODE>
struct PSet {
    bool b, d, i, cx, cy, cz;
    __device__ __forceinline__ explicit PSet(unsigned fl) {
        b = (MODE != M_LAPLACIAN);
        d = (MODE != M_RED && MODE != M_BLACK) && !(fl & TRIM_DIAG);
        i = (MODE == M_JACOBI || MODE == M_RED || MODE == M_BLACK) ? !(fl & TRIM_DIAG)
            : (MODE == M_SPAI0 ? !(fl & TRIM_SPAI0) : false);
        cx = !(fl & TRIM_X);
        cy = !(fl & TRIM_Y);
        cz = !(fl & TRIM_Z);
    }
    __device__ __forceinline__ unsigned count() const {
        return 1u + (b ? 1u : 0u) + (d ? 1u : 0u) + (i ? 1u : 0u) + (cx ? 1u : 0u) + (cy ? 1u : 0u) + (cz ? 1u : 0u);
    }
};

// thread 0: arrive on the stage's barrier with the byte count of all the
// leaf's copies, then issue the coefficient copies
template <int MODE, class LV>
__device__ __forceinline__ void pissue_static(const LV& L, int leaf, const PSet<MODE>& Q, unsigned char* st,
                                              uint64_t* bar) {
    using E = typename PipeLv<LV>::E;
    constexpr unsigned A = PipeE<E>::ARR;
    mbar_expect_tx(bar, A * Q.count());
    const long long o = (long long)leaf * UAAMG_LEAF;
    if (Q.d) bulk_g2s(st + PS_D * A, L.diag + o, A, bar);
    if (MODE != M_SPAI0 && Q.i) bulk_g2s(st + PS_I * A, L.invdiag + o, A, bar);
    if (Q.cx) bulk_g2s(st + PS_CX * A, L.cx + o, A, bar);
    if (Q.cy) bulk_g2s(st + PS_CY * A, L.cy + o, A, bar);
    if (Q.cz) bulk_g2s(st + PS_CZ * A, L.cz + o, A, bar);
}
// thread 0: the copies of the vectors (after the wait for the previous kernel)
template <int MODE, class LV>
__device__ __forceinline__ void pissue_dyn(const LV& L, int leaf, const PSet<MODE>& Q,
                                           const typename PipeLv<LV>::E* x, const typename PipeLv<LV>::E* b,
                                           unsigned char* st, uint64_t* bar) {
    using E = typename PipeLv<LV>::E;
    constexpr unsigned A = PipeE<E>::ARR;
    const long long o = (long long)leaf * UAAMG_LEAF;
    bulk_g2s(st + PS_X * A, x + o, A, bar);
    if (Q.b) bulk_g2s(st + PS_B * A, b + o, A, bar);
    if constexpr (MODE == M_SPAI0) {
        if (Q.i) bulk_g2s(st + PS_I * A, L.spai0 + o, A, bar);
    }
}

// a thread's halo: the neighbour leaves whose faces it reads and their face
// coefficients (static), and the neighbours' x values
struct PHalo {
    int xp, xm, yp, ym, z;
    float4 cxp, cyp;
    float cz;
};
struct PHaloX {
    float4 xp, xm, yp, ym;
    float z;
};
template <class LV>
__device__ __forceinline__ void phalo_static(const LV& L, int leaf, int t, PHalo& H) {
    using E = typename PipeLv<LV>::E;
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const int* nb = L.nbr + (long long)leaf * 6;
    const float df = L.def_face;
    H.xp = (X == 7) ? nb[1] : -1;
    H.xm = (X == 0) ? nb[0] : -1;
    H.yp = (Y == 7) ? nb[3] : -1;
    H.ym = (Y == 0) ? nb[2] : -1;
    H.z = (zh == 0) ? nb[4] : nb[5];
    H.cxp = H.cyp = f4splat(df);
    H.cz = df;
    if constexpr (PipeLv<LV>::SCALED) {
        // the stored 16-bit value of a trimmed leaf is the rounded default:
        // a trimmed neighbour reads the FP32 default (flags and values load together)
        if (H.xp >= 0) {
            const unsigned f = L.flags[H.xp];
            const float4 v = pscale4(L, PipeE<E>::g4(L.cx, H.xp, t - 112));
            if (!(f & TRIM_X)) H.cxp = v;
        }
        if (H.yp >= 0) {
            const unsigned f = L.flags[H.yp];
            const float4 v = pscale4(L, PipeE<E>::g4(L.cy, H.yp, t - 14));
            if (!(f & TRIM_Y)) H.cyp = v;
        }
        if (zh == 1 && H.z >= 0) {
            const unsigned f = L.flags[H.z];
            const float v = pscale1(L, PipeE<E>::g1(L.cz, (long long)H.z * UAAMG_LEAF + 4 * t - 4));
            if (!(f & TRIM_Z)) H.cz = v;
        }
    } else {
        // a trimmed FP32 leaf stores its default coefficients (finalize_leaf)
        if (H.xp >= 0) H.cxp = ld4(L.cx, H.xp, t - 112);
        if (H.yp >= 0) H.cyp = ld4(L.cy, H.yp, t - 14);
        if (zh == 1 && H.z >= 0) H.cz = L.cz[(long long)H.z * UAAMG_LEAF + 4 * t - 4];
    }
}
template <typename E>
__device__ __forceinline__ void phalo_dyn(const E* x, int t, const PHalo& H, PHaloX& V) {
    V.xp = (H.xp >= 0) ? PipeE<E>::g4(x, H.xp, t - 112) : f4zero();
    V.xm = (H.xm >= 0) ? PipeE<E>::g4(x, H.xm, t + 112) : f4zero();
    V.yp = (H.yp >= 0) ? PipeE<E>::g4(x, H.yp, t - 14) : f4zero();
    V.ym = (H.ym >= 0) ? PipeE<E>::g4(x, H.ym, t + 14) : f4zero();
    V.z = 0.f;
    if (H.z >= 0) V.z = PipeE<E>::g1(x, (long long)H.z * UAAMG_LEAF + ((t & 1) ? 4 * t - 4 : 4 * t + 7));
}

// the value of the thread's 4 voxels in MODE from a staged leaf (the
// operation sequence of staged_value)
template <int MODE, class LV>
__device__ __forceinline__ float4 pvalue(const LV& L, int t, unsigned fl, unsigned m, const unsigned char* st,
                                         const PHalo& H, const PHaloX& V, float w, float wsor, float one_minus_wsor,
                                         float4& xc) {
    using E = typename PipeLv<LV>::E;
    using P = PipeE<E>;
    constexpr unsigned A = P::ARR;
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const float df = L.def_face;
    const float4 dfv = f4splat(df);
    const unsigned char* sx = st + PS_X * A;
    const unsigned char* scx = st + PS_CX * A;
    const unsigned char* scy = st + PS_CY * A;
    const unsigned char* scz = st + PS_CZ * A;
    xc = P::s4(sx, t);
    const float4 xp = (X < 7) ? P::s4(sx, t + 16) : V.xp;
    const float4 xm = (X > 0) ? P::s4(sx, t - 16) : V.xm;
    const float4 yp = (Y < 7) ? P::s4(sx, t + 2) : V.yp;
    const float4 ym = (Y > 0) ? P::s4(sx, t - 2) : V.ym;
    const float4 cxp = (X < 7) ? ((fl & TRIM_X) ? dfv : pscale4(L, P::s4(scx, t + 16))) : H.cxp;
    const float4 cyp = (Y < 7) ? ((fl & TRIM_Y) ? dfv : pscale4(L, P::s4(scy, t + 2))) : H.cyp;
    const float4 cxm = (fl & TRIM_X) ? dfv : pscale4(L, P::s4(scx, t));
    const float4 cym = (fl & TRIM_Y) ? dfv : pscale4(L, P::s4(scy, t));
    const float4 czo = (fl & TRIM_Z) ? dfv : pscale4(L, P::s4(scz, t));
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = P::s1(sx, 4 * t + 4);
        czp3 = (fl & TRIM_Z) ? df : pscale1(L, P::s1(scz, 4 * t + 4));
        zm0 = V.z;
    } else {
        zm0 = P::s1(sx, 4 * t - 1);
        zp3 = V.z;
        czp3 = H.cz;
    }
    const float zp[4] = {xc.y, xc.z, xc.w, zp3};
    const float zm[4] = {zm0, xc.x, xc.y, xc.z};
    const float czp[4] = {czo.y, czo.z, czo.w, czp3};
    float4 off;
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
    float4 res = f4zero();
    if constexpr (MODE == M_RED || MODE == M_BLACK) {
        const float4 bb = pscale4(L, P::s4(st + PS_B * A, t));
        const float4 iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : piscale4(L, P::s4(st + PS_I * A, t));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int par = (X + Y + j) & 1;
            const bool upd = (MODE == M_RED) ? (par == 0) : (par == 1);
            float r = __fsub_rn(f4get(bb, j), f4get(off, j));
            r = __fmul_rn(r, f4get(iv, j));
            r = __fmul_rn(r, wsor);
            const float v = __fmaf_rn(f4get(xc, j), one_minus_wsor, r);
            f4set(res, j, upd ? v : f4get(xc, j));
        }
    } else {
        const float4 dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : pscale4(L, P::s4(st + PS_D * A, t));
        if constexpr (MODE == M_LAPLACIAN) {
#pragma unroll
            for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        } else {
            const float4 bb = pscale4(L, P::s4(st + PS_B * A, t));
            if constexpr (MODE == M_RESIDUAL) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
            } else if constexpr (MODE == M_JACOBI) {
                const float4 iv =
                    (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : piscale4(L, P::s4(st + PS_I * A, t));
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
                    r = __fmul_rn(r, f4get(iv, j));
                    f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
                }
            } else {  // SPAI0 (FP32 levels only)
                const float4 sp = (fl & TRIM_SPAI0) ? f4splat(L.def_spai0) : P::s4(st + PS_I * A, t);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
                    f4set(res, j, __fmaf_rn(f4get(sp, j), r, f4get(xc, j)));
                }
            }
        }
    }
    if (!(m & 1)) res.x = 0.f;
    if (!(m & 2)) res.y = 0.f;
    if (!(m & 4)) res.z = 0.f;
    if (!(m & 8)) res.w = 0.f;
    return res;
}

#ifndef PIPE_MINB
#define PIPE_MINB 8
#endif
// dynamic shared memory of a pipelined kernel: two stages of PS_N arrays
template <class LV>
constexpr size_t pipe_smem_bytes() {
    return 2u * PS_N * PipeE<typename PipeLv<LV>::E>::ARR;
}

// One sweep (RESTRICT false: out[leaf] = value, optionally scaled by *zscale
// and with the fused z.r of PCG lines 13-15) or one residual + restriction
// (RESTRICT true, MODE M_RESIDUAL: coarse = 0.125 * sum of the active fine
// residuals of each 2x2x2 block, times coarse_scale) over a level.
template <int MODE, class LV, typename TOut, bool RESTRICT>
__global__ void __launch_bounds__(128, PIPE_MINB)
    k_pipe(LV L, const typename PipeLv<LV>::E* x, const typename PipeLv<LV>::E* b, TOut* out, float w, float wsor,
           float one_minus_wsor, DotOut dot, const float* zscale, float coarse_scale, int* err) {
    using E = typename PipeLv<LV>::E;
    constexpr unsigned A = PipeE<E>::ARR;
    extern __shared__ __align__(128) unsigned char psm[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ __align__(16) float rs[RESTRICT ? UAAMG_LEAF : 4];
    __shared__ double shd[4];
    const int t = threadIdx.x;
    const int G = (int)gridDim.x;
    const int nl = L.nl;
    int leaf = (int)blockIdx.x;
    unsigned char* stg0 = psm;
    unsigned char* stg1 = psm + PS_N * A;
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    __syncthreads();
    // first leaf: static data before the wait
    unsigned fl = L.flags[leaf];
    PHalo H;
    phalo_static(L, leaf, t, H);
    if (t == 0) pissue_static<MODE>(L, leaf, PSet<MODE>(fl), stg0, &bar[0]);
    griddep_wait();
    griddep_launch();
    if (t == 0) pissue_dyn<MODE>(L, leaf, PSet<MODE>(fl), x, b, stg0, &bar[0]);
    int j = 0;
    bool ok = true, next_issued = false;
    for (; leaf < nl; ++j, leaf += G) {
        unsigned char* cur = (j & 1) ? stg1 : stg0;
        unsigned char* nst = (j & 1) ? stg0 : stg1;
        uint64_t* cbar = &bar[j & 1];
        uint64_t* nbar = &bar[(j & 1) ^ 1];
        const int nxt = leaf + G;
        unsigned fln = 0;
        next_issued = false;
        if (nxt < nl) {
            fln = L.flags[nxt];
            next_issued = true;
            if (t == 0) {
                const PSet<MODE> Qn(fln);
                pissue_static<MODE>(L, nxt, Qn, nst, nbar);
                pissue_dyn<MODE>(L, nxt, Qn, x, b, nst, nbar);
            }
        }
        PHaloX V;
        phalo_dyn(x, t, H, V);
        const unsigned m = mask4(L.mask, leaf, t);
        // the next leaf's neighbour data load while this leaf computes
        PHalo Hc = H;
        if (nxt < nl) phalo_static(L, nxt, t, H);
        ok = __syncthreads_and(mbar_wait_bounded(cbar, (unsigned)((j >> 1) & 1)) ? 1 : 0) != 0;
        if (!ok) break;
        float4 xc;
        float4 res = pvalue<MODE>(L, t, fl, m, cur, Hc, V, w, wsor, one_minus_wsor, xc);
        if constexpr (RESTRICT) {
            reinterpret_cast<float4*>(rs)[t] = res;
            __syncthreads();
            if (t < 64) {
                const int i = t >> 4, jj0 = (t >> 2) & 3, k = t & 3;
                const uint64_t* mk = L.mask + (long long)leaf * 8;
                float s = 0.f;
#pragma unroll
                for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                        for (int kk = 0; kk < 2; ++kk) {
                            const int fo = ((2 * i + ii) << 6) | ((2 * jj0 + jj) << 3) | (2 * k + kk);
                            if ((mk[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                        }
                const int o = L.octant[leaf];
                const int coff =
                    ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + jj0) << 3) | ((o & 1) * 4 + k);
                const long long ci = (long long)L.parent[leaf] * UAAMG_LEAF + coff;
                if constexpr (PipeLv<LV>::SCALED)
                    PipeE<TOut>::st1(out, ci, __fmul_rn(__fmul_rn(s, 0.125f), coarse_scale));
                else
                    PipeE<TOut>::st1(out, ci, __fmul_rn(s, 0.125f));
            }
        } else {
            if constexpr (PipeLv<LV>::SCALED) {
                if (zscale) {
                    const float zs = *zscale;
                    res = make_float4(__fmul_rn(res.x, zs), __fmul_rn(res.y, zs), __fmul_rn(res.z, zs),
                                      __fmul_rn(res.w, zs));
                }
            }
            PipeE<TOut>::st(out, leaf, t, res);
            if (dot.r) {  // rho_new = z . r, then beta and rho (PCG lines 13-15)
                float4 rr;
                if constexpr (PipeLv<LV>::SCALED) rr = ld4(dot.r, leaf, t);
                else rr = PipeE<E>::s4(cur + PS_B * A, t);  // the b of a level-0 sweep is r
                const double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z +
                                 (double)res.w * rr.w;
                const double part = block_sum128(s, shd);
                if (t == 0) dot.partials[RED_HEADER + leaf] = part;  // published after the loop
            }
        }
        fl = fln;
        __syncthreads();  // the stage just read is free for the copies issued next iteration
    }
    if (!ok) {
        // flag the timeout and let the copies in flight land before the CTA exits
        if (t == 0) {
            if (err) atomicExch(err, 1);
            mbar_wait_bounded(&bar[j & 1], (unsigned)((j >> 1) & 1));
            if (next_issued) mbar_wait_bounded(&bar[(j & 1) ^ 1], (unsigned)(((j + 1) >> 1) & 1));
        }
        __syncthreads();
        return;
    }
    if constexpr (!RESTRICT) {
        if (dot.r) {  // the leaves' z.r partials into the level's reduction
            const int K = (nl - (int)blockIdx.x + G - 1) / G;
            double tot = 0.0;
            if (red_publish_strided<false>(dot.partials, &dot.st->ticket[0], (int)blockIdx.x, G, K, nl, tot)) {
                if (t == 0) {
                    PcgState* st = dot.st;
                    const float rho_new = (float)tot;
                    st->rho_new = rho_new;
                    st->beta = st->first ? 0.f : __fdiv_rn(rho_new, st->rho);
                    st->rho = rho_new;
                    st->ticket[0] = 0;
                }
            }
        }
    }
}

}  // namespace uaamg
