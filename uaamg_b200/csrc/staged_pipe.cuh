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
// kernels.  A fused dot product sums each CTA's leaves in leaf order and
// reduces the PIPE_CTAS partials with reduce_sum: one ticket per CTA.
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

// level traits.  A 16-bit level (poisson_mixed.cuh) stores its coefficients
// and rhs divided by a power of two cs and 1/diag multiplied by it; since
// scaling by a power of two is exact, the pipelined kernels compute in the
// stored units -- off-diagonal sum, diagonal term and residual all come out
// divided by cs, and the product with the stored 1/diag is the true value --
// with the defaults of trimmed leaves brought to the same units (def_face /
// cs, def_diag / cs, def_invdiag * cs).  Each result equals the one computed
// from rescaled values.
template <class LV> struct PipeLv;
template <> struct PipeLv<DLevel> {
    using E = float;
    static constexpr bool SCALED = false;
    static __device__ __forceinline__ float def_face(const DLevel& L) { return L.def_face; }
    static __device__ __forceinline__ float def_diag(const DLevel& L) { return L.def_diag; }
    static __device__ __forceinline__ float def_invdiag(const DLevel& L) { return L.def_invdiag; }
};

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

// ---------------------------------------------------------------------------
// Stage layout (bytes): the PS_N leaf arrays, then the halo a leaf's stencil
// reads from its neighbours -- face chunks of 4 values (x of the +-x and +-y
// neighbours, c_x of the +x and c_y of the +y neighbour), the z-face values
// (x of the -z / +z neighbour per thread, c_z of the +z neighbour), the
// leaf's DOF mask and, for 16-bit levels, the flags of the +x, +y and +z
// neighbours (a trimmed neighbour reads the default).  Halo values are
// copied by the threads that use them (cp.async, 4-16 bytes), a 16-bit z
// value as the aligned pair that holds it.
template <typename E>
struct PLayout {
    static constexpr unsigned A = PipeE<E>::ARR;
    static constexpr unsigned C = 4u * (unsigned)sizeof(E);
    static constexpr unsigned HXP = PS_N * A;
    static constexpr unsigned HXM = HXP + 16 * C;
    static constexpr unsigned HYP = HXM + 16 * C;
    static constexpr unsigned HYM = HYP + 16 * C;
    static constexpr unsigned HCXP = HYM + 16 * C;
    static constexpr unsigned HCYP = HCXP + 16 * C;
    static constexpr unsigned HZ = HCYP + 16 * C;  // 128 x 4 B
    static constexpr unsigned HCZ = HZ + 512;      // 64 x 4 B
    static constexpr unsigned MASK = HCZ + 256;    // 8 x 8 B
    static constexpr unsigned FLG = MASK + 64;     // 3 x 4 B
    static constexpr unsigned STAGE = (FLG + 16 + 127) / 128 * 128;
};

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// the barrier's next phase also waits for this thread's cp.async copies so far
__device__ __forceinline__ void cpa_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <typename E>
__device__ __forceinline__ void cpa_chunk(unsigned char* dst, const E* src) {
    if constexpr (sizeof(E) == 4) cpa16(dst, src);
    else cpa8(dst, src);
}
template <typename E>
__device__ __forceinline__ void zero_chunk(unsigned char* dst) {
    if constexpr (sizeof(E) == 4) *reinterpret_cast<float4*>(dst) = f4zero();
    else *reinterpret_cast<uint2*>(dst) = make_uint2(0u, 0u);
}

// neighbour row of a leaf: -x +x -y +y -z +z
struct PNb {
    int v[6];
};
__device__ __forceinline__ PNb pnb_load(const int* nbr, int leaf) {
    const int2* p = reinterpret_cast<const int2*>(nbr + (long long)leaf * 6);
    const int2 a = p[0], b = p[1], c = p[2];
    PNb r;
    r.v[0] = a.x;
    r.v[1] = a.y;
    r.v[2] = b.x;
    r.v[3] = b.y;
    r.v[4] = c.x;
    r.v[5] = c.y;
    return r;
}

// Issue a thread's share of a leaf's halo: STAT the coefficient faces, the
// mask and the flags (no change during a solve), DYN the x faces.  Each
// group of 16 threads copies one kind of face chunk (threads 0-15 the -x
// face, 16-31 +x, 32-47 -y, 48-63 +y, 64-79 c_x of the +x neighbour, 80-95
// c_y of the +y neighbour, 96-127 c_z of the +z neighbour, two each), so
// the branches are uniform over half-warps; every thread copies its own
// z-face value.  The slots are those pvalue reads: a +-y face slot
// s = 2X + zh holds the chunk of the consumer thread 16X + 14 + zh (+y) or
// 16X + zh (-y).
template <bool STAT, bool DYN, class LV>
__device__ __forceinline__ void phalo_issue(const LV& L, int leaf, const PNb& N, int t, unsigned char* st,
                                            const typename PipeLv<LV>::E* x) {
    using E = typename PipeLv<LV>::E;
    using Lo = PLayout<E>;
    constexpr unsigned C = Lo::C;
    const int c = t >> 4, i = t & 15;
    const int ych = 16 * (i >> 1) + (i & 1);  // +y neighbour chunk of y-face slot i (-y: + 14)
    if constexpr (STAT) {
        if (c == 4) {
            const int n = N.v[1];
            unsigned char* d = st + Lo::HCXP + i * C;
            if (n >= 0) cpa_chunk(d, L.cx + (long long)n * UAAMG_LEAF + 4 * i);
            else if constexpr (!PipeLv<LV>::SCALED) *reinterpret_cast<float4*>(d) = f4splat(L.def_face);
        } else if (c == 5) {
            const int n = N.v[3];
            unsigned char* d = st + Lo::HCYP + i * C;
            if (n >= 0) cpa_chunk(d, L.cy + (long long)n * UAAMG_LEAF + 4 * ych);
            else if constexpr (!PipeLv<LV>::SCALED) *reinterpret_cast<float4*>(d) = f4splat(L.def_face);
        } else if (c >= 6) {
            // c_z entries e = 2j, 2j+1 of the consumers 2e+1 (zh = 1): elements 8e
            const int n = N.v[5];
            const int e0 = 2 * (t - 96);
            unsigned char* d = st + Lo::HCZ + 4 * e0;
            if (n >= 0) {
                cpa4(d, L.cz + (long long)n * UAAMG_LEAF + 8 * e0);
                cpa4(d + 4, L.cz + (long long)n * UAAMG_LEAF + 8 * e0 + 8);
            } else if constexpr (!PipeLv<LV>::SCALED) {
                *reinterpret_cast<float2*>(d) = make_float2(L.def_face, L.def_face);
            }
            if (t < 100) {
                cpa16(st + Lo::MASK + 16 * (t - 96),
                      reinterpret_cast<const unsigned char*>(L.mask + (long long)leaf * 8) + 16 * (t - 96));
            } else if constexpr (PipeLv<LV>::SCALED) {
                if (t < 103) {
                    const int nn = (t == 100) ? N.v[1] : ((t == 101) ? N.v[3] : N.v[5]);  // +x, +y, +z
                    unsigned char* f = st + Lo::FLG + 4 * (t - 100);
                    if (nn >= 0) cpa4(f, L.flags + nn);
                    else *reinterpret_cast<unsigned*>(f) = 0xFFFFFFFFu;  // missing: the default
                }
            }
        }
    }
    if constexpr (DYN) {
        if (c < 4) {
            const int n = (c == 0) ? N.v[0] : ((c == 1) ? N.v[1] : ((c == 2) ? N.v[2] : N.v[3]));
            const unsigned off = (c == 0) ? Lo::HXM : ((c == 1) ? Lo::HXP : ((c == 2) ? Lo::HYM : Lo::HYP));
            const int ch = (c == 0) ? i + 112 : ((c == 1) ? i : ((c == 2) ? ych + 14 : ych));
            unsigned char* d = st + off + i * C;
            if (n >= 0) cpa_chunk(d, x + (long long)n * UAAMG_LEAF + 4 * ch);
            else zero_chunk<E>(d);
        }
        const int zh = t & 1;
        const int n = zh ? N.v[5] : N.v[4];
        unsigned char* d = st + Lo::HZ + 4 * t;
        if (n >= 0) {
            // FP32: the value; 16-bit: the aligned pair holding it
            const long long e =
                (long long)n * UAAMG_LEAF + (zh ? 4 * t - 4 : (sizeof(E) == 4 ? 4 * t + 7 : 4 * t + 6));
            cpa4(d, x + e);
        } else {
            *reinterpret_cast<unsigned*>(d) = 0u;
        }
    }
}

// a z-face value read back from the stage (16-bit: high or low half of the pair)
template <typename E>
__device__ __forceinline__ float phz(const unsigned char* p, bool high) {
    if constexpr (sizeof(E) == 4) {
        return *reinterpret_cast<const float*>(p);
    } else {
        const unsigned u = *reinterpret_cast<const unsigned*>(p);
        return PipeE<E>::bits1((unsigned short)(high ? (u >> 16) : (u & 0xFFFFu)));
    }
}

// the value of the thread's 4 voxels in MODE from a staged leaf and its halo
// (the operation sequence of staged_value)
template <int MODE, class LV>
__device__ __forceinline__ float4 pvalue(const LV& L, int t, unsigned fl, const unsigned char* st, float w,
                                         float wsor, float one_minus_wsor) {
    using E = typename PipeLv<LV>::E;
    using P = PipeE<E>;
    using Lo = PLayout<E>;
    constexpr unsigned A = P::ARR;
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const int ys = 2 * X + zh;
    const float df = PipeLv<LV>::def_face(L);
    const float4 dfv = f4splat(df);
    const unsigned char* sx = st + PS_X * A;
    const unsigned char* scx = st + PS_CX * A;
    const unsigned char* scy = st + PS_CY * A;
    const unsigned char* scz = st + PS_CZ * A;
    const float4 xc = P::s4(sx, t);
    const float4 xp = (X < 7) ? P::s4(sx, t + 16) : P::s4(st + Lo::HXP, t - 112);
    const float4 xm = (X > 0) ? P::s4(sx, t - 16) : P::s4(st + Lo::HXM, t);
    const float4 yp = (Y < 7) ? P::s4(sx, t + 2) : P::s4(st + Lo::HYP, ys);
    const float4 ym = (Y > 0) ? P::s4(sx, t - 2) : P::s4(st + Lo::HYM, ys);
    const unsigned* nf = reinterpret_cast<const unsigned*>(st + Lo::FLG);
    float4 cxp, cyp;
    if (X < 7) {
        cxp = (fl & TRIM_X) ? dfv : P::s4(scx, t + 16);
    } else if constexpr (PipeLv<LV>::SCALED) {
        cxp = (nf[0] & TRIM_X) ? dfv : P::s4(st + Lo::HCXP, t - 112);
    } else {
        cxp = P::s4(st + Lo::HCXP, t - 112);
    }
    if (Y < 7) {
        cyp = (fl & TRIM_Y) ? dfv : P::s4(scy, t + 2);
    } else if constexpr (PipeLv<LV>::SCALED) {
        cyp = (nf[1] & TRIM_Y) ? dfv : P::s4(st + Lo::HCYP, ys);
    } else {
        cyp = P::s4(st + Lo::HCYP, ys);
    }
    const float4 cxm = (fl & TRIM_X) ? dfv : P::s4(scx, t);
    const float4 cym = (fl & TRIM_Y) ? dfv : P::s4(scy, t);
    const float4 czo = (fl & TRIM_Z) ? dfv : P::s4(scz, t);
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = P::s1(sx, 4 * t + 4);
        czp3 = (fl & TRIM_Z) ? df : P::s1(scz, 4 * t + 4);
        zm0 = phz<E>(st + Lo::HZ + 4 * t, true);
    } else {
        zm0 = P::s1(sx, 4 * t - 1);
        zp3 = phz<E>(st + Lo::HZ + 4 * t, false);
        if constexpr (PipeLv<LV>::SCALED)
            czp3 = (nf[2] & TRIM_Z) ? df : phz<E>(st + Lo::HCZ + 4 * (t >> 1), false);
        else
            czp3 = phz<E>(st + Lo::HCZ + 4 * (t >> 1), false);
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
    const uint64_t mw = reinterpret_cast<const uint64_t*>(st + Lo::MASK)[t >> 4];
    const unsigned m = (unsigned)((mw >> ((t & 15) * 4)) & 0xFull);
    float4 res = f4zero();
    if constexpr (MODE == M_RED || MODE == M_BLACK) {
        const float4 bb = P::s4(st + PS_B * A, t);
        const float4 iv = (fl & TRIM_DIAG) ? f4splat(PipeLv<LV>::def_invdiag(L)) : P::s4(st + PS_I * A, t);
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
        const float4 dg = (fl & TRIM_DIAG) ? f4splat(PipeLv<LV>::def_diag(L)) : P::s4(st + PS_D * A, t);
        if constexpr (MODE == M_LAPLACIAN) {
#pragma unroll
            for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        } else {
            const float4 bb = P::s4(st + PS_B * A, t);
            if constexpr (MODE == M_RESIDUAL) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
            } else if constexpr (MODE == M_JACOBI) {
                const float4 iv =
                    (fl & TRIM_DIAG) ? f4splat(PipeLv<LV>::def_invdiag(L)) : P::s4(st + PS_I * A, t);
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
#define PIPE_MINB 6  // FP32: 6 stages of 33.5 KB fill the shared memory of an SM
#endif
#ifndef PIPE_MINB16
#define PIPE_MINB16 7  // 16-bit stages are half the size: one more CTA per SM (8 spills)
#endif
// CTAs of a pipelined launch (at most one per leaf): 6 per SM on a 148-SM
// B200.  A constant rather than the occupancy of the GPU at hand, so the
// order of a fused dot product's sum depends only on the level.
#define PIPE_CTAS 888
// dynamic shared memory of a pipelined kernel: two stages
template <class LV>
constexpr size_t pipe_smem_bytes() {
    return 2u * PLayout<typename PipeLv<LV>::E>::STAGE;
}

// One sweep (RESTRICT false: out[leaf] = value, optionally scaled by *zscale
// and with the fused z.r of PCG lines 13-15) or one residual + restriction
// (RESTRICT true, MODE M_RESIDUAL: coarse = 0.125 * sum of the active fine
// residuals of each 2x2x2 block, times coarse_scale on 16-bit levels) over a
// level.  Everything a leaf reads -- its arrays by bulk copies (thread 0),
// its halo, mask and neighbour flags by cp.async (each thread its share) --
// is in flight into one stage while the CTA computes the leaf in the other;
// every thread's cp.async arrival and thread 0's byte count complete a
// stage's barrier phase.
//
// DOTK selects the fused dot of a sweep: 0 z.r with the b of a level-0 sweep
// or dot.r (PCG lines 13-15: rho, beta), 1 p.q with p the swept vector (the
// Laplacian of PCG lines 6-7: sigma, alpha).
template <int MODE, class LV, typename TOut, bool RESTRICT, int DOTK = 0>
__global__ void __launch_bounds__(128, PipeLv<LV>::SCALED ? PIPE_MINB16 : PIPE_MINB)
    k_pipe(LV L, const typename PipeLv<LV>::E* x, const typename PipeLv<LV>::E* b, TOut* out, float w, float wsor,
           float one_minus_wsor, DotOut dot, const float* zscale, float coarse_scale, int* err) {
    using E = typename PipeLv<LV>::E;
    using Lo = PLayout<E>;
    extern __shared__ __align__(128) unsigned char psm[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ __align__(16) float rs[RESTRICT ? UAAMG_LEAF : 4];
    __shared__ double shd[4];
    const int t = threadIdx.x;
    const int G = (int)gridDim.x;
    const int nl = L.nl;
    int leaf = (int)blockIdx.x;
    if (t == 0) {
        mbar_init(&bar[0], 1 + 128);  // thread 0's byte count + every thread's cp.async arrival
        mbar_init(&bar[1], 1 + 128);
    }
    __syncthreads();
    // first leaf: static data before the wait for the previous kernel
    unsigned fl = L.flags[leaf];
    PNb N = pnb_load(L.nbr, leaf);
    if (t == 0) pissue_static<MODE>(L, leaf, PSet<MODE>(fl), psm, &bar[0]);
    phalo_issue<true, false>(L, leaf, N, t, psm, x);
    griddep_wait();
    griddep_launch();
    if (t == 0) pissue_dyn<MODE>(L, leaf, PSet<MODE>(fl), x, b, psm, &bar[0]);
    phalo_issue<false, true>(L, leaf, N, t, psm, x);
    cpa_arrive(&bar[0]);
    // the next leaf's row and flags
    unsigned fln = 0;
    if (leaf + G < nl) {
        fln = L.flags[leaf + G];
        N = pnb_load(L.nbr, leaf + G);
    }
    int j = 0;
    bool ok = true, next_issued = false;
    double cta_dot = 0.0;  // thread 0: this CTA's leaves' z.r partials, in leaf order
    for (; leaf < nl; ++j, leaf += G) {
        unsigned char* cur = psm + (j & 1) * Lo::STAGE;
        unsigned char* nst = psm + ((j & 1) ^ 1) * Lo::STAGE;
        uint64_t* cbar = &bar[j & 1];
        uint64_t* nbar = &bar[(j & 1) ^ 1];
        const int nxt = leaf + G;
        next_issued = nxt < nl;
        if (next_issued) {
            if (t == 0) {
                const PSet<MODE> Qn(fln);
                pissue_static<MODE>(L, nxt, Qn, nst, nbar);
                pissue_dyn<MODE>(L, nxt, Qn, x, b, nst, nbar);
            }
            phalo_issue<true, true>(L, nxt, N, t, nst, x);
            cpa_arrive(nbar);
        }
        const unsigned flc = fl;
        fl = fln;
        if (nxt + G < nl) {  // row and flags two leaves ahead, in flight during this leaf
            fln = L.flags[nxt + G];
            N = pnb_load(L.nbr, nxt + G);
        }
        float4 rr = f4zero();
        if constexpr (!RESTRICT && PipeLv<LV>::SCALED && DOTK == 0) {
            if (dot.r) rr = ld4(dot.r, leaf, t);
        }
        int par = 0, oct = 0;
        if constexpr (RESTRICT) {
            if (t < 64) {
                par = L.parent[leaf];
                oct = L.octant[leaf];
            }
        }
        ok = __syncthreads_and(mbar_wait_bounded(cbar, (unsigned)((j >> 1) & 1)) ? 1 : 0) != 0;
        if (!ok) break;
        float4 res = pvalue<MODE>(L, t, flc, cur, w, wsor, one_minus_wsor);
        if constexpr (RESTRICT) {
            reinterpret_cast<float4*>(rs)[t] = res;
            __syncthreads();
            if (t < 64) {
                const int i = t >> 4, jj0 = (t >> 2) & 3, k = t & 3;
                const uint64_t* mk = reinterpret_cast<const uint64_t*>(cur + Lo::MASK);
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
                const int coff =
                    ((((oct >> 2) & 1) * 4 + i) << 6) | ((((oct >> 1) & 1) * 4 + jj0) << 3) | ((oct & 1) * 4 + k);
                const long long ci = (long long)par * UAAMG_LEAF + coff;
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
            if (dot.r) {  // this leaf's z.r (p.q) partial into the CTA's sum
                if constexpr (DOTK == 1) rr = PipeE<E>::s4(cur + PS_X * PipeE<E>::ARR, t);  // p
                else if constexpr (!PipeLv<LV>::SCALED) rr = PipeE<E>::s4(cur + PS_B * PipeE<E>::ARR, t);  // b is r
                const double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z +
                                 (double)res.w * rr.w;
                const double part = block_sum128(s, shd);
                if (t == 0) cta_dot += part;
            }
        }
        __syncthreads();  // the stage just read is free for the copies issued next iteration
    }
    if (!ok) {
        // flag the timeout and let the copies in flight land before the CTA exits
        cpa_wait_all();
        if (t == 0) {
            if (err) atomicExch(err, 1);
            mbar_wait_bounded(&bar[j & 1], (unsigned)((j >> 1) & 1));
            if (next_issued) mbar_wait_bounded(&bar[(j & 1) ^ 1], (unsigned)(((j + 1) >> 1) & 1));
        }
        __syncthreads();
        return;
    }
    if constexpr (!RESTRICT) {
        if (dot.r) {  // one partial per CTA into the launch's reduction (a ticket per CTA, not per leaf)
            double tot = 0.0;
            constexpr int TK = DOTK == 1 ? 2 : 0;
            if (reduce_sum(cta_dot, dot.partials, &dot.st->ticket[TK], (int)blockIdx.x, G, tot)) {
                if (t == 0) {
                    PcgState* st = dot.st;
                    if constexpr (DOTK == 1) {
                        const float sigma = (float)tot;
                        st->sigma = sigma;
                        st->alpha = __fdiv_rn(st->rho, sigma);
                        st->first = 0;
                    } else {
                        const float rho_new = (float)tot;
                        st->rho_new = rho_new;
                        st->beta = st->first ? 0.f : __fdiv_rn(rho_new, st->rho);
                        st->rho = rho_new;
                    }
                    st->ticket[TK] = 0;
                }
            }
        }
    }
}

}  // namespace uaamg
