// poisson_kernels.cuh -- sm_100a kernels of the pressure-Poisson UAAMG-PCG.
//
// Arithmetic follows LaplacianApplySIMD::LightWeightApplier::operator()
// (SIMD_UAAMG/simd_vdb_poisson.cpp:755-1031) operation by operation with
// round-to-nearest intrinsics, so every per-voxel result is bit-identical to
// the reference's AVX2 lanes; the library is built with --fmad=false so the
// compiler cannot contract what the reference keeps separate.
//
// One CTA of 128 threads per 8^3 leaf; thread t owns voxels 4t..4t+3
// (x = t>>4, y = (t>>1)&7, z = 4*(t&1)+j), i.e. one 16-byte float4 of each
// leaf-dense array, so a warp reads 512 contiguous bytes per array.  The +-z
// neighbours inside a leaf come from the partner thread (t^1) by shuffle,
// +-x/+-y neighbours from the L1-resident own or neighbour leaf.
#pragma once
#include "common.cuh"

namespace uaamg {

#define FULLMASK 0xffffffffu

// Programmatic dependent launch: every solve kernel is launched with
// programmatic stream serialisation, waits for its predecessor's memory
// before touching anything (griddepcontrol.wait), and lets its successor
// start launching right away, which hides the kernel-to-kernel launch gap of
// the many small coarse-level kernels.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------------------
// lhs sources: what the stencil reads as "x" at any voxel.  Besides a stored
// vector they compute, on the fly, the result of a pass the reference stores
// and immediately re-reads (first sweep from zero, prolongation-add), which
// removes a kernel launch and a full pass per use.
struct SrcPlain {
    const float* x;
    __device__ __forceinline__ float4 get4(const DLevel&, int leaf, int t) const { return ld4(x, leaf, t); }
    __device__ __forceinline__ float get1(const DLevel&, int leaf, int off) const {
        return x[(long long)leaf * UAAMG_LEAF + off];
    }
};

// setGridToResultAfterFirstJacobi (.cpp:1435-1479): x1 = w * (invdiag * b)
struct SrcFirstJacobi {
    const float* b;
    float w;
    __device__ __forceinline__ float4 get4(const DLevel& L, int leaf, int t) const {
        float4 bb = ld4(b, leaf, t);
        float4 iv = (L.flags[leaf] & TRIM_DIAG) ? f4splat(L.def_invdiag) : ld4(L.invdiag, leaf, t);
        return make_float4(__fmul_rn(w, __fmul_rn(iv.x, bb.x)), __fmul_rn(w, __fmul_rn(iv.y, bb.y)),
                           __fmul_rn(w, __fmul_rn(iv.z, bb.z)), __fmul_rn(w, __fmul_rn(iv.w, bb.w)));
    }
    __device__ __forceinline__ float get1(const DLevel& L, int leaf, int off) const {
        long long i = (long long)leaf * UAAMG_LEAF + off;
        float iv = (L.flags[leaf] & TRIM_DIAG) ? L.def_invdiag : L.invdiag[i];
        return __fmul_rn(w, __fmul_rn(iv, b[i]));
    }
};

// setGridToResultAfterFirstSPAI0 (.cpp:1481-1517): x1 = spai0 * b.  Before the
// level's first spai0Apply the reference's SPAI0 grid is still empty, so the
// default is used everywhere (`ready` is the device flag that tracks it).
struct SrcFirstSpai0 {
    const float* b;
    const int* ready;
    __device__ __forceinline__ float4 get4(const DLevel& L, int leaf, int t) const {
        float4 bb = ld4(b, leaf, t);
        float4 s = (!*ready || (L.flags[leaf] & TRIM_SPAI0)) ? f4splat(L.def_spai0) : ld4(L.spai0, leaf, t);
        return make_float4(__fmul_rn(s.x, bb.x), __fmul_rn(s.y, bb.y), __fmul_rn(s.z, bb.z), __fmul_rn(s.w, bb.w));
    }
    __device__ __forceinline__ float get1(const DLevel& L, int leaf, int off) const {
        long long i = (long long)leaf * UAAMG_LEAF + off;
        float s = (!*ready || (L.flags[leaf] & TRIM_SPAI0)) ? L.def_spai0 : L.spai0[i];
        return __fmul_rn(s, b[i]);
    }
};

// setGridToResultAfterFirstRBGS<redFirst> red part (.cpp:1519-1566):
// updated colour = w_sor * (invdiag * b), other colour = 0
struct SrcFirstRbgs {
    const float* b;
    float wsor;
    int red_first;
    __device__ __forceinline__ float one(const DLevel& L, int leaf, int off, float bv, float iv) const {
        int par = ((off >> 6) + (off >> 3) + off) & 1;  // (x+y+z) & 1, 0 = red
        int upd = red_first ? (par == 0) : (par == 1);
        return upd ? __fmul_rn(wsor, __fmul_rn(iv, bv)) : 0.f;
    }
    __device__ __forceinline__ float4 get4(const DLevel& L, int leaf, int t) const {
        float4 bb = ld4(b, leaf, t);
        float4 iv = (L.flags[leaf] & TRIM_DIAG) ? f4splat(L.def_invdiag) : ld4(L.invdiag, leaf, t);
        int o = 4 * t;
        return make_float4(one(L, leaf, o, bb.x, iv.x), one(L, leaf, o + 1, bb.y, iv.y),
                           one(L, leaf, o + 2, bb.z, iv.z), one(L, leaf, o + 3, bb.w, iv.w));
    }
    __device__ __forceinline__ float get1(const DLevel& L, int leaf, int off) const {
        long long i = (long long)leaf * UAAMG_LEAF + off;
        float iv = (L.flags[leaf] & TRIM_DIAG) ? L.def_invdiag : L.invdiag[i];
        return one(L, leaf, off, b[i], iv);
    }
};

// prolongation<inplace_add=true> (.cpp:1686-1754): active fine voxels get
// x + alpha * x_coarse(parent voxel)
struct SrcProlong {
    const float* x;
    const float* xc;  // coarse-level vector
    float alpha;
    __device__ __forceinline__ float4 get4(const DLevel& L, int leaf, int t) const {
        float4 v = ld4(x, leaf, t);
        unsigned m = mask4(L.mask, leaf, t);
        if (!m) return v;
        int P = L.parent[leaf];
        int o = L.octant[leaf];
        int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
        int coff = (((o >> 2) & 1) * 4 + (X >> 1)) * 64 + (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4 + 2 * zh;
        float2 c = *reinterpret_cast<const float2*>(xc + (long long)P * UAAMG_LEAF + coff);
        float c0 = __fmul_rn(alpha, c.x), c1 = __fmul_rn(alpha, c.y);
        if (m & 1) v.x = __fadd_rn(v.x, c0);
        if (m & 2) v.y = __fadd_rn(v.y, c0);
        if (m & 4) v.z = __fadd_rn(v.z, c1);
        if (m & 8) v.w = __fadd_rn(v.w, c1);
        return v;
    }
    __device__ __forceinline__ float get1(const DLevel& L, int leaf, int off) const {
        float v = x[(long long)leaf * UAAMG_LEAF + off];
        if (!((L.mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull)) return v;
        int P = L.parent[leaf];
        int o = L.octant[leaf];
        int X = off >> 6, Y = (off >> 3) & 7, Z = off & 7;
        int coff = (((o >> 2) & 1) * 4 + (X >> 1)) * 64 + (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4 + (Z >> 1);
        return __fadd_rn(v, __fmul_rn(alpha, xc[(long long)P * UAAMG_LEAF + coff]));
    }
};

// source kinds, for kernels that pick one at run time (batched solves)
enum { S_PLAIN = 0, S_FIRST_JACOBI = 1, S_FIRST_SPAI0 = 2, S_FIRST_RBGS = 3, S_PROLONG = 4 };

// ---------------------------------------------------------------------------
// The 6-neighbour off-diagonal sum of one float4 (4 z-consecutive voxels):
// off = ((x+ c_x+ + x- c_x-) + (y+ c_y+ + y- c_y-)) + (z+ c_z+ + z- c_z-)
// with c_k- this voxel's minus-face entry and c_k+ the +k neighbour's.
// A thread's static stencil data: the leaf's flags, the neighbour leaves it
// reads and the face coefficients.  None of it changes during a solve, so the
// sweep kernels load it before waiting for the previous kernel.
struct PStatic {
    unsigned fl;
    int nxp, nxm, nyp, nym, nzm, nzp;  // neighbour leaves this thread reads (-1: absent or not needed)
    float4 cxp, cyp, cxm, cym, czo;    // c_x+, c_y+ (neighbour faces), c_x-, c_y-, c_z- of the 4 voxels
    float czp3;                        // c_z+ of the last voxel
};
__device__ __forceinline__ void stencil_static(const DLevel& L, int leaf, int t, PStatic& S) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const unsigned fl = L.flags[leaf];
    const int* nb = L.nbr + (long long)leaf * 6;
    const float df = L.def_face;
    const float4 dfv = f4splat(df);
    S.fl = fl;
    S.nxp = S.nxm = S.nyp = S.nym = S.nzm = S.nzp = -1;
    if (X < 7) {
        S.cxp = (fl & TRIM_X) ? dfv : ld4(L.cx, leaf, t + 16);
    } else {
        const int n = nb[1];
        S.nxp = n;
        S.cxp = n >= 0 ? ((L.flags[n] & TRIM_X) ? dfv : ld4(L.cx, n, t - 112)) : dfv;
    }
    if (X == 0) S.nxm = nb[0];
    if (Y < 7) {
        S.cyp = (fl & TRIM_Y) ? dfv : ld4(L.cy, leaf, t + 2);
    } else {
        const int n = nb[3];
        S.nyp = n;
        S.cyp = n >= 0 ? ((L.flags[n] & TRIM_Y) ? dfv : ld4(L.cy, n, t - 14)) : dfv;
    }
    if (Y == 0) S.nym = nb[2];
    S.cxm = (fl & TRIM_X) ? dfv : ld4(L.cx, leaf, t);
    S.cym = (fl & TRIM_Y) ? dfv : ld4(L.cy, leaf, t);
    S.czo = (fl & TRIM_Z) ? dfv : ld4(L.cz, leaf, t);
    S.czp3 = df;
    if (zh == 0) {
        S.nzm = nb[4];
    } else {
        const int n = nb[5];
        S.nzp = n;
        if (n >= 0) S.czp3 = (L.flags[n] & TRIM_Z) ? df : L.cz[(long long)n * UAAMG_LEAF + 4 * t - 4];
    }
}

// The 6-neighbour off-diagonal sum of one float4 (4 z-consecutive voxels):
// off = ((x+ c_x+ + x- c_x-) + (y+ c_y+ + y- c_y-)) + (z+ c_z+ + z- c_z-)
// with c_k- this voxel's minus-face entry and c_k+ the +k neighbour's.
// SHFL: the partner half of the thread's z-line (thread t ^ 1, same warp)
// supplies x and c_z at z = 4 / 3 by shuffle; without it they are loaded
// (the same values), for threads whose partner computes something else.
template <class Src, bool SHFL = true>
__device__ __forceinline__ void stencil_dyn(const DLevel& L, int leaf, int t, const Src& src, const PStatic& S,
                                            float4& xc, float4& off) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    xc = src.get4(L, leaf, t);
    float4 xp, xm, yp, ym;
    if (X < 7) xp = src.get4(L, leaf, t + 16);
    else xp = S.nxp >= 0 ? src.get4(L, S.nxp, t - 112) : f4zero();
    if (X > 0) xm = src.get4(L, leaf, t - 16);
    else xm = S.nxm >= 0 ? src.get4(L, S.nxm, t + 112) : f4zero();
    if (Y < 7) yp = src.get4(L, leaf, t + 2);
    else yp = S.nyp >= 0 ? src.get4(L, S.nyp, t - 14) : f4zero();
    if (Y > 0) ym = src.get4(L, leaf, t - 2);
    else ym = S.nym >= 0 ? src.get4(L, S.nym, t + 14) : f4zero();
    const int base = 4 * t;
    float px, pw, pcz;
    if constexpr (SHFL) {
        px = __shfl_xor_sync(FULLMASK, xc.x, 1);
        pw = __shfl_xor_sync(FULLMASK, xc.w, 1);
        pcz = __shfl_xor_sync(FULLMASK, S.czo.x, 1);
    } else if (zh == 0) {  // partner t + 1: z = 4..7
        px = src.get1(L, leaf, base + 4);
        pcz = (S.fl & TRIM_Z) ? L.def_face : L.cz[(long long)leaf * UAAMG_LEAF + base + 4];
        pw = 0.f;
    } else {  // partner t - 1: z = 0..3
        pw = src.get1(L, leaf, base - 1);
        px = pcz = 0.f;
    }
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = px;
        czp3 = pcz;
        zm0 = (S.nzm >= 0) ? src.get1(L, S.nzm, base + 7) : 0.f;
    } else {
        zm0 = pw;
        zp3 = (S.nzp >= 0) ? src.get1(L, S.nzp, base - 4) : 0.f;
        czp3 = S.czp3;
    }
    const float zp[4] = {xc.y, xc.z, xc.w, zp3};
    const float zm[4] = {zm0, xc.x, xc.y, xc.z};
    const float czp[4] = {S.czo.y, S.czo.z, S.czo.w, czp3};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float f1 = __fmul_rn(f4get(xp, j), f4get(S.cxp, j));
        float f2 = __fmul_rn(f4get(xm, j), f4get(S.cxm, j));
        float f3 = __fmul_rn(f4get(yp, j), f4get(S.cyp, j));
        float f4 = __fmul_rn(f4get(ym, j), f4get(S.cym, j));
        float f5 = __fmul_rn(zp[j], czp[j]);
        float f6 = __fmul_rn(zm[j], f4get(S.czo, j));
        f1 = __fadd_rn(f1, f2);
        f3 = __fadd_rn(f3, f4);
        f5 = __fadd_rn(f5, f6);
        f1 = __fadd_rn(f1, f3);
        f1 = __fadd_rn(f1, f5);
        f4set(off, j, f1);
    }
}

template <class Src>
__device__ __forceinline__ void stencil4(const DLevel& L, int leaf, int t, const Src& src, float4& xc,
                                         float4& off) {
    PStatic S;
    stencil_static(L, leaf, t, S);
    stencil_dyn(L, leaf, t, src, S, xc, off);
}

// ---------------------------------------------------------------------------
// deterministic block reductions (128 threads) and last-block finalisation
__device__ __forceinline__ double block_sum128(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULLMASK, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0) r = ((sh[0] + sh[1]) + sh[2]) + sh[3];
    __syncthreads();
    return r;  // valid in thread 0
}
__device__ __forceinline__ float nanmax(float a, float b) {
    if (isnan(a) || isnan(b)) return __int_as_float(0x7fc00000);
    return fmaxf(a, b);
}
__device__ __forceinline__ float block_max128(float v, float* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(FULLMASK, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    float r = 0;
    if (threadIdx.x == 0) r = nanmax(nanmax(sh[0], sh[1]), nanmax(sh[2], sh[3]));
    __syncthreads();
    return r;
}
// |v| with non-finite values propagated (grid_abs_max_op, openvdb_grid_math_op.h:4-43)
__device__ __forceinline__ float absprop(float v) { return isfinite(v) ? fabsf(v) : (isnan(v) ? v : INFINITY); }

// Deterministic two-level reduction over the CTAs of one launch.  A
// reduction buffer holds RED_TICKETS group tickets (RED_HEADER doubles, zero
// between reductions), then one partial per CTA slot, then one partial per
// group of red_group_size(count) consecutive slots.  Every CTA stores its
// partial and takes a ticket of its group; the CTA that completes a group
// combines the group's partials and takes a ticket of the reduction; the CTA
// that completes the last group combines the group partials.  The order of
// the combination depends only on `count` and the block size, so results are
// reproducible; no CTA reads more than a group's worth of partials, and the
// reduction's own ticket sees one atomic per group rather than per CTA.
constexpr int RED_TICKETS = 2048;
constexpr int RED_HEADER = RED_TICKETS / 2;
__host__ __device__ __forceinline__ int red_group_size(int count) {
    return count <= 256 * RED_TICKETS ? 256 : (count + RED_TICKETS - 1) / RED_TICKETS;
}
// doubles a reduction buffer over `count` slots needs
__host__ __device__ __forceinline__ size_t red_buffer_doubles(size_t count) {
    return (size_t)RED_HEADER + count + RED_TICKETS;
}
template <bool MAX>
__device__ __forceinline__ double red_combine(double a, double b) {
    return MAX ? (double)nanmax((float)a, (float)b) : a + b;
}
// block-wide combination for any multiple of 32 threads up to 256; valid in thread 0
template <bool MAX>
__device__ __forceinline__ double block_reduce_n(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_combine<MAX>(v, __shfl_down_sync(FULLMASK, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0) {
        r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = red_combine<MAX>(r, sh[w]);
    }
    __syncthreads();
    return r;
}
// Publishes this CTA's partial (valid in thread 0) into slot `slot` of a
// reduction over `count` slots; returns true in every thread of the CTA that
// completes it, whose thread 0 then holds the result in `total`.  That CTA
// resets `ticket` itself (the group tickets are reset here).
template <bool MAX>
__device__ __forceinline__ bool red_publish(double part, double* buf, unsigned* ticket, int slot, int count,
                                            double& total) {
    __shared__ double rsh[8];
    __shared__ int rflag;
    unsigned* gt = reinterpret_cast<unsigned*>(buf);
    double* slots = buf + RED_HEADER;
    double* groups = slots + count;
    const int gs = red_group_size(count);
    const int g = slot / gs;
    const int g0 = g * gs;
    const int gn = min(gs, count - g0);
    const int ng = (count + gs - 1) / gs;
    if (threadIdx.x == 0) {
        slots[slot] = part;
        __threadfence();
        rflag = (atomicAdd(&gt[g], 1u) == (unsigned)gn - 1);
    }
    __syncthreads();
    if (!rflag) return false;
    __threadfence();
    double acc = 0.0;
    for (int i = threadIdx.x; i < gn; i += blockDim.x) acc = red_combine<MAX>(acc, __ldcg(slots + g0 + i));
    acc = block_reduce_n<MAX>(acc, rsh);
    if (ng == 1) {
        if (threadIdx.x == 0) gt[g] = 0;
        total = acc;
        return true;
    }
    if (threadIdx.x == 0) {
        gt[g] = 0;
        groups[g] = acc;
        __threadfence();
        rflag = (atomicAdd(ticket, 1u) == (unsigned)ng - 1);
    }
    __syncthreads();
    if (!rflag) return false;
    __threadfence();
    acc = 0.0;
    for (int i = threadIdx.x; i < ng; i += blockDim.x) acc = red_combine<MAX>(acc, __ldcg(groups + i));
    total = block_reduce_n<MAX>(acc, rsh);
    return true;
}
__device__ __forceinline__ bool reduce_sum(double part, double* buf, unsigned* ticket, int slot, int count,
                                           double& total) {
    return red_publish<false>(part, buf, ticket, slot, count, total);
}
__device__ __forceinline__ bool reduce_max(double part, double* buf, unsigned* ticket, int slot, int count,
                                           float& total) {
    double t = 0.0;
    const bool done = red_publish<true>(part, buf, ticket, slot, count, t);
    total = (float)t;
    return done;
}

// ---------------------------------------------------------------------------
// One sweep of the applier in any mode.  out may alias the stored lhs only for
// the Gauss-Seidel modes with SrcPlain (in-place red/black passes).
enum { M_JACOBI = 0, M_RESIDUAL = 1, M_LAPLACIAN = 2, M_RED = 3, M_BLACK = 4, M_SPAI0 = 5 };

struct DotOut {            // optional fused z.r for the PCG (rho_new, beta)
    const float* r;        // second operand; nullptr = no dot
    double* partials;
    PcgState* st;
};

// A thread's static sweep data: the stencil's, the DOF bits and the
// diagonal terms the mode reads.
struct SStatic {
    PStatic P;
    unsigned m;
    float4 dg, iv, sp;
};
template <int MODE>
__device__ __forceinline__ void sweep_static(const DLevel& L, int leaf, int t, SStatic& S) {
    stencil_static(L, leaf, t, S.P);
    S.m = mask4(L.mask, leaf, t);
    const unsigned fl = S.P.fl;
    if (MODE != M_RED && MODE != M_BLACK)
        S.dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : ld4(L.diag, leaf, t);
    if (MODE == M_RED || MODE == M_BLACK || MODE == M_JACOBI)
        S.iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : ld4(L.invdiag, leaf, t);
    if (MODE == M_SPAI0) S.sp = (fl & TRIM_SPAI0) ? f4splat(L.def_spai0) : ld4(L.spai0, leaf, t);
}

template <int MODE, class Src, bool SHFL = true>
__device__ __forceinline__ float4 sweep_value_s(const DLevel& L, int leaf, int t, const Src& src, const float* b,
                                                float w, float wsor, float one_minus_wsor, const SStatic& S,
                                                float4& xc, unsigned& m) {
    float4 off;
    stencil_dyn<Src, SHFL>(L, leaf, t, src, S.P, xc, off);
    m = S.m;
    float4 res = f4zero();
    if (MODE == M_RED || MODE == M_BLACK) {
        const float4 bb = ld4(b, leaf, t);
        const float4 iv = S.iv;
        const int X = t >> 4, Y = (t >> 1) & 7;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int par = (X + Y + j) & 1;  // z = 4*zh + j has the parity of j
            bool upd = (MODE == M_RED) ? (par == 0) : (par == 1);
            float r = __fsub_rn(f4get(bb, j), f4get(off, j));
            r = __fmul_rn(r, f4get(iv, j));
            r = __fmul_rn(r, wsor);
            float v = __fmaf_rn(f4get(xc, j), one_minus_wsor, r);
            f4set(res, j, upd ? v : f4get(xc, j));
        }
    } else {
        const float4 dg = S.dg;
        if (MODE == M_LAPLACIAN) {
#pragma unroll
            for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        } else {
            const float4 bb = ld4(b, leaf, t);
            if (MODE == M_RESIDUAL) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
            } else if (MODE == M_JACOBI) {
                const float4 iv = S.iv;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
                    r = __fmul_rn(r, f4get(iv, j));
                    f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
                }
            } else {  // SPAI0
                const float4 sp = S.sp;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
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

template <int MODE, class Src>
__device__ __forceinline__ float4 sweep_value(const DLevel& L, int leaf, int t, const Src& src, const float* b,
                                              float w, float wsor, float one_minus_wsor, float4& xc, unsigned& m) {
    SStatic S;
    sweep_static<MODE>(L, leaf, t, S);
    return sweep_value_s<MODE>(L, leaf, t, src, b, w, wsor, one_minus_wsor, S, xc, m);
}

// One leaf of a sweep (CTA = leaf of a level with `count` leaves, the slot
// range of the fused dot's partials).
// WAIT: static data first, then griddepcontrol.wait (false when the caller
// has waited already).  gate: a flag written by earlier kernels; the CTA does
// nothing when it is zero (batched solves: the instance has stopped).  A gate
// only goes from 1 to 0 while a solve runs (it is set again only before the
// first sweep), so a zero read before the wait is final and skips the static
// loads; the read after the wait decides.
template <int MODE, class Src, bool WAIT = false>
__device__ __forceinline__ void sweep_leaf(const DLevel& L, int leaf, int count, const Src& src, const float* b,
                                           float* out, float w, float wsor, float one_minus_wsor, const DotOut& dot,
                                           int* spai0_ready, const unsigned* gate = nullptr) {
    const int t = threadIdx.x;
    if (gate && !*gate) return;
    SStatic S;
    sweep_static<MODE>(L, leaf, t, S);
    if (WAIT) {
        griddep_wait();
        griddep_launch();
    }
    if (gate && !*gate) return;
    float4 xc;
    unsigned m;
    float4 res = sweep_value_s<MODE>(L, leaf, t, src, b, w, wsor, one_minus_wsor, S, xc, m);
    st4(out, leaf, t, res);
    if (MODE == M_SPAI0 && spai0_ready && leaf == 0 && t == 0) *spai0_ready = 1;
    if (dot.r) {  // rho_new = z . r (levelDot), then beta and rho (PCG lines 13-15)
        __shared__ double shd[4];
        float4 rr = ld4(dot.r, leaf, t);
        double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z + (double)res.w * rr.w;
        double part = block_sum128(s, shd);
        double tot;
        if (reduce_sum(part, dot.partials, &dot.st->ticket[0], leaf, count, tot)) {
            if (t == 0) {
                PcgState* st = dot.st;
                float rho_new = (float)tot;
                st->rho_new = rho_new;
                st->beta = st->first ? 0.f : __fdiv_rn(rho_new, st->rho);
                st->rho = rho_new;
                st->ticket[0] = 0;
            }
        }
    }
}

template <int MODE, class Src>
__global__ void __launch_bounds__(128) k_sweep(DLevel L, Src src, const float* b, float* out, float w, float wsor,
                                               float one_minus_wsor, DotOut dot, int* spai0_ready) {
    sweep_leaf<MODE, Src, true>(L, blockIdx.x, gridDim.x, src, b, out, w, wsor, one_minus_wsor, dot, spai0_ready);
}

// ---------------------------------------------------------------------------
// Two Jacobi sweeps in one launch: out = J_wb(J_wa(src)).  The second sweep at a
// voxel reads the first sweep's result at its six neighbours, so a CTA computes
// the first sweep for its leaf and for the face layers of its six neighbours
// (the values the neighbouring CTAs compute too, from the same inputs with the
// same operations: bit-identical), keeps them in a 10^3 shared cube and then
// does the second sweep on its leaf.  Results are those of two k_sweep
// launches.  src must not read `out` (neighbouring CTAs still read src).
// Threads: 0-127 the leaf's 4-voxel groups; 128-191 the groups of the -x, +x,
// -y, +y neighbours' face planes (x or y = 7 or 0 in that leaf); 192-319 one
// group of the -z / +z neighbours per (x, y) of the face, holding the voxel at
// z = 7 / 0.  The face groups compute without warp shuffles (their partner
// thread is not their z-line's other half).
#define SW2_THREADS 320
__device__ __forceinline__ int sw2_idx(int X, int Y, int Z) { return ((X + 1) * 10 + (Y + 1)) * 10 + (Z + 1); }
template <class Src>
__global__ void __launch_bounds__(SW2_THREADS, 2) k_sweep2(DLevel L, Src src, const float* b, float* out, float wa,
                                                           float wb) {
    __shared__ float cube[1000];
    const int t = threadIdx.x;
    const int leaf = blockIdx.x;
    const int* nb = L.nbr + (long long)leaf * 6;
    // the group this thread computes in the first sweep: leaf gl, group gt; cube origin (cX, cY, cZ0)
    int gl = leaf, gt = t, cX = t >> 4, cY = (t >> 1) & 7, cZ0 = 4 * (t & 1), zlane = -1;
    if (t >= 128 && t < 192) {
        const int h = t - 128, face = h >> 4, u = (h >> 1) & 7, zh = h & 1;
        gl = nb[face];
        cZ0 = 4 * zh;
        if (face < 2) {
            const int Xn = face == 0 ? 7 : 0;
            gt = (Xn << 4) | (u << 1) | zh;
            cX = face == 0 ? -1 : 8;
            cY = u;
        } else {
            const int Yn = face == 2 ? 7 : 0;
            gt = (u << 4) | (Yn << 1) | zh;
            cX = u;
            cY = face == 2 ? -1 : 8;
        }
    } else if (t >= 192) {
        const int h = t - 192, zf = h >> 6, X = (h >> 3) & 7, Y = h & 7;
        gl = nb[4 + zf];             // -z neighbour (its z = 4..7 group), then +z (its z = 0..3 group)
        gt = (X << 4) | (Y << 1) | (zf ? 0 : 1);
        cX = X;
        cY = Y;
        zlane = zf ? 0 : 3;          // the voxel at cube z = 8 / -1
        cZ0 = zf ? 8 : -4;
    }
    SStatic S;
    if (gl >= 0) sweep_static<M_JACOBI>(L, gl, gt, S);
    griddep_wait();
    griddep_launch();
    float4 T = f4zero(), xc;
    unsigned m = 0;
    if (t < 128) T = sweep_value_s<M_JACOBI, Src, true>(L, leaf, t, src, b, wa, 0.f, 1.f, S, xc, m);
    else if (gl >= 0) T = sweep_value_s<M_JACOBI, Src, false>(L, gl, gt, src, b, wa, 0.f, 1.f, S, xc, m);
    if (zlane < 0) {
        const int base = sw2_idx(cX, cY, cZ0);
        cube[base] = T.x;
        cube[base + 1] = T.y;
        cube[base + 2] = T.z;
        cube[base + 3] = T.w;
    } else {
        cube[sw2_idx(cX, cY, cZ0 + zlane)] = f4get(T, zlane);
    }
    __syncthreads();
    if (t >= 128) return;
    // second sweep on the leaf: stencil_dyn's operations with the first sweep's values from the cube
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1, Z0 = 4 * zh;
    const float pcz = __shfl_xor_sync(FULLMASK, S.P.czo.x, 1);
    const float czp3 = zh == 0 ? pcz : S.P.czp3;
    const float czp[4] = {S.P.czo.y, S.P.czo.z, S.P.czo.w, czp3};
    float4 off;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int Z = Z0 + j;
        float f1 = __fmul_rn(cube[sw2_idx(X + 1, Y, Z)], f4get(S.P.cxp, j));
        float f2 = __fmul_rn(cube[sw2_idx(X - 1, Y, Z)], f4get(S.P.cxm, j));
        float f3 = __fmul_rn(cube[sw2_idx(X, Y + 1, Z)], f4get(S.P.cyp, j));
        float f4 = __fmul_rn(cube[sw2_idx(X, Y - 1, Z)], f4get(S.P.cym, j));
        float f5 = __fmul_rn(cube[sw2_idx(X, Y, Z + 1)], czp[j]);
        float f6 = __fmul_rn(cube[sw2_idx(X, Y, Z - 1)], f4get(S.P.czo, j));
        f1 = __fadd_rn(f1, f2);
        f3 = __fadd_rn(f3, f4);
        f5 = __fadd_rn(f5, f6);
        f1 = __fadd_rn(f1, f3);
        f1 = __fadd_rn(f1, f5);
        f4set(off, j, f1);
    }
    const float4 bb = ld4(b, leaf, t);
    float4 res;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(T, j), f4get(S.dg, j), f4get(off, j)));
        r = __fmul_rn(r, f4get(S.iv, j));
        f4set(res, j, __fmaf_rn(wb, r, f4get(T, j)));
    }
    if (!(m & 1)) res.x = 0.f;
    if (!(m & 2)) res.y = 0.f;
    if (!(m & 4)) res.z = 0.f;
    if (!(m & 8)) res.w = 0.f;
    st4(out, leaf, t, res);
}

// out = value of a source (materialise a first sweep or a prolongation)
template <class Src>
// (grid-stride over the leaves: any grid size; large levels launch a few
// CTAs per SM rather than one per leaf, which the CTA launch rate would bound)
__global__ void __launch_bounds__(128) k_materialize(DLevel L, Src src, float* out) {
    griddep_wait();
    griddep_launch();
    const int t = threadIdx.x;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x) {
        float4 v = src.get4(L, leaf, t);
        unsigned m = mask4(L.mask, leaf, t);
        if (!(m & 1)) v.x = 0.f;
        if (!(m & 2)) v.y = 0.f;
        if (!(m & 4)) v.z = 0.f;
        if (!(m & 8)) v.w = 0.f;
        st4(out, leaf, t, v);
    }
}

// residual (RESID) or plain values, restricted to the parent level:
// coarse = 0.125 * sum of the active fine values of the 2x2x2 block (.cpp:1624-1684)
template <bool RESID, bool WAIT = false>
__device__ __forceinline__ void restrict_leaf(const DLevel& L, int leaf, const float* x, const float* b,
                                              float* coarse, const unsigned* gate = nullptr) {
    __shared__ float rs[UAAMG_LEAF];
    const int t = threadIdx.x;
    if (gate && !*gate) return;  // final when zero (see sweep_leaf)
    SStatic S;
    if (RESID) sweep_static<M_RESIDUAL>(L, leaf, t, S);
    if (WAIT) {
        griddep_wait();
        griddep_launch();
    }
    if (gate && !*gate) return;
    float4 r;
    if (RESID) {
        float4 xc;
        unsigned m;
        r = sweep_value_s<M_RESIDUAL>(L, leaf, t, SrcPlain{x}, b, 0.f, 0.f, 0.f, S, xc, m);
    } else {
        r = ld4(x, leaf, t);
    }
    reinterpret_cast<float4*>(rs)[t] = r;
    __syncthreads();
    if (t < 64) {
        const int i = t >> 4, j = (t >> 2) & 3, k = t & 3;
        const uint64_t* mk = L.mask + (long long)leaf * 8;
        float s = 0.f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    int fo = ((2 * i + ii) << 6) | ((2 * j + jj) << 3) | (2 * k + kk);
                    if ((mk[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                }
        const int o = L.octant[leaf];
        const int coff = ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + j) << 3) | ((o & 1) * 4 + k);
        coarse[(long long)L.parent[leaf] * UAAMG_LEAF + coff] = __fmul_rn(s, 0.125f);
    }
}
template <bool RESID>
__global__ void __launch_bounds__(128) k_restrict(DLevel L, const float* x, const float* b, float* coarse) {
    restrict_leaf<RESID, true>(L, blockIdx.x, x, b, coarse);
}

// ---------------------------------------------------------------------------
// Bulk-async staged sweeps.  One CTA per leaf: thread 0 issues
// cp.async.bulk copies (2 KB each) of the leaf's vectors and of the
// coefficient arrays that are stored for it (trimmed leaves hold the default
// and are not read) into shared memory, completing on an mbarrier; while they
// are in flight the boundary threads load the halo values of the six
// neighbour leaves; the stencil then reads the leaf from shared memory.
// Same arithmetic as sweep_value, so results are bit-identical.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (each try_wait blocks briefly).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < (1 << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// What a staged sweep needs in shared memory.
struct Staged {
    float* x;
    float* b;
    float* d;   // diag
    float* i;   // 1/diag or spai0
    float* cx;
    float* cy;
    float* cz;
};

// The bulk copies of one leaf (thread 0), in two parts: the coefficient
// arrays, which do not change during a solve, are issued before the wait for
// the previous kernel; x and b (and the SPAI0 array, built during a solve)
// after it.  The barrier expects all bytes from the first part on.
template <int MODE>
struct StageSet {
    bool b, d, i, cx, cy, cz;
    __device__ __forceinline__ StageSet(unsigned fl) {
        b = (MODE != M_LAPLACIAN);
        d = (MODE != M_RED && MODE != M_BLACK) && !(fl & TRIM_DIAG);
        i = (MODE == M_JACOBI || MODE == M_RED || MODE == M_BLACK) ? !(fl & TRIM_DIAG)
            : (MODE == M_SPAI0 ? !(fl & TRIM_SPAI0) : false);
        cx = !(fl & TRIM_X);
        cy = !(fl & TRIM_Y);
        cz = !(fl & TRIM_Z);
    }
    __device__ __forceinline__ unsigned bytes() const {
        return 2048u * (1u + (b ? 1u : 0u) + (d ? 1u : 0u) + (i ? 1u : 0u) + (cx ? 1u : 0u) + (cy ? 1u : 0u) +
                        (cz ? 1u : 0u));
    }
};
template <int MODE>
__device__ __forceinline__ void stage_issue_static(const DLevel& L, int leaf, const StageSet<MODE>& Q, const Staged& S,
                                                   uint64_t* bar) {
    mbar_expect_tx(bar, Q.bytes());
    const long long o = (long long)leaf * UAAMG_LEAF;
    if (Q.d) bulk_g2s(S.d, L.diag + o, 2048u, bar);
    if (Q.i && MODE != M_SPAI0) bulk_g2s(S.i, L.invdiag + o, 2048u, bar);
    if (Q.cx) bulk_g2s(S.cx, L.cx + o, 2048u, bar);
    if (Q.cy) bulk_g2s(S.cy, L.cy + o, 2048u, bar);
    if (Q.cz) bulk_g2s(S.cz, L.cz + o, 2048u, bar);
}
template <int MODE>
__device__ __forceinline__ void stage_issue_dyn(const DLevel& L, int leaf, const StageSet<MODE>& Q, const float* x,
                                                const float* b, const Staged& S, uint64_t* bar) {
    const long long o = (long long)leaf * UAAMG_LEAF;
    bulk_g2s(S.x, x + o, 2048u, bar);
    if (Q.b) bulk_g2s(S.b, b + o, 2048u, bar);
    if (Q.i && MODE == M_SPAI0) bulk_g2s(S.i, L.spai0 + o, 2048u, bar);
}

__device__ __forceinline__ float4 s4(const float* s, int t) { return reinterpret_cast<const float4*>(s)[t]; }

// Staged stencil: own-leaf values from shared memory, halo values (already
// loaded into registers by the caller) for the neighbour leaves.
template <int MODE>
__device__ __forceinline__ float4 staged_value(const DLevel& L, int leaf, int t, unsigned fl, const Staged& S,
                                               const float4& hxp, const float4& hxm, const float4& hyp,
                                               const float4& hym, const float4& hcxp, const float4& hcyp, float hz,
                                               float hcz, float w, float wsor, float one_minus_wsor, float4& xc,
                                               unsigned& m) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const float df = L.def_face;
    const float4 dfv = f4splat(df);
    xc = s4(S.x, t);
    const float4 xp = (X < 7) ? s4(S.x, t + 16) : hxp;
    const float4 xm = (X > 0) ? s4(S.x, t - 16) : hxm;
    const float4 yp = (Y < 7) ? s4(S.x, t + 2) : hyp;
    const float4 ym = (Y > 0) ? s4(S.x, t - 2) : hym;
    const float4 cxp = (X < 7) ? ((fl & TRIM_X) ? dfv : s4(S.cx, t + 16)) : hcxp;
    const float4 cyp = (Y < 7) ? ((fl & TRIM_Y) ? dfv : s4(S.cy, t + 2)) : hcyp;
    const float4 cxm = (fl & TRIM_X) ? dfv : s4(S.cx, t);
    const float4 cym = (fl & TRIM_Y) ? dfv : s4(S.cy, t);
    const float4 czo = (fl & TRIM_Z) ? dfv : s4(S.cz, t);
    // z neighbours inside the leaf from shared memory, across the leaf face from the halo
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = S.x[4 * t + 4];
        czp3 = (fl & TRIM_Z) ? df : S.cz[4 * t + 4];
        zm0 = hz;
    } else {
        zm0 = S.x[4 * t - 1];
        zp3 = hz;
        czp3 = hcz;
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
    m = mask4(L.mask, leaf, t);
    float4 res = f4zero();
    if (MODE == M_RED || MODE == M_BLACK) {
        const float4 bb = s4(S.b, t);
        const float4 iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : s4(S.i, t);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int par = (X + Y + j) & 1;
            bool upd = (MODE == M_RED) ? (par == 0) : (par == 1);
            float r = __fsub_rn(f4get(bb, j), f4get(off, j));
            r = __fmul_rn(r, f4get(iv, j));
            r = __fmul_rn(r, wsor);
            float v = __fmaf_rn(f4get(xc, j), one_minus_wsor, r);
            f4set(res, j, upd ? v : f4get(xc, j));
        }
    } else {
        const float4 dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : s4(S.d, t);
        if (MODE == M_LAPLACIAN) {
#pragma unroll
            for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        } else {
            const float4 bb = s4(S.b, t);
            if (MODE == M_RESIDUAL) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
            } else if (MODE == M_JACOBI) {
                const float4 iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : s4(S.i, t);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
                    r = __fmul_rn(r, f4get(iv, j));
                    f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
                }
            } else {  // SPAI0
                const float4 sp = (fl & TRIM_SPAI0) ? f4splat(L.def_spai0) : s4(S.i, t);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
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

// Halo loads of one thread, in two parts: the neighbour leaves and their
// face coefficients (static, before the wait) and the neighbours' x values
// (after it, while the bulk copies are in flight).
struct HaloNb {
    int xp, xm, yp, ym, z;  // neighbour leaf whose face this thread reads, or -1
};
__device__ __forceinline__ void staged_halo_static(const DLevel& L, int leaf, int t, HaloNb& H, float4& hcxp,
                                                   float4& hcyp, float& hcz) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const int* nb = L.nbr + (long long)leaf * 6;
    const float df = L.def_face;
    hcxp = hcyp = f4splat(df);
    hcz = df;
    H.xp = (X == 7) ? nb[1] : -1;
    H.xm = (X == 0) ? nb[0] : -1;
    H.yp = (Y == 7) ? nb[3] : -1;
    H.ym = (Y == 0) ? nb[2] : -1;
    H.z = (zh == 0) ? nb[4] : nb[5];
    // a trimmed leaf stores its default coefficients (finalize_leaf), so the
    // face values load without testing the neighbour's flags
    if (H.xp >= 0) hcxp = ld4(L.cx, H.xp, t - 112);
    if (H.yp >= 0) hcyp = ld4(L.cy, H.yp, t - 14);
    if (zh == 1 && H.z >= 0) hcz = L.cz[(long long)H.z * UAAMG_LEAF + 4 * t - 4];
}
__device__ __forceinline__ void staged_halo_dyn(const float* x, int t, const HaloNb& H, float4& hxp, float4& hxm,
                                                float4& hyp, float4& hym, float& hz) {
    hxp = (H.xp >= 0) ? ld4(x, H.xp, t - 112) : f4zero();
    hxm = (H.xm >= 0) ? ld4(x, H.xm, t + 112) : f4zero();
    hyp = (H.yp >= 0) ? ld4(x, H.yp, t - 14) : f4zero();
    hym = (H.ym >= 0) ? ld4(x, H.ym, t + 14) : f4zero();
    hz = 0.f;
    if (H.z >= 0) hz = x[(long long)H.z * UAAMG_LEAF + ((t & 1) ? 4 * t - 4 : 4 * t + 7)];
}

// minimum resident CTAs per SM the one-leaf staged kernels are compiled for
// (1: no register cap; higher values spill)
#ifndef STAGED_MINB
#define STAGED_MINB 1
#endif
#define STAGED_SMEM_DECL                                                         \
    __shared__ __align__(128) float sm_x[UAAMG_LEAF], sm_b[UAAMG_LEAF], sm_d[UAAMG_LEAF], \
        sm_i[UAAMG_LEAF], sm_cx[UAAMG_LEAF], sm_cy[UAAMG_LEAF], sm_cz[UAAMG_LEAF];      \
    __shared__ __align__(8) uint64_t sm_bar;                                     \
    const Staged S{sm_x, sm_b, sm_d, sm_i, sm_cx, sm_cy, sm_cz};

// Stage + halo + wait; false if the wait timed out (error flagged).  Waits
// for the previous kernel (programmatic dependent launch) after the static
// part.
template <int MODE>
__device__ __forceinline__ bool staged_prologue(const DLevel& L, int leaf, int t, const float* x, const float* b,
                                                const Staged& S, uint64_t* bar, unsigned& fl, float4& hxp,
                                                float4& hxm, float4& hyp, float4& hym, float4& hcxp, float4& hcyp,
                                                float& hz, float& hcz, int* err) {
    fl = L.flags[leaf];
    const StageSet<MODE> Q(fl);
    HaloNb H;
    staged_halo_static(L, leaf, t, H, hcxp, hcyp, hcz);
    if (t == 0) mbar_init(bar, 1);
    __syncthreads();
    if (t == 0) stage_issue_static<MODE>(L, leaf, Q, S, bar);
    griddep_wait();
    griddep_launch();
    if (t == 0) stage_issue_dyn<MODE>(L, leaf, Q, x, b, S, bar);
    staged_halo_dyn(x, t, H, hxp, hxm, hyp, hym, hz);
    // every thread of the CTA agrees on the outcome, so no thread leaves a
    // later barrier short-handed
    const bool ok = __syncthreads_and(mbar_wait_bounded(bar, 0) ? 1 : 0) != 0;
    if (!ok) {
        if (t == 0 && err) atomicExch(err, 1);
        mbar_wait_bounded(bar, 0);  // let the copies in flight land before the CTA exits
    }
    return ok;
}

template <int MODE>
__global__ void __launch_bounds__(128, STAGED_MINB) k_sweep_staged(DLevel L, const float* x, const float* b, float* out, float w,
                                                      float wsor, float one_minus_wsor, DotOut dot, int* err) {
    STAGED_SMEM_DECL
    const int leaf = blockIdx.x, t = threadIdx.x;
    unsigned fl;
    float4 hxp, hxm, hyp, hym, hcxp, hcyp;
    float hz, hcz;
    const bool ok = staged_prologue<MODE>(L, leaf, t, x, b, S, &sm_bar, fl, hxp, hxm, hyp, hym, hcxp, hcyp, hz, hcz, err);
    float4 xc, res = f4zero();
    unsigned m;
    if (ok) {
        res = staged_value<MODE>(L, leaf, t, fl, S, hxp, hxm, hyp, hym, hcxp, hcyp, hz, hcz, w, wsor,
                                 one_minus_wsor, xc, m);
        st4(out, leaf, t, res);
    }
    if (dot.r) {  // rho_new = z . r, then beta and rho (PCG lines 13-15)
        __shared__ double shd[4];
        float4 rr = ok ? s4(S.b, t) : f4zero();  // b of this sweep is r
        double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z + (double)res.w * rr.w;
        double part = block_sum128(s, shd);
        double tot;
        if (reduce_sum(part, dot.partials, &dot.st->ticket[0], blockIdx.x, gridDim.x, tot)) {
            if (t == 0) {
                PcgState* st = dot.st;
                float rho_new = (float)tot;
                st->rho_new = rho_new;
                st->beta = st->first ? 0.f : __fdiv_rn(rho_new, st->rho);
                st->rho = rho_new;
                st->ticket[0] = 0;
            }
        }
    }
}

// residual + restriction with the fine leaf staged
__global__ void __launch_bounds__(128, STAGED_MINB) k_restrict_staged(DLevel L, const float* x, const float* b, float* coarse,
                                                         int* err) {
    STAGED_SMEM_DECL
    const int leaf = blockIdx.x, t = threadIdx.x;
    unsigned fl;
    float4 hxp, hxm, hyp, hym, hcxp, hcyp;
    float hz, hcz;
    const bool ok =
        staged_prologue<M_RESIDUAL>(L, leaf, t, x, b, S, &sm_bar, fl, hxp, hxm, hyp, hym, hcxp, hcyp, hz, hcz, err);
    if (!ok) return;
    float4 xc;
    unsigned m;
    float4 r = staged_value<M_RESIDUAL>(L, leaf, t, fl, S, hxp, hxm, hyp, hym, hcxp, hcyp, hz, hcz, 0.f, 0.f, 0.f, xc, m);
    __syncthreads();  // every thread has read sm_x before it is reused for the residuals
    reinterpret_cast<float4*>(sm_x)[t] = r;
    __syncthreads();
    if (t < 64) {
        const int i = t >> 4, j = (t >> 2) & 3, k = t & 3;
        const uint64_t* mk = L.mask + (long long)leaf * 8;
        float s = 0.f;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    int fo = ((2 * i + ii) << 6) | ((2 * j + jj) << 3) | (2 * k + kk);
                    if ((mk[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, sm_x[fo]);
                }
        const int o = L.octant[leaf];
        const int coff = ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + j) << 3) | ((o & 1) * 4 + k);
        coarse[(long long)L.parent[leaf] * UAAMG_LEAF + coff] = __fmul_rn(s, 0.125f);
    }
}

// ---------------------------------------------------------------------------
// PCG vector kernels (PoissonSolver::solveMultigridPCG, .cpp:2155-2226)
__global__ void __launch_bounds__(128) k_mask_vec(DLevel L, float* v) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, t = threadIdx.x;
    unsigned m = mask4(L.mask, leaf, t);
    if (m == 0xF) return;
    float4 a = ld4(v, leaf, t);
    if (!(m & 1)) a.x = 0.f;
    if (!(m & 2)) a.y = 0.f;
    if (!(m & 4)) a.z = 0.f;
    if (!(m & 8)) a.w = 0.f;
    st4(v, leaf, t, a);
}

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use, unsigned v) {
    if (use) cudaGraphSetConditional(h, v);
}

// The PCG steps as per-leaf bodies (CTA = leaf of level 0 with `count`
// leaves): the single-solve kernels below run them with leaf = blockIdx.x,
// batched solves with the leaf of the CTA's (instance, leaf) entry.

// lines 2-3: r = b - A x; nu = |r|_inf; numax = tol * nu
__device__ __forceinline__ void pcg_init_leaf(const DLevel& L, int leaf, int count, const float* x, const float* b,
                                              float* r, double* partials, PcgState* st,
                                              cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ float shf[4];
    const int t = threadIdx.x;
    float4 xc;
    unsigned m;
    float4 res = sweep_value<M_RESIDUAL>(L, leaf, t, SrcPlain{x}, b, 0.f, 0.f, 0.f, xc, m);
    st4(r, leaf, t, res);
    float a = nanmax(nanmax(absprop(res.x), absprop(res.y)), nanmax(absprop(res.z), absprop(res.w)));
    float part = block_max128(a, shf);
    float nu;
    if (reduce_max(part, partials, &st->ticket[1], leaf, count, nu)) {
        if (t == 0) {
            st->nu = nu;
            st->nu_old = nu;
            st->numax = __fmul_rn(st->tol, nu);
            st->iter = 0;
            st->first = 1;
            st->iterations_taken = 0;
            st->alpha = 0.f;
            st->beta = 0.f;
            int status = PCG_RUNNING;
            if (nu <= st->numax) status = PCG_SUCCESS;
            else if (st->max_iter <= 0) status = PCG_FAILED_DIVERGED;  // no iteration: x untouched
            st->status = status;
            st->ticket[1] = 0;
            set_cond(cond, use_cond, status == PCG_RUNNING ? 1u : 0u);
        }
    }
}
__global__ void __launch_bounds__(128) k_pcg_init(DLevel L, const float* x, const float* b, float* r,
                                                  double* partials, PcgState* st,
                                                  cudaGraphConditionalHandle cond, int use_cond) {
    griddep_wait();
    griddep_launch();
    pcg_init_leaf(L, blockIdx.x, gridDim.x, x, b, r, partials, st, cond, use_cond);
}

// x += alpha_prev * p_prev (line 16, skipped in the first iteration); p = z + beta p (line 16)
__device__ __forceinline__ void pcg_update_p_leaf(int leaf, const float* z, float* p, float* x, const PcgState* st) {
    const int t = threadIdx.x;
    const float beta = st->beta, alpha = st->alpha;
    const int first = st->first;
    float4 zz = ld4(z, leaf, t), pp = ld4(p, leaf, t);
    if (!first) {
        float4 xx = ld4(x, leaf, t);
        xx.x = __fmaf_rn(alpha, pp.x, xx.x);
        xx.y = __fmaf_rn(alpha, pp.y, xx.y);
        xx.z = __fmaf_rn(alpha, pp.z, xx.z);
        xx.w = __fmaf_rn(alpha, pp.w, xx.w);
        st4(x, leaf, t, xx);
    }
    pp.x = __fmaf_rn(beta, pp.x, zz.x);
    pp.y = __fmaf_rn(beta, pp.y, zz.y);
    pp.z = __fmaf_rn(beta, pp.z, zz.z);
    pp.w = __fmaf_rn(beta, pp.w, zz.w);
    st4(p, leaf, t, pp);
}
__global__ void __launch_bounds__(128) k_pcg_update_p(DLevel L, const float* z, float* p, float* x,
                                                      const PcgState* st) {  // grid-stride over the leaves
    griddep_wait();
    griddep_launch();
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x) pcg_update_p_leaf(leaf, z, p, x, st);
}

// lines 6-7: q = A p; sigma = p.q; alpha = rho / sigma
__device__ __forceinline__ void pcg_Ap_leaf(const DLevel& L, int leaf, int count, const float* p, float* q,
                                            double* partials, PcgState* st) {
    __shared__ double shd[4];
    const int t = threadIdx.x;
    float4 xc;
    unsigned m;
    float4 res = sweep_value<M_LAPLACIAN>(L, leaf, t, SrcPlain{p}, nullptr, 0.f, 0.f, 0.f, xc, m);
    st4(q, leaf, t, res);
    double s = (double)xc.x * res.x + (double)xc.y * res.y + (double)xc.z * res.z + (double)xc.w * res.w;
    double part = block_sum128(s, shd);
    double tot;
    if (reduce_sum(part, partials, &st->ticket[2], leaf, count, tot)) {
        if (t == 0) {
            float sigma = (float)tot;
            st->sigma = sigma;
            st->alpha = __fdiv_rn(st->rho, sigma);
            st->first = 0;
            st->ticket[2] = 0;
        }
    }
}
__global__ void __launch_bounds__(128) k_pcg_Ap(DLevel L, const float* p, float* q, double* partials, PcgState* st) {
    griddep_wait();
    griddep_launch();
    pcg_Ap_leaf(L, blockIdx.x, gridDim.x, p, q, partials, st);
}

// lines 8-12: r -= alpha q; nu = |r|_inf; convergence / divergence test
// the thread's 4 voxels of r -= alpha q; returns their |r|_inf
__device__ __forceinline__ float pcg_update_r_apply(int leaf, const float* q, float* r, float na) {
    const int t = threadIdx.x;
    float4 qq = ld4(q, leaf, t), rr = ld4(r, leaf, t);
    rr.x = __fmaf_rn(na, qq.x, rr.x);
    rr.y = __fmaf_rn(na, qq.y, rr.y);
    rr.z = __fmaf_rn(na, qq.z, rr.z);
    rr.w = __fmaf_rn(na, qq.w, rr.w);
    st4(r, leaf, t, rr);
    return nanmax(nanmax(absprop(rr.x), absprop(rr.y)), nanmax(absprop(rr.z), absprop(rr.w)));
}
__device__ __forceinline__ void pcg_update_r_finish(float nu, PcgState* st, cudaGraphConditionalHandle cond,
                                                    int use_cond);
__device__ __forceinline__ void pcg_update_r_leaf(int leaf, int count, const float* q, float* r, double* partials,
                                                  PcgState* st, cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ float shf[4];
    const int t = threadIdx.x;
    const float a = pcg_update_r_apply(leaf, q, r, -st->alpha);
    float part = block_max128(a, shf);
    float nu;
    if (reduce_max(part, partials, &st->ticket[3], leaf, count, nu)) {
        if (t == 0) pcg_update_r_finish(nu, st, cond, use_cond);
    }
}
// nu, the convergence / divergence test and the loop condition (thread 0 of
// the CTA that completes the |r|_inf reduction)
__device__ __forceinline__ void pcg_update_r_finish(float nu, PcgState* st, cudaGraphConditionalHandle cond,
                                                    int use_cond) {
    const int k = st->iter;
    st->nu_old = st->nu;
    st->nu = nu;
    int status = PCG_RUNNING;
    if (nu <= st->numax) {
        status = PCG_SUCCESS;
        st->iterations_taken = k;
    } else if (nu > st->nu_old && k > 3) {
        status = PCG_FAILED_DIVERGED;
        st->iterations_taken = k;
    } else if (k + 1 >= st->max_iter) {
        status = PCG_FAILED_MAXITER;
        st->iterations_taken = st->max_iter;
    }
    st->iter = k + 1;
    st->status = status;
    st->ticket[3] = 0;
    set_cond(cond, use_cond, status == PCG_RUNNING ? 1u : 0u);
}
// grid-stride over the leaves, one |r|_inf partial per CTA (a maximum: the
// result does not depend on the grid)
__global__ void __launch_bounds__(128) k_pcg_update_r(DLevel L, const float* q, float* r, double* partials,
                                                      PcgState* st, cudaGraphConditionalHandle cond, int use_cond) {
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    const float na = -st->alpha;
    float a = 0.f;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x) a = nanmax(a, pcg_update_r_apply(leaf, q, r, na));
    const float part = block_max128(a, shf);
    float nu;
    if (reduce_max(part, partials, &st->ticket[3], blockIdx.x, gridDim.x, nu)) {
        if (threadIdx.x == 0) pcg_update_r_finish(nu, st, cond, use_cond);
    }
}

// line 10 on success, and line 16 of the last iteration when max_iter is reached
__device__ __forceinline__ bool pcg_finish_applies(const PcgState* st) {
    const int s = st->status;
    if (s != PCG_SUCCESS && s != PCG_FAILED_MAXITER) return false;
    if (st->iterations_taken == 0 && st->iter == 0) return false;  // converged before the loop
    return true;
}
__device__ __forceinline__ float4 pcg_finish_value(int leaf, const float* p, const float* x, const PcgState* st,
                                                   bool apply) {
    const int t = threadIdx.x;
    float4 xx = ld4(x, leaf, t);
    if (!apply) return xx;
    const float alpha = st->alpha;
    float4 pp = ld4(p, leaf, t);
    xx.x = __fmaf_rn(alpha, pp.x, xx.x);
    xx.y = __fmaf_rn(alpha, pp.y, xx.y);
    xx.z = __fmaf_rn(alpha, pp.z, xx.z);
    xx.w = __fmaf_rn(alpha, pp.w, xx.w);
    return xx;
}
__global__ void __launch_bounds__(128) k_pcg_finish(DLevel L, const float* p, float* x, const PcgState* st) {
    griddep_wait();
    griddep_launch();
    if (!pcg_finish_applies(st)) return;
    st4(x, blockIdx.x, threadIdx.x, pcg_finish_value(blockIdx.x, p, x, st, true));
}

// z.r over the DOF (levelDot) and the beta/rho step, for a hierarchy whose
// level 0 is the coarsest (no sweep is available to carry the dot)
__device__ __forceinline__ void dot_rho_leaf(const DLevel& L, int leaf, int count, const float* z, const float* r,
                                             double* partials, PcgState* st) {
    __shared__ double shd[4];
    const int t = threadIdx.x;
    float4 a = ld4(z, leaf, t), c = ld4(r, leaf, t);
    unsigned m = mask4(L.mask, leaf, t);
    double s = 0;
    if (m & 1) s += (double)a.x * c.x;
    if (m & 2) s += (double)a.y * c.y;
    if (m & 4) s += (double)a.z * c.z;
    if (m & 8) s += (double)a.w * c.w;
    double part = block_sum128(s, shd);
    double tot;
    if (reduce_sum(part, partials, &st->ticket[0], leaf, count, tot)) {
        if (t == 0) {
            float rho_new = (float)tot;
            st->rho_new = rho_new;
            st->beta = st->first ? 0.f : __fdiv_rn(rho_new, st->rho);
            st->rho = rho_new;
            st->ticket[0] = 0;
        }
    }
}

// v *= DOF mask (inputs of the PCG are zero off the DOF)
__device__ __forceinline__ float4 masked4(const DLevel& L, int leaf, float4 a) {
    unsigned m = mask4(L.mask, leaf, threadIdx.x);
    if (!(m & 1)) a.x = 0.f;
    if (!(m & 2)) a.y = 0.f;
    if (!(m & 4)) a.z = 0.f;
    if (!(m & 8)) a.w = 0.f;
    return a;
}

// r = b - A x and |r|_inf (residualApply + levelAbsMax), result in out[0]
__global__ void __launch_bounds__(128) k_residual_absmax(DLevel L, const float* x, const float* b, float* r,
                                                         double* partials, unsigned* ticket, float* out) {
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    const int leaf = blockIdx.x, t = threadIdx.x;
    float4 xc;
    unsigned m;
    float4 res = sweep_value<M_RESIDUAL>(L, leaf, t, SrcPlain{x}, b, 0.f, 0.f, 0.f, xc, m);
    st4(r, leaf, t, res);
    float a = nanmax(nanmax(absprop(res.x), absprop(res.y)), nanmax(absprop(res.z), absprop(res.w)));
    float part = block_max128(a, shf);
    float nu;
    if (reduce_max(part, partials, ticket, blockIdx.x, gridDim.x, nu)) {
        if (t == 0) {
            *out = nu;
            *ticket = 0;
        }
    }
}

// |v|_inf over a level (levelAbsMax), result in out[0]
__global__ void __launch_bounds__(128) k_absmax(DLevel L, const float* v, double* partials, unsigned* ticket,
                                                float* out) {
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    const int leaf = blockIdx.x, t = threadIdx.x;
    float4 a = ld4(v, leaf, t);
    unsigned m = mask4(L.mask, leaf, t);
    float mx = 0.f;
    if (m & 1) mx = nanmax(mx, absprop(a.x));
    if (m & 2) mx = nanmax(mx, absprop(a.y));
    if (m & 4) mx = nanmax(mx, absprop(a.z));
    if (m & 8) mx = nanmax(mx, absprop(a.w));
    float part = block_max128(mx, shf);
    float r;
    if (reduce_max(part, partials, ticket, blockIdx.x, gridDim.x, r)) {
        if (t == 0) {
            *out = r;
            *ticket = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Coarsest level: restatement of Eigen::ConjugateGradient<SparseMatrix<float>>
// (diagonal preconditioner, tolerance FLT_EPSILON, maxIterations 10, zero
// guess), one CTA, rows in DOF order with up to six off-diagonal entries.
struct DCoarsest {
    int n;
    const int* dof_slot;   // [n] leaf*512 + offset
    const float* diag;     // [n]
    const float* invd;     // [n] 1/diag (1 where diag == 0)
    const int* col;        // [n][6] (-1 = none)
    const float* val;      // [n][6]
};

// Thread-block shapes of the coarsest CG, by system size (rows per thread,
// threads): 512 threads with 2 or 4 rows each up to 2048 DOF, 1024 threads
// with 4 rows above; the rows' entries stay in registers.  The batched solve
// and the cluster bottom-cycle kernel use the same shape for the same size, so
// their results match the single solve bit for bit.
#define CG_MAX_DOF 4096
__host__ __device__ __forceinline__ int coarsest_class(int n) { return n <= 1024 ? 0 : (n <= 2048 ? 1 : 2); }

// Block reductions in one barrier: warps reduce with shfl_down into lane 0,
// lane 0 of each warp publishes its partial, and every thread then adds the
// NT/32 partials in one fixed pairwise order from shared memory (broadcast
// float4 reads), so all threads hold bit-identical scalars (the CG's control
// flow depends on them).  buf: 16-byte aligned, [2][32] floats for the pair
// form.
__device__ __forceinline__ float cg_warp_partial(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULLMASK, v, o);
    return v;  // the warp's sum in lane 0
}
template <int NW>  // 8, 16 or 32 partials
__device__ __forceinline__ float cg_tree_sum(const float* buf) {
    static_assert(NW == 8 || NW == 16 || NW == 32, "partials");
    float s[NW / 4];
#pragma unroll
    for (int q = 0; q < NW / 4; ++q) {
        const float4 v = reinterpret_cast<const float4*>(buf)[q];
        s[q] = (v.x + v.y) + (v.z + v.w);
    }
#pragma unroll
    for (int step = 1; step < NW / 4; step *= 2)
#pragma unroll
        for (int q = 0; q + step < NW / 4; q += 2 * step) s[q] += s[q + step];
    return s[0];
}
template <int NT>
__device__ __forceinline__ float cg_block_sum(float v, float* buf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = cg_warp_partial(v);
    if (lane == 0) buf[w] = v;
    __syncthreads();
    return cg_tree_sum<NT / 32>(buf);
}
template <int NT>
__device__ __forceinline__ float2 cg_block_sum2(float a, float b, float* buf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(FULLMASK, a, o);
        b += __shfl_down_sync(FULLMASK, b, o);
    }
    if (lane == 0) { buf[w] = a; buf[32 + w] = b; }
    __syncthreads();
    return make_float2(cg_tree_sum<NT / 32>(buf), cg_tree_sum<NT / 32>(buf + 32));
}

// ROWS rows per thread in a block of NT threads (row i = tid + k * NT); the
// matrix rows stay in registers for the whole solve (CgRows), so a kernel that
// solves the same system twice loads them once.  Three barriers per CG
// iteration.  (Publishing z and the old p with the second reduction, so that
// each thread forms its neighbours' new p itself and one barrier goes, doubles
// the shared-memory reads in flight and pushes the rows out of registers:
// measured 1.6 times slower.)
template <int ROWS>
struct CgRows {
    float dg[ROWS], iv[ROWS], val[ROWS][6];
    unsigned col[ROWS][6];  // shared-memory address of the column's p (the zero slot when absent)
    int slot[ROWS];
};
// ps: NT * ROWS + 4 floats in shared memory; slot NT * ROWS holds 0
template <int ROWS, int NT>
__device__ __forceinline__ void cg_rows_load(const DCoarsest& C, CgRows<ROWS>& M, const float* ps) {
    const int tid = threadIdx.x, n = C.n;
    const unsigned base = (unsigned)__cvta_generic_to_shared(ps);
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
        const int i = tid + k * NT;
        const bool ok = i < n;
        M.slot[k] = ok ? C.dof_slot[i] : -1;
        M.dg[k] = ok ? C.diag[i] : 0.f;
        M.iv[k] = ok ? C.invd[i] : 0.f;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const int c = ok ? C.col[i * 6 + e] : -1;
            M.col[k][e] = base + 4u * (unsigned)(c >= 0 ? c : NT * ROWS);
            M.val[k][e] = c >= 0 ? C.val[i * 6 + e] : 0.f;
        }
    }
}
__device__ __forceinline__ float lds_f32(unsigned addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}
// out[slot] = the 10-step CG solution for the rhs gathered from rhs[slot]
// (every thread of the NT-thread block takes part); ps: NT * ROWS + 4 floats,
// red: 16-byte aligned.  The products and sums use fused multiply-adds (the
// coarsest solve's summation order is this kernel's own; the unfused
// reference solve differs from it by rounding only).
template <int ROWS, int NT>
__device__ __forceinline__ void cg_rows_solve(const CgRows<ROWS>& M, const float* rhs, float* out, float* ps,
                                              float (*red)[64]) {
    const int tid = threadIdx.x;
    float x[ROWS], r[ROWS], p[ROWS], z[ROWS];
    float bb = 0.f;
    if (tid == 0) ps[NT * ROWS] = 0.f;  // the absent columns' slot (published by the first barrier)
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
        x[k] = 0.f;
        r[k] = M.slot[k] >= 0 ? rhs[M.slot[k]] : 0.f;
        bb = __fmaf_rn(r[k], r[k], bb);
    }
    int rb = 0;
    const float rhsNorm2 = cg_block_sum<NT>(bb, red[rb]);
    rb = rb == 2 ? 0 : rb + 1;
    const float threshold = fmaxf(__fmul_rn(__fmul_rn(FLT_EPSILON, FLT_EPSILON), rhsNorm2), FLT_MIN);
    // rhsNorm2 == 0 -> x = 0; residualNorm2 (== rhsNorm2 for x = 0) < threshold -> x = 0
    if (rhsNorm2 != 0.f && !(rhsNorm2 < threshold)) {
        float an = 0.f;
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            p[k] = __fmul_rn(M.iv[k], r[k]);
            an = __fmaf_rn(r[k], p[k], an);
        }
        float absNew = cg_block_sum<NT>(an, red[rb]);
        rb = rb == 2 ? 0 : rb + 1;
        for (int it = 0; it < 10; ++it) {
#pragma unroll
            for (int k = 0; k < ROWS; ++k) ps[tid + k * NT] = p[k];
            __syncthreads();
            float pt = 0.f, tq[ROWS];
#pragma unroll
            for (int k = 0; k < ROWS; ++k) {
                float s = __fmul_rn(M.dg[k], p[k]);
#pragma unroll
                for (int e = 0; e < 6; ++e) s = __fmaf_rn(M.val[k][e], lds_f32(M.col[k][e]), s);
                tq[k] = s;
                pt = __fmaf_rn(p[k], s, pt);
            }
            const float alpha = __fdiv_rn(absNew, cg_block_sum<NT>(pt, red[rb]));
            rb = rb == 2 ? 0 : rb + 1;
            float rr = 0.f, rz = 0.f;
#pragma unroll
            for (int k = 0; k < ROWS; ++k) {
                x[k] = __fmaf_rn(alpha, p[k], x[k]);
                r[k] = __fmaf_rn(-alpha, tq[k], r[k]);
                z[k] = __fmul_rn(M.iv[k], r[k]);
                rr = __fmaf_rn(r[k], r[k], rr);
                rz = __fmaf_rn(r[k], z[k], rz);
            }
            const float2 s2 = cg_block_sum2<NT>(rr, rz, red[rb]);
            rb = rb == 2 ? 0 : rb + 1;
            if (s2.x < threshold) break;
            const float absOld = absNew;
            absNew = s2.y;
            const float beta = __fdiv_rn(absNew, absOld);
#pragma unroll
            for (int k = 0; k < ROWS; ++k) p[k] = __fmaf_rn(beta, p[k], z[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < ROWS; ++k)
        if (M.slot[k] >= 0) out[M.slot[k]] = x[k];
}

// The whole coarsest solve.  WAIT: the body itself waits for the previous
// kernel (griddepcontrol) after loading the matrix, which does not change
// during a solve; false when the caller has waited already.
template <int ROWS, int NT, bool WAIT>
__device__ __forceinline__ void coarsest_cg_body(const DCoarsest& C, const float* rhs, float* out, float* ps,
                                                 float (*red)[64]) {
    CgRows<ROWS> M;
    cg_rows_load<ROWS, NT>(C, M, ps);
    if (WAIT) {
        griddep_wait();
        griddep_launch();
    }
    cg_rows_solve<ROWS, NT>(M, rhs, out, ps, red);
}

template <int ROWS, int NT>
__global__ void __launch_bounds__(NT, 1) k_coarsest_cg(DCoarsest C, const float* rhs, float* out) {
    __shared__ float ps[NT * ROWS + 4];
    __shared__ __align__(16) float red[3][64];  // rotating reduction buffers (no reuse within 2 barriers)
    coarsest_cg_body<ROWS, NT, true>(C, rhs, out, ps, red);
}

}  // namespace uaamg
