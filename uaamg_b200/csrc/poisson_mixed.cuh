// poisson_mixed.cuh -- the mixed-precision form of the pressure UAAMG-PCG.
//
// The preconditioner's hierarchy -- every level's coefficients (diag, 1/diag,
// c_x, c_y, c_z) and every mu-cycle vector -- is stored in 16-bit floats (FP16
// or BF16); the arithmetic is FP32 and follows the same operation sequence as
// the FP32 kernels (muCyclePreconditioner with scheduled relaxed Jacobi,
// simd_vdb_poisson.cpp:1844-1977).  The outer CG stays FP32 on the FP32
// level-0 operator with FP64 dot accumulation (the kernels of
// poisson_kernels.cuh), recomputes the true residual every 25 iterations, and
// the coarsest level is solved directly in FP64 (a dense inverse built once).
// Reading 2-byte instead of 4-byte values halves the traffic of the sweeps
// that bound the solve on large domains.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "poisson_kernels.cuh"
#include "staged_pipe.cuh"

namespace uaamg {

// ---------------------------------------------------------------------------
// 16-bit storage: 4 values (8 bytes) per thread, converted with round to nearest
template <typename T> struct H16;
template <> struct H16<__half> {
    static __device__ __forceinline__ float2 to2(unsigned u) {
        __half2 h = *reinterpret_cast<__half2*>(&u);
        return __half22float2(h);
    }
    static __device__ __forceinline__ unsigned from2(float a, float b) {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<unsigned*>(&h);
    }
    static __device__ __forceinline__ float to1(__half v) { return __half2float(v); }
    static __device__ __forceinline__ float bits1(unsigned short u) { return __half2float(__ushort_as_half(u)); }
    static __device__ __forceinline__ __half from1(float v) { return __float2half_rn(v); }
};
template <> struct H16<__nv_bfloat16> {
    static __device__ __forceinline__ float2 to2(unsigned u) {
        __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
        return __bfloat1622float2(h);
    }
    static __device__ __forceinline__ unsigned from2(float a, float b) {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<unsigned*>(&h);
    }
    static __device__ __forceinline__ float to1(__nv_bfloat16 v) { return __bfloat162float(v); }
    static __device__ __forceinline__ float bits1(unsigned short u) {
        return __bfloat162float(__ushort_as_bfloat16(u));
    }
    static __device__ __forceinline__ __nv_bfloat16 from1(float v) { return __float2bfloat16_rn(v); }
};

template <typename T>
__device__ __forceinline__ float4 ldh4(const T* p, long long leaf, int t) {
    const uint2 u = reinterpret_cast<const uint2*>(p)[leaf * UAAMG_LEAF4 + t];
    const float2 a = H16<T>::to2(u.x), b = H16<T>::to2(u.y);
    return make_float4(a.x, a.y, b.x, b.y);
}
template <typename T>
__device__ __forceinline__ float ldh1(const T* p, long long i) {
    return H16<T>::to1(p[i]);
}
template <typename T>
__device__ __forceinline__ void sth4(T* p, long long leaf, int t, float4 v) {
    uint2 u;
    u.x = H16<T>::from2(v.x, v.y);
    u.y = H16<T>::from2(v.z, v.w);
    reinterpret_cast<uint2*>(p)[leaf * UAAMG_LEAF4 + t] = u;
}
__device__ __forceinline__ void stv4(float* p, long long leaf, int t, float4 v) { st4(p, leaf, t, v); }
template <typename T>
__device__ __forceinline__ void stv4(T* p, long long leaf, int t, float4 v) { sth4(p, leaf, t, v); }

// A level of the 16-bit hierarchy: the FP32 level's topology and flags with
// 16-bit coefficient arrays; trimmed leaves read the FP32 defaults.
template <typename T>
struct MLevel {
    int nl;
    const uint64_t* mask;
    const int* nbr;
    const int* parent;
    const uint8_t* octant;
    const uint32_t* flags;
    const T* diag;
    const T* invdiag;
    const T* cx;
    const T* cy;
    const T* cz;
    float def_diag, def_face, def_invdiag;
    // storage scales (powers of two, so scaling adds no rounding): the
    // coefficients and the rhs are stored divided by cs, 1/diag multiplied by
    // cs, which keeps every stored value near 1 whatever dt/dx^2 is (FP16
    // overflows at 65504, and ghost-fluid diagonals reach 300 dt/dx^2)
    float cs, ics;
};
__device__ __forceinline__ float4 f4scale(float4 v, float s) {
    return make_float4(__fmul_rn(v.x, s), __fmul_rn(v.y, s), __fmul_rn(v.z, s), __fmul_rn(v.w, s));
}
// coefficient (scale cs), 1/diag (scale ics) and rhs (scale cs) loads
template <typename T>
__device__ __forceinline__ float4 ldc4(const MLevel<T>& L, const T* a, long long leaf, int t) {
    return f4scale(ldh4(a, leaf, t), L.cs);
}
template <typename T>
__device__ __forceinline__ float ldc1(const MLevel<T>& L, const T* a, long long i) {
    return __fmul_rn(ldh1(a, i), L.cs);
}
template <typename T>
__device__ __forceinline__ float4 ldi4(const MLevel<T>& L, long long leaf, int t) {
    return f4scale(ldh4(L.invdiag, leaf, t), L.ics);
}

// storage and level traits of the pipelined staged kernels (staged_pipe.cuh)
template <typename T>
struct PipeE16 {
    static constexpr unsigned ARR = UAAMG_LEAF * 2;
    static __device__ __forceinline__ float4 s4(const unsigned char* a, int t) {
        const uint2 u = reinterpret_cast<const uint2*>(a)[t];
        const float2 p = H16<T>::to2(u.x), q = H16<T>::to2(u.y);
        return make_float4(p.x, p.y, q.x, q.y);
    }
    static __device__ __forceinline__ float s1(const unsigned char* a, int i) {
        return H16<T>::bits1(reinterpret_cast<const unsigned short*>(a)[i]);
    }
    static __device__ __forceinline__ float bits1(unsigned short u) { return H16<T>::bits1(u); }
    static __device__ __forceinline__ float4 g4(const T* p, long long leaf, int t) { return ldh4(p, leaf, t); }
    static __device__ __forceinline__ float g1(const T* p, long long i) { return ldh1(p, i); }
    static __device__ __forceinline__ void st(T* p, long long leaf, int t, float4 v) { sth4(p, leaf, t, v); }
    static __device__ __forceinline__ void st1(T* p, long long i, float v) { p[i] = H16<T>::from1(v); }
};
template <> struct PipeE<__half> : PipeE16<__half> {};
template <> struct PipeE<__nv_bfloat16> : PipeE16<__nv_bfloat16> {};
template <typename T>
struct PipeLv<MLevel<T>> {  // computes in stored units (staged_pipe.cuh)
    using E = T;
    static constexpr bool SCALED = true;
    static __device__ __forceinline__ float def_face(const MLevel<T>& L) { return __fmul_rn(L.def_face, L.ics); }
    static __device__ __forceinline__ float def_diag(const MLevel<T>& L) { return __fmul_rn(L.def_diag, L.ics); }
    static __device__ __forceinline__ float def_invdiag(const MLevel<T>& L) { return __fmul_rn(L.def_invdiag, L.cs); }
};

// lhs sources (16-bit vectors)
template <typename T>
struct MSrcPlain {
    const T* x;
    __device__ __forceinline__ float4 get4(const MLevel<T>&, int leaf, int t) const { return ldh4(x, leaf, t); }
    __device__ __forceinline__ float get1(const MLevel<T>&, int leaf, int off) const {
        return ldh1(x, (long long)leaf * UAAMG_LEAF + off);
    }
};
// setGridToResultAfterFirstJacobi: x1 = w * (invdiag * b)
template <typename T>
struct MSrcFirstJacobi {
    const T* b;
    float w;
    __device__ __forceinline__ float4 get4(const MLevel<T>& L, int leaf, int t) const {
        const float4 bb = ldc4(L, b, leaf, t);
        const float4 iv = (L.flags[leaf] & TRIM_DIAG) ? f4splat(L.def_invdiag) : ldi4(L, leaf, t);
        return make_float4(__fmul_rn(w, __fmul_rn(iv.x, bb.x)), __fmul_rn(w, __fmul_rn(iv.y, bb.y)),
                           __fmul_rn(w, __fmul_rn(iv.z, bb.z)), __fmul_rn(w, __fmul_rn(iv.w, bb.w)));
    }
    __device__ __forceinline__ float get1(const MLevel<T>& L, int leaf, int off) const {
        const long long i = (long long)leaf * UAAMG_LEAF + off;
        const float iv = (L.flags[leaf] & TRIM_DIAG) ? L.def_invdiag : __fmul_rn(ldh1(L.invdiag, i), L.ics);
        return __fmul_rn(w, __fmul_rn(iv, ldc1(L, b, i)));
    }
};
// prolongation<true>: x + coarse parent value at active voxels
template <typename T>
struct MSrcProlong {
    const T* x;
    const T* xc;
    __device__ __forceinline__ float4 get4(const MLevel<T>& L, int leaf, int t) const {
        float4 v = ldh4(x, leaf, t);
        const unsigned m = mask4(L.mask, leaf, t);
        if (!m) return v;
        const int P = L.parent[leaf];
        const int o = L.octant[leaf];
        const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
        const int coff =
            (((o >> 2) & 1) * 4 + (X >> 1)) * 64 + (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4 + 2 * zh;
        const long long cb = (long long)P * UAAMG_LEAF + coff;
        const float c0 = ldh1(xc, cb), c1 = ldh1(xc, cb + 1);
        if (m & 1) v.x = __fadd_rn(v.x, c0);
        if (m & 2) v.y = __fadd_rn(v.y, c0);
        if (m & 4) v.z = __fadd_rn(v.z, c1);
        if (m & 8) v.w = __fadd_rn(v.w, c1);
        return v;
    }
    __device__ __forceinline__ float get1(const MLevel<T>& L, int leaf, int off) const {
        float v = ldh1(x, (long long)leaf * UAAMG_LEAF + off);
        if (!((L.mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull)) return v;
        const int P = L.parent[leaf];
        const int o = L.octant[leaf];
        const int X = off >> 6, Y = (off >> 3) & 7, Z = off & 7;
        const int coff =
            (((o >> 2) & 1) * 4 + (X >> 1)) * 64 + (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4 + (Z >> 1);
        return __fadd_rn(v, ldh1(xc, (long long)P * UAAMG_LEAF + coff));
    }
};

// The 7-point stencil of one float4 (same operation order as stencil4)
template <typename T, class Src>
__device__ __forceinline__ void mstencil4(const MLevel<T>& L, int leaf, int t, const Src& src, float4& xc,
                                          float4& off) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const unsigned fl = L.flags[leaf];
    const int* nb = L.nbr + (long long)leaf * 6;
    const float df = L.def_face;
    const float4 dfv = f4splat(df);
    xc = src.get4(L, leaf, t);
    float4 xp, xm, yp, ym, cxp, cyp;
    if (X < 7) {
        xp = src.get4(L, leaf, t + 16);
        cxp = (fl & TRIM_X) ? dfv : ldc4(L, L.cx, leaf, t + 16);
    } else {
        const int n = nb[1];
        if (n >= 0) {
            xp = src.get4(L, n, t - 112);
            cxp = (L.flags[n] & TRIM_X) ? dfv : ldc4(L, L.cx, n, t - 112);
        } else {
            xp = f4zero();
            cxp = dfv;
        }
    }
    if (X > 0) {
        xm = src.get4(L, leaf, t - 16);
    } else {
        const int n = nb[0];
        xm = (n >= 0) ? src.get4(L, n, t + 112) : f4zero();
    }
    if (Y < 7) {
        yp = src.get4(L, leaf, t + 2);
        cyp = (fl & TRIM_Y) ? dfv : ldc4(L, L.cy, leaf, t + 2);
    } else {
        const int n = nb[3];
        if (n >= 0) {
            yp = src.get4(L, n, t - 14);
            cyp = (L.flags[n] & TRIM_Y) ? dfv : ldc4(L, L.cy, n, t - 14);
        } else {
            yp = f4zero();
            cyp = dfv;
        }
    }
    if (Y > 0) {
        ym = src.get4(L, leaf, t - 2);
    } else {
        const int n = nb[2];
        ym = (n >= 0) ? src.get4(L, n, t + 14) : f4zero();
    }
    const float4 cxm = (fl & TRIM_X) ? dfv : ldc4(L, L.cx, leaf, t);
    const float4 cym = (fl & TRIM_Y) ? dfv : ldc4(L, L.cy, leaf, t);
    const float4 czo = (fl & TRIM_Z) ? dfv : ldc4(L, L.cz, leaf, t);
    const float px = __shfl_xor_sync(FULLMASK, xc.x, 1);
    const float pw = __shfl_xor_sync(FULLMASK, xc.w, 1);
    const float pcz = __shfl_xor_sync(FULLMASK, czo.x, 1);
    const int base = 4 * t;
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = px;
        czp3 = pcz;
        const int n = nb[4];
        zm0 = (n >= 0) ? src.get1(L, n, base + 7) : 0.f;
    } else {
        zm0 = pw;
        const int n = nb[5];
        if (n >= 0) {
            zp3 = src.get1(L, n, base - 4);
            czp3 = (L.flags[n] & TRIM_Z) ? df : ldc1(L, L.cz, (long long)n * UAAMG_LEAF + base - 4);
        } else {
            zp3 = 0.f;
            czp3 = df;
        }
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

// weighted Jacobi (RESID false) or residual (RESID true) at the thread's voxels
template <bool RESID, typename T, class Src>
__device__ __forceinline__ float4 mjacobi_value(const MLevel<T>& L, int leaf, int t, const Src& src, const T* b,
                                                float w) {
    float4 xc, off;
    mstencil4(L, leaf, t, src, xc, off);
    const unsigned m = mask4(L.mask, leaf, t);
    const unsigned fl = L.flags[leaf];
    const float4 dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : ldc4(L, L.diag, leaf, t);
    const float4 bb = ldc4(L, b, leaf, t);
    float4 res;
    if (RESID) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
    } else {
        const float4 iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : ldi4(L, leaf, t);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
            r = __fmul_rn(r, f4get(iv, j));
            f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
        }
    }
    if (!(m & 1)) res.x = 0.f;
    if (!(m & 2)) res.y = 0.f;
    if (!(m & 4)) res.z = 0.f;
    if (!(m & 8)) res.w = 0.f;
    return res;
}

// One Jacobi sweep of a 16-bit level; out is 16-bit, or FP32 for the last
// sweep of level 0 (the preconditioned residual z of the outer CG, with the
// fused z.r of PCG lines 13-15 when dot.r is set).
template <typename T, typename TOut, class Src>
__global__ void __launch_bounds__(128) k_msweep(MLevel<T> L, Src src, const T* b, TOut* out, float w, DotOut dot,
                                                const float* zscale) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, t = threadIdx.x;
    float4 res = mjacobi_value<false>(L, leaf, t, src, b, w);
    if (zscale) res = f4scale(res, *zscale);  // level 0: z = sigma * (solution of the normalised system)
    stv4(out, leaf, t, res);
    if (dot.r) {
        __shared__ double shd[4];
        const float4 rr = ld4(dot.r, leaf, t);
        const double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z + (double)res.w * rr.w;
        const double part = block_sum128(s, shd);
        double tot;
        if (reduce_sum(part, dot.partials, &dot.st->ticket[0], blockIdx.x, gridDim.x, tot)) {
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

// residual + restriction into the next level's 16-bit rhs
template <typename T>
__global__ void __launch_bounds__(128) k_mrestrict(MLevel<T> L, const T* x, const T* b, T* coarse, float coarse_ics) {
    griddep_wait();
    griddep_launch();
    __shared__ float rs[UAAMG_LEAF];
    const int leaf = blockIdx.x, t = threadIdx.x;
    reinterpret_cast<float4*>(rs)[t] = mjacobi_value<true>(L, leaf, t, MSrcPlain<T>{x}, b, 0.f);
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
                    const int fo = ((2 * i + ii) << 6) | ((2 * j + jj) << 3) | (2 * k + kk);
                    if ((mk[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                }
        const int o = L.octant[leaf];
        const int coff = ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + j) << 3) | ((o & 1) * 4 + k);
        coarse[(long long)L.parent[leaf] * UAAMG_LEAF + coff] =
            H16<T>::from1(__fmul_rn(__fmul_rn(s, 0.125f), coarse_ics));
    }
}

// FP32 -> 16-bit copy of a level vector (the outer CG's residual into the
// preconditioner's rhs)
// The CG residual into the preconditioner's level-0 rhs, normalised: sigma =
// 2^(ilogb(|r|_inf) - ilogb(default diagonal)) makes the level-0 solution
// O(1); the rhs is stored divided by sigma * cs.  sigma goes to *sigma_out
// for the last level-0 sweep.
template <typename T>
__global__ void __launch_bounds__(128) k_mto16(MLevel<T> L, const float* in, T* out, const PcgState* st,
                                               float* sigma_out) {
    griddep_wait();
    griddep_launch();
    const float nu = st->nu;
    float sigma = 1.0f;
    if (nu > 0.f && isfinite(nu)) sigma = ldexpf(1.0f, ilogbf(nu) - ilogbf(L.def_diag));
    if (blockIdx.x == 0 && threadIdx.x == 0) *sigma_out = sigma;
    const float sc = __fmul_rn(L.ics, 1.0f / sigma);  // exact: powers of two
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x)  // grid-stride
        sth4(out, leaf, threadIdx.x, f4scale(ld4(in, leaf, threadIdx.x), sc));
}

// 16-bit -> FP32 copy of a level vector (one-level hierarchies: z)
template <typename T>
__global__ void __launch_bounds__(128) k_mfrom16(const T* in, float* out, const float* sigma) {
    griddep_wait();
    griddep_launch();
    st4(out, blockIdx.x, threadIdx.x, f4scale(ldh4(in, blockIdx.x, threadIdx.x), *sigma));
}

// FP32 -> 16-bit copy of a coefficient array (hierarchy construction)
template <typename T>
__global__ void __launch_bounds__(256) k_mconvert(const float* in, T* out, long long n4, float scale) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n4) return;
    const float4 v = f4scale(reinterpret_cast<const float4*>(in)[i], scale);
    uint2 u;
    u.x = H16<T>::from2(v.x, v.y);
    u.y = H16<T>::from2(v.z, v.w);
    reinterpret_cast<uint2*>(out)[i] = u;
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Staged 16-bit sweeps for large levels: the leaf's 16-bit arrays (1 KB each)
// are bulk-copied into shared memory (the coefficient arrays before the wait
// for the previous kernel, x and b after it) while each thread loads its
// halo values from the neighbour leaves; a thread then computes its 4
// z-consecutive voxels from shared memory with the operation sequence of
// mstencil4 / mjacobi_value, so a staged sweep gives the same values as
// k_msweep with a plain source.
struct MStaged {
    uint16_t* x;
    uint16_t* b;
    uint16_t* d;
    uint16_t* i;
    uint16_t* cx;
    uint16_t* cy;
    uint16_t* cz;
};
template <typename T>
__device__ __forceinline__ float4 msh4(const uint16_t* s, int t) {
    const uint2 u = reinterpret_cast<const uint2*>(s)[t];
    const float2 a = H16<T>::to2(u.x), b = H16<T>::to2(u.y);
    return make_float4(a.x, a.y, b.x, b.y);
}
template <typename T>
__device__ __forceinline__ float msh1(const uint16_t* s, int i) {
    return H16<T>::bits1(s[i]);
}

struct MStageSet {
    bool d, i, cx, cy, cz;
    __device__ __forceinline__ MStageSet(unsigned fl) {
        d = i = !(fl & TRIM_DIAG);
        cx = !(fl & TRIM_X);
        cy = !(fl & TRIM_Y);
        cz = !(fl & TRIM_Z);
    }
};

// thread 0: arrive with the byte count of all copies and issue the
// coefficient copies (RESID needs no 1/diag)
template <typename T, bool RESID>
__device__ __forceinline__ void mstage_static(const MLevel<T>& L, int leaf, const MStageSet& Q, const MStaged& S,
                                              uint64_t* bar) {
    const bool ni = Q.i && !RESID;
    const unsigned bytes = 1024u * (2u + (Q.d ? 1u : 0u) + (ni ? 1u : 0u) + (Q.cx ? 1u : 0u) + (Q.cy ? 1u : 0u) +
                                    (Q.cz ? 1u : 0u));
    mbar_expect_tx(bar, bytes);
    const long long o = (long long)leaf * UAAMG_LEAF;
    if (Q.d) bulk_g2s(S.d, L.diag + o, 1024u, bar);
    if (ni) bulk_g2s(S.i, L.invdiag + o, 1024u, bar);
    if (Q.cx) bulk_g2s(S.cx, L.cx + o, 1024u, bar);
    if (Q.cy) bulk_g2s(S.cy, L.cy + o, 1024u, bar);
    if (Q.cz) bulk_g2s(S.cz, L.cz + o, 1024u, bar);
}

// a thread's halo: neighbour leaves and their face coefficients (static),
// then the neighbours' x values (after the wait)
struct MHalo {
    int xp, xm, yp, ym, z;
    float4 cxp, cyp;
    float cz;
    float4 xpv, xmv, ypv, ymv;
    float zv;
};
template <typename T>
__device__ __forceinline__ void mhalo_static(const MLevel<T>& L, int leaf, int t, MHalo& H) {
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
    // flags and values load together; a trimmed neighbour reads the FP32
    // default (its stored 16-bit value is the rounded default)
    if (H.xp >= 0) {
        const unsigned f = L.flags[H.xp];
        const float4 v = ldc4(L, L.cx, H.xp, t - 112);
        if (!(f & TRIM_X)) H.cxp = v;
    }
    if (H.yp >= 0) {
        const unsigned f = L.flags[H.yp];
        const float4 v = ldc4(L, L.cy, H.yp, t - 14);
        if (!(f & TRIM_Y)) H.cyp = v;
    }
    if (zh == 1 && H.z >= 0) {
        const unsigned f = L.flags[H.z];
        const float v = ldc1(L, L.cz, (long long)H.z * UAAMG_LEAF + 4 * t - 4);
        if (!(f & TRIM_Z)) H.cz = v;
    }
}
template <typename T>
__device__ __forceinline__ void mhalo_dyn(const T* x, int t, MHalo& H) {
    H.xpv = (H.xp >= 0) ? ldh4(x, H.xp, t - 112) : f4zero();
    H.xmv = (H.xm >= 0) ? ldh4(x, H.xm, t + 112) : f4zero();
    H.ypv = (H.yp >= 0) ? ldh4(x, H.yp, t - 14) : f4zero();
    H.ymv = (H.ym >= 0) ? ldh4(x, H.ym, t + 14) : f4zero();
    H.zv = 0.f;
    if (H.z >= 0) H.zv = ldh1(x, (long long)H.z * UAAMG_LEAF + ((t & 1) ? 4 * t - 4 : 4 * t + 7));
}

#ifndef MSTAGED_MINB  // minimum resident CTAs per SM (1: no register cap; higher values spill)
#define MSTAGED_MINB 1
#endif
#define MSTAGED_SMEM_DECL                                                                                    \
    __shared__ __align__(128) uint16_t msm_x[UAAMG_LEAF], msm_b[UAAMG_LEAF], msm_d[UAAMG_LEAF],             \
        msm_i[UAAMG_LEAF], msm_cx[UAAMG_LEAF], msm_cy[UAAMG_LEAF], msm_cz[UAAMG_LEAF];                      \
    __shared__ __align__(8) uint64_t msm_bar;                                                                \
    const MStaged S{msm_x, msm_b, msm_d, msm_i, msm_cx, msm_cy, msm_cz};

// static part, wait, x/b copies, halo, bounded wait on the copies; false if
// the wait timed out (error flagged)
template <typename T, bool RESID>
__device__ __forceinline__ bool mstaged_prologue(const MLevel<T>& L, int leaf, int t, const T* x, const T* b,
                                                 const MStaged& S, uint64_t* bar, unsigned& fl, MHalo& H, int* err) {
    fl = L.flags[leaf];
    const MStageSet Q(fl);
    mhalo_static(L, leaf, t, H);
    if (t == 0) mbar_init(bar, 1);
    __syncthreads();
    if (t == 0) mstage_static<T, RESID>(L, leaf, Q, S, bar);
    griddep_wait();
    griddep_launch();
    if (t == 0) {
        const long long o = (long long)leaf * UAAMG_LEAF;
        bulk_g2s(S.x, x + o, 1024u, bar);
        bulk_g2s(S.b, b + o, 1024u, bar);
    }
    mhalo_dyn(x, t, H);
    const bool ok = __syncthreads_and(mbar_wait_bounded(bar, 0) ? 1 : 0) != 0;
    if (!ok) {
        if (t == 0 && err) atomicExch(err, 1);
        mbar_wait_bounded(bar, 0);
    }
    return ok;
}

// weighted Jacobi (RESID false) or residual (RESID true) of the thread's 4
// voxels from the staged leaf
template <bool RESID, typename T>
__device__ __forceinline__ float4 mstaged_value(const MLevel<T>& L, int leaf, int t, unsigned fl, const MStaged& S,
                                                const MHalo& H, float w) {
    const int X = t >> 4, Y = (t >> 1) & 7, zh = t & 1;
    const float df = L.def_face;
    const float4 dfv = f4splat(df);
    const float cs = L.cs;
    const float4 xc = msh4<T>(S.x, t);
    const float4 xp = (X < 7) ? msh4<T>(S.x, t + 16) : H.xpv;
    const float4 xm = (X > 0) ? msh4<T>(S.x, t - 16) : H.xmv;
    const float4 yp = (Y < 7) ? msh4<T>(S.x, t + 2) : H.ypv;
    const float4 ym = (Y > 0) ? msh4<T>(S.x, t - 2) : H.ymv;
    const float4 cxp = (X < 7) ? ((fl & TRIM_X) ? dfv : f4scale(msh4<T>(S.cx, t + 16), cs)) : H.cxp;
    const float4 cyp = (Y < 7) ? ((fl & TRIM_Y) ? dfv : f4scale(msh4<T>(S.cy, t + 2), cs)) : H.cyp;
    const float4 cxm = (fl & TRIM_X) ? dfv : f4scale(msh4<T>(S.cx, t), cs);
    const float4 cym = (fl & TRIM_Y) ? dfv : f4scale(msh4<T>(S.cy, t), cs);
    const float4 czo = (fl & TRIM_Z) ? dfv : f4scale(msh4<T>(S.cz, t), cs);
    float zp3, zm0, czp3;
    if (zh == 0) {
        zp3 = msh1<T>(S.x, 4 * t + 4);
        czp3 = (fl & TRIM_Z) ? df : __fmul_rn(msh1<T>(S.cz, 4 * t + 4), cs);
        zm0 = H.zv;
    } else {
        zm0 = msh1<T>(S.x, 4 * t - 1);
        zp3 = H.zv;
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
    const unsigned m = mask4(L.mask, leaf, t);
    const float4 dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : f4scale(msh4<T>(S.d, t), cs);
    const float4 bb = f4scale(msh4<T>(S.b, t), cs);
    float4 res;
    if (RESID) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
    } else {
        const float4 iv = (fl & TRIM_DIAG) ? f4splat(L.def_invdiag) : f4scale(msh4<T>(S.i, t), L.ics);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
            r = __fmul_rn(r, f4get(iv, j));
            f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
        }
    }
    if (!(m & 1)) res.x = 0.f;
    if (!(m & 2)) res.y = 0.f;
    if (!(m & 4)) res.z = 0.f;
    if (!(m & 8)) res.w = 0.f;
    return res;
}

// One staged Jacobi sweep with a plain source; TOut float (with zscale and
// the optional z.r) for the last sweep of level 0, as k_msweep.
template <typename T, typename TOut>
__global__ void __launch_bounds__(128, MSTAGED_MINB) k_msweep_staged(MLevel<T> L, const T* x, const T* b, TOut* out, float w,
                                                       DotOut dot, const float* zscale, int* err) {
    MSTAGED_SMEM_DECL
    const int leaf = blockIdx.x, t = threadIdx.x;
    unsigned fl;
    MHalo H;
    const bool ok = mstaged_prologue<T, false>(L, leaf, t, x, b, S, &msm_bar, fl, H, err);
    float4 res = f4zero();
    if (ok) {
        res = mstaged_value<false>(L, leaf, t, fl, S, H, w);
        if (zscale) res = f4scale(res, *zscale);
        stv4(out, leaf, t, res);
    }
    if (dot.r) {
        __shared__ double shd[4];
        const float4 rr = ld4(dot.r, leaf, t);
        const double s = (double)res.x * rr.x + (double)res.y * rr.y + (double)res.z * rr.z + (double)res.w * rr.w;
        const double part = block_sum128(s, shd);
        double tot;
        if (reduce_sum(part, dot.partials, &dot.st->ticket[0], leaf, (int)gridDim.x, tot)) {
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

// staged residual + restriction into the next level's 16-bit rhs (as k_mrestrict)
template <typename T>
__global__ void __launch_bounds__(128, MSTAGED_MINB) k_mrestrict_staged(MLevel<T> L, const T* x, const T* b, T* coarse,
                                                          float coarse_ics, int* err) {
    MSTAGED_SMEM_DECL
    __shared__ __align__(16) float rs[UAAMG_LEAF];
    const int leaf = blockIdx.x, t = threadIdx.x;
    unsigned fl;
    MHalo H;
    if (!mstaged_prologue<T, true>(L, leaf, t, x, b, S, &msm_bar, fl, H, err)) return;
    reinterpret_cast<float4*>(rs)[t] = mstaged_value<true>(L, leaf, t, fl, S, H, 0.f);
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
                    const int fo = ((2 * i + ii) << 6) | ((2 * j + jj) << 3) | (2 * k + kk);
                    if ((mk[fo >> 6] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                }
        const int o = L.octant[leaf];
        const int coff = ((((o >> 2) & 1) * 4 + i) << 6) | ((((o >> 1) & 1) * 4 + j) << 3) | ((o & 1) * 4 + k);
        coarse[(long long)L.parent[leaf] * UAAMG_LEAF + coff] =
            H16<T>::from1(__fmul_rn(__fmul_rn(s, 0.125f), coarse_ics));
    }
}

// A computed source stored as a 16-bit vector (zero off the DOF): the first
// sweep's w * (1/diag * b), or the prolongation-add x + P x_c (in place)
template <typename T, class Src>
__global__ void __launch_bounds__(128) k_mmaterialize(MLevel<T> L, Src src, T* out) {  // grid-stride
    griddep_wait();
    griddep_launch();
    const int t = threadIdx.x;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x) {
        float4 v = src.get4(L, leaf, t);
        const unsigned m = mask4(L.mask, leaf, t);
        if (!(m & 1)) v.x = 0.f;
        if (!(m & 2)) v.y = 0.f;
        if (!(m & 4)) v.z = 0.f;
        if (!(m & 8)) v.w = 0.f;
        sth4(out, leaf, t, v);
    }
}

// ---------------------------------------------------------------------------
// Coarsest level in FP64: a dense inverse of the coarsest matrix, built once by
// Gauss-Jordan elimination (the matrix is symmetric positive definite when the
// domain has a free surface, so no pivoting), applied as an FP64 GEMV.
__global__ void __launch_bounds__(256) k_cdense(DCoarsest C, double* A) {
    const int i = blockIdx.x;  // row
    const int n = C.n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) A[(long long)i * n + j] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0) {
        A[(long long)i * n + i] = (double)C.diag[i];
        for (int e = 0; e < 6; ++e) {
            const int c = C.col[i * 6 + e];
            if (c >= 0) A[(long long)i * n + c] += (double)C.val[i * 6 + e];
        }
    }
}
// step k: save column k and the normalised row k
__global__ void __launch_bounds__(256) k_gj_pivot(double* A, int n, int k, double* fcol, double* rrow, int* err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const double p = A[(long long)k * n + k];
    if (j == 0 && !(p > 0.0)) atomicExch(err, 1);
    if (j >= n) return;
    fcol[j] = A[(long long)j * n + k];
    rrow[j] = (j == k ? 1.0 : A[(long long)k * n + j]) / p;
}
__global__ void __launch_bounds__(256) k_gj_update(double* A, int n, int k, const double* fcol, const double* rrow) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int i = (int)(idx / n), j = (int)(idx % n);
    if (i == k) {
        A[idx] = rrow[j];
    } else {
        const double a = (j == k) ? 0.0 : A[idx];
        A[idx] = a - fcol[i] * rrow[j];
    }
}
// out(slot i) = sum_j Ainv[i][j] rhs(slot j): one warp per row, FP64
template <typename T>
__global__ void __launch_bounds__(256) k_cgemv(int n, const double* Ainv, const int* slot, const T* rhs, T* out,
                                               float rhs_scale) {
    griddep_wait();
    griddep_launch();
    extern __shared__ double bs[];
    for (int j = threadIdx.x; j < n; j += blockDim.x) bs[j] = (double)ldh1(rhs, slot[j]) * (double)rhs_scale;
    __syncthreads();
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;
    const double* a = Ainv + (long long)row * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += a[j] * bs[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULLMASK, s, o);
    if (lane == 0) out[slot[row]] = H16<T>::from1((float)s);
}

// r = b - A x every `every` iterations of the outer CG (true-residual
// replacement); the other iterations leave r alone
__global__ void __launch_bounds__(128) k_pcg_replace(DLevel L, const float* x, const float* b, float* r,
                                                     const PcgState* st, int every) {
    griddep_wait();
    griddep_launch();
    const int it = st->iter;
    if (st->first || it == 0 || (it % every) != 0) return;
    const int t = threadIdx.x;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x) {  // grid-stride
        float4 xc;
        unsigned m;
        st4(r, leaf, t, sweep_value<M_RESIDUAL>(L, leaf, t, SrcPlain{x}, b, 0.f, 0.f, 0.f, xc, m));
    }
}

// |b - A x|_inf and |b|_inf over the DOF in FP64 (A x from the FP32
// level-0 coefficients in double arithmetic): the true relative residual of
// a solution, for accuracy checks.  out[0], out[1] (doubles) must start at 0.
__device__ __forceinline__ double f64get(const float4& v, int j) { return (double)f4get(v, j); }
__global__ void __launch_bounds__(128) k_res64(DLevel L, const float* x, const float* b, unsigned long long* out) {
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int X = t >> 4, Y = (t >> 1) & 7;
    const unsigned m = mask4(L.mask, leaf, t);
    const unsigned fl = L.flags[leaf];
    const float4 dfv = f4splat(L.def_face);
    const int* nb = L.nbr + (long long)leaf * 6;
    double rmax = 0.0, bmax = 0.0;
    if (m) {
        const float4 xc = ld4(x, leaf, t), bb = ld4(b, leaf, t);
        const float4 dg = (fl & TRIM_DIAG) ? f4splat(L.def_diag) : ld4(L.diag, leaf, t);
        const float4 cxm = (fl & TRIM_X) ? dfv : ld4(L.cx, leaf, t);
        const float4 cym = (fl & TRIM_Y) ? dfv : ld4(L.cy, leaf, t);
        const float4 czo = (fl & TRIM_Z) ? dfv : ld4(L.cz, leaf, t);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!((m >> j) & 1)) continue;
            const int off = 4 * t + j, Z = off & 7;
            auto xat = [&](int lf, int o) -> double { return lf >= 0 ? (double)x[(long long)lf * UAAMG_LEAF + o] : 0.0; };
            auto cat = [&](const float* c, unsigned bit, int lf, int o) -> double {
                if (lf < 0) return (double)L.def_face;
                return (L.flags[lf] & bit) ? (double)L.def_face : (double)c[(long long)lf * UAAMG_LEAF + o];
            };
            double ax = f64get(dg, j) * f64get(xc, j);
            // minus faces: this voxel's coefficient, the neighbour's value
            ax += f64get(cxm, j) * (X > 0 ? xat(leaf, off - 64) : xat(nb[0], off + 448));
            ax += f64get(cym, j) * (Y > 0 ? xat(leaf, off - 8) : xat(nb[2], off + 56));
            ax += f64get(czo, j) * (Z > 0 ? xat(leaf, off - 1) : xat(nb[4], off + 7));
            // plus faces: the neighbour's coefficient and value
            ax += (X < 7 ? cat(L.cx, TRIM_X, leaf, off + 64) * xat(leaf, off + 64)
                         : cat(L.cx, TRIM_X, nb[1], off - 448) * xat(nb[1], off - 448));
            ax += (Y < 7 ? cat(L.cy, TRIM_Y, leaf, off + 8) * xat(leaf, off + 8)
                         : cat(L.cy, TRIM_Y, nb[3], off - 56) * xat(nb[3], off - 56));
            ax += (Z < 7 ? cat(L.cz, TRIM_Z, leaf, off + 1) * xat(leaf, off + 1)
                         : cat(L.cz, TRIM_Z, nb[5], off - 7) * xat(nb[5], off - 7));
            rmax = fmax(rmax, fabs(f64get(bb, j) - ax));
            bmax = fmax(bmax, fabs(f64get(bb, j)));
        }
    }
    // non-negative doubles order like their bit patterns
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(rmax));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(bmax));
}

}  // namespace uaamg
