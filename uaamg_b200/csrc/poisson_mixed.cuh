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
    sth4(out, blockIdx.x, threadIdx.x, f4scale(ld4(in, blockIdx.x, threadIdx.x), sc));
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
// z-line kernels: one thread per 8-voxel z-line (x = t >> 3, y = t & 7,
// offset 64x + 8y + z), 64 threads per leaf.  A line of a 16-bit array is
// one 16-byte load, so a warp reads 512 contiguous bytes per array and each
// thread keeps ~10 independent loads in flight; the +-z neighbours inside the
// line are register shifts.  Same per-voxel operations and order as
// mstencil4 / mjacobi_value.
struct F8 {
    float v[8];
};
template <typename T>
__device__ __forceinline__ F8 ldl8(const T* p, long long leaf, int line) {  // 8 values of a z-line
    const uint4 u = reinterpret_cast<const uint4*>(p)[leaf * 64 + line];
    F8 r;
    float2 a = H16<T>::to2(u.x), b = H16<T>::to2(u.y), c = H16<T>::to2(u.z), d = H16<T>::to2(u.w);
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
    r.v[4] = c.x; r.v[5] = c.y; r.v[6] = d.x; r.v[7] = d.y;
    return r;
}
template <typename T>
__device__ __forceinline__ void stl8(T* p, long long leaf, int line, const F8& f) {
    uint4 u;
    u.x = H16<T>::from2(f.v[0], f.v[1]);
    u.y = H16<T>::from2(f.v[2], f.v[3]);
    u.z = H16<T>::from2(f.v[4], f.v[5]);
    u.w = H16<T>::from2(f.v[6], f.v[7]);
    reinterpret_cast<uint4*>(p)[leaf * 64 + line] = u;
}
__device__ __forceinline__ void stl8(float* p, long long leaf, int line, const F8& f) {
    float4* q = reinterpret_cast<float4*>(p + leaf * UAAMG_LEAF + line * 8);
    q[0] = make_float4(f.v[0], f.v[1], f.v[2], f.v[3]);
    q[1] = make_float4(f.v[4], f.v[5], f.v[6], f.v[7]);
}
__device__ __forceinline__ F8 f8splat(float x) {
    F8 r;
#pragma unroll
    for (int j = 0; j < 8; ++j) r.v[j] = x;
    return r;
}
__device__ __forceinline__ F8 f8scale(F8 a, float s) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a.v[j] = __fmul_rn(a.v[j], s);
    return a;
}
template <typename T>
__device__ __forceinline__ F8 ldc8(const MLevel<T>& L, const T* a, long long leaf, int line) {
    return f8scale(ldl8(a, leaf, line), L.cs);
}

// line sources
template <typename T>
struct LSrcPlain {
    const T* x;
    __device__ __forceinline__ F8 line(const MLevel<T>&, int leaf, int ln) const { return ldl8(x, leaf, ln); }
    __device__ __forceinline__ float one(const MLevel<T>&, int leaf, int off) const {
        return ldh1(x, (long long)leaf * UAAMG_LEAF + off);
    }
};
template <typename T>
struct LSrcFirstJacobi {  // w * (invdiag * b)
    const T* b;
    float w;
    __device__ __forceinline__ F8 line(const MLevel<T>& L, int leaf, int ln) const {
        const F8 bb = ldc8(L, b, leaf, ln);
        const F8 iv = (L.flags[leaf] & TRIM_DIAG) ? f8splat(L.def_invdiag) : f8scale(ldl8(L.invdiag, leaf, ln), L.ics);
        F8 r;
#pragma unroll
        for (int j = 0; j < 8; ++j) r.v[j] = __fmul_rn(w, __fmul_rn(iv.v[j], bb.v[j]));
        return r;
    }
    __device__ __forceinline__ float one(const MLevel<T>& L, int leaf, int off) const {
        const long long i = (long long)leaf * UAAMG_LEAF + off;
        const float iv = (L.flags[leaf] & TRIM_DIAG) ? L.def_invdiag : __fmul_rn(ldh1(L.invdiag, i), L.ics);
        return __fmul_rn(w, __fmul_rn(iv, ldc1(L, b, i)));
    }
};
template <typename T>
struct LSrcProlong {  // x + coarse parent value at active voxels
    const T* x;
    const T* xc;
    __device__ __forceinline__ F8 line(const MLevel<T>& L, int leaf, int ln) const {
        F8 v = ldl8(x, leaf, ln);
        const int X = ln >> 3, Y = ln & 7;
        const unsigned m = (unsigned)((L.mask[(long long)leaf * 8 + X] >> (8 * Y)) & 0xFFull);
        if (!m) return v;
        const int P = L.parent[leaf];
        const int o = L.octant[leaf];
        const long long cb = (long long)P * UAAMG_LEAF + (((o >> 2) & 1) * 4 + (X >> 1)) * 64 +
                             (((o >> 1) & 1) * 4 + (Y >> 1)) * 8 + (o & 1) * 4;
        const uint2 u = *reinterpret_cast<const uint2*>(xc + cb);  // 4 coarse values (z pairs)
        const float2 c01 = H16<T>::to2(u.x), c23 = H16<T>::to2(u.y);
        const float c[4] = {c01.x, c01.y, c23.x, c23.y};
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if ((m >> j) & 1) v.v[j] = __fadd_rn(v.v[j], c[j >> 1]);
        return v;
    }
    __device__ __forceinline__ float one(const MLevel<T>& L, int leaf, int off) const {
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

template <typename T, class Src>
__device__ __forceinline__ void mstencil8(const MLevel<T>& L, int leaf, int ln, const Src& src, F8& xc, F8& off) {
    const int X = ln >> 3, Y = ln & 7;
    const unsigned fl = L.flags[leaf];
    const int* nb = L.nbr + (long long)leaf * 6;
    const float df = L.def_face;
    xc = src.line(L, leaf, ln);
    F8 xp, xm, yp, ym, cxp, cyp;
    if (X < 7) {
        xp = src.line(L, leaf, ln + 8);
        cxp = (fl & TRIM_X) ? f8splat(df) : ldc8(L, L.cx, leaf, ln + 8);
    } else {
        const int n = nb[1];
        if (n >= 0) {
            xp = src.line(L, n, ln - 56);
            cxp = (L.flags[n] & TRIM_X) ? f8splat(df) : ldc8(L, L.cx, n, ln - 56);
        } else {
            xp = f8splat(0.f);
            cxp = f8splat(df);
        }
    }
    if (X > 0) {
        xm = src.line(L, leaf, ln - 8);
    } else {
        const int n = nb[0];
        xm = (n >= 0) ? src.line(L, n, ln + 56) : f8splat(0.f);
    }
    if (Y < 7) {
        yp = src.line(L, leaf, ln + 1);
        cyp = (fl & TRIM_Y) ? f8splat(df) : ldc8(L, L.cy, leaf, ln + 1);
    } else {
        const int n = nb[3];
        if (n >= 0) {
            yp = src.line(L, n, ln - 7);
            cyp = (L.flags[n] & TRIM_Y) ? f8splat(df) : ldc8(L, L.cy, n, ln - 7);
        } else {
            yp = f8splat(0.f);
            cyp = f8splat(df);
        }
    }
    if (Y > 0) {
        ym = src.line(L, leaf, ln - 1);
    } else {
        const int n = nb[2];
        ym = (n >= 0) ? src.line(L, n, ln + 7) : f8splat(0.f);
    }
    const F8 cxm = (fl & TRIM_X) ? f8splat(df) : ldc8(L, L.cx, leaf, ln);
    const F8 cym = (fl & TRIM_Y) ? f8splat(df) : ldc8(L, L.cy, leaf, ln);
    const F8 czo = (fl & TRIM_Z) ? f8splat(df) : ldc8(L, L.cz, leaf, ln);
    // the line's ends: z = -1 from the -z leaf, z = 8 (value and c_z) from the +z leaf
    const int nzm = nb[4], nzp = nb[5];
    const float zm0 = nzm >= 0 ? src.one(L, nzm, ln * 8 + 7) : 0.f;
    float zp7 = 0.f, czp7 = df;
    if (nzp >= 0) {
        zp7 = src.one(L, nzp, ln * 8);
        czp7 = (L.flags[nzp] & TRIM_Z) ? df : ldc1(L, L.cz, (long long)nzp * UAAMG_LEAF + ln * 8);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float zp = j < 7 ? xc.v[j + 1] : zp7;
        const float zm = j > 0 ? xc.v[j - 1] : zm0;
        const float czp = j < 7 ? czo.v[j + 1] : czp7;
        float f1 = __fmul_rn(xp.v[j], cxp.v[j]);
        float f2 = __fmul_rn(xm.v[j], cxm.v[j]);
        float f3 = __fmul_rn(yp.v[j], cyp.v[j]);
        float f4 = __fmul_rn(ym.v[j], cym.v[j]);
        float f5 = __fmul_rn(zp, czp);
        float f6 = __fmul_rn(zm, czo.v[j]);
        f1 = __fadd_rn(f1, f2);
        f3 = __fadd_rn(f3, f4);
        f5 = __fadd_rn(f5, f6);
        f1 = __fadd_rn(f1, f3);
        off.v[j] = __fadd_rn(f1, f5);
    }
}

template <bool RESID, typename T, class Src>
__device__ __forceinline__ F8 mjacobi8(const MLevel<T>& L, int leaf, int ln, const Src& src, const T* b, float w) {
    F8 xc, off;
    mstencil8(L, leaf, ln, src, xc, off);
    const int X = ln >> 3, Y = ln & 7;
    const unsigned m = (unsigned)((L.mask[(long long)leaf * 8 + X] >> (8 * Y)) & 0xFFull);
    const unsigned fl = L.flags[leaf];
    const F8 dg = (fl & TRIM_DIAG) ? f8splat(L.def_diag) : ldc8(L, L.diag, leaf, ln);
    const F8 bb = ldc8(L, b, leaf, ln);
    F8 res;
    if (RESID) {
#pragma unroll
        for (int j = 0; j < 8; ++j) res.v[j] = __fsub_rn(bb.v[j], __fmaf_rn(xc.v[j], dg.v[j], off.v[j]));
    } else {
        const F8 iv = (fl & TRIM_DIAG) ? f8splat(L.def_invdiag) : f8scale(ldl8(L.invdiag, leaf, ln), L.ics);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float r = __fsub_rn(bb.v[j], __fmaf_rn(xc.v[j], dg.v[j], off.v[j]));
            r = __fmul_rn(r, iv.v[j]);
            res.v[j] = __fmaf_rn(w, r, xc.v[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (!((m >> j) & 1)) res.v[j] = 0.f;
    return res;
}

template <typename T, typename TOut, class Src>
__global__ void __launch_bounds__(64) k_msweep8(MLevel<T> L, Src src, const T* b, TOut* out, float w, DotOut dot,
                                               const float* zscale) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, ln = threadIdx.x;
    F8 res = mjacobi8<false>(L, leaf, ln, src, b, w);
    if (zscale) res = f8scale(res, *zscale);
    stl8(out, leaf, ln, res);
    if (dot.r) {
        __shared__ double shd[2];
        const float4* rp = reinterpret_cast<const float4*>(dot.r + (long long)leaf * UAAMG_LEAF + ln * 8);
        const float4 r0 = rp[0], r1 = rp[1];
        double s = (double)res.v[0] * r0.x + (double)res.v[1] * r0.y + (double)res.v[2] * r0.z +
                   (double)res.v[3] * r0.w + (double)res.v[4] * r1.x + (double)res.v[5] * r1.y +
                   (double)res.v[6] * r1.z + (double)res.v[7] * r1.w;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULLMASK, s, o);
        if ((threadIdx.x & 31) == 0) shd[threadIdx.x >> 5] = s;
        __syncthreads();
        const double part = shd[0] + shd[1];
        double tot;
        if (reduce_sum(part, dot.partials, &dot.st->ticket[0], leaf, (int)gridDim.x, tot)) {
            if (threadIdx.x == 0) {
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

template <typename T>
__global__ void __launch_bounds__(64) k_mrestrict8(MLevel<T> L, const T* x, const T* b, T* coarse, float coarse_ics) {
    griddep_wait();
    griddep_launch();
    __shared__ float rs[UAAMG_LEAF];
    const int leaf = blockIdx.x, ln = threadIdx.x;
    const F8 r = mjacobi8<true>(L, leaf, ln, LSrcPlain<T>{x}, b, 0.f);
    float4* q = reinterpret_cast<float4*>(rs + ln * 8);
    q[0] = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
    q[1] = make_float4(r.v[4], r.v[5], r.v[6], r.v[7]);
    __syncthreads();
    const int t = threadIdx.x;  // 64 coarse voxels of the octant
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
    coarse[(long long)L.parent[leaf] * UAAMG_LEAF + coff] = H16<T>::from1(__fmul_rn(__fmul_rn(s, 0.125f), coarse_ics));
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
    const int leaf = blockIdx.x, t = threadIdx.x;
    float4 xc;
    unsigned m;
    st4(r, leaf, t, sweep_value<M_RESIDUAL>(L, leaf, t, SrcPlain{x}, b, 0.f, 0.f, 0.f, xc, m));
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
