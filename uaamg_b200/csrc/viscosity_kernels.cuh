// viscosity_kernels.cuh -- sm_100a kernels of the variational-viscosity
// UAAMG-PCG (the solve phase).
//
// Arithmetic follows L_with_level::light_weight_applier::component_operator<c>
// (SIMD_UAAMG/simd_viscosity3d.cpp:2849-3603) operation by operation with
// round-to-nearest intrinsics (the library is built with --fmad=false), so the
// per-voxel results are bit-identical to the reference's AVX2 lanes.
//
// Layout of a level (one leaf set for all three velocity channels: the leaves
// of the union of the channel DOF masks dilated by the coefficient pattern):
//   dof   uint64 [3][nl][8]     per-channel DOF masks (word x = plane x)
//   nb    int32  [nl][27]       3x3x3 neighbour leaves, (dx+1)*9+(dy+1)*3+dz+1
//   coef  float  [27][nl][512]  array (c*9 + a): diag, invdiag, neg_x, neg_y,
//                               neg_z, T00, T01, T10, T11 of channel c
//   vectors float [3][nl][512], zero at every non-DOF voxel
// One CTA of 128 threads per (leaf, channel); thread t owns voxels 4t..4t+3
// (x = t>>4, y = (t>>1)&7, z = 4*(t&1)+j): one float4 of every array.
#pragma once
#include "common.cuh"
#include "poisson_kernels.cuh"

namespace uaamg {

#define VNA 9
enum { VA_DIAG = 0, VA_INV = 1, VA_NEGX = 2, VA_NEGY = 3, VA_NEGZ = 4, VA_T00 = 5, VA_T01 = 6, VA_T10 = 7,
       VA_T11 = 8 };
enum { VM_NORMAL = 0, VM_RESIDUAL = 1, VM_JACOBI = 2, VM_RED = 3, VM_BLACK = 4 };

struct VLevel {
    int nl;
    const uint64_t* dof;          // [3][nl][8]
    const int* nb;                // [nl][27]
    const int* cnb;               // [nl][27] nb for coefficient reads: -1 at fully trimmed leaves; NULL = nb
    const float* coef;            // [27][nl][512]
    const uint32_t* trim;         // [nl] bit (c*9+a): leaf holds the default
    const float* defpage;         // [27][512] applier default of every array
    const float* zpage;           // [512] zeros
    const int* parent;            // [nl] coarse leaf, -1 if none
    const unsigned char* octant;  // [nl] position in the parent: x<<2 | y<<1 | z
    const int* child;             // [nl][8] fine leaf per octant, -1 if none
    float app[27];                // light_weight_applier defaults (missing leaf)
};

__device__ __forceinline__ unsigned vmask4(const VLevel& L, int c, int leaf, int t) {
    return (unsigned)((L.dof[((long long)c * L.nl + leaf) * 8 + (t >> 4)] >> ((t & 15) * 4)) & 0xFull);
}
__device__ __forceinline__ bool vdof_bit(const VLevel& L, int c, int leaf, int off) {
    return (L.dof[((long long)c * L.nl + leaf) * 8 + (off >> 6)] >> (off & 63)) & 1ull;
}
__device__ __forceinline__ int vnb_index(int X, int Y, int Z) {
    const int a = X < 0 ? 0 : (X > 7 ? 2 : 1), b = Y < 0 ? 0 : (Y > 7 ? 2 : 1), c = Z < 0 ? 0 : (Z > 7 ? 2 : 1);
    return a * 9 + b * 3 + c;
}
__device__ __forceinline__ int voff3(int X, int Y, int Z) { return ((X & 7) << 6) | ((Y & 7) << 3) | (Z & 7); }

// The 27-neighbourhood of the CTA's leaf, staged in shared memory once per
// CTA: every later load depends only on a shared-memory read, so all of a
// thread's global loads are in flight together instead of in dependent
// chains.  (Trimmed level-0 leaves need no check here: their blocks hold the
// applier default itself, written by k_vtrim_fill.)
// Coefficient reads use a second table in which a leaf whose 27 arrays are
// all trimmed is replaced by -1: its blocks hold exactly the applier defaults,
// which the default page also holds, and that page stays in L1 while the
// leaf's own blocks would stream from DRAM.
struct VNbSh {
    int nb[27];
    int cnb[27];
};
// call with all threads of the CTA (contains __syncthreads)
__device__ __forceinline__ void vnb_prologue(const VLevel& L, int leaf, VNbSh& sh) {
    const int t = threadIdx.x;
    if (t < 27) {
        const int v = L.nb[(long long)leaf * 27 + t];
        sh.nb[t] = v;
        sh.cnb[t] = L.cnb ? L.cnb[(long long)leaf * 27 + t] : v;
    }
    __syncthreads();
}

// Address of the leaf block holding neighbourhood slot k of array arr: the
// fallback page when the leaf does not exist (or, for coefficients, is fully
// trimmed).
template <bool COEF = false>
__device__ __forceinline__ const float* vsel(const float* arr, const float* fallback, const VNbSh& sh, int k) {
    const int lf = COEF ? sh.cnb[k] : sh.nb[k];
    return lf >= 0 ? arr + (long long)lf * UAAMG_LEAF : fallback;
}

// Values of a [nl][512] array at the thread's four voxels shifted by
// (dx, dy, dz), dz in {-1, 0, 1}: missing leaves read the fallback page
// (zeros for vectors, the applier default for coefficients).
template <bool COEF = false>
__device__ __forceinline__ float4 vload4(const float* arr, const float* fb, const VNbSh& sh, int x, int y, int z0,
                                         int dx, int dy, int dz) {
    const int X = x + dx, Y = y + dy;
    const float* p = vsel<COEF>(arr, fb, sh, vnb_index(X, Y, z0));
    const float4 a = *reinterpret_cast<const float4*>(p + voff3(X, Y, z0));
    if (dz == 0) return a;
    if (dz > 0) {
        const float* q = vsel<COEF>(arr, fb, sh, vnb_index(X, Y, z0 + 4));
        return make_float4(a.y, a.z, a.w, q[voff3(X, Y, z0 + 4)]);
    }
    const float* q = vsel<COEF>(arr, fb, sh, vnb_index(X, Y, z0 - 1));
    return make_float4(q[voff3(X, Y, z0 - 1)], a.x, a.y, a.z);
}

struct VArr {  // one coefficient array of a level with its default page
    const float* a;
    const float* def;
};
__device__ __forceinline__ VArr varr(const VLevel& L, int c, int a) {
    VArr r;
    r.a = L.coef + (long long)(c * VNA + a) * L.nl * UAAMG_LEAF;
    r.def = L.defpage + (c * VNA + a) * UAAMG_LEAF;
    return r;
}
__device__ __forceinline__ float4 cload4(const VArr& A, const VNbSh& sh, int x, int y, int z0, int dx, int dy,
                                         int dz) {
    return vload4<true>(A.a, A.def, sh, x, y, z0, dx, dy, dz);
}
__device__ __forceinline__ float4 uload4(const float* v, const VLevel& L, int c, const VNbSh& sh, int x, int y, int z0,
                                         int dx, int dy, int dz) {
    return vload4(v + (long long)c * L.nl * UAAMG_LEAF, L.zpage, sh, x, y, z0, dx, dy, dz);
}

// Off-diagonal sum of channel c at the thread's four voxels (faced_result[1]
// after the cross terms, :3084-3490) and the centre value.
__device__ __forceinline__ float4 voffdiag(const VLevel& L, const VNbSh& sh, int c, int t, const float* x,
                                          float4& xc) {
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    xc = uload4(x, L, c, sh, X, Y, Z0, 0, 0, 0);
    // same channel, absolute axes x, y, z: u(g+e)*neg(g+e) and u(g-e)*neg(g)
    float4 fr[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const VArr W = varr(L, c, VA_NEGX + ax);
        const float4 up = uload4(x, L, c, sh, X, Y, Z0, px, py, pz);
        const float4 wp = cload4(W, sh, X, Y, Z0, px, py, pz);
        const float4 um = uload4(x, L, c, sh, X, Y, Z0, -px, -py, -pz);
        const float4 wm = cload4(W, sh, X, Y, Z0, 0, 0, 0);
        fr[2 * ax] = make_float4(__fmul_rn(up.x, wp.x), __fmul_rn(up.y, wp.y), __fmul_rn(up.z, wp.z),
                                 __fmul_rn(up.w, wp.w));
        fr[2 * ax + 1] = make_float4(__fmul_rn(um.x, wm.x), __fmul_rn(um.y, wm.y), __fmul_rn(um.z, wm.z),
                                     __fmul_rn(um.w, wm.w));
    }
    // Td2 (m_cross_channel[d2], channel d1 velocities) and Td1
    // (m_cross_channel[d1], channel d2 velocities)
    const float4 u1_g = uload4(x, L, d1, sh, X, Y, Z0, 0, 0, 0);
    const float4 u1_p1 = uload4(x, L, d1, sh, X, Y, Z0, e1[0], e1[1], e1[2]);
    const float4 u1_m0 = uload4(x, L, d1, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u1_m0p1 = uload4(x, L, d1, sh, X, Y, Z0, e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]);
    const float4 u2_g = uload4(x, L, d2, sh, X, Y, Z0, 0, 0, 0);
    const float4 u2_m0 = uload4(x, L, d2, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u2_p2 = uload4(x, L, d2, sh, X, Y, Z0, e2[0], e2[1], e2[2]);
    const float4 u2_m0p2 = uload4(x, L, d2, sh, X, Y, Z0, e2[0] - e0[0], e2[1] - e0[1], e2[2] - e0[2]);
    const float4 a00 = cload4(varr(L, d2, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    const float4 a01 = cload4(varr(L, d2, VA_T01), sh, X, Y, Z0, 0, 0, 0);
    const float4 a10 = cload4(varr(L, d2, VA_T10), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 a11 = cload4(varr(L, d2, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 b00 = cload4(varr(L, d1, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    const float4 b01 = cload4(varr(L, d1, VA_T01), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 b10 = cload4(varr(L, d1, VA_T10), sh, X, Y, Z0, 0, 0, 0);
    const float4 b11 = cload4(varr(L, d1, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    float4 off;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float f1 = __fadd_rn(f4get(fr[0], j), f4get(fr[1], j));
        float f3 = __fadd_rn(f4get(fr[2], j), f4get(fr[3], j));
        float f5 = __fadd_rn(f4get(fr[4], j), f4get(fr[5], j));
        f1 = __fadd_rn(f1, f3);
        f1 = __fadd_rn(f1, f5);
        const float R0 = __fmul_rn(f4get(u1_g, j), f4get(a00, j));
        const float R1 = __fmul_rn(f4get(a01, j), f4get(u1_p1, j));
        const float R2 = __fmul_rn(f4get(a10, j), f4get(u1_m0, j));
        const float R3 = __fmul_rn(f4get(a11, j), f4get(u1_m0p1, j));
        const float Q0 = __fmul_rn(f4get(b00, j), f4get(u2_g, j));
        const float Q1 = __fmul_rn(f4get(b01, j), f4get(u2_m0, j));
        const float Q2 = __fmul_rn(f4get(b10, j), f4get(u2_p2, j));
        const float Q3 = __fmul_rn(f4get(b11, j), f4get(u2_m0p2, j));
        const float td2 = __fadd_rn(__fadd_rn(R0, R1), __fadd_rn(R2, R3));
        const float td1 = __fadd_rn(__fadd_rn(Q0, Q1), __fadd_rn(Q2, Q3));
        f1 = __fadd_rn(f1, td2);
        f1 = __fadd_rn(f1, td1);
        f4set(off, j, f1);
    }
    return off;
}

// The coefficients one applier pass of channel c reads at the thread's
// voxels.  They do not change during a solve, so k_vapply loads them before it
// waits for the previous kernel (programmatic dependent launch): only the
// vector loads remain on the critical path after the wait.
struct VCoef {
    float4 wp[3], wm[3];                    // neg_x/y/z at g + e_ax and at g
    float4 a00, a01, a10, a11;              // m_cross_channel[d2]
    float4 b00, b01, b10, b11;              // m_cross_channel[d1]
    float4 dg;                              // 1/diag (GS, Jacobi) or diag (normal, residual)
};
// at the 4-voxel group (X, Y, Z0..Z0+3) relative to the CTA's leaf, X and Y in
// -1..8, Z0 in {0, 4}; inv: 1/diag instead of diag
template <int c>
__device__ __forceinline__ void vload_coef_at(const VLevel& L, const VNbSh& sh, int X, int Y, int Z0, bool inv,
                                              VCoef& k) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    int e0[3] = {0, 0, 0};
    e0[d0] = 1;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const VArr W = varr(L, c, VA_NEGX + ax);
        k.wp[ax] = cload4(W, sh, X, Y, Z0, px, py, pz);
        k.wm[ax] = cload4(W, sh, X, Y, Z0, 0, 0, 0);
    }
    k.a00 = cload4(varr(L, d2, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    k.a01 = cload4(varr(L, d2, VA_T01), sh, X, Y, Z0, 0, 0, 0);
    k.a10 = cload4(varr(L, d2, VA_T10), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.a11 = cload4(varr(L, d2, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.b00 = cload4(varr(L, d1, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    k.b01 = cload4(varr(L, d1, VA_T01), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.b10 = cload4(varr(L, d1, VA_T10), sh, X, Y, Z0, 0, 0, 0);
    k.b11 = cload4(varr(L, d1, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.dg = cload4(varr(L, c, inv ? VA_INV : VA_DIAG), sh, X, Y, Z0, 0, 0, 0);
}
template <int MODE, int c>
__device__ __forceinline__ void vload_coef(const VLevel& L, const VNbSh& sh, int t, VCoef& k) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int e0[3] = {0, 0, 0};
    e0[d0] = 1;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const VArr W = varr(L, c, VA_NEGX + ax);
        k.wp[ax] = cload4(W, sh, X, Y, Z0, px, py, pz);
        k.wm[ax] = cload4(W, sh, X, Y, Z0, 0, 0, 0);
    }
    k.a00 = cload4(varr(L, d2, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    k.a01 = cload4(varr(L, d2, VA_T01), sh, X, Y, Z0, 0, 0, 0);
    k.a10 = cload4(varr(L, d2, VA_T10), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.a11 = cload4(varr(L, d2, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.b00 = cload4(varr(L, d1, VA_T00), sh, X, Y, Z0, 0, 0, 0);
    k.b01 = cload4(varr(L, d1, VA_T01), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    k.b10 = cload4(varr(L, d1, VA_T10), sh, X, Y, Z0, 0, 0, 0);
    k.b11 = cload4(varr(L, d1, VA_T11), sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const bool inv = (MODE == VM_RED || MODE == VM_BLACK || MODE == VM_JACOBI);
    k.dg = cload4(varr(L, c, inv ? VA_INV : VA_DIAG), sh, X, Y, Z0, 0, 0, 0);
}

// voffdiag with the coefficients already loaded (same operations and order);
// the channel is a template parameter so every stencil offset is a constant
template <int c>
__device__ __forceinline__ float4 voffdiag_k(const VLevel& L, const VNbSh& sh, int t, const float* x,
                                             const VCoef& k, float4& xc) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    xc = uload4(x, L, c, sh, X, Y, Z0, 0, 0, 0);
    float4 fr[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const float4 up = uload4(x, L, c, sh, X, Y, Z0, px, py, pz);
        const float4 um = uload4(x, L, c, sh, X, Y, Z0, -px, -py, -pz);
        const float4 wp = k.wp[ax], wm = k.wm[ax];
        fr[2 * ax] = make_float4(__fmul_rn(up.x, wp.x), __fmul_rn(up.y, wp.y), __fmul_rn(up.z, wp.z),
                                 __fmul_rn(up.w, wp.w));
        fr[2 * ax + 1] = make_float4(__fmul_rn(um.x, wm.x), __fmul_rn(um.y, wm.y), __fmul_rn(um.z, wm.z),
                                     __fmul_rn(um.w, wm.w));
    }
    const float4 u1_g = uload4(x, L, d1, sh, X, Y, Z0, 0, 0, 0);
    const float4 u1_p1 = uload4(x, L, d1, sh, X, Y, Z0, e1[0], e1[1], e1[2]);
    const float4 u1_m0 = uload4(x, L, d1, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u1_m0p1 = uload4(x, L, d1, sh, X, Y, Z0, e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]);
    const float4 u2_g = uload4(x, L, d2, sh, X, Y, Z0, 0, 0, 0);
    const float4 u2_m0 = uload4(x, L, d2, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u2_p2 = uload4(x, L, d2, sh, X, Y, Z0, e2[0], e2[1], e2[2]);
    const float4 u2_m0p2 = uload4(x, L, d2, sh, X, Y, Z0, e2[0] - e0[0], e2[1] - e0[1], e2[2] - e0[2]);
    float4 off;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float f1 = __fadd_rn(f4get(fr[0], j), f4get(fr[1], j));
        float f3 = __fadd_rn(f4get(fr[2], j), f4get(fr[3], j));
        float f5 = __fadd_rn(f4get(fr[4], j), f4get(fr[5], j));
        f1 = __fadd_rn(f1, f3);
        f1 = __fadd_rn(f1, f5);
        const float R0 = __fmul_rn(f4get(u1_g, j), f4get(k.a00, j));
        const float R1 = __fmul_rn(f4get(k.a01, j), f4get(u1_p1, j));
        const float R2 = __fmul_rn(f4get(k.a10, j), f4get(u1_m0, j));
        const float R3 = __fmul_rn(f4get(k.a11, j), f4get(u1_m0p1, j));
        const float Q0 = __fmul_rn(f4get(k.b00, j), f4get(u2_g, j));
        const float Q1 = __fmul_rn(f4get(k.b01, j), f4get(u2_m0, j));
        const float Q2 = __fmul_rn(f4get(k.b10, j), f4get(u2_p2, j));
        const float Q3 = __fmul_rn(f4get(k.b11, j), f4get(u2_m0p2, j));
        const float td2 = __fadd_rn(__fadd_rn(R0, R1), __fadd_rn(R2, R3));
        const float td1 = __fadd_rn(__fadd_rn(Q0, Q1), __fadd_rn(Q2, Q3));
        f1 = __fadd_rn(f1, td2);
        f1 = __fadd_rn(f1, td1);
        f4set(off, j, f1);
    }
    return off;
}

// vapply_value with the coefficients already loaded
template <int MODE, int c>
__device__ __forceinline__ float4 vapply_value_k(const VLevel& L, const VNbSh& sh, int t, const float* x,
                                                 const float* b, float w, unsigned m, const VCoef& k, float4& xc) {
    const float4 off = voffdiag_k<c>(L, sh, t, x, k, xc);
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 res = xc;
    if (MODE == VM_RED || MODE == VM_BLACK) {
        const float4 bb = uload4(b, L, c, sh, X, Y, Z0, 0, 0, 0);
        const float4 iv = k.dg;
        const float one_minus_w = __fsub_rn(1.0f, w);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int par = (X + Y + Z0 + j) & 1;
            const bool upd = (MODE == VM_RED) ? (par == 0) : (par == 1);
            float r = __fsub_rn(f4get(bb, j), f4get(off, j));
            r = __fmul_rn(r, f4get(iv, j));
            r = __fmul_rn(r, w);
            const float v = __fmaf_rn(f4get(xc, j), one_minus_w, r);
            f4set(res, j, upd ? v : f4get(xc, j));
        }
    } else if (MODE == VM_NORMAL) {
#pragma unroll
        for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(k.dg, j), f4get(off, j)));
    } else if (MODE == VM_RESIDUAL) {
        const float4 bb = uload4(b, L, c, sh, X, Y, Z0, 0, 0, 0);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(k.dg, j), f4get(off, j))));
    } else {  // JACOBI: diag from memory, 1/diag preloaded
        const float4 bb = uload4(b, L, c, sh, X, Y, Z0, 0, 0, 0);
        const float4 dg = cload4(varr(L, c, VA_DIAG), sh, X, Y, Z0, 0, 0, 0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
            r = __fmul_rn(r, f4get(k.dg, j));
            f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
        }
    }
    if (!(m & 1)) res.x = 0.f;
    if (!(m & 2)) res.y = 0.f;
    if (!(m & 4)) res.z = 0.f;
    if (!(m & 8)) res.w = 0.f;
    return res;
}

// One applier pass for channel c at the thread's voxels; m = DOF bits.
template <int MODE>
__device__ __forceinline__ float4 vapply_value(const VLevel& L, const VNbSh& sh, int c, int t, const float* x,
                                               const float* b, float w, unsigned m, float4& xc) {
    const float4 off = voffdiag(L, sh, c, t, x, xc);
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 res = xc;
    if (MODE == VM_RED || MODE == VM_BLACK) {
        const float4 bb = uload4(b, L, c, sh, X, Y, Z0, 0, 0, 0);
        const float4 iv = cload4(varr(L, c, VA_INV), sh, X, Y, Z0, 0, 0, 0);
        const float one_minus_w = __fsub_rn(1.0f, w);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int par = (X + Y + Z0 + j) & 1;
            const bool upd = (MODE == VM_RED) ? (par == 0) : (par == 1);
            float r = __fsub_rn(f4get(bb, j), f4get(off, j));
            r = __fmul_rn(r, f4get(iv, j));
            r = __fmul_rn(r, w);
            const float v = __fmaf_rn(f4get(xc, j), one_minus_w, r);
            f4set(res, j, upd ? v : f4get(xc, j));
        }
    } else {
        const float4 dg = cload4(varr(L, c, VA_DIAG), sh, X, Y, Z0, 0, 0, 0);
        if (MODE == VM_NORMAL) {
#pragma unroll
            for (int j = 0; j < 4; ++j) f4set(res, j, __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
        } else {
            const float4 bb = uload4(b, L, c, sh, X, Y, Z0, 0, 0, 0);
            if (MODE == VM_RESIDUAL) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    f4set(res, j, __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j))));
            } else {  // JACOBI
                const float4 iv = cload4(varr(L, c, VA_INV), sh, X, Y, Z0, 0, 0, 0);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float r = __fsub_rn(f4get(bb, j), __fmaf_rn(f4get(xc, j), f4get(dg, j), f4get(off, j)));
                    r = __fmul_rn(r, f4get(iv, j));
                    f4set(res, j, __fmaf_rn(w, r, f4get(xc, j)));
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

// One applier pass over one leaf and channel c (a constant); m = DOF bits.
// Static data first (DOF mask, neighbourhood, coefficients): they are not
// written during a solve, so they load while the previous kernel is still
// running; the vectors are read after griddepcontrol.wait.
template <int MODE, int c>
__device__ __forceinline__ void vapply_leaf(const VLevel& L, VNbSh& sh, int leaf, const float* x, const float* b,
                                            float* out, float w) {
    const int t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    vnb_prologue(L, leaf, sh);
    VCoef k;
    if (m) vload_coef<MODE, c>(L, sh, t, k);
    griddep_wait();
    griddep_launch();
    if (!m) return;
    float4 xc;
    const float4 res = vapply_value_k<MODE, c>(L, sh, t, x, b, w, m, k, xc);
    reinterpret_cast<float4*>(out + (long long)c * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = res;
}

#ifndef VAPPLY_MINB
#define VAPPLY_MINB 3  // CTAs per SM: no register spills (fewer registers spill and run slower)
#endif
// RED / BLACK: one channel C, grid (nl), x updated in place (out == x).
// NORMAL / RESIDUAL / JACOBI: C = -1, grid (nl, 3), blockIdx.y = channel.
// Voxel groups without DOFs are not written: every vector holds zeros there.
template <int MODE, int C>
__global__ void __launch_bounds__(128, VAPPLY_MINB) k_vapply(VLevel L, const float* x, const float* b, float* out,
                                                             float w) {
    __shared__ VNbSh sh;
    const int leaf = blockIdx.x;
    if constexpr (C >= 0) {
        vapply_leaf<MODE, C>(L, sh, leaf, x, b, out, w);
    } else {
        if (blockIdx.y == 0) vapply_leaf<MODE, 0>(L, sh, leaf, x, b, out, w);
        else if (blockIdx.y == 1) vapply_leaf<MODE, 1>(L, sh, leaf, x, b, out, w);
        else vapply_leaf<MODE, 2>(L, sh, leaf, x, b, out, w);
    }
}

// ---------------------------------------------------------------------------
// One red-black Gauss-Seidel step of one channel in one launch: the first
// colour's update followed by the second's (XYZ_RBGS_apply runs red then black
// per channel, ZYX_RBGS_apply black then red; simd_viscosity3d.cpp:2238-2302).
//
// The first-colour update at a voxel reads only second-colour values of its
// own channel and the other two channels, none of which that update changes,
// so a CTA can compute it for its own leaf and for the first-colour voxels of
// the six face layers around it (the ones its second-colour voxels read),
// which the neighbouring CTAs compute as well from the same inputs in the same
// order: bit-identical values, no exchange between CTAs.  The second colour
// then reads its same-channel neighbours from shared memory; its cross-channel
// sums are the first colour's, kept in registers.  The step reads channel c
// from one buffer and writes it to another (neighbouring CTAs still read the
// old values), so a pair of steps over the three channels ends where it began.
//
// Threads: 0-127 the leaf's 4-voxel groups (as k_vapply); 128-191 the groups
// of the -x, +x, -y, +y face layers (x or y = -1 or 8, z0 = 0 or 4); 192-255
// the first-colour voxels of the -z and +z layers, one each.
struct VRbIo {
    const float* xc;  // channel c before the step
    const float* x1;  // channel (c + 1) % 3
    const float* x2;  // channel (c + 2) % 3
    const float* b;   // channel c of the right-hand side
    float* out;       // channel c after the step
};
#define VRB_THREADS 256
#ifndef VRB_MINB
#define VRB_MINB 2
#endif
#define VRB_HALO 10  // shared-memory cube: the leaf and one voxel around it
__device__ __forceinline__ int vrb_idx(int X, int Y, int Z) {
    return ((X + 1) * VRB_HALO + (Y + 1)) * VRB_HALO + (Z + 1);
}

// faced_result[1] of one voxel from its seven products and two cross sums,
// in the order of voffdiag
__device__ __forceinline__ float vsum_off(float p0, float p1, float p2, float p3, float p4, float p5, float td2,
                                          float td1) {
    float f1 = __fadd_rn(p0, p1);
    const float f3 = __fadd_rn(p2, p3);
    const float f5 = __fadd_rn(p4, p5);
    f1 = __fadd_rn(f1, f3);
    f1 = __fadd_rn(f1, f5);
    f1 = __fadd_rn(f1, td2);
    return __fadd_rn(f1, td1);
}
// Gauss-Seidel update of vapply_value_k
__device__ __forceinline__ float vgs_update(float bb, float off, float iv, float w, float one_minus_w, float xc) {
    float r = __fsub_rn(bb, off);
    r = __fmul_rn(r, iv);
    r = __fmul_rn(r, w);
    return __fmaf_rn(xc, one_minus_w, r);
}
template <bool COEF = false>
__device__ __forceinline__ float vload1(const float* arr, const float* fb, const VNbSh& sh, int X, int Y, int Z) {
    return vsel<COEF>(arr, fb, sh, vnb_index(X, Y, Z))[voff3(X, Y, Z)];
}

// Cross-channel sums (td2, td1 of voffdiag) at a 4-voxel group.
template <int c>
__device__ __forceinline__ void vcross4(const VLevel& L, const VNbSh& sh, const VRbIo& io, int X, int Y, int Z0,
                                        const VCoef& k, float4& td2, float4& td1) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    const float* zp = L.zpage;
    const float4 u1_g = vload4(io.x1, zp, sh, X, Y, Z0, 0, 0, 0);
    const float4 u1_p1 = vload4(io.x1, zp, sh, X, Y, Z0, e1[0], e1[1], e1[2]);
    const float4 u1_m0 = vload4(io.x1, zp, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u1_m0p1 = vload4(io.x1, zp, sh, X, Y, Z0, e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]);
    const float4 u2_g = vload4(io.x2, zp, sh, X, Y, Z0, 0, 0, 0);
    const float4 u2_m0 = vload4(io.x2, zp, sh, X, Y, Z0, -e0[0], -e0[1], -e0[2]);
    const float4 u2_p2 = vload4(io.x2, zp, sh, X, Y, Z0, e2[0], e2[1], e2[2]);
    const float4 u2_m0p2 = vload4(io.x2, zp, sh, X, Y, Z0, e2[0] - e0[0], e2[1] - e0[1], e2[2] - e0[2]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float R0 = __fmul_rn(f4get(u1_g, j), f4get(k.a00, j));
        const float R1 = __fmul_rn(f4get(k.a01, j), f4get(u1_p1, j));
        const float R2 = __fmul_rn(f4get(k.a10, j), f4get(u1_m0, j));
        const float R3 = __fmul_rn(f4get(k.a11, j), f4get(u1_m0p1, j));
        const float Q0 = __fmul_rn(f4get(k.b00, j), f4get(u2_g, j));
        const float Q1 = __fmul_rn(f4get(k.b01, j), f4get(u2_m0, j));
        const float Q2 = __fmul_rn(f4get(k.b10, j), f4get(u2_p2, j));
        const float Q3 = __fmul_rn(f4get(k.b11, j), f4get(u2_m0p2, j));
        f4set(td2, j, __fadd_rn(__fadd_rn(R0, R1), __fadd_rn(R2, R3)));
        f4set(td1, j, __fadd_rn(__fadd_rn(Q0, Q1), __fadd_rn(Q2, Q3)));
    }
}

// First-colour update of a 4-voxel group (lanes of the other colour keep xc);
// m = DOF bits of the group, non-DOF lanes 0.
template <int c, int FP>
__device__ __forceinline__ float4 vrb_first4(const VLevel& L, const VNbSh& sh, const VRbIo& io, int X, int Y,
                                             int Z0, unsigned m, float w, const VCoef& k, float4& td2, float4& td1,
                                             float4& bb) {
    const float* zp = L.zpage;
    const float4 xc = vload4(io.xc, zp, sh, X, Y, Z0, 0, 0, 0);
    float4 fr[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const float4 up = vload4(io.xc, zp, sh, X, Y, Z0, px, py, pz);
        const float4 um = vload4(io.xc, zp, sh, X, Y, Z0, -px, -py, -pz);
        fr[2 * ax] = make_float4(__fmul_rn(up.x, k.wp[ax].x), __fmul_rn(up.y, k.wp[ax].y),
                                 __fmul_rn(up.z, k.wp[ax].z), __fmul_rn(up.w, k.wp[ax].w));
        fr[2 * ax + 1] = make_float4(__fmul_rn(um.x, k.wm[ax].x), __fmul_rn(um.y, k.wm[ax].y),
                                     __fmul_rn(um.z, k.wm[ax].z), __fmul_rn(um.w, k.wm[ax].w));
    }
    vcross4<c>(L, sh, io, X, Y, Z0, k, td2, td1);
    bb = vload4(io.b, zp, sh, X, Y, Z0, 0, 0, 0);
    const float one_minus_w = __fsub_rn(1.0f, w);
    float4 res;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float off = vsum_off(f4get(fr[0], j), f4get(fr[1], j), f4get(fr[2], j), f4get(fr[3], j),
                                   f4get(fr[4], j), f4get(fr[5], j), f4get(td2, j), f4get(td1, j));
        const bool upd = ((X + Y + Z0 + j) & 1) == FP;
        const float v = vgs_update(f4get(bb, j), off, f4get(k.dg, j), w, one_minus_w, f4get(xc, j));
        f4set(res, j, (m >> j & 1) ? (upd ? v : f4get(xc, j)) : 0.f);
    }
    return res;
}

// The coefficients of one voxel (VCoef's fifteen values).
struct VCoef1 {
    float wp[3], wm[3], a00, a01, a10, a11, b00, b01, b10, b11, iv;
};
template <int c>
__device__ __forceinline__ void vload_coef1(const VLevel& L, const VNbSh& sh, int X, int Y, int Z, VCoef1& k) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    int e0[3] = {0, 0, 0};
    e0[d0] = 1;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        const VArr W = varr(L, c, VA_NEGX + ax);
        k.wp[ax] = vload1<true>(W.a, W.def, sh, X + px, Y + py, Z + pz);
        k.wm[ax] = vload1<true>(W.a, W.def, sh, X, Y, Z);
    }
    const VArr A00 = varr(L, d2, VA_T00), A01 = varr(L, d2, VA_T01), A10 = varr(L, d2, VA_T10),
               A11 = varr(L, d2, VA_T11), B00 = varr(L, d1, VA_T00), B01 = varr(L, d1, VA_T01),
               B10 = varr(L, d1, VA_T10), B11 = varr(L, d1, VA_T11), IV = varr(L, c, VA_INV);
    const int Xm = X - e0[0], Ym = Y - e0[1], Zm = Z - e0[2];
    k.a00 = vload1<true>(A00.a, A00.def, sh, X, Y, Z);
    k.a01 = vload1<true>(A01.a, A01.def, sh, X, Y, Z);
    k.a10 = vload1<true>(A10.a, A10.def, sh, Xm, Ym, Zm);
    k.a11 = vload1<true>(A11.a, A11.def, sh, Xm, Ym, Zm);
    k.b00 = vload1<true>(B00.a, B00.def, sh, X, Y, Z);
    k.b01 = vload1<true>(B01.a, B01.def, sh, Xm, Ym, Zm);
    k.b10 = vload1<true>(B10.a, B10.def, sh, X, Y, Z);
    k.b11 = vload1<true>(B11.a, B11.def, sh, Xm, Ym, Zm);
    k.iv = vload1<true>(IV.a, IV.def, sh, X, Y, Z);
}
// First-colour update of one DOF voxel (X, Y, Z), one of them -1 or 8.
template <int c>
__device__ __forceinline__ float vrb_first1(const VLevel& L, const VNbSh& sh, const VRbIo& io, int X, int Y, int Z,
                                            float w, const VCoef1& k) {
    constexpr int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    const float* zp = L.zpage;
    const float xc = vload1(io.xc, zp, sh, X, Y, Z);
    float fr[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int px = ax == 0, py = ax == 1, pz = ax == 2;
        fr[2 * ax] = __fmul_rn(vload1(io.xc, zp, sh, X + px, Y + py, Z + pz), k.wp[ax]);
        fr[2 * ax + 1] = __fmul_rn(vload1(io.xc, zp, sh, X - px, Y - py, Z - pz), k.wm[ax]);
    }
    const int Xm = X - e0[0], Ym = Y - e0[1], Zm = Z - e0[2];
    const float u1_g = vload1(io.x1, zp, sh, X, Y, Z);
    const float u1_p1 = vload1(io.x1, zp, sh, X + e1[0], Y + e1[1], Z + e1[2]);
    const float u1_m0 = vload1(io.x1, zp, sh, Xm, Ym, Zm);
    const float u1_m0p1 = vload1(io.x1, zp, sh, Xm + e1[0], Ym + e1[1], Zm + e1[2]);
    const float u2_g = vload1(io.x2, zp, sh, X, Y, Z);
    const float u2_m0 = vload1(io.x2, zp, sh, Xm, Ym, Zm);
    const float u2_p2 = vload1(io.x2, zp, sh, X + e2[0], Y + e2[1], Z + e2[2]);
    const float u2_m0p2 = vload1(io.x2, zp, sh, Xm + e2[0], Ym + e2[1], Zm + e2[2]);
    const float bb = vload1(io.b, zp, sh, X, Y, Z);
    const float R0 = __fmul_rn(u1_g, k.a00);
    const float R1 = __fmul_rn(k.a01, u1_p1);
    const float R2 = __fmul_rn(k.a10, u1_m0);
    const float R3 = __fmul_rn(k.a11, u1_m0p1);
    const float Q0 = __fmul_rn(k.b00, u2_g);
    const float Q1 = __fmul_rn(k.b01, u2_m0);
    const float Q2 = __fmul_rn(k.b10, u2_p2);
    const float Q3 = __fmul_rn(k.b11, u2_m0p2);
    const float td2 = __fadd_rn(__fadd_rn(R0, R1), __fadd_rn(R2, R3));
    const float td1 = __fadd_rn(__fadd_rn(Q0, Q1), __fadd_rn(Q2, Q3));
    const float off = vsum_off(fr[0], fr[1], fr[2], fr[3], fr[4], fr[5], td2, td1);
    return vgs_update(bb, off, k.iv, w, __fsub_rn(1.0f, w), xc);
}

// FP: parity of the first colour (0 red first, XYZ order; 1 black first, ZYX).
// grid (nl), VRB_THREADS threads.
template <int c, int FP>
__global__ void __launch_bounds__(VRB_THREADS, VRB_MINB) k_vrbgs(VLevel L, VRbIo io, float w) {
    __shared__ VNbSh sh;
    __shared__ float cur[VRB_HALO * VRB_HALO * VRB_HALO];
    const int t = threadIdx.x;
    const int leaf = blockIdx.x;
    vnb_prologue(L, leaf, sh);
    // static data before the wait: group / voxel coordinates, DOF bits, coefficients
    int X, Y, Z0;
    unsigned m = 0;
    VCoef k;
    VCoef1 k1;
    if (t < 128) {
        X = t >> 4;
        Y = (t >> 1) & 7;
        Z0 = (t & 1) * 4;
        m = vmask4(L, c, leaf, t);
        if (m) vload_coef_at<c>(L, sh, X, Y, Z0, true, k);
    } else if (t < 192) {
        const int h = t - 128, face = h >> 4, u = (h >> 1) & 7;
        Z0 = (h & 1) * 4;
        if (face < 2) {
            X = face ? 8 : -1;
            Y = u;
        } else {
            X = u;
            Y = face == 3 ? 8 : -1;
        }
        const int lf = sh.nb[vnb_index(X, Y, Z0)];
        if (lf >= 0) {
            const int tg = ((X & 7) << 4) | ((Y & 7) << 1) | (Z0 >> 2);
            m = vmask4(L, c, lf, tg);
        }
        if (m) vload_coef_at<c>(L, sh, X, Y, Z0, true, k);
    } else {
        const int h = t - 192, i = h & 31;
        Z0 = (h >> 5) ? 8 : -1;  // the voxel's z
        X = i >> 2;
        Y = 2 * (i & 3) + ((FP + Z0 + X) & 1);
        const int lf = sh.nb[vnb_index(X, Y, Z0)];
        if (lf >= 0 && vdof_bit(L, c, lf, voff3(X, Y, Z0))) m = 1;
        if (m) vload_coef1<c>(L, sh, X, Y, Z0, k1);
    }
    griddep_wait();
    griddep_launch();
    // first colour: every first-colour position of the cube is written (0 where
    // there is no DOF), the only positions the second colour reads
    float4 td2, td1, bb, res = f4zero();
    if (t < 192) {
        if (m) res = vrb_first4<c, FP>(L, sh, io, X, Y, Z0, m, w, k, td2, td1, bb);
        const int base = vrb_idx(X, Y, Z0);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (((X + Y + Z0 + j) & 1) == FP) cur[base + j] = f4get(res, j);
    } else {
        cur[vrb_idx(X, Y, Z0)] = m ? vrb_first1<c>(L, sh, io, X, Y, Z0, w, k1) : 0.f;
    }
    __syncthreads();
    if (t >= 128 || !m) return;
    // second colour: same-channel neighbours (all first colour) from shared memory
    const float one_minus_w = __fsub_rn(1.0f, w);
    float4 out = res;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int Z = Z0 + j;
        if (((X + Y + Z) & 1) == FP || !(m >> j & 1)) continue;
        const float p0 = __fmul_rn(cur[vrb_idx(X + 1, Y, Z)], f4get(k.wp[0], j));
        const float p1 = __fmul_rn(cur[vrb_idx(X - 1, Y, Z)], f4get(k.wm[0], j));
        const float p2 = __fmul_rn(cur[vrb_idx(X, Y + 1, Z)], f4get(k.wp[1], j));
        const float p3 = __fmul_rn(cur[vrb_idx(X, Y - 1, Z)], f4get(k.wm[1], j));
        const float p4 = __fmul_rn(cur[vrb_idx(X, Y, Z + 1)], f4get(k.wp[2], j));
        const float p5 = __fmul_rn(cur[vrb_idx(X, Y, Z - 1)], f4get(k.wm[2], j));
        const float off = vsum_off(p0, p1, p2, p3, p4, p5, f4get(td2, j), f4get(td1, j));
        f4set(out, j, vgs_update(f4get(bb, j), off, f4get(k.dg, j), w, one_minus_w, f4get(res, j)));
    }
    reinterpret_cast<float4*>(io.out)[(long long)leaf * UAAMG_LEAF4 + t] = out;
}

// k_vapply<RED / BLACK, c> over many leaves: a grid of a few CTAs per SM, each
// looping over leaves blockIdx.x, blockIdx.x + gridDim.x, ...  A one-leaf CTA
// starts with a dependent chain (neighbour table into shared memory, barrier,
// then the coefficient and vector loads); here the next leaf's table entries
// and DOF bits load while the current leaf computes, so every leaf after the
// first starts at its coefficient loads.  Same per-voxel arithmetic as
// k_vapply.
template <int MODE, int c>
__global__ void __launch_bounds__(128, VAPPLY_MINB) k_vapply_seq(VLevel L, const float* x, const float* b, float* out,
                                                                 float w) {
    __shared__ VNbSh sh[2];
    const int t = threadIdx.x;
    int leaf = blockIdx.x;
    unsigned m = 0;
    if (leaf < L.nl) {
        if (t < 27) {
            const int v = L.nb[(long long)leaf * 27 + t];
            sh[0].nb[t] = v;
            sh[0].cnb[t] = L.cnb ? L.cnb[(long long)leaf * 27 + t] : v;
        }
        m = vmask4(L, c, leaf, t);
    }
    __syncthreads();
    bool waited = false;
    for (int it = 0; leaf < L.nl; ++it, leaf += gridDim.x) {
        const VNbSh& cur = sh[it & 1];
        const int next = leaf + (int)gridDim.x;
        int nb_n = -1, cnb_n = -1;
        unsigned m_n = 0;
        if (next < L.nl) {
            if (t < 27) {
                nb_n = L.nb[(long long)next * 27 + t];
                cnb_n = L.cnb ? L.cnb[(long long)next * 27 + t] : nb_n;
            }
            m_n = vmask4(L, c, next, t);
        }
        VCoef k;
        if (m) vload_coef<MODE, c>(L, cur, t, k);
        if (!waited) {
            griddep_wait();
            griddep_launch();
            waited = true;
        }
        if (m) {
            float4 xc;
            const float4 res = vapply_value_k<MODE, c>(L, cur, t, x, b, w, m, k, xc);
            reinterpret_cast<float4*>(out + (long long)c * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = res;
        }
        if (t < 27) {
            sh[(it + 1) & 1].nb[t] = nb_n;
            sh[(it + 1) & 1].cnb[t] = cnb_n;
        }
        m = m_n;
        __syncthreads();
    }
    if (!waited) {
        griddep_wait();
        griddep_launch();
    }
}

// restriction (:2353-2413) for one (coarse leaf, channel): coarse = (sum of the
// DOF children) * 0.125 * 0.5 * 2, zero at coarse non-DOF voxels
__device__ __forceinline__ void vrestrict_item(const VLevel& F, const VLevel& C, const float* fine, float* coarse,
                                               int leaf, int c, int t) {
    // static data (masks, child table) before the wait for the fine vector
    const unsigned m = vmask4(C, c, leaf, t);
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int fl = -1;
    uint64_t fw[2] = {0ull, 0ull};  // fine DOF mask words of planes 2X, 2X+1
    if (m) {
        const int q = ((X >= 4) << 2) | ((Y >= 4) << 1) | (Z0 >= 4);
        fl = C.child[leaf * 8 + q];
        if (fl >= 0) {
            const uint64_t* fm = F.dof + ((long long)c * F.nl + fl) * 8;
            fw[0] = fm[(2 * X) & 7];
            fw[1] = fm[(2 * X + 1) & 7];
        }
    }
    griddep_wait();
    griddep_launch();
    float4 res = f4zero();
    if (m && fl >= 0) {
        const float* fv = fine + ((long long)c * F.nl + fl) * UAAMG_LEAF;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!(m >> j & 1)) continue;
            const int base = voff3(2 * X, 2 * Y, 2 * (Z0 + j));
            float s = 0.f;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int bq = 0; bq < 2; ++bq)
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        const int fo = base + 64 * a + 8 * bq + k;
                        if ((fw[a] >> (fo & 63)) & 1ull) s = __fadd_rn(s, fv[fo]);
                    }
            f4set(res, j, __fmul_rn(__fmul_rn(__fmul_rn(s, 0.125f), 0.5f), 2.0f));
        }
    }
    reinterpret_cast<float4*>(coarse + (long long)c * C.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = res;
}
__global__ void __launch_bounds__(128) k_vrestrict(VLevel F, VLevel C, const float* fine, float* coarse) {
    vrestrict_item(F, C, fine, coarse, blockIdx.x, blockIdx.y, threadIdx.x);
}

// residual_apply followed by restriction (the two steps of a mu-cycle visit
// before the coarse visits, :3837-3884) in one pass over the fine leaves: a
// CTA computes the residual of its fine leaf in shared memory and writes the
// restricted values of its octant of the parent leaf.  Same operations and
// summation order as k_vapply<VM_RESIDUAL> + k_vrestrict; the coarse voxels of
// octants without a fine leaf are never written (they hold no DOF, and the
// coarse rhs is zero there from allocation).
template <int c>
__device__ __forceinline__ void vresrestrict_leaf(const VLevel& F, const VLevel& C, VNbSh& sh, float* rs, int leaf,
                                                  const float* x, const float* b, float* coarse, float* coarse_lhs) {
    const int t = threadIdx.x;
    const unsigned m = vmask4(F, c, leaf, t);
    vnb_prologue(F, leaf, sh);
    VCoef k;
    if (m) vload_coef<VM_RESIDUAL, c>(F, sh, t, k);
    // static: parent, octant, the DOF mask words of this thread's coarse
    // voxel (t < 64: one of the 4x4x4 coarse voxels of the octant)
    const int P = F.parent[leaf];
    const int oc = F.octant[leaf];
    const int ci = t >> 4, cj = (t >> 2) & 3, ck = t & 3;
    const int cx = ((oc >> 2) & 1) * 4 + ci, cy = ((oc >> 1) & 1) * 4 + cj, cz = (oc & 1) * 4 + ck;
    bool cdof = false;
    uint64_t fw[2] = {0ull, 0ull};
    if (t < 64 && P >= 0) {
        cdof = vdof_bit(C, c, P, voff3(cx, cy, cz));
        const uint64_t* fm = F.dof + ((long long)c * F.nl + leaf) * 8;
        fw[0] = fm[2 * ci];
        fw[1] = fm[2 * ci + 1];
    }
    griddep_wait();
    griddep_launch();
    float4 res = f4zero();
    if (m) {
        float4 xc;
        res = vapply_value_k<VM_RESIDUAL, c>(F, sh, t, x, b, 1.f, m, k, xc);
    }
    reinterpret_cast<float4*>(rs)[t] = res;
    __syncthreads();
    if (t < 64 && P >= 0) {
        float s = 0.f;
        if (cdof) {
            const int base = voff3(2 * ci, 2 * cj, 2 * ck);
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int bq = 0; bq < 2; ++bq)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const int fo = base + 64 * a + 8 * bq + kk;
                        if ((fw[a] >> (fo & 63)) & 1ull) s = __fadd_rn(s, rs[fo]);
                    }
            s = __fmul_rn(__fmul_rn(__fmul_rn(s, 0.125f), 0.5f), 2.0f);
        }
        coarse[((long long)c * C.nl + P) * UAAMG_LEAF + voff3(cx, cy, cz)] = s;
        // the coarse visit that follows starts from zero: every coarse DOF of channel c lies in an octant whose
        // fine leaf has a DOF of c, so these writes cover them (the memset they replace was a graph node of its own)
        if (coarse_lhs) coarse_lhs[((long long)c * C.nl + P) * UAAMG_LEAF + voff3(cx, cy, cz)] = 0.f;
    }
}
__global__ void __launch_bounds__(128, VAPPLY_MINB) k_vresrestrict(VLevel F, VLevel C, const float* x, const float* b,
                                                                   float* coarse, float* coarse_lhs) {
    __shared__ VNbSh sh;
    __shared__ __align__(16) float rs[UAAMG_LEAF];
    const int leaf = blockIdx.x;
    if (blockIdx.y == 0) vresrestrict_leaf<0>(F, C, sh, rs, leaf, x, b, coarse, coarse_lhs);
    else if (blockIdx.y == 1) vresrestrict_leaf<1>(F, C, sh, rs, leaf, x, b, coarse, coarse_lhs);
    else vresrestrict_leaf<2>(F, C, sh, rs, leaf, x, b, coarse, coarse_lhs);
}

// v = 0 over n floats (grid-stride, float4), a kernel so that it keeps the
// chain of programmatic dependent launches
__global__ void __launch_bounds__(256) k_vzero(float4* v, long long n4) {
    griddep_wait();
    griddep_launch();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x)
        v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// prolongation<true> (:2659-2729) for one (fine leaf, channel): fine += coarse parent
__device__ __forceinline__ void vprolong_item(const VLevel& F, const VLevel& C, const float* coarse, float* fine,
                                              int leaf, int c, int t) {
    // static data (mask, parent, octant) before the wait for the vectors
    const unsigned m = vmask4(F, c, leaf, t);
    const int P = m ? F.parent[leaf] : -1;
    const int oc = m ? F.octant[leaf] : 0;
    griddep_wait();
    griddep_launch();
    if (!m || P < 0) return;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    const int cx = ((oc >> 2) & 1) * 4 + (X >> 1), cy = ((oc >> 1) & 1) * 4 + (Y >> 1);
    const float* cv = coarse + ((long long)c * C.nl + P) * UAAMG_LEAF;
    float4* fp = reinterpret_cast<float4*>(fine + (long long)c * F.nl * UAAMG_LEAF) + (long long)leaf * UAAMG_LEAF4 + t;
    float4 v = *fp;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!(m >> j & 1)) continue;
        const int cz = (oc & 1) * 4 + ((Z0 + j) >> 1);
        f4set(v, j, __fadd_rn(f4get(v, j), cv[(cx << 6) | (cy << 3) | cz]));
    }
    *fp = v;
}
__global__ void __launch_bounds__(128) k_vprolong(VLevel F, VLevel C, const float* coarse, float* fine) {
    vprolong_item(F, C, coarse, fine, blockIdx.x, blockIdx.y, threadIdx.x);
}

// zero every non-DOF voxel of a 3-channel vector (inputs from callers)
__global__ void __launch_bounds__(128) k_vmask(VLevel L, float* v) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    float4* p = reinterpret_cast<float4*>(v + (long long)c * L.nl * UAAMG_LEAF) + (long long)leaf * UAAMG_LEAF4 + t;
    if (m == 0xF) return;
    float4 a = *p;
    if (!(m & 1)) a.x = 0.f;
    if (!(m & 2)) a.y = 0.f;
    if (!(m & 4)) a.z = 0.f;
    if (!(m & 8)) a.w = 0.f;
    *p = a;
}

// ---------------------------------------------------------------------------
// PCG of simd_viscosity3d::pcg_solve (:3691-3754) with device-resident scalars.
// Reductions: per-block partials (FP64 for dots), the last block to arrive
// combines them in block order, so results do not depend on scheduling.
__device__ __forceinline__ bool vpublish(double part, double* partials, unsigned* ticket, bool* sh_last) {
    const unsigned bid = blockIdx.x + blockIdx.y * gridDim.x, nb = gridDim.x * gridDim.y;
    if (threadIdx.x == 0) {
        partials[bid] = part;
        __threadfence();
        const unsigned tk = atomicAdd(ticket, 1u);
        *sh_last = (tk == nb - 1);
    }
    __syncthreads();
    return *sh_last;
}
__device__ __forceinline__ double vgather_sum(const double* partials, double* sh) {
    const int nb = gridDim.x * gridDim.y;
    double acc = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += __ldcg(partials + i);
    return block_sum128(acc, sh);
}
__device__ __forceinline__ float vgather_max(const double* partials, float* sh) {
    const int nb = gridDim.x * gridDim.y;
    float acc = 0.f;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc = nanmax(acc, (float)__ldcg(partials + i));
    return block_max128(acc, sh);
}
__device__ __forceinline__ float vabs4(float4 v, unsigned m) {
    float a = 0.f;
    if (m & 1) a = nanmax(a, absprop(v.x));
    if (m & 2) a = nanmax(a, absprop(v.y));
    if (m & 4) a = nanmax(a, absprop(v.z));
    if (m & 8) a = nanmax(a, absprop(v.w));
    return a;
}

// lines 2-3: r = b - A x; nu = |r|_inf; numax = tol * nu
__global__ void __launch_bounds__(128) k_vpcg_init(VLevel L, const float* x, const float* b, float* r,
                                                   double* partials, PcgState* st, cudaGraphConditionalHandle cond,
                                                   int use_cond) {
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    __shared__ bool last;
    __shared__ VNbSh sh;
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    vnb_prologue(L, leaf, sh);
    float a = 0.f;
    if (m) {
        float4 xc;
        const float4 res = vapply_value<VM_RESIDUAL>(L, sh, c, t, x, b, 1.f, m, xc);
        reinterpret_cast<float4*>(r + (long long)c * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = res;
        a = vabs4(res, m);
    }
    const float part = block_max128(a, shf);
    if (vpublish((double)part, partials, &st->ticket[1], &last)) {
        const float nu = vgather_max(partials, shf);
        if (t == 0) {
            st->nu = nu;
            st->numax = __fmul_rn(st->tol, nu);
            st->iter = 0;
            st->first = 1;
            st->iterations_taken = 0;
            st->alpha = 0.f;
            st->beta = 0.f;
            int status = PCG_RUNNING;
            if (nu <= st->numax) status = PCG_SUCCESS;
            else if (st->max_iter <= 0) status = PCG_FAILED_MAXITER;  // loop never runs: x untouched
            st->status = status;
            st->ticket[1] = 0;
            set_cond(cond, use_cond, status == PCG_RUNNING ? 1u : 0u);
        }
    }
}

// lv_dot (:3769-3780) with grid_dot_op (openvdb_grid_math_op.h:45-75): float
// accumulation of a*b over the DOF voxels of a leaf in offset order, then of
// the leaf partials in leaf order per channel, then of the three channel
// sums.  (TBB may split the reference's sum anywhere; this is the serial
// schedule, so the PCG follows the reference's float rounding.)
// One kernel: a thread per (channel, leaf) item adds the products of its
// leaf's DOF voxels in offset order; the last CTA to finish (ticket) adds the
// item partials channel by channel in leaf order and updates the PCG scalar:
// which = 0: rho_new = z.r (line 13; first iteration: rho = rho_new, beta = 0,
// later beta = rho_new / rho, rho = rho_new); which = 1: sigma = p.q,
// alpha = rho / sigma (lines 6-7).
#define VDOT_THREADS 256
#define VDOT_ITEMS 16      // (channel, leaf) items per CTA
#define VDOT_CHUNK 2048
#define VDOT_PITCH 516     // product row pitch (floats): rows start in different banks, 16-byte aligned
// lv_dot (:3756-3835) in the reference's order: per (channel, leaf) item a
// sequential float sum of the DOF products in offset order, then the items
// of each channel in leaf order, then the three channel sums.  A CTA stages
// the products of VDOT_ITEMS consecutive items in shared memory with
// coalesced loads; one thread per item then adds them in order.  The CTA
// that finishes last adds the per-item sums (ticket).
__global__ void __launch_bounds__(VDOT_THREADS) k_vdot(VLevel L, const float* a, const float* b, float* part,
                                                       PcgState* st, int which) {
    __shared__ __align__(16) float buf[VDOT_ITEMS * VDOT_PITCH];  // products; reused as [3][VDOT_CHUNK]
    __shared__ uint64_t mw[VDOT_ITEMS][8];
    __shared__ float cs[3];
    __shared__ bool last;
    const int t = threadIdx.x;
    const long long nitems = 3LL * L.nl;
    const long long item0 = (long long)blockIdx.x * VDOT_ITEMS;
    if (t < VDOT_ITEMS * 8) {  // DOF masks: static, loaded before the wait
        const long long it = item0 + (t >> 3);
        mw[t >> 3][t & 7] = it < nitems ? L.dof[it * 8 + (t & 7)] : 0ull;
    }
    griddep_wait();
    griddep_launch();
    // products a*b of every voxel of the CTA's items (non-DOF entries are not read later)
#pragma unroll 4
    for (int k = t; k < VDOT_ITEMS * UAAMG_LEAF4; k += VDOT_THREADS) {
        const int li = k >> 7, q = k & 127;
        const long long it = item0 + li;
        float4 pr = f4zero();
        if (it < nitems) {
            const float4 x = reinterpret_cast<const float4*>(a + it * UAAMG_LEAF)[q];
            const float4 y = reinterpret_cast<const float4*>(b + it * UAAMG_LEAF)[q];
            pr = make_float4(__fmul_rn(x.x, y.x), __fmul_rn(x.y, y.y), __fmul_rn(x.z, y.z), __fmul_rn(x.w, y.w));
        }
        *reinterpret_cast<float4*>(buf + li * VDOT_PITCH + 4 * q) = pr;
    }
    __syncthreads();
    if (t < VDOT_ITEMS && item0 + t < nitems) {
        const float* pr = buf + t * VDOT_PITCH;
        float acc = 0.f;
        for (int q = 0; q < 8; ++q) {
            const uint64_t word = mw[t][q];
            if (!word) continue;
#pragma unroll
            for (int k = 0; k < 16; ++k) {  // DOF in offset order
                const unsigned nib = (unsigned)(word >> (4 * k)) & 0xFu;
                const float4 v = *reinterpret_cast<const float4*>(pr + q * 64 + 4 * k);
                if (nib & 1u) acc = __fadd_rn(acc, v.x);
                if (nib & 2u) acc = __fadd_rn(acc, v.y);
                if (nib & 4u) acc = __fadd_rn(acc, v.z);
                if (nib & 8u) acc = __fadd_rn(acc, v.w);
            }
        }
        part[item0 + t] = acc;
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = (atomicAdd(&st->ticket[5], 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    float* chunk = buf;  // [3][VDOT_CHUNK] (3 * 2048 <= 16 * 516)
    const int nl = L.nl;
    float acc = 0.f;  // thread c < 3: running sum of channel c
    for (int base = 0; base < nl; base += VDOT_CHUNK) {
        const int len = min(VDOT_CHUNK, nl - base);
        __syncthreads();
        for (int c = 0; c < 3; ++c)
            for (int i = t; i < len; i += VDOT_THREADS) chunk[c * VDOT_CHUNK + i] = __ldcg(part + (long long)c * nl + base + i);
        __syncthreads();
        if (t < 3) {
            const float* bb = chunk + t * VDOT_CHUNK;
            int i = 0;
            for (; i + 4 <= len; i += 4) {
                const float4 v = *reinterpret_cast<const float4*>(bb + i);
                acc = __fadd_rn(acc, v.x);
                acc = __fadd_rn(acc, v.y);
                acc = __fadd_rn(acc, v.z);
                acc = __fadd_rn(acc, v.w);
            }
            for (; i < len; ++i) acc = __fadd_rn(acc, bb[i]);
        }
    }
    if (t < 3) cs[t] = acc;
    __syncthreads();
    if (t == 0) {
        float r = 0.f;
        r = __fadd_rn(r, cs[0]);
        r = __fadd_rn(r, cs[1]);
        r = __fadd_rn(r, cs[2]);
        if (which == 0) {
            st->beta = st->first ? 0.f : __fdiv_rn(r, st->rho);
            st->rho = r;
        } else {
            st->sigma = r;
            st->alpha = __fdiv_rn(st->rho, r);
            st->first = 0;
        }
        st->ticket[5] = 0;
    }
}

// line 16: x += alpha p (not in the first iteration); p = z + beta p
__global__ void __launch_bounds__(128) k_vpcg_update_p(VLevel L, const float* z, float* p, float* x,
                                                       const PcgState* st) {
    // one grid-stride stream over the level's three channels (a few CTAs per
    // SM); non-DOF voxels hold 0 in x, p and z, and 0 + a * 0 keeps them 0
    griddep_wait();
    griddep_launch();
    const long long n4 = 3LL * L.nl * UAAMG_LEAF4;
    const float beta = st->beta, alpha = st->alpha;
    const bool first = st->first;
    float4* p4 = reinterpret_cast<float4*>(p);
    float4* x4 = reinterpret_cast<float4*>(x);
    const float4* z4 = reinterpret_cast<const float4*>(z);
#pragma unroll 2
    for (long long i = (long long)blockIdx.x * 128 + threadIdx.x; i < n4; i += (long long)gridDim.x * 128) {
        float4 pp = p4[i];
        const float4 zz = z4[i];
        if (!first) {
            float4 xx = x4[i];
            xx.x = __fadd_rn(xx.x, __fmul_rn(alpha, pp.x));
            xx.y = __fadd_rn(xx.y, __fmul_rn(alpha, pp.y));
            xx.z = __fadd_rn(xx.z, __fmul_rn(alpha, pp.z));
            xx.w = __fadd_rn(xx.w, __fmul_rn(alpha, pp.w));
            x4[i] = xx;
        }
        pp.x = __fadd_rn(zz.x, __fmul_rn(beta, pp.x));
        pp.y = __fadd_rn(zz.y, __fmul_rn(beta, pp.y));
        pp.z = __fadd_rn(zz.z, __fmul_rn(beta, pp.z));
        pp.w = __fadd_rn(zz.w, __fmul_rn(beta, pp.w));
        p4[i] = pp;
    }
}

// line 6: q = A p (sigma and alpha follow in k_vdot)
__global__ void __launch_bounds__(128) k_vpcg_Ap(VLevel L, const float* p, float* q) {
    __shared__ VNbSh sh;
    const int leaf = blockIdx.x;
    if (blockIdx.y == 0) vapply_leaf<VM_NORMAL, 0>(L, sh, leaf, p, nullptr, q, 1.f);
    else if (blockIdx.y == 1) vapply_leaf<VM_NORMAL, 1>(L, sh, leaf, p, nullptr, q, 1.f);
    else vapply_leaf<VM_NORMAL, 2>(L, sh, leaf, p, nullptr, q, 1.f);
}

// lines 8-9: r -= alpha q; nu = |r|_inf; stop when nu <= numax or at the
// last allowed iteration (no divergence test in this solver)
__global__ void __launch_bounds__(128) k_vpcg_update_r(VLevel L, const float* q, float* r, double* partials,
                                                       PcgState* st, cudaGraphConditionalHandle cond, int use_cond) {
    // one grid-stride stream over the level's three channels; non-DOF voxels
    // hold 0 in r and q (0 - alpha * 0 keeps them 0), so the max over every
    // voxel is the max over the DOFs
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    __shared__ bool last;
    const int t = threadIdx.x;
    const long long n4 = 3LL * L.nl * UAAMG_LEAF4;
    const float na = -st->alpha;
    float4* r4 = reinterpret_cast<float4*>(r);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    float a = 0.f;
#pragma unroll 2
    for (long long i = (long long)blockIdx.x * 128 + t; i < n4; i += (long long)gridDim.x * 128) {
        const float4 qq = q4[i];
        float4 rr = r4[i];
        rr.x = __fadd_rn(rr.x, __fmul_rn(na, qq.x));
        rr.y = __fadd_rn(rr.y, __fmul_rn(na, qq.y));
        rr.z = __fadd_rn(rr.z, __fmul_rn(na, qq.z));
        rr.w = __fadd_rn(rr.w, __fmul_rn(na, qq.w));
        r4[i] = rr;
        a = nanmax(a, vabs4(rr, 0xFu));
    }
    const float part = block_max128(a, shf);
    if (vpublish((double)part, partials, &st->ticket[4], &last)) {
        const float nu = vgather_max(partials, shf);
        if (t == 0) {
            const int k = st->iter;
            st->nu = nu;
            int status = PCG_RUNNING;
            if (nu <= st->numax) {
                status = PCG_SUCCESS;
                st->iterations_taken = k;
            } else if (k == st->max_iter - 1) {
                status = PCG_FAILED_MAXITER;
                st->iterations_taken = k;
            }
            st->iter = k + 1;
            st->status = status;
            st->ticket[4] = 0;
            set_cond(cond, use_cond, status == PCG_RUNNING ? 1u : 0u);
        }
    }
}

// line 10: x += alpha p after the stopping iteration
__global__ void __launch_bounds__(128) k_vpcg_finish(VLevel L, const float* p, float* x, const PcgState* st) {
    griddep_wait();
    griddep_launch();
    if (st->iter == 0) return;  // stopped before the loop
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const long long i = (long long)c * L.nl * UAAMG_LEAF4 + (long long)leaf * UAAMG_LEAF4 + t;
    const float alpha = st->alpha;
    const float4 pp = reinterpret_cast<const float4*>(p)[i];
    float4 xx = reinterpret_cast<float4*>(x)[i];
    xx.x = __fadd_rn(xx.x, __fmul_rn(alpha, pp.x));
    xx.y = __fadd_rn(xx.y, __fmul_rn(alpha, pp.y));
    xx.z = __fadd_rn(xx.z, __fmul_rn(alpha, pp.z));
    xx.w = __fadd_rn(xx.w, __fmul_rn(alpha, pp.w));
    reinterpret_cast<float4*>(x)[i] = xx;
}

// |v|_inf (lv_abs_max) or v.w (lv_dot) over a level, result in out[0]
__global__ void __launch_bounds__(128) k_vreduce(VLevel L, const float* v, const float* w, double* partials,
                                                 unsigned* ticket, float* out) {
    griddep_wait();
    griddep_launch();
    __shared__ float shf[4];
    __shared__ double shd[4];
    __shared__ bool last;
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    const long long i = (long long)c * L.nl * UAAMG_LEAF4 + (long long)leaf * UAAMG_LEAF4 + t;
    const float4 a = reinterpret_cast<const float4*>(v)[i];
    if (w) {
        const float4 bb = reinterpret_cast<const float4*>(w)[i];
        double s = 0.0;
        if (m & 1) s += (double)a.x * bb.x;
        if (m & 2) s += (double)a.y * bb.y;
        if (m & 4) s += (double)a.z * bb.z;
        if (m & 8) s += (double)a.w * bb.w;
        const double part = block_sum128(s, shd);
        if (vpublish(part, partials, ticket, &last)) {
            const double tot = vgather_sum(partials, shd);
            if (t == 0) { *out = (float)tot; *ticket = 0; }
        }
    } else {
        const float part = block_max128(vabs4(a, m), shf);
        if (vpublish((double)part, partials, ticket, &last)) {
            const float mx = vgather_max(partials, shf);
            if (t == 0) { *out = mx; *ticket = 0; }
        }
    }
}

// ---------------------------------------------------------------------------
// Coarsest level: Eigen::ConjugateGradient<RowMajor, Upper|Lower> with the
// diagonal preconditioner, tolerance FLT_EPSILON, maxIterations 10, zero guess
// (construct_exact_solver / solve_exact, :2645-2657), one CTA.  The explicit
// matrix rows (explicit_matrix_reducer, :2415-2605) are stored as an ELL of
// width 15 with columns ascending, the order of a RowMajor row after
// setFromTriplets.
#define VCG_W 15
struct DCoarsestV {
    int n;
    const long long* slot;  // [n] c*nl*512 + leaf*512 + offset
    const float* invd;      // [n] 1/diag (1 where diag == 0)
    const int* col;         // [n][15] (-1 = padding)
    const float* val;       // [n][15]
};

// Restatement of Eigen::ConjugateGradient (Upper|Lower, diagonal
// preconditioner, tolerance FLT_EPSILON, maxIterations 10, zero guess) on the
// coarsest level, one CTA of VCG_THREADS threads: row i = tid + k *
// VCG_THREADS, ROWS rows per thread.  With ROWS <= 4 a thread keeps its rows'
// ELL entries in registers for the whole solve; more rows read them through
// L1.  Few warps keep the three barriers and two reductions of an iteration
// short.
#define VCG_THREADS 256
#define VCG_WARPS (VCG_THREADS / 32)
// Block sums in one barrier: a shuffle-down tree inside each warp, then every
// thread adds the 8 warp sums from shared memory as ((w0+w1)+(w2+w3)) +
// ((w4+w5)+(w6+w7)) (cg_tree_sum), so every thread gets the same bits.
// buf: 16-byte aligned.
__device__ __forceinline__ float vcg_block_sum(float v, float* buf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = cg_warp_partial(v);
    if (lane == 0) buf[w] = v;
    __syncthreads();
    return cg_tree_sum<VCG_WARPS>(buf);
}
__device__ __forceinline__ float2 vcg_block_sum2(float a, float b, float* buf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    a = cg_warp_partial(a);
    b = cg_warp_partial(b);
    if (lane == 0) {
        buf[w] = a;
        buf[32 + w] = b;
    }
    __syncthreads();
    return make_float2(cg_tree_sum<VCG_WARPS>(buf), cg_tree_sum<VCG_WARPS>(buf + 32));
}

// Rows of ROWS <= 4 stay in registers with the shared-memory address of each
// entry's p (padding entries: value 0 at a slot that holds 0); larger systems
// read their rows from global memory each iteration.  A row's product is
// s = fma(v_e, p[c_e], s) over its VCG_W entries, padding included.
template <int ROWS>
__global__ void __launch_bounds__(VCG_THREADS, 1) k_vcoarsest_cg(DCoarsestV C, const float* rhs, float* out) {
    constexpr bool REG = ROWS <= 4;
    constexpr int ZERO = VCG_THREADS * ROWS;  // the zero slot
    __shared__ float ps[VCG_THREADS * ROWS + 4];
    __shared__ __align__(16) float red[3][64];
    const int tid = threadIdx.x, n = C.n;
    const unsigned psb = (unsigned)__cvta_generic_to_shared(ps);
    float x[ROWS], r[ROWS], p[ROWS], z[ROWS], iv[ROWS];
    unsigned rc[REG ? ROWS : 1][VCG_W];
    float rv[REG ? ROWS : 1][VCG_W];
    long long sl[ROWS];
    // static data (rows, 1/diag, slots) before the wait for rhs
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
        const int i = tid + k * VCG_THREADS;
        sl[k] = i < n ? C.slot[i] : -1;
        iv[k] = i < n ? C.invd[i] : 0.f;
        if (REG) {
#pragma unroll
            for (int e = 0; e < VCG_W; ++e) {
                const int cc = i < n ? __ldg(C.col + (long long)i * VCG_W + e) : -1;
                rc[REG ? k : 0][e] = psb + 4u * (unsigned)(cc >= 0 ? cc : ZERO);
                rv[REG ? k : 0][e] = cc >= 0 ? __ldg(C.val + (long long)i * VCG_W + e) : 0.f;
            }
        }
    }
    if (tid == 0) ps[ZERO] = 0.f;  // published by the first reduction's barrier
    griddep_wait();
    griddep_launch();
    float bb = 0.f;
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
        x[k] = 0.f;
        r[k] = sl[k] >= 0 ? rhs[sl[k]] : 0.f;
        p[k] = 0.f;
        bb = __fmaf_rn(r[k], r[k], bb);
    }
    int rb = 0;
    const float rhsNorm2 = vcg_block_sum(bb, red[rb]);
    rb = rb == 2 ? 0 : rb + 1;
    const float threshold = fmaxf(__fmul_rn(__fmul_rn(FLT_EPSILON, FLT_EPSILON), rhsNorm2), FLT_MIN);
    if (rhsNorm2 != 0.f && !(rhsNorm2 < threshold)) {
        float an = 0.f;
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            p[k] = __fmul_rn(iv[k], r[k]);
            an = __fmaf_rn(r[k], p[k], an);
        }
        float absNew = vcg_block_sum(an, red[rb]);
        rb = rb == 2 ? 0 : rb + 1;
        for (int it = 0; it < 10; ++it) {
#pragma unroll
            for (int k = 0; k < ROWS; ++k) ps[tid + k * VCG_THREADS] = p[k];
            __syncthreads();
            float pt = 0.f, tq[ROWS];
#pragma unroll
            for (int k = 0; k < ROWS; ++k) {
                const int i = tid + k * VCG_THREADS;
                float s = 0.f;
                if (REG) {
#pragma unroll
                    for (int e = 0; e < VCG_W; ++e) s = __fmaf_rn(rv[REG ? k : 0][e], lds_f32(rc[REG ? k : 0][e]), s);
                } else if (i < n) {
                    const int* cr = C.col + (long long)i * VCG_W;
                    const float* vr = C.val + (long long)i * VCG_W;
#pragma unroll
                    for (int e = 0; e < VCG_W; ++e) {
                        const int cc = __ldg(cr + e);
                        s = __fmaf_rn(cc >= 0 ? __ldg(vr + e) : 0.f, ps[cc >= 0 ? cc : ZERO], s);
                    }
                }
                tq[k] = s;
                pt = __fmaf_rn(p[k], s, pt);
            }
            const float alpha = __fdiv_rn(absNew, vcg_block_sum(pt, red[rb]));
            rb = rb == 2 ? 0 : rb + 1;
            float rr = 0.f, rz = 0.f;
#pragma unroll
            for (int k = 0; k < ROWS; ++k) {
                x[k] = __fmaf_rn(alpha, p[k], x[k]);
                r[k] = __fmaf_rn(-alpha, tq[k], r[k]);
                z[k] = __fmul_rn(iv[k], r[k]);
                rr = __fmaf_rn(r[k], r[k], rr);
                rz = __fmaf_rn(r[k], z[k], rz);
            }
            const float2 s2 = vcg_block_sum2(rr, rz, red[rb]);
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
        if (sl[k] >= 0) out[sl[k]] = x[k];
}

}  // namespace uaamg
