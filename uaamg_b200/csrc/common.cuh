// common.cuh -- shared definitions for the UAAMG-PCG CUDA library (sm_100a).
//
// Layout of every level in HBM (one "leaf" = one 8^3 block of the sparse grid,
// the unit OpenVDB also uses; voxel offset = 64x + 8y + z):
//   mask   uint64 [nl][8]        DOF value mask (word x holds the (y,z) plane x)
//   nbr    int32  [nl][6]        face-neighbour leaf (-x,+x,-y,+y,-z,+z), -1 if absent
//   coefficient and vector arrays float [nl][512], 2 KB contiguous per leaf
// A thread owns 4 consecutive z voxels (one float4); 128 threads cover a leaf.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define UAAMG_LEAF 512
#define UAAMG_LEAF4 128

// per-leaf "trimmed" flags: the leaf holds the level's default value for the
// array (LaplacianWithLevel::trimDefaultNodes), so kernels skip loading it.
#define TRIM_DIAG 1u
#define TRIM_X 2u
#define TRIM_Y 4u
#define TRIM_Z 8u
#define TRIM_SPAI0 16u

// PCG status word
#define PCG_RUNNING 0
#define PCG_SUCCESS 1
#define PCG_FAILED_DIVERGED 2
#define PCG_FAILED_MAXITER 3

struct DLevel {
    int nl;
    const uint64_t* mask;    // [nl][8]
    const int* nbr;          // [nl][6]
    const int* child;        // [nl][8] fine children (levels >= 1)
    const int* parent;       // [nl] coarse parent leaf (levels below the coarsest)
    const uint8_t* octant;   // [nl] position inside the parent leaf: x<<2 | y<<1 | z
    const float* diag;
    const float* cx;
    const float* cy;
    const float* cz;
    const float* invdiag;
    const float* spai0;
    const uint32_t* flags;   // [nl]
    float def_diag, def_face, def_invdiag, def_spai0;
};

// Scalars of the device-driven PCG (all in device memory so the whole solve
// can run inside one CUDA graph with a conditional WHILE node).
struct PcgState {
    float rho, rho_new, sigma, alpha, beta, nu, nu_old, numax;
    float tol;
    int iter, status, max_iter, first, iterations_taken;
    int error;  // set by a kernel whose bounded wait timed out
    unsigned int ticket[8];
};

__device__ __forceinline__ float4 f4zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float4 f4splat(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float f4get(const float4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}
__device__ __forceinline__ void f4set(float4& v, int j, float s) {
    if (j == 0) v.x = s; else if (j == 1) v.y = s; else if (j == 2) v.z = s; else v.w = s;
}
__device__ __forceinline__ float4 ld4(const float* p, long long leaf, int t) {
    return reinterpret_cast<const float4*>(p)[leaf * UAAMG_LEAF4 + t];
}
__device__ __forceinline__ void st4(float* p, long long leaf, int t, float4 v) {
    reinterpret_cast<float4*>(p)[leaf * UAAMG_LEAF4 + t] = v;
}
// 4 mask bits of thread t (voxels 4t..4t+3): word x = t>>4, bits (t&15)*4
__device__ __forceinline__ unsigned mask4(const uint64_t* mask, long long leaf, int t) {
    return (unsigned)((mask[leaf * 8 + (t >> 4)] >> ((t & 15) * 4)) & 0xFull);
}
