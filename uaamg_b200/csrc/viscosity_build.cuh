// viscosity_build.cuh -- sm_100a kernels that assemble the variational
// viscosity hierarchy (L_with_level, SIMD_UAAMG/simd_viscosity3d.cpp):
// subcell SDF and liquid volume fractions, control volumes, solid faces and
// DOFs, level-0 coefficients, Galerkin coarsening, default-leaf trimming, the
// coarsest explicit matrix and the right-hand side.  Float arithmetic follows
// the reference operation by operation (round-to-nearest intrinsics).
#pragma once
#include <float.h>

#include "poisson_build.cuh"
#include "viscosity_kernels.cuh"

namespace uaamg {

// Dense leaf-index volume of a leaf set (device copy of HostMap).
struct DMap {
    const int* map;
    int lo0, lo1, lo2, d0, d1, d2;
    __device__ __forceinline__ int find(int x, int y, int z) const {  // voxel coordinates
        if (!map) return -1;
        const int a = (x >> 3) - lo0, b = (y >> 3) - lo1, c = (z >> 3) - lo2;
        if ((unsigned)a >= (unsigned)d0 || (unsigned)b >= (unsigned)d1 || (unsigned)c >= (unsigned)d2) return -1;
        return map[((long long)a * d1 + b) * d2 + c];
    }
};

// A float field over a leaf set with getValue semantics (0 outside).
struct DField {
    DMap m;
    const float* v;  // [n][512]
    __device__ __forceinline__ float get(int x, int y, int z) const {
        const int li = m.find(x, y, z);
        if (li < 0) return 0.f;
        return v[(long long)li * UAAMG_LEAF + voff3(x, y, z)];
    }
};

// ---------------------------------------------------------------------------
// OpenVDB BoxSampler::sample (tools/Interpolation.h): floor, fractional
// weights in double, three levels of a + float((double)(b - a) * w).
__device__ __forceinline__ float vdb_lerp(float a, float b, double w) {
    const float d = __fsub_rn(b, a);
    return __fadd_rn(a, __double2float_rn(__dmul_rn((double)d, w)));
}
__device__ __forceinline__ float box_interp(float d000, float d001, float d010, float d011, float d100, float d101,
                                            float d110, float d111, double u, double v, double w) {
    const float a0 = vdb_lerp(vdb_lerp(d000, d001, w), vdb_lerp(d010, d011, w), v);
    const float a1 = vdb_lerp(vdb_lerp(d100, d101, w), vdb_lerp(d110, d111, w), v);
    return vdb_lerp(a0, a1, u);
}
__device__ __forceinline__ float box_sample(const DGrid& g, double px, double py, double pz) {
    const double fx = floor(px), fy = floor(py), fz = floor(pz);
    const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    const double u = __dsub_rn(px, fx), v = __dsub_rn(py, fy), w = __dsub_rn(pz, fz);
    return box_interp(g.get(ix, iy, iz, 0), g.get(ix, iy, iz + 1, 0), g.get(ix, iy + 1, iz, 0),
                      g.get(ix, iy + 1, iz + 1, 0), g.get(ix + 1, iy, iz, 0), g.get(ix + 1, iy, iz + 1, 0),
                      g.get(ix + 1, iy + 1, iz, 0), g.get(ix + 1, iy + 1, iz + 1, 0), u, v, w);
}

// box_sample over a 10^3 block of a grid staged in shared memory, the block's
// voxel (0,0,0) at (bx, by, bz); the caller guarantees floor(p) + 1 lies in it.
__device__ __forceinline__ float box_sample_block(const float (*blk)[10][10], int bx, int by, int bz, double px,
                                                  double py, double pz) {
    const double fx = floor(px), fy = floor(py), fz = floor(pz);
    const int ix = (int)fx - bx, iy = (int)fy - by, iz = (int)fz - bz;
    return box_interp(blk[ix][iy][iz], blk[ix][iy][iz + 1], blk[ix][iy + 1][iz], blk[ix][iy + 1][iz + 1],
                      blk[ix + 1][iy][iz], blk[ix + 1][iy][iz + 1], blk[ix + 1][iy + 1][iz],
                      blk[ix + 1][iy + 1][iz + 1], __dsub_rn(px, fx), __dsub_rn(py, fy), __dsub_rn(pz, fz));
}

// volume_fractions.cpp:82-120 (float versions)
__device__ __forceinline__ void vswap(float& a, float& b) {
    const float t = a;
    a = b;
    b = t;
}
__device__ __forceinline__ float sorted_tet_fraction(float p0, float p1, float p2, float p3) {
    const float num = __fmul_rn(__fmul_rn(p0, p0), p0);
    const float den = __fmul_rn(__fmul_rn(__fsub_rn(p0, p1), __fsub_rn(p0, p2)), __fsub_rn(p0, p3));
    return __fdiv_rn(num, den);
}
__device__ __forceinline__ float sorted_prism_fraction(float p0, float p1, float p2, float p3) {
    const float a = __fdiv_rn(p0, __fsub_rn(p0, p2)), b = __fdiv_rn(p0, __fsub_rn(p0, p3));
    const float c = __fdiv_rn(p1, __fsub_rn(p1, p3)), d = __fdiv_rn(p1, __fsub_rn(p1, p2));
    const float t1 = __fmul_rn(__fmul_rn(a, b), __fsub_rn(1.f, d));
    const float t2 = __fmul_rn(__fmul_rn(b, __fsub_rn(1.f, c)), d);
    return __fadd_rn(__fadd_rn(t1, t2), __fmul_rn(c, d));
}
__device__ __forceinline__ float tet_fraction(float p0, float p1, float p2, float p3) {
    if (p0 > p1) vswap(p0, p1);  // util.h sort(a, b, c, d)
    if (p2 > p3) vswap(p2, p3);
    if (p0 > p2) vswap(p0, p2);
    if (p1 > p3) vswap(p1, p3);
    if (p1 > p2) vswap(p1, p2);
    if (p3 <= 0) return 1.f;
    if (p2 <= 0) return __fsub_rn(1.f, sorted_tet_fraction(p3, p2, p1, p0));
    if (p1 <= 0) return sorted_prism_fraction(p0, p1, p2, p3);
    if (p0 <= 0) return sorted_tet_fraction(p0, p1, p2, p3);
    return 0.f;
}
__device__ __forceinline__ float cube_fraction(float p000, float p100, float p010, float p110, float p001,
                                               float p101, float p011, float p111) {
    if (p000 < 0.f && p100 < 0.f && p010 < 0.f && p110 < 0.f && p001 < 0.f && p101 < 0.f && p011 < 0.f &&
        p111 < 0.f)
        return 1.0f;
    // all corners outside: every tet fraction is +0, so is the mean
    if (p000 > 0.f && p100 > 0.f && p010 > 0.f && p110 > 0.f && p001 > 0.f && p101 > 0.f && p011 > 0.f &&
        p111 > 0.f)
        return 0.0f;
    float s = tet_fraction(p000, p001, p101, p011);
    s = __fadd_rn(s, tet_fraction(p000, p101, p100, p110));
    s = __fadd_rn(s, tet_fraction(p000, p010, p011, p110));
    s = __fadd_rn(s, tet_fraction(p101, p011, p111, p110));
    s = __fadd_rn(s, __fmul_rn(2.f, tet_fraction(p000, p011, p101, p110)));
    s = __fadd_rn(s, tet_fraction(p100, p101, p001, p111));
    s = __fadd_rn(s, tet_fraction(p100, p001, p000, p010));
    s = __fadd_rn(s, tet_fraction(p100, p110, p111, p010));
    s = __fadd_rn(s, tet_fraction(p001, p111, p011, p010));
    s = __fadd_rn(s, __fmul_rn(2.f, tet_fraction(p100, p111, p001, p010)));
    return __fdiv_rn(s, 12.f);
}

// ---------------------------------------------------------------------------
// calculate_subcell_sdf_volume (:258-330).  The subcell leaves of liquid leaf
// i (of the liquid leaves dilated by one voxel) are 8*i + q, q = the octant of
// 2*origin + 8*(q>>2, (q>>1)&1, q&1); subcell corner s sits at liquid index
// s/2 - 1/2.
__device__ __forceinline__ int sub_leaf_of(const DMap& a1, int sx, int sy, int sz) {
    const int li = a1.find(sx >> 1, sy >> 1, sz >> 1);
    if (li < 0) return -1;
    return li * 8 + (((sx >> 3) & 1) << 2) + (((sy >> 3) & 1) << 1) + ((sz >> 3) & 1);
}

// One subcell leaf per CTA (8 per liquid leaf of the dilated set): the
// subcell SDF at the 9^3 corners the leaf's cubes need, then the cubes'
// liquid fractions.  The SDF at subcell s is min(BoxSampler of the liquid SDF
// at s/2 - 1/2, 1.5 dx) where s's subcell leaf exists, else 1.5 dx (the
// subcell grid's background).  The liquid values those samples read -- a 6^3
// block from s0/2 - 1 -- are staged in shared memory first, so each cube reads
// its 8 corners from shared memory instead of through the leaf map.
__global__ void __launch_bounds__(128) k_vsub(DGrid liq, DMap a1, const int* a1org, float bg, float* svol) {
    __shared__ float lq[6][6][6];
    __shared__ float cs[9][9][9];
    __shared__ int halo[8];
    const int b = blockIdx.x, t = threadIdx.x;
    const int li = b >> 3, q = b & 7;
    const int ox = 2 * a1org[3 * li] + 8 * (q >> 2), oy = 2 * a1org[3 * li + 1] + 8 * ((q >> 1) & 1),
              oz = 2 * a1org[3 * li + 2] + 8 * (q & 1);
    const int lx = (ox >> 1) - 1, ly = (oy >> 1) - 1, lz = (oz >> 1) - 1;
    for (int i = t; i < 216; i += 128) lq[i / 36][(i / 6) % 6][i % 6] = liq.get(lx + i / 36, ly + (i / 6) % 6, lz + i % 6, 0);
    if (t < 8) halo[t] = sub_leaf_of(a1, ox + 8 * (t >> 2), oy + 8 * ((t >> 1) & 1), oz + 8 * (t & 1)) >= 0;
    __syncthreads();
    for (int i = t; i < 729; i += 128) {
        const int k0 = i / 81, k1 = (i / 9) % 9, k2 = i % 9;
        float v = bg;
        if (halo[((k0 >> 3) << 2) | ((k1 >> 3) << 1) | (k2 >> 3)]) {
            const double px = 0.5 * (ox + k0) - 0.5, py = 0.5 * (oy + k1) - 0.5, pz = 0.5 * (oz + k2) - 0.5;
            const double fx = floor(px), fy = floor(py), fz = floor(pz);
            const int ix = (int)fx - lx, iy = (int)fy - ly, iz = (int)fz - lz;
            const float sv = box_interp(lq[ix][iy][iz], lq[ix][iy][iz + 1], lq[ix][iy + 1][iz], lq[ix][iy + 1][iz + 1],
                                        lq[ix + 1][iy][iz], lq[ix + 1][iy][iz + 1], lq[ix + 1][iy + 1][iz],
                                        lq[ix + 1][iy + 1][iz + 1], __dsub_rn(px, fx), __dsub_rn(py, fy),
                                        __dsub_rn(pz, fz));
            v = sv < bg ? sv : bg;
        }
        cs[k0][k1][k2] = v;
    }
    __syncthreads();
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 r;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int Z = Z0 + j;
        const float f = cube_fraction(cs[X][Y][Z], cs[X + 1][Y][Z], cs[X][Y + 1][Z], cs[X + 1][Y + 1][Z],
                                      cs[X][Y][Z + 1], cs[X + 1][Y][Z + 1], cs[X][Y + 1][Z + 1],
                                      cs[X + 1][Y + 1][Z + 1]);
        f4set(r, j, f > 0 ? f : 0.f);
    }
    reinterpret_cast<float4*>(svol)[(long long)b * UAAMG_LEAF4 + t] = r;
}

// calculate_matrix_coefficients_volume (:332-406) over the liquid leaves
// dilated by two voxels: out[0] voxel, out[1+c] face c, out[4+c] edge c.
// The 3^3 subcells around 2g of every voxel g of the leaf lie in the 17^3
// block of subcells from 2*origin - 1; the block is staged in shared memory
// (0 where the subcell leaf does not exist) with the 8 liquid leaves it
// touches looked up once.
__global__ void __launch_bounds__(128) k_vvol(DMap a1, const int* a2org, int n2, const float* svol, float* out) {
    __shared__ float sb[17][17][17];
    __shared__ int lv[8];  // liquid leaf of (origin + 8*(i>>2, (i>>1)&1, i&1) - 8), or -1
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int ax = a2org[3 * leaf], ay = a2org[3 * leaf + 1], az = a2org[3 * leaf + 2];
    if (t < 8) lv[t] = a1.find(ax - 8 + 8 * (t >> 2), ay - 8 + 8 * ((t >> 1) & 1), az - 8 + 8 * (t & 1));
    __syncthreads();
    const int s0x = 2 * ax - 1, s0y = 2 * ay - 1, s0z = 2 * az - 1;
    for (int i = t; i < 17 * 17 * 17; i += 128) {
        const int a = i / 289, b = (i / 17) % 17, c = i % 17;
        const int sx = s0x + a, sy = s0y + b, sz = s0z + c;
        // liquid voxel sx>>1 lies in the leaf before the origin's (a == 0) or in the origin's own
        const int l = lv[((a > 0) << 2) | ((b > 0) << 1) | (c > 0)];
        float v = 0.f;
        if (l >= 0) {
            const int sl = l * 8 + (((sx >> 3) & 1) << 2) + (((sy >> 3) & 1) << 1) + ((sz >> 3) & 1);
            v = svol[(long long)sl * UAAMG_LEAF + voff3(sx, sy, sz)];
        }
        sb[a][b][c] = v;
    }
    __syncthreads();
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 res[7];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int bx = 2 * X, by = 2 * Y, bz = 2 * (Z0 + j);  // subcell 2g - 1 in the block
        float vol_c = 0.f, vf[3] = {0.f, 0.f, 0.f}, ve[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj)
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    vol_c = __fadd_rn(vol_c, sb[bx + i + 1][by + jj + 1][bz + k + 1]);
                    // face c: subcell - e_c; edge c: subcell - (1,1,1) + e_c
                    vf[0] = __fadd_rn(vf[0], sb[bx + i][by + jj + 1][bz + k + 1]);
                    ve[0] = __fadd_rn(ve[0], sb[bx + i + 1][by + jj][bz + k]);
                    vf[1] = __fadd_rn(vf[1], sb[bx + i + 1][by + jj][bz + k + 1]);
                    ve[1] = __fadd_rn(ve[1], sb[bx + i][by + jj + 1][bz + k]);
                    vf[2] = __fadd_rn(vf[2], sb[bx + i + 1][by + jj + 1][bz + k]);
                    ve[2] = __fadd_rn(ve[2], sb[bx + i][by + jj][bz + k + 1]);
                }
        f4set(res[0], j, vol_c > 0 ? __fmul_rn(vol_c, 0.125f) : 0.f);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            f4set(res[1 + c], j, vf[c] > 0 ? __fmul_rn(vf[c], 0.125f) : 0.f);
            f4set(res[4 + c], j, ve[c] > 0 ? __fmul_rn(ve[c], 0.125f) : 0.f);
        }
    }
#pragma unroll
    for (int k = 0; k < 7; ++k)
        reinterpret_cast<float4*>(out + (long long)k * n2 * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = res[k];
}

// 4 bits per thread -> 32-bit words of a [nl][8] uint64 mask (thread t owns
// bits (t&7)*4.. of 32-bit word t>>3)
__device__ __forceinline__ void store_bits(uint32_t* words, int leaf, int t, unsigned nib) {
    unsigned v = nib << ((t & 7) * 4);
    v |= __shfl_xor_sync(FULLMASK, v, 1);
    v |= __shfl_xor_sync(FULLMASK, v, 2);
    v |= __shfl_xor_sync(FULLMASK, v, 4);
    if ((t & 7) == 0) words[(long long)leaf * 16 + (t >> 3)] = v;
}

// mark_dof (:408-498) over the liquid leaves face-dilated by one voxel:
// is_solid (solid SDF at the face centre < 0) and the DOF rule.
struct VolFields {
    DField voxel, face[3], edge[3];
};
// The solid samples at the minus-face centres g - e_c / 2 read the solid SDF
// at g - e_c .. g + 1: the 10^3 block from origin - 1, staged in shared memory.
__global__ void __launch_bounds__(128) k_vdof(DGrid sol, VolFields V, const int* org, int n, uint32_t* dofw,
                                              uint32_t* solidw) {
    __shared__ float sb[10][10][10];
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
    for (int i = t; i < 1000; i += 128) sb[i / 100][(i / 10) % 10][i % 10] = sol.get(ox - 1 + i / 100, oy - 1 + (i / 10) % 10, oz - 1 + i % 10, 0);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
        unsigned dn = 0, sn = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int g[3] = {ox + X, oy + Y, oz + Z0 + j};
            double p[3] = {(double)g[0], (double)g[1], (double)g[2]};
            p[c] -= 0.5;
            // box_sample over the staged block: floor(p) - (origin - 1) in 0..8
            const double fx = floor(p[0]), fy = floor(p[1]), fz = floor(p[2]);
            const int ix = (int)fx - ox + 1, iy = (int)fy - oy + 1, iz = (int)fz - oz + 1;
            const float s = box_interp(sb[ix][iy][iz], sb[ix][iy][iz + 1], sb[ix][iy + 1][iz], sb[ix][iy + 1][iz + 1],
                                       sb[ix + 1][iy][iz], sb[ix + 1][iy][iz + 1], sb[ix + 1][iy + 1][iz],
                                       sb[ix + 1][iy + 1][iz + 1], __dsub_rn(p[0], fx), __dsub_rn(p[1], fy),
                                       __dsub_rn(p[2], fz));
            if (s < 0) {
                sn |= 1u << j;
                continue;
            }
            bool on = V.face[c].get(g[0], g[1], g[2]) > 0;
            if (!on) {
                int m[3] = {g[0], g[1], g[2]};
                m[c] -= 1;
                on = V.voxel.get(g[0], g[1], g[2]) > 0 || V.voxel.get(m[0], m[1], m[2]) > 0;
            }
            if (!on) {
                int q2[3] = {g[0], g[1], g[2]}, q1[3] = {g[0], g[1], g[2]};
                q2[d2] += 1;
                q1[d1] += 1;
                on = V.edge[d1].get(g[0], g[1], g[2]) > 0 || V.edge[d1].get(q2[0], q2[1], q2[2]) > 0 ||
                     V.edge[d2].get(g[0], g[1], g[2]) > 0 || V.edge[d2].get(q1[0], q1[1], q1[2]) > 0;
            }
            if (on) dn |= 1u << j;
        }
        store_bits(dofw + (long long)c * n * 16, leaf, t, dn);
        store_bits(solidw + (long long)c * n * 16, leaf, t, sn);
    }
}

// ---------------------------------------------------------------------------
// DOF test at a voxel of a level given by local coordinates (-1..8) around a
// leaf, through its 27-neighbourhood
__device__ __forceinline__ bool vdof_at(const VLevel& L, const int* nbrow, int c, int X, int Y, int Z) {
    const int lf = nbrow[vnb_index(X, Y, Z)];
    if (lf < 0) return false;
    return vdof_bit(L, c, lf, voff3(X, Y, Z));
}

// finest_level_matrix_setter::channel_op (:617-844), grid (nl, 3).  Voxels of
// pattern leaves outside the DOF pattern get the same formulas; nothing reads
// them (every read is within two voxels of a DOF).
template <int C>
__device__ __forceinline__ void vcoef0_body(const VLevel& L, const int* org, const VolFields& V, const DGrid& mu,
                                            float factor, float ddiag, float* coef, float (*mub)[10][10]) {
    const int leaf = blockIdx.x, c = C, t = threadIdx.x;
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int bx = org[3 * leaf] - 1, by = org[3 * leaf + 1] - 1, bz = org[3 * leaf + 2] - 1;
    const int* nbrow = L.nb + (long long)leaf * 27;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    const float two_f = __fmul_rn(2.f, factor);
    float4 out[VNA];
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const int lz = Z0 + j;
        const int g[3] = {org[3 * leaf] + X, org[3 * leaf + 1] + Y, org[3 * leaf + 2] + lz};
        float val[VNA];
        if (vdof_at(L, nbrow, c, X, Y, lz)) {
            float fv = V.face[d0].get(g[0], g[1], g[2]);
            if (fv < 1e-1f) fv = 1e-1f;
            float diag = __fadd_rn(0.f, fv);
            {
                const float term = __fmul_rn(__fmul_rn(two_f, V.voxel.get(g[0], g[1], g[2])), mub[X + 1][Y + 1][lz + 1]);
                diag = __fadd_rn(diag, term);
            }
            float negv[3];
            {
                const int m[3] = {g[0] - e0[0], g[1] - e0[1], g[2] - e0[2]};
                const float term = __fmul_rn(__fmul_rn(two_f, V.voxel.get(m[0], m[1], m[2])), mub[m[0] - bx][m[1] - by][m[2] - bz]);
                diag = __fadd_rn(diag, term);
                negv[0] = vdof_at(L, nbrow, c, X - e0[0], Y - e0[1], lz - e0[2]) ? -term : 0.f;
            }
            float fc[3] = {(float)g[0], (float)g[1], (float)g[2]};
            fc[d0] = __fsub_rn(fc[d0], 0.5f);
            // +d1, -d1 (edge d2), +d2, -d2 (edge d1)
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int ax = s < 2 ? d1 : d2;
                const int ech = s < 2 ? d2 : d1;
                const bool pos = (s & 1) == 0;
                int q[3] = {g[0], g[1], g[2]};
                if (pos) q[ax] += 1;
                const float ev = V.edge[ech].get(q[0], q[1], q[2]);
                float p[3] = {fc[0], fc[1], fc[2]};
                p[ax] = pos ? __fadd_rn(p[ax], 0.5f) : __fsub_rn(p[ax], 0.5f);
                const float sm = box_sample_block(mub, bx, by, bz, p[0], p[1], p[2]);
                const float term = __fmul_rn(__fmul_rn(factor, ev), sm);
                diag = __fadd_rn(diag, term);
                if (!pos) {
                    int l[3] = {X, Y, lz};
                    l[ax] -= 1;
                    negv[s < 2 ? 1 : 2] = vdof_at(L, nbrow, c, l[0], l[1], l[2]) ? -term : 0.f;
                }
            }
            val[VA_DIAG] = diag;
            val[VA_INV] = diag != 0.f ? __fdiv_rn(1.0f, diag) : 0.f;
            // negv[k] is the entry along axis d_k; store by absolute axis with
            // static indices only
            if (c == 0) {
                val[VA_NEGX] = negv[0]; val[VA_NEGY] = negv[1]; val[VA_NEGZ] = negv[2];
            } else if (c == 1) {
                val[VA_NEGY] = negv[0]; val[VA_NEGZ] = negv[1]; val[VA_NEGX] = negv[2];
            } else {
                val[VA_NEGZ] = negv[0]; val[VA_NEGX] = negv[1]; val[VA_NEGY] = negv[2];
            }
        } else {
            val[VA_DIAG] = ddiag;  // setValueOff keeps the default
            val[VA_INV] = 0.f;
            val[VA_NEGX] = val[VA_NEGY] = val[VA_NEGZ] = 0.f;
        }
        const bool dof1n = vdof_at(L, nbrow, d1, X, Y, lz);
        const bool dof1p = vdof_at(L, nbrow, d1, X + e1[0], Y + e1[1], lz + e1[2]);
        const bool dof2n = vdof_at(L, nbrow, d2, X, Y, lz);
        const bool dof2p = vdof_at(L, nbrow, d2, X + e2[0], Y + e2[1], lz + e2[2]);
#pragma unroll
        for (int jk = 0; jk < 4; ++jk) {
            const int jj = jk >> 1, kk = jk & 1;
            const bool ok = (jj ? dof1p : dof1n) && (kk ? dof2p : dof2n);
            if (!ok) {
                val[VA_T00 + jk] = 0.f;
                continue;
            }
            int q[3] = {g[0], g[1], g[2]};
            q[d1] += jj;
            q[d2] += kk;
            const float ev = V.edge[d0].get(q[0], q[1], q[2]);
            float p[3] = {(float)g[0], (float)g[1], (float)g[2]};
            p[d1] = jj ? __fadd_rn(p[d1], 0.5f) : __fsub_rn(p[d1], 0.5f);
            p[d2] = kk ? __fadd_rn(p[d2], 0.5f) : __fsub_rn(p[d2], 0.5f);
            const float sm = box_sample_block(mub, bx, by, bz, p[0], p[1], p[2]);
            const float f = (jj == kk) ? factor : -factor;
            val[VA_T00 + jk] = __fmul_rn(__fmul_rn(f, ev), sm);
        }
#pragma unroll
        for (int a = 0; a < VNA; ++a) f4set(out[a], j, val[a]);
    }
#pragma unroll
    for (int a = 0; a < VNA; ++a)
        reinterpret_cast<float4*>(coef + (long long)(c * VNA + a) * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] =
            out[a];
}

__global__ void __launch_bounds__(128) k_vcoef0(VLevel L, const int* org, VolFields V, DGrid mu, float factor,
                                                float ddiag, float* coef) {
    // mu on the 10^3 block from origin - 1: every sample lies within half a voxel of the leaf's voxels
    __shared__ float mub[10][10][10];
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int bx = org[3 * leaf] - 1, by = org[3 * leaf + 1] - 1, bz = org[3 * leaf + 2] - 1;
    for (int i = t; i < 1000; i += 128) mub[i / 100][(i / 10) % 10][i % 10] = mu.get(bx + i / 100, by + (i / 10) % 10, bz + i % 10, 0);
    __syncthreads();
    if (blockIdx.y == 0) vcoef0_body<0>(L, org, V, mu, factor, ddiag, coef, mub);
    else if (blockIdx.y == 1) vcoef0_body<1>(L, org, V, mu, factor, ddiag, coef, mub);
    else vcoef0_body<2>(L, org, V, mu, factor, ddiag, coef, mub);
}

// coarse_matrix_coef_setter (:1068-1350), grid (coarse nl, 3, 4): R A P with
// rap_factor 0.125 from the fine level's (untrimmed) coefficients
__global__ void __launch_bounds__(128) k_vcoarse_coef(VLevel F, VLevel C, float* coef) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const int d[3] = {c, (c + 1) % 3, (c + 2) % 3};
    const int* nbrow = C.nb + (long long)leaf * 27;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    const float rap = 0.125f;
    const float* fdiag = F.coef + (long long)(c * VNA + VA_DIAG) * F.nl * UAAMG_LEAF;
    {
        const int j = blockIdx.z;  // one voxel per thread: the grid's z splits a thread's 4 z-consecutive voxels
        const int lz = Z0 + j;
        const int L3[3] = {X, Y, lz};
        const int q = ((X >= 4) << 2) | ((Y >= 4) << 1) | (lz >= 4);
        const int fl = C.child[leaf * 8 + q];
        const int* fnb = fl >= 0 ? F.nb + (long long)fl * 27 : nullptr;
        const int fb[3] = {2 * (X & 3), 2 * (Y & 3), 2 * (lz & 3)};  // fine local base in leaf fl
        float val[VNA];
        if (vdof_at(C, nbrow, c, X, Y, lz)) {
            float nd = 0.f, nn[3] = {0.f, 0.f, 0.f};
            if (fl >= 0) {
#pragma unroll 1
                for (int ii = 0; ii < 2; ++ii)
#pragma unroll 1
                    for (int jj = 0; jj < 2; ++jj)
#pragma unroll 1
                        for (int kk = 0; kk < 2; ++kk) {
                            int f[3] = {fb[0], fb[1], fb[2]};
                            f[d[0]] += ii;
                            f[d[1]] += jj;
                            f[d[2]] += kk;
                            const int fo = voff3(f[0], f[1], f[2]);
                            if (!vdof_bit(F, c, fl, fo)) continue;
                            nd = __fadd_rn(nd, fdiag[(long long)fl * UAAMG_LEAF + fo]);
                            const int idx[3] = {ii, jj, kk};
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                const float nt =
                                    F.coef[(long long)(c * VNA + VA_NEGX + d[k]) * F.nl * UAAMG_LEAF + (long long)fl * UAAMG_LEAF + fo];
                                int nb3[3] = {f[0], f[1], f[2]};
                                nb3[d[k]] -= 1;
                                if (!vdof_at(F, fnb, c, nb3[0], nb3[1], nb3[2])) continue;
                                if (idx[k] == 0) nn[k] = __fadd_rn(nn[k], nt);
                                else nd = __fadd_rn(nd, __fmul_rn(nt, 2.0f));
                            }
                        }
            }
            val[VA_DIAG] = __fmul_rn(rap, nd);
            val[VA_INV] = nd != 0.f ? __fdiv_rn(1.0f, __fmul_rn(rap, nd)) : 0.f;
            float ng[3];  // along d_k
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                int l[3] = {X, Y, lz};
                l[d[k]] -= 1;
                ng[k] = vdof_at(C, nbrow, c, l[0], l[1], l[2]) ? __fmul_rn(rap, nn[k]) : 0.f;
            }
            if (c == 0) {
                val[VA_NEGX] = ng[0]; val[VA_NEGY] = ng[1]; val[VA_NEGZ] = ng[2];
            } else if (c == 1) {
                val[VA_NEGY] = ng[0]; val[VA_NEGZ] = ng[1]; val[VA_NEGX] = ng[2];
            } else {
                val[VA_NEGZ] = ng[0]; val[VA_NEGX] = ng[1]; val[VA_NEGY] = ng[2];
            }
        } else {
            val[VA_DIAG] = val[VA_INV] = 0.f;
            val[VA_NEGX] = val[VA_NEGY] = val[VA_NEGZ] = 0.f;
        }
#pragma unroll
        for (int tt = 0; tt < 4; ++tt) {  // unrolled: val[] takes static indices only
            float s = 0.f;
            if (fl >= 0) {
                const float* T0 = F.coef + (long long)(c * VNA + VA_T00) * F.nl * UAAMG_LEAF + (long long)fl * UAAMG_LEAF;
                const long long st = (long long)F.nl * UAAMG_LEAF;
#pragma unroll 1
                for (int ii = 0; ii < 2; ++ii)
#pragma unroll 1
                    for (int jj = 0; jj < 2; ++jj)
#pragma unroll 1
                        for (int kk = 0; kk < 2; ++kk) {
                            int f[3] = {fb[0], fb[1], fb[2]};
                            f[d[0]] += ii;
                            f[d[1]] += jj;
                            f[d[2]] += kk;
                            const int fo = voff3(f[0], f[1], f[2]);
                            switch (tt) {
                            case 0:
                                s = __fadd_rn(s, T0[fo]);
                                if (kk == 0) s = __fadd_rn(s, T0[st + fo]);
                                if (jj == 0) s = __fadd_rn(s, T0[2 * st + fo]);
                                if (kk == 0 && jj == 0) s = __fadd_rn(s, T0[3 * st + fo]);
                                break;
                            case 1:
                                if (kk == 1) s = __fadd_rn(s, T0[st + fo]);
                                if (jj == 0 && kk == 1) s = __fadd_rn(s, T0[3 * st + fo]);
                                break;
                            case 2:
                                if (jj == 1) s = __fadd_rn(s, T0[2 * st + fo]);
                                if (jj == 1 && kk == 0) s = __fadd_rn(s, T0[3 * st + fo]);
                                break;
                            default:
                                if (jj == 1 && kk == 1) s = __fadd_rn(s, T0[3 * st + fo]);
                            }
                        }
            }
            int a1[3] = {X, Y, lz}, a2[3] = {X, Y, lz};
            if (tt & 2) a1[d[1]] += 1;
            if (tt & 1) a2[d[2]] += 1;
            const bool ok = vdof_at(C, nbrow, d[1], a1[0], a1[1], a1[2]) && vdof_at(C, nbrow, d[2], a2[0], a2[1], a2[2]);
            val[VA_T00 + tt] = ok ? __fmul_rn(rap, s) : 0.f;
        }
        (void)L3;
#pragma unroll
        for (int a = 0; a < VNA; ++a)
            coef[(long long)(c * VNA + a) * C.nl * UAAMG_LEAF + (long long)leaf * UAAMG_LEAF + 4 * t + j] = val[a];
    }
}

// trim_default_nodes (:1692-1721) with LaplacianWithLevel::trimDefaultNodes
// (simd_vdb_poisson.cpp:1772-1811): a leaf whose active values (what
// setValueOn marked) all lie within |default * 1e-3| of the default is
// replaced by the default.  One CTA per leaf; sets trim bits only.
__global__ void __launch_bounds__(128) k_vtrim(VLevel L, uint32_t* trim) {
    griddep_wait();
    griddep_launch();
    // A leaf's array is trimmed when max over its active voxels of |v - default| (NaN differences skipped, 0
    // when there are none) is <= |default * 1e-3|: every active voxel's difference is NaN or <= the tolerance,
    // and the tolerance is not NaN.  All 27 arrays are tested at once and AND-reduced over the block.
    __shared__ uint32_t shm[4];
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int* nbrow = L.nb + (long long)leaf * 27;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    uint32_t ok = 0, tolok = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int d1 = (c + 1) % 3, d2 = (c + 2) % 3;
        const int e1[3] = {d1 == 0, d1 == 1, d1 == 2}, e2[3] = {d2 == 0, d2 == 1, d2 == 2};
        bool own[4], mneg[3][4], a1n[4], a1p[4], a2n[4], a2p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int lz = Z0 + j;
            own[j] = vdof_at(L, nbrow, c, X, Y, lz);
            mneg[0][j] = vdof_at(L, nbrow, c, X - 1, Y, lz);
            mneg[1][j] = vdof_at(L, nbrow, c, X, Y - 1, lz);
            mneg[2][j] = vdof_at(L, nbrow, c, X, Y, lz - 1);
            a1n[j] = vdof_at(L, nbrow, d1, X, Y, lz);
            a1p[j] = vdof_at(L, nbrow, d1, X + e1[0], Y + e1[1], lz + e1[2]);
            a2n[j] = vdof_at(L, nbrow, d2, X, Y, lz);
            a2p[j] = vdof_at(L, nbrow, d2, X + e2[0], Y + e2[1], lz + e2[2]);
        }
#pragma unroll
        for (int a = 0; a < VNA; ++a) {
            const float def = L.app[c * VNA + a];
            const float tol = fabsf(__fmul_rn(def, 1e-3f));
            const float4 v = reinterpret_cast<const float4*>(L.coef + (long long)(c * VNA + a) * L.nl * UAAMG_LEAF)
                [(long long)leaf * UAAMG_LEAF4 + t];
            bool good = true;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                bool act;
                if (a == VA_DIAG || a == VA_INV) act = own[j];
                else if (a <= VA_NEGZ) act = own[j] && mneg[a - VA_NEGX][j];
                else act = (((a - VA_T00) & 2) ? a1p[j] : a1n[j]) && (((a - VA_T00) & 1) ? a2p[j] : a2n[j]);
                if (act && fabsf(__fsub_rn(f4get(v, j), def)) > tol) good = false;
            }
            if (good) ok |= 1u << (c * VNA + a);
            if (tol == tol) tolok |= 1u << (c * VNA + a);
        }
    }
    ok = __reduce_and_sync(FULLMASK, ok);
    if ((t & 31) == 0) shm[t >> 5] = ok;
    __syncthreads();
    if (t == 0) trim[leaf] = shm[0] & shm[1] & shm[2] & shm[3] & tolok;
}

// A trimmed leaf reads its array's applier default: write that default into
// the leaf's block of every trimmed array, so the solve kernels read the
// block as for any other leaf (same values, no trim test per load).
__global__ void __launch_bounds__(128) k_vtrim_fill(VLevel L, const uint32_t* trim, float* coef) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, t = threadIdx.x;
    const uint32_t bits = trim[leaf];
    if (!bits) return;
#pragma unroll 1
    for (int ca = 0; ca < 3 * VNA; ++ca) {
        if (!((bits >> ca) & 1u)) continue;
        const float d = L.app[ca];
        reinterpret_cast<float4*>(coef + (long long)ca * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] =
            make_float4(d, d, d, d);
    }
}

// Coefficient neighbour table of a trimmed level: slot k of leaf i is -1 where
// nb is -1 or names a leaf whose 27 arrays are all trimmed (its blocks hold the
// defaults that the default page holds), else nb.  grid ceil(nl*27 / 128).
__global__ void __launch_bounds__(128) k_vcnb(VLevel L, const uint32_t* trim, int* cnb) {
    griddep_wait();
    griddep_launch();
    const long long i = (long long)blockIdx.x * 128 + threadIdx.x;
    if (i >= (long long)L.nl * 27) return;
    const int lf = L.nb[i];
    cnb[i] = (lf >= 0 && trim[lf] == (1u << (3 * VNA)) - 1u) ? -1 : lf;
}

// explicit_matrix_reducer (:2415-2605): one ELL row per DOF, columns ascending
__device__ __forceinline__ int vdof_number(const VLevel& L, const int* dof_base, const int* nbrow, int c, int X, int Y,
                                           int Z) {
    const int lf = nbrow[vnb_index(X, Y, Z)];
    if (lf < 0) return -1;
    const int off = voff3(X, Y, Z);
    const uint64_t* m = L.dof + ((long long)c * L.nl + lf) * 8;
    if (!((m[off >> 6] >> (off & 63)) & 1ull)) return -1;
    int d = dof_base[c * L.nl + lf];
    for (int w = 0; w < (off >> 6); ++w) d += __popcll(m[w]);
    const uint64_t below = (off & 63) ? (m[off >> 6] & ((1ull << (off & 63)) - 1ull)) : 0ull;
    return d + __popcll(below);
}
__device__ __forceinline__ float vcoef_at(const VLevel& L, const int* nbrow, int c, int a, int X, int Y, int Z) {
    const int lf = nbrow[vnb_index(X, Y, Z)];
    if (lf < 0) return 0.f;
    if (L.trim && (L.trim[lf] >> (c * VNA + a) & 1u)) return L.app[c * VNA + a];
    return L.coef[(long long)(c * VNA + a) * L.nl * UAAMG_LEAF + (long long)lf * UAAMG_LEAF + voff3(X, Y, Z)];
}

__global__ void __launch_bounds__(128) k_vcoarsest_ell(VLevel L, const int* dof_base, int* col, float* val,
                                                       float* invd, long long* slot) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const int* nbrow = L.nb + (long long)leaf * 27;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0};
    e0[d0] = 1;
    e1[d1] = 1;
    e2[d2] = 1;
    {
        const int lz = Z0 + blockIdx.z;  // one voxel per thread: the grid's z splits a thread's 4 voxels
        const int row = vdof_number(L, dof_base, nbrow, c, X, Y, lz);
        if (row < 0) return;
        int cc[VCG_W];
        float vv[VCG_W];
        int n = 0;
        const float dg = vcoef_at(L, nbrow, c, VA_DIAG, X, Y, lz);
        cc[n] = row;
        vv[n++] = dg;
#pragma unroll 1
        for (int f = 0; f < 6; ++f) {
            const int ax = f >> 1;
            int nb3[3] = {X, Y, lz};
            nb3[ax] += (f & 1) ? -1 : 1;
            const int nd = vdof_number(L, dof_base, nbrow, c, nb3[0], nb3[1], nb3[2]);
            if (nd < 0) continue;
            const float term = (f & 1) ? vcoef_at(L, nbrow, c, VA_NEGX + ax, X, Y, lz)
                                       : vcoef_at(L, nbrow, c, VA_NEGX + ax, nb3[0], nb3[1], nb3[2]);
            cc[n] = nd;
            vv[n++] = term;
        }
        // Td2 (channel d1 unknowns, coefficients of channel d2) then Td1
        const int m0[3] = {X - e0[0], Y - e0[1], lz - e0[2]};
        const int pos[8][3] = {{X, Y, lz},
                               {X + e1[0], Y + e1[1], lz + e1[2]},
                               {m0[0], m0[1], m0[2]},
                               {m0[0] + e1[0], m0[1] + e1[1], m0[2] + e1[2]},
                               {X, Y, lz},
                               {m0[0], m0[1], m0[2]},
                               {X + e2[0], Y + e2[1], lz + e2[2]},
                               {m0[0] + e2[0], m0[1] + e2[1], m0[2] + e2[2]}};
        const int atm0[8] = {0, 0, 1, 1, 0, 1, 0, 1};
        const int arr[8] = {VA_T00, VA_T01, VA_T10, VA_T11, VA_T00, VA_T01, VA_T10, VA_T11};
#pragma unroll 1
        for (int k = 0; k < 8; ++k) {
            const int ch = k < 4 ? d1 : d2, ach = k < 4 ? d2 : d1;
            const int nd = vdof_number(L, dof_base, nbrow, ch, pos[k][0], pos[k][1], pos[k][2]);
            if (nd < 0) continue;
            const int* at = atm0[k] ? m0 : nullptr;
            cc[n] = nd;
            vv[n++] = at ? vcoef_at(L, nbrow, ach, arr[k], m0[0], m0[1], m0[2]) : vcoef_at(L, nbrow, ach, arr[k], X, Y, lz);
        }
        for (int a = 1; a < n; ++a) {  // insertion sort by column
            const int kc = cc[a];
            const float kv = vv[a];
            int b = a - 1;
            while (b >= 0 && cc[b] > kc) {
                cc[b + 1] = cc[b];
                vv[b + 1] = vv[b];
                --b;
            }
            cc[b + 1] = kc;
            vv[b + 1] = kv;
        }
        for (int e = 0; e < VCG_W; ++e) {
            col[(long long)row * VCG_W + e] = e < n ? cc[e] : -1;
            val[(long long)row * VCG_W + e] = e < n ? vv[e] : 0.f;
        }
        invd[row] = dg != 0.f ? __fdiv_rn(1.0f, dg) : 1.0f;
        slot[row] = ((long long)c * L.nl + leaf) * UAAMG_LEAF + voff3(X, Y, lz);
    }
}

// ---------------------------------------------------------------------------
// build_rhs (:2005-2087): rhs = u * max(face volume, 0.1) at every DOF
struct VelGrids {
    DGrid v[3];
};
__global__ void __launch_bounds__(128) k_vrhs(VLevel L, const int* org, VolFields V, VelGrids U, float* rhs) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    if (!m) return;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 r = f4zero();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!(m >> j & 1)) continue;
        const int g0 = org[3 * leaf] + X, g1 = org[3 * leaf + 1] + Y, g2 = org[3 * leaf + 2] + Z0 + j;
        float fv = V.face[c].get(g0, g1, g2);
        if (fv < 1e-1f) fv = 1e-1f;
        f4set(r, j, __fmul_rn(U.v[c].get(g0, g1, g2, 0), fv));
    }
    reinterpret_cast<float4*>(rhs + (long long)c * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = r;
}

// The velocity at every DOF (the warm start of FLIP_vdb.cpp:3188-3198).
__global__ void __launch_bounds__(128) k_vgather(VLevel L, const int* org, VelGrids U, float* out) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    float4 r = f4zero();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!(m >> j & 1)) continue;
        f4set(r, j, U.v[c].get(org[3 * leaf] + X, org[3 * leaf + 1] + Y, org[3 * leaf + 2] + Z0 + j, 0));
    }
    reinterpret_cast<float4*>(out + (long long)c * L.nl * UAAMG_LEAF)[(long long)leaf * UAAMG_LEAF4 + t] = r;
}

// Solid-velocity part of build_rhs: rhs_reducer (:1724-2002) scatters
// -coefficient * solid velocity of every solid face coupled to a DOF; here
// each DOF gathers its contributions in a fixed order: the same-channel sum,
// then the cross terms of channel c+1 (where c is its second face) and of
// channel c+2 (where c is its first face), each in 00, 01, 10, 11 order.
struct SolidInfo {
    DMap m;                 // leaves of the is_solid grids
    const uint32_t* words;  // [3][n][16]
    int n;
    __device__ __forceinline__ bool at(int c, int x, int y, int z) const {
        const int li = m.find(x, y, z);
        if (li < 0) return false;
        const int off = voff3(x, y, z);
        return (words[((long long)c * n + li) * 16 + (off >> 5)] >> (off & 31)) & 1u;
    }
};
__device__ __forceinline__ float vcross_term(const VolFields& V, const DGrid& mu, float factor, int cp, const int* p,
                                             int jk) {
    const int d1 = (cp + 1) % 3, d2 = (cp + 2) % 3;
    const int jj = jk >> 1, kk = jk & 1;
    int e[3] = {p[0], p[1], p[2]};
    e[d1] += jj;
    e[d2] += kk;
    const float ev = V.edge[cp].get(e[0], e[1], e[2]);
    float q[3] = {(float)p[0], (float)p[1], (float)p[2]};
    q[d1] = jj ? __fadd_rn(q[d1], 0.5f) : __fsub_rn(q[d1], 0.5f);
    q[d2] = kk ? __fadd_rn(q[d2], 0.5f) : __fsub_rn(q[d2], 0.5f);
    const float sm = box_sample(mu, q[0], q[1], q[2]);
    const float f = (jj == kk) ? factor : -factor;
    return __fmul_rn(__fmul_rn(f, ev), sm);
}
__global__ void __launch_bounds__(128) k_vrhs_solid(VLevel L, const int* org, VolFields V, DGrid mu, SolidInfo S,
                                                    DGrid sv, float factor, float* rhs) {
    griddep_wait();
    griddep_launch();
    const int leaf = blockIdx.x, c = blockIdx.y, t = threadIdx.x;
    const unsigned m = vmask4(L, c, leaf, t);
    if (!m) return;
    const int* nbrow = L.nb + (long long)leaf * 27;
    const int X = t >> 4, Y = (t >> 1) & 7, Z0 = (t & 1) * 4;
    const int d0 = c, d1 = (c + 1) % 3, d2 = (c + 2) % 3;
    const float two_f = __fmul_rn(2.f, factor);
    float4* rp = reinterpret_cast<float4*>(rhs + (long long)c * L.nl * UAAMG_LEAF) + (long long)leaf * UAAMG_LEAF4 + t;
    float4 r = *rp;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        if (!(m >> j & 1)) continue;
        const int lz = Z0 + j;
        const int g[3] = {org[3 * leaf] + X, org[3 * leaf + 1] + Y, org[3 * leaf + 2] + lz};
        const int l[3] = {X, Y, lz};
        float acc = 0.f;
        bool have = false;
        auto add = [&](float v) {
            if (have) acc = __fadd_rn(acc, v);
            else { acc = v; have = true; }
        };
        auto dof_g = [&](int ch, const int* q) {  // q global
            return vdof_at(L, nbrow, ch, l[0] + q[0] - g[0], l[1] + q[1] - g[1], l[2] + q[2] - g[2]);
        };
        float temp_rhs = 0.f;
#pragma unroll 1
        for (int s = 0; s < 2; ++s) {  // +d0, -d0
            int q[3] = {g[0], g[1], g[2]};
            q[d0] += s == 0 ? 1 : -1;
            const int* vg = s == 0 ? g : q;
            const float term = __fmul_rn(__fmul_rn(two_f, V.voxel.get(vg[0], vg[1], vg[2])), mu.get(vg[0], vg[1], vg[2], 0));
            if (!dof_g(c, q) && S.at(c, q[0], q[1], q[2]))
                temp_rhs = __fadd_rn(temp_rhs, __fmul_rn(term, sv.get(q[0], q[1], q[2], d0)));
        }
        float fc[3] = {(float)g[0], (float)g[1], (float)g[2]};
        fc[d0] = __fsub_rn(fc[d0], 0.5f);
#pragma unroll 1
        for (int s = 0; s < 4; ++s) {  // +d1, -d1, +d2, -d2
            const int ax = s < 2 ? d1 : d2, ech = s < 2 ? d2 : d1;
            const bool pos = (s & 1) == 0;
            int e[3] = {g[0], g[1], g[2]};
            if (pos) e[ax] += 1;
            const float ev = V.edge[ech].get(e[0], e[1], e[2]);
            float p[3] = {fc[0], fc[1], fc[2]};
            p[ax] = pos ? __fadd_rn(p[ax], 0.5f) : __fsub_rn(p[ax], 0.5f);
            const float term = __fmul_rn(__fmul_rn(factor, ev), box_sample(mu, p[0], p[1], p[2]));
            int q[3] = {g[0], g[1], g[2]};
            q[ax] += pos ? 1 : -1;
            if (!dof_g(c, q) && S.at(c, q[0], q[1], q[2]))
                temp_rhs = __fadd_rn(temp_rhs, __fmul_rn(term, sv.get(q[0], q[1], q[2], d0)));
        }
        if (temp_rhs != 0.f) add(temp_rhs);
        int gm[3] = {g[0], g[1], g[2]};
        gm[c] -= 1;
        {  // channel c+1 with c as its second face; its first face a1 = c+2
            const int cp = (c + 1) % 3, a1 = (cp + 1) % 3;
            int q[3];
            if (!dof_g(a1, g) && S.at(a1, g[0], g[1], g[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, g, 0), sv.get(g[0], g[1], g[2], a1)));
            if (!dof_g(a1, gm) && S.at(a1, gm[0], gm[1], gm[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, gm, 1), sv.get(gm[0], gm[1], gm[2], a1)));
            q[0] = g[0]; q[1] = g[1]; q[2] = g[2];
            q[a1] += 1;
            if (!dof_g(a1, q) && S.at(a1, q[0], q[1], q[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, g, 2), sv.get(q[0], q[1], q[2], a1)));
            q[0] = gm[0]; q[1] = gm[1]; q[2] = gm[2];
            q[a1] += 1;
            if (!dof_g(a1, q) && S.at(a1, q[0], q[1], q[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, gm, 3), sv.get(q[0], q[1], q[2], a1)));
        }
        {  // channel c+2 with c as its first face; its second face a2 = c+1
            const int cp = (c + 2) % 3, a2 = (cp + 2) % 3;
            int q[3];
            if (!dof_g(a2, g) && S.at(a2, g[0], g[1], g[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, g, 0), sv.get(g[0], g[1], g[2], a2)));
            q[0] = g[0]; q[1] = g[1]; q[2] = g[2];
            q[a2] += 1;
            if (!dof_g(a2, q) && S.at(a2, q[0], q[1], q[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, g, 1), sv.get(q[0], q[1], q[2], a2)));
            if (!dof_g(a2, gm) && S.at(a2, gm[0], gm[1], gm[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, gm, 2), sv.get(gm[0], gm[1], gm[2], a2)));
            q[0] = gm[0]; q[1] = gm[1]; q[2] = gm[2];
            q[a2] += 1;
            if (!dof_g(a2, q) && S.at(a2, q[0], q[1], q[2]))
                add(__fmul_rn(-vcross_term(V, mu, factor, cp, gm, 3), sv.get(q[0], q[1], q[2], a2)));
        }
        if (have) f4set(r, j, __fadd_rn(f4get(r, j), acc));
    }
    *rp = r;
}

}  // namespace uaamg
