// poisson_build.cuh -- sm_100a kernels that assemble the Poisson hierarchy:
// level-0 coefficients from the liquid SDF and solid face fractions, Galerkin
// (unsmoothed-aggregation) coarsening, default-leaf trimming, SPAI0, the
// coarsest explicit matrix and the right-hand side.
#pragma once
#include <float.h>

#include "common.cuh"

namespace uaamg {

// A flattened input grid with OpenVDB ConstAccessor::getValue semantics:
// the value stored in the leaf containing the voxel (active or not), else the
// background.  Leaves are found through a dense index volume over the
// bounding box of leaf coordinates.
struct DGrid {
    const float* val;  // [n][512][comps]
    const int* map;    // dense [d0][d1][d2] leaf index or -1
    int lo0, lo1, lo2, d0, d1, d2;
    int comps;
    float bg0, bg1, bg2;
    __device__ __forceinline__ int leaf_of(int x, int y, int z) const {
        if (!map) return -1;
        int a = (x >> 3) - lo0, b = (y >> 3) - lo1, c = (z >> 3) - lo2;
        if ((unsigned)a >= (unsigned)d0 || (unsigned)b >= (unsigned)d1 || (unsigned)c >= (unsigned)d2) return -1;
        return map[((long long)a * d1 + b) * d2 + c];
    }
    __device__ __forceinline__ float get(int x, int y, int z, int c) const {
        int li = leaf_of(x, y, z);
        if (li < 0) return c == 0 ? bg0 : (c == 1 ? bg1 : bg2);
        int off = ((x & 7) << 6) | ((y & 7) << 3) | (z & 7);
        return val[((long long)li * UAAMG_LEAF + off) * comps + c];
    }
};

// A grid seen from one leaf: the leaf indices of the leaf at `o` and of its six
// face neighbours, resolved once per CTA (slot 0: the leaf; 1 + 2 axis +
// (+ side): the neighbour), so a read at a voxel of the leaf or one voxel
// across a face costs one load instead of a map lookup and a load.  get()
// returns what DGrid::get returns for those voxels.
struct DGridNb {
    const DGrid* g;
    const int* li;  // [7], shared memory
    int ox, oy, oz;
    __device__ __forceinline__ float get(int x, int y, int z, int c) const {
        const int lx = (x - ox) >> 3, ly = (y - oy) >> 3, lz = (z - oz) >> 3;
        const int slot = lx ? (lx < 0 ? 1 : 2) : (ly ? (ly < 0 ? 3 : 4) : (lz ? (lz < 0 ? 5 : 6) : 0));
        const int l = li[slot];
        if (l < 0) return c == 0 ? g->bg0 : (c == 1 ? g->bg1 : g->bg2);
        const int off = ((x & 7) << 6) | ((y & 7) << 3) | (z & 7);
        return g->val[((long long)l * UAAMG_LEAF + off) * g->comps + c];
    }
};
// the seven leaf indices of grid g around origin o, by threads t < 7 (the caller syncs)
__device__ __forceinline__ void nb7_resolve(const DGrid& g, int ox, int oy, int oz, int t, int* li) {
    if (t < 7) {
        const int ax = (t - 1) >> 1, sg = ((t - 1) & 1) ? 8 : -8;
        li[t] = g.leaf_of(ox + (t > 0 && ax == 0 ? sg : 0), oy + (t > 0 && ax == 1 ? sg : 0),
                          oz + (t > 0 && ax == 2 ? sg : 0));
    }
}

// levelset_util.cpp:4-13
__device__ __forceinline__ float fraction_inside1(float l, float r) {
    if (l < 0 && r < 0) return 1.f;
    if (l < 0 && r >= 0) return __fdiv_rn(l, __fsub_rn(l, r));
    if (l >= 0 && r < 0) return __fdiv_rn(r, __fsub_rn(r, l));
    return 0.f;
}

struct LevelOut {
    float* diag;
    float* cx;
    float* cy;
    float* cz;
    float* invdiag;
    uint32_t* flags;
    float def_diag, def_face;  // trim defaults: 6 dt/dx^2 and -dt/dx^2
    float eps_diag, eps_face;  // |default| * 1e-5
    float inv_bg;              // 1 / background of the diagonal grid
    float def_invdiag;         // 1 / (6 dt/dx^2)
};

// BuildFinestMatrix for one voxel (simd_vdb_poisson.cpp:520-584): returns diag
// (0 = not a DOF) and the three minus-face entries.
template <class GP, class GF>
__device__ __forceinline__ float finest_voxel(const GP& phi, const GF& fw, int gx, int gy, int gz, float phic,
                                              float dtOverDxSqr, float* xyz) {
    float dg = 0.f;
    xyz[0] = xyz[1] = xyz[2] = 0.f;
    const int g[3] = {gx, gy, gz};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int comp = f >> 1;
        const bool pos = (f & 1) == 0;
        int wc[3] = {g[0], g[1], g[2]}, pc[3] = {g[0], g[1], g[2]};
        if (pos) { wc[comp] += 1; pc[comp] += 1; } else { pc[comp] -= 1; }
        const float weight = fw.get(wc[0], wc[1], wc[2], comp);
        const float phiOther = phi.get(pc[0], pc[1], pc[2], 0);
        const float term = __fmul_rn(weight, dtOverDxSqr);
        if (phiOther < 0.f) {
            dg = __fadd_rn(dg, term);
            if (!pos) xyz[comp] = -term;
        } else {
            float theta = fraction_inside1(phic, phiOther);
            if (theta < 0.02f) theta = 0.02f;
            dg = __fadd_rn(dg, __fdiv_rn(term, theta));
        }
    }
    return dg;
}

// ---------------------------------------------------------------------------
// Inputs in pinned host memory: only the leaves the construction reads cross
// the bus.  The DOF mask, the coefficients and the rhs read a face grid (face
// weights, face velocities, solid velocity) at the six faces of liquid voxels
// (active, phi < 0): in the voxel's own leaf and, for its + faces on a leaf
// boundary, in the next leaf along x, y or z.  So a face-grid leaf is read
// exactly when the liquid-SDF leaf at its origin or one leaf below it along x,
// y or z holds a liquid voxel.

// per liquid-SDF leaf: does it hold a liquid voxel?
__global__ void __launch_bounds__(128) k_liquid_leaves(DGrid phi, const uint64_t* phi_mask, uint8_t* out) {
    const int leaf = blockIdx.x, t = threadIdx.x;
    bool any = false;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int off = 4 * t + j;
        if (phi_mask && !((phi_mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull)) continue;
        if (phi.val[(long long)leaf * UAAMG_LEAF + off] < 0.f) any = true;
    }
    any = __syncthreads_or(any) != 0;
    if (t == 0) out[leaf] = any ? 1 : 0;
}
// per leaf of a face grid (origins org[n][3]): does the construction read it?
__global__ void k_face_leaves_read(const int* org, int n, DGrid phi, const uint8_t* liquid, uint8_t* need) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ox = org[3 * i], oy = org[3 * i + 1], oz = org[3 * i + 2];
    const int l0 = phi.leaf_of(ox, oy, oz), lx = phi.leaf_of(ox - 8, oy, oz), ly = phi.leaf_of(ox, oy - 8, oz),
              lz = phi.leaf_of(ox, oy, oz - 8);
    need[i] = ((l0 >= 0 && liquid[l0]) || (lx >= 0 && liquid[lx]) || (ly >= 0 && liquid[ly]) ||
               (lz >= 0 && liquid[lz]))
                  ? 1
                  : 0;
}
// A face grid's values [n][512][comps] from pinned host memory (read by the
// kernel through its device mapping): the leaves the construction reads are
// copied, the others hold NaN, which no result may depend on.  A few CTAs
// (one per SM) walk the leaves, each thread with the loads of GATHER_LEAVES
// leaves in flight: that keeps the bus busy while leaving the SMs to the
// kernels that run beside the copy (one CTA per leaf filled every SM with
// CTAs waiting on the bus, and the construction's kernels queued behind them).
constexpr int GATHER_LEAVES = 4;
__global__ void __launch_bounds__(128) k_gather_host_leaves(const float4* __restrict__ src, int comps, int n,
                                                            const uint8_t* __restrict__ need,
                                                            float4* __restrict__ dst) {
    const int t = threadIdx.x;
    const float q = __int_as_float(0x7fffffff);
    const float4 nan4 = make_float4(q, q, q, q);
    for (int l0 = blockIdx.x; l0 < n; l0 += gridDim.x * GATHER_LEAVES) {
        float4 v[GATHER_LEAVES][3];
#pragma unroll
        for (int u = 0; u < GATHER_LEAVES; ++u) {
            const int leaf = l0 + u * (int)gridDim.x;
            const bool rd = leaf < n && need[leaf];
            const long long base = (long long)leaf * comps * (UAAMG_LEAF / 4);
#pragma unroll
            for (int c = 0; c < 3; ++c) v[u][c] = (rd && c < comps) ? src[base + c * 128 + t] : nan4;
        }
#pragma unroll
        for (int u = 0; u < GATHER_LEAVES; ++u) {
            const int leaf = l0 + u * (int)gridDim.x;
            if (leaf >= n) break;
            const long long base = (long long)leaf * comps * (UAAMG_LEAF / 4);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (c < comps) dst[base + c * 128 + t] = v[u][c];
        }
    }
}

// pass 0: DOF masks of every input leaf (liquid, active, diag != 0)
__global__ void __launch_bounds__(128) k_finest_mask(DGrid phi, const uint64_t* phi_mask, const int* phi_org, DGrid fw,
                                                     float dtOverDxSqr, uint64_t* out_mask) {
    __shared__ uint32_t bits[16];
    __shared__ int pli[7], fli[7];
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (t < 16) bits[t] = 0;
    const int ox = phi_org[3 * leaf], oy = phi_org[3 * leaf + 1], oz = phi_org[3 * leaf + 2];
    nb7_resolve(phi, ox, oy, oz, t, pli);
    nb7_resolve(fw, ox, oy, oz, t, fli);
    __syncthreads();
    const DGridNb P{&phi, pli, ox, oy, oz}, W{&fw, fli, ox, oy, oz};
    unsigned my = 0;
    for (int j = 0; j < 4; ++j) {
        const int off = 4 * t + j;
        if (phi_mask && !((phi_mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull)) continue;
        const float phic = phi.val[(long long)leaf * UAAMG_LEAF + off];
        if (!(phic < 0.f)) continue;
        float xyz[3];
        float dg = finest_voxel(P, W, ox + (off >> 6), oy + ((off >> 3) & 7), oz + (off & 7), phic, dtOverDxSqr, xyz);
        if (dg != 0.f) my |= 1u << j;
    }
    // thread t's 4 bits belong to word t>>4 at bit (t&15)*4: 8 threads per 32-bit half
    atomicOr(&bits[t >> 3], my << ((t & 7) * 4));
    __syncthreads();
    if (t < 8) out_mask[(long long)leaf * 8 + t] = (uint64_t)bits[2 * t] | ((uint64_t)bits[2 * t + 1] << 32);
}

__device__ __forceinline__ float block_max128f(float v, float* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    float r = fmaxf(fmaxf(sh[0], sh[1]), fmaxf(sh[2], sh[3]));
    __syncthreads();
    return r;
}

// trimDefaultNodes (.cpp:1756-1811) + initInvDiagonal (.cpp:1081-1111) for one
// leaf whose 4 arrays are in registers (4 voxels per thread); writes the
// effective values (defaults for trimmed leaves), 1/diag and the flags.
__device__ __forceinline__ void finalize_leaf(const LevelOut& O, int leaf, int t, unsigned m, float4 dg, float4 vx,
                                              float4 vy, float4 vz) {
    __shared__ float sh[4];
    float e[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        float a = fabsf(__fsub_rn(f4get(dg, j), O.def_diag));
        float b = fabsf(__fsub_rn(f4get(vx, j), O.def_face));
        float c = fabsf(__fsub_rn(f4get(vy, j), O.def_face));
        float d = fabsf(__fsub_rn(f4get(vz, j), O.def_face));
        if (a > e[0]) e[0] = a;
        if (b > e[1]) e[1] = b;
        if (c > e[2]) e[2] = c;
        if (d > e[3]) e[3] = d;
    }
    const bool td = block_max128f(e[0], sh) <= O.eps_diag;
    const bool tx = block_max128f(e[1], sh) <= O.eps_face;
    const bool ty = block_max128f(e[2], sh) <= O.eps_face;
    const bool tz = block_max128f(e[3], sh) <= O.eps_face;
    if (td) dg = f4splat(O.def_diag);
    if (tx) vx = f4splat(O.def_face);
    if (ty) vy = f4splat(O.def_face);
    if (tz) vz = f4splat(O.def_face);
    float4 iv;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float v;
        if (td) v = O.def_invdiag;
        else if (!((m >> j) & 1)) v = O.inv_bg;
        else v = (f4get(dg, j) == 0.f) ? 0.f : __fdiv_rn(1.0f, f4get(dg, j));
        f4set(iv, j, v);
    }
    st4(O.diag, leaf, t, dg);
    st4(O.cx, leaf, t, vx);
    st4(O.cy, leaf, t, vy);
    st4(O.cz, leaf, t, vz);
    st4(O.invdiag, leaf, t, iv);
    if (t == 0) O.flags[leaf] = (td ? TRIM_DIAG : 0u) | (tx ? TRIM_X : 0u) | (ty ? TRIM_Y : 0u) | (tz ? TRIM_Z : 0u);
}

// pass 1: level-0 coefficients into the compacted (DOF-leaf) order
__global__ void __launch_bounds__(128) k_finest_coef(DGrid phi, const int* phi_org, DGrid fw, float dtOverDxSqr,
                                                     const int* src_leaf, const uint64_t* mask, LevelOut O) {
    __shared__ int pli[7], fli[7];
    const int leaf = blockIdx.x, t = threadIdx.x;
    const int s = src_leaf[leaf];
    const int ox = phi_org[3 * s], oy = phi_org[3 * s + 1], oz = phi_org[3 * s + 2];
    nb7_resolve(phi, ox, oy, oz, t, pli);
    nb7_resolve(fw, ox, oy, oz, t, fli);
    __syncthreads();
    const DGridNb P{&phi, pli, ox, oy, oz}, W{&fw, fli, ox, oy, oz};
    const unsigned m = mask4(mask, leaf, t);
    float4 dg = f4splat(O.def_diag), vx = f4splat(O.def_face), vy = vx, vz = vx;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        const int off = 4 * t + j;
        const float phic = phi.val[(long long)s * UAAMG_LEAF + off];
        float xyz[3];
        float d = finest_voxel(P, W, ox + (off >> 6), oy + ((off >> 3) & 7), oz + (off & 7), phic, dtOverDxSqr, xyz);
        f4set(dg, j, d);
        f4set(vx, j, xyz[0]);
        f4set(vy, j, xyz[1]);
        f4set(vz, j, xyz[2]);
    }
    finalize_leaf(O, leaf, t, m, dg, vx, vy, vz);
}

// Galerkin coarsening of the 7-point operator (initializeFromFineLevel,
// .cpp:353-467): 0.5 * R A P with R = 1/8 sum, P = injection.  One CTA per
// coarse leaf.  Its 8 child leaves' diag, c_x, c_y, c_z (the effective
// values; a trimmed leaf holds its default) and the DOF masks a fine voxel
// consults (its own leaf's and its -x, -y, -z neighbours') are staged into
// shared memory with coalesced loads first; each thread then sums its 4
// coarse voxels' 8 fine voxels in the order of the unstaged loop.  (Loading
// per fine voxel, every thread ran a chain of 32 dependent global loads: 50 us
// for a 284-leaf level.)
constexpr int COARSEN_SMEM = 4 * 8 * UAAMG_LEAF * 4;  // dynamic shared memory of k_coarsen (64 KB)
__global__ void __launch_bounds__(128) k_coarsen(DLevel F, const int* child, const uint64_t* cmask, LevelOut O) {
    extern __shared__ __align__(16) float cst[];  // [4 arrays][8 children][512]
    __shared__ uint64_t msk[8][4][8];            // [child][own, -x, -y, -z][word]
    __shared__ int kid[8];
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (t < 8) kid[t] = child[leaf * 8 + t];
    __syncthreads();
    for (int i = t; i < 8 * 4 * 8; i += 128) {
        const int q = i >> 5, r = (i >> 3) & 3, w = i & 7;
        const int fl = kid[q];
        uint64_t v = 0;
        if (fl >= 0) {
            const int src = r == 0 ? fl : F.nbr[(long long)fl * 6 + 2 * (r - 1)];
            if (src >= 0) v = F.mask[(long long)src * 8 + w];
        }
        msk[q][r][w] = v;
    }
    const float* arr[4] = {F.diag, F.cx, F.cy, F.cz};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int fl = kid[q];
        if (fl < 0) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a)
            reinterpret_cast<float4*>(cst + (a * 8 + q) * UAAMG_LEAF)[t] = ld4(arr[a], fl, t);
    }
    __syncthreads();
    const unsigned m = mask4(cmask, leaf, t);
    float4 dg = f4splat(O.def_diag), vx = f4splat(O.def_face), vy = vx, vz = vx;
    const float factor = 0.5f * (1.0f / 8.0f);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        const int off = 4 * t + j;
        const int X = off >> 6, Y = (off >> 3) & 7, Z = off & 7;
        const int q = ((X >= 4) << 2) | ((Y >= 4) << 1) | (Z >= 4);
        const uint64_t* fm = msk[q][0];
        const float* sd = cst + (0 * 8 + q) * UAAMG_LEAF;
        const float* sx = cst + (1 * 8 + q) * UAAMG_LEAF;
        const float* sy = cst + (2 * 8 + q) * UAAMG_LEAF;
        const float* sz = cst + (3 * 8 + q) * UAAMG_LEAF;
        float d = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
        for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
                for (int kk = 0; kk < 2; ++kk) {
                    const int fx = (2 * X + ii) & 7, fy = (2 * Y + jj) & 7, fz = (2 * Z + kk) & 7;
                    const int fo = (fx << 6) | (fy << 3) | fz;
                    if (!((fm[fo >> 6] >> (fo & 63)) & 1ull)) continue;
                    d = __fadd_rn(d, sd[fo]);
                    // -x neighbour a DOF?
                    bool on;
                    if (fx > 0) on = (fm[(fo - 64) >> 6] >> ((fo - 64) & 63)) & 1ull;
                    else on = (msk[q][1][7] >> ((fo + 448) & 63)) & 1ull;
                    if (on) { if (ii == 0) tx = __fadd_rn(tx, sx[fo]); else d = __fadd_rn(d, __fmul_rn(2.f, sx[fo])); }
                    if (fy > 0) on = (fm[(fo - 8) >> 6] >> ((fo - 8) & 63)) & 1ull;
                    else on = (msk[q][2][(fo + 56) >> 6] >> ((fo + 56) & 63)) & 1ull;
                    if (on) { if (jj == 0) ty = __fadd_rn(ty, sy[fo]); else d = __fadd_rn(d, __fmul_rn(2.f, sy[fo])); }
                    if (fz > 0) on = (fm[(fo - 1) >> 6] >> ((fo - 1) & 63)) & 1ull;
                    else on = (msk[q][3][(fo + 7) >> 6] >> ((fo + 7) & 63)) & 1ull;
                    if (on) { if (kk == 0) tz = __fadd_rn(tz, sz[fo]); else d = __fadd_rn(d, __fmul_rn(2.f, sz[fo])); }
                }
        f4set(dg, j, __fmul_rn(d, factor));
        f4set(vx, j, __fmul_rn(tx, factor));
        f4set(vy, j, __fmul_rn(ty, factor));
        f4set(vz, j, __fmul_rn(tz, factor));
    }
    finalize_leaf(O, leaf, t, m, dg, vx, vy, vz);
}

// init_SPAI0 (.cpp:1113-1190): a_kk / ||a_k||^2, trimmed against 6/(7 diag_bg)
__global__ void __launch_bounds__(128) k_spai0(DLevel L, float* spai0, uint32_t* flags, float defaultSPAI0Val,
                                               float eps) {
    __shared__ float sh[4];
    const int leaf = blockIdx.x, t = threadIdx.x;
    const unsigned m = mask4(L.mask, leaf, t);
    const int* nb = L.nbr + (long long)leaf * 6;
    float4 out = f4splat(defaultSPAI0Val);
    float err = 0.f;
    const float* arr[3] = {L.cx, L.cy, L.cz};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        const int off = 4 * t + j;
        const long long me = (long long)leaf * UAAMG_LEAF + off;
        float rs = 0.f;
        for (int c = 0; c < 3; ++c) {
            const int sh_ = (c == 0) ? 64 : (c == 1 ? 8 : 1);
            const int loc = (c == 0) ? (off >> 6) : (c == 1 ? ((off >> 3) & 7) : (off & 7));
            // + neighbour: its own minus-face entry
            int nl = leaf, no = off + sh_;
            if (loc == 7) { nl = nb[2 * c + 1]; no = off - 7 * sh_; }
            if (nl >= 0 && ((L.mask[(long long)nl * 8 + (no >> 6)] >> (no & 63)) & 1ull)) {
                float v = arr[c][(long long)nl * UAAMG_LEAF + no];
                rs = __fadd_rn(rs, __fmul_rn(v, v));
            }
            // - neighbour: this voxel's minus-face entry
            nl = leaf; no = off - sh_;
            if (loc == 0) { nl = nb[2 * c]; no = off + 7 * sh_; }
            if (nl >= 0 && ((L.mask[(long long)nl * 8 + (no >> 6)] >> (no & 63)) & 1ull)) {
                float v = arr[c][me];
                rs = __fadd_rn(rs, __fmul_rn(v, v));
            }
        }
        const float d = L.diag[me];
        const float s = (d == 0.f) ? 0.f : __fdiv_rn(d, __fadd_rn(__fmul_rn(d, d), rs));
        f4set(out, j, s);
        err = fmaxf(err, fabsf(__fsub_rn(s, defaultSPAI0Val)));
    }
    const bool trimmed = block_max128f(err, sh) <= eps;
    if (trimmed) out = f4splat(L.def_spai0);
    st4(spai0, leaf, t, out);
    if (t == 0 && trimmed) flags[leaf] |= TRIM_SPAI0;
}

// explicit coarsest matrix in DOF order (getTriplets, .cpp:129-206)
__global__ void __launch_bounds__(128) k_coarsest_ell(DLevel L, const int* dof_base, int* dof_slot, float* diag,
                                                      float* invd, int* col, float* val) {
    // the leaf's and its six face neighbours' DOF masks and DOF bases, staged
    // once (slot 0: the leaf, 1 + 2c + s: neighbour -/+ along axis c)
    __shared__ uint64_t mks[7][8];
    __shared__ int nbl[7], nbase[7];
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (t < 7) {
        const int n = t == 0 ? leaf : L.nbr[(long long)leaf * 6 + t - 1];
        nbl[t] = n;
        nbase[t] = n >= 0 ? dof_base[n] : 0;
    }
    __syncthreads();
    if (t < 56) mks[t >> 3][t & 7] = nbl[t >> 3] >= 0 ? L.mask[(long long)nbl[t >> 3] * 8 + (t & 7)] : 0ull;
    __syncthreads();
    const unsigned m = mask4(L.mask, leaf, t);
    const uint64_t* mk = mks[0];
    const float* arr[3] = {L.cx, L.cy, L.cz};
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        const int off = 4 * t + j;
        const long long me = (long long)leaf * UAAMG_LEAF + off;
        int row = nbase[0];
        for (int w = 0; w < (off >> 6); ++w) row += __popcll(mk[w]);
        row += __popcll(mk[off >> 6] & ((1ull << (off & 63)) - 1ull));
        dof_slot[row] = (int)me;
        const float dgv = L.diag[me];
        diag[row] = dgv;
        invd[row] = (dgv != 0.f) ? __fdiv_rn(1.0f, dgv) : 1.0f;
        for (int c = 0; c < 3; ++c) {
            const int sh_ = (c == 0) ? 64 : (c == 1 ? 8 : 1);
            const int loc = (c == 0) ? (off >> 6) : (c == 1 ? ((off >> 3) & 7) : (off & 7));
            for (int s = 0; s < 2; ++s) {
                int slot = 0, no;
                if (s == 0) { no = off - sh_; if (loc == 0) { slot = 1 + 2 * c; no = off + 7 * sh_; } }
                else { no = off + sh_; if (loc == 7) { slot = 2 + 2 * c; no = off - 7 * sh_; } }
                const int nl = nbl[slot];
                const int e = 2 * c + s;
                const uint64_t* nm = mks[slot];
                if (nl >= 0 && ((nm[no >> 6] >> (no & 63)) & 1ull)) {
                    int d = nbase[slot];
                    for (int w = 0; w < (no >> 6); ++w) d += __popcll(nm[w]);
                    d += __popcll(nm[no >> 6] & ((1ull << (no & 63)) - 1ull));
                    col[row * 6 + e] = d;
                    val[row * 6 + e] = (s == 0) ? arr[c][me] : arr[c][(long long)nl * UAAMG_LEAF + no];
                } else {
                    col[row * 6 + e] = -1;
                    val[row * 6 + e] = 0.f;
                }
            }
        }
    }
}

// BuildPoissonRhs (.cpp:19-93): rhs = -(1/dx) sum_k [F_k(c+e_k) - F_k(c)],
// F = w u + (1-w) u_solid; zero when all six face weights are zero.
__global__ void __launch_bounds__(128) k_build_rhs(const uint64_t* mask, const int* org, DGrid fw, DGrid vx, DGrid vy,
                                                   DGrid vz, DGrid sv, float invdx, float* rhs) {
    __shared__ int li[5][7];
    const int leaf = blockIdx.x, t = threadIdx.x;
    const unsigned m = mask4(mask, leaf, t);
    float4 out = f4zero();
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
    nb7_resolve(fw, ox, oy, oz, t, li[0]);
    nb7_resolve(vx, ox, oy, oz, t, li[1]);
    nb7_resolve(vy, ox, oy, oz, t, li[2]);
    nb7_resolve(vz, ox, oy, oz, t, li[3]);
    nb7_resolve(sv, ox, oy, oz, t, li[4]);
    __syncthreads();
    const DGridNb FW{&fw, li[0], ox, oy, oz}, SV{&sv, li[4], ox, oy, oz};
    const DGridNb VX{&vx, li[1], ox, oy, oz}, VY{&vy, li[2], ox, oy, oz}, VZ{&vz, li[3], ox, oy, oz};
    const DGridNb* vel[3] = {&VX, &VY, &VZ};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!((m >> j) & 1)) continue;
        const int off = 4 * t + j;
        const int g[3] = {ox + (off >> 6), oy + ((off >> 3) & 7), oz + (off & 7)};
        float r = 0.f;
        bool nz = false;
        for (int f = 0; f < 6; ++f) {
            const int ch = f >> 1;
            const bool pos = (f & 1) == 0;
            int c[3] = {g[0], g[1], g[2]};
            if (pos) c[ch] += 1;
            const float w = FW.get(c[0], c[1], c[2], ch);
            if (w != 0.f) nz = true;
            const float v = vel[ch]->get(c[0], c[1], c[2], 0);
            const float s = SV.get(c[0], c[1], c[2], ch);
            const float flux = __fmul_rn(invdx, __fadd_rn(__fmul_rn(w, v), __fmul_rn(__fsub_rn(1.0f, w), s)));
            r = pos ? __fsub_rn(r, flux) : __fadd_rn(r, flux);
        }
        f4set(out, j, nz ? r : 0.f);
    }
    st4(rhs, leaf, t, out);
}

}  // namespace uaamg
