// projection.cu -- the two steps either side of the pressure solve in a FLIP
// projection, on the device: the solid face weights the solver reads
// (FLIP_Solver_OpenVDB::calculate_face_weights, FLIP_vdb/FLIP_vdb.cpp:2669-2752)
// and the pressure-gradient velocity update that consumes its solution
// (FLIP_Solver_OpenVDB::apply_pressure_gradient, FLIP_vdb.cpp:2571-2667), and
// the ghost-fluid adjustment of the liquid SDF inside solids between them
// (FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids, FLIP_vdb.cpp:2856-2942).
// Included by uaamg_lib.cu after poisson.cu (grids, handle, errors).

namespace uaamg {

// fraction_inside(phi_bl, phi_br, phi_tl, phi_tr) (SIMD_UAAMG/levelset_util.cpp:23-100):
// the fraction of a square with the given corner values that is inside.  The
// corners are visited in the order bl, br, tr, tl and rotated as the
// reference's cycle_array does; float operations in the reference's order.
__device__ __forceinline__ float fi4_rotate_to(float* l, int k) {  // rotate left by k (0..3)
    float t[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) t[i] = l[(i + k) & 3];
#pragma unroll
    for (int i = 0; i < 4; ++i) l[i] = t[i];
    return 0.f;
}
__device__ __forceinline__ float fraction_inside4(float bl, float br, float tl, float tr) {
    const int inside = (bl < 0 ? 1 : 0) + (tl < 0 ? 1 : 0) + (br < 0 ? 1 : 0) + (tr < 0 ? 1 : 0);
    float l[4] = {bl, br, tr, tl};
    if (inside == 4) return 1.f;
    if (inside == 3) {
        int k = 0;
        while (k < 3 && l[k] < 0) ++k;  // the corner that is not inside
        fi4_rotate_to(l, k);
        const float side0 = __fsub_rn(1.f, fraction_inside1(l[0], l[3]));
        const float side1 = __fsub_rn(1.f, fraction_inside1(l[0], l[1]));
        return __fsub_rn(1.f, __fmul_rn(__fmul_rn(0.5f, side0), side1));
    }
    if (inside == 2) {
        // rotate until a negative value is first and the next negative is in slot 1 or 2
        int k = 0;
        for (; k < 4; ++k) {  // the reference's loop condition, negated
            const float a = l[k & 3], b = l[(k + 1) & 3], c = l[(k + 2) & 3];
            if (!(a >= 0 || !(b < 0 || c < 0))) break;
        }
        fi4_rotate_to(l, k & 3);
        if (l[1] < 0) {  // matching signs adjacent
            const float left = fraction_inside1(l[0], l[3]);
            const float right = fraction_inside1(l[1], l[2]);
            return __fmul_rn(0.5f, __fadd_rn(left, right));
        }
        // matching signs diagonally opposite: the centre's sign disambiguates
        const float mid = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(l[0], l[1]), l[2]), l[3]));
        if (mid < 0) {
            float area = 0.f;
            const float side1 = __fsub_rn(1.f, fraction_inside1(l[0], l[3]));
            const float side3 = __fsub_rn(1.f, fraction_inside1(l[2], l[3]));
            area = __fadd_rn(area, __fmul_rn(__fmul_rn(0.5f, side1), side3));
            const float side2 = __fsub_rn(1.f, fraction_inside1(l[2], l[1]));
            const float side0 = __fsub_rn(1.f, fraction_inside1(l[0], l[1]));
            area = __fadd_rn(area, __fmul_rn(__fmul_rn(0.5f, side0), side2));
            return __fsub_rn(1.f, area);
        }
        float area = 0.f;
        const float side0 = fraction_inside1(l[0], l[1]);
        const float side1 = fraction_inside1(l[0], l[3]);
        area = __fadd_rn(area, __fmul_rn(__fmul_rn(0.5f, side0), side1));
        const float side2 = fraction_inside1(l[2], l[1]);
        const float side3 = fraction_inside1(l[2], l[3]);
        area = __fadd_rn(area, __fmul_rn(__fmul_rn(0.5f, side2), side3));
        return area;
    }
    if (inside == 1) {
        int k = 0;
        while (k < 3 && l[k] >= 0) ++k;  // the negative corner
        fi4_rotate_to(l, k);
        const float side0 = fraction_inside1(l[0], l[3]);
        const float side1 = fraction_inside1(l[0], l[1]);
        return __fmul_rn(__fmul_rn(0.5f, side0), side1);
    }
    return 0.f;
}

// std::max(0.f, std::min(v, 1.f)) with the standard library's comparisons
// (a NaN becomes 0)
__device__ __forceinline__ float clamp01(float v) {
    const float m = (1.f < v) ? 1.f : v;
    return (0.f < m) ? m : 0.f;
}

// calculate_face_weights for the active voxels of the output leaves: the
// fraction of each of the voxel's three minus faces that is not inside the
// solid, from the solid SDF at the 8 voxel corners (g + {0,1}^3); weights
// below 1e-2 become 0.  out: [leaf][512][3], inactive voxels keep (1, 1, 1)
// (the output grid's background).
__global__ void __launch_bounds__(128) k_face_weights(DGrid solid, const int* org, const uint64_t* mask, int nl,
                                                      float* out) {
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (leaf >= nl) return;
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const int off = 4 * t + j;
        float* o = out + ((long long)leaf * UAAMG_LEAF + off) * 3;
        if (mask && !((mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull)) {
            o[0] = o[1] = o[2] = 1.f;
            continue;
        }
        const int gx = ox + (off >> 6), gy = oy + ((off >> 3) & 7), gz = oz + (off & 7);
        float s[2][2][2];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int m = 0; m < 2; ++m) s[i][k][m] = solid.get(gx + i, gy + k, gz + m, 0);
        float w0 = clamp01(__fsub_rn(1.f, fraction_inside4(s[0][0][0], s[0][1][0], s[0][0][1], s[0][1][1])));
        float w1 = clamp01(__fsub_rn(1.f, fraction_inside4(s[0][0][0], s[0][0][1], s[1][0][0], s[1][0][1])));
        float w2 = clamp01(__fsub_rn(1.f, fraction_inside4(s[0][0][0], s[1][0][0], s[0][1][0], s[1][1][0])));
        if (w0 < 1e-2f) w0 = 0.f;
        if (w1 < 1e-2f) w1 = 0.f;
        if (w2 < 1e-2f) w2 = 0.f;
        o[0] = w0;
        o[1] = w1;
        o[2] = w2;
    }
}

// The pressure vector of a Poisson handle's level 0 as an accessor:
// getValue (the stored value, 0 outside the leaves) and isValueOn (a DOF).
struct PGrid {
    const float* p;
    const uint64_t* mask;
    const int* map;
    int lo0, lo1, lo2, d0, d1, d2;
    __device__ __forceinline__ int leaf_of(int x, int y, int z) const {
        const int a = (x >> 3) - lo0, b = (y >> 3) - lo1, c = (z >> 3) - lo2;
        if ((unsigned)a >= (unsigned)d0 || (unsigned)b >= (unsigned)d1 || (unsigned)c >= (unsigned)d2) return -1;
        return map[((long long)a * d1 + b) * d2 + c];
    }
    __device__ __forceinline__ void get(int x, int y, int z, float& v, bool& on) const {
        const int li = leaf_of(x, y, z);
        if (li < 0) {
            v = 0.f;
            on = false;
            return;
        }
        const int off = ((x & 7) << 6) | ((y & 7) << 3) | (z & 7);
        v = p[(long long)li * UAAMG_LEAF + off];
        on = (mask[(long long)li * 8 + (off >> 6)] >> (off & 63)) & 1ull;
    }
};

// apply_pressure_gradient for one velocity channel c over the active voxels
// of its leaves: where the face has a positive weight and a DOF on either
// side, u += -dt (p - p_below) / dx / theta (theta: the liquid fraction of the
// segment between the two cell centres, at least 0.02, when either side is
// air), the reflected velocity is u + the update, and a partly solid face
// blends in the solid velocity by (1 - w) * friction.  Voxels without an
// update become inactive (mask_out) and keep their value; update_out holds
// the update where there is one, else the input value (the reference's copy
// of the velocity grid); reflected_out likewise.
__global__ void __launch_bounds__(128) k_pressure_gradient(DGrid phi, DGrid fw, DGrid sv, PGrid P, int c,
                                                           const int* org, const uint64_t* mask_in, float* vel,
                                                           uint64_t* mask_out, float* upd_out, float* refl_out,
                                                           float dt, float dx, float friction) {
    __shared__ uint32_t bits[16];
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (t < 16) bits[t] = 0;
    __syncthreads();
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
    const float ndt = -dt;
    unsigned my = 0;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const int off = 4 * t + j;
        const long long i = (long long)leaf * UAAMG_LEAF + off;
        const float u = vel[i];
        float up = u, refl = u;
        const bool active = !mask_in || ((mask_in[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull);
        bool has = false;
        if (active) {
            int g[3] = {ox + (off >> 6), oy + ((off >> 3) & 7), oz + (off & 7)};
            int b[3] = {g[0], g[1], g[2]};
            b[c] -= 1;
            const float w = fw.get(g[0], g[1], g[2], c);
            if (w > 0.f) {
                float p_this, p_below;
                bool on_this, on_below;
                P.get(g[0], g[1], g[2], p_this, on_this);
                P.get(b[0], b[1], b[2], p_below, on_below);
                if (on_this || on_below) {
                    has = true;
                    const float phi_this = phi.get(g[0], g[1], g[2], 0);
                    const float phi_below = phi.get(b[0], b[1], b[2], 0);
                    float theta = 1.f;
                    if (phi_this >= 0 || phi_below >= 0) {
                        theta = fraction_inside1(phi_below, phi_this);
                        if (theta < 0.02f) theta = 0.02f;
                    }
                    float d = __fmul_rn(ndt, __fsub_rn(p_this, p_below));
                    d = __fdiv_rn(d, dx);
                    d = __fdiv_rn(d, theta);
                    float nv = __fadd_rn(u, d);
                    refl = __fadd_rn(nv, d);
                    if (w < 1.0f) {
                        const float svel = sv.get(g[0], g[1], g[2], c);
                        const float sf = __fmul_rn(__fsub_rn(1.f, w), friction);
                        nv = __fadd_rn(__fmul_rn(__fsub_rn(1.f, sf), nv), __fmul_rn(sf, svel));
                    }
                    vel[i] = nv;
                    up = d;
                }
            }
        }
        if (upd_out) upd_out[i] = up;
        if (refl_out) refl_out[i] = refl;
        if (has) my |= 1u << j;
    }
    atomicOr(&bits[t >> 3], my << ((t & 7) * 4));
    __syncthreads();
    if (t < 8) mask_out[(long long)leaf * 8 + t] = (uint64_t)bits[2 * t] | ((uint64_t)bits[2 * t + 1] << 32);
}

}  // namespace uaamg

// ---------------------------------------------------------------------------
// C ABI

namespace {

// the output topology of the face weights: origins (multiples of 8) and optional masks
static void check_topology(int64_t n, const int32_t* org, const char* name) {
    if (n < 0 || (n > 0 && !org)) {
        set_error("%s: invalid leaf list", name);
        throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
    }
    for (int64_t i = 0; i < 3 * n; ++i)
        if (org[i] & 7) {
            set_error("%s: leaf origins must be multiples of 8", name);
            throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
        }
}

static void face_weights_impl(const uaamg_leaf_grid* solid, int64_t n, const int32_t* org, const uint64_t* masks,
                              float* d_out, cudaStream_t s) {
    check_grid(solid, 1, "solid_sdf");
    check_topology(n, org, "face weights");
    if (n == 0) return;
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    std::vector<void*> tofree;
    HostMap m;
    DevGrid g;
    upload_grid_cs(ctx, s, solid, g, m, tofree);
    void* mem = nullptr;
    const size_t ob = carve_size((size_t)n * 3, 4), mb = masks ? carve_size((size_t)n * 8, 8) : 0;
    CK(ctx_dev_alloc(ctx, &mem, ob + mb, s));
    tofree.push_back(mem);
    char* cur = (char*)mem;
    int* dorg = carve<int>(cur, (size_t)n * 3);
    uint64_t* dmask = masks ? carve<uint64_t>(cur, (size_t)n * 8) : nullptr;
    CK(cudaMemcpyAsync(dorg, org, (size_t)n * 12, cudaMemcpyHostToDevice, s));
    if (masks) CK(cudaMemcpyAsync(dmask, masks, (size_t)n * 64, cudaMemcpyHostToDevice, s));
    k_face_weights<<<(unsigned)n, 128, 0, s>>>(g.g, dorg, dmask, (int)n, d_out);
    CHECK_LAUNCH();
    for (void* p : tofree) CK(cudaFreeAsync(p, s));
}

static void pressure_gradient_impl(uaamg_poisson* h, const uaamg_leaf_grid* phi, const uaamg_leaf_grid* fw,
                                   const uaamg_leaf_grid* sv, const float* d_pressure, int channel,
                                   const uaamg_leaf_grid* vel, float* d_vel, uint64_t* d_mask_out, float* d_upd,
                                   float* d_refl, float dt, float friction) {
    check_grid(phi, 1, "liquid_phi");
    check_grid(fw, 3, "face_weights");
    check_grid(sv, 3, "solid_velocity");
    check_grid(vel, 1, "velocity");
    require(channel >= 0 && channel <= 2, "channel must be 0, 1 or 2");
    require(d_pressure || h->lv[0].L.nl == 0, "NULL pressure");
    const int64_t n = vel->leaf_count;
    if (n == 0) return;
    require(d_vel && d_mask_out, "NULL velocity or mask output");
    cudaStream_t s = h->stream;
    std::vector<void*> tofree;
    HostMap m0, m1, m2;
    DevGrid g0, g1, g2;
    upload_grid(h, phi, g0, m0, tofree);
    upload_grid(h, fw, g1, m1, tofree);
    upload_grid(h, sv, g2, m2, tofree);
    // the pressure's accessor: the handle's level-0 leaf map and DOF masks
    const HostMap& pm = h->host[0].map;
    PGrid P{};
    P.p = d_pressure;
    P.mask = h->lv[0].L.mask;
    const size_t mapn = pm.idx.size();
    const size_t vn = (size_t)n;
    void* mem = nullptr;
    CK(ctx_dev_alloc(h->ctx, &mem, carve_size(mapn ? mapn : 1, 4) + carve_size(vn * 3, 4) +
                                       (vel->masks ? carve_size(vn * 8, 8) : 0), s));
    tofree.push_back(mem);
    char* cur = (char*)mem;
    int* dmap = carve<int>(cur, mapn ? mapn : 1);
    int* dorg = carve<int>(cur, vn * 3);
    uint64_t* dmin = vel->masks ? carve<uint64_t>(cur, vn * 8) : nullptr;
    if (mapn) CK(cudaMemcpyAsync(dmap, pm.idx.data(), mapn * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dorg, vel->origins, vn * 12, cudaMemcpyHostToDevice, s));
    if (dmin) CK(cudaMemcpyAsync(dmin, vel->masks, vn * 64, cudaMemcpyHostToDevice, s));
    P.map = dmap;
    P.lo0 = pm.lo[0]; P.lo1 = pm.lo[1]; P.lo2 = pm.lo[2];
    P.d0 = mapn ? pm.dim[0] : 0; P.d1 = pm.dim[1]; P.d2 = pm.dim[2];
    k_pressure_gradient<<<(unsigned)n, 128, 0, s>>>(g0.g, g1.g, g2.g, P, channel, dorg, dmin, d_vel, d_mask_out,
                                                    d_upd, d_refl, dt, h->lv[0].dx, friction);
    CHECK_LAUNCH();
    h->launches++;
    for (void* p : tofree) CK(cudaFreeAsync(p, s));
}

// immerse_liquid_phi_in_solids (FLIP_vdb/FLIP_vdb.cpp:2856-2942), the value
// passes, over the liquid SDF's leaves as they were before its 26-neighbour
// dilation (the reference's LeafManager is built at :2876, before the dilation
// at :2881, and reused at :2938).  A leaf takes part when the solid SDF has a
// leaf at its origin (probeConstLeaf).  The solid SDF is sampled at voxel
// centres with BoxSampler.  Pass 1 (:2860-2877): active voxels inside the
// solid get phi - dx/2; the result is the reference copy `ref` of both passes.
__global__ void __launch_bounds__(128) k_immerse_correct(DGrid solid, DGrid liq, const int* org,
                                                         const uint64_t* mask, int nl, float half_dx, float* ref) {
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (leaf >= nl) return;
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
    const bool gated = solid.leaf_of(ox, oy, oz) >= 0;
    const float* vin = liq.val + (long long)leaf * UAAMG_LEAF;
    float* r = ref + (long long)leaf * UAAMG_LEAF;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const int off = t + 128 * j;
        float v = vin[off];
        if (gated && (!mask || ((mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull))) {
            const float sv = box_sample(solid, (double)(ox + (off >> 6)) + 0.5, (double)(oy + ((off >> 3) & 7)) + 0.5,
                                        (double)(oz + (off & 7)) + 0.5);
            if (sv < 0.f) v = __fsub_rn(v, half_dx);
        }
        r[off] = v;
    }
}

// Pass 2 (:2883-2938): every voxel active after the dilation (itself or one of
// its 26 neighbours active in `mask`) whose solid sample is negative takes the
// least of 3 dx and the reference values of its face neighbours, visited in
// the order +x, -x, +y, -y, +z, -z up to the first negative one, if there is
// one (std::min: a NaN neighbour is skipped); else a negative value becomes
// std::max(background, -solid).  Other voxels keep the reference value.
// refg: the liquid's leaf map over `ref`, background = the liquid's.
__global__ void __launch_bounds__(128) k_immerse_solid(DGrid solid, DGrid refg, const int* org, const uint64_t* mask,
                                                       int nl, float three_dx, float* out) {
    const int leaf = blockIdx.x, t = threadIdx.x;
    if (leaf >= nl) return;
    const int ox = org[3 * leaf], oy = org[3 * leaf + 1], oz = org[3 * leaf + 2];
    const bool gated = solid.leaf_of(ox, oy, oz) >= 0;
    const float* r = refg.val + (long long)leaf * UAAMG_LEAF;
    float* o = out + (long long)leaf * UAAMG_LEAF;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const int off = t + 128 * j;
        float v = r[off];
        if (gated) {
            const int gx = ox + (off >> 6), gy = oy + ((off >> 3) & 7), gz = oz + (off & 7);
            bool on = false;
#pragma unroll 1
            for (int a = -1; a <= 1 && !on; ++a)
#pragma unroll 1
                for (int b = -1; b <= 1 && !on; ++b)
#pragma unroll 1
                    for (int c = -1; c <= 1 && !on; ++c) {
                        const int x = gx + a, y = gy + b, z = gz + c;
                        const int q = refg.leaf_of(x, y, z);
                        if (q >= 0) {
                            const int qo = voff3(x, y, z);
                            on = !mask || ((mask[(long long)q * 8 + (qo >> 6)] >> (qo & 63)) & 1ull);
                        }
                    }
            if (on) {
                const float sv = box_sample(solid, (double)gx + 0.5, (double)gy + 0.5, (double)gz + 0.5);
                if (sv < 0.f) {
                    bool found = false;
                    float mn = three_dx;
#pragma unroll 1
                    for (int i = 0; i < 6 && !found; ++i) {
                        const int sx = (i == 0) - (i == 1), sy = (i == 2) - (i == 3), sz = (i == 4) - (i == 5);
                        const float rv = refg.get(gx + sx, gy + sy, gz + sz, 0);
                        mn = (rv < mn) ? rv : mn;
                        found = found || (rv < 0.f);
                    }
                    if (found) {
                        v = mn;
                    } else if (v < 0.f) {
                        const float ns = -sv;
                        v = (refg.bg0 < ns) ? ns : refg.bg0;
                    }
                }
            }
        }
        o[off] = v;
    }
}

static void immerse_impl(const uaamg_leaf_grid* solid, const uaamg_leaf_grid* liquid, float dx, float* d_out,
                         cudaStream_t s) {
    check_grid(solid, 1, "solid_sdf");
    check_grid(liquid, 1, "liquid_phi");
    require(std::isfinite(dx) && dx > 0.f, "dx must be positive");
    const int64_t n = liquid->leaf_count;
    if (n == 0) return;
    require(d_out != nullptr, "NULL output");
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    std::vector<void*> tofree;
    try {
        HostMap ms, ml;
        DevGrid gs, gl;
        upload_grid_cs(ctx, s, solid, gs, ms, tofree);
        upload_grid_cs(ctx, s, liquid, gl, ml, tofree);
        for (int64_t i = 0; i < n; ++i)
            if (ml.idx[ml.cell(liquid->origins[3 * i] >> 3, liquid->origins[3 * i + 1] >> 3,
                               liquid->origins[3 * i + 2] >> 3)] != (int32_t)i) {
                set_error("liquid_phi: duplicate leaf origin");
                throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
            }
        const size_t vn = (size_t)n;
        void* mem = nullptr;
        CK(ctx_dev_alloc(ctx, &mem, carve_size(vn * 3, 4) + (liquid->masks ? carve_size(vn * 8, 8) : 0) +
                                        carve_size(vn * UAAMG_LEAF, 4), s));
        tofree.push_back(mem);
        char* cur = (char*)mem;
        int* dorg = carve<int>(cur, vn * 3);
        uint64_t* dmask = liquid->masks ? carve<uint64_t>(cur, vn * 8) : nullptr;
        float* ref = carve<float>(cur, vn * UAAMG_LEAF);
        CK(cudaMemcpyAsync(dorg, liquid->origins, vn * 12, cudaMemcpyHostToDevice, s));
        if (dmask) CK(cudaMemcpyAsync(dmask, liquid->masks, vn * 64, cudaMemcpyHostToDevice, s));
        k_immerse_correct<<<(unsigned)n, 128, 0, s>>>(gs.g, gl.g, dorg, dmask, (int)n, 0.5f * dx, ref);
        CHECK_LAUNCH();
        DGrid refg = gl.g;
        refg.val = ref;
        k_immerse_solid<<<(unsigned)n, 128, 0, s>>>(gs.g, refg, dorg, dmask, (int)n, dx * 3.0f, d_out);
        CHECK_LAUNCH();
    } catch (...) {
        for (void* p : tofree) cudaFreeAsync(p, s);
        throw;
    }
    for (void* p : tofree) CK(cudaFreeAsync(p, s));
}

}  // namespace

extern "C" {

int uaamg_face_weights(const uaamg_leaf_grid* solid_sdf, int64_t leaf_count, const int32_t* origins,
                       const uint64_t* masks, float* weights) {
    ABI_BEGIN
    require(weights || leaf_count == 0, "NULL output");
    if (leaf_count <= 0) { check_topology(leaf_count, origins, "face weights"); return UAAMG_SUCCESS; }
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = nullptr;
    CK(ctx_stream_acquire(ctx, &s));
    float* d = nullptr;
    const size_t bytes = (size_t)leaf_count * UAAMG_LEAF * 3 * sizeof(float);
    try {
        CK(ctx_dev_alloc(ctx, (void**)&d, bytes, s));
        face_weights_impl(solid_sdf, leaf_count, origins, masks, d, s);
        CK(cudaMemcpyAsync(weights, d, bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(d, s));
        CK(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        ctx_stream_release(ctx, s);
        throw;
    }
    ctx_stream_release(ctx, s);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_face_weights_device(const uaamg_leaf_grid* solid_sdf, int64_t leaf_count, const int32_t* origins,
                              const uint64_t* masks, float* d_weights, void* stream) {
    ABI_BEGIN
    require(d_weights || leaf_count == 0, "NULL output");
    face_weights_impl(solid_sdf, leaf_count, origins, masks, d_weights, (cudaStream_t)stream);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_apply_pressure_gradient(uaamg_poisson* h, const uaamg_leaf_grid* liquid_phi,
                                          const uaamg_leaf_grid* face_weights, const uaamg_leaf_grid* solid_velocity,
                                          const float* pressure, float dt, float friction, int channel,
                                          const uaamg_leaf_grid* velocity, float* velocity_out, uint64_t* mask_out,
                                          float* update_out, float* reflected_out) {
    ABI_BEGIN
    require(h && velocity && velocity_out && mask_out, "NULL argument");
    require(!velocity->values_on_device, "host form: velocity values must be host pointers");
    const int64_t n = velocity->leaf_count;
    if (n <= 0) return UAAMG_SUCCESS;
    cudaStream_t s = h->stream;
    const size_t vb = (size_t)n * UAAMG_LEAF * 4, pb = vec_bytes(h, 0);
    float* d = nullptr;
    CK(ctx_dev_alloc(h->ctx, (void**)&d, 3 * vb + (size_t)n * 64 + pb + 256, s));
    float* dvel = d;
    float* dupd = d + vb / 4;
    float* drefl = d + 2 * (vb / 4);
    uint64_t* dmask = reinterpret_cast<uint64_t*>(d + 3 * (vb / 4));
    float* dp = reinterpret_cast<float*>(dmask + (size_t)n * 8);
    try {
        CK(cudaMemcpyAsync(dvel, velocity->values, vb, cudaMemcpyHostToDevice, s));
        if (pb) CK(cudaMemcpyAsync(dp, pressure, pb, cudaMemcpyHostToDevice, s));
        pressure_gradient_impl(h, liquid_phi, face_weights, solid_velocity, dp, channel, velocity, dvel, dmask,
                               update_out ? dupd : nullptr, reflected_out ? drefl : nullptr, dt, friction);
        CK(cudaMemcpyAsync(velocity_out, dvel, vb, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(mask_out, dmask, (size_t)n * 64, cudaMemcpyDeviceToHost, s));
        if (update_out) CK(cudaMemcpyAsync(update_out, dupd, vb, cudaMemcpyDeviceToHost, s));
        if (reflected_out) CK(cudaMemcpyAsync(reflected_out, drefl, vb, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(d, s));
        CK(cudaStreamSynchronize(s));
    } catch (...) {
        cudaFreeAsync(d, s);
        cudaStreamSynchronize(s);
        throw;
    }
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_apply_pressure_gradient_device(uaamg_poisson* h, const uaamg_leaf_grid* liquid_phi,
                                                 const uaamg_leaf_grid* face_weights,
                                                 const uaamg_leaf_grid* solid_velocity, const float* d_pressure,
                                                 float dt, float friction, int channel,
                                                 const uaamg_leaf_grid* velocity, float* d_velocity,
                                                 uint64_t* d_mask_out, float* d_update_out, float* d_reflected_out) {
    ABI_BEGIN
    require(h && velocity, "NULL argument");
    pressure_gradient_impl(h, liquid_phi, face_weights, solid_velocity, d_pressure, channel, velocity, d_velocity,
                           d_mask_out, d_update_out, d_reflected_out, dt, friction);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_immerse_liquid_phi(const uaamg_leaf_grid* solid_sdf, const uaamg_leaf_grid* liquid_phi, float dx,
                             float* values_out) {
    ABI_BEGIN
    require(liquid_phi != nullptr, "liquid_phi is NULL");
    const int64_t n = liquid_phi->leaf_count;
    if (n <= 0) {
        check_grid(solid_sdf, 1, "solid_sdf");
        return UAAMG_SUCCESS;
    }
    require(values_out != nullptr, "NULL output");
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = nullptr;
    CK(ctx_stream_acquire(ctx, &s));
    float* d = nullptr;
    const size_t bytes = (size_t)n * UAAMG_LEAF * sizeof(float);
    try {
        CK(ctx_dev_alloc(ctx, (void**)&d, bytes, s));
        immerse_impl(solid_sdf, liquid_phi, dx, d, s);
        CK(cudaMemcpyAsync(values_out, d, bytes, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(d, s));
        d = nullptr;
        CK(cudaStreamSynchronize(s));
    } catch (...) {
        if (d) cudaFreeAsync(d, s);
        cudaStreamSynchronize(s);
        ctx_stream_release(ctx, s);
        throw;
    }
    ctx_stream_release(ctx, s);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_immerse_liquid_phi_device(const uaamg_leaf_grid* solid_sdf, const uaamg_leaf_grid* liquid_phi, float dx,
                                    float* d_values_out, void* stream) {
    ABI_BEGIN
    require(liquid_phi != nullptr, "liquid_phi is NULL");
    immerse_impl(solid_sdf, liquid_phi, dx, d_values_out, (cudaStream_t)stream);
    return UAAMG_SUCCESS;
    ABI_END
}

}  // extern "C"
