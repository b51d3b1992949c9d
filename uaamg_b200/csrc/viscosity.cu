// viscosity.cu -- host side of the B200 variational-viscosity UAAMG-PCG
// (the reference's simd_viscosity3d / L_with_level) and its C ABI.
//
// What runs where
//  * host (C++): leaf sets of the OpenVDB dilations (bit operations on the
//    64-byte masks, O(leaves)), leaf ordering, DOF numbering bases, neighbour /
//    child tables and the coarse DOF masks, then one upload per level;
//  * device: every numeric step -- subcell SDF and volume fractions, control
//    volumes, solid faces and DOF marking, level-0 coefficients, Galerkin
//    coarsening, trimming, the coarsest explicit matrix, the right-hand side
//    and the whole PCG (mu-cycle with red-black Gauss-Seidel, device-resident
//    scalars, optionally one CUDA graph with a conditional WHILE node).
// Compiled into the same translation unit as poisson.cu (uaamg_lib.cu) and
// shares its error handling, resource pools and launch helpers.
#include <climits>

#include "viscosity_build.cuh"

namespace {

// ---------------------------------------------------------------------------
// Leaves of dilateActiveValues(tree, r, NN_FACE_EDGE_VERTEX | NN_FACE) for a
// tree with the given leaves and active masks: the input leaves plus every
// neighbour leaf that a dilated active voxel enters.  Result in OpenVDB tree
// order.
static inline uint64_t zband(int lo, int hi) {  // bits with z in [lo, hi] in every (y) byte
    uint64_t b = 0;
    for (int z = lo; z <= hi; ++z) b |= 1ull << z;
    return b * 0x0101010101010101ull;
}
static inline uint64_t yband(int lo, int hi) {
    uint64_t b = 0;
    for (int y = lo; y <= hi; ++y) b |= 0xFFull << (8 * y);
    return b;
}
static void sort_unique_vdb(std::vector<int32_t>& org) {
    const size_t n = org.size() / 3;
    std::vector<std::pair<unsigned __int128, uint32_t>> keys(n);
    for (size_t i = 0; i < n; ++i) keys[i] = {vdb_key128(&org[3 * i]), (uint32_t)i};
    // a dense scan of a bounding box inside one 128^3 node is in tree order already
    if (!std::is_sorted(keys.begin(), keys.end())) std::sort(keys.begin(), keys.end());
    std::vector<int32_t> out;
    out.reserve(org.size());
    for (size_t i = 0; i < n; ++i) {
        if (i > 0 && keys[i - 1].first == keys[i].first) continue;
        const int32_t* o = &org[3 * keys[i].second];
        out.insert(out.end(), o, o + 3);
    }
    org.swap(out);
}
// Tree order of distinct leaves listed by a dense x-major scan of their cells:
// inside one 128^3 node the tree order is the x-major order of the node's
// leaf cells (vdb_key's last field), which the scan already follows, so only
// the nodes need ordering -- a counting pass by node rank, with the few nodes
// sorted by key, instead of a sort of every leaf's 128-bit key.
static void order_dense_scan(std::vector<int32_t>& org) {
    const size_t n = org.size() / 3;
    if (n < 2) return;
    int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            const int v = org[3 * i + c] >> 7;
            lo[c] = std::min(lo[c], v);
            hi[c] = std::max(hi[c], v);
        }
    const int64_t d1 = hi[1] - lo[1] + 1, d2 = hi[2] - lo[2] + 1;
    const int64_t ncell = (hi[0] - lo[0] + 1) * d1 * d2;
    if (ncell == 1) return;
    std::vector<uint32_t> cnt((size_t)ncell, 0), cell(n);
    for (size_t i = 0; i < n; ++i) {
        cell[i] = (uint32_t)(((int64_t)((org[3 * i] >> 7) - lo[0]) * d1 + ((org[3 * i + 1] >> 7) - lo[1])) * d2 +
                             ((org[3 * i + 2] >> 7) - lo[2]));
        cnt[cell[i]]++;
    }
    std::vector<std::pair<unsigned __int128, uint32_t>> nodes;
    for (int64_t k = 0; k < ncell; ++k)
        if (cnt[(size_t)k]) {
            const int32_t o[3] = {(int32_t)((k / (d1 * d2) + lo[0]) * 128), (int32_t)(((k / d2) % d1 + lo[1]) * 128),
                                  (int32_t)((k % d2 + lo[2]) * 128)};
            nodes.push_back({vdb_key128(o), (uint32_t)k});
        }
    std::sort(nodes.begin(), nodes.end());
    std::vector<uint32_t> start((size_t)ncell, 0);
    uint32_t acc = 0;
    for (const auto& nd : nodes) {
        start[nd.second] = acc;
        acc += cnt[nd.second];
    }
    std::vector<int32_t> out(org.size());
    for (size_t i = 0; i < n; ++i) {
        const size_t d = start[cell[i]]++;
        out[3 * d] = org[3 * i];
        out[3 * d + 1] = org[3 * i + 1];
        out[3 * d + 2] = org[3 * i + 2];
    }
    org.swap(out);
}
static void dilate_leaves(const int32_t* org, int64_t n, const uint64_t* masks, int r, bool face_only,
                          std::vector<int32_t>& out, bool vdb_order) {
    out.clear();
    if (n <= 0) return;
    // dense occupancy over the leaf bounding box with a one-leaf margin
    int mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            mn[c] = std::min(mn[c], org[3 * i + c] >> 3);
            mx[c] = std::max(mx[c], org[3 * i + c] >> 3);
        }
    const int64_t d0 = mx[0] - mn[0] + 3, d1 = mx[1] - mn[1] + 3, d2 = mx[2] - mn[2] + 3;
    if (d0 * d1 * d2 > (int64_t(1) << 30)) {
        set_error("leaf bounding box too large for the dense leaf map (%lld cells)", (long long)(d0 * d1 * d2));
        throw UaamgError{UAAMG_ERR_DOMAIN_TOO_LARGE};
    }
    std::vector<uint8_t> mark((size_t)(d0 * d1 * d2), 0);
    auto cell = [&](int a, int b, int c) { return ((size_t)(a - mn[0] + 1) * d1 + (b - mn[1] + 1)) * d2 + (c - mn[2] + 1); };
    const uint64_t ylo = yband(0, r - 1), yhi = yband(8 - r, 7), zlo = zband(0, r - 1), zhi = zband(8 - r, 7);
    for (int64_t i = 0; i < n; ++i) {
        const int a0 = org[3 * i] >> 3, b0 = org[3 * i + 1] >> 3, c0 = org[3 * i + 2] >> 3;
        mark[cell(a0, b0, c0)] = 1;
        uint64_t w[8];
        for (int k = 0; k < 8; ++k) w[k] = masks ? masks[8 * i + k] : ~0ull;
        uint64_t xa = 0, xl = 0, xh = 0;
        for (int k = 0; k < 8; ++k) {
            xa |= w[k];
            if (k <= r - 1) xl |= w[k];
            if (k >= 8 - r) xh |= w[k];
        }
        if (!xa) continue;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    const int nz = (dx != 0) + (dy != 0) + (dz != 0);
                    if (nz == 0 || (face_only && nz != 1)) continue;
                    uint64_t p = dx < 0 ? xl : (dx > 0 ? xh : xa);
                    if (dy < 0) p &= ylo; else if (dy > 0) p &= yhi;
                    if (dz < 0) p &= zlo; else if (dz > 0) p &= zhi;
                    if (p) mark[cell(a0 + dx, b0 + dy, c0 + dz)] = 1;
                }
    }
    for (int64_t a = 0; a < d0; ++a)
        for (int64_t b = 0; b < d1; ++b)
            for (int64_t c = 0; c < d2; ++c)
                if (mark[((size_t)a * d1 + b) * d2 + c]) {
                    out.push_back((int32_t)((a + mn[0] - 1) * 8));
                    out.push_back((int32_t)((b + mn[1] - 1) * 8));
                    out.push_back((int32_t)((c + mn[2] - 1) * 8));
                }
    if (vdb_order) order_dense_scan(out);  // the scan lists each leaf once
}

struct VHostLevel {
    int nl = 0;
    std::vector<int32_t> org;       // [nl][3]
    std::vector<uint64_t> dof;      // [3][nl][8]
    std::vector<int32_t> nb;        // [nl][27]
    std::vector<int32_t> dof_base;  // [3][nl]
    std::vector<int32_t> child;     // [nl][8]
    std::vector<int32_t> parent;    // [nl]
    std::vector<uint8_t> octant;    // [nl]
    int64_t ndof = 0;
    HostMap map;
};

// set_dof (:500-538): per channel, leaves in tree order, offsets ascending;
// numbering continues across channels
static void finalize_vlevel(VHostLevel& L) {
    // a one-leaf margin puts every leaf's 27 neighbour cells inside the map
    L.map.build(L.nl, L.org.data(), 1);
    L.nb.assign((size_t)L.nl * 27, -1);
    if (L.nl > 0) {
        const int64_t s0 = (int64_t)L.map.dim[1] * L.map.dim[2], s1 = L.map.dim[2];
        int64_t off[27];
        for (int a = 0; a < 27; ++a) off[a] = (a / 9 - 1) * s0 + ((a / 3) % 3 - 1) * s1 + (a % 3 - 1);
        const int32_t* idx = L.map.idx.data();
        for (int i = 0; i < L.nl; ++i) {
            const int32_t* o = &L.org[3 * i];
            const int64_t base = L.map.cell(o[0] >> 3, o[1] >> 3, o[2] >> 3);
            int32_t* nb = &L.nb[27 * (size_t)i];
            for (int a = 0; a < 27; ++a) nb[a] = idx[base + off[a]];
        }
    }
    L.dof_base.assign((size_t)3 * L.nl, 0);
    int64_t acc = 0;
    for (int c = 0; c < 3; ++c)
        acc = popc_prefix(&L.dof[(size_t)c * L.nl * 8], (size_t)L.nl, &L.dof_base[(size_t)c * L.nl], acc);
    L.ndof = acc;
    L.child.assign((size_t)L.nl * 8, -1);
    L.parent.assign((size_t)L.nl, -1);
    L.octant.assign((size_t)L.nl, 0);
}

// pattern leaves (DOF union dilated by r) carrying the given DOF masks
static void make_pattern_level(const std::vector<int32_t>& dl, const std::vector<uint64_t>& dm /*[3][nd][8]*/, int r,
                               VHostLevel& L) {
    const int64_t nd = (int64_t)(dl.size() / 3);
    std::vector<uint64_t> uni((size_t)nd * 8);
    for (int64_t i = 0; i < nd; ++i)
        for (int w = 0; w < 8; ++w)
            uni[8 * i + w] = dm[(0 * nd + i) * 8 + w] | dm[(1 * nd + i) * 8 + w] | dm[(2 * nd + i) * 8 + w];
    dilate_leaves(dl.data(), nd, uni.data(), r, false, L.org, true);
    L.nl = (int)(L.org.size() / 3);
    L.dof.assign((size_t)3 * L.nl * 8, 0);
    HostMap dmap;
    dmap.build(nd, dl.data());
    for (int i = 0; i < L.nl; ++i) {
        const int32_t* o = &L.org[3 * i];
        const int j = dmap.find_leaf(o[0] >> 3, o[1] >> 3, o[2] >> 3);
        if (j < 0) continue;
        for (int c = 0; c < 3; ++c)
            memcpy(&L.dof[((size_t)c * L.nl + i) * 8], &dm[((size_t)c * nd + j) * 8], 64);
    }
    finalize_vlevel(L);
}

// mark_dof_from_child (:1017-1065): coarse leaves are the parents of the fine
// leaves with DOFs; a coarse voxel is a DOF of channel c if any of its 2x2x2
// fine voxels is.  The coarse pattern dilates by 3 (:1361).
static void coarsen_vlevel(VHostLevel& F, VHostLevel& C) {
    std::vector<int32_t> dl;
    for (int i = 0; i < F.nl; ++i) {
        uint64_t any = 0;
        for (int c = 0; c < 3; ++c)
            for (int w = 0; w < 8; ++w) any |= F.dof[((size_t)c * F.nl + i) * 8 + w];
        if (!any) continue;
        for (int a = 0; a < 3; ++a) dl.push_back((F.org[3 * i + a] / 2) & ~7);
    }
    sort_unique_vdb(dl);
    const int64_t nd = (int64_t)(dl.size() / 3);
    std::vector<uint64_t> dm((size_t)3 * nd * 8, 0);
    for (int64_t i = 0; i < nd; ++i)
        for (int a = 0; a < 8; ++a) {
            const int fo[3] = {2 * dl[3 * i] + ((a >> 2) & 1) * 8, 2 * dl[3 * i + 1] + ((a >> 1) & 1) * 8,
                               2 * dl[3 * i + 2] + (a & 1) * 8};
            const int fl = F.map.find_leaf(fo[0] >> 3, fo[1] >> 3, fo[2] >> 3);
            if (fl < 0) continue;
            const int ox = (a >> 2) & 1, oy = (a >> 1) & 1, oz = a & 1;
            for (int c = 0; c < 3; ++c) {
                const uint64_t* fm = &F.dof[((size_t)c * F.nl + fl) * 8];
                for (int px = 0; px < 4; ++px) {
                    uint64_t p = fm[2 * px] | fm[2 * px + 1];
                    p |= (p >> 1);
                    p |= (p >> 8);
                    // bit 16*yy + 2*zz holds coarse voxel (yy, zz): compress each 16-bit group's bits 0, 2, 4, 6
                    // into its low nibble, then place nibble yy at row oy*4 + yy, columns oz*4 ..
                    uint64_t x = p & 0x0055005500550055ull;
                    x = (x | (x >> 1)) & 0x0033003300330033ull;
                    x = (x | (x >> 2)) & 0x000F000F000F000Full;
                    uint64_t& w = dm[((size_t)c * nd + i) * 8 + ox * 4 + px];
                    for (int yy = 0; yy < 4; ++yy) w |= ((x >> (16 * yy)) & 0xFull) << ((oy * 4 + yy) * 8 + oz * 4);
                }
            }
        }
    make_pattern_level(dl, dm, 3, C);
    for (int i = 0; i < C.nl; ++i)
        for (int a = 0; a < 8; ++a) {
            const int32_t* o = &C.org[3 * i];
            const int fl = F.map.find_leaf((2 * o[0] >> 3) + ((a >> 2) & 1), (2 * o[1] >> 3) + ((a >> 1) & 1),
                                           (2 * o[2] >> 3) + (a & 1));
            C.child[8 * i + a] = fl;
            if (fl >= 0) {
                F.parent[fl] = i;
                F.octant[fl] = (uint8_t)a;
            }
        }
}

struct VLevelDev {
    VLevel L{};
    float* lhs = nullptr;
    float* rhs = nullptr;
    float* alt = nullptr;  // second buffer of the fused red-black steps (zero at non-DOF voxel groups), when used
    int* dof_base = nullptr;
    int* org = nullptr;
};

}  // namespace

struct uaamg_viscosity {
    DeviceCtx* ctx = nullptr;
    void* pin_state = nullptr;
    size_t pin_state_cap = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t body_stream = nullptr;
    std::vector<VHostLevel> host;
    std::vector<VLevelDev> lv;
    int nlev = 0;
    // levels of at most this many leaves smooth with the fused red-black step
    // (k_vrbgs): latency-bound levels of about one wave at 2 CTAs per SM; larger
    // levels are issue-bound and the step's face-layer recomputation costs more
    // than the launch it saves
    int rb_fused_max_leaves = 0;
    // levels of more leaves run their red / black passes as k_vapply_seq
    // (more leaves than resident CTAs: the next leaf's table loads hide behind
    // the current leaf)
    int seq_min_leaves = INT_MAX;
    std::vector<void*> allocs;
    // level-0 construction products kept for the right-hand side
    VolFields V{};
    DGrid mu{};
    SolidInfo S{};
    int* org0 = nullptr;
    float* zpage = nullptr;  // [512] zeros
    DCoarsestV C{};
    float *x = nullptr, *b = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    double* partials = nullptr;
    PcgState* st = nullptr;
    PcgState* st_host = nullptr;
    float* scalar_dev = nullptr;
    float* scalar_host = nullptr;
    float dt = 0, rho = 0, dx = 0, factor = 0, def_off = 0, def_diag = 0;
    int max_iter = 100;
    float tol = 1e-6f;
    int use_graph = 1;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t graph = nullptr;
    std::shared_ptr<SolveGraph> shared_graph;  // set when graph / graph_exec belong to the solve-graph cache
    int64_t setup_launches = 0, body_launches = 0, finish_launches = 0;
    int64_t launches = 0, last_launches = 0;
    int iterations = 0;
    int status = UAAMG_SUCCESS;
    float final_residual = 0.f;
    int64_t solves = 0;
};

namespace {

static void* valloc(uaamg_viscosity* h, size_t bytes) {
    void* p = nullptr;
    CK(ctx_dev_alloc(h->ctx, &p, bytes ? bytes : 256, h->stream));
    h->allocs.push_back(p);
    return p;
}
template <typename T>
static T* vupload(uaamg_viscosity* h, const T* src, size_t count) {
    T* d = (T*)valloc(h, count * sizeof(T));
    if (count) CK(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return d;
}
static void vfree_now(uaamg_viscosity* h, void* p) {
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if (it != h->allocs.end()) h->allocs.erase(it);
    CK(cudaFreeAsync(p, h->stream));
}
static DMap vupload_map(uaamg_viscosity* h, const HostMap& m) {
    DMap d{};
    if (m.idx.empty()) return d;
    d.map = vupload(h, m.idx.data(), m.idx.size());
    d.lo0 = m.lo[0]; d.lo1 = m.lo[1]; d.lo2 = m.lo[2];
    d.d0 = m.dim[0]; d.d1 = m.dim[1]; d.d2 = m.dim[2];
    return d;
}
static DGrid vupload_grid(uaamg_viscosity* h, const uaamg_leaf_grid* gr) {
    DGrid g{};
    g.comps = gr->components;
    g.bg0 = gr->background[0];
    g.bg1 = gr->components > 1 ? gr->background[1] : 0.f;
    g.bg2 = gr->components > 2 ? gr->background[2] : 0.f;
    if (gr->leaf_count == 0) return g;
    HostMap map;
    map.build(gr->leaf_count, gr->origins);
    DMap dm = vupload_map(h, map);
    g.map = dm.map;
    g.lo0 = dm.lo0; g.lo1 = dm.lo1; g.lo2 = dm.lo2;
    g.d0 = dm.d0; g.d1 = dm.d1; g.d2 = dm.d2;
    const size_t nv = (size_t)gr->leaf_count * UAAMG_LEAF * gr->components;
    g.val = gr->values_on_device ? gr->values : vupload(h, gr->values, nv);
    return g;
}

template <typename... KArgs, typename... Args>
static void launch2(void (*kern)(KArgs...), dim3 grid, unsigned block, cudaStream_t s, Args... args) {
    if (grid.x == 0 || grid.y == 0) return;
    if (t_rec) {  // recording a solve for the solve-graph cache
        rec_launch(kern, grid, dim3(block), 0, g_use_pdl ? 1 : 0, args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_use_pdl ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

static void upload_vlevel(uaamg_viscosity* h, const VHostLevel& H, VLevelDev& D, bool has_children) {
    D.L.nl = H.nl;
    D.L.dof = vupload(h, H.dof.data(), H.dof.size());
    D.L.nb = vupload(h, H.nb.data(), H.nb.size());
    D.dof_base = vupload(h, H.dof_base.data(), H.dof_base.size());
    D.org = vupload(h, H.org.data(), H.org.size());
    if (has_children) D.L.child = vupload(h, H.child.data(), H.child.size());
    D.L.trim = nullptr;
    const size_t vb = (size_t)3 * H.nl * UAAMG_LEAF * sizeof(float);
    D.lhs = (float*)valloc(h, vb);
    D.rhs = (float*)valloc(h, vb);
    CK(cudaMemsetAsync(D.lhs, 0, vb, h->stream));
    if (H.nl <= h->rb_fused_max_leaves) {
        D.alt = (float*)valloc(h, vb);
        CK(cudaMemsetAsync(D.alt, 0, vb, h->stream));
    }
    CK(cudaMemsetAsync(D.rhs, 0, vb, h->stream));  // restriction leaves voxels without fine leaves untouched
    D.L.coef = (float*)valloc(h, (size_t)27 * H.nl * UAAMG_LEAF * sizeof(float));
    D.L.zpage = h->zpage;
}
// [27][512] pages holding each array's applier default (read for missing and
// trimmed leaves)
static void upload_defpage(uaamg_viscosity* h, VLevelDev& D) {
    std::vector<float> page((size_t)27 * UAAMG_LEAF);
    for (int ca = 0; ca < 27; ++ca)
        for (int k = 0; k < UAAMG_LEAF; ++k) page[(size_t)ca * UAAMG_LEAF + k] = D.L.app[ca];
    D.L.defpage = vupload(h, page.data(), page.size());
}
static void upload_parents(uaamg_viscosity* h, const VHostLevel& H, VLevelDev& D) {
    D.L.parent = vupload(h, H.parent.data(), H.parent.size());
    D.L.octant = vupload(h, H.octant.data(), H.octant.size());
}

static void build_viscosity(uaamg_viscosity* h, const uaamg_leaf_grid* mu_g, const uaamg_leaf_grid* liq,
                            const uaamg_leaf_grid* sol, float dt, float rho, float dx) {
    double trace_t0 = trace_now();
    check_grid(mu_g, 1, "viscosity");
    check_grid(liq, 1, "liquid_sdf");
    check_grid(sol, 1, "solid_sdf");
    require(dx > 0.f && rho > 0.f, "dx and rho must be positive");
    h->dt = dt;
    h->rho = rho;
    h->dx = dx;
    h->factor = dt / (rho * dx * dx);
    h->def_off = h->factor * mu_g->background[0];
    h->def_diag = 1.0f + 8.0f * h->def_off;
    cudaStream_t s = h->stream;

    // leaf sets of the three dilations of the liquid topology; the subcell kernel, which needs only the first,
    // runs while the host builds the other two
    std::vector<int32_t> a1, a2, a1f;
    dilate_leaves(liq->origins, liq->leaf_count, liq->masks, 1, false, a1, false);
    const int n1 = (int)(a1.size() / 3);
    HostMap m1;
    m1.build(n1, a1.data());
    DGrid dliq = vupload_grid(h, liq);
    DMap d1 = vupload_map(h, m1);
    int* a1org = vupload(h, a1.data(), a1.size());
    const float sub_bg = 1.5f * dx;
    float* svol = (float*)valloc(h, (size_t)8 * n1 * UAAMG_LEAF * 4);
    if (n1) {
        k_vsub<<<(unsigned)(8 * n1), 128, 0, s>>>(dliq, d1, a1org, sub_bg, svol);
        CHECK_LAUNCH();
    }
    dilate_leaves(liq->origins, liq->leaf_count, liq->masks, 2, false, a2, false);
    dilate_leaves(liq->origins, liq->leaf_count, liq->masks, 1, true, a1f, false);
    const int n2 = (int)(a2.size() / 3), n1f = (int)(a1f.size() / 3);
    HostMap m2, m1f;
    m2.build(n2, a2.data());
    m1f.build(n1f, a1f.data());
    TRACE("visc host leaf sets");

    DGrid dsol = vupload_grid(h, sol);
    h->mu = vupload_grid(h, mu_g);
    DMap d2 = vupload_map(h, m2), d1f = vupload_map(h, m1f);
    int* a2org = vupload(h, a2.data(), a2.size());
    int* a1forg = vupload(h, a1f.data(), a1f.size());
    float* vol7 = (float*)valloc(h, (size_t)7 * n2 * UAAMG_LEAF * 4);
    uint32_t* dofw = (uint32_t*)valloc(h, (size_t)3 * n1f * 64);
    uint32_t* solw = (uint32_t*)valloc(h, (size_t)3 * n1f * 64);
    if (n2) {
        k_vvol<<<(unsigned)n2, 128, 0, s>>>(d1, a2org, n2, svol, vol7);
        CHECK_LAUNCH();
    }
    vfree_now(h, svol);
    h->V.voxel = DField{d2, vol7};
    for (int c = 0; c < 3; ++c) {
        h->V.face[c] = DField{d2, vol7 + (size_t)(1 + c) * n2 * UAAMG_LEAF};
        h->V.edge[c] = DField{d2, vol7 + (size_t)(4 + c) * n2 * UAAMG_LEAF};
    }
    if (n1f) {
        k_vdof<<<(unsigned)n1f, 128, 0, s>>>(dsol, h->V, a1forg, n1f, dofw, solw);
        CHECK_LAUNCH();
    }
    h->S = SolidInfo{d1f, solw, n1f};
    std::vector<uint64_t> dofh((size_t)3 * n1f * 8);
    if (n1f) CK(cudaMemcpyAsync(dofh.data(), dofw, dofh.size() * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    TRACE("visc volumes + dof marking");

    h->zpage = (float*)valloc(h, UAAMG_LEAF * sizeof(float));
    CK(cudaMemsetAsync(h->zpage, 0, UAAMG_LEAF * sizeof(float), s));
    // level 0: DOF leaves (pruned) and the pattern dilated by 2
    std::vector<int32_t> dl;
    std::vector<int> keep;
    for (int i = 0; i < n1f; ++i) {
        uint64_t any = 0;
        for (int c = 0; c < 3; ++c)
            for (int w = 0; w < 8; ++w) any |= dofh[((size_t)c * n1f + i) * 8 + w];
        if (!any) continue;
        keep.push_back(i);
        dl.insert(dl.end(), &a1f[3 * i], &a1f[3 * i] + 3);
    }
    const int nd = (int)keep.size();
    std::vector<uint64_t> dm((size_t)3 * nd * 8);
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < nd; ++k)
            memcpy(&dm[((size_t)c * nd + k) * 8], &dofh[((size_t)c * n1f + keep[k]) * 8], 64);
    h->host.reserve(32);
    h->host.emplace_back();
    make_pattern_level(dl, dm, 2, h->host[0]);
    h->lv.reserve(32);
    h->lv.emplace_back();
    TRACE("visc level-0 topology");
    {
        VHostLevel& H = h->host[0];
        VLevelDev& D = h->lv[0];
        upload_vlevel(h, H, D, false);
        for (int c = 0; c < 3; ++c) {
            float* a = D.L.app + c * VNA;
            a[VA_DIAG] = h->def_diag;
            a[VA_INV] = 1.0f / h->def_diag;
            for (int ax = 0; ax < 3; ++ax) a[VA_NEGX + ax] = (ax == c) ? -2.0f * h->def_off : -h->def_off;
            a[VA_T00] = h->def_off;
            a[VA_T01] = -h->def_off;
            a[VA_T10] = -h->def_off;
            a[VA_T11] = h->def_off;
        }
        h->org0 = D.org;
        upload_defpage(h, D);
        launch2(k_vcoef0, dim3((unsigned)H.nl, 3), 128, s, D.L, (const int*)D.org, h->V, h->mu, h->factor, h->def_diag,
                (float*)D.L.coef);
    }
    TRACE("visc level-0 coefficients");
    // coarse levels while ndof > 4000 (simd_viscosity3d ctor, :3639-3645)
    while (h->host.back().ndof > 4000 && h->host.size() < 30) {
        const int fl = (int)h->host.size() - 1;
        h->host.emplace_back();
        coarsen_vlevel(h->host[fl], h->host[fl + 1]);
        h->lv.emplace_back();
        VLevelDev& D = h->lv[fl + 1];
        upload_vlevel(h, h->host[fl + 1], D, true);
        upload_parents(h, h->host[fl], h->lv[fl]);
        for (int c = 0; c < 3; ++c) {
            float* a = D.L.app + c * VNA;  // m_default_diag = m_default_off_diag = 1 (:66-68)
            a[VA_DIAG] = 1.f;
            a[VA_INV] = 1.f;
            for (int ax = 0; ax < 3; ++ax) a[VA_NEGX + ax] = (ax == c) ? -2.f : -1.f;
            a[VA_T00] = 1.f;
            a[VA_T01] = -1.f;
            a[VA_T10] = -1.f;
            a[VA_T11] = 1.f;
        }
        upload_defpage(h, D);
        launch2(k_vcoarse_coef, dim3((unsigned)h->host[fl + 1].nl, 3, 4), 128, s, h->lv[fl].L, D.L, (float*)D.L.coef);
    }
    h->nlev = (int)h->host.size();
    {
        VLevelDev& D = h->lv[h->nlev - 1];
        D.L.parent = nullptr;
        D.L.octant = nullptr;
    }
    TRACE("visc coarse levels");
    // trim level 0 after the coarse levels (:3649)
    {
        VLevelDev& D = h->lv[0];
        uint32_t* trim = (uint32_t*)valloc(h, (size_t)(D.L.nl ? D.L.nl : 1) * 4);
        if (D.L.nl) {
            launch2(k_vtrim, dim3((unsigned)D.L.nl), 128, s, D.L, trim);
            launch2(k_vtrim_fill, dim3((unsigned)D.L.nl), 128, s, D.L, (const uint32_t*)trim, (float*)D.L.coef);
            int* cnb = (int*)valloc(h, (size_t)D.L.nl * 27 * sizeof(int));
            launch2(k_vcnb, dim3((unsigned)(((long long)D.L.nl * 27 + 127) / 128)), 128, s, D.L,
                    (const uint32_t*)trim, cnb);
            D.L.cnb = cnb;
        }
        D.L.trim = trim;
    }
    // coarsest explicit matrix (construct_exact_solver, :3650)
    {
        VHostLevel& H = h->host[h->nlev - 1];
        VLevelDev& D = h->lv[h->nlev - 1];
        const int n = (int)H.ndof;
        h->C.n = n;
        if (n > 16 * VCG_THREADS) {
            set_error("coarsest level has %d DOFs (more than %d)", n, 16 * VCG_THREADS);
            throw UaamgError{UAAMG_ERR_DOMAIN_TOO_LARGE};
        }
        int* col = (int*)valloc(h, (size_t)(n ? n : 1) * VCG_W * 4);
        float* val = (float*)valloc(h, (size_t)(n ? n : 1) * VCG_W * 4);
        float* invd = (float*)valloc(h, (size_t)(n ? n : 1) * 4);
        long long* slot = (long long*)valloc(h, (size_t)(n ? n : 1) * 8);
        if (n) launch2(k_vcoarsest_ell, dim3((unsigned)H.nl, 3, 4), 128, s, D.L, (const int*)D.dof_base, col, val, invd, slot);
        h->C.col = col;
        h->C.val = val;
        h->C.invd = invd;
        h->C.slot = slot;
    }
    // PCG vectors and scalars
    {
        const size_t vb = (size_t)3 * h->host[0].nl * UAAMG_LEAF * 4;
        float** vecs[6] = {&h->x, &h->b, &h->r, &h->z, &h->p, &h->q};
        for (float** v : vecs) {
            *v = (float*)valloc(h, vb);
            CK(cudaMemsetAsync(*v, 0, vb, s));
        }
        size_t maxb = 1;
        for (auto& H : h->host) maxb = std::max(maxb, (size_t)3 * H.nl);
        h->partials = (double*)valloc(h, maxb * sizeof(double));
        h->st = (PcgState*)valloc(h, sizeof(PcgState) + 64);
        CK(cudaMemsetAsync(h->st, 0, sizeof(PcgState), s));
        h->scalar_dev = (float*)((char*)h->st + ((sizeof(PcgState) + 15) & ~size_t(15)));
    }
    CK(cudaStreamSynchronize(s));
    TRACE("visc trim + coarsest + vectors");
}

// ---------------------------------------------------------------------------
struct VEnq {
    uaamg_viscosity* h;
    cudaStream_t s;
    int64_t count = 0;
    std::vector<ProfRec>* prof = nullptr;
    void pb(const std::string& label) {
        if (!prof) return;
        ProfRec r;
        r.label = label;
        CK(cudaEventCreate(&r.a));
        CK(cudaEventCreate(&r.b));
        CK(cudaEventRecord(r.a, s));
        prof->push_back(r);
    }
    void pe() {
        if (!prof) return;
        CK(cudaEventRecord(prof->back().b, s));
    }
    template <int MODE>
    void apply(int l, int c, const float* x, const float* b, float* out) {
        const VLevelDev& D = h->lv[l];
        const bool gs = (MODE == VM_RED || MODE == VM_BLACK);
        static const char* names[] = {"normal", "residual", "jacobi", "red_gs", "black_gs"};
        if (prof) pb("L" + std::to_string(l) + " " + names[MODE] + (gs ? " c" + std::to_string(c) : std::string()));
        if constexpr (MODE == VM_RED || MODE == VM_BLACK) {
            if (D.L.nl >= h->seq_min_leaves) {
                const dim3 g((unsigned)std::min(D.L.nl, VAPPLY_MINB * g_sms));
                if (c == 0) launch2(k_vapply_seq<MODE, 0>, g, 128, s, D.L, x, b, out, 1.0f);
                else if (c == 1) launch2(k_vapply_seq<MODE, 1>, g, 128, s, D.L, x, b, out, 1.0f);
                else launch2(k_vapply_seq<MODE, 2>, g, 128, s, D.L, x, b, out, 1.0f);
            } else {
                const dim3 g((unsigned)D.L.nl);
                if (c == 0) launch2(k_vapply<MODE, 0>, g, 128, s, D.L, x, b, out, 1.0f);
                else if (c == 1) launch2(k_vapply<MODE, 1>, g, 128, s, D.L, x, b, out, 1.0f);
                else launch2(k_vapply<MODE, 2>, g, 128, s, D.L, x, b, out, 1.0f);
            }
        } else {
            launch2(k_vapply<MODE, -1>, dim3((unsigned)D.L.nl, 3u), 128, s, D.L, x, b, out, 1.0f);
        }
        pe();
        count++;
    }
    // Two red-black sweeps (XYZ or ZYX order) of level l on x in place.  A level
    // the fused step covers runs one k_vrbgs per channel and sweep, alternating
    // between x and the level's second buffer; each channel moves twice, so the
    // result is back in x.
    void rbgs2(int l, bool xyz, float* x, const float* b) {
        const VLevelDev& D = h->lv[l];
        if (!D.alt) {
            rbgs(l, xyz, x, b);
            rbgs(l, xyz, x, b);
            return;
        }
        const size_t cs = (size_t)D.L.nl * UAAMG_LEAF;
        float* buf[2] = {x, D.alt};
        int where[3] = {0, 0, 0};
        for (int i = 0; i < 2; ++i)
            for (int s3 = 0; s3 < 3; ++s3) {
                const int c = xyz ? s3 : 2 - s3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                VRbIo io;
                io.xc = buf[where[c]] + c * cs;
                io.x1 = buf[where[c1]] + c1 * cs;
                io.x2 = buf[where[c2]] + c2 * cs;
                io.b = b + c * cs;
                io.out = buf[where[c] ^ 1] + c * cs;
                if (prof) pb("L" + std::to_string(l) + " rbgs step c" + std::to_string(c));
                const dim3 g((unsigned)D.L.nl);
                if (xyz) {
                    if (c == 0) launch2(k_vrbgs<0, 0>, g, VRB_THREADS, s, D.L, io, 1.0f);
                    else if (c == 1) launch2(k_vrbgs<1, 0>, g, VRB_THREADS, s, D.L, io, 1.0f);
                    else launch2(k_vrbgs<2, 0>, g, VRB_THREADS, s, D.L, io, 1.0f);
                } else {
                    if (c == 0) launch2(k_vrbgs<0, 1>, g, VRB_THREADS, s, D.L, io, 1.0f);
                    else if (c == 1) launch2(k_vrbgs<1, 1>, g, VRB_THREADS, s, D.L, io, 1.0f);
                    else launch2(k_vrbgs<2, 1>, g, VRB_THREADS, s, D.L, io, 1.0f);
                }
                pe();
                count++;
                where[c] ^= 1;
            }
    }
    void rbgs(int l, bool xyz, float* x, const float* b) {
        if (xyz) {
            for (int c = 0; c < 3; ++c) {
                apply<VM_RED>(l, c, x, b, x);
                apply<VM_BLACK>(l, c, x, b, x);
            }
        } else {
            for (int c = 2; c >= 0; --c) {
                apply<VM_BLACK>(l, c, x, b, x);
                apply<VM_RED>(l, c, x, b, x);
            }
        }
    }
    void restrict_(int l, const float* fine, float* coarse) {
        if (prof) pb("L" + std::to_string(l) + " restrict");
        launch2(k_vrestrict, dim3((unsigned)h->lv[l + 1].L.nl, 3), 128, s, h->lv[l].L, h->lv[l + 1].L, fine, coarse);
        pe();
        count++;
    }
    // residual of level l restricted into the rhs of level l + 1 (fused); coarse_lhs (optional) is zeroed
    void residual_restrict(int l, const float* x, const float* b, float* coarse, float* coarse_lhs) {
        if (prof) pb("L" + std::to_string(l) + " residual+restrict");
        launch2(k_vresrestrict, dim3((unsigned)h->lv[l].L.nl, 3), 128, s, h->lv[l].L, h->lv[l + 1].L, x, b, coarse,
                coarse_lhs);
        pe();
        count++;
    }
    void prolong(int l, const float* coarse, float* fine) {
        if (prof) pb("L" + std::to_string(l) + " prolong");
        launch2(k_vprolong, dim3((unsigned)h->lv[l].L.nl, 3), 128, s, h->lv[l].L, h->lv[l + 1].L, coarse, fine);
        pe();
        count++;
    }
    void coarsest(const float* rhs, float* out) {
        if (h->C.n == 0) return;
        if (prof) pb("coarsest cg");
        const int n = h->C.n;
        if (n <= 2 * VCG_THREADS) launch2(k_vcoarsest_cg<2>, dim3(1), VCG_THREADS, s, h->C, rhs, out);
        else if (n <= 4 * VCG_THREADS) launch2(k_vcoarsest_cg<4>, dim3(1), VCG_THREADS, s, h->C, rhs, out);
        else if (n <= 8 * VCG_THREADS) launch2(k_vcoarsest_cg<8>, dim3(1), VCG_THREADS, s, h->C, rhs, out);
        else launch2(k_vcoarsest_cg<16>, dim3(1), VCG_THREADS, s, h->C, rhs, out);
        pe();
        count++;
    }
    void zero(int l, float* v) {
        const long long n4 = (long long)3 * h->lv[l].L.nl * (UAAMG_LEAF / 4);
        if (n4 == 0) return;
        const long long g = std::min<long long>((n4 + 255) / 256, (long long)g_sms * 8);
        launch2(k_vzero, dim3((unsigned)g), 256, s, reinterpret_cast<float4*>(v), n4);
        count++;
    }
};

// simd_viscosity3d::mucycle (:3837-3884) with mu = 2, n = 2.  The second
// visit of the coarsest level solves the same rhs from the same zero guess as
// the first, so it is not repeated.
// lhs_zeroed: the restriction before this visit already zeroed lhs.
static void enqueue_mucycle(VEnq& E, int l, float* lhs, const float* rhs, bool for_precon, bool lhs_zeroed = false) {
    uaamg_viscosity* h = E.h;
    if (l == h->nlev - 1) {
        E.coarsest(rhs, lhs);
        return;
    }
    if (for_precon && !lhs_zeroed) E.zero(l, lhs);
    E.rbgs2(l, true, lhs, rhs);
    VLevelDev& D = h->lv[l];
    VLevelDev& P = h->lv[l + 1];
    const bool coarse_visit = l + 1 != h->nlev - 1;  // the coarsest solve writes its own result
    E.residual_restrict(l, lhs, rhs, P.rhs, coarse_visit ? P.lhs : nullptr);
    enqueue_mucycle(E, l + 1, P.lhs, P.rhs, true, coarse_visit);
    if (l + 1 != h->nlev - 1) enqueue_mucycle(E, l + 1, P.lhs, P.rhs, false);
    E.prolong(l, P.lhs, lhs);
    E.rbgs2(l, false, lhs, rhs);
}

// grid of the level-0 vector streams: 16 CTAs of 128 threads per SM at most
static dim3 vstream_grid(int nl) {
    const long long n4 = 3LL * nl * UAAMG_LEAF4;
    return dim3((unsigned)std::max(1LL, std::min((n4 + 127) / 128, 16LL * g_sms)));
}

static void venqueue_setup(VEnq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_viscosity* h = E.h;
    const VLevelDev& D = h->lv[0];
    const dim3 g((unsigned)D.L.nl, 3);
    E.zero(0, h->p);
    launch2(k_vmask, g, 128, E.s, D.L, h->x);
    launch2(k_vmask, g, 128, E.s, D.L, h->b);
    if (E.prof) E.pb("L0 pcg init (residual+absmax)");
    launch2(k_vpcg_init, g, 128, E.s, D.L, (const float*)h->x, (const float*)h->b, h->r, h->partials, h->st, cond,
            use_cond);
    E.pe();
    E.count += 3;
}
static void venqueue_body(VEnq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_viscosity* h = E.h;
    const VLevelDev& D = h->lv[0];
    const dim3 g((unsigned)D.L.nl, 3);
    enqueue_mucycle(E, 0, h->z, h->r, true);
    const dim3 gd((unsigned)((3 * D.L.nl + VDOT_ITEMS - 1) / VDOT_ITEMS));
    float* part = reinterpret_cast<float*>(h->partials);
    if (E.prof) E.pb("L0 pcg rho (z.r)");
    launch2(k_vdot, gd, VDOT_THREADS, E.s, D.L, (const float*)h->z, (const float*)h->r, part, h->st, 0);
    E.pe();
    if (E.prof) E.pb("L0 pcg x,p update");
    launch2(k_vpcg_update_p, vstream_grid(D.L.nl), 128, E.s, D.L, (const float*)h->z, h->p, h->x,
            (const PcgState*)h->st);
    E.pe();
    if (E.prof) E.pb("L0 pcg Ap");
    launch2(k_vpcg_Ap, g, 128, E.s, D.L, (const float*)h->p, h->q);
    E.pe();
    if (E.prof) E.pb("L0 pcg sigma (p.q)");
    launch2(k_vdot, gd, VDOT_THREADS, E.s, D.L, (const float*)h->p, (const float*)h->q, part, h->st, 1);
    E.pe();
    if (E.prof) E.pb("L0 pcg r update+absmax");
    launch2(k_vpcg_update_r, vstream_grid(D.L.nl), 128, E.s, D.L, (const float*)h->q, h->r, h->partials, h->st,
            cond, use_cond);
    E.pe();
    E.count += 5;
}
static void venqueue_finish(VEnq& E) {
    uaamg_viscosity* h = E.h;
    const VLevelDev& D = h->lv[0];
    if (E.prof) E.pb("L0 pcg finish");
    launch2(k_vpcg_finish, dim3((unsigned)D.L.nl, 3), 128, E.s, D.L, (const float*)h->p, h->x, (const PcgState*)h->st);
    E.pe();
    E.count += 1;
}

static void vdestroy_graph(uaamg_viscosity* h) {
    if (h->shared_graph) {
        h->shared_graph.reset();
    } else {
        if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
        if (h->graph) cudaGraphDestroy(h->graph);
    }
    h->graph_exec = nullptr;
    h->graph = nullptr;
}

// The recording of one PCG solve's enqueue (setup, body, finish) as the
// graph captures it (the solve-graph cache of poisson.cu).
static std::vector<unsigned char> vrecord_solve(uaamg_viscosity* h) {
    LaunchRec rec;
    rec.val((unsigned char)'V');
    rec.val(g_use_pdl);
    rec.val(h->ctx->device);
    t_rec = &rec;
    try {
        VEnq E{h, h->stream};
        venqueue_setup(E, 0, 1);
        rec.val((unsigned char)'|');
        VEnq B{h, h->body_stream};
        venqueue_body(B, 0, 1);
        rec.val((unsigned char)'|');
        VEnq F{h, h->stream};
        venqueue_finish(F);
    } catch (...) {
        t_rec = nullptr;
        throw;
    }
    t_rec = nullptr;
    return std::move(rec.bytes);
}

static void vbuild_graph(uaamg_viscosity* h) {
    vdestroy_graph(h);
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    VEnq E{h, h->stream};
    CK(cudaStreamBeginCaptureToGraph(h->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        venqueue_setup(E, cond, 1);
        h->setup_launches = E.count;
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraph_t cg = nullptr;
        CK(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cg, &deps, &ndeps));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t wnode;
        CK(cudaGraphAddNode(&wnode, cg, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(h->stream, &wnode, 1, cudaStreamSetCaptureDependencies));
        VEnq B{h, h->body_stream};
        CK(cudaStreamBeginCaptureToGraph(h->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        venqueue_body(B, cond, 1);
        cudaGraph_t bodyout = nullptr;
        CK(cudaStreamEndCapture(h->body_stream, &bodyout));
        h->body_launches = B.count;
        VEnq F{h, h->stream};
        venqueue_finish(F);
        h->finish_launches = F.count;
    } catch (...) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(h->stream, &dummy);
        cudaStreamEndCapture(h->body_stream, &dummy);
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(h->stream, &out));
    CK(cudaGraphInstantiate(&h->graph_exec, g, 0));
    h->graph = g;
}

static void vinit_state(uaamg_viscosity* h) {
    PcgState s;
    memset(&s, 0, sizeof(s));
    s.tol = h->tol;
    s.max_iter = h->max_iter;
    *h->st_host = s;
    CK(cudaMemcpyAsync(h->st, h->st_host, sizeof(PcgState), cudaMemcpyHostToDevice, h->stream));
}

// x, b (h->x, h->b) on the device; returns UAAMG_SUCCESS when the stopping
// test held, UAAMG_FAILED when the loop returned at max_iter - 1
static int vrun_pcg(uaamg_viscosity* h, std::vector<ProfRec>* prof = nullptr) {
    if (h->lv[0].L.nl == 0 || h->host[0].ndof == 0) {
        h->iterations = 0;
        h->final_residual = 0.f;
        h->status = UAAMG_SUCCESS;
        return UAAMG_SUCCESS;
    }
    vinit_state(h);
    int64_t launches = 0;
    bool use_graph = !prof && h->use_graph && (h->use_graph == 2 || h->solves > 0);
    std::shared_ptr<SolveGraph> hit;
    std::vector<unsigned char> sig;
    bool share = false;
    if (!prof && !use_graph && h->use_graph == 1 && g_solve_graph_cache) {  // the cache may take this first solve
        sig = vrecord_solve(h);
        share = solve_graph_lookup(sig, hit);
        use_graph = hit || share;
    }
    h->solves++;
    if (use_graph) {
        if (hit) {
            vdestroy_graph(h);
            h->shared_graph = hit;
            h->graph = hit->g;
            h->graph_exec = hit->x;
            h->setup_launches = hit->setup;
            h->body_launches = hit->body;
            h->finish_launches = hit->finish;
        } else if (!h->graph_exec) {
            vbuild_graph(h);
            if (share)
                h->shared_graph = solve_graph_insert(std::move(sig), h->graph, h->graph_exec, h->setup_launches,
                                                     h->body_launches, h->finish_launches);
        }
        CK(cudaGraphLaunch(h->graph_exec, h->stream));
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        launches = h->setup_launches + (int64_t)h->st_host->iter * h->body_launches + h->finish_launches;
    } else {
        VEnq E{h, h->stream};
        E.prof = prof;
        venqueue_setup(E, 0, 0);
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        while (h->st_host->status == PCG_RUNNING) {
            venqueue_body(E, 0, 0);
            CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        venqueue_finish(E);
        CK(cudaStreamSynchronize(h->stream));
        launches = E.count;
    }
    h->last_launches = launches;
    h->launches += launches;
    const PcgState& s = *h->st_host;
    if (s.error) {
        set_error("a kernel's bounded wait for its bulk copies timed out");
        throw UaamgError{UAAMG_ERR_CUDA};
    }
    h->iterations = s.iterations_taken;
    h->final_residual = s.nu;
    h->status = (s.status == PCG_SUCCESS) ? UAAMG_SUCCESS : UAAMG_FAILED;
    return h->status;
}

static size_t vvec_bytes(const uaamg_viscosity* h, int level) {
    return (size_t)3 * h->lv[level].L.nl * UAAMG_LEAF * sizeof(float);
}
static void vcheck_level(const uaamg_viscosity* h, int level) {
    require(h != nullptr, "handle is NULL");
    require(level >= 0 && level < h->nlev, "level out of range");
}

static void vgrids3(const uaamg_leaf_grid* u, const uaamg_leaf_grid* v, const uaamg_leaf_grid* w) {
    check_grid(u, 1, "u");
    check_grid(v, 1, "v");
    check_grid(w, 1, "w");
}

static void vbuild_rhs_dev(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                           const uaamg_leaf_grid* w, const uaamg_leaf_grid* sv, float* d_out) {
    vgrids3(u, v, w);
    const size_t mark = h->allocs.size();
    VelGrids U;
    U.v[0] = vupload_grid(h, u);
    U.v[1] = vupload_grid(h, v);
    U.v[2] = vupload_grid(h, w);
    const VLevelDev& D = h->lv[0];
    CK(cudaMemsetAsync(d_out, 0, vvec_bytes(h, 0), h->stream));
    launch2(k_vrhs, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, h->V, U, d_out);
    bool moving = false;
    if (sv) {
        check_grid(sv, 3, "solid_velocity");
        moving = sv->leaf_count > 0 || sv->background[0] != 0.f || sv->background[1] != 0.f || sv->background[2] != 0.f;
    }
    if (moving) {
        DGrid dsv = vupload_grid(h, sv);
        launch2(k_vrhs_solid, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, h->V, h->mu, h->S, dsv,
                h->factor, d_out);
    }
    CK(cudaStreamSynchronize(h->stream));
    while (h->allocs.size() > mark) {
        CK(cudaFreeAsync(h->allocs.back(), h->stream));
        h->allocs.pop_back();
    }
}
static void vgather_dev(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                        const uaamg_leaf_grid* w, float* d_out) {
    vgrids3(u, v, w);
    const size_t mark = h->allocs.size();
    VelGrids U;
    U.v[0] = vupload_grid(h, u);
    U.v[1] = vupload_grid(h, v);
    U.v[2] = vupload_grid(h, w);
    const VLevelDev& D = h->lv[0];
    launch2(k_vgather, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, U, d_out);
    CK(cudaStreamSynchronize(h->stream));
    while (h->allocs.size() > mark) {
        CK(cudaFreeAsync(h->allocs.back(), h->stream));
        h->allocs.pop_back();
    }
}

struct VScratch {  // temporary device buffers of one host-pointer call
    uaamg_viscosity* h;
    std::vector<void*> bufs;
    float* get(size_t bytes) {
        void* p = nullptr;
        CK(ctx_dev_alloc(h->ctx, &p, bytes ? bytes : 256, h->stream));
        bufs.push_back(p);
        return (float*)p;
    }
    ~VScratch() {
        for (void* p : bufs) cudaFreeAsync(p, h->stream);
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
extern "C" {

int uaamg_viscosity_create(const uaamg_leaf_grid* viscosity, const uaamg_leaf_grid* liquid_sdf,
                           const uaamg_leaf_grid* solid_sdf, float dt, float rho, float dx, uaamg_viscosity** out) {
    return uaamg_viscosity_create_on_stream(viscosity, liquid_sdf, solid_sdf, dt, rho, dx, nullptr, out);
}

int uaamg_viscosity_create_on_stream(const uaamg_leaf_grid* viscosity, const uaamg_leaf_grid* liquid_sdf,
                                     const uaamg_leaf_grid* solid_sdf, float dt, float rho, float dx, void* stream,
                                     uaamg_viscosity** out) {
    {
        const char* e = getenv("UAAMG_PDL");
        g_use_pdl = !(e && e[0] == '0');
        e = getenv("UAAMG_SOLVE_GRAPH_CACHE");
        g_solve_graph_cache = !(e && e[0] == '0');
    }
    if (!out) { set_error("out is NULL"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return UAAMG_ERR_NO_DEVICE;
    }
    uaamg_viscosity* h = new (std::nothrow) uaamg_viscosity();
    if (!h) { set_error("host out of memory"); return UAAMG_ERR_OUT_OF_MEMORY; }
    try {
        cudaError_t ce = cudaSuccess;
        h->ctx = device_ctx(&ce);
        CK(ce);
        CK(ctx_stream_acquire(h->ctx, &h->own_stream));
        CK(ctx_stream_acquire(h->ctx, &h->body_stream));
        h->stream = stream ? (cudaStream_t)stream : h->own_stream;
        CK(ctx_pinned_acquire(h->ctx, sizeof(PcgState) + 256, &h->pin_state, &h->pin_state_cap));
        h->st_host = reinterpret_cast<PcgState*>(h->pin_state);
        h->scalar_host = reinterpret_cast<float*>((char*)h->pin_state + ((sizeof(PcgState) + 63) & ~size_t(63)));
        {
            int sms = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->ctx->device) == cudaSuccess && sms > 0)
                g_sms = sms;
        }
        h->rb_fused_max_leaves = 2 * g_sms;
        h->seq_min_leaves = 2 * g_sms + 1;
        if (const char* e = getenv("UAAMG_VISC_FUSED_RB_LEAVES")) h->rb_fused_max_leaves = atoi(e);
        if (const char* e = getenv("UAAMG_VISC_SEQ_LEAVES")) h->seq_min_leaves = atoi(e);
        build_viscosity(h, viscosity, liquid_sdf, solid_sdf, dt, rho, dx);
    } catch (const UaamgError& e) {
        uaamg_viscosity_destroy(h);
        return e.code;
    } catch (const std::bad_alloc&) {
        uaamg_viscosity_destroy(h);
        set_error("host out of memory");
        return UAAMG_ERR_OUT_OF_MEMORY;
    }
    *out = h;
    return UAAMG_SUCCESS;
}

int uaamg_viscosity_destroy(uaamg_viscosity* h) {
    if (!h) return UAAMG_SUCCESS;
    if (h->stream) cudaStreamSynchronize(h->stream);
    vdestroy_graph(h);
    if (h->ctx) {
        for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
        h->allocs.clear();
        if (h->stream) cudaStreamSynchronize(h->stream);
        ctx_pinned_release(h->ctx, h->pin_state, h->pin_state_cap);
        ctx_stream_release(h->ctx, h->body_stream);
        ctx_stream_release(h->ctx, h->own_stream);
    }
    delete h;
    return UAAMG_SUCCESS;
}

int uaamg_viscosity_set_max_iterations(uaamg_viscosity* h, int m) {
    ABI_BEGIN
    require(h != nullptr, "handle is NULL");
    h->max_iter = m;
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_iterations(const uaamg_viscosity* h) { return h ? h->iterations : 0; }
float uaamg_viscosity_final_residual(const uaamg_viscosity* h) { return h ? h->final_residual : 0.f; }
int uaamg_viscosity_num_levels(const uaamg_viscosity* h) { return h ? h->nlev : 0; }
int64_t uaamg_viscosity_num_dof(const uaamg_viscosity* h, int level) {
    if (!h || level < 0 || level >= h->nlev) return -1;
    return h->host[level].ndof;
}
int64_t uaamg_viscosity_leaf_count(const uaamg_viscosity* h, int level) {
    if (!h || level < 0 || level >= h->nlev) return -1;
    return h->host[level].nl;
}
int uaamg_viscosity_topology(const uaamg_viscosity* h, int level, int32_t* origins, uint64_t* dof_masks) {
    ABI_BEGIN
    vcheck_level(h, level);
    const VHostLevel& H = h->host[level];
    if (origins) memcpy(origins, H.org.data(), H.org.size() * 4);
    if (dof_masks) memcpy(dof_masks, H.dof.data(), H.dof.size() * 8);
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_dof_index(const uaamg_viscosity* h, int level, int32_t* out) {
    ABI_BEGIN
    vcheck_level(h, level);
    require(out != nullptr, "out is NULL");
    const VHostLevel& H = h->host[level];
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < H.nl; ++i) {
            int32_t d = H.dof_base[(size_t)c * H.nl + i];
            const uint64_t* m = &H.dof[((size_t)c * H.nl + i) * 8];
            int32_t* o = out + ((size_t)c * H.nl + i) * UAAMG_LEAF;
            for (int off = 0; off < UAAMG_LEAF; ++off) o[off] = ((m[off >> 6] >> (off & 63)) & 1ull) ? d++ : -1;
        }
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_viscosity_build_rhs(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                              const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity, float* rhs_out) {
    ABI_BEGIN
    require(h != nullptr && rhs_out != nullptr, "NULL argument");
    VScratch sc{h};
    float* d = sc.get(vvec_bytes(h, 0));
    vbuild_rhs_dev(h, u, v, w, solid_velocity, d);
    CK(cudaMemcpyAsync(rhs_out, d, vvec_bytes(h, 0), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_build_rhs_device(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                     const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity, float* d_rhs_out) {
    ABI_BEGIN
    require(h != nullptr && d_rhs_out != nullptr, "NULL argument");
    vbuild_rhs_dev(h, u, v, w, solid_velocity, d_rhs_out);
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_gather_velocity(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                    const uaamg_leaf_grid* w, float* out) {
    ABI_BEGIN
    require(h != nullptr && out != nullptr, "NULL argument");
    VScratch sc{h};
    float* d = sc.get(vvec_bytes(h, 0));
    vgather_dev(h, u, v, w, d);
    CK(cudaMemcpyAsync(out, d, vvec_bytes(h, 0), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_gather_velocity_device(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                           const uaamg_leaf_grid* w, float* d_out) {
    ABI_BEGIN
    require(h != nullptr && d_out != nullptr, "NULL argument");
    vgather_dev(h, u, v, w, d_out);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_viscosity_solve_pcg(uaamg_viscosity* h, float* velocity, const float* rhs, float tolerance, int* iterations) {
    ABI_BEGIN
    require(h != nullptr && velocity != nullptr && rhs != nullptr, "NULL argument");
    const size_t vb = vvec_bytes(h, 0);
    h->tol = tolerance;
    CK(cudaMemcpyAsync(h->x, velocity, vb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->b, rhs, vb, cudaMemcpyHostToDevice, h->stream));
    const int st = vrun_pcg(h);
    CK(cudaMemcpyAsync(velocity, h->x, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}
int uaamg_viscosity_solve_pcg_device(uaamg_viscosity* h, float* d_velocity, const float* d_rhs, float tolerance,
                                     int* iterations) {
    ABI_BEGIN
    require(h != nullptr && d_velocity != nullptr && d_rhs != nullptr, "NULL argument");
    const size_t vb = vvec_bytes(h, 0);
    h->tol = tolerance;
    CK(cudaMemcpyAsync(h->x, d_velocity, vb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->b, d_rhs, vb, cudaMemcpyDeviceToDevice, h->stream));
    const int st = vrun_pcg(h);
    CK(cudaMemcpyAsync(d_velocity, h->x, vb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}

int uaamg_viscosity_solve_velocity(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                   const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity, float tolerance,
                                   float* velocity_out, int* iterations) {
    ABI_BEGIN
    require(h != nullptr && velocity_out != nullptr, "NULL argument");
    vgrids3(u, v, w);
    bool moving = false;
    if (solid_velocity) {
        check_grid(solid_velocity, 3, "solid_velocity");
        moving = solid_velocity->leaf_count > 0 || solid_velocity->background[0] != 0.f ||
                 solid_velocity->background[1] != 0.f || solid_velocity->background[2] != 0.f;
    }
    const size_t mark = h->allocs.size();
    int st = UAAMG_FAILED;
    try {
        VelGrids U;
        U.v[0] = vupload_grid(h, u);
        U.v[1] = vupload_grid(h, v);
        U.v[2] = vupload_grid(h, w);
        const VLevelDev& D = h->lv[0];
        const size_t vb = vvec_bytes(h, 0);
        // the rhs (simd_viscosity3d ctor, .cpp:3660-3689) and the warm start (FLIP_vdb.cpp:3186-3198) straight
        // into the PCG vectors
        CK(cudaMemsetAsync(h->b, 0, vb, h->stream));
        launch2(k_vrhs, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, h->V, U, h->b);
        if (moving) {
            DGrid dsv = vupload_grid(h, solid_velocity);
            launch2(k_vrhs_solid, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, h->V, h->mu,
                    h->S, dsv, h->factor, h->b);
        }
        launch2(k_vgather, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, (const int*)D.org, U, h->x);
        h->tol = tolerance;
        st = vrun_pcg(h);
        CK(cudaMemcpyAsync(velocity_out, h->x, vb, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    } catch (...) {
        cudaStreamSynchronize(h->stream);
        while (h->allocs.size() > mark) {
            cudaFreeAsync(h->allocs.back(), h->stream);
            h->allocs.pop_back();
        }
        throw;
    }
    while (h->allocs.size() > mark) {
        CK(cudaFreeAsync(h->allocs.back(), h->stream));
        h->allocs.pop_back();
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}

// level operations (host pointers; parity tests)
int uaamg_viscosity_level_apply(uaamg_viscosity* h, int level, int mode, int channel, const float* lhs,
                                const float* rhs, float* out) {
    ABI_BEGIN
    vcheck_level(h, level);
    require(mode >= VM_NORMAL && mode <= VM_BLACK, "mode out of range");
    require(lhs && out && (mode == VM_NORMAL || rhs), "NULL argument");
    const bool gs = mode == VM_RED || mode == VM_BLACK;
    require(!gs || (channel >= 0 && channel < 3), "channel out of range");
    const size_t vb = vvec_bytes(h, level);
    VScratch sc{h};
    float* x = sc.get(vb);
    float* b = sc.get(vb);
    float* o = gs ? x : sc.get(vb);
    CK(cudaMemcpyAsync(x, lhs, vb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(b, rhs ? rhs : lhs, vb, cudaMemcpyHostToDevice, h->stream));
    if (!gs) CK(cudaMemsetAsync(o, 0, vb, h->stream));
    const VLevelDev& D = h->lv[level];
    launch2(k_vmask, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, x);
    VEnq E{h, h->stream};
    switch (mode) {
    case VM_NORMAL: E.apply<VM_NORMAL>(level, 0, x, b, o); break;
    case VM_RESIDUAL: E.apply<VM_RESIDUAL>(level, 0, x, b, o); break;
    case VM_JACOBI: E.apply<VM_JACOBI>(level, 0, x, b, o); break;
    case VM_RED: E.apply<VM_RED>(level, channel, x, b, o); break;
    default: E.apply<VM_BLACK>(level, channel, x, b, o); break;
    }
    CK(cudaMemcpyAsync(out, o, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_level_rbgs(uaamg_viscosity* h, int level, int order, float* lhs, const float* rhs) {
    ABI_BEGIN
    vcheck_level(h, level);
    require(lhs && rhs, "NULL argument");
    const size_t vb = vvec_bytes(h, level);
    VScratch sc{h};
    float* x = sc.get(vb);
    float* b = sc.get(vb);
    CK(cudaMemcpyAsync(x, lhs, vb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(b, rhs, vb, cudaMemcpyHostToDevice, h->stream));
    const VLevelDev& D = h->lv[level];
    launch2(k_vmask, dim3((unsigned)D.L.nl, 3), 128, h->stream, D.L, x);
    VEnq E{h, h->stream};
    E.rbgs(level, order == 0, x, b);
    CK(cudaMemcpyAsync(lhs, x, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_level_restrict(uaamg_viscosity* h, int fine_level, const float* fine, float* coarse) {
    ABI_BEGIN
    vcheck_level(h, fine_level);
    require(fine_level + 1 < h->nlev, "no coarser level");
    require(fine && coarse, "NULL argument");
    VScratch sc{h};
    float* f = sc.get(vvec_bytes(h, fine_level));
    float* c = sc.get(vvec_bytes(h, fine_level + 1));
    CK(cudaMemcpyAsync(f, fine, vvec_bytes(h, fine_level), cudaMemcpyHostToDevice, h->stream));
    launch2(k_vmask, dim3((unsigned)h->lv[fine_level].L.nl, 3), 128, h->stream, h->lv[fine_level].L, f);
    VEnq E{h, h->stream};
    E.restrict_(fine_level, f, c);
    CK(cudaMemcpyAsync(coarse, c, vvec_bytes(h, fine_level + 1), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_level_prolongate(uaamg_viscosity* h, int fine_level, const float* coarse, float* fine) {
    ABI_BEGIN
    vcheck_level(h, fine_level);
    require(fine_level + 1 < h->nlev, "no coarser level");
    require(fine && coarse, "NULL argument");
    VScratch sc{h};
    float* f = sc.get(vvec_bytes(h, fine_level));
    float* c = sc.get(vvec_bytes(h, fine_level + 1));
    CK(cudaMemcpyAsync(f, fine, vvec_bytes(h, fine_level), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(c, coarse, vvec_bytes(h, fine_level + 1), cudaMemcpyHostToDevice, h->stream));
    launch2(k_vmask, dim3((unsigned)h->lv[fine_level].L.nl, 3), 128, h->stream, h->lv[fine_level].L, f);
    launch2(k_vmask, dim3((unsigned)h->lv[fine_level + 1].L.nl, 3), 128, h->stream, h->lv[fine_level + 1].L, c);
    VEnq E{h, h->stream};
    E.prolong(fine_level, c, f);
    CK(cudaMemcpyAsync(fine, f, vvec_bytes(h, fine_level), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_level_coefficients(const uaamg_viscosity* h, int level, float* coef, uint32_t* trim) {
    ABI_BEGIN
    vcheck_level(h, level);
    const VLevelDev& D = h->lv[level];
    const size_t n = (size_t)27 * D.L.nl * UAAMG_LEAF;
    if (coef && n) CK(cudaMemcpyAsync(coef, D.L.coef, n * 4, cudaMemcpyDeviceToHost, h->stream));
    std::vector<uint32_t> tb((size_t)D.L.nl, 0);
    if (D.L.trim && D.L.nl) CK(cudaMemcpyAsync(tb.data(), D.L.trim, (size_t)D.L.nl * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (trim) memcpy(trim, tb.data(), tb.size() * 4);
    // effective values: a trimmed leaf reads its default
    if (coef)
        for (int i = 0; i < D.L.nl; ++i) {
            if (!tb[i]) continue;
            for (int ca = 0; ca < 27; ++ca) {
                if (!(tb[i] >> ca & 1u)) continue;
                float* v = coef + ((size_t)ca * D.L.nl + i) * UAAMG_LEAF;
                for (int k = 0; k < UAAMG_LEAF; ++k) v[k] = D.L.app[ca];
            }
        }
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_coarsest_solve(uaamg_viscosity* h, const float* rhs, float* out) {
    ABI_BEGIN
    require(h && rhs && out, "NULL argument");
    const int l = h->nlev - 1;
    const size_t vb = vvec_bytes(h, l);
    VScratch sc{h};
    float* b = sc.get(vb);
    float* x = sc.get(vb);
    CK(cudaMemcpyAsync(b, rhs, vb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(x, 0, vb, h->stream));
    VEnq E{h, h->stream};
    E.coarsest(b, x);
    CK(cudaMemcpyAsync(out, x, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_precondition(uaamg_viscosity* h, const float* r, float* z) {
    ABI_BEGIN
    require(h && r && z, "NULL argument");
    const size_t vb = vvec_bytes(h, 0);
    VScratch sc{h};
    float* rr = sc.get(vb);
    float* zz = sc.get(vb);
    CK(cudaMemcpyAsync(rr, r, vb, cudaMemcpyHostToDevice, h->stream));
    launch2(k_vmask, dim3((unsigned)h->lv[0].L.nl, 3), 128, h->stream, h->lv[0].L, rr);
    VEnq E{h, h->stream};
    enqueue_mucycle(E, 0, zz, rr, true);
    CK(cudaMemcpyAsync(z, zz, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_viscosity_profile_pcg(uaamg_viscosity* h, float* d_velocity, const float* d_rhs, float tolerance,
                                int max_classes, char* names, double* total_ms, int64_t* counts, int* nclasses) {
    ABI_BEGIN
    require(h && d_velocity && d_rhs && names && total_ms && counts && nclasses, "NULL argument");
    const size_t vb = vvec_bytes(h, 0);
    *nclasses = 0;
    h->tol = tolerance;
    CK(cudaMemcpyAsync(h->x, d_velocity, vb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->b, d_rhs, vb, cudaMemcpyDeviceToDevice, h->stream));
    std::vector<ProfRec> prof;
    const int st = vrun_pcg(h, &prof);
    CK(cudaMemcpyAsync(d_velocity, h->x, vb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<std::string> lab;
    for (auto& r : prof) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, r.a, r.b));
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
        int k = (int)(std::find(lab.begin(), lab.end(), r.label) - lab.begin());
        if (k == (int)lab.size()) {
            if (k >= max_classes) continue;
            lab.push_back(r.label);
            total_ms[k] = 0;
            counts[k] = 0;
            snprintf(names + 64 * k, 64, "%s", r.label.c_str());
        }
        total_ms[k] += ms;
        counts[k] += 1;
    }
    *nclasses = (int)lab.size();
    return st;
    ABI_END
}

int uaamg_viscosity_set_stream(uaamg_viscosity* h, void* stream) {
    ABI_BEGIN
    require(h != nullptr, "handle is NULL");
    CK(cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_viscosity_get_stream(const uaamg_viscosity* h, void** stream) {
    if (!h || !stream) { set_error("NULL argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *stream = (void*)h->stream;
    return UAAMG_SUCCESS;
}
int uaamg_viscosity_set_graph_mode(uaamg_viscosity* h, int use_graph) {
    ABI_BEGIN
    require(h != nullptr, "handle is NULL");
    require(use_graph >= 0 && use_graph <= 2, "graph mode must be 0, 1 or 2");
    h->use_graph = use_graph;
    return UAAMG_SUCCESS;
    ABI_END
}
int64_t uaamg_viscosity_kernel_launches(const uaamg_viscosity* h) { return h ? h->launches : 0; }

}  // extern "C"
