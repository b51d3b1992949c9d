// poisson.cu -- host side of the B200 UAAMG-PCG pressure solver and its C ABI.
//
// What runs where
//  * host (C++): leaf ordering, DOF-leaf compaction, neighbour / child tables
//    and the coarse-level masks (bit operations on 64-byte masks; O(leaves)),
//    then one upload of all tables.
//  * device: every numeric step -- level-0 coefficients, Galerkin coarsening,
//    trimming, SPAI0, the coarsest explicit matrix, right-hand side, and the
//    whole PCG: the W-cycle preconditioner and the CG vector steps keep all
//    scalars in device memory, and the iteration runs as a CUDA graph with a
//    conditional WHILE node, so a solve is a single graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <immintrin.h>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/uaamg.h"
#include "common.cuh"
#include "poisson_build.cuh"
#include "poisson_kernels.cuh"
#include "staged_pipe.cuh"
#include "poisson_bottom.cuh"
#include "resources.cuh"

using namespace uaamg;

// ---------------------------------------------------------------------------
// errors
static thread_local std::string g_last_error;
static void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}
struct UaamgError {
    int code;
};
#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            throw UaamgError{e_ == cudaErrorMemoryAllocation ? UAAMG_ERR_OUT_OF_MEMORY : UAAMG_ERR_CUDA}; \
        }                                                                                         \
    } while (0)
#define CHECK_LAUNCH() CK(cudaGetLastError())

// ---------------------------------------------------------------------------
// host-side topology helpers
namespace {

struct VdbKey {
    int32_t k[5];
};
// OpenVDB tree order of a leaf origin (5-4-3 tree): RootNode std::map keyed by
// the 4096^3 tile origin (compared x, y, z), then the child offsets of the two
// internal node levels.  Same leaf order as LeafManager, hence the same DOF
// numbering as setDofIndex.
static inline VdbKey vdb_key(const int32_t* o) {
    VdbKey r;
    r.k[0] = o[0] & ~4095;
    r.k[1] = o[1] & ~4095;
    r.k[2] = o[2] & ~4095;
    r.k[3] = (((o[0] & 4095) >> 7) << 10) | (((o[1] & 4095) >> 7) << 5) | ((o[2] & 4095) >> 7);
    r.k[4] = (((o[0] & 127) >> 3) << 8) | (((o[1] & 127) >> 3) << 4) | ((o[2] & 127) >> 3);
    return r;
}
static inline bool key_less(const VdbKey& a, const VdbKey& b) {
    for (int c = 0; c < 5; ++c) {
        if (a.k[c] != b.k[c]) return a.k[c] < b.k[c];
    }
    return false;
}

// vdb_key packed into one unsigned 128-bit number with the same order: the
// root tile origins (multiples of 4096) biased into 20 bits each, then the
// 15-bit and 12-bit child offsets of the two internal levels.
static inline unsigned __int128 vdb_key128(const int32_t* o) {
    const VdbKey k = vdb_key(o);
    const uint64_t rx = (uint64_t)((k.k[0] >> 12) + (1 << 19)), ry = (uint64_t)((k.k[1] >> 12) + (1 << 19)),
                   rz = (uint64_t)((k.k[2] >> 12) + (1 << 19));
    const uint64_t hi = (rx << 40) | (ry << 20) | rz;
    const uint64_t lo = ((uint64_t)k.k[3] << 12) | (uint64_t)k.k[4];
    return ((unsigned __int128)hi << 27) | lo;
}

// The coarse DOF bits one fine leaf contributes to its parent (a coarse voxel
// is a DOF if any of its 2x2x2 fine voxels is): fine word x holds the (y,z)
// plane (bit 8y + z); pairs of planes are OR-ed, then pairs in y and z, and the
// 4x4 bits at (2yy, 2zz) are compressed into nibbles and placed at the
// octant's (y, z) quarter of the coarse words ox*4 .. ox*4+3.
__attribute__((target("avx2"))) static void coarse_bits_from_child_avx2(const uint64_t* fm, int a, uint64_t* cw) {
    // the four plane pairs (2px, 2px+1) as the four lanes: the same integer steps as the scalar form
    const int ox = (a >> 2) & 1, oy = (a >> 1) & 1, oz = a & 1;
    __m256i p = _mm256_or_si256(_mm256_setr_epi64x((long long)fm[0], (long long)fm[2], (long long)fm[4], (long long)fm[6]),
                                _mm256_setr_epi64x((long long)fm[1], (long long)fm[3], (long long)fm[5], (long long)fm[7]));
    p = _mm256_or_si256(p, _mm256_srli_epi64(p, 1));
    p = _mm256_or_si256(p, _mm256_srli_epi64(p, 8));
    __m256i q = _mm256_and_si256(p, _mm256_set1_epi64x(0x0055005500550055ll));
    q = _mm256_and_si256(_mm256_or_si256(q, _mm256_srli_epi64(q, 1)), _mm256_set1_epi64x(0x0033003300330033ll));
    q = _mm256_and_si256(_mm256_or_si256(q, _mm256_srli_epi64(q, 2)), _mm256_set1_epi64x(0x000F000F000F000Fll));
    const __m256i nib = _mm256_set1_epi64x(0xF);
    __m256i dep = _mm256_and_si256(q, nib);
    dep = _mm256_or_si256(dep, _mm256_slli_epi64(_mm256_and_si256(_mm256_srli_epi64(q, 16), nib), 8));
    dep = _mm256_or_si256(dep, _mm256_slli_epi64(_mm256_and_si256(_mm256_srli_epi64(q, 32), nib), 16));
    dep = _mm256_or_si256(dep, _mm256_slli_epi64(_mm256_and_si256(_mm256_srli_epi64(q, 48), nib), 24));
    dep = _mm256_sll_epi64(dep, _mm_cvtsi32_si128(oy * 32 + oz * 4));
    __m256i* dst = reinterpret_cast<__m256i*>(cw + ox * 4);
    _mm256_storeu_si256(dst, _mm256_or_si256(_mm256_loadu_si256(dst), dep));
}
static inline void coarse_bits_from_child(const uint64_t* fm, int a, uint64_t* cw) {
    const int ox = (a >> 2) & 1, oy = (a >> 1) & 1, oz = a & 1;
    for (int px = 0; px < 4; ++px) {
        uint64_t p = fm[2 * px] | fm[2 * px + 1];
        p |= p >> 1;  // z pairs
        p |= p >> 8;  // y pairs
        uint64_t q = p & 0x0055005500550055ull;       // bits 16 yy + 2 zz
        q = (q | (q >> 1)) & 0x0033003300330033ull;
        q = (q | (q >> 2)) & 0x000F000F000F000Full;   // nibble yy (bit zz) at bit 16 yy
        const uint64_t dep = (q & 0xFull) | (((q >> 16) & 0xFull) << 8) | (((q >> 32) & 0xFull) << 16) |
                             (((q >> 48) & 0xFull) << 24);
        cw[ox * 4 + px] |= dep << (oy * 32 + oz * 4);
    }
}

// population count of a 64-bit mask on the host (SWAR bit count; inline, no
// library call on CPUs compiled without a popcount instruction)
static inline int host_popc64(uint64_t x);
// base[i] = acc + the set bits of the 8-word masks before leaf i; returns the
// total.  The CPU's popcount instruction where it has one (a DOF-numbering
// pass over a level's masks is on the host side of every construction).
__attribute__((target("popcnt"))) static int64_t popc_prefix_hw(const uint64_t* m, size_t nleaves, int32_t* base,
                                                                 int64_t acc) {
    for (size_t i = 0; i < nleaves; ++i) {
        base[i] = (int32_t)acc;
        for (int w = 0; w < 8; ++w) acc += __builtin_popcountll(m[8 * i + w]);
    }
    return acc;
}
static int64_t popc_prefix_sw(const uint64_t* m, size_t nleaves, int32_t* base, int64_t acc) {
    for (size_t i = 0; i < nleaves; ++i) {
        base[i] = (int32_t)acc;
        for (int w = 0; w < 8; ++w) acc += host_popc64(m[8 * i + w]);
    }
    return acc;
}
static int64_t popc_prefix(const uint64_t* m, size_t nleaves, int32_t* base, int64_t acc) {
    static const bool hw = __builtin_cpu_supports("popcnt");
    return hw ? popc_prefix_hw(m, nleaves, base, acc) : popc_prefix_sw(m, nleaves, base, acc);
}
static inline int host_popc64(uint64_t x) {
    x = x - ((x >> 1) & 0x5555555555555555ull);
    x = (x & 0x3333333333333333ull) + ((x >> 2) & 0x3333333333333333ull);
    x = (x + (x >> 4)) & 0x0F0F0F0F0F0F0F0Full;
    return (int)((x * 0x0101010101010101ull) >> 56);
}

struct HostMap {  // dense leaf-index volume over the bounding box
    int lo[3] = {0, 0, 0}, dim[3] = {0, 0, 0};
    std::vector<int32_t> idx;
    void build(int64_t n, const int32_t* org, int pad = 0) {
        idx.clear();
        if (n <= 0) { dim[0] = dim[1] = dim[2] = 0; return; }
        int mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
        for (int64_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) {
                int v = org[3 * i + c] >> 3;
                mn[c] = std::min(mn[c], v);
                mx[c] = std::max(mx[c], v);
            }
        int64_t tot = 1;
        for (int c = 0; c < 3; ++c) {
            lo[c] = mn[c] - pad;
            dim[c] = mx[c] - mn[c] + 1 + 2 * pad;
            tot *= dim[c];
        }
        if (tot > (int64_t(1) << 31)) {
            set_error("leaf bounding box too large for the dense leaf map (%lld cells)", (long long)tot);
            throw UaamgError{UAAMG_ERR_DOMAIN_TOO_LARGE};
        }
        idx.assign((size_t)tot, -1);
        for (int64_t i = 0; i < n; ++i) idx[cell(org[3 * i] >> 3, org[3 * i + 1] >> 3, org[3 * i + 2] >> 3)] = (int32_t)i;
    }
    inline int64_t cell(int a, int b, int c) const {
        return ((int64_t)(a - lo[0]) * dim[1] + (b - lo[1])) * dim[2] + (c - lo[2]);
    }
    inline int32_t find_leaf(int lx, int ly, int lz) const {  // leaf coordinates (origin >> 3)
        if (idx.empty()) return -1;
        int a = lx - lo[0], b = ly - lo[1], c = lz - lo[2];
        if ((unsigned)a >= (unsigned)dim[0] || (unsigned)b >= (unsigned)dim[1] || (unsigned)c >= (unsigned)dim[2]) return -1;
        return idx[((int64_t)a * dim[1] + b) * dim[2] + c];
    }
};

struct HostLevel {
    int nl = 0;
    int64_t ndof = 0;
    std::vector<int32_t> org;     // [nl][3]
    std::vector<uint64_t> mask;   // [nl][8]
    std::vector<int32_t> nbr;     // [nl][6]
    std::vector<int32_t> child;   // [nl][8]
    std::vector<int32_t> parent;  // [nl]
    std::vector<uint8_t> octant;  // [nl]
    std::vector<int32_t> dof_base;
    HostMap map;
    float dt = 0, dx = 0;
};

static void finalize_host_level(HostLevel& L) {
    // a one-leaf margin puts every leaf's face-neighbour cells inside the map
    L.map.build(L.nl, L.org.data(), 1);
    L.nbr.assign((size_t)L.nl * 6, -1);
    if (L.nl > 0) {
        const int64_t s0 = (int64_t)L.map.dim[1] * L.map.dim[2], s1 = L.map.dim[2];
        const int64_t off[6] = {-s0, s0, -s1, s1, -1, 1};
        const int32_t* idx = L.map.idx.data();
        for (int i = 0; i < L.nl; ++i) {
            const int32_t* o = &L.org[3 * i];
            const int64_t base = L.map.cell(o[0] >> 3, o[1] >> 3, o[2] >> 3);
            for (int d = 0; d < 6; ++d) L.nbr[6 * i + d] = idx[base + off[d]];
        }
    }
    L.dof_base.resize(L.nl);
    L.ndof = popc_prefix(L.mask.data(), (size_t)L.nl, L.dof_base.data(), 0);
}

// coarse level topology from the fine level (TouchCoarseLeafReducer,
// SIMD_UAAMG_Ops.h:4-38, and the coarse DOF rule of initializeFromFineLevel,
// simd_vdb_poisson.cpp:283-311: a coarse voxel is a DOF if any of its 2x2x2
// fine voxels is).
static void coarsen_topology(HostLevel& F, HostLevel& C) {
    C.dt = F.dt;
    C.dx = 2.0f * F.dx;
    // the coarse leaf of fine leaf l (origin / 2, leaf-aligned) is at leaf
    // coordinate l >> 1; unique coarse leaves through a dense mark over their
    // bounding box, then only those sorted into tree order
    const int clo[3] = {F.map.lo[0] >> 1, F.map.lo[1] >> 1, F.map.lo[2] >> 1};
    const int cdim[3] = {((F.map.lo[0] + F.map.dim[0] - 1) >> 1) - clo[0] + 1,
                         ((F.map.lo[1] + F.map.dim[1] - 1) >> 1) - clo[1] + 1,
                         ((F.map.lo[2] + F.map.dim[2] - 1) >> 1) - clo[2] + 1};
    std::vector<uint8_t> seen((size_t)cdim[0] * cdim[1] * cdim[2], 0);
    std::vector<std::pair<unsigned __int128, int>> keys;
    std::vector<int32_t> corg;
    keys.reserve(F.nl / 4 + 8);
    corg.reserve((size_t)(F.nl / 4 + 8) * 3);
    for (int i = 0; i < F.nl; ++i) {
        const int l[3] = {F.org[3 * i] >> 4, F.org[3 * i + 1] >> 4, F.org[3 * i + 2] >> 4};
        const size_t cell = ((size_t)(l[0] - clo[0]) * cdim[1] + (l[1] - clo[1])) * cdim[2] + (l[2] - clo[2]);
        if (seen[cell]) continue;
        seen[cell] = 1;
        const int k = (int)keys.size();
        corg.push_back(l[0] * 8);
        corg.push_back(l[1] * 8);
        corg.push_back(l[2] * 8);
        keys.push_back({vdb_key128(&corg[3 * (size_t)k]), k});
    }
    if (!std::is_sorted(keys.begin(), keys.end())) std::sort(keys.begin(), keys.end());
    const int nu = (int)keys.size();
    std::vector<int32_t> uorg((size_t)nu * 3);
    for (int i = 0; i < nu; ++i) std::copy(&corg[3 * (size_t)keys[i].second], &corg[3 * (size_t)keys[i].second] + 3, &uorg[3 * (size_t)i]);
    std::vector<uint64_t> cmask((size_t)nu * 8, 0);
    std::vector<int32_t> child((size_t)nu * 8, -1);
    // the children of coarse leaf c are the fine leaves 2c + {0,1}^3: inside the fine map's one-leaf margin
    const int64_t fs0 = (int64_t)F.map.dim[1] * F.map.dim[2], fs1 = F.map.dim[2];
    const int64_t coff[8] = {0, 1, fs1, fs1 + 1, fs0, fs0 + 1, fs0 + fs1, fs0 + fs1 + 1};
    const int32_t* fidx = F.map.idx.data();
    static const bool avx2 = __builtin_cpu_supports("avx2");
    for (int i = 0; i < nu; ++i) {
        const int64_t c0 = F.map.cell(uorg[3 * i] >> 2, uorg[3 * i + 1] >> 2, uorg[3 * i + 2] >> 2);
        for (int a = 0; a < 8; ++a) {
            const int fl = fidx[c0 + coff[a]];
            child[8 * i + a] = fl;
            if (fl < 0) continue;
            if (avx2) coarse_bits_from_child_avx2(&F.mask[8 * (size_t)fl], a, &cmask[8 * (size_t)i]);
            else coarse_bits_from_child(&F.mask[8 * (size_t)fl], a, &cmask[8 * (size_t)i]);
        }
    }
    // drop leaves without DOF
    int nc = 0;
    for (int i = 0; i < nu; ++i) {
        uint64_t any = 0;
        for (int w = 0; w < 8; ++w) any |= cmask[8 * i + w];
        nc += any != 0;
    }
    C.org.resize((size_t)nc * 3);
    C.mask.resize((size_t)nc * 8);
    C.child.resize((size_t)nc * 8);
    for (int i = 0, k = 0; i < nu; ++i) {
        uint64_t any = 0;
        for (int w = 0; w < 8; ++w) any |= cmask[8 * i + w];
        if (!any) continue;
        std::copy(&uorg[3 * i], &uorg[3 * i] + 3, &C.org[3 * (size_t)k]);
        std::copy(&cmask[8 * i], &cmask[8 * i] + 8, &C.mask[8 * (size_t)k]);
        std::copy(&child[8 * i], &child[8 * i] + 8, &C.child[8 * (size_t)k]);
        ++k;
    }
    C.nl = nc;
    finalize_host_level(C);
    F.parent.assign(F.nl, -1);
    F.octant.assign(F.nl, 0);
    for (int i = 0; i < C.nl; ++i)
        for (int a = 0; a < 8; ++a) {
            int fl = C.child[8 * i + a];
            if (fl >= 0) { F.parent[fl] = i; F.octant[fl] = (uint8_t)a; }
        }
}

// ---------------------------------------------------------------------------
// Bump allocator over a pinned host block.  Small tables go up through it: a
// cudaMemcpyAsync from pageable memory first waits for the work already in the
// stream (the large input copies), a copy from pinned memory does not.  An
// item that does not fit goes up from its pageable source.
struct PinStage {
    char* base = nullptr;
    size_t cap = 0, off = 0;
    const void* put(const void* src, size_t bytes) {
        if (!base || off + bytes > cap) return src;
        char* p = base + off;
        memcpy(p, src, bytes);
        off = (off + bytes + 15) & ~size_t(15);
        return p;
    }
    void* reserve(size_t bytes) {  // pinned space for a download, or nullptr
        if (!base || off + bytes > cap) return nullptr;
        char* p = base + off;
        off = (off + bytes + 15) & ~size_t(15);
        return p;
    }
};

struct DevGrid {  // device copy of an input grid + its leaf map
    DGrid g{};
    void* mem = nullptr;
    const uint8_t* read = nullptr;  // per leaf: read by the construction (set when only those were copied)
};

// What a face grid in pinned host memory needs to copy only the leaves the
// construction reads (k_face_leaves_read): the liquid SDF on the device and its
// per-leaf liquid flags.
struct FaceGather {
    const DGrid* phi;
    const uint8_t* liquid;
    int64_t* launches;
};
// The device address of pinned (page-locked, mapped) host memory, or null for
// pageable memory or an address a float4 load cannot start at.
static const void* host_mapped(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer || ((uintptr_t)a.devicePointer & 15)) return nullptr;
    return a.devicePointer;
}

}  // namespace

struct LevelDev {
    DLevel L{};
    float* lhs = nullptr;
    float* rhs = nullptr;
    float* tmp = nullptr;
    float* tmp2 = nullptr;  // second scratch vector: the intermediate of a fused sweep pair (k_sweep2)
    float* spai0 = nullptr;
    uint32_t* flags = nullptr;
    int* spai0_ready = nullptr;
    int* dof_base = nullptr;
    int* org = nullptr;
    float w_sor = 1.2f;
    float dt = 0, dx = 0;
};

struct MixedData;  // the mixed-precision form's data (mixed.cu)

struct uaamg_poisson {
    DeviceCtx* ctx = nullptr;
    void* pin_state = nullptr;  // pinned block holding st_host and scalar_host
    size_t pin_state_cap = 0;
    void* pin_stage = nullptr;  // pinned staging of the level-0 table upload
    size_t pin_stage_cap = 0;
    void* pin_stage2 = nullptr;  // pinned staging of the coarse levels' table upload
    size_t pin_stage2_cap = 0;
    void* pin_in = nullptr;  // pinned staging of the small input tables (leaf maps, origins, masks)
    size_t pin_in_cap = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t body_stream = nullptr;
    std::vector<HostLevel> host;
    std::vector<LevelDev> lv;
    int nlev = 0;
    // hierarchy memory (one allocation)
    char* dmem = nullptr;   // level 0 and the PCG's vectors
    size_t dmem_bytes = 0;
    char* dmem2 = nullptr;  // the coarse levels and the coarsest system
    // coarsest
    DCoarsest C{};
    // PCG
    float *x = nullptr, *b = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    double* partials = nullptr;
    PcgState* st = nullptr;
    PcgState* st_host = nullptr;  // pinned
    float* scalar_dev = nullptr;
    float* scalar_host = nullptr;  // pinned
    // options
    int smoother = UAAMG_SMOOTHER_SCHEDULED_RELAXED_JACOBI;
    int max_iter = 100;
    float rel_tol = 1e-7f;
    int use_graph = 1;
    // graph
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_key = -1;
    std::shared_ptr<struct SolveGraph> shared_graph;  // set when graph / graph_exec belong to the solve-graph cache
    bool use_sweep2 = true;  // fused Jacobi sweep pairs (Enq::pair), fixed at creation
    int64_t body_launches = 0, setup_launches = 0, finish_launches = 0;
    int64_t launches = 0;
    int64_t last_launches = 0;
    int iterations = 0;
    float final_residual = 0.f;
    bool spai0_built = false;
    float dt = 0, dx = 0;
    int64_t solves = 0;
    MixedData* mixed = nullptr;  // 16-bit hierarchy copy, FP64 coarsest inverse, graph
    int replace_every = 25;      // true-residual replacement interval of the mixed form
    void* noalloc_scratch = nullptr;  // device address of the allocation-free entry point's array
    float* rhs0 = nullptr;  // the rhs built by uaamg_poisson_create_with_rhs (level-0 vector)
    bool rhs_resident = false;
    // the bottom of the W-cycle in one cluster launch (k_bottom): decided once
    // per handle; level lb = nlev - 2, P leaves per CTA, a cluster of bot_C
    int bot_state = -1;  // -1 undecided, 0 not used (or turned off by UAAMG_BOTTOM=0 at creation), 1 used
    int bot_C = 0, bot_P = 0, bot_rows = 0;
    size_t bot_smem = 0;
};

namespace {

template <typename T>
static T* carve(char*& cur, size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(cur);
    cur += bytes;
    return p;
}
static size_t carve_size(size_t count, size_t elem) { return (count * elem + 255) & ~size_t(255); }

// Device copy of an input grid and its leaf map.  When `share` (a grid whose
// device map `share_dg` is already built) lists the same leaves in the same
// order, as the face-velocity channels and the face weights of a staggered
// grid usually do, its map is reused and only the values go up.  With `fg`, a
// face grid whose values are in pinned host memory is gathered by a kernel
// that reads only the leaves the construction reads (the others are NaN).
static void upload_grid_cs(DeviceCtx* ctx, cudaStream_t stream, const uaamg_leaf_grid* gr, DevGrid& dg, HostMap& map,
                           std::vector<void*>& tofree, const uaamg_leaf_grid* share = nullptr,
                           const DevGrid* share_dg = nullptr, PinStage* stage = nullptr,
                           const FaceGather* fg = nullptr) {
    const bool same = share && share_dg && share_dg->g.map && share->leaf_count == gr->leaf_count &&
                      gr->leaf_count > 0 &&
                      (share->origins == gr->origins ||
                       memcmp(share->origins, gr->origins, (size_t)gr->leaf_count * 3 * sizeof(int32_t)) == 0);
    if (!same) map.build(gr->leaf_count, gr->origins);
    dg.g = DGrid{};
    dg.g.comps = gr->components;
    dg.g.bg0 = gr->background[0];
    dg.g.bg1 = gr->components > 1 ? gr->background[1] : 0.f;
    dg.g.bg2 = gr->components > 2 ? gr->background[2] : 0.f;
    if (gr->leaf_count == 0) return;
    size_t mapn = same ? 0 : map.idx.size();
    const size_t n = (size_t)gr->leaf_count;
    size_t vbytes = n * UAAMG_LEAF * gr->components * sizeof(float);
    const void* mapped = (fg && !gr->values_on_device) ? host_mapped(gr->values) : nullptr;
    const bool own_read = mapped && !(same && share_dg->read);  // this grid's read flags are computed here
    size_t total = carve_size(mapn, 4) + (gr->values_on_device ? 0 : carve_size(vbytes, 1)) +
                   (own_read ? carve_size(n * 3, 4) + carve_size(n, 1) : 0);
    void* mem = nullptr;
    CK(ctx_dev_alloc(ctx, &mem, total, stream));
    tofree.push_back(mem);
    char* cur = (char*)mem;
    int* dmap = nullptr;
    if (same) {
        dmap = const_cast<int*>(share_dg->g.map);
        dg.g.lo0 = share_dg->g.lo0; dg.g.lo1 = share_dg->g.lo1; dg.g.lo2 = share_dg->g.lo2;
        dg.g.d0 = share_dg->g.d0; dg.g.d1 = share_dg->g.d1; dg.g.d2 = share_dg->g.d2;
    } else {
        dmap = carve<int>(cur, mapn);
        const void* src = stage ? stage->put(map.idx.data(), mapn * 4) : map.idx.data();
        CK(cudaMemcpyAsync(dmap, src, mapn * 4, cudaMemcpyHostToDevice, stream));
    }
    const float* vals = gr->values;
    if (!gr->values_on_device) {
        float* dv = carve<float>(cur, vbytes / 4);
        if (mapped) {
            const uint8_t* read = same ? share_dg->read : nullptr;
            if (own_read) {
                int* dorg = carve<int>(cur, n * 3);
                uint8_t* rd = carve<uint8_t>(cur, n);
                const void* osrc = stage ? stage->put(gr->origins, n * 12) : gr->origins;
                CK(cudaMemcpyAsync(dorg, osrc, n * 12, cudaMemcpyHostToDevice, stream));
                k_face_leaves_read<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(dorg, (int)n, *fg->phi, fg->liquid,
                                                                                    rd);
                CHECK_LAUNCH();
                ++*fg->launches;
                read = rd;
            }
            const int gctas = (int)std::min<int64_t>(n, std::max(1, ctx->sms));
            k_gather_host_leaves<<<(unsigned)gctas, 128, 0, stream>>>(static_cast<const float4*>(mapped),
                                                                      gr->components, (int)n, read,
                                                                      reinterpret_cast<float4*>(dv));
            CHECK_LAUNCH();
            ++*fg->launches;
            dg.read = read;
        } else {
            CK(cudaMemcpyAsync(dv, gr->values, vbytes, cudaMemcpyHostToDevice, stream));
        }
        vals = dv;
    }
    dg.g.val = vals;
    dg.g.map = dmap;
    if (!same) {
        dg.g.lo0 = map.lo[0]; dg.g.lo1 = map.lo[1]; dg.g.lo2 = map.lo[2];
        dg.g.d0 = map.dim[0]; dg.g.d1 = map.dim[1]; dg.g.d2 = map.dim[2];
    }
}

static void upload_grid(uaamg_poisson* h, const uaamg_leaf_grid* gr, DevGrid& dg, HostMap& map,
                        std::vector<void*>& tofree, PinStage* stage = nullptr) {
    upload_grid_cs(h->ctx, h->stream, gr, dg, map, tofree, nullptr, nullptr, stage);
}

static void check_grid(const uaamg_leaf_grid* g, int comps, const char* name) {
    if (!g) { set_error("%s is NULL", name); throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT}; }
    if (g->components != comps) {
        set_error("%s must have %d component(s), got %d", name, comps, g->components);
        throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
    }
    if (g->leaf_count < 0 || (g->leaf_count > 0 && (!g->origins || !g->values))) {
        set_error("%s has no origins/values", name);
        throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
    }
    int32_t low = 0;  // the OR of every origin coordinate's low bits (one vectorisable pass)
    for (int64_t i = 0; i < 3 * g->leaf_count; ++i) low |= g->origins[i];
    if (low & 7) {
        set_error("%s: leaf origins must be multiples of 8", name);
        throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
    }
}

static LevelOut level_out(LevelDev& d) {
    LevelOut O;
    O.diag = const_cast<float*>(d.L.diag);
    O.cx = const_cast<float*>(d.L.cx);
    O.cy = const_cast<float*>(d.L.cy);
    O.cz = const_cast<float*>(d.L.cz);
    O.invdiag = const_cast<float*>(d.L.invdiag);
    O.flags = d.flags;
    // trimDefaultNodes (simd_vdb_poisson.cpp:1756-1770)
    float term = -d.dt / (d.dx * d.dx);
    float diagonalTerm = -6.0f * term;
    O.def_diag = diagonalTerm;
    O.def_face = term;
    O.eps_diag = fabsf(diagonalTerm * 1e-5f);
    O.eps_face = fabsf(term * 1e-5f);
    O.inv_bg = 1.0f / d.L.def_diag;
    O.def_invdiag = d.L.def_invdiag;
    return O;
}

}  // namespace

// ---------------------------------------------------------------------------
// hierarchy construction
#include <chrono>
static double trace_now() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static bool trace_on() {
    static int on = -1;
    if (on < 0) { const char* e = getenv("UAAMG_TRACE"); on = (e && e[0] == '1') ? 1 : 0; }
    return on == 1;
}
#define TRACE(label)                                                                   \
    do {                                                                               \
        if (trace_on()) {                                                              \
            double t_ = trace_now();                                                   \
            fprintf(stderr, "[uaamg] %-28s %8.3f ms\n", label, t_ - trace_t0);        \
            trace_t0 = t_;                                                             \
        }                                                                              \
    } while (0)

struct EventGuard {
    cudaEvent_t e = nullptr;
    ~EventGuard() {
        if (e) cudaEventDestroy(e);
    }
};

// The face-velocity inputs of the right-hand side, when the hierarchy build
// also builds it (uaamg_poisson_create_with_rhs).
struct RhsInputs {
    const uaamg_leaf_grid *vx, *vy, *vz, *sv;
};

static void build_hierarchy(uaamg_poisson* h, const uaamg_leaf_grid* phi, const uaamg_leaf_grid* fw, float dt,
                            float dx, const RhsInputs* ri = nullptr) {
    double trace_t0 = trace_now();
    check_grid(phi, 1, "liquid_phi");
    check_grid(fw, 3, "face_weights");
    if (ri) {
        check_grid(ri->vx, 1, "vx");
        check_grid(ri->vy, 1, "vy");
        check_grid(ri->vz, 1, "vz");
        check_grid(ri->sv, 3, "solid_velocity");
    }
    if (!(dx > 0.f)) { set_error("dx must be positive"); throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT}; }
    h->dt = dt;
    h->dx = dx;
    cudaStream_t s = h->stream;
    std::vector<void*> tofree;
    const int64_t nphi = phi->leaf_count;
    h->host.clear();
    h->host.reserve(32);  // references into it are held while levels are appended
    h->host.emplace_back();
    HostLevel& L0 = h->host[0];
    L0.dt = dt;
    L0.dx = dx;
    if (nphi > 0) {
        // ---- inputs to the device
        HostMap phimap, fwmap;
        DevGrid dphi, dfw;
        // the small input tables go up through a pinned block the handle keeps
        CK(ctx_pinned_acquire(h->ctx, (size_t)4 << 20, &h->pin_in, &h->pin_in_cap));
        PinStage stage{(char*)h->pin_in, h->pin_in_cap, 0};
        upload_grid(h, phi, dphi, phimap, tofree, &stage);
        TRACE("  liquid SDF up");
        // the liquid SDF's origins and active masks, its DOF masks, its per-leaf liquid flags
        size_t extra = carve_size((size_t)nphi * 8, 8) * 2 + carve_size((size_t)nphi * 3, 4) + carve_size((size_t)nphi, 1);
        void* mem = nullptr;
        CK(ctx_dev_alloc(h->ctx, &mem, extra, s));
        tofree.push_back(mem);
        char* cur = (char*)mem;
        uint64_t* dphimask = carve<uint64_t>(cur, (size_t)nphi * 8);
        uint64_t* ddofmask = carve<uint64_t>(cur, (size_t)nphi * 8);
        int* dphiorg = carve<int>(cur, (size_t)nphi * 3);
        uint8_t* dliquid = carve<uint8_t>(cur, (size_t)nphi);
        CK(cudaMemcpyAsync(dphiorg, stage.put(phi->origins, (size_t)nphi * 12), (size_t)nphi * 12,
                           cudaMemcpyHostToDevice, s));
        const uint64_t* pm = nullptr;
        if (phi->masks) {
            CK(cudaMemcpyAsync(dphimask, stage.put(phi->masks, (size_t)nphi * 64), (size_t)nphi * 64,
                               cudaMemcpyHostToDevice, s));
            pm = dphimask;
        }
        // Face grids in pinned host memory cross the bus only where the construction reads them (the leaves
        // at and above liquid leaves): the liquid flags come first.
        FaceGather fgather{&dphi.g, dliquid, &h->launches};
        const FaceGather* fgp = nullptr;
        {
            bool host_faces = !fw->values_on_device;
            if (ri)
                for (const uaamg_leaf_grid* g : {ri->vx, ri->vy, ri->vz, ri->sv})
                    host_faces = host_faces || (!g->values_on_device && g->leaf_count > 0);
            if (host_faces) {
                k_liquid_leaves<<<(unsigned)nphi, 128, 0, s>>>(dphi.g, pm, dliquid);
                CHECK_LAUNCH();
                h->launches++;
                fgp = &fgather;
            }
        }
        TRACE("  SDF tables up");
        upload_grid_cs(h->ctx, s, fw, dfw, fwmap, tofree, nullptr, nullptr, &stage, fgp);
        TRACE("  face weights up");
        // The velocities of the right-hand side go up on a second stream once
        // the SDF and the face weights are up, so their copies overlap the DOF
        // mask kernel, the host topology and the coefficient kernels.
        HostMap vmap[4];
        DevGrid dvel[4];
        EventGuard ev_in, ev_vel, ev_l0;
        if (ri) {
            cudaStream_t s2 = h->body_stream;
            CK(cudaEventCreateWithFlags(&ev_in.e, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ev_vel.e, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ev_l0.e, cudaEventDisableTiming));
            CK(cudaEventRecord(ev_in.e, s));
            CK(cudaStreamWaitEvent(s2, ev_in.e, 0));
            const uaamg_leaf_grid* vg[4] = {ri->vx, ri->vy, ri->vz, ri->sv};
            // the channels' maps come from the face weights' when the leaves match (the face-weight map
            // was uploaded on the first stream, which the second stream waits for)
            for (int k = 0; k < 4; ++k)
                upload_grid_cs(h->ctx, s2, vg[k], dvel[k], vmap[k], tofree, fw, &dfw, &stage, fgp);
        }
        TRACE("upload inputs");
        const float dtOverDxSqr = dt / (dx * dx);
        k_finest_mask<<<(unsigned)nphi, 128, 0, s>>>(dphi.g, pm, dphiorg, dfw.g, dtOverDxSqr, ddofmask);
        CHECK_LAUNCH();
        h->launches++;
        // the DOF masks come back into pinned memory, so the copy does not hold the host
        std::vector<uint64_t> dofmask_pageable;
        uint64_t* dofmask = static_cast<uint64_t*>(stage.reserve((size_t)nphi * 64));
        if (!dofmask) {
            dofmask_pageable.resize((size_t)nphi * 8);
            dofmask = dofmask_pageable.data();
        }
        CK(cudaMemcpyAsync(dofmask, ddofmask, (size_t)nphi * 64, cudaMemcpyDeviceToHost, s));
        // while the mask kernel and its copy run: the tree-order key of every liquid-SDF leaf, and whether
        // the leaves are in tree order already (as an OpenVDB leaf iteration gives them)
        std::vector<unsigned __int128> pkey((size_t)nphi);
        bool phi_sorted = true;
        for (int64_t i = 0; i < nphi; ++i) {
            pkey[i] = vdb_key128(&phi->origins[3 * i]);
            if (i > 0 && pkey[i] < pkey[i - 1]) phi_sorted = false;
        }
        CK(cudaStreamSynchronize(s));
        TRACE("DOF mask kernel + D2H");
        // ---- level-0 DOF leaves in tree order
        std::vector<std::pair<unsigned __int128, int>> keys;
        keys.reserve(nphi);
        for (int64_t i = 0; i < nphi; ++i) {
            uint64_t any = 0;
            for (int w = 0; w < 8; ++w) any |= dofmask[8 * i + w];
            if (any) keys.push_back({pkey[i], (int)i});
        }
        if (!phi_sorted) std::sort(keys.begin(), keys.end());  // a subset of sorted leaves is sorted
        TRACE("  level-0 leaves ordered");
        std::vector<int32_t> src(keys.size());
        L0.org.resize(keys.size() * 3);
        L0.mask.resize(keys.size() * 8);
        for (size_t i = 0; i < keys.size(); ++i) {
            const int sidx = keys[i].second;
            src[i] = sidx;
            std::copy(&phi->origins[3 * sidx], &phi->origins[3 * sidx] + 3, &L0.org[3 * i]);
            std::copy(&dofmask[8 * (size_t)sidx], &dofmask[8 * (size_t)sidx] + 8, &L0.mask[8 * i]);
        }
        L0.nl = (int)keys.size();
        finalize_host_level(L0);
        TRACE("  level-0 tables");
        // ---- level 0 goes to the device first: its tables go up and its
        // coefficients (and the rhs) are computed while the host coarsens the
        // topology.  Two device blocks: level 0 with the PCG's vectors, then the
        // coarse levels, level 0's parent / octant tables (which coarsening
        // makes) and the coarsest system.  Each block's host-built tables lie
        // contiguous at its start, so their pinned image goes up in one copy;
        // the rest of the block is zeroed on the device.
        const size_t n0 = (size_t)L0.nl * UAAMG_LEAF;
        h->lv.assign(1, LevelDev());
        // the arrays of one level (coefficients, flags, vectors) and its DLevel fields
        auto carve_arrays = [&](const HostLevel& H, LevelDev& D, char*& cur) {
            const size_t n = (size_t)H.nl;
            D.dt = H.dt;
            D.dx = H.dx;
            D.flags = carve<uint32_t>(cur, n);
            D.spai0_ready = carve<int>(cur, 1);
            float* dg = carve<float>(cur, n * UAAMG_LEAF);
            float* cx = carve<float>(cur, n * UAAMG_LEAF);
            float* cy = carve<float>(cur, n * UAAMG_LEAF);
            float* cz = carve<float>(cur, n * UAAMG_LEAF);
            float* iv = carve<float>(cur, n * UAAMG_LEAF);
            D.spai0 = carve<float>(cur, n * UAAMG_LEAF);
            D.lhs = carve<float>(cur, n * UAAMG_LEAF);
            D.rhs = carve<float>(cur, n * UAAMG_LEAF);
            D.tmp = carve<float>(cur, n * UAAMG_LEAF);
            D.tmp2 = carve<float>(cur, n * UAAMG_LEAF);
            const float t = H.dt / (H.dx * H.dx);  // LaplacianApplySIMD ctor (.cpp:1045-1065)
            DLevel& L = D.L;
            L.nl = (int)n;
            L.diag = dg; L.cx = cx; L.cy = cy; L.cz = cz; L.invdiag = iv; L.spai0 = D.spai0; L.flags = D.flags;
            L.def_face = -t;
            L.def_diag = 6.f * t;
            L.def_invdiag = 1.0f / (6.f * t);
            L.def_spai0 = 1.0f / (7.f * t);
        };
        auto arrays_bytes = [](size_t n) {
            return carve_size(n, 4) + carve_size(1, 4) + 10 * carve_size(n * UAAMG_LEAF, 4);  // flags ... tmp2
        };
        using Up = std::pair<void*, std::pair<const void*, size_t>>;
        // a block's table image through pinned memory the handle keeps until destroy (create() need not wait for
        // the copy); the arrays not uploaded and the alignment gaps are zero, as the device memset made them
        auto upload_tables = [&](char* block, size_t table_bytes, const std::vector<Up>& ups, void** pin,
                                 size_t* cap) {
            CK(ctx_pinned_acquire(h->ctx, table_bytes + 512, pin, cap));
            char* img = (char*)*pin;
            memset(img, 0, table_bytes);
            for (const Up& u : ups) memcpy(img + ((char*)u.first - block), u.second.first, u.second.second);
            CK(cudaMemcpyAsync(block, img, table_bytes, cudaMemcpyHostToDevice, s));
        };
        int* dsrc = nullptr;
        {
            const size_t n = (size_t)L0.nl;
            size_t bytes = carve_size(n * 8, 8) + carve_size(n * 6, 4) + carve_size(n * 8, 4) + carve_size(n, 4) +
                           carve_size(n * 3, 4) + carve_size(src.size(), 4) + arrays_bytes(n);
            bytes += (ri ? 7 : 6) * carve_size(n0, 4);  // x b r z p q (+ the built rhs)
            bytes += carve_size(red_buffer_doubles(std::max<size_t>(n, 1)), 8);
            bytes += carve_size(sizeof(PcgState), 1) + carve_size(64, 4);
            CK(ctx_dev_alloc(h->ctx, (void**)&h->dmem, bytes, s));
            h->dmem_bytes = bytes;
            char* cur = h->dmem;
            LevelDev& D0 = h->lv[0];
            std::vector<Up> ups;
            uint64_t* m = carve<uint64_t>(cur, n * 8);
            int* nb = carve<int>(cur, n * 6);
            int* ch = carve<int>(cur, n * 8);
            D0.dof_base = carve<int>(cur, n);
            D0.org = carve<int>(cur, n * 3);
            dsrc = carve<int>(cur, src.size());
            ups.push_back({m, {L0.mask.data(), n * 64}});
            ups.push_back({nb, {L0.nbr.data(), n * 24}});
            ups.push_back({D0.dof_base, {L0.dof_base.data(), n * 4}});
            ups.push_back({D0.org, {L0.org.data(), n * 12}});
            ups.push_back({dsrc, {src.data(), src.size() * 4}});
            const size_t table_bytes = (size_t)(cur - h->dmem);
            CK(cudaMemsetAsync(cur, 0, bytes - table_bytes, s));
            carve_arrays(L0, D0, cur);
            D0.L.mask = m;
            D0.L.nbr = nb;
            D0.L.child = ch;
            h->x = carve<float>(cur, n0);
            h->b = carve<float>(cur, n0);
            h->r = carve<float>(cur, n0);
            h->z = carve<float>(cur, n0);
            h->p = carve<float>(cur, n0);
            h->q = carve<float>(cur, n0);
            if (ri) h->rhs0 = carve<float>(cur, n0);
            h->partials = carve<double>(cur, red_buffer_doubles(std::max<size_t>(n, 1)));
            h->st = reinterpret_cast<PcgState*>(carve<char>(cur, sizeof(PcgState)));
            h->scalar_dev = carve<float>(cur, 64);
            upload_tables(h->dmem, table_bytes, ups, &h->pin_stage, &h->pin_stage_cap);
        }
        if (ri) {
            // createPressurePoissonRightHandSide into the PCG's b (the face
            // weights uploaded once serve the matrix and the rhs), on the
            // velocities' stream once they and level 0's tables are up: the
            // coarse levels' kernels that follow on the first stream do not
            // wait for the velocities, which the first stream joins at the end
            cudaStream_t s2 = h->body_stream;
            LevelDev& D0 = h->lv[0];
            if (D0.L.nl > 0) {
                CK(cudaEventRecord(ev_l0.e, s));
                CK(cudaStreamWaitEvent(s2, ev_l0.e, 0));
                k_build_rhs<<<(unsigned)D0.L.nl, 128, 0, s2>>>(D0.L.mask, D0.org, dfw.g, dvel[0].g, dvel[1].g,
                                                               dvel[2].g, dvel[3].g, 1.0f / dx, h->rhs0);
                CHECK_LAUNCH();
                h->launches++;
            }
            CK(cudaEventRecord(ev_vel.e, s2));
            h->rhs_resident = true;
        }
        if (L0.nl > 0) {
            LevelDev& D0 = h->lv[0];
            k_finest_coef<<<(unsigned)L0.nl, 128, 0, s>>>(dphi.g, dphiorg, dfw.g, dtOverDxSqr, dsrc, D0.L.mask,
                                                          level_out(D0));
            CHECK_LAUNCH();
            h->launches++;
        }
        TRACE("level 0 up, its kernels enqueued");
        // ---- coarse topology: constructMultigridHierarchy (.cpp:1813-1842)
        while (h->host.back().ndof > 4000 && h->host.size() < 32) {
            h->host.emplace_back();
            HostLevel& F = h->host[h->host.size() - 2];
            HostLevel& C = h->host.back();
            coarsen_topology(F, C);
            TRACE("  coarse level");
        }
        const int nlev = (int)h->host.size();
        const HostLevel& HC = h->host.back();
        size_t nc = (size_t)HC.ndof;
        if (nc > (size_t)CG_MAX_DOF) {
            set_error("coarsening stalled: %zu DOF on the coarsest level (max %d)", nc, CG_MAX_DOF);
            throw UaamgError{UAAMG_ERR_DOMAIN_TOO_LARGE};
        }
        h->lv.resize(nlev);
        int *dslot = nullptr, *ccol = nullptr;
        float *cdiag = nullptr, *cinvd = nullptr, *cval = nullptr;
        // ---- the coarse block
        {
            const size_t nl0 = (size_t)L0.nl;
            size_t bytes = carve_size(nl0, 4) + carve_size(nl0, 1);  // level 0's parent, octant
            for (int l = 1; l < nlev; ++l) {
                const size_t n = (size_t)h->host[l].nl;
                bytes += carve_size(n * 8, 8) + carve_size(n * 6, 4) + carve_size(n * 8, 4) + carve_size(n, 4) +
                         carve_size(n, 1) + carve_size(n, 4) + carve_size(n * 3, 4) + arrays_bytes(n);
            }
            bytes += carve_size(nc, 4) * 3 + carve_size(nc * 6, 4) * 2;
            CK(ctx_dev_alloc(h->ctx, (void**)&h->dmem2, bytes, s));
            char* cur = h->dmem2;
            std::vector<Up> ups;
            int* par0 = carve<int>(cur, nl0);
            uint8_t* oc0 = carve<uint8_t>(cur, nl0);
            if (!L0.parent.empty()) ups.push_back({par0, {L0.parent.data(), nl0 * 4}});
            if (!L0.octant.empty()) ups.push_back({oc0, {L0.octant.data(), nl0}});
            h->lv[0].L.parent = par0;
            h->lv[0].L.octant = oc0;
            for (int l = 1; l < nlev; ++l) {
                HostLevel& H = h->host[l];
                LevelDev& D = h->lv[l];
                const size_t n = (size_t)H.nl;
                uint64_t* m = carve<uint64_t>(cur, n * 8);
                int* nb = carve<int>(cur, n * 6);
                int* ch = carve<int>(cur, n * 8);
                int* par = carve<int>(cur, n);
                uint8_t* oc = carve<uint8_t>(cur, n);
                D.dof_base = carve<int>(cur, n);
                D.org = carve<int>(cur, n * 3);
                ups.push_back({m, {H.mask.data(), n * 64}});
                ups.push_back({nb, {H.nbr.data(), n * 24}});
                if (!H.child.empty()) ups.push_back({ch, {H.child.data(), n * 32}});
                if (!H.parent.empty()) ups.push_back({par, {H.parent.data(), n * 4}});
                if (!H.octant.empty()) ups.push_back({oc, {H.octant.data(), n}});
                ups.push_back({D.dof_base, {H.dof_base.data(), n * 4}});
                ups.push_back({D.org, {H.org.data(), n * 12}});
                D.L.mask = m; D.L.nbr = nb; D.L.child = ch; D.L.parent = par; D.L.octant = oc;
            }
            const size_t table_bytes = (size_t)(cur - h->dmem2);
            CK(cudaMemsetAsync(cur, 0, bytes - table_bytes, s));
            for (int l = 1; l < nlev; ++l) carve_arrays(h->host[l], h->lv[l], cur);
            h->C.n = (int)nc;
            dslot = carve<int>(cur, nc);
            cdiag = carve<float>(cur, nc);
            cinvd = carve<float>(cur, nc);
            ccol = carve<int>(cur, nc * 6);
            cval = carve<float>(cur, nc * 6);
            h->C.dof_slot = dslot; h->C.diag = cdiag; h->C.invd = cinvd; h->C.col = ccol; h->C.val = cval;
            upload_tables(h->dmem2, table_bytes, ups, &h->pin_stage2, &h->pin_stage2_cap);
        }
        TRACE("coarse levels up");
        for (int l = 1; l < nlev; ++l) {
            LevelDev& D = h->lv[l];
            if (D.L.nl == 0) continue;
            static bool coarsen_smem_set = false;
            if (!coarsen_smem_set) {
                CK(cudaFuncSetAttribute(k_coarsen, cudaFuncAttributeMaxDynamicSharedMemorySize, COARSEN_SMEM));
                coarsen_smem_set = true;
            }
            k_coarsen<<<(unsigned)D.L.nl, 128, COARSEN_SMEM, s>>>(h->lv[l - 1].L, D.L.child, D.L.mask, level_out(D));
            CHECK_LAUNCH();
            h->launches++;
        }
        if (h->lv[nlev - 1].L.nl > 0) {
            LevelDev& D = h->lv[nlev - 1];
            k_coarsest_ell<<<(unsigned)D.L.nl, 128, 0, s>>>(D.L, D.dof_base, dslot, cdiag, cinvd, ccol, cval);
            CHECK_LAUNCH();
            h->launches++;
        }
        // the rhs and the velocities' buffers: done before the inputs are freed and the handle is used
        if (ri) CK(cudaStreamWaitEvent(s, ev_vel.e, 0));
        for (void* pmem : tofree) CK(cudaFreeAsync(pmem, s));
        tofree.clear();
        TRACE("coefficient kernels enqueued");
        h->nlev = nlev;
    } else {
        h->nlev = 1;
        h->lv.assign(1, LevelDev());
        h->rhs_resident = ri != nullptr;
    }
}

static void ensure_spai0(uaamg_poisson* h) {
    if (h->spai0_built) return;
    for (int l = 0; l < h->nlev; ++l) {
        LevelDev& D = h->lv[l];
        if (D.L.nl == 0) continue;
        float bg = D.L.def_diag;  // mDiagonal->background()
        float defaultSPAI0Val = 6.0f / (7.f * bg);
        k_spai0<<<(unsigned)D.L.nl, 128, 0, h->stream>>>(D.L, D.spai0, D.flags, defaultSPAI0Val,
                                                         fabsf(defaultSPAI0Val * 1e-5f));
        CHECK_LAUNCH();
        h->launches++;
    }
    h->spai0_built = true;
}

// ---------------------------------------------------------------------------
// kernel enqueue helpers
namespace {

// Launch with programmatic stream serialisation (PDL); the kernels start with
// griddepcontrol.wait, so ordering is preserved while launch latency overlaps.
static bool g_use_pdl = true;
// Level sweeps with SrcPlain on levels of at least STAGED_MIN_LEAVES leaves run
// the bulk-async staged kernels (UAAMG_STAGED=0 turns them off).
static bool g_use_staged = true;
static bool g_use_sweep2 = true;  // fused Jacobi sweep pairs (Enq::pair)
// Kernel shapes by level size (uaamg_set_tuning): the defaults below, or the
// table an autotuner wrote.  Every choice gives the same results; only the
// speed differs.  g_tune_gen is part of every graph's key, so a change rebuilds
// cached graphs.
static uaamg_tuning g_tune = {64, 1024, 8192, 16, 1};
static int g_tune_gen = 0;
static int g_sms = 148;  // SMs of the device (set when a handle is created)
#define STAGED_MIN_LEAVES (g_tune.staged_min_leaves)
// On levels of at least SPLIT_MIN_LEAVES leaves a sweep whose source is
// computed (the first sweep from a zero guess, the prolongation-add) runs as
// k_materialize of the source and a staged plain sweep: the fused kernel
// recomputes the source at every stencil neighbour from dependent loads,
// which costs more than one extra elementwise pass on large levels.  The
// stored values are the ones the fused kernel computes, so the results are
// identical.
#define SPLIT_MIN_LEAVES (g_tune.split_min_leaves)
// Levels of at least PIPE_MIN_LEAVES leaves sweep with the persistent
// pipelined kernels (several leaves per CTA); smaller staged levels with the
// one-leaf staged kernels, which start faster.
#define PIPE_MIN_LEAVES (g_tune.pipe_min_leaves)
// A pass that carries a level-0 dot product (the last post-smoothing sweep
// with z.r, A p with p.q) uses the pipelined kernel from this fixed size on:
// its per-CTA partials set the dot's summation order, which must not depend
// on the tuning.  The mixed-precision form uses it for all its passes.
#define PIPE_DOT_MIN_LEAVES 8192
// Grid of the grid-stride elementwise kernels (k_materialize, the PCG
// vector updates): 16 CTAs of 128 threads per SM of a 148-SM B200, at most
// one per leaf.  One CTA per leaf would make a large level's elementwise
// pass cost the GPU's CTA launch rate (about a nanosecond per CTA) instead
// of its bytes.
static unsigned elem_grid(int nl) { return (unsigned)std::min(nl, g_tune.elem_ctas_per_sm * g_sms); }
// ---------------------------------------------------------------------------
// Launch recorder.  While t_rec is set (on this thread), the launch helpers
// append each launch -- kernel, grid, block, shared memory, attributes and the
// bytes of its arguments -- and each memset to t_rec instead of issuing it.
// Two recordings of the PCG's enqueue code are equal exactly when the graphs
// captured from them would be equal (the conditional handle is recorded as 0),
// which lets a new handle replay a graph captured for an earlier handle whose
// buffers sat at the same addresses (solve_graph_cache).
struct LaunchRec {
    std::vector<unsigned char> bytes;
    void put(const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        bytes.insert(bytes.end(), c, c + n);
    }
    template <class T>
    void val(const T& v) {
        static_assert(std::is_trivially_copyable<T>::value, "recorded argument");
        put(&v, sizeof(T));
    }
};
static thread_local LaunchRec* t_rec = nullptr;
template <typename... KArgs, typename... Args>
static void rec_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, int attrs, Args... args) {
    LaunchRec& r = *t_rec;
    r.val((unsigned char)'K');
    r.val(reinterpret_cast<const void*>(kern));
    r.val(grid);
    r.val(block);
    r.val(smem);
    r.val(attrs);
    (r.val(static_cast<KArgs>(args)), ...);
}
static void enq_memset(void* p, int v, size_t n, cudaStream_t s) {
    if (t_rec) {
        t_rec->val((unsigned char)'M');
        t_rec->val(p);
        t_rec->val(v);
        t_rec->val(n);
        return;
    }
    CK(cudaMemsetAsync(p, v, n, s));
}

template <typename... KArgs, typename... Args>
static void launch(void (*kern)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
    if (t_rec) {
        rec_launch(kern, dim3(grid), dim3(block), 0, g_use_pdl ? 1 : 0, args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_use_pdl ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

// Launch of a pipelined staged kernel (staged_pipe.cuh) over nl leaves:
// PIPE_CTAS CTAs, at most one per leaf.
template <typename... KArgs, typename... Args>
static void launch_pipe(void (*kern)(KArgs...), int nl, size_t smem, cudaStream_t s, Args... args) {
    const int g = std::min(nl, PIPE_CTAS);
    if (t_rec) {
        rec_launch(kern, dim3((unsigned)g), dim3(128), smem, g_use_pdl ? 1 : 0, args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)g);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_use_pdl ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

// Optional per-kernel timing (diagnostics): a CUDA event pair around every launch.
struct ProfRec {
    std::string label;
    cudaEvent_t a, b;
};

// sums the event-timed launches per label (first max_classes labels, in
// first-seen order) and destroys the events
static void prof_collect(std::vector<ProfRec>& prof, int max_classes, char* names, double* total_ms, int64_t* counts,
                         int* nclasses) {
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
    prof.clear();
    *nclasses = (int)lab.size();
}

template <class Src> struct SrcName { static const char* get() { return ""; } };
template <> struct SrcName<SrcFirstJacobi> { static const char* get() { return "+first"; } };
template <> struct SrcName<SrcFirstSpai0> { static const char* get() { return "+first"; } };
template <> struct SrcName<SrcFirstRbgs> { static const char* get() { return "+first"; } };
template <> struct SrcName<SrcProlong> { static const char* get() { return "+prolong"; } };
static const char* mode_name(int m) {
    static const char* n[] = {"jacobi", "residual", "laplacian", "red_gs", "black_gs", "spai0"};
    return n[m];
}

struct Enq {
    uaamg_poisson* h;
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

    template <int MODE, class Src>
    void sweep(int l, const Src& src, const float* b, float* out, float w, DotOut dot = DotOut{nullptr, nullptr, nullptr},
               bool mark_spai0 = false) {
        LevelDev& D = h->lv[l];
        float ws = D.w_sor;
        if constexpr (std::is_same<Src, SrcPlain>::value) {
            if (g_use_staged && D.L.nl >= STAGED_MIN_LEAVES && !(MODE == M_SPAI0 && mark_spai0)) {
                if (prof) pb("L" + std::to_string(l) + " " + mode_name(MODE) + " staged" + (dot.r ? "+dot" : ""));
                if (D.L.nl >= (dot.r ? PIPE_DOT_MIN_LEAVES : PIPE_MIN_LEAVES))
                    launch_pipe(k_pipe<MODE, DLevel, float, false>, D.L.nl, pipe_smem_bytes<DLevel>(), s, D.L,
                                (const float*)src.x, b, out, w, ws, 1.0f - ws, dot, (const float*)nullptr, 0.f,
                                &h->st->error);
                else
                    launch(k_sweep_staged<MODE>, (unsigned)D.L.nl, 128, s, D.L, (const float*)src.x, b, out, w, ws,
                           1.0f - ws, dot, &h->st->error);
                pe();
                count++;
                return;
            }
        }
        if (prof) pb("L" + std::to_string(l) + " " + mode_name(MODE) + SrcName<Src>::get() + (dot.r ? "+dot" : ""));
        launch(k_sweep<MODE, Src>, (unsigned)D.L.nl, 128, s, D.L, src, b, out, w, ws, 1.0f - ws, dot,
               mark_spai0 ? D.spai0_ready : nullptr);
        pe();
        count++;
    }
    bool split(int l) const { return g_use_staged && h->lv[l].L.nl >= SPLIT_MIN_LEAVES; }
    // whether two consecutive Jacobi sweeps of level l run as one k_sweep2:
    // latency-bound levels of about one wave at 2 CTAs per SM (from the staged
    // size on); on larger levels the face-layer recomputation costs more than
    // the launch it saves (measured: 776 and 784 leaves slower, 120-284 faster)
    bool pair(int l) const {
        const int nl = h->lv[l].L.nl;
        return h->use_sweep2 && !split(l) && nl >= STAGED_MIN_LEAVES && nl <= 2 * g_sms;
    }
    template <class Src>
    void sweep2(int l, const Src& src, const float* b, float* out, float wa, float wb) {
        LevelDev& D = h->lv[l];
        if (prof) pb("L" + std::to_string(l) + " jacobi pair" + SrcName<Src>::get());
        launch(k_sweep2<Src>, (unsigned)D.L.nl, SW2_THREADS, s, D.L, src, b, out, wa, wb);
        pe();
        count++;
    }
    template <class Src>
    void materialize(int l, const Src& src, float* out) {
        LevelDev& D = h->lv[l];
        if (prof) pb("L" + std::to_string(l) + " materialize" + SrcName<Src>::get());
        launch(k_materialize<Src>, elem_grid(D.L.nl), 128, s, D.L, src, out);
        pe();
        count++;
    }
    void restrict_resid(int l, const float* x, const float* b) {
        LevelDev& D = h->lv[l];
        if (g_use_staged && D.L.nl >= STAGED_MIN_LEAVES) {
            if (prof) pb("L" + std::to_string(l) + " residual+restrict staged");
            if (D.L.nl >= PIPE_MIN_LEAVES)
                launch_pipe(k_pipe<M_RESIDUAL, DLevel, float, true>, D.L.nl, pipe_smem_bytes<DLevel>(), s, D.L, x,
                            b, h->lv[l + 1].rhs, 0.f, 0.f, 0.f, DotOut{nullptr, nullptr, nullptr},
                            (const float*)nullptr, 0.f, &h->st->error);
            else
                launch(k_restrict_staged, (unsigned)D.L.nl, 128, s, D.L, x, b, h->lv[l + 1].rhs, &h->st->error);
            pe();
            count++;
            return;
        }
        if (prof) pb("L" + std::to_string(l) + " residual+restrict");
        launch(k_restrict<true>, (unsigned)D.L.nl, 128, s, D.L, x, b, h->lv[l + 1].rhs);
        pe();
        count++;
    }
    // both mu-visits of level lb = nlev - 2 with their coarsest solves, in one cluster launch
    void bottom(int lb, float* lhs, const float* rhs, const float w[3]) {
        BottomArgs A;
        memset(&A, 0, sizeof(A));  // padding included: the recorder compares argument bytes
        A.L = h->lv[lb].L;
        A.rhs = rhs;
        A.lhs = lhs;
        A.C = h->C;
        A.nlc = h->lv[lb + 1].L.nl;
        A.P = h->bot_P;
        A.w[0] = w[0]; A.w[1] = w[1]; A.w[2] = w[2];
        if (prof) pb("L" + std::to_string(lb) + " bottom (2 visits + coarsest)");
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)h->bot_C);
        cfg.blockDim = dim3(BOT_THREADS);
        cfg.dynamicSmemBytes = h->bot_smem;
        cfg.stream = s;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)h->bot_C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = g_use_pdl ? 2 : 1;
        if (t_rec) {
            const int attrs = (int)cfg.numAttrs * 1000 + h->bot_C;  // the cluster shape
            if (h->bot_rows == 2) rec_launch(k_bottom<2>, cfg.gridDim, cfg.blockDim, cfg.dynamicSmemBytes, attrs, A);
            else rec_launch(k_bottom<4>, cfg.gridDim, cfg.blockDim, cfg.dynamicSmemBytes, attrs, A);
        } else if (h->bot_rows == 2) {
            CK(cudaLaunchKernelEx(&cfg, k_bottom<2>, A));
        } else {
            CK(cudaLaunchKernelEx(&cfg, k_bottom<4>, A));
        }
        pe();
        count++;
    }
    void coarsest(const float* rhs, float* out) {
        if (h->C.n == 0) return;
        pb("coarsest cg");
        switch (coarsest_class(h->C.n)) {
            case 0: launch(k_coarsest_cg<2, 512>, 1, 512, s, h->C, rhs, out); break;
            case 1: launch(k_coarsest_cg<4, 512>, 1, 512, s, h->C, rhs, out); break;
            default: launch(k_coarsest_cg<4, 1024>, 1, 1024, s, h->C, rhs, out); break;
        }
        pe();
        count++;
    }
};

// Whether the two visits of level nlev - 2 (with the coarsest solves) run as
// one k_bottom cluster launch: Jacobi-family smoothers, at least three levels,
// a coarsest system the 256-thread CG shape takes (at most 2048 DOF), and a
// cluster of at most 16 CTAs whose shared memory holds level nlev - 2 and
// that the device can schedule.  The shape is decided once per handle.
static bool g_use_bottom = true;
template <int R>
static int bottom_clusters(int C, size_t smem, int max_dynamic) {
    // the largest size any handle may use, so that no handle's setting limits another's launches
    CK(cudaFuncSetAttribute(k_bottom<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic));
    CK(cudaFuncSetAttribute(k_bottom<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)C);
    cfg.blockDim = dim3(BOT_THREADS);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_bottom<R>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
static bool use_bottom(uaamg_poisson* h) {
    if (h->smoother != UAAMG_SMOOTHER_SCHEDULED_RELAXED_JACOBI && h->smoother != UAAMG_SMOOTHER_WEIGHTED_JACOBI)
        return false;
    if (h->bot_state >= 0) return h->bot_state == 1;
    h->bot_state = 0;
    if (h->nlev < 3) return false;
    const int lb = h->nlev - 2;
    const int nl = h->lv[lb].L.nl, nlc = h->lv[lb + 1].L.nl;
    if (nl <= 0 || nlc <= 0 || h->C.n <= 0 || coarsest_class(h->C.n) > 1) return false;
    const int P = (nl + BOT_MAX_CLUSTER - 1) / BOT_MAX_CLUSTER;
    const int C = (nl + P - 1) / P;
    const int rows = coarsest_class(h->C.n) == 0 ? 2 : 4;
    const size_t smem = bottom_smem_bytes(P, nlc, rows);
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->ctx->device));
    const int max_dynamic = optin - 1024;  // above the kernel's static shared memory
    if (smem > (size_t)max_dynamic) return false;
    if ((rows == 2 ? bottom_clusters<2>(C, smem, max_dynamic) : bottom_clusters<4>(C, smem, max_dynamic)) < 1)
        return false;
    h->bot_C = C;
    h->bot_P = P;
    h->bot_rows = rows;
    h->bot_smem = smem;
    h->bot_state = 1;
    return true;
}

static float sched_weight_precond(int n, int it) {
    // muCyclePreconditioner's get_scheduled_weight (simd_vdb_poisson.cpp:1848-1866)
    if (it >= n) return 6.0f / 7.0f;
    if (n == 1) return 6.0f / 7.0f;
    if (n == 2) { const float w[2] = {1.7319f, 0.5695f}; return w[it]; }
    const float w[3] = {2.2473f, 0.8571f, 0.5296f};
    return w[it];
}
static float sched_weight_iter(int n, int it) {
    // muCycleIterative's get_scheduled_weight (simd_vdb_poisson.cpp:1983-2000)
    if (it >= n) return 6.0f / 7.0f;
    if (n == 2) { const float w[2] = {1.7319f, 0.5695f}; return w[it]; }
    if (n >= 3) { const float w[3] = {2.2473f, 0.8571f, 0.5296f}; return w[it]; }
    return 6.0f / 7.0f;
}

}  // namespace

// The materialised z.r for a one-level hierarchy (the coarsest solve is the
// whole preconditioner, so no sweep is available to carry the dot).
__global__ void __launch_bounds__(128) k_dot_rho(DLevel L, const float* z, const float* r, double* partials,
                                                 PcgState* st) {
    griddep_wait();
    griddep_launch();
    dot_rho_leaf(L, blockIdx.x, gridDim.x, z, r, partials, st);
}

// muCyclePreconditioner<2, skip_first> (simd_vdb_poisson.cpp:1844-1977) at
// level l: lhs <- M^-1 rhs.  Fusions (bit-identical to the unfused sequence):
// first sweep from zero + second sweep; residual + restriction;
// prolongation-add + first post-smoothing sweep; z.r into the last level-0
// sweep.  The W-cycle's second visit of the coarsest level re-solves the same
// system from a zero guess, so it is skipped.
static void enqueue_precond(Enq& E, int l, float* lhs, const float* rhs, bool skip_first, DotOut dot) {
    uaamg_poisson* h = E.h;
    LevelDev& D = h->lv[l];
    const int n = 3;
    const int sm = h->smoother;
    if (l == h->nlev - 1) {
        E.coarsest(rhs, lhs);
        if (dot.r) {
            E.pb("L0 dot");
            launch(k_dot_rho, (unsigned)D.L.nl, 128, E.s, D.L, (const float*)lhs, dot.r, dot.partials, dot.st);
            E.pe();
            E.count++;
        }
        return;
    }
    float* T = D.tmp;
    LevelDev& P = h->lv[l + 1];
    auto wpre = [&](int i) { return sm == UAAMG_SMOOTHER_WEIGHTED_JACOBI ? 6.0f / 7.0f : sched_weight_precond(n, i); };
    float* cur = nullptr;
    if (sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL) {
        int i0 = 0;
        if (skip_first) {
            E.sweep<M_BLACK>(l, SrcFirstRbgs{rhs, D.w_sor, 1}, rhs, lhs, 0.f);
            i0 = 1;
        }
        for (int i = i0; i < n; ++i) {
            E.sweep<M_RED>(l, SrcPlain{lhs}, rhs, lhs, 0.f);
            E.sweep<M_BLACK>(l, SrcPlain{lhs}, rhs, lhs, 0.f);
        }
        cur = lhs;
        E.restrict_resid(l, cur, rhs);
        enqueue_precond(E, l + 1, P.lhs, P.rhs, true, DotOut{nullptr, nullptr, nullptr});
        if (l + 1 != h->nlev - 1) enqueue_precond(E, l + 1, P.lhs, P.rhs, false, DotOut{nullptr, nullptr, nullptr});
        // post: (black, red) x n; the first black pass adds the prolongation,
        // writes T; the last red pass writes back into lhs
        if (E.split(l)) {
            E.materialize(l, SrcProlong{lhs, P.lhs, 1.0f}, lhs);
            E.sweep<M_BLACK>(l, SrcPlain{lhs}, rhs, T, 0.f);
        } else {
            E.sweep<M_BLACK>(l, SrcProlong{lhs, P.lhs, 1.0f}, rhs, T, 0.f);
        }
        for (int i = 0; i < n; ++i) {
            if (i > 0) E.sweep<M_BLACK>(l, SrcPlain{T}, rhs, T, 0.f);
            if (i < n - 1) E.sweep<M_RED>(l, SrcPlain{T}, rhs, T, 0.f);
            else E.sweep<M_RED>(l, SrcPlain{T}, rhs, lhs, 0.f, dot);
        }
        return;
    }
    const bool spai = (sm == UAAMG_SMOOTHER_SPAI0);
    // pre-smoothing, ends in T
    if (skip_first) {
        if (E.split(l)) {  // T is free until the second sweep writes it
            if (spai) E.materialize(l, SrcFirstSpai0{rhs, D.spai0_ready}, T);
            else E.materialize(l, SrcFirstJacobi{rhs, wpre(0)}, T);
            if (spai) E.sweep<M_SPAI0>(l, SrcPlain{T}, rhs, lhs, 0.f);
            else E.sweep<M_JACOBI>(l, SrcPlain{T}, rhs, lhs, wpre(1));
        } else if (spai) {
            E.sweep<M_SPAI0>(l, SrcFirstSpai0{rhs, D.spai0_ready}, rhs, lhs, 0.f);
        } else if (E.pair(l)) {  // first sweep from zero + second + third in one launch, into T
            E.sweep2(l, SrcFirstJacobi{rhs, wpre(0)}, rhs, T, wpre(1), wpre(2));
        } else {
            E.sweep<M_JACOBI>(l, SrcFirstJacobi{rhs, wpre(0)}, rhs, lhs, wpre(1));
        }
        if (spai) E.sweep<M_SPAI0>(l, SrcPlain{lhs}, rhs, T, 0.f, DotOut{nullptr, nullptr, nullptr}, true);
        else if (E.split(l) || !E.pair(l)) E.sweep<M_JACOBI>(l, SrcPlain{lhs}, rhs, T, wpre(2));
    } else {
        if (spai) {
            E.sweep<M_SPAI0>(l, SrcPlain{lhs}, rhs, T, 0.f, DotOut{nullptr, nullptr, nullptr}, true);
            E.sweep<M_SPAI0>(l, SrcPlain{T}, rhs, lhs, 0.f);
            E.sweep<M_SPAI0>(l, SrcPlain{lhs}, rhs, T, 0.f);
        } else if (E.pair(l)) {  // the first two sweeps in one launch through tmp2
            E.sweep2(l, SrcPlain{lhs}, rhs, D.tmp2, wpre(0), wpre(1));
            E.sweep<M_JACOBI>(l, SrcPlain{D.tmp2}, rhs, T, wpre(2));
        } else {
            E.sweep<M_JACOBI>(l, SrcPlain{lhs}, rhs, T, wpre(0));
            E.sweep<M_JACOBI>(l, SrcPlain{T}, rhs, lhs, wpre(1));
            E.sweep<M_JACOBI>(l, SrcPlain{lhs}, rhs, T, wpre(2));
        }
    }
    cur = T;
    E.restrict_resid(l, cur, rhs);
    if (l + 1 == h->nlev - 2 && use_bottom(h)) {
        const float w[3] = {wpre(0), wpre(1), wpre(2)};
        E.bottom(l + 1, P.lhs, P.rhs, w);
    } else {
        enqueue_precond(E, l + 1, P.lhs, P.rhs, true, DotOut{nullptr, nullptr, nullptr});
        if (l + 1 != h->nlev - 1) enqueue_precond(E, l + 1, P.lhs, P.rhs, false, DotOut{nullptr, nullptr, nullptr});
    }
    // post-smoothing with reversed weights: T(+P x_c) -> lhs -> T -> lhs
    if (E.split(l)) {  // T += P x_c in place (T is not read again before it is rewritten)
        E.materialize(l, SrcProlong{T, P.lhs, 1.0f}, T);
        if (spai) {
            E.sweep<M_SPAI0>(l, SrcPlain{T}, rhs, lhs, 0.f);
            E.sweep<M_SPAI0>(l, SrcPlain{lhs}, rhs, T, 0.f);
            E.sweep<M_SPAI0>(l, SrcPlain{T}, rhs, lhs, 0.f, dot);
        } else {
            E.sweep<M_JACOBI>(l, SrcPlain{T}, rhs, lhs, wpre(2));
            E.sweep<M_JACOBI>(l, SrcPlain{lhs}, rhs, T, wpre(1));
            E.sweep<M_JACOBI>(l, SrcPlain{T}, rhs, lhs, wpre(0), dot);
        }
        return;
    }
    if (spai) {
        E.sweep<M_SPAI0>(l, SrcProlong{T, P.lhs, 1.0f}, rhs, lhs, 0.f);
        E.sweep<M_SPAI0>(l, SrcPlain{lhs}, rhs, T, 0.f);
        E.sweep<M_SPAI0>(l, SrcPlain{T}, rhs, lhs, 0.f, dot);
    } else if (E.pair(l)) {  // prolongation + the first two sweeps in one launch through tmp2
        E.sweep2(l, SrcProlong{T, P.lhs, 1.0f}, rhs, D.tmp2, wpre(2), wpre(1));
        E.sweep<M_JACOBI>(l, SrcPlain{D.tmp2}, rhs, lhs, wpre(0), dot);
    } else {
        E.sweep<M_JACOBI>(l, SrcProlong{T, P.lhs, 1.0f}, rhs, lhs, wpre(2));
        E.sweep<M_JACOBI>(l, SrcPlain{lhs}, rhs, T, wpre(1));
        E.sweep<M_JACOBI>(l, SrcPlain{T}, rhs, lhs, wpre(0), dot);
    }
}

static int graph_key(const uaamg_poisson* h);

// muCycleIterative<2> (simd_vdb_poisson.cpp:1979-2110): the MG-as-solver
// cycle; coarse levels start from whatever their lhs holds, as in the reference.
static void enqueue_mg_cycle(Enq& E, int l, float* lhs, const float* rhs) {
    uaamg_poisson* h = E.h;
    LevelDev& D = h->lv[l];
    const int n = 3;
    const int sm = h->smoother;
    float* T = D.tmp;
    auto w = [&](int i) { return sm == UAAMG_SMOOTHER_WEIGHTED_JACOBI ? 6.0f / 7.0f : sched_weight_iter(n, i); };
    if (sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL) D.w_sor = 1.0f;
    auto smooth = [&](int i, int red_first, float*& cur, float*& oth) {
        if (sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL) {
            if (red_first) { E.sweep<M_RED>(l, SrcPlain{cur}, rhs, cur, 0.f); E.sweep<M_BLACK>(l, SrcPlain{cur}, rhs, cur, 0.f); }
            else { E.sweep<M_BLACK>(l, SrcPlain{cur}, rhs, cur, 0.f); E.sweep<M_RED>(l, SrcPlain{cur}, rhs, cur, 0.f); }
        } else if (sm == UAAMG_SMOOTHER_SPAI0) {
            E.sweep<M_SPAI0>(l, SrcPlain{cur}, rhs, oth, 0.f, DotOut{nullptr, nullptr, nullptr}, true);
            std::swap(cur, oth);
        } else {
            E.sweep<M_JACOBI>(l, SrcPlain{cur}, rhs, oth, w(i));
            std::swap(cur, oth);
        }
    };
    float* cur = lhs;
    float* oth = T;
    if (l == h->nlev - 1) {
        for (int i = 0; i < 10 * n; ++i) smooth(i, 1, cur, oth);
        if (cur != lhs) { CK(cudaMemcpyAsync(lhs, cur, (size_t)D.L.nl * UAAMG_LEAF * 4, cudaMemcpyDeviceToDevice, E.s)); }
        return;
    }
    for (int i = 0; i < n; ++i) smooth(i, 1, cur, oth);
    LevelDev& P = h->lv[l + 1];
    E.restrict_resid(l, cur, rhs);
    for (int mu = 0; mu < 2; ++mu) enqueue_mg_cycle(E, l + 1, P.lhs, P.rhs);
    // prolongation (alpha 0.5) + post-smoothing
    if (sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL) {
        launch(k_materialize<SrcProlong>, (unsigned)D.L.nl, 128, E.s, D.L, SrcProlong{cur, P.lhs, 0.5f}, oth);
        E.count++;
        std::swap(cur, oth);
        for (int i = 0; i < n; ++i) smooth(n - 1 - i, 0, cur, oth);
    } else {
        if (sm == UAAMG_SMOOTHER_SPAI0) E.sweep<M_SPAI0>(l, SrcProlong{cur, P.lhs, 0.5f}, rhs, oth, 0.f);
        else E.sweep<M_JACOBI>(l, SrcProlong{cur, P.lhs, 0.5f}, rhs, oth, w(n - 1));
        std::swap(cur, oth);
        for (int i = 1; i < n; ++i) smooth(n - 1 - i, 0, cur, oth);
    }
    if (cur != lhs) CK(cudaMemcpyAsync(lhs, cur, (size_t)D.L.nl * UAAMG_LEAF * 4, cudaMemcpyDeviceToDevice, E.s));
}

// ---------------------------------------------------------------------------
// PCG (PoissonSolver::solveMultigridPCG, simd_vdb_poisson.cpp:2155-2226), loop
// rotated so that the convergence test ends the iteration:
//   setup:  r = b - A x, nu0, numax                        [k_pcg_init]
//   while running:
//     z = M^-1 r, rho_new = z.r, beta, rho                 [W-cycle]
//     x += alpha_prev p (not in the first pass); p = z + beta p
//     q = A p, sigma, alpha = rho / sigma
//     r -= alpha q, nu, convergence / divergence test
//   finish: x += alpha p when converged or out of iterations
static void enqueue_setup(Enq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_poisson* h = E.h;
    LevelDev& D0 = h->lv[0];
    const size_t n0 = (size_t)D0.L.nl * UAAMG_LEAF;
    enq_memset(h->p, 0, n0 * 4, E.s);
    E.pb("L0 mask inputs");
    launch(k_mask_vec, (unsigned)D0.L.nl, 128, E.s, D0.L, h->x);
    launch(k_mask_vec, (unsigned)D0.L.nl, 128, E.s, D0.L, h->b);
    E.pe();
    E.pb("L0 pcg init (residual+absmax)");
    launch(k_pcg_init, (unsigned)D0.L.nl, 128, E.s, D0.L, (const float*)h->x, (const float*)h->b, h->r, h->partials,
           h->st, cond, use_cond);
    E.pe();
    E.count += 3;
}
// PCG lines 6-7: q = A p with sigma = p.q and alpha (pipelined staged kernel
// on large levels)
static void enqueue_Ap(Enq& E) {
    uaamg_poisson* h = E.h;
    LevelDev& D0 = h->lv[0];
    if (g_use_staged && D0.L.nl >= PIPE_DOT_MIN_LEAVES)
        launch_pipe(k_pipe<M_LAPLACIAN, DLevel, float, false, 1>, D0.L.nl, pipe_smem_bytes<DLevel>(), E.s, D0.L,
                    (const float*)h->p, (const float*)nullptr, h->q, 0.f, 0.f, 0.f,
                    DotOut{h->p, h->partials, h->st}, (const float*)nullptr, 0.f, &h->st->error);
    else
        launch(k_pcg_Ap, (unsigned)D0.L.nl, 128, E.s, D0.L, (const float*)h->p, h->q, h->partials, h->st);
}
static void enqueue_body(Enq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_poisson* h = E.h;
    LevelDev& D0 = h->lv[0];
    enqueue_precond(E, 0, h->z, h->r, true, DotOut{h->r, h->partials, h->st});
    E.pb("L0 pcg x,p update");
    launch(k_pcg_update_p, (unsigned)D0.L.nl, 128, E.s, D0.L, (const float*)h->z, h->p, h->x, (const PcgState*)h->st);
    E.pe();
    E.pb("L0 pcg Ap+dot");
    enqueue_Ap(E);
    E.pe();
    E.pb("L0 pcg r update+absmax");
    launch(k_pcg_update_r, elem_grid(D0.L.nl), 128, E.s, D0.L, (const float*)h->q, h->r, h->partials, h->st, cond,
           use_cond);
    E.pe();
    E.count += 3;
}
static void enqueue_finish(Enq& E) {
    uaamg_poisson* h = E.h;
    LevelDev& D0 = h->lv[0];
    E.pb("L0 pcg finish");
    launch(k_pcg_finish, (unsigned)D0.L.nl, 128, E.s, D0.L, (const float*)h->p, h->x, (const PcgState*)h->st);
    E.pe();
    E.count += 1;
}

static int graph_key(const uaamg_poisson* h) {
    int k = h->smoother + 4 * g_tune_gen;
    for (int l = 0; l < h->nlev; ++l) k = k * 3 + (h->lv[l].w_sor == 1.2f ? 0 : 1);
    return k;
}

// ---------------------------------------------------------------------------
// Solve-graph cache of the process.  A FLIP-style caller creates a fresh
// hierarchy every substep, and a fresh handle's first solve runs host-driven
// (capturing a graph costs about what it saves).  When a new handle's
// recording (t_rec) equals the one a cached graph was captured from -- the same
// kernels, shapes and argument bytes, i.e. its buffers sit where a destroyed
// handle's did -- its first solve replays that graph.  A graph is captured
// for the cache only for a recording seen once before, so a stream of
// different hierarchies keeps the host-driven first solve.  The cache lives
// on the heap for the whole process (no destruction after the CUDA runtime).
struct SolveGraph {
    std::vector<unsigned char> sig;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    int64_t setup = 0, body = 0, finish = 0;
    ~SolveGraph() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};
struct SolveGraphCache {
    std::mutex mu;
    std::vector<std::shared_ptr<SolveGraph>> graphs;  // most recent first
    std::vector<uint64_t> seen;                       // recordings without a graph, most recent first
    int64_t hits = 0, captures = 0;
};
static SolveGraphCache& solve_graph_cache() {
    static SolveGraphCache* c = new SolveGraphCache();
    return *c;
}
static constexpr size_t SGC_GRAPHS = 4, SGC_SEEN = 16;
static bool g_solve_graph_cache = true;
static uint64_t fnv1a(const std::vector<unsigned char>& v) {
    uint64_t x = 1469598103934665603ull;
    for (unsigned char c : v) x = (x ^ c) * 1099511628211ull;
    return x;
}

// A recording's cached graph (hit), or whether to capture one for the cache:
// true on its second sighting.
static bool solve_graph_lookup(const std::vector<unsigned char>& sig, std::shared_ptr<SolveGraph>& hit) {
    const uint64_t hs = fnv1a(sig);
    SolveGraphCache& c = solve_graph_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    for (size_t i = 0; i < c.graphs.size(); ++i)
        if (c.graphs[i]->sig == sig) {
            hit = c.graphs[i];
            c.graphs.erase(c.graphs.begin() + (long)i);
            c.graphs.insert(c.graphs.begin(), hit);
            c.hits++;
            return false;
        }
    auto f = std::find(c.seen.begin(), c.seen.end(), hs);
    if (f != c.seen.end()) {
        c.seen.erase(f);
        return true;
    }
    c.seen.insert(c.seen.begin(), hs);
    if (c.seen.size() > SGC_SEEN) c.seen.pop_back();
    return false;
}
// Hands a just-captured graph to the cache (the handle keeps a reference).
static std::shared_ptr<SolveGraph> solve_graph_insert(std::vector<unsigned char> sig, cudaGraph_t g,
                                                      cudaGraphExec_t x, int64_t setup, int64_t body,
                                                      int64_t finish) {
    auto sg = std::make_shared<SolveGraph>();
    sg->sig = std::move(sig);
    sg->g = g;
    sg->x = x;
    sg->setup = setup;
    sg->body = body;
    sg->finish = finish;
    SolveGraphCache& c = solve_graph_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    c.graphs.insert(c.graphs.begin(), sg);
    if (c.graphs.size() > SGC_GRAPHS) c.graphs.pop_back();
    c.captures++;
    return sg;
}

static void destroy_graph(uaamg_poisson* h) {
    if (h->shared_graph) {
        h->shared_graph.reset();
    } else {
        if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
        if (h->graph) cudaGraphDestroy(h->graph);
    }
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->graph_key = -1;
}

static void build_graph(uaamg_poisson* h) {
    double trace_t0 = trace_now();
    destroy_graph(h);
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    Enq E{h, h->stream};
    CK(cudaStreamBeginCaptureToGraph(h->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_setup(E, cond, 1);
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
        Enq B{h, h->body_stream};
        CK(cudaStreamBeginCaptureToGraph(h->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        enqueue_body(B, cond, 1);
        cudaGraph_t bodyout = nullptr;
        CK(cudaStreamEndCapture(h->body_stream, &bodyout));
        h->body_launches = B.count;
        Enq F{h, h->stream};
        enqueue_finish(F);
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
    TRACE("solve graph captured");
    CK(cudaGraphInstantiate(&h->graph_exec, g, 0));
    TRACE("solve graph instantiated");
    h->graph = g;
    h->graph_key = graph_key(h);
}

// The recording of one PCG solve's enqueue (setup, body, finish) as the
// graph captures it.
static std::vector<unsigned char> record_solve(uaamg_poisson* h) {
    LaunchRec rec;
    rec.val((unsigned char)'P');
    rec.val(g_use_pdl);
    rec.val(h->ctx->device);
    t_rec = &rec;
    try {
        Enq E{h, h->stream};
        enqueue_setup(E, 0, 1);
        rec.val((unsigned char)'|');
        Enq B{h, h->body_stream};
        enqueue_body(B, 0, 1);
        rec.val((unsigned char)'|');
        Enq F{h, h->stream};
        enqueue_finish(F);
    } catch (...) {
        t_rec = nullptr;
        throw;
    }
    t_rec = nullptr;
    return std::move(rec.bytes);
}

static void init_state(uaamg_poisson* h) {
    PcgState s;
    memset(&s, 0, sizeof(s));
    s.tol = h->rel_tol;
    s.max_iter = h->max_iter;
    *h->st_host = s;
    CK(cudaMemcpyAsync(h->st, h->st_host, sizeof(PcgState), cudaMemcpyHostToDevice, h->stream));
}

// x, b (h->x, h->b) already on the device; returns status
static int run_pcg(uaamg_poisson* h) {
    if (h->lv[0].L.nl == 0 || h->lv[0].L.nl == 0) {
        h->iterations = 0;
        h->final_residual = 0.f;
        return UAAMG_SUCCESS;
    }
    if (h->smoother == UAAMG_SMOOTHER_SPAI0) ensure_spai0(h);
    init_state(h);
    int64_t launches = 0;
    // A handle's first solve runs host-driven: capturing and instantiating the
    // graph costs about as much as the launches it saves, and a FLIP substep
    // solves each hierarchy once.  Later solves on the handle use the graph.
    bool use_graph = h->use_graph && (h->use_graph == 2 || h->solves > 0);
    std::shared_ptr<SolveGraph> hit;
    std::vector<unsigned char> sig;
    bool share = false;
    if (!use_graph && h->use_graph == 1 && g_solve_graph_cache) {  // the cache may take this first solve
        sig = record_solve(h);
        share = solve_graph_lookup(sig, hit);
        use_graph = hit || share;
    }
    h->solves++;
    if (use_graph) {
        if (hit) {
            destroy_graph(h);
            h->shared_graph = hit;
            h->graph = hit->g;
            h->graph_exec = hit->x;
            h->graph_key = graph_key(h);
            h->setup_launches = hit->setup;
            h->body_launches = hit->body;
            h->finish_launches = hit->finish;
        } else if (!h->graph_exec || h->graph_key != graph_key(h)) {
            build_graph(h);
            if (share)
                h->shared_graph = solve_graph_insert(std::move(sig), h->graph, h->graph_exec, h->setup_launches,
                                                     h->body_launches, h->finish_launches);
        }
        CK(cudaGraphLaunch(h->graph_exec, h->stream));
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        int iters_run = h->st_host->iter;  // body executions
        launches = h->setup_launches + (int64_t)iters_run * h->body_launches + h->finish_launches;
    } else {
            Enq E{h, h->stream};
        enqueue_setup(E, 0, 0);
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        while (h->st_host->status == PCG_RUNNING) {
            enqueue_body(E, 0, 0);
            CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        enqueue_finish(E);
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
    return (s.status == PCG_SUCCESS) ? UAAMG_SUCCESS : UAAMG_FAILED;
}

// PoissonSolver::solvePureMultigrid (simd_vdb_poisson.cpp:2228-2267)
static int run_mg(uaamg_poisson* h) {
    LevelDev& D0 = h->lv[0];
    if (D0.L.nl == 0) { h->iterations = 0; h->final_residual = 0.f; return UAAMG_SUCCESS; }
    if (h->smoother == UAAMG_SMOOTHER_SPAI0) ensure_spai0(h);
    Enq E{h, h->stream};
    k_mask_vec<<<(unsigned)D0.L.nl, 128, 0, E.s>>>(D0.L, h->x);
    k_mask_vec<<<(unsigned)D0.L.nl, 128, 0, E.s>>>(D0.L, h->b);
    E.count += 2;
    auto resid_norm = [&]() {
        E.sweep<M_RESIDUAL>(0, SrcPlain{h->x}, h->b, h->r, 0.f);
        k_absmax<<<(unsigned)D0.L.nl, 128, 0, E.s>>>(D0.L, h->r, h->partials, &h->st->ticket[4], h->scalar_dev);
        CHECK_LAUNCH();
        E.count++;
        CK(cudaMemcpyAsync(h->scalar_host, h->scalar_dev, 4, cudaMemcpyDeviceToHost, E.s));
        CK(cudaStreamSynchronize(E.s));
        return h->scalar_host[0];
    };
    init_state(h);
    float nu = resid_norm();
    const float numax = h->rel_tol * nu;
    int it = 0, status = UAAMG_FAILED;
    if (nu <= numax) {
        status = UAAMG_SUCCESS;
    } else {
        float nu_old = nu;
        for (; it < h->max_iter; ++it) {
            enqueue_mg_cycle(E, 0, h->x, h->b);
            nu_old = nu;
            nu = resid_norm();
            if (nu <= numax) { status = UAAMG_SUCCESS; break; }
            if (nu > nu_old && it > 8) { status = UAAMG_FAILED; break; }
        }
    }
    h->iterations = it;
    h->final_residual = nu;
    h->last_launches = E.count;
    h->launches += E.count;
    return status;
}

// ---------------------------------------------------------------------------
// C ABI
#define ABI_BEGIN try {
#define ABI_END                                            \
    }                                                      \
    catch (const UaamgError& e) { return e.code; }         \
    catch (const std::bad_alloc&) {                        \
        set_error("host out of memory");                   \
        return UAAMG_ERR_OUT_OF_MEMORY;                    \
    }                                                      \
    catch (...) {                                          \
        set_error("unexpected exception");                 \
        return UAAMG_ERR_CUDA;                             \
    }

static void require(bool c, const char* msg) {
    if (!c) { set_error("%s", msg); throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT}; }
}
static size_t vec_bytes(const uaamg_poisson* h, int level) { return (size_t)h->lv[level].L.nl * UAAMG_LEAF * 4; }

extern "C" {

const char* uaamg_last_error(void) { return g_last_error.c_str(); }

int uaamg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int uaamg_poisson_create(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights, float dt, float dx,
                         uaamg_poisson** out) {
    return uaamg_poisson_create_on_stream(liquid_phi, face_weights, dt, dx, nullptr, out);
}

static void noalloc_resolve(uaamg_poisson* h);

static int create_impl(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights, float dt, float dx,
                       void* stream, const RhsInputs* ri, uaamg_poisson** out) {
    {
        const char* e = getenv("UAAMG_PDL");
        g_use_pdl = !(e && e[0] == '0');
        e = getenv("UAAMG_STAGED");
        g_use_staged = !(e && e[0] == '0');
        e = getenv("UAAMG_BOTTOM");
        g_use_bottom = !(e && e[0] == '0');
        e = getenv("UAAMG_SOLVE_GRAPH_CACHE");
        g_solve_graph_cache = !(e && e[0] == '0');
        e = getenv("UAAMG_SWEEP2");
        g_use_sweep2 = !(e && e[0] == '0');
    }
    if (!out) { set_error("out is NULL"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return UAAMG_ERR_NO_DEVICE;
    }
    uaamg_poisson* h = new (std::nothrow) uaamg_poisson();
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
        noalloc_resolve(h);
        h->bot_state = (g_use_bottom && g_tune.bottom_cycle) ? -1 : 0;
        h->use_sweep2 = g_use_sweep2;
        {
            int sms = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->ctx->device) == cudaSuccess && sms > 0)
                g_sms = sms;
        }
        build_hierarchy(h, liquid_phi, face_weights, dt, dx, ri);
    } catch (const UaamgError& e) {
        uaamg_poisson_destroy(h);
        return e.code;
    } catch (const std::bad_alloc&) {
        uaamg_poisson_destroy(h);
        set_error("host out of memory");
        return UAAMG_ERR_OUT_OF_MEMORY;
    }
    *out = h;
    return UAAMG_SUCCESS;
}

int uaamg_poisson_create_on_stream(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights, float dt,
                                   float dx, void* stream, uaamg_poisson** out) {
    return create_impl(liquid_phi, face_weights, dt, dx, stream, nullptr, out);
}

int uaamg_poisson_create_with_rhs(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights,
                                  const uaamg_leaf_grid* vx, const uaamg_leaf_grid* vy, const uaamg_leaf_grid* vz,
                                  const uaamg_leaf_grid* solid_velocity, float dt, float dx, void* stream,
                                  uaamg_poisson** out) {
    RhsInputs ri{vx, vy, vz, solid_velocity};
    return create_impl(liquid_phi, face_weights, dt, dx, stream, &ri, out);
}

static void mixed_free(uaamg_poisson* h);

int uaamg_poisson_destroy(uaamg_poisson* h) {
    if (!h) return UAAMG_SUCCESS;
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroy_graph(h);
    if (h->ctx) mixed_free(h);
    if (h->ctx) {
        if (h->dmem) cudaFreeAsync(h->dmem, h->stream);
        if (h->dmem2) cudaFreeAsync(h->dmem2, h->stream);
        if (h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
        ctx_pinned_release(h->ctx, h->pin_state, h->pin_state_cap);
        ctx_pinned_release(h->ctx, h->pin_stage, h->pin_stage_cap);
        ctx_pinned_release(h->ctx, h->pin_stage2, h->pin_stage2_cap);
        ctx_pinned_release(h->ctx, h->pin_in, h->pin_in_cap);
        ctx_stream_release(h->ctx, h->body_stream);
        ctx_stream_release(h->ctx, h->own_stream);
    }
    delete h;
    return UAAMG_SUCCESS;
}

int uaamg_poisson_set_smoother(uaamg_poisson* h, int smoother) {
    if (!h || smoother < 0 || smoother > 3) { set_error("invalid smoother"); return UAAMG_ERR_INVALID_ARGUMENT; }
    h->smoother = smoother;
    return UAAMG_SUCCESS;
}
int uaamg_poisson_set_max_iterations(uaamg_poisson* h, int m) {
    if (!h) { set_error("NULL handle"); return UAAMG_ERR_INVALID_ARGUMENT; }
    h->max_iter = m;
    return UAAMG_SUCCESS;
}
int uaamg_poisson_set_relative_tolerance(uaamg_poisson* h, float t) {
    if (!h) { set_error("NULL handle"); return UAAMG_ERR_INVALID_ARGUMENT; }
    h->rel_tol = t;
    return UAAMG_SUCCESS;
}
int uaamg_poisson_iterations(const uaamg_poisson* h) { return h ? h->iterations : 0; }
float uaamg_poisson_final_residual(const uaamg_poisson* h) { return h ? h->final_residual : 0.f; }
int uaamg_poisson_num_levels(const uaamg_poisson* h) { return h ? h->nlev : 0; }
int64_t uaamg_poisson_num_dof(const uaamg_poisson* h, int level) {
    if (!h || level < 0 || level >= (int)h->host.size()) return -1;
    return h->host[level].ndof;
}
int64_t uaamg_poisson_leaf_count(const uaamg_poisson* h, int level) {
    if (!h || level < 0 || level >= (int)h->host.size()) return -1;
    return h->host[level].nl;
}
int uaamg_poisson_dof_topology(const uaamg_poisson* h, int level, int32_t* origins, uint64_t* masks) {
    if (!h || level < 0 || level >= (int)h->host.size()) { set_error("invalid level"); return UAAMG_ERR_INVALID_ARGUMENT; }
    const HostLevel& H = h->host[level];
    if (origins && H.nl) memcpy(origins, H.org.data(), (size_t)H.nl * 12);
    if (masks && H.nl) memcpy(masks, H.mask.data(), (size_t)H.nl * 64);
    return UAAMG_SUCCESS;
}
int uaamg_poisson_dof_index(const uaamg_poisson* h, int level, int32_t* out) {
    if (!h || !out || level < 0 || level >= (int)h->host.size()) { set_error("invalid argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    const HostLevel& H = h->host[level];
    for (int i = 0; i < H.nl; ++i) {
        int32_t d = H.dof_base[i];
        for (int off = 0; off < UAAMG_LEAF; ++off)
            out[(size_t)i * UAAMG_LEAF + off] = ((H.mask[8 * i + (off >> 6)] >> (off & 63)) & 1ull) ? d++ : -1;
    }
    return UAAMG_SUCCESS;
}

static int build_rhs_impl(uaamg_poisson* h, const uaamg_leaf_grid* fw, const uaamg_leaf_grid* vx,
                          const uaamg_leaf_grid* vy, const uaamg_leaf_grid* vz, const uaamg_leaf_grid* sv, float dt,
                          float* d_out) {
    (void)dt;  // the reference's BuildPoissonRhs carries dt but does not use it (.cpp:84-86)
    check_grid(fw, 3, "face_weights");
    check_grid(vx, 1, "vx");
    check_grid(vy, 1, "vy");
    check_grid(vz, 1, "vz");
    check_grid(sv, 3, "solid_velocity");
    LevelDev& D0 = h->lv[0];
    if (D0.L.nl == 0) return UAAMG_SUCCESS;
    std::vector<void*> tofree;
    HostMap m0, m1, m2, m3, m4;
    DevGrid g0, g1, g2, g3, g4;
    upload_grid(h, fw, g0, m0, tofree);
    upload_grid(h, vx, g1, m1, tofree);
    upload_grid(h, vy, g2, m2, tofree);
    upload_grid(h, vz, g3, m3, tofree);
    upload_grid(h, sv, g4, m4, tofree);
    float invdx = 1.0f / D0.dx;
    k_build_rhs<<<(unsigned)D0.L.nl, 128, 0, h->stream>>>(D0.L.mask, D0.org, g0.g, g1.g, g2.g, g3.g, g4.g, invdx, d_out);
    CHECK_LAUNCH();
    h->launches++;
    for (void* p : tofree) CK(cudaFreeAsync(p, h->stream));
    return UAAMG_SUCCESS;
}

int uaamg_poisson_build_rhs(uaamg_poisson* h, const uaamg_leaf_grid* fw, const uaamg_leaf_grid* vx,
                            const uaamg_leaf_grid* vy, const uaamg_leaf_grid* vz, const uaamg_leaf_grid* sv, float dt,
                            float* rhs_out) {
    ABI_BEGIN
    require(h && rhs_out, "NULL argument");
    int rc = build_rhs_impl(h, fw, vx, vy, vz, sv, dt, h->b);
    if (rc) return rc;
    CK(cudaMemcpyAsync(rhs_out, h->b, vec_bytes(h, 0), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}
int uaamg_poisson_build_rhs_device(uaamg_poisson* h, const uaamg_leaf_grid* fw, const uaamg_leaf_grid* vx,
                                   const uaamg_leaf_grid* vy, const uaamg_leaf_grid* vz, const uaamg_leaf_grid* sv,
                                   float dt, float* d_rhs_out) {
    ABI_BEGIN
    require(h && d_rhs_out, "NULL argument");
    return build_rhs_impl(h, fw, vx, vy, vz, sv, dt, d_rhs_out);
    ABI_END
}

int uaamg_poisson_solve_pcg(uaamg_poisson* h, float* pressure, const float* rhs, int* iterations) {
    ABI_BEGIN
    require(h && pressure && rhs, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemcpyAsync(h->x, pressure, nb, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->b, rhs, nb, cudaMemcpyHostToDevice, h->stream));
    }
    int st = run_pcg(h);
    if (nb) {
        CK(cudaMemcpyAsync(pressure, h->x, nb, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}
int uaamg_poisson_solve_pcg_device(uaamg_poisson* h, float* d_pressure, const float* d_rhs, int* iterations) {
    ABI_BEGIN
    require(h && d_pressure && d_rhs, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        if (d_pressure != h->x) CK(cudaMemcpyAsync(h->x, d_pressure, nb, cudaMemcpyDeviceToDevice, h->stream));
        if (d_rhs != h->b) CK(cudaMemcpyAsync(h->b, d_rhs, nb, cudaMemcpyDeviceToDevice, h->stream));
    }
    int st = run_pcg(h);
    if (nb && d_pressure != h->x) {
        CK(cudaMemcpyAsync(d_pressure, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}
int uaamg_poisson_solve_mg(uaamg_poisson* h, float* pressure, const float* rhs, int* iterations) {
    ABI_BEGIN
    require(h && pressure && rhs, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemcpyAsync(h->x, pressure, nb, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->b, rhs, nb, cudaMemcpyHostToDevice, h->stream));
    }
    int st = run_mg(h);
    if (nb) {
        CK(cudaMemcpyAsync(pressure, h->x, nb, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}
int uaamg_poisson_solve_mg_device(uaamg_poisson* h, float* d_pressure, const float* d_rhs, int* iterations) {
    ABI_BEGIN
    require(h && d_pressure && d_rhs, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemcpyAsync(h->x, d_pressure, nb, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->b, d_rhs, nb, cudaMemcpyDeviceToDevice, h->stream));
    }
    int st = run_mg(h);
    if (nb) {
        CK(cudaMemcpyAsync(d_pressure, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}

// Solves from a zero pressure with the rhs built by uaamg_poisson_create_with_rhs.
static int solve_resident(uaamg_poisson* h, float* pressure, int* iterations, bool on_device, bool mg) {
    require(h && pressure, "NULL argument");
    if (!h->rhs_resident) {
        set_error("the handle holds no right-hand side (create it with uaamg_poisson_create_with_rhs)");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemsetAsync(h->x, 0, nb, h->stream));
        CK(cudaMemcpyAsync(h->b, h->rhs0, nb, cudaMemcpyDeviceToDevice, h->stream));
    }
    int st = mg ? run_mg(h) : run_pcg(h);
    if (nb) {
        CK(cudaMemcpyAsync(pressure, h->x, nb, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
}
int uaamg_poisson_solve_pcg_resident(uaamg_poisson* h, float* pressure, int* iterations) {
    ABI_BEGIN
    return solve_resident(h, pressure, iterations, false, false);
    ABI_END
}
int uaamg_poisson_solve_pcg_resident_device(uaamg_poisson* h, float* d_pressure, int* iterations) {
    ABI_BEGIN
    return solve_resident(h, d_pressure, iterations, true, false);
    ABI_END
}
int uaamg_poisson_solve_mg_resident(uaamg_poisson* h, float* pressure, int* iterations) {
    ABI_BEGIN
    return solve_resident(h, pressure, iterations, false, true);
    ABI_END
}
int uaamg_poisson_copy_rhs(uaamg_poisson* h, float* rhs_out) {
    ABI_BEGIN
    require(h && rhs_out, "NULL argument");
    if (!h->rhs_resident) {
        set_error("the handle holds no right-hand side (create it with uaamg_poisson_create_with_rhs)");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemcpyAsync(rhs_out, h->rhs0, nb, cudaMemcpyDefault, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return UAAMG_SUCCESS;
    ABI_END
}

// ---- per-level operators (host pointers); scratch = the level's lhs/rhs/tmp
// buffers are NOT used so the multigrid state is not disturbed
struct Scratch {
    float* a = nullptr;
    float* b = nullptr;
    float* c = nullptr;
    cudaStream_t s;
    Scratch(size_t bytes, cudaStream_t st) : s(st) {
        cudaError_t ce = cudaSuccess;
        DeviceCtx* dc = device_ctx(&ce);
        CK(ce);
        CK(ctx_dev_alloc(dc, (void**)&a, std::max<size_t>(bytes, 16) * 3, s));
        b = a + std::max<size_t>(bytes, 16) / 4;
        c = b + std::max<size_t>(bytes, 16) / 4;
    }
    ~Scratch() { cudaFreeAsync(a, s); }
};

static void check_level(const uaamg_poisson* h, int level) {
    require(h != nullptr, "NULL handle");
    require(level >= 0 && level < h->nlev, "invalid level");
}

int uaamg_poisson_level_apply(uaamg_poisson* h, int level, int mode, float weight, float w_sor, const float* lhs,
                              const float* rhs, float* out) {
    ABI_BEGIN
    check_level(h, level);
    require(lhs && out && mode >= 0 && mode <= 5, "invalid argument");
    if (mode == UAAMG_MODE_SPAI0) ensure_spai0(h);
    size_t nb = vec_bytes(h, level);
    if (!nb) return UAAMG_SUCCESS;
    Scratch S(nb, h->stream);
    CK(cudaMemcpyAsync(S.a, lhs, nb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(S.b, rhs ? rhs : lhs, nb, cudaMemcpyHostToDevice, h->stream));
    LevelDev& D = h->lv[level];
    float save = D.w_sor;
    D.w_sor = w_sor;
    Enq E{h, h->stream};
    switch (mode) {
        case UAAMG_MODE_WEIGHTED_JACOBI: E.sweep<M_JACOBI>(level, SrcPlain{S.a}, S.b, S.c, weight); break;
        case UAAMG_MODE_RESIDUAL: E.sweep<M_RESIDUAL>(level, SrcPlain{S.a}, S.b, S.c, weight); break;
        case UAAMG_MODE_LAPLACIAN: E.sweep<M_LAPLACIAN>(level, SrcPlain{S.a}, S.b, S.c, weight); break;
        case UAAMG_MODE_RED_GS: E.sweep<M_RED>(level, SrcPlain{S.a}, S.b, S.a, weight); break;
        case UAAMG_MODE_BLACK_GS: E.sweep<M_BLACK>(level, SrcPlain{S.a}, S.b, S.a, weight); break;
        default: E.sweep<M_SPAI0>(level, SrcPlain{S.a}, S.b, S.c, weight, DotOut{nullptr, nullptr, nullptr}, true); break;
    }
    D.w_sor = save;
    float* res = (mode == UAAMG_MODE_RED_GS || mode == UAAMG_MODE_BLACK_GS) ? S.a : S.c;
    CK(cudaMemcpyAsync(out, res, nb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_level_first_sweep(uaamg_poisson* h, int level, int kind, float weight, float w_sor, const float* rhs,
                                    float* out) {
    ABI_BEGIN
    check_level(h, level);
    require(rhs && out && kind >= 0 && kind <= 2, "invalid argument");
    if (kind == 1) ensure_spai0(h);
    size_t nb = vec_bytes(h, level);
    if (!nb) return UAAMG_SUCCESS;
    Scratch S(nb, h->stream);
    CK(cudaMemcpyAsync(S.b, rhs, nb, cudaMemcpyHostToDevice, h->stream));
    LevelDev& D = h->lv[level];
    cudaStream_t s = h->stream;
    if (kind == 0) {
        k_materialize<SrcFirstJacobi><<<(unsigned)D.L.nl, 128, 0, s>>>(D.L, SrcFirstJacobi{S.b, weight}, S.c);
    } else if (kind == 1) {
        k_materialize<SrcFirstSpai0><<<(unsigned)D.L.nl, 128, 0, s>>>(D.L, SrcFirstSpai0{S.b, D.spai0_ready}, S.c);
    } else {
        float save = D.w_sor;
        D.w_sor = w_sor;
        Enq E{h, s};
        E.sweep<M_BLACK>(level, SrcFirstRbgs{S.b, w_sor, 1}, S.b, S.c, 0.f);
        D.w_sor = save;
    }
    CHECK_LAUNCH();
    CK(cudaMemcpyAsync(out, S.c, nb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_level_restrict(uaamg_poisson* h, int fine_level, const float* fine, float* coarse) {
    ABI_BEGIN
    check_level(h, fine_level);
    require(fine_level + 1 < h->nlev && fine && coarse, "invalid argument");
    size_t nf = vec_bytes(h, fine_level), nc = vec_bytes(h, fine_level + 1);
    Scratch S(std::max(nf, nc), h->stream);
    CK(cudaMemcpyAsync(S.a, fine, nf, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(S.c, 0, nc, h->stream));
    LevelDev& D = h->lv[fine_level];
    k_restrict<false><<<(unsigned)D.L.nl, 128, 0, h->stream>>>(D.L, S.a, nullptr, S.c);
    CHECK_LAUNCH();
    CK(cudaMemcpyAsync(coarse, S.c, nc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_level_prolongate(uaamg_poisson* h, int fine_level, const float* coarse, float* fine, float alpha) {
    ABI_BEGIN
    check_level(h, fine_level);
    require(fine_level + 1 < h->nlev && fine && coarse, "invalid argument");
    size_t nf = vec_bytes(h, fine_level), nc = vec_bytes(h, fine_level + 1);
    Scratch S(std::max(nf, nc), h->stream);
    CK(cudaMemcpyAsync(S.a, fine, nf, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(S.b, coarse, nc, cudaMemcpyHostToDevice, h->stream));
    LevelDev& D = h->lv[fine_level];
    k_materialize<SrcProlong><<<(unsigned)D.L.nl, 128, 0, h->stream>>>(D.L, SrcProlong{S.a, S.b, alpha}, S.c);
    CHECK_LAUNCH();
    CK(cudaMemcpyAsync(fine, S.c, nf, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_level_coefficients(const uaamg_poisson* h, int level, float* diag, float* cx, float* cy, float* cz,
                                     uint8_t* flags) {
    ABI_BEGIN
    check_level(h, level);
    const LevelDev& D = h->lv[level];
    size_t nb = (size_t)D.L.nl * UAAMG_LEAF * 4;
    if (!nb) return UAAMG_SUCCESS;
    if (diag) CK(cudaMemcpyAsync(diag, D.L.diag, nb, cudaMemcpyDeviceToHost, h->stream));
    if (cx) CK(cudaMemcpyAsync(cx, D.L.cx, nb, cudaMemcpyDeviceToHost, h->stream));
    if (cy) CK(cudaMemcpyAsync(cy, D.L.cy, nb, cudaMemcpyDeviceToHost, h->stream));
    if (cz) CK(cudaMemcpyAsync(cz, D.L.cz, nb, cudaMemcpyDeviceToHost, h->stream));
    std::vector<uint32_t> f(D.L.nl);
    CK(cudaMemcpyAsync(f.data(), D.flags, (size_t)D.L.nl * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (flags)
        for (int i = 0; i < D.L.nl; ++i) flags[i] = (uint8_t)(f[i] & 15u);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_coarsest_solve(uaamg_poisson* h, const float* rhs, float* out) {
    ABI_BEGIN
    require(h && rhs && out, "NULL argument");
    int l = h->nlev - 1;
    size_t nb = vec_bytes(h, l);
    if (!nb) return UAAMG_SUCCESS;
    Scratch S(nb, h->stream);
    CK(cudaMemcpyAsync(S.a, rhs, nb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(S.c, 0, nb, h->stream));
    Enq E{h, h->stream};
    E.coarsest(S.a, S.c);
    CK(cudaMemcpyAsync(out, S.c, nb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_precondition(uaamg_poisson* h, const float* r, float* z) {
    ABI_BEGIN
    require(h && r && z, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    if (!nb) return UAAMG_SUCCESS;
    if (h->smoother == UAAMG_SMOOTHER_SPAI0) ensure_spai0(h);
    Scratch S(nb, h->stream);
    CK(cudaMemcpyAsync(S.b, r, nb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(S.a, 0, nb, h->stream));
    Enq E{h, h->stream};
    enqueue_precond(E, 0, S.a, S.b, true, DotOut{nullptr, nullptr, nullptr});
    CK(cudaMemcpyAsync(z, S.a, nb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_residual_norm_device(uaamg_poisson* h, const float* d_x, const float* d_b, float* d_r,
                                       float* d_norm) {
    ABI_BEGIN
    require(h && d_x && d_b && d_r && d_norm, "NULL argument");
    LevelDev& D0 = h->lv[0];
    if (D0.L.nl == 0) {
        CK(cudaMemsetAsync(d_norm, 0, sizeof(float), h->stream));
        return UAAMG_SUCCESS;
    }
    launch(k_residual_absmax, (unsigned)D0.L.nl, 128, h->stream, D0.L, d_x, d_b, d_r, h->partials,
           &h->st->ticket[5], d_norm);
    h->launches++;
    return UAAMG_SUCCESS;
    ABI_END
}

// ---------------------------------------------------------------------------
// Allocation-free variant of uaamg_poisson_residual_norm_device.  Its reduction
// scratch (a reduction buffer over up to UAAMG_NOALLOC_MAX_LEAVES level-0
// leaves, then the finishing ticket) lives in this file-scope array, which
// every GPU that loads the library holds until the process exits; the call
// itself allocates nothing.
#define UAAMG_NOALLOC_MAX_LEAVES 262144
#define UAAMG_NOALLOC_RED_DOUBLES (RED_HEADER + UAAMG_NOALLOC_MAX_LEAVES + RED_TICKETS)
static __device__ __align__(256) unsigned char g_noalloc_scratch[(UAAMG_NOALLOC_RED_DOUBLES + 32) * sizeof(double)];

// The array's device address on the handle's device, looked up when the handle
// is created (its device is current then).  Host code may not use the symbol
// itself: it names a host-side stand-in, not device memory.  Keeping the
// address in the handle ties it to the context the handle lives in.
static void noalloc_resolve(uaamg_poisson* h) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    h->noalloc_scratch = p;
}

// Level-0 leaf limit of the allocation-free variant; a test may lower it
// through UAAMG_NOALLOC_TEST_MAX_LEAVES to reach the rejection path on a small
// domain (it can only be lowered).
static int noalloc_max_leaves() {
    const char* e = getenv("UAAMG_NOALLOC_TEST_MAX_LEAVES");
    if (e && e[0]) {
        long v = strtol(e, nullptr, 10);
        if (v >= 0 && v < UAAMG_NOALLOC_MAX_LEAVES) return (int)v;
    }
    return UAAMG_NOALLOC_MAX_LEAVES;
}

int uaamg_poisson_residual_norm_noalloc(uaamg_poisson* h, const float* d_x, const float* d_b, float* d_r,
                                        float* d_norm) {
    ABI_BEGIN
    require(h && d_x && d_b && d_r && d_norm, "NULL argument");
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != h->ctx->device || !h->noalloc_scratch) {
        set_error("uaamg_poisson_residual_norm_noalloc: the handle lives on device %d but device %d is current",
                  h->ctx->device, cur);
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    LevelDev& D0 = h->lv[0];
    const int maxl = noalloc_max_leaves();
    if (D0.L.nl > maxl) {
        set_error("uaamg_poisson_residual_norm_noalloc: level 0 has %d leaves, the allocation-free variant "
                  "handles at most %d (use uaamg_poisson_residual_norm_device)",
                  D0.L.nl, maxl);
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    char* scratch = (char*)h->noalloc_scratch;
    double* partials = reinterpret_cast<double*>(scratch);
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + (size_t)UAAMG_NOALLOC_RED_DOUBLES * sizeof(double));
    if (D0.L.nl == 0) {
        CK(cudaMemsetAsync(d_norm, 0, sizeof(float), h->stream));
        return UAAMG_SUCCESS;
    }
    // the array keeps the previous call's contents: the tickets must start at zero
    CK(cudaMemsetAsync(partials, 0, (size_t)RED_HEADER * sizeof(double), h->stream));
    CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), h->stream));
    launch(k_residual_absmax, (unsigned)D0.L.nl, 128, h->stream, D0.L, d_x, d_b, d_r, partials, ticket, d_norm);
    h->launches++;
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_profile_pcg(uaamg_poisson* h, float* d_pressure, const float* d_rhs, int max_classes, char* names,
                              double* total_ms, int64_t* counts, int* nclasses) {
    ABI_BEGIN
    require(h && d_pressure && d_rhs && names && total_ms && counts && nclasses, "NULL argument");
    size_t nb = vec_bytes(h, 0);
    *nclasses = 0;
    if (!nb) return UAAMG_SUCCESS;
    if (h->smoother == UAAMG_SMOOTHER_SPAI0) ensure_spai0(h);
    CK(cudaMemcpyAsync(h->x, d_pressure, nb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->b, d_rhs, nb, cudaMemcpyDeviceToDevice, h->stream));
    init_state(h);
    std::vector<ProfRec> prof;
    Enq E{h, h->stream};
    E.prof = &prof;
    enqueue_setup(E, 0, 0);
    CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    while (h->st_host->status == PCG_RUNNING) {
        enqueue_body(E, 0, 0);
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    enqueue_finish(E);
    CK(cudaStreamSynchronize(h->stream));
    h->launches += E.count;
    h->iterations = h->st_host->iterations_taken;
    prof_collect(prof, max_classes, names, total_ms, counts, nclasses);
    CK(cudaMemcpyAsync(d_pressure, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return h->st_host->status == PCG_SUCCESS ? UAAMG_SUCCESS : UAAMG_FAILED;
    ABI_END
}

int uaamg_get_tuning(uaamg_tuning* out) {
    if (!out) { set_error("out is NULL"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *out = g_tune;
    return UAAMG_SUCCESS;
}
int uaamg_set_tuning(const uaamg_tuning* t) {
    if (!t) { set_error("tuning is NULL"); return UAAMG_ERR_INVALID_ARGUMENT; }
    if (t->staged_min_leaves < 1 || t->split_min_leaves < 1 || t->pipe_min_leaves < 1 || t->elem_ctas_per_sm < 1 ||
        t->elem_ctas_per_sm > 32 || (t->bottom_cycle != 0 && t->bottom_cycle != 1)) {
        set_error("tuning out of range (leaf thresholds >= 1, elem_ctas_per_sm 1..32, bottom_cycle 0/1)");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    g_tune = *t;
    ++g_tune_gen;
    return UAAMG_SUCCESS;
}

int uaamg_poisson_set_stream(uaamg_poisson* h, void* stream) {
    if (!h) { set_error("NULL handle"); return UAAMG_ERR_INVALID_ARGUMENT; }
    cudaStream_t s = stream ? (cudaStream_t)stream : h->own_stream;
    if (s != h->stream) {
        cudaStreamSynchronize(h->stream);
        h->stream = s;
    }
    return UAAMG_SUCCESS;
}
int uaamg_poisson_get_stream(const uaamg_poisson* h, void** stream) {
    if (!h || !stream) { set_error("NULL argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *stream = (void*)h->stream;
    return UAAMG_SUCCESS;
}
int uaamg_poisson_set_graph_mode(uaamg_poisson* h, int use_graph) {
    if (!h || use_graph < 0 || use_graph > 2) { set_error("invalid graph mode"); return UAAMG_ERR_INVALID_ARGUMENT; }
    h->use_graph = use_graph;
    return UAAMG_SUCCESS;
}
int64_t uaamg_poisson_kernel_launches(const uaamg_poisson* h) { return h ? h->launches : 0; }

int uaamg_solve_graph_cache_stats(int64_t* hits, int64_t* captures) {
    SolveGraphCache& c = solve_graph_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    if (hits) *hits = c.hits;
    if (captures) *captures = c.captures;
    return UAAMG_SUCCESS;
}

}  // extern "C"
