// packed3.cu -- packed_FloatGrid3 (SIMD_UAAMG/packed3grids.cpp) on the device:
// a staggered Vec3fGrid split into its three channel FloatGrids and merged
// back.  The reference's channel grids also carry a world transform shifted
// by -dx/2 along their axis (:22-26); a uaamg_leaf_grid is in index space and
// carries no transform, so only the values and the topology are converted.
// Compiled into the same translation unit as poisson.cu (uaamg_lib.cu).
#include <algorithm>
#include <vector>

namespace {

// from_vec3 (:11-43): the channel grids copy the vec3 grid's topology with
// every value set to the channel's background (Tree(other, background,
// TopologyCopy)); then each active voxel takes component c of the input.
// One CTA per leaf, 4 voxels per thread (their 12 floats are 48 contiguous bytes).
__global__ void __launch_bounds__(128) k_packed3_split(const float* __restrict__ in, const uint64_t* __restrict__ masks,
                                                       float bg0, float bg1, float bg2, float* __restrict__ o0,
                                                       float* __restrict__ o1, float* __restrict__ o2) {
    const long long leaf = blockIdx.x;
    const int t = threadIdx.x;
    const float4* p = reinterpret_cast<const float4*>(in + (leaf * UAAMG_LEAF + 4 * t) * 3);
    const float4 a = p[0], b = p[1], c = p[2];
    const float v[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    const unsigned m = masks ? (unsigned)((masks[leaf * 8 + (t >> 4)] >> ((t & 15) * 4)) & 0xFull) : 0xFu;
    const float bg[3] = {bg0, bg1, bg2};
    float* out[3] = {o0, o1, o2};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float4 r;
        r.x = (m & 1) ? v[0 + ch] : bg[ch];
        r.y = (m & 2) ? v[3 + ch] : bg[ch];
        r.z = (m & 4) ? v[6 + ch] : bg[ch];
        r.w = (m & 8) ? v[9 + ch] : bg[ch];
        reinterpret_cast<float4*>(out[ch])[leaf * (UAAMG_LEAF / 4) + t] = r;
    }
}

// to_vec3 (:46-83): the output holds the union of the channels' topologies
// (background (0,0,0)); component c is set at the active voxels of channel c.
// src[3 * leaf + c]: the leaf of channel c at the output leaf's origin, or -1.
struct Packed3Ch {
    const float* val;
    const uint64_t* mask;  // null: every voxel of the channel's leaves is active
};
__global__ void __launch_bounds__(128) k_packed3_merge(const int* __restrict__ src, Packed3Ch c0, Packed3Ch c1,
                                                       Packed3Ch c2, float* __restrict__ out) {
    const long long leaf = blockIdx.x;
    const int t = threadIdx.x;
    const Packed3Ch ch[3] = {c0, c1, c2};
    float v[12];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int s = src[3 * leaf + c];
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned m = 0;
        if (s >= 0) {
            x = reinterpret_cast<const float4*>(ch[c].val)[(long long)s * (UAAMG_LEAF / 4) + t];
            m = ch[c].mask ? (unsigned)((ch[c].mask[(long long)s * 8 + (t >> 4)] >> ((t & 15) * 4)) & 0xFull) : 0xFu;
        }
        v[0 + c] = (m & 1) ? x.x : 0.f;
        v[3 + c] = (m & 2) ? x.y : 0.f;
        v[6 + c] = (m & 4) ? x.z : 0.f;
        v[9 + c] = (m & 8) ? x.w : 0.f;
    }
    float4* o = reinterpret_cast<float4*>(out + (leaf * UAAMG_LEAF + 4 * t) * 3);
    o[0] = make_float4(v[0], v[1], v[2], v[3]);
    o[1] = make_float4(v[4], v[5], v[6], v[7]);
    o[2] = make_float4(v[8], v[9], v[10], v[11]);
}

static void packed3_check(const uaamg_leaf_grid* g, int comps, const char* name) {
    check_grid(g, comps, name);
}

// The union topology of the three channels: leaves in OpenVDB tree order, the
// OR of their active masks, and per output leaf the channel leaf at its origin.
struct Packed3Union {
    std::vector<int32_t> org;
    std::vector<uint64_t> mask;
    std::vector<int> src;  // [n][3]
};
static void packed3_union(const uaamg_leaf_grid* const ch[3], Packed3Union& U) {
    std::vector<std::pair<unsigned __int128, std::pair<int, int>>> keys;  // (key, (channel, leaf))
    size_t tot = 0;
    for (int c = 0; c < 3; ++c) tot += (size_t)ch[c]->leaf_count;
    keys.reserve(tot);
    for (int c = 0; c < 3; ++c)
        for (int64_t i = 0; i < ch[c]->leaf_count; ++i)
            keys.push_back({vdb_key128(&ch[c]->origins[3 * i]), {c, (int)i}});
    std::sort(keys.begin(), keys.end());
    U.org.clear();
    U.mask.clear();
    U.src.clear();
    for (size_t k = 0; k < keys.size(); ++k) {
        if (k == 0 || keys[k].first != keys[k - 1].first) {
            const int c = keys[k].second.first, i = keys[k].second.second;
            U.org.insert(U.org.end(), &ch[c]->origins[3 * i], &ch[c]->origins[3 * i] + 3);
            U.mask.insert(U.mask.end(), 8, 0ull);
            U.src.insert(U.src.end(), 3, -1);
        }
        const int c = keys[k].second.first, i = keys[k].second.second;
        const size_t o = U.src.size() / 3 - 1;
        if (U.src[3 * o + c] >= 0) {
            set_error("channel %d lists the leaf at (%d, %d, %d) twice", c, ch[c]->origins[3 * i],
                      ch[c]->origins[3 * i + 1], ch[c]->origins[3 * i + 2]);
            throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
        }
        U.src[3 * o + c] = i;
        for (int w = 0; w < 8; ++w) U.mask[8 * o + w] |= ch[c]->masks ? ch[c]->masks[8 * (size_t)i + w] : ~0ull;
    }
}

// merge into device memory d_out on stream s (channel values device-resident at
// dval[c]); the union is computed here
static void packed3_merge_dev(const uaamg_leaf_grid* const ch[3], const float* const dval[3], const Packed3Union& U,
                              float* d_out, DeviceCtx* ctx, cudaStream_t s, std::vector<void*>& tofree) {
    const size_t n = U.src.size() / 3;
    if (n == 0) return;
    size_t mbytes[3];
    size_t total = carve_size(n * 3, 4);
    for (int c = 0; c < 3; ++c) {
        mbytes[c] = ch[c]->masks && ch[c]->leaf_count ? (size_t)ch[c]->leaf_count * 64 : 0;
        total += carve_size(mbytes[c], 1);
    }
    void* mem = nullptr;
    CK(ctx_dev_alloc(ctx, &mem, total, s));
    tofree.push_back(mem);
    char* cur = (char*)mem;
    int* dsrc = carve<int>(cur, n * 3);
    CK(cudaMemcpyAsync(dsrc, U.src.data(), n * 3 * 4, cudaMemcpyHostToDevice, s));
    Packed3Ch pc[3];
    for (int c = 0; c < 3; ++c) {
        pc[c].val = dval[c];
        pc[c].mask = nullptr;
        if (mbytes[c]) {
            uint64_t* dm = carve<uint64_t>(cur, mbytes[c] / 8);
            CK(cudaMemcpyAsync(dm, ch[c]->masks, mbytes[c], cudaMemcpyHostToDevice, s));
            pc[c].mask = dm;
        }
    }
    k_packed3_merge<<<(unsigned)n, 128, 0, s>>>(dsrc, pc[0], pc[1], pc[2], d_out);
    CHECK_LAUNCH();
    // (the host tables are pageable: each copy returns once its source is staged, so they may go out of scope)
}

static void packed3_split_dev(const uaamg_leaf_grid* v, const float* d_in, float* const d_out[3], DeviceCtx* ctx,
                              cudaStream_t s, std::vector<void*>& tofree) {
    const int64_t n = v->leaf_count;
    if (n == 0) return;
    const uint64_t* dm = nullptr;
    if (v->masks) {
        void* mem = nullptr;
        CK(ctx_dev_alloc(ctx, &mem, (size_t)n * 64, s));
        tofree.push_back(mem);
        CK(cudaMemcpyAsync(mem, v->masks, (size_t)n * 64, cudaMemcpyHostToDevice, s));
        dm = (const uint64_t*)mem;
    }
    k_packed3_split<<<(unsigned)n, 128, 0, s>>>(d_in, dm, v->background[0], v->background[1], v->background[2],
                                                d_out[0], d_out[1], d_out[2]);
    CHECK_LAUNCH();
}

// a stream of the context for the duration of a host-pointer call
struct Packed3Call {
    DeviceCtx* ctx = nullptr;
    cudaStream_t s = nullptr;
    std::vector<void*> tofree;
    Packed3Call() {
        cudaError_t ce = cudaSuccess;
        ctx = device_ctx(&ce);
        CK(ce);
        CK(ctx_stream_acquire(ctx, &s));
    }
    ~Packed3Call() {
        for (void* p : tofree) cudaFreeAsync(p, s);
        cudaStreamSynchronize(s);
        ctx_stream_release(ctx, s);
    }
};

}  // namespace

extern "C" {

int uaamg_packed3_from_vec3(const uaamg_leaf_grid* vec3, float* out_c0, float* out_c1, float* out_c2) {
    ABI_BEGIN
    packed3_check(vec3, 3, "vec3");
    require(!vec3->values_on_device, "vec3 values are on the device: use uaamg_packed3_from_vec3_device");
    const int64_t n = vec3->leaf_count;
    if (n == 0) return UAAMG_SUCCESS;
    require(out_c0 && out_c1 && out_c2, "NULL output");
    Packed3Call call;
    const size_t cb = (size_t)n * UAAMG_LEAF * 4;
    void* mem = nullptr;
    CK(ctx_dev_alloc(call.ctx, &mem, carve_size(cb * 3, 1) + 3 * carve_size(cb, 1), call.s));
    call.tofree.push_back(mem);
    char* cur = (char*)mem;
    float* din = carve<float>(cur, (size_t)n * UAAMG_LEAF * 3);
    float* dout[3];
    for (int c = 0; c < 3; ++c) dout[c] = carve<float>(cur, (size_t)n * UAAMG_LEAF);
    CK(cudaMemcpyAsync(din, vec3->values, cb * 3, cudaMemcpyHostToDevice, call.s));
    packed3_split_dev(vec3, din, dout, call.ctx, call.s, call.tofree);
    float* host[3] = {out_c0, out_c1, out_c2};
    for (int c = 0; c < 3; ++c) CK(cudaMemcpyAsync(host[c], dout[c], cb, cudaMemcpyDeviceToHost, call.s));
    CK(cudaStreamSynchronize(call.s));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_packed3_from_vec3_device(const uaamg_leaf_grid* vec3, float* d_c0, float* d_c1, float* d_c2, void* stream) {
    ABI_BEGIN
    packed3_check(vec3, 3, "vec3");
    require(vec3->values_on_device || vec3->leaf_count == 0, "vec3 values must be device memory");
    if (vec3->leaf_count == 0) return UAAMG_SUCCESS;
    require(d_c0 && d_c1 && d_c2, "NULL output");
    require(!(((uintptr_t)vec3->values | (uintptr_t)d_c0 | (uintptr_t)d_c1 | (uintptr_t)d_c2) & 15),
            "device arrays must be 16-byte aligned");
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<void*> tofree;
    float* dout[3] = {d_c0, d_c1, d_c2};
    packed3_split_dev(vec3, vec3->values, dout, ctx, s, tofree);
    for (void* p : tofree) CK(cudaFreeAsync(p, s));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_packed3_to_vec3_topology(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                                   int64_t* leaf_count, int32_t* out_origins, uint64_t* out_masks) {
    ABI_BEGIN
    require(leaf_count, "NULL leaf_count");
    packed3_check(c0, 1, "c0");
    packed3_check(c1, 1, "c1");
    packed3_check(c2, 1, "c2");
    const uaamg_leaf_grid* ch[3] = {c0, c1, c2};
    Packed3Union U;
    packed3_union(ch, U);
    const int64_t n = (int64_t)U.src.size() / 3;
    if (out_origins) {
        if (*leaf_count < n) {
            set_error("out_origins holds %lld leaves, the union has %lld", (long long)*leaf_count, (long long)n);
            throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
        }
        std::copy(U.org.begin(), U.org.end(), out_origins);
        if (out_masks) std::copy(U.mask.begin(), U.mask.end(), out_masks);
    }
    *leaf_count = n;
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_packed3_to_vec3(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                          float* out_values) {
    ABI_BEGIN
    const uaamg_leaf_grid* ch[3] = {c0, c1, c2};
    const char* names[3] = {"c0", "c1", "c2"};
    for (int c = 0; c < 3; ++c) {
        packed3_check(ch[c], 1, names[c]);
        require(!ch[c]->values_on_device, "channel values are on the device: use uaamg_packed3_to_vec3_device");
    }
    Packed3Union U;
    packed3_union(ch, U);
    const size_t n = U.src.size() / 3;
    if (n == 0) return UAAMG_SUCCESS;
    require(out_values, "NULL output");
    Packed3Call call;
    size_t total = carve_size(n * UAAMG_LEAF * 3 * 4, 1);
    for (int c = 0; c < 3; ++c) total += carve_size((size_t)ch[c]->leaf_count * UAAMG_LEAF * 4, 1);
    void* mem = nullptr;
    CK(ctx_dev_alloc(call.ctx, &mem, total, call.s));
    call.tofree.push_back(mem);
    char* cur = (char*)mem;
    float* dout = carve<float>(cur, n * UAAMG_LEAF * 3);
    const float* dval[3];
    for (int c = 0; c < 3; ++c) {
        const size_t b = (size_t)ch[c]->leaf_count * UAAMG_LEAF * 4;
        float* d = carve<float>(cur, b / 4);
        if (b) CK(cudaMemcpyAsync(d, ch[c]->values, b, cudaMemcpyHostToDevice, call.s));
        dval[c] = d;
    }
    packed3_merge_dev(ch, dval, U, dout, call.ctx, call.s, call.tofree);
    CK(cudaMemcpyAsync(out_values, dout, n * UAAMG_LEAF * 3 * 4, cudaMemcpyDeviceToHost, call.s));
    CK(cudaStreamSynchronize(call.s));
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_packed3_to_vec3_device(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                                 float* d_out_values, void* stream) {
    ABI_BEGIN
    const uaamg_leaf_grid* ch[3] = {c0, c1, c2};
    const char* names[3] = {"c0", "c1", "c2"};
    for (int c = 0; c < 3; ++c) {
        packed3_check(ch[c], 1, names[c]);
        require(ch[c]->values_on_device || ch[c]->leaf_count == 0, "channel values must be device memory");
    }
    Packed3Union U;
    packed3_union(ch, U);
    if (U.src.empty()) return UAAMG_SUCCESS;
    require(d_out_values, "NULL output");
    require(!(((uintptr_t)c0->values | (uintptr_t)c1->values | (uintptr_t)c2->values | (uintptr_t)d_out_values) & 15),
            "device arrays must be 16-byte aligned");
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<void*> tofree;
    const float* dval[3] = {c0->values, c1->values, c2->values};
    packed3_merge_dev(ch, dval, U, d_out_values, ctx, s, tofree);
    for (void* p : tofree) CK(cudaFreeAsync(p, s));
    return UAAMG_SUCCESS;
    ABI_END
}

}  // extern "C"
