// extrapolate.cu -- velocity extrapolation into a band of new voxels on the
// device: vdb_velocity_extrapolator::union_extrapolate
// (FLIP_vdb/vdb_velocity_extrapolator.cpp:585-662), which runs around the
// viscosity solve of a FLIP substep.  The topology set operations of the
// reference (union of the channels, dilation, difference, touchLeaf) are done
// by the caller, which passes per channel the leaves of the output grid and the
// voxels to fill; each layer is one kernel over those leaves.
// Included by uaamg_lib.cu after poisson.cu (grids, errors, resources).

namespace uaamg {

// One layer of value_extrapolator (:621-652) for the channel grid `out`
// (values [n_out][512] updated in place, active masks `snap` before the layer):
// every voxel of the fill set of leaf e (rem[e], still to fill) with at least
// one active face neighbour gets the mean of those neighbours' values (summed
// in the order -x, +x, -y, +y, -z, +z), becomes active in `next` and leaves
// the fill set.  `next` holds a copy of `snap` on entry.  Only neighbours
// active in `snap` are read and only voxels inactive in it are written, so the
// layer does not depend on the order of the leaves.
__global__ void __launch_bounds__(128) k_extrapolate_layer(int n_fill, const int* fill_leaf, uint64_t* rem,
                                                           const int* out_org, const int* map, int lo0, int lo1,
                                                           int lo2, int d0, int d1, int d2, const uint64_t* snap,
                                                           uint64_t* next, float* val) {
    __shared__ uint32_t nbits[16], rbits[16];
    const int e = blockIdx.x, t = threadIdx.x;
    if (e >= n_fill) return;
    if (t < 16) nbits[t] = rbits[t] = 0;
    __syncthreads();
    const int li = fill_leaf[e];
    const int ox = out_org[3 * li], oy = out_org[3 * li + 1], oz = out_org[3 * li + 2];
    unsigned filled = 0, remaining = 0;
    for (int j = 0; j < 4; ++j) {
        const int off = 4 * t + j;
        if (!((rem[(long long)e * 8 + (off >> 6)] >> (off & 63)) & 1ull)) continue;
        const int g[3] = {ox + (off >> 6), oy + ((off >> 3) & 7), oz + (off & 7)};
        int wcount = 0;
        float sum = 0.f;
#pragma unroll
        for (int d = 0; d < 6; ++d) {
            int q[3] = {g[0], g[1], g[2]};
            q[d >> 1] += (d & 1) ? 1 : -1;
            const int a = (q[0] >> 3) - lo0, b = (q[1] >> 3) - lo1, c = (q[2] >> 3) - lo2;
            if ((unsigned)a >= (unsigned)d0 || (unsigned)b >= (unsigned)d1 || (unsigned)c >= (unsigned)d2) continue;
            const int nl = map[((long long)a * d1 + b) * d2 + c];
            if (nl < 0) continue;
            const int qo = ((q[0] & 7) << 6) | ((q[1] & 7) << 3) | (q[2] & 7);
            if (!((snap[(long long)nl * 8 + (qo >> 6)] >> (qo & 63)) & 1ull)) continue;
            ++wcount;
            sum = __fadd_rn(sum, val[(long long)nl * UAAMG_LEAF + qo]);
        }
        if (wcount) {
            val[(long long)li * UAAMG_LEAF + off] = __fdiv_rn(sum, (float)wcount);
            filled |= 1u << j;
        } else {
            remaining |= 1u << j;
        }
    }
    atomicOr(&nbits[t >> 3], filled << ((t & 7) * 4));
    atomicOr(&rbits[t >> 3], remaining << ((t & 7) * 4));
    __syncthreads();
    if (t < 8) {
        const uint64_t f = (uint64_t)nbits[2 * t] | ((uint64_t)nbits[2 * t + 1] << 32);
        next[(long long)li * 8 + t] = snap[(long long)li * 8 + t] | f;
        rem[(long long)e * 8 + t] = (uint64_t)rbits[2 * t] | ((uint64_t)rbits[2 * t + 1] << 32);
    }
}

// Host-side checks of one channel's inputs; builds the dense leaf map of the
// output leaves.  Returns UAAMG_SUCCESS or the error code (message set).
static int extrapolate_check(int n_layer, int64_t n_out, const int32_t* out_origins, int64_t n_fill,
                             const int32_t* fill_leaf, const uint64_t* fill_masks, HostMap& map) {
    if (n_layer < 0 || n_out < 0 || n_fill < 0) {
        set_error("extrapolate: negative count");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    if ((n_out && !out_origins) || (n_fill && (!fill_leaf || !fill_masks))) {
        set_error("extrapolate: NULL leaf origins or fill set");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < 3 * n_out; ++i)
        if (out_origins[i] & 7) {
            set_error("extrapolate: leaf origins must be multiples of 8");
            return UAAMG_ERR_INVALID_ARGUMENT;
        }
    std::vector<char> seen((size_t)n_out, 0);  // one fill entry per output leaf (a block owns its leaf's masks)
    for (int64_t e = 0; e < n_fill; ++e) {
        if (fill_leaf[e] < 0 || fill_leaf[e] >= n_out) {
            set_error("extrapolate: fill leaf %d out of range", (int)fill_leaf[e]);
            return UAAMG_ERR_INVALID_ARGUMENT;
        }
        if (seen[(size_t)fill_leaf[e]]++) {
            set_error("extrapolate: output leaf %d listed twice in the fill set", (int)fill_leaf[e]);
            return UAAMG_ERR_INVALID_ARGUMENT;
        }
    }
    map.build(n_out, out_origins);
    for (int64_t i = 0; i < n_out; ++i)
        if (map.idx[map.cell(out_origins[3 * i] >> 3, out_origins[3 * i + 1] >> 3, out_origins[3 * i + 2] >> 3)] !=
            (int32_t)i) {
            set_error("extrapolate: duplicate output leaf origin");
            return UAAMG_ERR_INVALID_ARGUMENT;
        }
    return UAAMG_SUCCESS;
}

// The layers on stream s over device values/masks [n_out] (updated in place).
// Both mask buffers start as the input masks; a layer rewrites the masks of
// fill-set leaves only, so the other leaves stay equal in both and no copy is
// needed between layers.  Enqueued only (the scratch is freed stream-ordered).
static void extrapolate_enqueue(DeviceCtx* ctx, cudaStream_t s, const HostMap& map, int n_layer, int64_t n_out,
                                const int32_t* out_origins, float* dval, uint64_t* dmask, int64_t n_fill,
                                const int32_t* fill_leaf, const uint64_t* fill_masks) {
    const size_t mb = (size_t)n_out * 64;
    const size_t tot = carve_size(map.idx.size(), 4) + carve_size((size_t)n_out * 3, 4) + carve_size(mb, 1) +
                       carve_size((size_t)n_fill, 4) + carve_size((size_t)n_fill * 64, 1);
    void* mem = nullptr;
    CK(ctx_dev_alloc(ctx, &mem, tot, s));
    try {
        char* cur = (char*)mem;
        int* dmap = carve<int>(cur, map.idx.size());
        int* dorg = carve<int>(cur, (size_t)n_out * 3);
        uint64_t* m1 = carve<uint64_t>(cur, (size_t)n_out * 8);
        int* dfl = carve<int>(cur, (size_t)n_fill);
        uint64_t* drem = carve<uint64_t>(cur, (size_t)n_fill * 8);
        CK(cudaMemcpyAsync(dmap, map.idx.data(), map.idx.size() * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dorg, out_origins, (size_t)n_out * 12, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dfl, fill_leaf, (size_t)n_fill * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(drem, fill_masks, (size_t)n_fill * 64, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(m1, dmask, mb, cudaMemcpyDeviceToDevice, s));
        uint64_t *m0 = dmask, *mn = m1;
        for (int layer = 0; layer < n_layer; ++layer) {
            k_extrapolate_layer<<<(unsigned)n_fill, 128, 0, s>>>((int)n_fill, dfl, drem, dorg, dmap, map.lo[0],
                                                                 map.lo[1], map.lo[2], map.dim[0], map.dim[1],
                                                                 map.dim[2], m0, mn, dval);
            CHECK_LAUNCH();
            std::swap(m0, mn);
        }
        if (m0 != dmask) CK(cudaMemcpyAsync(dmask, m0, mb, cudaMemcpyDeviceToDevice, s));
    } catch (...) {
        cudaFreeAsync(mem, s);
        throw;
    }
    CK(cudaFreeAsync(mem, s));
}

}  // namespace uaamg

extern "C" {

int uaamg_extrapolate_channel(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                              uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf,
                              const uint64_t* fill_masks) {
    ABI_BEGIN
    require(n_out == 0 || (values && masks), "NULL output grid");
    HostMap map;
    const int rc = extrapolate_check(n_layer, n_out, out_origins, n_fill, fill_leaf, fill_masks, map);
    if (rc != UAAMG_SUCCESS) return rc;
    if (n_out == 0 || n_fill == 0 || n_layer == 0) return UAAMG_SUCCESS;
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = nullptr;
    CK(ctx_stream_acquire(ctx, &s));
    void* mem = nullptr;
    try {
        const size_t vb = (size_t)n_out * UAAMG_LEAF * 4, mb = (size_t)n_out * 64;
        CK(ctx_dev_alloc(ctx, &mem, carve_size(vb, 1) + carve_size(mb, 1), s));
        char* cur = (char*)mem;
        float* dval = carve<float>(cur, vb / 4);
        uint64_t* dmask = carve<uint64_t>(cur, (size_t)n_out * 8);
        CK(cudaMemcpyAsync(dval, values, vb, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dmask, masks, mb, cudaMemcpyHostToDevice, s));
        extrapolate_enqueue(ctx, s, map, n_layer, n_out, out_origins, dval, dmask, n_fill, fill_leaf, fill_masks);
        CK(cudaMemcpyAsync(values, dval, vb, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(masks, dmask, mb, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(mem, s));
        mem = nullptr;
        CK(cudaStreamSynchronize(s));
    } catch (...) {
        if (mem) cudaFreeAsync(mem, s);
        cudaStreamSynchronize(s);
        ctx_stream_release(ctx, s);
        throw;
    }
    ctx_stream_release(ctx, s);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_extrapolate_channel_device(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                                     uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf,
                                     const uint64_t* fill_masks, void* stream) {
    ABI_BEGIN
    require(n_out == 0 || (values && masks), "NULL output grid");
    HostMap map;
    const int rc = extrapolate_check(n_layer, n_out, out_origins, n_fill, fill_leaf, fill_masks, map);
    if (rc != UAAMG_SUCCESS) return rc;
    if (n_out == 0 || n_fill == 0 || n_layer == 0) return UAAMG_SUCCESS;
    cudaError_t ce = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&ce);
    CK(ce);
    cudaStream_t s = (cudaStream_t)stream;
    extrapolate_enqueue(ctx, s, map, n_layer, n_out, out_origins, values, masks, n_fill, fill_leaf, fill_masks);
    return UAAMG_SUCCESS;
    ABI_END
}

}  // extern "C"
