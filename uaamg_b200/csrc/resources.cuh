// resources.cuh -- per-device pools that make solver handles cheap to create.
//
// A FLIP substep builds a new hierarchy for every pressure solve
// (FLIP_vdb.cpp:3132-3141), so the fixed cost of a handle matters as much as
// the solve.  cudaMalloc/cudaFree, pinned host allocation and stream creation
// each cost tens of microseconds to milliseconds and synchronise the device,
// so handles draw all three from per-device pools instead:
//  * device memory: a private stream-ordered memory pool whose release
//    threshold is "never", so freed blocks are reused without OS calls;
//  * streams and pinned host blocks: free lists.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

namespace uaamg {

struct DeviceCtx {
    int device = -1;
    int sms = 0;  // streaming multiprocessors of the device
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    std::vector<cudaStream_t> streams;
    std::vector<std::pair<size_t, void*>> pinned;  // free pinned blocks (capacity, pointer)
};

inline std::mutex& ctx_registry_mutex() {
    static std::mutex m;
    return m;
}

// Context of the current device (created on first use).
inline DeviceCtx* device_ctx(cudaError_t* err) {
    static DeviceCtx* ctxs[64] = {nullptr};
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= 64) { *err = cudaErrorInvalidDevice; return nullptr; }
    std::lock_guard<std::mutex> lk(ctx_registry_mutex());
    if (!ctxs[dev]) {
        DeviceCtx* c = new DeviceCtx();
        c->device = dev;
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        *err = cudaMemPoolCreate(&c->pool, &props);
        if (*err != cudaSuccess) { delete c; return nullptr; }
        uint64_t thr = UINT64_MAX;
        *err = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr);
        if (*err != cudaSuccess) { delete c; return nullptr; }
        *err = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
        if (*err != cudaSuccess) { delete c; return nullptr; }
        ctxs[dev] = c;
    }
    return ctxs[dev];
}

inline cudaError_t ctx_stream_acquire(DeviceCtx* c, cudaStream_t* s) {
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if (!c->streams.empty()) {
            *s = c->streams.back();
            c->streams.pop_back();
            return cudaSuccess;
        }
    }
    return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
}
inline void ctx_stream_release(DeviceCtx* c, cudaStream_t s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(c->mu);
    c->streams.push_back(s);
}

// pinned host block of at least `bytes`; *cap receives its capacity
inline cudaError_t ctx_pinned_acquire(DeviceCtx* c, size_t bytes, void** p, size_t* cap) {
    {
        std::lock_guard<std::mutex> lk(c->mu);
        size_t best = (size_t)-1;
        int bi = -1;
        for (size_t i = 0; i < c->pinned.size(); ++i)
            if (c->pinned[i].first >= bytes && c->pinned[i].first < best) { best = c->pinned[i].first; bi = (int)i; }
        if (bi >= 0) {
            *cap = c->pinned[bi].first;
            *p = c->pinned[bi].second;
            c->pinned.erase(c->pinned.begin() + bi);
            return cudaSuccess;
        }
    }
    size_t sz = 4096;
    while (sz < bytes) sz <<= 1;
    *cap = sz;
    return cudaMallocHost(p, sz);
}
inline void ctx_pinned_release(DeviceCtx* c, void* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(c->mu);
    c->pinned.push_back({cap, p});
}

inline cudaError_t ctx_dev_alloc(DeviceCtx* c, void** p, size_t bytes, cudaStream_t s) {
    return cudaMallocFromPoolAsync(p, bytes ? bytes : 256, c->pool, s);
}

}  // namespace uaamg
