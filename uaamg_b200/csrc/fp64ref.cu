// fp64ref.cu -- FP64 reference solve of the level-0 pressure system.
//
// The accuracy of every solver form (FP32, the 16-bit hierarchies) is stated
// against the exact solution of the same system, which the benchmark names as
// an FP64 Eigen CG solved to 1e-12 (Eigen is not available here).  This is that
// solve: the level-0 matrix assembled from the FP32 coefficients (each entry
// a float, held exactly in FP64; getTriplets, SIMD_UAAMG/simd_vdb_poisson.cpp:
// 129-206), FP64 vectors and FP64 dot products, and a flexible preconditioned
// CG (Polak-Ribiere beta, so a preconditioner computed in FP32 is admissible)
// that stops when the TRUE residual |b - A x|_2 <= rel_tol |b|_2 (Eigen's CG
// criterion), recomputing the residual from x before it accepts convergence.
// The preconditioner is the handle's FP32 W-cycle applied to the residual
// scaled by a power of two (|r / s|_inf in [1, 2), so no FP32 underflow as the
// residual falls by twelve orders of magnitude), its result scaled back.
// No counterpart in the reference.

namespace uaamg {

#define F64_CTAS 2368  // grid of the grid-stride FP64 passes (16 CTAs of 128 threads per SM)

// (A x)_v in FP64 at voxel `off` of `leaf` (the FP32 coefficients promoted; the
// plus-face entry is the neighbour's minus-face coefficient)
__device__ __forceinline__ double a64_at(const DLevel& L, int leaf, int off, const double* x) {
    const unsigned fl = L.flags[leaf];
    const int* nb = L.nbr + (long long)leaf * 6;
    const int X = off >> 6, Y = (off >> 3) & 7, Z = off & 7;
    const long long i = (long long)leaf * UAAMG_LEAF + off;
    auto xat = [&](int lf, int o) -> double { return lf >= 0 ? x[(long long)lf * UAAMG_LEAF + o] : 0.0; };
    auto cat = [&](const float* c, unsigned bit, int lf, int o) -> double {
        if (lf < 0) return (double)L.def_face;
        return (L.flags[lf] & bit) ? (double)L.def_face : (double)c[(long long)lf * UAAMG_LEAF + o];
    };
    const double dg = (fl & TRIM_DIAG) ? (double)L.def_diag : (double)L.diag[i];
    double ax = dg * x[i];
    ax += cat(L.cx, TRIM_X, leaf, off) * (X > 0 ? xat(leaf, off - 64) : xat(nb[0], off + 448));
    ax += cat(L.cy, TRIM_Y, leaf, off) * (Y > 0 ? xat(leaf, off - 8) : xat(nb[2], off + 56));
    ax += cat(L.cz, TRIM_Z, leaf, off) * (Z > 0 ? xat(leaf, off - 1) : xat(nb[4], off + 7));
    ax += X < 7 ? cat(L.cx, TRIM_X, leaf, off + 64) * xat(leaf, off + 64)
                : cat(L.cx, TRIM_X, nb[1], off - 448) * xat(nb[1], off - 448);
    ax += Y < 7 ? cat(L.cy, TRIM_Y, leaf, off + 8) * xat(leaf, off + 8)
                : cat(L.cy, TRIM_Y, nb[3], off - 56) * xat(nb[3], off - 56);
    ax += Z < 7 ? cat(L.cz, TRIM_Z, leaf, off + 1) * xat(leaf, off + 1)
                : cat(L.cz, TRIM_Z, nb[5], off - 7) * xat(nb[5], off - 7);
    return ax;
}
__device__ __forceinline__ bool dof_at(const DLevel& L, int leaf, int off) {
    return (L.mask[(long long)leaf * 8 + (off >> 6)] >> (off & 63)) & 1ull;
}

// y = A x (out = A x), or y = b - A x (RESID); zero off the DOF
template <bool RESID>
__global__ void __launch_bounds__(128) k64_apply(DLevel L, const double* x, const double* b, double* y) {
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x)
        for (int off = threadIdx.x; off < UAAMG_LEAF; off += 128) {
            const long long i = (long long)leaf * UAAMG_LEAF + off;
            double v = 0.0;
            if (dof_at(L, leaf, off)) {
                const double ax = a64_at(L, leaf, off, x);
                v = RESID ? b[i] - ax : ax;
            }
            y[i] = v;
        }
}

// per-CTA partial sums of a . b over the DOF (then k64_sum: fixed order)
__global__ void __launch_bounds__(128) k64_dot(DLevel L, const double* a, const double* b, double* partials) {
    __shared__ double sh[4];
    double s = 0.0;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x)
        for (int off = threadIdx.x; off < UAAMG_LEAF; off += 128) {
            const long long i = (long long)leaf * UAAMG_LEAF + off;
            if (dof_at(L, leaf, off)) s += a[i] * b[i];
        }
    const double p = block_sum128(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = p;
}
// per-CTA partial maxima of |a| over the DOF
__global__ void __launch_bounds__(128) k64_absmax(DLevel L, const double* a, double* partials) {
    __shared__ double sh[4];
    double m = 0.0;
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x)
        for (int off = threadIdx.x; off < UAAMG_LEAF; off += 128) {
            const long long i = (long long)leaf * UAAMG_LEAF + off;
            if (dof_at(L, leaf, off)) m = fmax(m, fabs(a[i]));
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(FULLMASK, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) partials[blockIdx.x] = fmax(fmax(sh[0], sh[1]), fmax(sh[2], sh[3]));
}
// out[0] = the partials combined in index order (sum or max)
template <bool MAX>
__global__ void __launch_bounds__(32) k64_combine(const double* partials, int n, double* out) {
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = MAX ? fmax(s, partials[i]) : s + partials[i];
    out[0] = s;
}

// y = x + a y (XPAY) or y += a x; n = elements (grid-stride)
template <bool XPAY>
__global__ void __launch_bounds__(256) k64_axpy(long long n, double a, const double* x, double* y) {
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        y[i] = XPAY ? x[i] + a * y[i] : y[i] + a * x[i];
}
// double <-> float with a power-of-two scale (exact apart from the float rounding)
__global__ void __launch_bounds__(256) k64_to_float(long long n, const double* in, float* out, double scale) {
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        out[i] = (float)(in[i] * scale);
}
__global__ void __launch_bounds__(256) k64_from_float(long long n, const float* in, double* out, double scale) {
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        out[i] = (double)in[i] * scale;
}
// b64 = b on the DOF, 0 elsewhere
__global__ void __launch_bounds__(128) k64_rhs(DLevel L, const float* b, double* out) {
    for (int leaf = blockIdx.x; leaf < L.nl; leaf += gridDim.x)
        for (int off = threadIdx.x; off < UAAMG_LEAF; off += 128) {
            const long long i = (long long)leaf * UAAMG_LEAF + off;
            out[i] = dof_at(L, leaf, off) ? (double)b[i] : 0.0;
        }
}

}  // namespace uaamg

namespace {

struct F64Solver {
    uaamg_poisson* h;
    cudaStream_t s;
    DLevel L;
    long long n;   // vector elements (leaves * 512)
    unsigned grid;
    double* part;  // [F64_CTAS]
    double* scal;  // [1] device scalar
    double* scal_host;

    double reduce_dot(const double* a, const double* b) {
        k64_dot<<<grid, 128, 0, s>>>(L, a, b, part);
        k64_combine<false><<<1, 32, 0, s>>>(part, (int)grid, scal);
        return fetch();
    }
    double reduce_absmax(const double* a) {
        k64_absmax<<<grid, 128, 0, s>>>(L, a, part);
        k64_combine<true><<<1, 32, 0, s>>>(part, (int)grid, scal);
        return fetch();
    }
    double fetch() {
        CHECK_LAUNCH();
        CK(cudaMemcpyAsync(scal_host, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return *scal_host;
    }
    unsigned egrid() const { return (unsigned)std::min<long long>((n + 255) / 256, F64_CTAS); }
    // z = M^-1 r with the FP32 W-cycle on r / s (s a power of two near |r|_inf)
    void precondition(const double* r, double* z) {
        const double rmax = reduce_absmax(r);
        if (!(rmax > 0.0) || !std::isfinite(rmax)) {
            CK(cudaMemsetAsync(z, 0, (size_t)n * sizeof(double), s));
            return;
        }
        const double sc = std::ldexp(1.0, std::ilogb(rmax));
        k64_to_float<<<egrid(), 256, 0, s>>>(n, r, h->r, 1.0 / sc);
        CHECK_LAUNCH();
        CK(cudaMemsetAsync(h->z, 0, (size_t)n * sizeof(float), s));
        Enq E{h, s};
        enqueue_precond(E, 0, h->z, h->r, true, DotOut{nullptr, nullptr, nullptr});
        k64_from_float<<<egrid(), 256, 0, s>>>(n, h->z, z, sc);
        CHECK_LAUNCH();
        h->launches += E.count + 2;
    }
};

}  // namespace

extern "C" {

int uaamg_poisson_solve_fp64_reference(uaamg_poisson* h, const float* d_rhs, double* d_x, double rel_tol,
                                       int max_iter, int* iterations, double* rel_residual) {
    ABI_BEGIN
    require(h && d_rhs && d_x, "NULL argument");
    require(rel_tol > 0.0 && max_iter > 0, "rel_tol and max_iter must be positive");
    if (iterations) *iterations = 0;
    if (rel_residual) *rel_residual = 0.0;
    LevelDev& D0 = h->lv[0];
    const long long n = (long long)D0.L.nl * UAAMG_LEAF;
    if (n == 0) return UAAMG_SUCCESS;
    if (h->smoother == UAAMG_SMOOTHER_SPAI0) ensure_spai0(h);
    cudaStream_t s = h->stream;
    F64Solver F;
    F.h = h;
    F.s = s;
    F.L = D0.L;
    F.n = n;
    F.grid = (unsigned)std::min(D0.L.nl, F64_CTAS);
    // FP64 work vectors b, r, z, z_old, p, q and the reduction buffer (pool memory, freed at the end)
    const size_t vb = (size_t)n * sizeof(double);
    char* mem = nullptr;
    CK(ctx_dev_alloc(h->ctx, (void**)&mem, 6 * vb + (F64_CTAS + 2) * sizeof(double), s));
    double* b = (double*)mem;
    double* r = (double*)(mem + vb);
    double* z = (double*)(mem + 2 * vb);
    double* zo = (double*)(mem + 3 * vb);
    double* p = (double*)(mem + 4 * vb);
    double* q = (double*)(mem + 5 * vb);
    F.part = (double*)(mem + 6 * vb);
    F.scal = F.part + F64_CTAS;
    F.scal_host = reinterpret_cast<double*>(h->scalar_host);  // pinned, 64 floats
    int status = UAAMG_FAILED, it = 0;
    double rel = 0.0;
    try {
        const unsigned lg = F.grid;
        k64_rhs<<<lg, 128, 0, s>>>(D0.L, d_rhs, b);
        CHECK_LAUNCH();
        CK(cudaMemsetAsync(d_x, 0, vb, s));
        const double bn = std::sqrt(F.reduce_dot(b, b));
        if (bn == 0.0) {
            status = UAAMG_SUCCESS;
        } else {
            CK(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
            F.precondition(r, z);
            CK(cudaMemcpyAsync(p, z, vb, cudaMemcpyDeviceToDevice, s));
            double rz = F.reduce_dot(r, z);
            for (it = 1; it <= max_iter; ++it) {
                k64_apply<false><<<lg, 128, 0, s>>>(D0.L, p, nullptr, q);
                CHECK_LAUNCH();
                const double alpha = rz / F.reduce_dot(p, q);
                k64_axpy<false><<<F.egrid(), 256, 0, s>>>(n, alpha, p, d_x);
                k64_axpy<false><<<F.egrid(), 256, 0, s>>>(n, -alpha, q, r);
                CHECK_LAUNCH();
                rel = std::sqrt(F.reduce_dot(r, r)) / bn;
                if (!std::isfinite(rel)) break;
                if (rel <= rel_tol) {
                    // accept only on the true residual; otherwise continue from it
                    k64_apply<true><<<lg, 128, 0, s>>>(D0.L, d_x, b, r);
                    CHECK_LAUNCH();
                    rel = std::sqrt(F.reduce_dot(r, r)) / bn;
                    if (rel <= rel_tol) {
                        status = UAAMG_SUCCESS;
                        break;
                    }
                }
                std::swap(z, zo);
                F.precondition(r, z);
                const double rz_new = F.reduce_dot(r, z);
                const double rz_mix = F.reduce_dot(r, zo);
                const double beta = (rz_new - rz_mix) / rz;  // Polak-Ribiere (flexible CG)
                rz = rz_new;
                k64_axpy<true><<<F.egrid(), 256, 0, s>>>(n, beta, z, p);
                CHECK_LAUNCH();
            }
            if (it > max_iter) it = max_iter;
        }
    } catch (...) {
        cudaFreeAsync(mem, s);
        throw;
    }
    CK(cudaFreeAsync(mem, s));
    CK(cudaStreamSynchronize(s));
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = rel;
    return status;
    ABI_END
}

}  // extern "C"
