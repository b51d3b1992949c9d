// mixed.cu -- host side of the mixed-precision pressure solve (kernels in
// poisson_mixed.cuh): a 16-bit copy of a handle's hierarchy, the FP64
// coarsest inverse, the 16-bit mu-cycle and the outer FP32 CG as one CUDA
// graph, and an FP64 true-residual check.
#include "poisson_mixed.cuh"

namespace {

struct MixedLevel {
    void* diag = nullptr;
    void* invdiag = nullptr;
    void* cx = nullptr;
    void* cy = nullptr;
    void* cz = nullptr;
    void* lhs = nullptr;
    void* rhs = nullptr;
    void* tmp = nullptr;
};

}  // namespace

struct MixedData {
    int precision = 0;  // UAAMG_PRECISION_FP16 / _BF16
    char* mem = nullptr;
    std::vector<MixedLevel> lv;
    double* ainv = nullptr;  // [nc][nc] inverse of the coarsest matrix
    float* sigma = nullptr;  // normalisation of the current preconditioner application
    int nc = 0;
    int replace_every = 25;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_every = -1;
    int64_t setup_launches = 0, body_launches = 0, finish_launches = 0;
    unsigned long long* res64 = nullptr;  // k_res64 output
    double setup_ms = 0.0;
};

namespace {

// storage scale of a level: the power of two nearest below its default diagonal
static float level_scale(const DLevel& L) {
    const float d = L.def_diag;
    return (d > 0.f && std::isfinite(d)) ? std::ldexp(1.0f, std::ilogb(d)) : 1.0f;
}

template <typename T>
static MLevel<T> mlevel(const uaamg_poisson* h, int l) {
    const LevelDev& D = h->lv[l];
    const MixedLevel& M = h->mixed->lv[l];
    MLevel<T> L;
    L.nl = D.L.nl;
    L.mask = D.L.mask;
    L.nbr = D.L.nbr;
    L.parent = D.L.parent;
    L.octant = D.L.octant;
    L.flags = D.L.flags;
    L.diag = (const T*)M.diag;
    L.invdiag = (const T*)M.invdiag;
    L.cx = (const T*)M.cx;
    L.cy = (const T*)M.cy;
    L.cz = (const T*)M.cz;
    L.def_diag = D.L.def_diag;
    L.def_face = D.L.def_face;
    L.def_invdiag = D.L.def_invdiag;
    L.cs = level_scale(D.L);
    L.ics = 1.0f / L.cs;
    return L;
}

static void mixed_destroy_graph(MixedData* M) {
    if (M->exec) cudaGraphExecDestroy(M->exec);
    if (M->graph) cudaGraphDestroy(M->graph);
    M->exec = nullptr;
    M->graph = nullptr;
    M->graph_every = -1;
}

}  // namespace

// called by uaamg_poisson_destroy
static void mixed_free(uaamg_poisson* h) {
    MixedData* M = h->mixed;
    if (!M) return;
    mixed_destroy_graph(M);
    if (M->mem) cudaFreeAsync(M->mem, h->stream);
    delete M;
    h->mixed = nullptr;
}

namespace {

template <typename T>
static void mixed_build_t(uaamg_poisson* h) {
    MixedData* M = h->mixed;
    cudaStream_t s = h->stream;
    const int nlev = h->nlev;
    size_t bytes = 0;
    for (int l = 0; l < nlev; ++l) bytes += 8 * carve_size((size_t)h->lv[l].L.nl * UAAMG_LEAF, sizeof(T));
    const int nc = h->C.n;
    bytes += carve_size((size_t)nc * nc, 8) + 2 * carve_size((size_t)nc, 8) + carve_size(4, 4) + carve_size(2, 8) +
             carve_size(1, 4);
    CK(ctx_dev_alloc(h->ctx, (void**)&M->mem, bytes, s));
    CK(cudaMemsetAsync(M->mem, 0, bytes, s));
    char* cur = M->mem;
    M->lv.assign(nlev, MixedLevel());
    for (int l = 0; l < nlev; ++l) {
        const LevelDev& D = h->lv[l];
        const size_t n = (size_t)D.L.nl * UAAMG_LEAF;
        MixedLevel& ML = M->lv[l];
        const float* src[5] = {D.L.diag, D.L.invdiag, D.L.cx, D.L.cy, D.L.cz};
        void** dst[5] = {&ML.diag, &ML.invdiag, &ML.cx, &ML.cy, &ML.cz};
        const float cs = level_scale(D.L);
        for (int a = 0; a < 5; ++a) {
            *dst[a] = carve<T>(cur, n);
            const long long n4 = (long long)n / 4;
            if (n4) {
                k_mconvert<T><<<(unsigned)((n4 + 255) / 256), 256, 0, s>>>(src[a], (T*)*dst[a], n4,
                                                                           a == 1 ? cs : 1.0f / cs);
                CHECK_LAUNCH();
            }
        }
        ML.lhs = carve<T>(cur, n);
        ML.rhs = carve<T>(cur, n);
        ML.tmp = carve<T>(cur, n);
    }
    M->nc = nc;
    M->ainv = carve<double>(cur, (size_t)nc * nc);
    double* fcol = carve<double>(cur, (size_t)nc);
    double* rrow = carve<double>(cur, (size_t)nc);
    int* err = carve<int>(cur, 4);
    M->res64 = carve<unsigned long long>(cur, 2);
    M->sigma = carve<float>(cur, 1);
    if (nc > 0) {
        k_cdense<<<(unsigned)nc, 256, 0, s>>>(h->C, M->ainv);
        CHECK_LAUNCH();
        const unsigned gp = (unsigned)((nc + 255) / 256);
        const unsigned gu = (unsigned)(((long long)nc * nc + 255) / 256);
        for (int k = 0; k < nc; ++k) {
            k_gj_pivot<<<gp, 256, 0, s>>>(M->ainv, nc, k, fcol, rrow, err);
            k_gj_update<<<gu, 256, 0, s>>>(M->ainv, nc, k, fcol, rrow);
        }
        CHECK_LAUNCH();
        int herr = 0;
        CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (herr) {
            set_error("the coarsest matrix is not positive definite (a domain without free surface?): "
                      "no FP64 direct coarsest solve");
            throw UaamgError{UAAMG_ERR_INVALID_ARGUMENT};
        }
    }
}

static void mixed_prepare(uaamg_poisson* h, int precision) {
    require(precision == UAAMG_PRECISION_FP16 || precision == UAAMG_PRECISION_BF16, "precision must be FP16 or BF16");
    require(h->smoother == UAAMG_SMOOTHER_SCHEDULED_RELAXED_JACOBI || h->smoother == UAAMG_SMOOTHER_WEIGHTED_JACOBI,
            "the mixed-precision form runs the Jacobi smoothers");
    if (h->mixed && h->mixed->precision == precision) return;
    mixed_free(h);
    const double t0 = trace_now();
    h->mixed = new MixedData();
    h->mixed->precision = precision;
    try {
        if (precision == UAAMG_PRECISION_FP16) mixed_build_t<__half>(h);
        else mixed_build_t<__nv_bfloat16>(h);
        CK(cudaStreamSynchronize(h->stream));
    } catch (...) {
        mixed_free(h);
        throw;
    }
    h->mixed->setup_ms = trace_now() - t0;
}

struct MEnq {
    uaamg_poisson* h;
    cudaStream_t s;
    int64_t count = 0;
    std::vector<ProfRec>* prof = nullptr;

    void pb(const char* what, int l) {
        if (!prof) return;
        ProfRec r;
        r.label = "L" + std::to_string(l) + " " + what;
        CK(cudaEventCreate(&r.a));
        CK(cudaEventCreate(&r.b));
        CK(cudaEventRecord(r.a, s));
        prof->push_back(r);
    }
    void pe() {
        if (prof) CK(cudaEventRecord(prof->back().b, s));
        count++;
    }
    template <typename... KArgs, typename... Args>
    void run(const char* what, int l, void (*kern)(KArgs...), unsigned g, unsigned b, Args... args) {
        pb(what, l);
        launch(kern, g, b, s, args...);
        pe();
    }
    template <typename... KArgs, typename... Args>
    void run_pipe(const char* what, int l, void (*kern)(KArgs...), int nl, size_t smem, Args... args) {
        pb(what, l);
        launch_pipe(kern, nl, smem, s, args...);
        pe();
    }
};

// muCyclePreconditioner<2, skip_first> (simd_vdb_poisson.cpp:1844-1977) on
// the 16-bit hierarchy: the launch sequence of enqueue_precond for the Jacobi
// smoothers; at level 0 the rhs is the 16-bit copy of the CG residual and the
// last sweep writes z in FP32 together with z.r.  Levels of at least
// STAGED_MIN_LEAVES leaves sweep with the staged kernels, and from
// SPLIT_MIN_LEAVES on the first sweep's source and the prolongation-add are
// stored first (k_mmaterialize) so that every sweep is a staged plain one.
template <typename T>
static void menq_visit(MEnq& E, int l, bool skip_first, DotOut dot, float* z) {
    uaamg_poisson* h = E.h;
    MixedData* M = h->mixed;
    const int last = h->nlev - 1;
    const MLevel<T> L = mlevel<T>(h, l);
    T* lhs = (T*)M->lv[l].lhs;
    T* rhs = (T*)M->lv[l].rhs;
    T* tmp = (T*)M->lv[l].tmp;
    const unsigned g = (unsigned)L.nl;
    const DotOut nodot{nullptr, nullptr, nullptr};
    const float* ns = nullptr;
    if (l == last) {
        if (M->nc > 0) {
            const unsigned rows = (unsigned)((M->nc + 7) / 8);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(rows);
            cfg.blockDim = dim3(256);
            cfg.dynamicSmemBytes = (size_t)M->nc * sizeof(double);
            cfg.stream = E.s;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            E.pb("coarsest fp64 gemv", l);
            CK(cudaLaunchKernelEx(&cfg, k_cgemv<T>, M->nc, (const double*)M->ainv, (const int*)h->C.dof_slot,
                                  (const T*)rhs, lhs, L.cs));
            E.pe();
        }
        return;
    }
    const int sm = h->smoother;
    auto wpre = [&](int i) { return sm == UAAMG_SMOOTHER_WEIGHTED_JACOBI ? 6.0f / 7.0f : sched_weight_precond(3, i); };
    const bool staged = g_use_staged && L.nl >= STAGED_MIN_LEAVES;
    const bool split = g_use_staged && L.nl >= SPLIT_MIN_LEAVES;
    int* err = &h->st->error;
    const size_t psm = pipe_smem_bytes<MLevel<T>>();
    const bool pipe = staged && L.nl >= PIPE_DOT_MIN_LEAVES;
    auto sweep = [&](const T* x, T* out, float w) {  // plain source
        if (pipe)
            E.run_pipe("jacobi staged", l, k_pipe<M_JACOBI, MLevel<T>, T, false>, L.nl, psm, L, x, (const T*)rhs, out,
                       w, 0.f, 0.f, nodot, ns, 0.f, err);
        else if (staged)
            E.run("jacobi staged", l, k_msweep_staged<T, T>, g, 128, L, x, (const T*)rhs, out, w, nodot, ns, err);
        else
            E.run("jacobi", l, k_msweep<T, T, MSrcPlain<T>>, g, 128, L, MSrcPlain<T>{x}, (const T*)rhs, out, w, nodot,
                  ns);
    };
    if (skip_first) {
        if (split) {
            E.run("materialize first", l, k_mmaterialize<T, MSrcFirstJacobi<T>>, elem_grid(L.nl), 128, L,
                  MSrcFirstJacobi<T>{rhs, wpre(0)}, tmp);
            sweep(tmp, lhs, wpre(1));
        } else {
            E.run("jacobi first", l, k_msweep<T, T, MSrcFirstJacobi<T>>, g, 128, L, MSrcFirstJacobi<T>{rhs, wpre(0)},
                  (const T*)rhs, lhs, wpre(1), nodot, ns);
        }
        sweep(lhs, tmp, wpre(2));
    } else {
        sweep(lhs, tmp, wpre(0));
        sweep(tmp, lhs, wpre(1));
        sweep(lhs, tmp, wpre(2));
    }
    const float cics = 1.0f / level_scale(h->lv[l + 1].L);
    T* crhs = (T*)M->lv[l + 1].rhs;
    if (pipe)  // the pipelined kernel computes in stored units: its scale is cs / cs'
        E.run_pipe("restrict staged", l, k_pipe<M_RESIDUAL, MLevel<T>, T, true>, L.nl, psm, L, (const T*)tmp,
                   (const T*)rhs, crhs, 0.f, 0.f, 0.f, nodot, ns, L.cs * cics, err);
    else if (staged)
        E.run("restrict staged", l, k_mrestrict_staged<T>, g, 128, L, (const T*)tmp, (const T*)rhs, crhs, cics, err);
    else
        E.run("restrict", l, k_mrestrict<T>, g, 128, L, (const T*)tmp, (const T*)rhs, crhs, cics);
    menq_visit<T>(E, l + 1, true, nodot, nullptr);
    if (l + 1 != last) menq_visit<T>(E, l + 1, false, nodot, nullptr);
    const T* clhs = (const T*)M->lv[l + 1].lhs;
    if (split) {  // tmp += P x_c in place (tmp is rewritten before it is read again)
        E.run("materialize prolong", l, k_mmaterialize<T, MSrcProlong<T>>, elem_grid(L.nl), 128, L,
              MSrcProlong<T>{tmp, clhs}, tmp);
        sweep(tmp, lhs, wpre(2));
    } else {
        E.run("jacobi prolong", l, k_msweep<T, T, MSrcProlong<T>>, g, 128, L, MSrcProlong<T>{tmp, clhs},
              (const T*)rhs, lhs, wpre(2), nodot, ns);
    }
    sweep(lhs, tmp, wpre(1));
    if (l == 0) {
        if (pipe)
            E.run_pipe("jacobi staged to fp32 +dot", l, k_pipe<M_JACOBI, MLevel<T>, float, false>, L.nl, psm, L,
                       (const T*)tmp, (const T*)rhs, z, wpre(0), 0.f, 0.f, dot, (const float*)M->sigma, 0.f, err);
        else if (staged)
            E.run("jacobi staged to fp32 +dot", l, k_msweep_staged<T, float>, g, 128, L, (const T*)tmp,
                  (const T*)rhs, z, wpre(0), dot, (const float*)M->sigma, err);
        else
            E.run("jacobi to fp32 +dot", l, k_msweep<T, float, MSrcPlain<T>>, g, 128, L, MSrcPlain<T>{tmp},
                  (const T*)rhs, z, wpre(0), dot, (const float*)M->sigma);
    } else {
        sweep(tmp, lhs, wpre(0));
    }
}

template <typename T>
static void menq_precond(MEnq& E) {
    uaamg_poisson* h = E.h;
    MixedData* M = h->mixed;
    const LevelDev& D0 = h->lv[0];
    const unsigned g = (unsigned)D0.L.nl;
    const DotOut dot{h->r, h->partials, h->st};
    E.run("r to 16-bit", 0, k_mto16<T>, elem_grid((int)g), 128, mlevel<T>(h, 0), (const float*)h->r, (T*)M->lv[0].rhs,
          (const PcgState*)h->st, M->sigma);
    if (h->nlev == 1) {  // the coarsest solve is the whole preconditioner
        menq_visit<T>(E, 0, true, dot, h->z);
        E.run("z to fp32", 0, k_mfrom16<T>, g, 128, (const T*)M->lv[0].lhs, h->z, (const float*)M->sigma);
        E.run("dot z.r", 0, k_dot_rho, g, 128, D0.L, (const float*)h->z, (const float*)h->r, h->partials, h->st);
        return;
    }
    menq_visit<T>(E, 0, true, dot, h->z);
}

template <typename T>
static void menq_body(MEnq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_poisson* h = E.h;
    const LevelDev& D0 = h->lv[0];
    const unsigned g = (unsigned)D0.L.nl;
    menq_precond<T>(E);
    E.run("pcg update p", 0, k_pcg_update_p, g, 128, D0.L, (const float*)h->z, h->p, h->x, (const PcgState*)h->st);
    E.run("pcg replace", 0, k_pcg_replace, elem_grid((int)g), 128, D0.L, (const float*)h->x, (const float*)h->b, h->r,
          (const PcgState*)h->st, h->mixed->replace_every);
    E.pb("pcg Ap", 0);
    Enq A{h, E.s};
    enqueue_Ap(A);
    E.pe();
    E.run("pcg update r", 0, k_pcg_update_r, elem_grid((int)g), 128, D0.L, (const float*)h->q, h->r, h->partials, h->st, cond,
          use_cond);
}

template <typename T>
static void mixed_build_graph(uaamg_poisson* h) {
    MixedData* M = h->mixed;
    mixed_destroy_graph(M);
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    Enq S{h, h->stream};
    CK(cudaStreamBeginCaptureToGraph(h->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_setup(S, cond, 1);
        M->setup_launches = S.count;
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
        MEnq B{h, h->body_stream};
        CK(cudaStreamBeginCaptureToGraph(h->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        menq_body<T>(B, cond, 1);
        cudaGraph_t bodyout = nullptr;
        CK(cudaStreamEndCapture(h->body_stream, &bodyout));
        M->body_launches = B.count;
        Enq F{h, h->stream};
        enqueue_finish(F);
        M->finish_launches = F.count;
    } catch (...) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(h->stream, &dummy);
        cudaStreamEndCapture(h->body_stream, &dummy);
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(h->stream, &out));
    CK(cudaGraphInstantiate(&M->exec, g, 0));
    M->graph = g;
    M->graph_every = M->replace_every;
}

// x, b (h->x, h->b) on the device; returns the status.  With prof the loop
// is host-driven and every launch is timed with CUDA events.
static int mixed_run_pcg(uaamg_poisson* h, std::vector<ProfRec>* prof = nullptr) {
    MixedData* M = h->mixed;
    if (h->lv[0].L.nl == 0) {
        h->iterations = 0;
        h->final_residual = 0.f;
        return UAAMG_SUCCESS;
    }
    init_state(h);
    int64_t launches = 0;
    if (h->use_graph && !prof) {
        if (!M->exec || M->graph_every != M->replace_every) {
            if (M->precision == UAAMG_PRECISION_FP16) mixed_build_graph<__half>(h);
            else mixed_build_graph<__nv_bfloat16>(h);
        }
        CK(cudaGraphLaunch(M->exec, h->stream));
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        launches = M->setup_launches + (int64_t)h->st_host->iter * M->body_launches + M->finish_launches;
    } else {  // host-driven loop (diagnostics: every kernel a separate launch)
        Enq S{h, h->stream};
        S.prof = prof;
        enqueue_setup(S, 0, 0);
        CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        MEnq B{h, h->stream};
        B.prof = prof;
        while (h->st_host->status == PCG_RUNNING) {
            if (M->precision == UAAMG_PRECISION_FP16) menq_body<__half>(B, 0, 0);
            else menq_body<__nv_bfloat16>(B, 0, 0);
            CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(PcgState), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        Enq F{h, h->stream};
        F.prof = prof;
        enqueue_finish(F);
        CK(cudaStreamSynchronize(h->stream));
        launches = S.count + B.count + F.count;
    }
    const PcgState& s = *h->st_host;
    h->last_launches = launches;
    h->launches += launches;
    if (s.error) {
        set_error("a kernel's bounded wait for its bulk copies timed out");
        throw UaamgError{UAAMG_ERR_CUDA};
    }
    h->iterations = s.iterations_taken;
    h->final_residual = s.nu;
    return (s.status == PCG_SUCCESS) ? UAAMG_SUCCESS : UAAMG_FAILED;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI (mixed-precision form)

int uaamg_poisson_prepare_mixed(uaamg_poisson* h, int precision, double* setup_ms) {
    ABI_BEGIN
    require(h != nullptr, "NULL handle");
    mixed_prepare(h, precision);
    if (setup_ms) *setup_ms = h->mixed->setup_ms;
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_set_residual_replacement(uaamg_poisson* h, int every) {
    if (!h || every < 1) { set_error("NULL handle or interval < 1"); return UAAMG_ERR_INVALID_ARGUMENT; }
    h->replace_every = every;
    if (h->mixed) h->mixed->replace_every = every;
    return UAAMG_SUCCESS;
}

int uaamg_poisson_solve_pcg_mixed_device(uaamg_poisson* h, int precision, float* d_pressure, const float* d_rhs,
                                         int* iterations) {
    ABI_BEGIN
    require(h && d_pressure && d_rhs, "NULL argument");
    mixed_prepare(h, precision);
    h->mixed->replace_every = h->replace_every;
    const size_t nb = vec_bytes(h, 0);
    if (nb) {
        if (d_pressure != h->x) CK(cudaMemcpyAsync(h->x, d_pressure, nb, cudaMemcpyDeviceToDevice, h->stream));
        if (d_rhs != h->b) CK(cudaMemcpyAsync(h->b, d_rhs, nb, cudaMemcpyDeviceToDevice, h->stream));
    }
    const int st = mixed_run_pcg(h);
    if (nb && d_pressure != h->x) {
        CK(cudaMemcpyAsync(d_pressure, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}

int uaamg_poisson_solve_pcg_mixed(uaamg_poisson* h, int precision, float* pressure, const float* rhs,
                                  int* iterations) {
    ABI_BEGIN
    require(h && pressure && rhs, "NULL argument");
    mixed_prepare(h, precision);
    h->mixed->replace_every = h->replace_every;
    const size_t nb = vec_bytes(h, 0);
    if (nb) {
        CK(cudaMemcpyAsync(h->x, pressure, nb, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->b, rhs, nb, cudaMemcpyHostToDevice, h->stream));
    }
    const int st = mixed_run_pcg(h);
    if (nb) {
        CK(cudaMemcpyAsync(pressure, h->x, nb, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (iterations) *iterations = h->iterations;
    return st;
    ABI_END
}

int uaamg_poisson_true_residual_fp64(uaamg_poisson* h, const float* d_x, const float* d_b, double* out) {
    ABI_BEGIN
    require(h && d_x && d_b && out, "NULL argument");
    const LevelDev& D0 = h->lv[0];
    out[0] = out[1] = 0.0;
    if (D0.L.nl == 0) return UAAMG_SUCCESS;
    unsigned long long* buf = nullptr;
    if (h->mixed) {
        buf = h->mixed->res64;
    } else {
        CK(ctx_dev_alloc(h->ctx, (void**)&buf, 16, h->stream));
    }
    CK(cudaMemsetAsync(buf, 0, 16, h->stream));
    k_res64<<<(unsigned)D0.L.nl, 128, 0, h->stream>>>(D0.L, d_x, d_b, buf);
    CHECK_LAUNCH();
    unsigned long long hb[2];
    CK(cudaMemcpyAsync(hb, buf, 16, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (!h->mixed) CK(cudaFreeAsync(buf, h->stream));
    memcpy(&out[0], &hb[0], 8);
    memcpy(&out[1], &hb[1], 8);
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_poisson_profile_pcg_mixed(uaamg_poisson* h, int precision, float* d_pressure, const float* d_rhs,
                                    int max_classes, char* names, double* total_ms, int64_t* counts, int* nclasses) {
    ABI_BEGIN
    require(h && d_pressure && d_rhs && names && total_ms && counts && nclasses, "NULL argument");
    *nclasses = 0;
    mixed_prepare(h, precision);
    h->mixed->replace_every = h->replace_every;
    const size_t nb = vec_bytes(h, 0);
    if (!nb) return UAAMG_SUCCESS;
    CK(cudaMemcpyAsync(h->x, d_pressure, nb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->b, d_rhs, nb, cudaMemcpyDeviceToDevice, h->stream));
    std::vector<ProfRec> prof;
    const int st = mixed_run_pcg(h, &prof);
    prof_collect(prof, max_classes, names, total_ms, counts, nclasses);
    CK(cudaMemcpyAsync(d_pressure, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return st;
    ABI_END
}
