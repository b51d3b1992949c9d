// batch.cu -- many independent pressure-Poisson UAAMG-PCG solves in one CUDA
// graph launch (the batched form of PoissonSolver::solveMultigridPCG,
// SIMD_UAAMG/simd_vdb_poisson.cpp:2155-2226).
//
// A batch references existing solver handles (uaamg_poisson), each with its
// own hierarchy of any depth, and runs all their W-cycles and CG steps
// together: every kernel launch of the batched cycle covers the leaves of
// every instance that has work at that point, so the launch and latency cost
// of a cycle is that of the deepest instance, not the sum over instances.
//
// Device side
//  * a record per (depth, instance) (BRec): the instance's level (DLevel),
//    its vectors by role, its coarsest system, PCG state and partials;
//  * block maps: entry k of a map is the (instance, leaf) that CTA k works
//    on; one map for level 0 of all instances and one per depth d for the
//    instances that smooth there (hierarchy deeper than d);
//  * per instance an "active" flag: an instance that has converged (or
//    stopped) skips all later work, while the graph's WHILE loop runs until
//    no instance is active.
// Every CTA runs the same per-leaf device code as the single-instance
// kernels, and each reduction keeps the instance's leaf slots and order, so
// each instance's result, iteration count and status are bit-identical to its
// standalone solve.
#include <array>

namespace {

enum { BR_LHS = 0, BR_RHS, BR_TMP, BR_CLHS, BR_CRHS, BR_X, BR_B, BR_R, BR_Z, BR_P, BR_Q, BR_NROLE };

}  // namespace

struct BRec {  // one instance at one depth
    DLevel L;
    float* v[BR_NROLE];  // lhs, rhs, tmp of this level; lhs, rhs of the next; PCG vectors (depth 0)
    DCoarsest C;         // the instance's coarsest system (used at its last depth)
    PcgState* st;
    double* partials;
    int* spai0_ready;
    float w_sor;
    int pad_;
};

struct BGlobal {
    unsigned ticket;  // CTAs of the current launch that have finished
    int running;      // instances still iterating (after the last test)
};

namespace uaamg {

// After a CTA's own work: the CTA that finishes last in the launch refreshes
// the active flags from the instances' PCG states and sets the loop condition.
__device__ __forceinline__ void batch_refresh_active(const BRec* recs0, int n, unsigned* active, BGlobal* g,
                                                     cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ bool lastg;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned tk = atomicAdd(&g->ticket, 1u);
        lastg = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!lastg) return;
    __threadfence();
    int run = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const PcgState* st = recs0[i].st;
        const unsigned a = (st != nullptr && __ldcg(&st->status) == PCG_RUNNING) ? 1u : 0u;
        active[i] = a;
        run |= (int)a;
    }
    run = __syncthreads_or(run);
    if (threadIdx.x == 0) {
        g->running = run;
        g->ticket = 0;
        set_cond(cond, use_cond, run ? 1u : 0u);
    }
}

// The block map and the records do not change during a solve: they and the
// static stencil data load before the wait; the instance's active flag is
// read after it.
template <int MODE, int SRC>
__global__ void __launch_bounds__(128, 7) k_bsweep(const BRec* __restrict__ recs, const int2* __restrict__ map,
                                                const unsigned* active, int xr, int br, int outr,
                                                float w, float wsrc, int dot, int mark) {
    const int2 e = map[blockIdx.x];
    const BRec& R = recs[e.x];
    const DLevel& L = R.L;
    const float ws = R.w_sor;
    const DotOut d = dot ? DotOut{R.v[BR_R], R.partials, R.st} : DotOut{nullptr, nullptr, nullptr};
    int* ready = mark ? R.spai0_ready : nullptr;
    const float* b = R.v[br];
    float* out = R.v[outr];
    const unsigned* g = active + e.x;
    if (SRC == S_PLAIN)
        sweep_leaf<MODE, SrcPlain, true>(L, e.y, L.nl, SrcPlain{R.v[xr]}, b, out, w, ws, 1.0f - ws, d, ready, g);
    else if (SRC == S_FIRST_JACOBI)
        sweep_leaf<MODE, SrcFirstJacobi, true>(L, e.y, L.nl, SrcFirstJacobi{b, wsrc}, b, out, w, ws, 1.0f - ws, d,
                                               ready, g);
    else if (SRC == S_FIRST_SPAI0)
        sweep_leaf<MODE, SrcFirstSpai0, true>(L, e.y, L.nl, SrcFirstSpai0{b, R.spai0_ready}, b, out, w, ws,
                                              1.0f - ws, d, ready, g);
    else if (SRC == S_FIRST_RBGS)
        sweep_leaf<MODE, SrcFirstRbgs, true>(L, e.y, L.nl, SrcFirstRbgs{b, ws, 1}, b, out, w, ws, 1.0f - ws, d,
                                             ready, g);
    else
        sweep_leaf<MODE, SrcProlong, true>(L, e.y, L.nl, SrcProlong{R.v[xr], R.v[BR_CLHS], 1.0f}, b, out, w, ws,
                                           1.0f - ws, d, ready, g);
}

__global__ void __launch_bounds__(128, 7) k_brestrict(const BRec* __restrict__ recs, const int2* __restrict__ map,
                                                   const unsigned* active, int xr, int br) {
    const int2 e = map[blockIdx.x];
    const BRec& R = recs[e.x];
    restrict_leaf<true, true>(R.L, e.y, R.v[xr], R.v[br], R.v[BR_CRHS], active + e.x);
}

template <int ROWS, int NT>
__global__ void __launch_bounds__(NT, 1) k_bcoarsest(const BRec* __restrict__ recs, const int* __restrict__ list,
                                                     const unsigned* __restrict__ active, int br, int outr) {
    griddep_wait();
    griddep_launch();
    __shared__ float ps[NT * ROWS + 4];
    __shared__ __align__(16) float red[3][64];
    const int i = list[blockIdx.x];
    if (!active[i]) return;
    const BRec& R = recs[i];
    coarsest_cg_body<ROWS, NT, false>(R.C, R.v[br], R.v[outr], ps, red);
}

__global__ void __launch_bounds__(128) k_bdot_rho(const BRec* __restrict__ recs, const int2* __restrict__ map,
                                                  const unsigned* __restrict__ active) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    if (!active[e.x]) return;
    const BRec& R = recs[e.x];
    dot_rho_leaf(R.L, e.y, R.L.nl, R.v[BR_Z], R.v[BR_R], R.partials, R.st);
}

// PoissonSolver state of every instance reset for a new solve
__global__ void k_binit(const BRec* __restrict__ recs0, int n, float tol, int max_iter, BGlobal* g) {
    griddep_wait();
    griddep_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        g->ticket = 0;
        g->running = 0;
    }
    if (i >= n) return;
    PcgState* st = recs0[i].st;
    if (!st) return;
    PcgState s;
    memset(&s, 0, sizeof(s));
    s.tol = tol;
    s.max_iter = max_iter;
    *st = s;
}

// x and b from the caller's vectors, zero off the DOF; p = 0
__global__ void __launch_bounds__(128) k_bload(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                               const float* const* __restrict__ ux,
                                               const float* const* __restrict__ ub) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    const BRec& R = recs0[e.x];
    const int t = threadIdx.x;
    st4(R.v[BR_X], e.y, t, masked4(R.L, e.y, ld4(ux[e.x], e.y, t)));
    st4(R.v[BR_B], e.y, t, masked4(R.L, e.y, ld4(ub[e.x], e.y, t)));
    st4(R.v[BR_P], e.y, t, f4zero());
}

__global__ void __launch_bounds__(128) k_bpcg_init(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                                   int n, unsigned* active, BGlobal* g,
                                                   cudaGraphConditionalHandle cond, int use_cond) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    const BRec& R = recs0[e.x];
    pcg_init_leaf(R.L, e.y, R.L.nl, R.v[BR_X], R.v[BR_B], R.v[BR_R], R.partials, R.st, 0, 0);
    batch_refresh_active(recs0, n, active, g, cond, use_cond);
}

__global__ void __launch_bounds__(128) k_bpcg_update_p(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                                       const unsigned* __restrict__ active) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    if (!active[e.x]) return;
    const BRec& R = recs0[e.x];
    pcg_update_p_leaf(e.y, R.v[BR_Z], R.v[BR_P], R.v[BR_X], R.st);
}

__global__ void __launch_bounds__(128) k_bpcg_Ap(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                                 const unsigned* __restrict__ active) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    if (!active[e.x]) return;
    const BRec& R = recs0[e.x];
    pcg_Ap_leaf(R.L, e.y, R.L.nl, R.v[BR_P], R.v[BR_Q], R.partials, R.st);
}

__global__ void __launch_bounds__(128) k_bpcg_update_r(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                                       int n, unsigned* active, BGlobal* g,
                                                       cudaGraphConditionalHandle cond, int use_cond) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    if (active[e.x]) {
        const BRec& R = recs0[e.x];
        pcg_update_r_leaf(e.y, R.L.nl, R.v[BR_Q], R.v[BR_R], R.partials, R.st, 0, 0);
    }
    batch_refresh_active(recs0, n, active, g, cond, use_cond);
}

// the last x update (k_pcg_finish) written straight into the caller's vector
__global__ void __launch_bounds__(128) k_bpcg_finish(const BRec* __restrict__ recs0, const int2* __restrict__ map,
                                                     float* const* __restrict__ ux) {
    griddep_wait();
    griddep_launch();
    const int2 e = map[blockIdx.x];
    const BRec& R = recs0[e.x];
    const bool apply = pcg_finish_applies(R.st);
    st4(ux[e.x], e.y, threadIdx.x, pcg_finish_value(e.y, R.v[BR_P], R.v[BR_X], R.st, apply));
}

__global__ void k_bstates(const BRec* __restrict__ recs0, int n, PcgState* out) {
    griddep_wait();
    griddep_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (recs0[i].st) out[i] = *recs0[i].st;
    else memset(&out[i], 0, sizeof(PcgState));
}

}  // namespace uaamg

struct uaamg_batch {
    DeviceCtx* ctx = nullptr;
    cudaStream_t own_stream = nullptr, body_stream = nullptr, stream = nullptr;
    std::vector<uaamg_poisson*> inst;
    std::vector<cudaEvent_t> ev;
    int n = 0, depth = 0;
    int smoother = UAAMG_SMOOTHER_SCHEDULED_RELAXED_JACOBI, max_iter = 100;
    float rel_tol = 1e-7f;
    int use_graph = 1;
    int64_t solves = 0;
    // device tables (one allocation)
    char* dmem = nullptr;
    BRec* recs = nullptr;  // [depth][n]
    int2* maps = nullptr;
    int* lists = nullptr;
    unsigned* active = nullptr;
    float** ux = nullptr;
    const float** ub = nullptr;
    BGlobal* g = nullptr;
    PcgState* states = nullptr;
    // pinned staging: records, pointer arrays, states
    void* pin = nullptr;
    size_t pin_cap = 0;
    struct Range {
        int off = 0, count = 0;
    };
    Range all0, dot1;
    std::vector<Range> smooth;                  // [depth]
    std::vector<std::array<Range, 3>> coarse;   // [depth][ROWS 1, 2, 4]
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_key = -1;
    int64_t setup_launches = 0, body_launches = 0, finish_launches = 0;
    int64_t launches = 0, last_launches = 0;
    std::vector<int> iterations, status;
    std::vector<float> residual;
};

namespace {

struct BEnq {
    uaamg_batch* b;
    cudaStream_t s;
    int64_t count = 0;
    const BRec* recs(int d) const { return b->recs + (size_t)d * b->n; }
    const int2* map(const uaamg_batch::Range& r) const { return b->maps + r.off; }
    bool smooths(int d) const { return d < (int)b->smooth.size() && b->smooth[d].count > 0; }

    template <int MODE, int SRC>
    void sweep(int d, int xr, int br, int outr, float w, float wsrc = 0.f, int dot = 0, int mark = 0) {
        const uaamg_batch::Range& r = b->smooth[d];
        launch(k_bsweep<MODE, SRC>, (unsigned)r.count, 128, s, recs(d), map(r), (const unsigned*)b->active, xr, br,
               outr, w, wsrc, dot, mark);
        count++;
    }
    void restrict_resid(int d, int xr, int br) {
        const uaamg_batch::Range& r = b->smooth[d];
        launch(k_brestrict, (unsigned)r.count, 128, s, recs(d), map(r), (const unsigned*)b->active, xr, br);
        count++;
    }
    // coarsest solves of the instances whose hierarchy ends at depth d (rows
    // per thread as in the single solve), then z.r for one-level hierarchies
    void coarsest(int d, int br, int outr, bool dot) {
        const std::array<uaamg_batch::Range, 3>& c = b->coarse[d];
        const unsigned* act = b->active;
        if (c[0].count) launch(k_bcoarsest<2, 512>, (unsigned)c[0].count, 512, s, recs(d), b->lists + c[0].off, act, br, outr);
        if (c[1].count) launch(k_bcoarsest<4, 512>, (unsigned)c[1].count, 512, s, recs(d), b->lists + c[1].off, act, br, outr);
        if (c[2].count) launch(k_bcoarsest<4, 1024>, (unsigned)c[2].count, 1024, s, recs(d), b->lists + c[2].off, act, br, outr);
        count += (c[0].count > 0) + (c[1].count > 0) + (c[2].count > 0);
        if (dot && d == 0 && b->dot1.count) {
            launch(k_bdot_rho, (unsigned)b->dot1.count, 128, s, recs(0), map(b->dot1), act);
            count++;
        }
    }
};

// muCyclePreconditioner<2, skip_first> (simd_vdb_poisson.cpp:1844-1977) over
// every instance at depth d: the same launch sequence as enqueue_precond,
// with vectors named by role.  lhs/rhs are BR_Z/BR_R at depth 0.
static void benqueue_precond(BEnq& E, int d, int lhs, int rhs, bool skip_first, bool dot) {
    uaamg_batch* b = E.b;
    if (skip_first) E.coarsest(d, rhs, lhs, dot);
    if (!E.smooths(d)) return;
    const int n = 3;
    const int sm = b->smoother;
    const int T = BR_TMP;
    auto wpre = [&](int i) { return sm == UAAMG_SMOOTHER_WEIGHTED_JACOBI ? 6.0f / 7.0f : sched_weight_precond(n, i); };
    auto recurse = [&]() {
        E.restrict_resid(d, sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL ? lhs : T, rhs);
        benqueue_precond(E, d + 1, BR_LHS, BR_RHS, true, false);
        if (E.smooths(d + 1)) benqueue_precond(E, d + 1, BR_LHS, BR_RHS, false, false);
    };
    if (sm == UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL) {
        int i0 = 0;
        if (skip_first) {
            E.sweep<M_BLACK, S_FIRST_RBGS>(d, lhs, rhs, lhs, 0.f);
            i0 = 1;
        }
        for (int i = i0; i < n; ++i) {
            E.sweep<M_RED, S_PLAIN>(d, lhs, rhs, lhs, 0.f);
            E.sweep<M_BLACK, S_PLAIN>(d, lhs, rhs, lhs, 0.f);
        }
        recurse();
        E.sweep<M_BLACK, S_PROLONG>(d, lhs, rhs, T, 0.f);
        for (int i = 0; i < n; ++i) {
            if (i > 0) E.sweep<M_BLACK, S_PLAIN>(d, T, rhs, T, 0.f);
            if (i < n - 1) E.sweep<M_RED, S_PLAIN>(d, T, rhs, T, 0.f);
            else E.sweep<M_RED, S_PLAIN>(d, T, rhs, lhs, 0.f, 0.f, dot ? 1 : 0);
        }
        return;
    }
    const bool spai = (sm == UAAMG_SMOOTHER_SPAI0);
    if (skip_first) {
        if (spai) E.sweep<M_SPAI0, S_FIRST_SPAI0>(d, lhs, rhs, lhs, 0.f);
        else E.sweep<M_JACOBI, S_FIRST_JACOBI>(d, lhs, rhs, lhs, wpre(1), wpre(0));
        if (spai) E.sweep<M_SPAI0, S_PLAIN>(d, lhs, rhs, T, 0.f, 0.f, 0, 1);
        else E.sweep<M_JACOBI, S_PLAIN>(d, lhs, rhs, T, wpre(2));
    } else {
        if (spai) {
            E.sweep<M_SPAI0, S_PLAIN>(d, lhs, rhs, T, 0.f, 0.f, 0, 1);
            E.sweep<M_SPAI0, S_PLAIN>(d, T, rhs, lhs, 0.f);
            E.sweep<M_SPAI0, S_PLAIN>(d, lhs, rhs, T, 0.f);
        } else {
            E.sweep<M_JACOBI, S_PLAIN>(d, lhs, rhs, T, wpre(0));
            E.sweep<M_JACOBI, S_PLAIN>(d, T, rhs, lhs, wpre(1));
            E.sweep<M_JACOBI, S_PLAIN>(d, lhs, rhs, T, wpre(2));
        }
    }
    recurse();
    if (spai) {
        E.sweep<M_SPAI0, S_PROLONG>(d, T, rhs, lhs, 0.f);
        E.sweep<M_SPAI0, S_PLAIN>(d, lhs, rhs, T, 0.f);
        E.sweep<M_SPAI0, S_PLAIN>(d, T, rhs, lhs, 0.f, 0.f, dot ? 1 : 0);
    } else {
        E.sweep<M_JACOBI, S_PROLONG>(d, T, rhs, lhs, wpre(2));
        E.sweep<M_JACOBI, S_PLAIN>(d, lhs, rhs, T, wpre(1));
        E.sweep<M_JACOBI, S_PLAIN>(d, T, rhs, lhs, wpre(0), 0.f, dot ? 1 : 0);
    }
}

static void benqueue_setup(BEnq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_batch* b = E.b;
    launch(k_binit, (unsigned)((b->n + 127) / 128), 128, E.s, E.recs(0), b->n, b->rel_tol, b->max_iter, b->g);
    launch(k_bload, (unsigned)b->all0.count, 128, E.s, E.recs(0), E.map(b->all0), (const float* const*)b->ux,
           (const float* const*)b->ub);
    launch(k_bpcg_init, (unsigned)b->all0.count, 128, E.s, E.recs(0), E.map(b->all0), b->n, b->active, b->g, cond,
           use_cond);
    E.count += 3;
}
static void benqueue_body(BEnq& E, cudaGraphConditionalHandle cond, int use_cond) {
    uaamg_batch* b = E.b;
    benqueue_precond(E, 0, BR_Z, BR_R, true, true);
    const unsigned g0 = (unsigned)b->all0.count;
    launch(k_bpcg_update_p, g0, 128, E.s, E.recs(0), E.map(b->all0), (const unsigned*)b->active);
    launch(k_bpcg_Ap, g0, 128, E.s, E.recs(0), E.map(b->all0), (const unsigned*)b->active);
    launch(k_bpcg_update_r, g0, 128, E.s, E.recs(0), E.map(b->all0), b->n, b->active, b->g, cond, use_cond);
    E.count += 3;
}
static void benqueue_finish(BEnq& E) {
    uaamg_batch* b = E.b;
    launch(k_bpcg_finish, (unsigned)b->all0.count, 128, E.s, E.recs(0), E.map(b->all0), (float* const*)b->ux);
    launch(k_bstates, (unsigned)((b->n + 127) / 128), 128, E.s, E.recs(0), b->n, b->states);
    E.count += 2;
}

static void bdestroy_graph(uaamg_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_key = -1;
}

static void bbuild_graph(uaamg_batch* b) {
    bdestroy_graph(b);
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    BEnq E{b, b->stream};
    CK(cudaStreamBeginCaptureToGraph(b->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        benqueue_setup(E, cond, 1);
        b->setup_launches = E.count;
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraph_t cg = nullptr;
        CK(cudaStreamGetCaptureInfo(b->stream, &cs, nullptr, &cg, &deps, &ndeps));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t wnode;
        CK(cudaGraphAddNode(&wnode, cg, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(b->stream, &wnode, 1, cudaStreamSetCaptureDependencies));
        BEnq B{b, b->body_stream};
        CK(cudaStreamBeginCaptureToGraph(b->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        benqueue_body(B, cond, 1);
        cudaGraph_t bodyout = nullptr;
        CK(cudaStreamEndCapture(b->body_stream, &bodyout));
        b->body_launches = B.count;
        BEnq F{b, b->stream};
        benqueue_finish(F);
        b->finish_launches = F.count;
    } catch (...) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(b->stream, &dummy);
        cudaStreamEndCapture(b->body_stream, &dummy);
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(b->stream, &out));
    CK(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph = g;
    b->graph_key = b->smoother;
}

static size_t bpin_records_bytes(const uaamg_batch* b) { return (size_t)b->depth * b->n * sizeof(BRec); }

// The per-(depth, instance) records from the instances' current state.
static void bfill_records(uaamg_batch* b, BRec* out) {
    memset(out, 0, bpin_records_bytes(b));
    for (int i = 0; i < b->n; ++i) {
        uaamg_poisson* h = b->inst[i];
        if (h->lv.empty() || h->lv[0].L.nl == 0) continue;
        for (int d = 0; d < h->nlev; ++d) {
            BRec& R = out[(size_t)d * b->n + i];
            LevelDev& D = h->lv[d];
            R.L = D.L;
            R.v[BR_LHS] = D.lhs;
            R.v[BR_RHS] = D.rhs;
            R.v[BR_TMP] = D.tmp;
            if (d + 1 < h->nlev) {
                R.v[BR_CLHS] = h->lv[d + 1].lhs;
                R.v[BR_CRHS] = h->lv[d + 1].rhs;
            }
            R.v[BR_X] = h->x;
            R.v[BR_B] = h->b;
            R.v[BR_R] = h->r;
            R.v[BR_Z] = h->z;
            R.v[BR_P] = h->p;
            R.v[BR_Q] = h->q;
            R.C = h->C;
            R.st = h->st;
            R.partials = h->partials;
            R.spai0_ready = D.spai0_ready;
            R.w_sor = D.w_sor;
        }
    }
}

// Block maps and coarsest lists from the instances' hierarchies.
static void bbuild_tables(uaamg_batch* b) {
    const int n = b->n;
    b->depth = 1;
    for (uaamg_poisson* h : b->inst)
        if (!h->lv.empty() && h->lv[0].L.nl > 0) b->depth = std::max(b->depth, h->nlev);
    std::vector<int2> maps;
    std::vector<int> lists;
    auto add_map = [&](auto&& pick, uaamg_batch::Range& r, auto&& level_of) {
        r.off = (int)maps.size();
        for (int i = 0; i < n; ++i) {
            uaamg_poisson* h = b->inst[i];
            if (h->lv.empty() || h->lv[0].L.nl == 0 || !pick(h)) continue;
            const int nl = h->lv[level_of(h)].L.nl;
            for (int leaf = 0; leaf < nl; ++leaf) maps.push_back(make_int2(i, leaf));
        }
        r.count = (int)maps.size() - r.off;
    };
    add_map([](uaamg_poisson*) { return true; }, b->all0, [](uaamg_poisson*) { return 0; });
    add_map([](uaamg_poisson* h) { return h->nlev == 1; }, b->dot1, [](uaamg_poisson*) { return 0; });
    b->smooth.assign(b->depth, uaamg_batch::Range());
    b->coarse.assign(b->depth, std::array<uaamg_batch::Range, 3>());
    for (int d = 0; d < b->depth; ++d) {
        add_map([d](uaamg_poisson* h) { return h->nlev - 1 > d; }, b->smooth[d], [d](uaamg_poisson*) { return d; });
        for (int k = 0; k < 3; ++k) {
            uaamg_batch::Range& r = b->coarse[d][k];
            r.off = (int)lists.size();
            for (int i = 0; i < n; ++i) {
                uaamg_poisson* h = b->inst[i];
                if (h->lv.empty() || h->lv[0].L.nl == 0 || h->nlev - 1 != d || h->C.n == 0) continue;
                const int cls = coarsest_class(h->C.n);
                if (cls == k) lists.push_back(i);
            }
            r.count = (int)lists.size() - r.off;
        }
    }
    // one device allocation: records, maps, lists, active flags, pointer
    // arrays, global counters, gathered states
    const size_t nrec = (size_t)b->depth * n;
    size_t bytes = carve_size(nrec, sizeof(BRec)) + carve_size(std::max<size_t>(maps.size(), 1), sizeof(int2)) +
                   carve_size(std::max<size_t>(lists.size(), 1), 4) + carve_size(n, 4) + 2 * carve_size(n, 8) +
                   carve_size(1, sizeof(BGlobal)) + carve_size(n, sizeof(PcgState));
    CK(ctx_dev_alloc(b->ctx, (void**)&b->dmem, bytes, b->stream));
    CK(cudaMemsetAsync(b->dmem, 0, bytes, b->stream));
    char* cur = b->dmem;
    b->recs = carve<BRec>(cur, nrec);
    b->maps = carve<int2>(cur, std::max<size_t>(maps.size(), 1));
    b->lists = carve<int>(cur, std::max<size_t>(lists.size(), 1));
    b->active = carve<unsigned>(cur, n);
    b->ux = carve<float*>(cur, n);
    b->ub = carve<const float*>(cur, n);
    b->g = carve<BGlobal>(cur, 1);
    b->states = carve<PcgState>(cur, n);
    // pinned staging: records | ux | ub | states | tables (upload once)
    const size_t pin_bytes = bpin_records_bytes(b) + 2 * (size_t)n * 8 + (size_t)n * sizeof(PcgState) +
                             maps.size() * sizeof(int2) + lists.size() * 4 + 1024;
    CK(ctx_pinned_acquire(b->ctx, pin_bytes, &b->pin, &b->pin_cap));
    char* tab = (char*)b->pin + bpin_records_bytes(b) + 2 * (size_t)n * 8 + (size_t)n * sizeof(PcgState);
    tab = (char*)(((uintptr_t)tab + 255) & ~uintptr_t(255));
    if (!maps.empty()) {
        memcpy(tab, maps.data(), maps.size() * sizeof(int2));
        CK(cudaMemcpyAsync(b->maps, tab, maps.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
        tab += (maps.size() * sizeof(int2) + 255) & ~size_t(255);
    }
    if (!lists.empty()) {
        memcpy(tab, lists.data(), lists.size() * 4);
        CK(cudaMemcpyAsync(b->lists, tab, lists.size() * 4, cudaMemcpyHostToDevice, b->stream));
    }
}

static BRec* bpin_records(uaamg_batch* b) { return reinterpret_cast<BRec*>(b->pin); }
static float** bpin_ux(uaamg_batch* b) { return reinterpret_cast<float**>((char*)b->pin + bpin_records_bytes(b)); }
static const float** bpin_ub(uaamg_batch* b) {
    return reinterpret_cast<const float**>((char*)b->pin + bpin_records_bytes(b) + (size_t)b->n * 8);
}
static PcgState* bpin_states(uaamg_batch* b) {
    return reinterpret_cast<PcgState*>((char*)b->pin + bpin_records_bytes(b) + 2 * (size_t)b->n * 8);
}

// The instances' own pending work (hierarchy build, rhs, SPAI0 factors)
// comes before anything the batch enqueues.
static void bwait_instances(uaamg_batch* b) {
    for (int i = 0; i < b->n; ++i) {
        uaamg_poisson* h = b->inst[i];
        if (b->smoother == UAAMG_SMOOTHER_SPAI0 && !h->lv.empty() && h->lv[0].L.nl > 0) ensure_spai0(h);
        if (h->stream != b->stream) {
            CK(cudaEventRecord(b->ev[i], h->stream));
            CK(cudaStreamWaitEvent(b->stream, b->ev[i], 0));
        }
    }
}

// Solve every instance: x (in/out) and b are device vectors per instance.
static int brun_pcg(uaamg_batch* b, float* const* d_x, const float* const* d_b) {
    const int n = b->n;
    BRec* rec = bpin_records(b);
    bfill_records(b, rec);
    float** ux = bpin_ux(b);
    const float** ub = bpin_ub(b);
    for (int i = 0; i < n; ++i) {
        ux[i] = d_x[i];
        ub[i] = d_b[i];
    }
    CK(cudaMemcpyAsync(b->recs, rec, bpin_records_bytes(b), cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->ux, ux, (size_t)n * 8, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->ub, ub, (size_t)n * 8, cudaMemcpyHostToDevice, b->stream));
    int64_t launches = 0;
    PcgState* hs = bpin_states(b);
    // A batch's first solve runs host-driven, as a handle's does: a batch
    // formed for one solve (a served round whose set of requests changed)
    // would pay the graph's capture and instantiation for a single launch.
    const bool graph = b->use_graph == 2 || (b->use_graph == 1 && b->solves > 0);
    b->solves++;
    if (b->all0.count > 0) {
        if (graph) {
            if (!b->exec || b->graph_key != b->smoother) bbuild_graph(b);
            CK(cudaGraphLaunch(b->exec, b->stream));
            CK(cudaMemcpyAsync(hs, b->states, (size_t)n * sizeof(PcgState), cudaMemcpyDeviceToHost, b->stream));
            CK(cudaStreamSynchronize(b->stream));
            int body_runs = 0;
            for (int i = 0; i < n; ++i) body_runs = std::max(body_runs, hs[i].iter);
            launches = b->setup_launches + (int64_t)body_runs * b->body_launches + b->finish_launches;
        } else {
            BEnq E{b, b->stream};
            benqueue_setup(E, 0, 0);
            int running = 0;
            CK(cudaMemcpyAsync(&hs[0].status, &b->g->running, 4, cudaMemcpyDeviceToHost, b->stream));
            CK(cudaStreamSynchronize(b->stream));
            running = hs[0].status;
            while (running) {
                benqueue_body(E, 0, 0);
                CK(cudaMemcpyAsync(&hs[0].status, &b->g->running, 4, cudaMemcpyDeviceToHost, b->stream));
                CK(cudaStreamSynchronize(b->stream));
                running = hs[0].status;
            }
            benqueue_finish(E);
            CK(cudaMemcpyAsync(hs, b->states, (size_t)n * sizeof(PcgState), cudaMemcpyDeviceToHost, b->stream));
            CK(cudaStreamSynchronize(b->stream));
            launches = E.count;
        }
    }
    b->last_launches = launches;
    b->launches += launches;
    b->iterations.assign(n, 0);
    b->status.assign(n, UAAMG_SUCCESS);
    b->residual.assign(n, 0.f);
    int all = UAAMG_SUCCESS;
    for (int i = 0; i < n; ++i) {
        uaamg_poisson* h = b->inst[i];
        if (h->lv.empty() || h->lv[0].L.nl == 0) continue;
        const PcgState& s = hs[i];
        if (s.error) {
            set_error("instance %d: a kernel's bounded wait timed out", i);
            throw UaamgError{UAAMG_ERR_CUDA};
        }
        b->iterations[i] = s.iterations_taken;
        b->status[i] = (s.status == PCG_SUCCESS) ? UAAMG_SUCCESS : UAAMG_FAILED;
        b->residual[i] = s.nu;
        h->iterations = s.iterations_taken;
        h->final_residual = s.nu;
        h->solves++;
        if (b->status[i] != UAAMG_SUCCESS) all = UAAMG_FAILED;
    }
    return all;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI (batched form)

int uaamg_batch_create(int count, uaamg_poisson* const* instances, uaamg_batch** out) {
    ABI_BEGIN
    require(out != nullptr && count >= 1 && instances != nullptr, "NULL argument or empty batch");
    *out = nullptr;
    for (int i = 0; i < count; ++i) require(instances[i] != nullptr, "NULL instance handle");
    for (int i = 0; i < count; ++i)
        for (int j = 0; j < i; ++j) require(instances[i] != instances[j], "an instance appears twice in the batch");
    uaamg_batch* b = new uaamg_batch();
    try {
        cudaError_t ce;
        b->ctx = device_ctx(&ce);
        CK(ce);
        CK(ctx_stream_acquire(b->ctx, &b->own_stream));
        CK(ctx_stream_acquire(b->ctx, &b->body_stream));
        b->stream = b->own_stream;
        b->n = count;
        b->inst.assign(instances, instances + count);
        b->ev.assign(count, nullptr);
        for (int i = 0; i < count; ++i) CK(cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming));
        b->smoother = instances[0]->smoother;
        b->max_iter = instances[0]->max_iter;
        b->rel_tol = instances[0]->rel_tol;
        for (int i = 0; i < count; ++i) {
            uaamg_poisson* h = b->inst[i];
            if (h->stream != b->stream) {
                CK(cudaEventRecord(b->ev[i], h->stream));
                CK(cudaStreamWaitEvent(b->stream, b->ev[i], 0));
            }
        }
        bbuild_tables(b);
        CK(cudaStreamSynchronize(b->stream));
    } catch (...) {
        uaamg_batch_destroy(b);
        throw;
    }
    *out = b;
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_batch_destroy(uaamg_batch* b) {
    if (!b) return UAAMG_SUCCESS;
    if (b->stream) cudaStreamSynchronize(b->stream);
    bdestroy_graph(b);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->ctx) {
        if (b->dmem) cudaFreeAsync(b->dmem, b->stream);
        if (b->stream != b->own_stream) cudaStreamSynchronize(b->stream);
        ctx_pinned_release(b->ctx, b->pin, b->pin_cap);
        ctx_stream_release(b->ctx, b->body_stream);
        ctx_stream_release(b->ctx, b->own_stream);
    }
    delete b;
    return UAAMG_SUCCESS;
}

int uaamg_batch_size(const uaamg_batch* b) { return b ? b->n : 0; }

int uaamg_batch_set_smoother(uaamg_batch* b, int smoother) {
    if (!b || smoother < 0 || smoother > 3) { set_error("invalid smoother"); return UAAMG_ERR_INVALID_ARGUMENT; }
    b->smoother = smoother;
    return UAAMG_SUCCESS;
}
int uaamg_batch_set_max_iterations(uaamg_batch* b, int m) {
    if (!b) { set_error("NULL batch"); return UAAMG_ERR_INVALID_ARGUMENT; }
    b->max_iter = m;
    return UAAMG_SUCCESS;
}
int uaamg_batch_set_relative_tolerance(uaamg_batch* b, float t) {
    if (!b) { set_error("NULL batch"); return UAAMG_ERR_INVALID_ARGUMENT; }
    b->rel_tol = t;
    return UAAMG_SUCCESS;
}

int uaamg_batch_solve_pcg_device(uaamg_batch* b, float* const* d_pressure, const float* const* d_rhs,
                                 int* iterations, int* status) {
    ABI_BEGIN
    require(b && d_pressure && d_rhs, "NULL argument");
    for (int i = 0; i < b->n; ++i)
        require(b->inst[i]->lv[0].L.nl == 0 || (d_pressure[i] && d_rhs[i]), "NULL instance vector");
    bwait_instances(b);
    int all = brun_pcg(b, d_pressure, d_rhs);
    for (int i = 0; i < b->n; ++i) {
        if (iterations) iterations[i] = b->iterations[i];
        if (status) status[i] = b->status[i];
    }
    return all;
    ABI_END
}

int uaamg_batch_solve_pcg(uaamg_batch* b, float* const* pressure, const float* const* rhs, int* iterations,
                          int* status) {
    ABI_BEGIN
    require(b && pressure && rhs, "NULL argument");
    std::vector<float*> dx(b->n, nullptr);
    std::vector<const float*> db(b->n, nullptr);
    bwait_instances(b);
    for (int i = 0; i < b->n; ++i) {
        uaamg_poisson* h = b->inst[i];
        const size_t nb = vec_bytes(h, 0);
        if (!nb) continue;
        require(pressure[i] && rhs[i], "NULL instance vector");
        CK(cudaMemcpyAsync(h->x, pressure[i], nb, cudaMemcpyHostToDevice, b->stream));
        CK(cudaMemcpyAsync(h->b, rhs[i], nb, cudaMemcpyHostToDevice, b->stream));
        dx[i] = h->x;
        db[i] = h->b;
    }
    int all = brun_pcg(b, dx.data(), db.data());
    for (int i = 0; i < b->n; ++i) {
        uaamg_poisson* h = b->inst[i];
        const size_t nb = vec_bytes(h, 0);
        if (nb) CK(cudaMemcpyAsync(pressure[i], h->x, nb, cudaMemcpyDeviceToHost, b->stream));
        if (iterations) iterations[i] = b->iterations[i];
        if (status) status[i] = b->status[i];
    }
    CK(cudaStreamSynchronize(b->stream));
    return all;
    ABI_END
}

int uaamg_batch_results(const uaamg_batch* b, int* iterations, int* status, float* final_residual) {
    if (!b) { set_error("NULL batch"); return UAAMG_ERR_INVALID_ARGUMENT; }
    for (int i = 0; i < b->n && i < (int)b->iterations.size(); ++i) {
        if (iterations) iterations[i] = b->iterations[i];
        if (status) status[i] = b->status[i];
        if (final_residual) final_residual[i] = b->residual[i];
    }
    return UAAMG_SUCCESS;
}

int uaamg_batch_set_stream(uaamg_batch* b, void* stream) {
    if (!b) { set_error("NULL batch"); return UAAMG_ERR_INVALID_ARGUMENT; }
    cudaStream_t s = stream ? (cudaStream_t)stream : b->own_stream;
    if (s != b->stream) {
        cudaStreamSynchronize(b->stream);
        b->stream = s;
    }
    return UAAMG_SUCCESS;
}

int uaamg_batch_get_stream(const uaamg_batch* b, void** stream) {
    if (!b || !stream) { set_error("NULL argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *stream = (void*)b->stream;
    return UAAMG_SUCCESS;
}
int uaamg_batch_set_graph_mode(uaamg_batch* b, int use_graph) {
    if (!b || use_graph < 0 || use_graph > 2) { set_error("NULL batch or invalid graph mode"); return UAAMG_ERR_INVALID_ARGUMENT; }
    b->use_graph = use_graph;
    return UAAMG_SUCCESS;
}

int64_t uaamg_batch_kernel_launches(const uaamg_batch* b) { return b ? b->last_launches : 0; }
