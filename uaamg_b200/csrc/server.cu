// server.cu -- the served form: many simulations' solves on one GPU.
//
// A request is one simulation domain that asks for `substeps` solves of one
// kind: FLIP_vdb's pressure projection (FLIP_vdb.cpp:3118-3168) or its
// viscosity step (:3170-3216).  Each substep brings new face velocities.  The
// server (no counterpart in the reference, which solves one domain per call):
//  * admits queued requests in submission order while their estimated device
//    footprint fits the budget and the resident caps, building their
//    hierarchies on the device; a request's hierarchy, its face weights and
//    its warm start (the previous substep's pressure) stay on the device
//    until its last substep;
//  * runs pressure rounds: every resident pressure request with a pending
//    substep gets its right-hand side built on the device, and all of them
//    are solved in one batched CUDA graph (uaamg_batch, kept while the set
//    of requests is unchanged), or one after another when batching is off.
//    A set seen for the first time is also solved one request after another
//    (each handle replays its own solve graph); the batch is built when the
//    same set comes back in the next round, since a batch's first solve runs
//    host-driven and pays off only over the rounds that reuse it;
//    requests admitted meanwhile join the next round;
//  * runs each viscosity request on a lane of its own (a host thread and a
//    CUDA stream) that solves its substeps as their velocities arrive, in
//    both modes, so the plain form differs from the batched one only in the
//    pressure batching;
//  * checks every pressure result in FP64 (|b - A x|_inf / |b|_inf with the
//    FP32-assembled matrix) and keeps it with the status and the iterations.
// The loop runs on a thread of its own; submissions, velocity pushes and
// result fetches may come from any thread.  Results are identical alone and
// in the mix: the batched pressure solve is bit-identical to a standalone one
// and viscosity solves are independent.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <thread>

namespace {

using srv_clock = std::chrono::steady_clock;

// a C-ABI call's status: negative codes become the error (the message is set)
#define CKC(expr)                                  \
    do {                                           \
        const int rc_ = (expr);                    \
        if (rc_ < 0) throw UaamgError{rc_};        \
    } while (0)

// device memory for server-owned copies: the device's stream-ordered pool
// (no device-wide synchronisation), allocated and copied on `s`, which is
// synchronised before the memory is used elsewhere
static float* srv_alloc(size_t bytes, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    DeviceCtx* ctx = device_ctx(&e);
    CK(e);
    void* p = nullptr;
    CK(ctx_dev_alloc(ctx, &p, bytes, s));
    return reinterpret_cast<float*>(p);
}

// A server-owned copy of an input grid.  Host grids are copied into host
// memory, device grids into device memory (synchronously), so the caller may
// free its grids as soon as the call returns.
struct SrvGrid {
    std::vector<int32_t> org;
    std::vector<uint64_t> mask;
    std::vector<float> hval;
    float* dval = nullptr;
    cudaStream_t stream = nullptr;  // of the device copy
    int64_t n = 0;
    int comps = 1;
    float bg[3] = {0.f, 0.f, 0.f};
    SrvGrid() = default;
    SrvGrid(const SrvGrid&) = delete;
    SrvGrid& operator=(const SrvGrid&) = delete;
    ~SrvGrid() {
        if (dval) cudaFreeAsync(dval, stream);
    }
    // `s`: the server's copy stream (device grids are copied on it, and it is
    // synchronised before the call returns)
    void copy_from(const uaamg_leaf_grid* g, cudaStream_t s) {
        n = g->leaf_count;
        comps = g->components;
        for (int c = 0; c < 3; ++c) bg[c] = g->background[c];
        if (n <= 0) return;
        org.assign(g->origins, g->origins + 3 * n);
        if (g->masks) mask.assign(g->masks, g->masks + 8 * n);
        const size_t nv = (size_t)n * UAAMG_LEAF * comps;
        if (g->values_on_device) {
            stream = s;
            dval = srv_alloc(nv * sizeof(float), s);
            CK(cudaMemcpyAsync(dval, g->values, nv * sizeof(float), cudaMemcpyDeviceToDevice, s));
            CK(cudaStreamSynchronize(s));
        } else {
            hval.assign(g->values, g->values + nv);
        }
    }
    uaamg_leaf_grid view() const {
        uaamg_leaf_grid g{};
        g.leaf_count = n;
        g.origins = n ? org.data() : nullptr;
        g.masks = mask.empty() ? nullptr : mask.data();
        g.values = dval ? dval : (hval.empty() ? nullptr : hval.data());
        g.values_on_device = dval ? 1 : 0;
        g.components = comps;
        for (int c = 0; c < 3; ++c) g.background[c] = bg[c];
        return g;
    }
};

struct SrvSubstep {
    SrvGrid u, v, w;
};

struct SrvResult {
    int status = 0, iterations = 0;
    double residual = -1.0;  // FP64 true relative residual (pressure), -1 when not checked
    double done_s = 0.0;
    std::vector<float> x;    // the solution, when the server keeps results
};

enum { RQ_QUEUED = 0, RQ_ADMITTING = 1, RQ_RESIDENT = 2, RQ_DONE = 3, RQ_FAILED = 4 };

struct SrvReq {
    int64_t id = 0;
    int kind = 0;  // UAAMG_SERVER_POISSON / UAAMG_SERVER_VISCOSITY
    int substeps = 0;
    int pushed = 0;  // velocities pushed (a substep in flight is in neither pending nor results)
    int64_t cost = 0;
    SrvGrid a, b, c, sv;  // pressure: liquid SDF, face weights; viscosity: viscosity, liquid SDF, solid SDF
    float dt = 0, dx = 0, rho = 0;
    std::deque<std::unique_ptr<SrvSubstep>> pending;
    std::vector<SrvResult> results;
    int state = RQ_QUEUED;
    std::string error;
    double submit_s = 0, admit_s = -1, done_s = -1;
    int64_t leaves = 0;
    uaamg_poisson* hp = nullptr;
    uaamg_viscosity* hv = nullptr;
    float *dx_ = nullptr, *drhs = nullptr;  // device solution (warm start) and rhs
    float* dfw = nullptr;                   // pressure: the face weights on the device
    cudaStream_t lane_stream = nullptr;
    std::thread lane;
    std::atomic<bool> lane_running{false};
};

}  // namespace

struct uaamg_server {
    uaamg_server_options opt{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv;  // new work or new results
    std::map<int64_t, std::unique_ptr<SrvReq>> reqs;
    std::deque<int64_t> queue;
    int64_t used = 0, peak = 0, next_id = 1;
    int64_t rounds = 0, solves = 0, batch_builds = 0;
    int64_t pressure_solves = 0;
    double pressure_busy_s = 0.0;  // wall time inside pressure rounds (rhs, solves, FP64 checks)
    srv_clock::time_point t0;
    std::thread loop;
    std::atomic<bool> stop{false};
    cudaStream_t pstream = nullptr;
    cudaStream_t cstream = nullptr;  // copies of device inputs at submission
    std::mutex copy_mu;              // one submission copy at a time on cstream
    uaamg_batch* batch = nullptr;
    std::vector<int64_t> batch_key;
    std::vector<int64_t> last_key;  // the previous pressure round's set of requests
    std::string loop_error;
    double now() const { return std::chrono::duration<double>(srv_clock::now() - t0).count(); }
};

namespace {

// Device footprint estimate of a request (hierarchy, vectors, inputs kept on
// the device), from its level-0-sized input: a pressure request keeps about
// 20 leaf-sized float arrays per input leaf (coefficients, mu-cycle and PCG
// vectors over ~1.15 leaves of hierarchy per level-0 leaf, the face weights,
// the solution and rhs); a viscosity request about 110 (27 coefficient arrays
// per leaf, three-channel vectors, the subcell construction).
static int64_t srv_estimate(const SrvReq& r) {
    const int64_t leaves = r.kind == UAAMG_SERVER_POISSON ? std::max(r.a.n, r.b.n) : std::max(r.b.n, r.c.n);
    const int64_t per = r.kind == UAAMG_SERVER_POISSON ? 20 : 110;
    return leaves * (int64_t)UAAMG_LEAF * 4 * per + (64ll << 20);
}

static void srv_release_device(SrvReq& r, cudaStream_t s) {
    if (r.hp) uaamg_poisson_destroy(r.hp);
    if (r.hv) uaamg_viscosity_destroy(r.hv);
    r.hp = nullptr;
    r.hv = nullptr;
    if (r.dx_) cudaFreeAsync(r.dx_, s);
    if (r.drhs) cudaFreeAsync(r.drhs, s);
    if (r.dfw) cudaFreeAsync(r.dfw, s);
    r.dx_ = r.drhs = r.dfw = nullptr;
    if (r.lane_stream) cudaStreamDestroy(r.lane_stream);
    r.lane_stream = nullptr;
}

// Admission work of a pressure request (outside the lock): its hierarchy on
// the pressure stream, the face weights kept on the device, a zero warm start.
static void srv_admit_poisson(uaamg_server* s, SrvReq& r) {
    uaamg_leaf_grid phi = r.a.view(), fw = r.b.view();
    CKC(uaamg_poisson_create_on_stream(&phi, &fw, r.dt, r.dx, s->pstream, &r.hp));
    CKC(uaamg_poisson_set_relative_tolerance(r.hp, s->opt.pressure_tolerance));
    r.leaves = uaamg_poisson_leaf_count(r.hp, 0);
    const size_t nb = (size_t)std::max<int64_t>(r.leaves, 1) * UAAMG_LEAF * sizeof(float);
    r.dx_ = srv_alloc(nb, s->pstream);
    r.drhs = srv_alloc(nb, s->pstream);
    CK(cudaMemsetAsync(r.dx_, 0, nb, s->pstream));
    if (r.b.n > 0 && !r.b.dval) {
        const size_t fb = (size_t)r.b.n * UAAMG_LEAF * 3 * sizeof(float);
        r.dfw = srv_alloc(fb, s->pstream);
        CK(cudaMemcpyAsync(r.dfw, r.b.hval.data(), fb, cudaMemcpyHostToDevice, s->pstream));
        CK(cudaStreamSynchronize(s->pstream));
        std::vector<float>().swap(r.b.hval);
    }
}

static uaamg_leaf_grid srv_fw_view(const SrvReq& r) {
    uaamg_leaf_grid g = r.b.view();
    if (r.dfw) {
        g.values = r.dfw;
        g.values_on_device = 1;
    }
    return g;
}

static void srv_notify(uaamg_server* s) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->cv.notify_all();
}

// A viscosity request's lane: its matrix and hierarchy, then each substep as
// its velocities arrive: rhs and warm start (the velocity at the DOFs) on the
// device, PCG, result.
static void srv_viscosity_lane(uaamg_server* s, SrvReq* r) {
    try {
        CK(cudaSetDevice(s->device));
        CK(cudaStreamCreateWithFlags(&r->lane_stream, cudaStreamNonBlocking));
        uaamg_leaf_grid mu = r->a.view(), liq = r->b.view(), sol = r->c.view();
        CKC(uaamg_viscosity_create_on_stream(&mu, &liq, &sol, r->dt, r->rho, r->dx, r->lane_stream, &r->hv));
        r->leaves = uaamg_viscosity_leaf_count(r->hv, 0);
        const size_t nb = (size_t)std::max<int64_t>(r->leaves, 1) * 3 * UAAMG_LEAF * sizeof(float);
        r->dx_ = srv_alloc(nb, r->lane_stream);
        r->drhs = srv_alloc(nb, r->lane_stream);
        for (int k = 0; k < r->substeps; ++k) {
            std::unique_ptr<SrvSubstep> sub;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                s->cv.wait(lk, [&] { return !r->pending.empty() || s->stop.load(); });
                if (r->pending.empty()) break;  // stopping
                sub = std::move(r->pending.front());
                r->pending.pop_front();
            }
            uaamg_leaf_grid u = sub->u.view(), v = sub->v.view(), w = sub->w.view(), sv = r->sv.view();
            CKC(uaamg_viscosity_build_rhs_device(r->hv, &u, &v, &w, &sv, r->drhs));
            CKC(uaamg_viscosity_gather_velocity_device(r->hv, &u, &v, &w, r->dx_));
            SrvResult res;
            int it = 0;
            const int st = uaamg_viscosity_solve_pcg_device(r->hv, r->dx_, r->drhs, s->opt.viscosity_tolerance, &it);
            CKC(st);
            res.status = st;
            res.iterations = it;
            if (s->opt.keep_results) {
                res.x.resize(nb / sizeof(float));
                CK(cudaMemcpyAsync(res.x.data(), r->dx_, nb, cudaMemcpyDeviceToHost, r->lane_stream));
            }
            CK(cudaStreamSynchronize(r->lane_stream));
            res.done_s = s->now();
            std::lock_guard<std::mutex> lk(s->mu);
            r->results.push_back(std::move(res));
            s->solves++;
            s->cv.notify_all();
        }
    } catch (const UaamgError& e) {
        std::lock_guard<std::mutex> lk(s->mu);
        r->error = uaamg_last_error();
        r->state = RQ_FAILED;
        (void)e;
    } catch (...) {
        std::lock_guard<std::mutex> lk(s->mu);
        r->error = "viscosity lane failed";
        r->state = RQ_FAILED;
    }
    r->lane_running = false;
    srv_notify(s);
}

// One pressure round over `act` (requests with a pending substep whose
// inputs were taken out of their queues into `subs`).
static void srv_fail(uaamg_server* s, SrvReq& r, const char* what) {
    std::lock_guard<std::mutex> lk(s->mu);
    r.state = RQ_FAILED;
    r.error = std::string(what) + ": " + uaamg_last_error();
    s->cv.notify_all();
}

static void srv_pressure_round(uaamg_server* s, std::vector<SrvReq*>& act_in,
                               std::vector<std::unique_ptr<SrvSubstep>>& subs) {
    const double t_start = s->now();
    // the substep's rhs of every request; a request whose inputs fail leaves the round, failed
    std::vector<SrvReq*> act;
    for (size_t i = 0; i < act_in.size(); ++i) {
        SrvReq& r = *act_in[i];
        uaamg_leaf_grid fw = srv_fw_view(r), u = subs[i]->u.view(), v = subs[i]->v.view(), w = subs[i]->w.view();
        uaamg_leaf_grid sv = r.sv.view();
        if (uaamg_poisson_build_rhs_device(r.hp, &fw, &u, &v, &w, &sv, r.dt, r.drhs) < 0) {
            srv_fail(s, r, "right-hand side");
            continue;
        }
        act.push_back(&r);
    }
    const size_t n = act.size();
    if (n == 0) return;
    std::vector<int> iters(n, 0), status(n, 0);
    std::vector<int64_t> key(n);
    for (size_t i = 0; i < n; ++i) key[i] = act[i]->id;
    const bool repeat = key == s->last_key;
    s->last_key = key;
    if (s->opt.batching && ((s->batch && key == s->batch_key) || repeat)) {
        if (!s->batch || key != s->batch_key) {
            if (s->batch) uaamg_batch_destroy(s->batch);
            s->batch = nullptr;
            std::vector<uaamg_poisson*> hs(n);
            for (size_t i = 0; i < n; ++i) hs[i] = act[i]->hp;
            CKC(uaamg_batch_create((int)n, hs.data(), &s->batch));
            CKC(uaamg_batch_set_relative_tolerance(s->batch, s->opt.pressure_tolerance));
            CKC(uaamg_batch_set_stream(s->batch, s->pstream));
            s->batch_key = key;
            s->batch_builds++;
        }
        std::vector<float*> xs(n);
        std::vector<const float*> bs(n);
        for (size_t i = 0; i < n; ++i) {
            xs[i] = act[i]->dx_;
            bs[i] = act[i]->drhs;
        }
        CKC(uaamg_batch_solve_pcg_device(s->batch, xs.data(), bs.data(), iters.data(), status.data()));
    } else {
        for (size_t i = 0; i < n; ++i) {
            CKC(uaamg_poisson_set_stream(act[i]->hp, s->pstream));
            status[i] = uaamg_poisson_solve_pcg_device(act[i]->hp, act[i]->dx_, act[i]->drhs, &iters[i]);
            CKC(status[i]);
        }
    }
    std::vector<SrvResult> res(n);
    for (size_t i = 0; i < n; ++i) {
        SrvReq& r = *act[i];
        double out[2] = {0.0, 0.0};
        CKC(uaamg_poisson_true_residual_fp64(r.hp, r.dx_, r.drhs, out));
        res[i].status = status[i];
        res[i].iterations = iters[i];
        res[i].residual = out[1] > 0.0 ? out[0] / out[1] : 0.0;
        if (s->opt.keep_results) {
            res[i].x.resize((size_t)r.leaves * UAAMG_LEAF);
            if (r.leaves)
                CK(cudaMemcpyAsync(res[i].x.data(), r.dx_, res[i].x.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                   s->pstream));
        }
    }
    CK(cudaStreamSynchronize(s->pstream));
    const double t = s->now();
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < n; ++i) {
        res[i].done_s = t;
        act[i]->results.push_back(std::move(res[i]));
    }
    s->rounds++;
    s->solves += (int64_t)n;
    s->pressure_solves += (int64_t)n;
    s->pressure_busy_s += t - t_start;
    s->cv.notify_all();
}

// Retire requests whose every substep is solved (under the lock); their
// device memory is freed by the caller outside the lock.
static void srv_collect_done(uaamg_server* s, std::vector<SrvReq*>& freed) {
    for (auto& kv : s->reqs) {
        SrvReq& r = *kv.second;
        if ((r.state == RQ_RESIDENT && (int)r.results.size() >= r.substeps && !r.lane_running) ||
            (r.state == RQ_FAILED && r.cost > 0 && !r.lane_running)) {
            if (r.state == RQ_RESIDENT) {
                r.state = RQ_DONE;
                r.done_s = r.results.empty() ? s->now() : r.results.back().done_s;
            }
            s->used -= r.cost;
            r.cost = 0;
            freed.push_back(&r);
        }
    }
}

static void srv_loop(uaamg_server* s) {
    try {
        CK(cudaSetDevice(s->device));
        while (true) {
            std::vector<SrvReq*> admit, freed;
            std::vector<SrvReq*> act;
            std::vector<std::unique_ptr<SrvSubstep>> subs;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                srv_collect_done(s, freed);
                // admission in submission order while the budget and the caps allow
                int np = 0, nv = 0;
                for (auto& kv : s->reqs)
                    if (kv.second->state == RQ_RESIDENT || kv.second->state == RQ_ADMITTING)
                        (kv.second->kind == UAAMG_SERVER_POISSON ? np : nv)++;
                while (!s->queue.empty() && (int)admit.size() < s->opt.admit_per_round) {
                    SrvReq& r = *s->reqs.at(s->queue.front());
                    const bool pois = r.kind == UAAMG_SERVER_POISSON;
                    if ((pois ? np : nv) >= (pois ? s->opt.max_poisson : s->opt.max_viscosity)) break;
                    if (s->used + r.cost > s->opt.budget_bytes) break;
                    s->queue.pop_front();
                    r.state = RQ_ADMITTING;
                    s->used += r.cost;
                    s->peak = std::max(s->peak, s->used);
                    (pois ? np : nv)++;
                    admit.push_back(&r);
                }
                // the pressure requests with a pending substep
                for (auto& kv : s->reqs) {
                    SrvReq& r = *kv.second;
                    if (r.kind == UAAMG_SERVER_POISSON && r.state == RQ_RESIDENT && !r.pending.empty() &&
                        (int)(r.results.size()) < r.substeps) {
                        act.push_back(&r);
                        subs.push_back(std::move(r.pending.front()));
                        r.pending.pop_front();
                    }
                }
                if (admit.empty() && act.empty() && freed.empty()) {
                    if (s->stop.load()) break;
                    s->cv.wait_for(lk, std::chrono::milliseconds(2));
                    continue;
                }
            }
            for (SrvReq* r : freed) {
                if (r->lane.joinable()) r->lane.join();
                srv_release_device(*r, s->pstream);
            }
            for (SrvReq* r : admit) {
                try {
                    if (r->kind == UAAMG_SERVER_POISSON) {
                        srv_admit_poisson(s, *r);
                        std::lock_guard<std::mutex> lk(s->mu);
                        r->state = RQ_RESIDENT;
                        r->admit_s = s->now();
                    } else {
                        {
                            std::lock_guard<std::mutex> lk(s->mu);
                            r->state = RQ_RESIDENT;
                            r->admit_s = s->now();
                        }
                        r->lane_running = true;
                        r->lane = std::thread(srv_viscosity_lane, s, r);
                    }
                } catch (const UaamgError&) {
                    srv_fail(s, *r, "admission");
                }
            }
            if (!act.empty()) {
                try {
                    srv_pressure_round(s, act, subs);
                } catch (const UaamgError&) {
                    // a solve of the round failed: its requests fail, the server goes on
                    std::string msg = uaamg_last_error();
                    if (s->batch) uaamg_batch_destroy(s->batch);
                    s->batch = nullptr;
                    s->batch_key.clear();
                    s->last_key.clear();
                    for (SrvReq* r : act) srv_fail(s, *r, ("pressure round: " + msg).c_str());
                }
            }
            if (!admit.empty() || !act.empty()) srv_notify(s);
        }
    } catch (const UaamgError&) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->loop_error = uaamg_last_error();
        s->cv.notify_all();
    } catch (...) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->loop_error = "server loop failed";
        s->cv.notify_all();
    }
}

static int srv_submit(uaamg_server* s, std::unique_ptr<SrvReq> r, int64_t* request) {
    r->cost = std::min(srv_estimate(*r), s->opt.budget_bytes + 1);
    if (r->cost > s->opt.budget_bytes) {
        set_error("request needs about %lld bytes, more than the server budget of %lld", (long long)r->cost,
                  (long long)s->opt.budget_bytes);
        return UAAMG_ERR_OUT_OF_MEMORY;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->loop_error.empty()) {
        set_error("server loop stopped: %s", s->loop_error.c_str());
        return UAAMG_ERR_CUDA;
    }
    r->id = s->next_id++;
    r->submit_s = s->now();
    *request = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    s->cv.notify_all();
    return UAAMG_SUCCESS;
}

}  // namespace

extern "C" {

int uaamg_server_default_options(uaamg_server_options* o) {
    if (!o) { set_error("NULL argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    o->budget_bytes = 64ll << 30;
    o->max_poisson = 256;
    o->max_viscosity = 16;
    o->admit_per_round = 8;
    o->batching = 1;
    o->keep_results = 0;
    o->pressure_tolerance = 1e-7f;
    o->viscosity_tolerance = 1e-6f;
    return UAAMG_SUCCESS;
}

int uaamg_server_create(const uaamg_server_options* opt, uaamg_server** out) {
    if (!opt || !out) { set_error("NULL argument"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    if (opt->budget_bytes <= 0 || opt->max_poisson < 1 || opt->max_viscosity < 0 || opt->admit_per_round < 1 ||
        !(opt->pressure_tolerance > 0.f) || !(opt->viscosity_tolerance > 0.f)) {
        set_error("invalid server options");
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return UAAMG_ERR_NO_DEVICE;
    }
    uaamg_server* s = new (std::nothrow) uaamg_server();
    if (!s) { set_error("host out of memory"); return UAAMG_ERR_OUT_OF_MEMORY; }
    s->opt = *opt;
    s->t0 = srv_clock::now();
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        delete s;
        set_error("cudaGetDevice failed");
        return UAAMG_ERR_CUDA;
    }
    // pressure rounds are short and latency-bound: their stream has the
    // highest priority, so their kernels go ahead of the viscosity lanes'
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&s->pstream, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking) != cudaSuccess) {
        if (s->pstream) cudaStreamDestroy(s->pstream);
        delete s;
        set_error("stream creation failed");
        return UAAMG_ERR_CUDA;
    }
    s->loop = std::thread(srv_loop, s);
    *out = s;
    return UAAMG_SUCCESS;
}

int uaamg_server_destroy(uaamg_server* s) {
    if (!s) return UAAMG_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->loop.joinable()) s->loop.join();
    for (auto& kv : s->reqs) {
        SrvReq& r = *kv.second;
        if (r.lane.joinable()) r.lane.join();
        srv_release_device(r, s->pstream);
    }
    if (s->batch) uaamg_batch_destroy(s->batch);
    s->reqs.clear();  // the requests' device copies are freed on their copy stream
    if (s->pstream) cudaStreamSynchronize(s->pstream);
    if (s->cstream) cudaStreamSynchronize(s->cstream);
    if (s->pstream) cudaStreamDestroy(s->pstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    delete s;
    return UAAMG_SUCCESS;
}

int uaamg_server_submit_poisson(uaamg_server* s, const uaamg_leaf_grid* liquid_phi,
                                const uaamg_leaf_grid* face_weights, const uaamg_leaf_grid* solid_velocity, float dt,
                                float dx, int substeps, int64_t* request) {
    ABI_BEGIN
    require(s && liquid_phi && face_weights && solid_velocity && request, "NULL argument");
    require(substeps >= 1 && dx > 0.f, "substeps must be >= 1 and dx positive");
    check_grid(liquid_phi, 1, "liquid_phi");
    check_grid(face_weights, 3, "face_weights");
    check_grid(solid_velocity, 3, "solid_velocity");
    auto r = std::make_unique<SrvReq>();
    r->kind = UAAMG_SERVER_POISSON;
    r->substeps = substeps;
    r->dt = dt;
    r->dx = dx;
    {
        std::lock_guard<std::mutex> lk(s->copy_mu);
        r->a.copy_from(liquid_phi, s->cstream);
        r->b.copy_from(face_weights, s->cstream);
        r->sv.copy_from(solid_velocity, s->cstream);
    }
    return srv_submit(s, std::move(r), request);
    ABI_END
}

int uaamg_server_submit_viscosity(uaamg_server* s, const uaamg_leaf_grid* viscosity,
                                  const uaamg_leaf_grid* liquid_sdf, const uaamg_leaf_grid* solid_sdf,
                                  const uaamg_leaf_grid* solid_velocity, float dt, float rho, float dx, int substeps,
                                  int64_t* request) {
    ABI_BEGIN
    require(s && viscosity && liquid_sdf && solid_sdf && solid_velocity && request, "NULL argument");
    require(substeps >= 1 && dx > 0.f && rho > 0.f, "substeps must be >= 1, dx and rho positive");
    require(s->opt.max_viscosity > 0, "the server takes no viscosity requests (max_viscosity 0)");
    check_grid(viscosity, 1, "viscosity");
    check_grid(liquid_sdf, 1, "liquid_sdf");
    check_grid(solid_sdf, 1, "solid_sdf");
    check_grid(solid_velocity, 3, "solid_velocity");
    auto r = std::make_unique<SrvReq>();
    r->kind = UAAMG_SERVER_VISCOSITY;
    r->substeps = substeps;
    r->dt = dt;
    r->rho = rho;
    r->dx = dx;
    {
        std::lock_guard<std::mutex> lk(s->copy_mu);
        r->a.copy_from(viscosity, s->cstream);
        r->b.copy_from(liquid_sdf, s->cstream);
        r->c.copy_from(solid_sdf, s->cstream);
        r->sv.copy_from(solid_velocity, s->cstream);
    }
    return srv_submit(s, std::move(r), request);
    ABI_END
}

int uaamg_server_push_velocity(uaamg_server* s, int64_t request, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                               const uaamg_leaf_grid* w) {
    ABI_BEGIN
    require(s && u && v && w, "NULL argument");
    check_grid(u, 1, "u");
    check_grid(v, 1, "v");
    check_grid(w, 1, "w");
    auto sub = std::make_unique<SrvSubstep>();
    {
        std::lock_guard<std::mutex> lk(s->copy_mu);
        sub->u.copy_from(u, s->cstream);
        sub->v.copy_from(v, s->cstream);
        sub->w.copy_from(w, s->cstream);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) { set_error("unknown request %lld", (long long)request); return UAAMG_ERR_INVALID_ARGUMENT; }
    SrvReq& r = *it->second;
    if (r.pushed >= r.substeps) {
        set_error("request %lld already has all its %d substeps", (long long)request, r.substeps);
        return UAAMG_ERR_INVALID_ARGUMENT;
    }
    if (r.state == RQ_FAILED) { set_error("request %lld failed: %s", (long long)request, r.error.c_str()); return UAAMG_ERR_CUDA; }
    r.pending.push_back(std::move(sub));
    ++r.pushed;
    s->cv.notify_all();
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_server_wait(uaamg_server* s, int64_t request, int substep, double timeout_s, int* status, int* iterations,
                      double* fp64_residual, double* latency_s) {
    ABI_BEGIN
    require(s, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) { set_error("unknown request %lld", (long long)request); return UAAMG_ERR_INVALID_ARGUMENT; }
    SrvReq& r = *it->second;
    if (substep < 0 || substep >= r.substeps) { set_error("substep out of range"); return UAAMG_ERR_INVALID_ARGUMENT; }
    const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return (int)r.results.size() > substep || r.state == RQ_FAILED || !s->loop_error.empty();
    });
    if ((int)r.results.size() <= substep) {
        if (r.state == RQ_FAILED) { set_error("request %lld failed: %s", (long long)request, r.error.c_str()); return UAAMG_ERR_CUDA; }
        if (!s->loop_error.empty()) { set_error("server loop stopped: %s", s->loop_error.c_str()); return UAAMG_ERR_CUDA; }
        (void)ok;
        set_error("timed out");
        return UAAMG_ERR_TIMEOUT;
    }
    const SrvResult& res = r.results[substep];
    if (status) *status = res.status;
    if (iterations) *iterations = res.iterations;
    if (fp64_residual) *fp64_residual = res.residual;
    if (latency_s) *latency_s = res.done_s - r.submit_s;
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_server_result(uaamg_server* s, int64_t request, int substep, int64_t* leaf_count, float* x) {
    ABI_BEGIN
    require(s && leaf_count, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) { set_error("unknown request %lld", (long long)request); return UAAMG_ERR_INVALID_ARGUMENT; }
    SrvReq& r = *it->second;
    if (substep < 0 || substep >= (int)r.results.size()) { set_error("substep not solved yet"); return UAAMG_ERR_INVALID_ARGUMENT; }
    *leaf_count = r.leaves;
    const SrvResult& res = r.results[substep];
    if (x) {
        if (res.x.empty() && r.leaves) { set_error("the server keeps no solutions (keep_results 0)"); return UAAMG_ERR_INVALID_ARGUMENT; }
        std::copy(res.x.begin(), res.x.end(), x);
    }
    return UAAMG_SUCCESS;
    ABI_END
}

int uaamg_server_stats(uaamg_server* s, uaamg_server_stats_t* out) {
    ABI_BEGIN
    require(s && out, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = (int64_t)s->reqs.size();
    out->queued = (int64_t)s->queue.size();
    out->resident = 0;
    out->done = 0;
    out->failed = 0;
    for (auto& kv : s->reqs) {
        const int st = kv.second->state;
        out->resident += st == RQ_RESIDENT || st == RQ_ADMITTING;
        out->done += st == RQ_DONE;
        out->failed += st == RQ_FAILED;
    }
    out->solves = s->solves;
    out->rounds = s->rounds;
    out->batch_builds = s->batch_builds;
    out->used_bytes = s->used;
    out->peak_bytes = s->peak;
    out->pressure_solves = s->pressure_solves;
    out->pressure_busy_us = (int64_t)(s->pressure_busy_s * 1e6);
    return UAAMG_SUCCESS;
    ABI_END
}

}  // extern "C"
