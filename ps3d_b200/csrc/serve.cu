// serve.cu — a request loop for optimal-balance integrations.
//
// A request is one diag_opt_balance (for_src/diag_opt_balance.f90:55-179)
// on its own grid and initial state, or one ensemble run: n members of any
// grid sizes advanced nsteps main-loop steps together in batched launches
// (ps3d_ensemble_*), their final states returned.  Requests are admitted in arrival order
// as execution slots and HBM free up: a request's device footprint is
// computed from its grid before admission and the sum over running requests
// never exceeds the budget.  Every admitted request owns a context with its
// own CUDA stream, driven by a worker thread, so the kernels of concurrent
// requests overlap on the GPU while each request's arithmetic stays exactly
// what it would be alone (no data is shared, reductions are deterministic).
// Every wait is bounded; nothing here blocks without a limit.
//
// A finished request's context is kept idle, still counted in the budget,
// and handed to the next request with the same parameters after a reset to
// its just-created state (the request mix repeats grid sizes, and creating
// and destroying a context per request costs allocations, table uploads and
// device-synchronising frees that stall the other requests); idle contexts
// are destroyed, oldest first, when an admission needs their memory.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>
#include "ctx.h"

using ps3d::Ctx;
using Clock = std::chrono::steady_clock;

namespace ps3d {
int ensemble_create(const ps3d_params* members, int n, int device, bool tune, ps3d_ensemble** out);
}

namespace {

enum State { kQueued, kRunning, kDone, kFailed, kCancelled };

struct Request;
// requests admitted together as the instances of one batched context
struct Group {
    std::vector<Request*> members;
    std::atomic<int> cancel{0};   // set once every member is cancelled
};

struct Request {
    long long id = 0;
    int kind = 0;                   // 0: optimal balance, 1: ensemble run
    ps3d_params prm{};
    ps3d_optbal opt{};
    std::vector<ps3d_params> members;   // ensemble run: the members, nsteps each
    int nsteps = 0;
    std::vector<std::vector<double>> ein, eout;   // ensemble run: [member * 4 + field], halo layout
    std::vector<double> in[4];      // halo-layout input fields
    std::vector<double> out[4];     // balanced fields (u_bal..b_bal)
    size_t footprint = 0;
    State state = kQueued;
    int status = PS3D_OK;
    double norm = 0.0;
    int iters = 0;
    Clock::time_point t_submit, t_start, t_end;
    std::atomic<int> cancel{0};
    std::shared_ptr<Group> group;   // batched with other requests (null: alone)
};

}  // namespace

// Device bytes a context for `p` allocates for a full optimal-balance run.
static size_t footprint_of(const ps3d_params& p) {
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    const size_t M = (size_t)(p.nx / 2 + 1) * p.ny * p.nz;
    const bool mixed = p.precision == PS3D_MIXED || p.precision == PS3D_MIXED_REFINED;
    const size_t ts = mixed ? 4 : 8;
    size_t b = 0;
    b += 12 * N * 8;                       // 3 state buffers x 4 fields
    b += N * 8;                            // p
    b += 9 * N * ts + 3 * N * 8;           // 3 tendency levels x 4 fields (w always FP64)
    b += M * (mixed ? 8 : 16);             // Poisson spectral array
    b += 6 * M * 16;                       // projection spectra, g0_base, scratch
    b += 4 * 4 * N * 8;                    // balanced, base, saved, zero-order field sets
    b += N * 8 + 9 * N * ts + 3 * N * 8;   // saved p and tendencies
    if (p.nz > 0) b += 6 * (size_t)p.nz * p.nz * 8;   // mode matrices and their transposes
    b += (size_t)(p.nx + 4) * (p.ny + 4) * (p.nz + 4) * 8;   // host-layout staging
    return b + (64u << 20);                // tables, plans, reductions, allocator slack
}

struct IdleCtx {
    ps3d_params prm;
    int batch;                  // instances the context holds (serves groups of up to this many)
    std::unique_ptr<Ctx> ctx;
    size_t footprint;
};

struct ps3d_server {
    int device = 0;
    std::deque<IdleCtx> idle;   // finished requests' contexts, oldest first (counted in `used`)
    size_t budget = 0, used = 0, peak_used = 0;
    int max_active = 1, active = 0, peak_active = 0;
    int max_batch = 1;          // same-parameter requests run together (ps3d_server_set_batching)
    std::atomic<long long> created{0}, reused{0};   // request contexts created, and taken from the pool
    long batch_points = 1L << 22;   // ... while the group's grid points stay within this
    long long next_id = 1;
    bool stopping = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<long long, std::shared_ptr<Request>> all;
    std::vector<std::thread> workers;

    void worker_loop();
    std::unique_ptr<Ctx> run(std::vector<std::shared_ptr<Request>>& g, std::unique_ptr<Ctx> reuse);
};

static bool same_params(const ps3d_params& a, const ps3d_params& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }
static bool same_opt(const ps3d_optbal& a, const ps3d_optbal& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }
// requests that may share a batched context: no biharmonic friction (its
// generic-path kernels take one grid)
static bool batchable(const Request& r) {
    const ps3d_params& p = r.prm;
    return r.kind == 0 && !(p.Ahbi > 0 || p.Avbi > 0 || p.Khbi > 0 || p.Kvbi > 0);
}

// An ensemble run: batched contexts of its own (not pooled), advanced in
// chunks of 30 steps (a multiple of the graph period 3) with the cancel flag
// checked between chunks.
static int run_ensemble(Request& r, int device) {
    const int n = (int)r.members.size();
    ps3d_ensemble* e = nullptr;
    int rc = ps3d::ensemble_create(r.members.data(), n, device, false, &e);
    for (int m = 0; m < n && !rc; ++m)
        rc = ps3d_ensemble_upload(e, m, r.ein[4 * m].data(), r.ein[4 * m + 1].data(), r.ein[4 * m + 2].data(),
                                  r.ein[4 * m + 3].data());
    for (int left = r.nsteps; left > 0 && !rc;) {
        if (r.cancel.load(std::memory_order_relaxed)) { rc = PS3D_ERR_CANCELLED; break; }
        const int c = left < 30 ? left : 30;
        rc = ps3d_ensemble_integrate(e, c);
        left -= c;
    }
    if (!rc) {
        r.eout.assign(4 * (size_t)n, std::vector<double>());
        for (int m = 0; m < n && !rc; ++m) {
            const ps3d_params& q = r.members[m];
            const size_t n3 = (size_t)(q.nx + 4) * (q.ny + 4) * (q.nz + 4);
            for (int f = 0; f < 4; ++f) r.eout[4 * m + f].assign(n3, 0.0);
            std::vector<double> pbuf(n3);
            rc = ps3d_ensemble_download(e, m, r.eout[4 * m].data(), r.eout[4 * m + 1].data(), r.eout[4 * m + 2].data(),
                                        r.eout[4 * m + 3].data(), pbuf.data());
        }
    }
    if (e) ps3d_ensemble_destroy(e);
    return rc;
}

// Runs the group g (one request, or several same-parameter optimal balances
// as the instances of one batched context) on `reuse` (an idle context of
// the same parameters and batch) or on a new context; returns the context
// for the idle pool when every request of the group succeeded.
std::unique_ptr<Ctx> ps3d_server::run(std::vector<std::shared_ptr<Request>>& g, std::unique_ptr<Ctx> reuse) {
    cudaSetDevice(device);
    Request& r0 = *g[0];
    if (r0.kind == 1) {
        r0.status = run_ensemble(r0, device);
        return nullptr;
    }
    const int nb = (int)g.size();
    std::unique_ptr<Ctx> cp = std::move(reuse);
    int rc = PS3D_OK;
    if (cp) {
        ++reused;
        rc = cp->reset_request();
        if (!rc) rc = cp->set_active_batch(nb);
    } else {
        ++created;
        cp.reset(new Ctx());
        // no autotuning runs here: they would time their candidates while
        // other requests share the GPU, and one context at a time (the
        // tuner's lock); cached choices or the defaults are taken instead
        cp->tune_timing = false;
        rc = cp->init(r0.prm, device, nb);
    }
    Ctx& c = *cp;
    std::atomic<int> one{0};
    if (!rc) {
        c.cancel_flag = nb > 1 ? &r0.group->cancel : &r0.cancel;
        for (int m = 0; m < nb && !rc; ++m)
            for (int f = 0; f < 4 && !rc; ++f) rc = c.upload_field(c.member_field(f, m), g[m]->in[f].data());
    }
    std::vector<double> norms(nb, 0.0);
    std::vector<int> iters(nb, 0);
    if (!rc) rc = c.opt_balance(r0.opt, norms.data(), iters.data());
    std::vector<int> st(nb, rc);
    if (!rc) {
        ps3d::DevBuf* bal = c.fieldset(PS3D_FIELDS_BALANCED);
        for (int f = 0; f < 4 && !rc; ++f)
            if (cudaMemcpyAsync(c.field(f), bal[f].p, c.N * nb * sizeof(double), cudaMemcpyDeviceToDevice, c.stream))
                rc = PS3D_ERR_CUDA;
        for (int m = 0; m < nb; ++m) {
            st[m] = rc;
            double ke, pe, um, wm;
            // a non-finite balanced state fails this request only
            if (!st[m]) st[m] = c.diagnose(&ke, &pe, &um, &wm, m);
            if (!st[m]) {
                const size_t n3 = (size_t)(r0.prm.nx + 4) * (r0.prm.ny + 4) * (r0.prm.nz + 4);
                for (int f = 0; f < 4 && !st[m]; ++f) {
                    g[m]->out[f].assign(n3, 0.0);
                    st[m] = c.download_field(c.member_field(f, m), g[m]->out[f].data(), 0);
                }
            }
        }
    }
    c.cancel_flag = nullptr;
    bool all_ok = true;
    for (int m = 0; m < nb; ++m) {
        Request& r = *g[m];
        r.norm = norms[m];
        r.iters = iters[m];
        r.status = st[m];
        if (!st[m] && r.cancel.load()) r.status = PS3D_ERR_CANCELLED;   // cancelled while its group ran on
        if (r.status) all_ok = false;
    }
    if (rc || !all_ok) cp.reset();
    return cp;
}

void ps3d_server::worker_loop() {
    for (;;) {
        std::vector<std::shared_ptr<Request>> g;   // the request(s) admitted together
        size_t gfoot = 0;
        std::unique_ptr<Ctx> reuse;
        std::vector<std::unique_ptr<Ctx>> evicted;   // destroyed after the lock is released
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (stopping) return;
                // admit the oldest request if a slot and its HBM footprint are free,
                // with the queued requests that share its parameters (up to
                // max_batch): on an idle context of the same parameters and
                // batch, or after freeing idle ones
                if (!queue.empty() && active < max_active) {
                    const std::shared_ptr<Request>& q = queue.front();
                    std::vector<std::shared_ptr<Request>> cand{q};
                    const long qpts = (long)q->prm.nx * q->prm.ny * q->prm.nz;
                    // group only when more requests wait than slots are free: with
                    // free slots, lone requests run side by side on their own
                    // streams, and a group would take that concurrency away
                    const bool backlog = (long)queue.size() > (long)(max_active - active);
                    if (max_batch > 1 && backlog && batchable(*q))
                        for (size_t k = 1; k < queue.size() && (int)cand.size() < max_batch &&
                                           (long)(cand.size() + 1) * qpts <= batch_points;
                             ++k)
                            if (batchable(*queue[k]) && same_params(queue[k]->prm, q->prm) &&
                                same_opt(queue[k]->opt, q->opt))
                                cand.push_back(queue[k]);
                    // the largest group whose footprint fits, given what idle contexts could
                    // free, of a power-of-two size: a finished group's context then serves
                    // later groups of the same parameters (the pool matches the batch)
                    size_t idle_bytes = 0;
                    for (const IdleCtx& ic : idle) idle_bytes += ic.footprint;
                    while (cand.size() > 1 && used - idle_bytes + cand.size() * q->footprint > budget) cand.pop_back();
                    while (cand.size() & (cand.size() - 1)) cand.pop_back();
                    const int nb = (int)cand.size();
                    const size_t foot = nb * q->footprint;
                    // an idle context of the same parameters holding at least nb
                    // instances, the smallest such (a group runs the first nb)
                    long hit = -1;
                    for (size_t i = 0; i < idle.size() && q->kind == 0; ++i)
                        if (idle[i].batch >= nb && same_params(idle[i].prm, q->prm) &&
                            (hit < 0 || idle[i].batch < idle[hit].batch))
                            hit = (long)i;
                    bool fits = hit >= 0;
                    while (!fits && !idle.empty() && used + foot > budget) {   // no hit: free idle ones
                        evicted.push_back(std::move(idle.front().ctx));
                        used -= idle.front().footprint;
                        idle.pop_front();
                    }
                    if (!fits) fits = used + foot <= budget;
                    if (fits) {
                        g = cand;
                        for (const auto& r : g)
                            for (auto it = queue.begin(); it != queue.end(); ++it)
                                if (*it == r) { queue.erase(it); break; }
                        if (hit >= 0) {
                            reuse = std::move(idle[hit].ctx);   // its footprint is already counted
                            gfoot = idle[hit].footprint;
                            idle.erase(idle.begin() + hit);
                        } else {
                            used += foot;
                            gfoot = foot;
                        }
                        if (nb > 1) {
                            auto grp = std::make_shared<Group>();
                            for (const auto& r : g) { grp->members.push_back(r.get()); r->group = grp; }
                        }
                        ++active;
                        peak_used = std::max(peak_used, used);
                        peak_active = std::max(peak_active, active);
                        const auto now = Clock::now();
                        for (const auto& r : g) { r->state = kRunning; r->t_start = now; }
                        break;
                    }
                }
                if (!evicted.empty()) break;   // free them, then look again
                cv_work.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
        if (!evicted.empty()) {
            cudaSetDevice(device);
            evicted.clear();
            if (g.empty()) continue;
        }
        std::unique_ptr<Ctx> done = run(g, std::move(reuse));
        {
            std::lock_guard<std::mutex> lk(mu);
            const auto now = Clock::now();
            for (const auto& r : g) {
                r->t_end = now;
                r->state = r->status == PS3D_OK ? kDone : (r->status == PS3D_ERR_CANCELLED ? kCancelled : kFailed);
                for (int f = 0; f < 4; ++f) { r->in[f].clear(); r->in[f].shrink_to_fit(); }
                r->ein.clear();
                r->ein.shrink_to_fit();
                r->group.reset();
            }
            --active;
            if (done && !stopping) {
                const int capn = done->cap;
                idle.push_back({g[0]->prm, capn, std::move(done), gfoot});
            }
            else used -= gfoot;
            // keep at most 2 max_active idle contexts (with batching, groups of
            // different sizes of one grid each keep theirs)
            while ((int)idle.size() > 2 * max_active) {
                evicted.push_back(std::move(idle.front().ctx));
                used -= idle.front().footprint;
                idle.pop_front();
            }
        }
        if (!evicted.empty() || done) {
            cudaSetDevice(device);
            evicted.clear();
            done.reset();   // not kept (server stopping)
        }
        cv_work.notify_all();
        cv_done.notify_all();
    }
}

#define SGUARD_BEGIN try {
#define SGUARD_END                                         \
    }                                                      \
    catch (const std::bad_alloc&) { return PS3D_ERR_OOM; } \
    catch (...) { return PS3D_ERR_CUDA; }

extern "C" {

PS3D_API int ps3d_server_create(int device, size_t hbm_budget_bytes, int max_active, ps3d_server** out) {
    SGUARD_BEGIN
    if (!out || max_active < 1) return PS3D_ERR_BADPARAM;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return PS3D_ERR_CUDA;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return PS3D_ERR_CUDA;
    std::unique_ptr<ps3d_server> s(new ps3d_server());
    s->device = device;
    s->budget = hbm_budget_bytes ? std::min(hbm_budget_bytes, fr) : (size_t)(0.8 * fr);
    s->max_active = max_active;
    for (int t = 0; t < max_active; ++t) s->workers.emplace_back([p = s.get()] { p->worker_loop(); });
    *out = s.release();
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_server_destroy(ps3d_server* s) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        for (auto& q : s->queue) { q->state = kCancelled; q->status = PS3D_ERR_CANCELLED; }
        s->queue.clear();
        for (auto& kv : s->all) {
            kv.second->cancel.store(1);
            if (kv.second->group) kv.second->group->cancel.store(1);   // a running batched group stops too
        }
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    cudaSetDevice(s->device);
    delete s;
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_server_submit(ps3d_server* s, const ps3d_params* prm, const ps3d_optbal* opt,
                                const double* u, const double* v, const double* w, const double* b,
                                long long* ticket) {
    SGUARD_BEGIN
    if (!s || !prm || !opt || !ticket || !u || !v || !w || !b) return PS3D_ERR_BADPARAM;
    const ps3d_params& p = *prm;
    const bool rigid = p.enable_vertical_boundaries != 0;
    if (p.nx < 2 || p.ny < 2 || p.nz < 2 || p.nx % 2 || p.ny % 2 || (!rigid && p.nz % 2)) return PS3D_ERR_BADPARAM;
    if (!ps3d::fft_length_ok(p.nx / 2) || !ps3d::fft_length_ok(p.ny) || (!rigid && !ps3d::fft_length_ok(p.nz)))
        return PS3D_ERR_BADPARAM;
    if (!(p.dt > 0) || !(opt->period > 0) || opt->max_itts < 1) return PS3D_ERR_BADPARAM;
    if (p.precision != PS3D_FP64 && (p.Ahbi > 0 || p.Avbi > 0 || p.Khbi > 0 || p.Kvbi > 0)) return PS3D_ERR_UNSUPPORTED;
    auto r = std::make_shared<Request>();
    r->prm = p;
    r->opt = *opt;
    r->opt.adopt = 0;
    r->footprint = footprint_of(p);
    if (r->footprint > s->budget) return PS3D_ERR_OOM;   // can never be admitted
    const size_t n3 = (size_t)(p.nx + 4) * (p.ny + 4) * (p.nz + 4);
    const double* f[4] = {u, v, w, b};
    for (int q = 0; q < 4; ++q) r->in[q].assign(f[q], f[q] + n3);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return PS3D_ERR_CANCELLED;
        r->id = s->next_id++;
        s->all[r->id] = r;
        s->queue.push_back(r);
    }
    s->cv_work.notify_all();
    *ticket = r->id;
    return PS3D_OK;
    SGUARD_END
}

// An ensemble run as a request: n members (any grid sizes; members with
// identical parameters share launches), each advanced nsteps main-loop steps
// from the given halo-layout state.  Admitted by the sum of the members'
// footprints like any request.
PS3D_API int ps3d_server_submit_ensemble(ps3d_server* s, const ps3d_params* members, int n, int nsteps,
                                         const double* const* u, const double* const* v, const double* const* w,
                                         const double* const* b, long long* ticket) {
    SGUARD_BEGIN
    if (!s || !members || n < 1 || nsteps < 0 || !u || !v || !w || !b || !ticket) return PS3D_ERR_BADPARAM;
    auto r = std::make_shared<Request>();
    r->kind = 1;
    r->nsteps = nsteps;
    r->members.assign(members, members + n);
    r->footprint = 0;
    for (int m = 0; m < n; ++m) {
        const ps3d_params& p = members[m];
        const bool rigid = p.enable_vertical_boundaries != 0;
        if (p.nx < 2 || p.ny < 2 || p.nz < 2 || p.nx % 2 || p.ny % 2 || (!rigid && p.nz % 2)) return PS3D_ERR_BADPARAM;
        if (!ps3d::fft_length_ok(p.nx / 2) || !ps3d::fft_length_ok(p.ny) || (!rigid && !ps3d::fft_length_ok(p.nz)))
            return PS3D_ERR_BADPARAM;
        if (!u[m] || !v[m] || !w[m] || !b[m]) return PS3D_ERR_BADPARAM;
        r->footprint += footprint_of(p);
    }
    if (r->footprint > s->budget) return PS3D_ERR_OOM;   // can never be admitted
    r->ein.resize(4 * (size_t)n);
    for (int m = 0; m < n; ++m) {
        const ps3d_params& p = members[m];
        const size_t n3 = (size_t)(p.nx + 4) * (p.ny + 4) * (p.nz + 4);
        const double* f[4] = {u[m], v[m], w[m], b[m]};
        for (int q = 0; q < 4; ++q) r->ein[4 * m + q].assign(f[q], f[q] + n3);
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return PS3D_ERR_CANCELLED;
        r->id = s->next_id++;
        s->all[r->id] = r;
        s->queue.push_back(r);
    }
    s->cv_work.notify_all();
    *ticket = r->id;
    return PS3D_OK;
    SGUARD_END
}

// Wait up to timeout_ms for a request.  On success the balanced fields are
// copied out (any pointer may be NULL) and res receives
// {status, final norm, iterations, latency ms, queue ms, run ms}.
PS3D_API int ps3d_server_wait(ps3d_server* s, long long ticket, int timeout_ms,
                              double* u_bal, double* v_bal, double* w_bal, double* b_bal, double* res) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    std::shared_ptr<Request> r;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return PS3D_ERR_BADPARAM;
    r = it->second;
    const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
    while (r->state == kQueued || r->state == kRunning) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
            (r->state == kQueued || r->state == kRunning))
            return PS3D_ERR_TIMEOUT;
    }
    double* out[4] = {u_bal, v_bal, w_bal, b_bal};
    if (r->state == kDone && r->kind == 0)
        for (int q = 0; q < 4; ++q)
            if (out[q] && !r->out[q].empty()) std::memcpy(out[q], r->out[q].data(), r->out[q].size() * sizeof(double));
    if (res) {
        auto ms = [](Clock::time_point a, Clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        res[0] = r->status;
        res[1] = r->norm;
        res[2] = r->iters;
        const bool ran = r->state != kCancelled || r->t_start.time_since_epoch().count() != 0;
        res[3] = ms(r->t_submit, r->t_end);
        res[4] = ran ? ms(r->t_submit, r->t_start) : res[3];
        res[5] = ran ? ms(r->t_start, r->t_end) : 0.0;
    }
    const int st = r->status;
    s->all.erase(ticket);   // results are handed out once
    return st;
    SGUARD_END
}

// Wait for an ensemble run; on success member m's final u, v, w, b (halo
// layout) are copied to u[m] .. b[m] (an array, or one of its entries, may
// be NULL); res as for ps3d_server_wait (norm 0, iterations = nsteps).
PS3D_API int ps3d_server_wait_ensemble(ps3d_server* s, long long ticket, int timeout_ms, double* const* u,
                                       double* const* v, double* const* w, double* const* b, double* res) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end() || it->second->kind != 1) return PS3D_ERR_BADPARAM;
    std::shared_ptr<Request> r = it->second;
    const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
    while (r->state == kQueued || r->state == kRunning) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
            (r->state == kQueued || r->state == kRunning))
            return PS3D_ERR_TIMEOUT;
    }
    double* const* out[4] = {u, v, w, b};
    if (r->state == kDone)
        for (size_t m = 0; m < r->members.size(); ++m)
            for (int q = 0; q < 4; ++q)
                if (out[q] && out[q][m] && !r->eout[4 * m + q].empty())
                    std::memcpy(out[q][m], r->eout[4 * m + q].data(), r->eout[4 * m + q].size() * sizeof(double));
    if (res) {
        auto ms = [](Clock::time_point a, Clock::time_point c) {
            return std::chrono::duration<double, std::milli>(c - a).count();
        };
        res[0] = r->status;
        res[1] = 0.0;
        res[2] = r->nsteps;
        const bool ran = r->state != kCancelled || r->t_start.time_since_epoch().count() != 0;
        res[3] = ms(r->t_submit, r->t_end);
        res[4] = ran ? ms(r->t_submit, r->t_start) : res[3];
        res[5] = ran ? ms(r->t_start, r->t_end) : 0.0;
    }
    const int st = r->status;
    s->all.erase(ticket);
    return st;
    SGUARD_END
}

PS3D_API int ps3d_server_cancel(ps3d_server* s, long long ticket) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->all.find(ticket);
        if (it == s->all.end()) return PS3D_ERR_BADPARAM;
        Request& r = *it->second;
        if (r.state == kQueued) {
            for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
                if ((*q)->id == ticket) { s->queue.erase(q); break; }
            r.state = kCancelled;
            r.status = PS3D_ERR_CANCELLED;
            r.t_end = Clock::now();
        } else if (r.state == kRunning) {
            r.cancel.store(1);
            if (r.group) {   // a batched group stops once every member is cancelled
                bool all = true;
                for (Request* m : r.group->members) all = all && m->cancel.load() != 0;
                if (all) r.group->cancel.store(1);
            }
        }
    }
    s->cv_done.notify_all();
    return PS3D_OK;
    SGUARD_END
}

// stats: [0] active, [1] queued, [2] bytes in use, [3] peak bytes, [4] peak active, [5] budget
PS3D_API int ps3d_server_stats(ps3d_server* s, double* stats) {
    if (!s || !stats) return PS3D_ERR_BADPARAM;
    std::lock_guard<std::mutex> lk(s->mu);
    stats[0] = s->active;
    stats[1] = (double)s->queue.size();
    stats[2] = (double)s->used;
    stats[3] = (double)s->peak_used;
    stats[4] = s->peak_active;
    stats[5] = (double)s->budget;
    return PS3D_OK;
}

PS3D_API long long ps3d_server_footprint(const ps3d_params* prm) { return prm ? (long long)footprint_of(*prm) : -1; }

PS3D_API int ps3d_server_context_stats(ps3d_server* s, long long* created, long long* reused) {
    if (!s) return PS3D_ERR_BADPARAM;
    if (created) *created = s->created.load();
    if (reused) *reused = s->reused.load();
    return PS3D_OK;
}

PS3D_API int ps3d_server_set_batching(ps3d_server* s, int max_batch, long long max_points) {
    if (!s || max_batch < 1 || max_points < 0) return PS3D_ERR_BADPARAM;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->max_batch = max_batch;
        s->batch_points = max_points ? (long)max_points : (1L << 22);
    }
    s->cv_work.notify_all();
    return PS3D_OK;
}

}  // extern "C"
