// ensemble.cu — batched ensembles of uneven grids.
//
// The reference runs one grid per MPI job; an ensemble is a new capability.
// Members with identical parameters (same grid, physics and time step) form
// one group; a group is a batched context whose kernels carry the member
// index in their grid, so one launch of each kernel advances every member of
// the group.  Each group runs on its own stream, forked from the ensemble's
// stream and joined back at every step, so the groups' kernels (which share
// no data) run side by side on the GPU; for constant parameters three
// consecutive steps of every group are captured into a single CUDA graph —
// one branch per group — that is replayed (tau and the state buffers cycle
// with period 3).
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <vector>
#include "ctx.h"

using ps3d::Ctx;

struct ps3d_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<std::unique_ptr<Ctx>> groups;
    cudaEvent_t fork = nullptr;              // the ensemble stream's point the groups start from
    std::vector<cudaEvent_t> joins;          // each group's end of a step
    std::vector<std::pair<int, int>> where;   // member -> (group, index in group)
    cudaGraphExec_t gexec = nullptr;
    bool graph_valid = false;
    bool grouped = false;                    // the groups' step kernels in one launch
    int itt = 0;
    ~ps3d_ensemble() {
        if (gexec) cudaGraphExecDestroy(gexec);
        groups.clear();
        if (fork) cudaEventDestroy(fork);
        for (cudaEvent_t j : joins) cudaEventDestroy(j);
        if (stream) { cudaStreamSynchronize(stream); cudaStreamDestroy(stream); }
    }
};

namespace {

bool same_params(const ps3d_params& a, const ps3d_params& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

// The groups' step kernels as one launch on the ensemble stream
// (PS3D_ENSEMBLE_GROUPED=1 at creation; measured slower than one launch per
// group on its own stream, so off by default): every group runs the fused
// step (no generic friction or callback path), in one precision,
// unprofiled, and there are at most kMaxStepGroups of them.
bool grouped_step(const ps3d_ensemble* e) {
    const size_t G = e->groups.size();
    if (!e->grouped || G < 2 || G > (size_t)ps3d::kMaxStepGroups) return false;
    for (auto& g : e->groups)
        if (!g->fused_step() || g->prof || g->split_solve || g->hist32 != e->groups[0]->hist32) return false;
    return true;
}

// one step of every group: each group's stream waits for the ensemble
// stream, runs its step, and the ensemble stream waits for every group.
// Grouped: the step kernels of all groups run first, as one launch on the
// ensemble stream, and the groups' streams then run their pressure solves.
int step_all(ps3d_ensemble* e) {
    if (grouped_step(e)) {
        const size_t G = e->groups.size();
        ps3d::StepArgs args[ps3d::kMaxStepGroups];
        for (size_t q = 0; q < G; ++q) {
            Ctx& g = *e->groups[q];
            g.defer_step = &args[q];
            const int rc = g.step(g.itt, g.tau, g.taum1, g.taum2);
            g.defer_step = nullptr;
            if (rc) return rc;
        }
        bool same = true;
        for (size_t q = 1; q < G; ++q) same = same && ps3d::step_flavour(args[q]) == ps3d::step_flavour(args[0]);
        const bool f32 = e->groups[0]->hist32;
        if (same) {
            if (ps3d::launch_step_groups(args, (int)G, f32, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
            ++e->groups[0]->launches;
        } else {
            for (size_t q = 0; q < G; ++q) {
                if (ps3d::launch_step(args[q], f32, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
                ++e->groups[q]->launches;
            }
        }
        if (cudaEventRecord(e->fork, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
        for (size_t q = 0; q < G; ++q) {
            Ctx& g = *e->groups[q];
            if (cudaStreamWaitEvent(g.stream, e->fork, 0) != cudaSuccess) return PS3D_ERR_CUDA;
            const int rc = g.step_finish();
            if (rc) return rc;
            g.rotate();
            g.time = g.time + g.P.dt;
            ++g.itt;
            if (cudaEventRecord(e->joins[q], g.stream) != cudaSuccess) return PS3D_ERR_CUDA;
            if (cudaStreamWaitEvent(e->stream, e->joins[q], 0) != cudaSuccess) return PS3D_ERR_CUDA;
        }
        ++e->itt;
        return PS3D_OK;
    }
    if (cudaEventRecord(e->fork, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
    for (size_t q = 0; q < e->groups.size(); ++q) {
        Ctx& g = *e->groups[q];
        if (cudaStreamWaitEvent(g.stream, e->fork, 0) != cudaSuccess) return PS3D_ERR_CUDA;
        int rc = g.step(g.itt, g.tau, g.taum1, g.taum2);
        if (rc) return rc;
        g.rotate();
        g.time = g.time + g.P.dt;
        ++g.itt;
        if (cudaEventRecord(e->joins[q], g.stream) != cudaSuccess) return PS3D_ERR_CUDA;
        if (cudaStreamWaitEvent(e->stream, e->joins[q], 0) != cudaSuccess) return PS3D_ERR_CUDA;
    }
    ++e->itt;
    return PS3D_OK;
}

bool all_graphable(ps3d_ensemble* e) {
    for (auto& g : e->groups)
        if (!g->graphable()) return false;
    return true;
}

int capture(ps3d_ensemble* e) {
    if (e->gexec) { cudaGraphExecDestroy(e->gexec); e->gexec = nullptr; }
    struct Book { int itt, tau, t1, t2, cur[4]; double time; long long launches; bool pend; const double* pcor; double dtp; bool warm; };
    std::vector<Book> saved;
    for (auto& g : e->groups)
        saved.push_back({g->itt, g->tau, g->taum1, g->taum2, {g->cur[0], g->cur[1], g->cur[2], g->cur[3]}, g->time,
                         g->launches, g->pending, g->pcor, g->dtp, g->p_warm});
    const int itt0 = e->itt;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return PS3D_ERR_CUDA;
    int rc = PS3D_OK;
    for (int s = 0; s < 3 && !rc; ++s) rc = step_all(e);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
    for (size_t q = 0; q < e->groups.size(); ++q) {
        Ctx& g = *e->groups[q];
        g.g_launches = g.launches - saved[q].launches;
        g.itt = saved[q].itt; g.tau = saved[q].tau; g.taum1 = saved[q].t1; g.taum2 = saved[q].t2;
        for (int f = 0; f < 4; ++f) g.cur[f] = saved[q].cur[f];
        g.time = saved[q].time;
        g.launches = saved[q].launches;
        g.g_pend_out = g.pending; g.g_pcor_out = g.pcor; g.g_dtp_out = g.dtp; g.g_warm_out = g.p_warm;
        g.pending = saved[q].pend; g.pcor = saved[q].pcor; g.dtp = saved[q].dtp; g.p_warm = saved[q].warm;
        g.g_pend_in = g.pending; g.g_pcor_in = g.pcor; g.g_dtp_in = g.dtp; g.g_warm_in = g.p_warm;
        g.g_tau = g.tau; g.g_cur = g.cur[0];   // the phase of the cycle the graph starts at
    }
    e->itt = itt0;
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (ce != cudaSuccess) return PS3D_ERR_CUDA;
    ce = cudaGraphInstantiate(&e->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return PS3D_ERR_CUDA;
    e->graph_valid = true;
    return PS3D_OK;
}

int advance(ps3d_ensemble* e, int nsteps) {
    // the ensemble stream (where grouped step kernels run) waits for what the
    // groups' streams hold (uploads, the previous call's work)
    for (size_t q = 0; q < e->groups.size(); ++q) {
        if (cudaEventRecord(e->joins[q], e->groups[q]->stream) != cudaSuccess) return PS3D_ERR_CUDA;
        if (cudaStreamWaitEvent(e->stream, e->joins[q], 0) != cudaSuccess) return PS3D_ERR_CUDA;
    }
    while (nsteps > 0) {
        if (nsteps >= 3 && e->itt >= 2 && all_graphable(e)) {
            bool same = true;
            // the same phase of the (tau, state buffer) cycle and the same
            // pending correction and warm start as at the capture
            for (auto& g : e->groups)
                same = same && g->g_pend_in == g->pending && g->g_pcor_in == g->pcor && g->g_dtp_in == g->dtp &&
                       g->g_warm_in == g->p_warm && g->g_tau == g->tau && g->g_cur == g->cur[0];
            if (!e->graph_valid || !same) {
                int rc = capture(e);
                if (rc) return rc;
            }
            if (cudaGraphLaunch(e->gexec, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
            for (auto& g : e->groups)
                for (int s = 0; s < 3; ++s) {
                    g->rotate();
                    for (int f = 0; f < 4; ++f) g->cur[f] = (g->cur[f] + 1) % 3;
                    g->time = g->time + g->P.dt;
                    ++g->itt;
                }
            for (auto& g : e->groups) {
                g->launches += g->g_launches;
                g->pending = g->g_pend_out; g->pcor = g->g_pcor_out; g->dtp = g->g_dtp_out; g->p_warm = g->g_warm_out;
            }
            e->itt += 3;
            nsteps -= 3;
            continue;
        }
        int rc = step_all(e);
        if (rc) return rc;
        --nsteps;
    }
    // what a group's stream runs next (an upload, a download) waits for
    // everything queued so far, graph replays included
    if (cudaEventRecord(e->fork, e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
    for (auto& g : e->groups)
        if (cudaStreamWaitEvent(g->stream, e->fork, 0) != cudaSuccess) return PS3D_ERR_CUDA;
    return PS3D_OK;
}

}  // namespace

namespace ps3d {
// ps3d_ensemble_create with the autotuner's timing runs optional (the
// serving loop creates ensembles while other requests run)
int ensemble_create(const ps3d_params* members, int n, int device, bool tune, ps3d_ensemble** out);
}

#define EGUARD_BEGIN try {
#define EGUARD_END                                         \
    }                                                      \
    catch (const std::bad_alloc&) { return PS3D_ERR_OOM; } \
    catch (...) { return PS3D_ERR_CUDA; }

extern "C" {

PS3D_API int ps3d_ensemble_create(const ps3d_params* members, int n, int device, ps3d_ensemble** out) {
    return ps3d::ensemble_create(members, n, device, true, out);
}

}  // extern "C"

int ps3d::ensemble_create(const ps3d_params* members, int n, int device, bool tune, ps3d_ensemble** out) {
    EGUARD_BEGIN
    if (!members || n < 1 || !out) return PS3D_ERR_BADPARAM;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return PS3D_ERR_CUDA;
    std::unique_ptr<ps3d_ensemble> e(new ps3d_ensemble());
    e->device = device;
    {
        const char* v = std::getenv("PS3D_ENSEMBLE_GROUPED");
        e->grouped = v && v[0] == '1';
    }
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return PS3D_ERR_CUDA;
    // group members with identical parameters, in first-seen order
    std::vector<int> gid(n, -1);
    std::vector<int> leader, count;
    for (int m = 0; m < n; ++m) {
        for (size_t q = 0; q < leader.size(); ++q)
            if (same_params(members[leader[q]], members[m])) { gid[m] = (int)q; break; }
        if (gid[m] < 0) { gid[m] = (int)leader.size(); leader.push_back(m); count.push_back(0); }
        e->where.push_back({gid[m], count[gid[m]]++});
    }
    if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) return PS3D_ERR_CUDA;
    for (size_t q = 0; q < leader.size(); ++q) {
        std::unique_ptr<Ctx> c(new Ctx());
        c->tune_timing = tune;
        int rc = c->init(members[leader[q]], device, count[q]);   // on a stream of its own
        if (rc) return rc;
        e->groups.push_back(std::move(c));
        cudaEvent_t j = nullptr;
        if (cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) return PS3D_ERR_CUDA;
        e->joins.push_back(j);
    }
    *out = e.release();
    return PS3D_OK;
    EGUARD_END
}

extern "C" {

PS3D_API int ps3d_ensemble_destroy(ps3d_ensemble* e) {
    EGUARD_BEGIN
    if (!e) return PS3D_ERR_BADPARAM;
    cudaSetDevice(e->device);
    delete e;
    return PS3D_OK;
    EGUARD_END
}

PS3D_API int ps3d_ensemble_upload(ps3d_ensemble* e, int member, const double* u, const double* v, const double* w,
                                  const double* b) {
    EGUARD_BEGIN
    if (!e || member < 0 || member >= (int)e->where.size()) return PS3D_ERR_BADPARAM;
    cudaSetDevice(e->device);
    Ctx& g = *e->groups[e->where[member].first];
    const int m = e->where[member].second;
    { int rc = g.materialize(); if (rc) return rc; }
    e->graph_valid = false;
    g.p_warm = false;   // the group's next step starts cold (every member)
    const double* f[4] = {u, v, w, b};
    for (int q = 0; q < 4; ++q) {
        int rc = g.upload_field(g.member_field(q, m), f[q]);
        if (rc) return rc;
    }
    return PS3D_OK;
    EGUARD_END
}

PS3D_API int ps3d_ensemble_download(ps3d_ensemble* e, int member, double* u, double* v, double* w, double* b,
                                    double* p) {
    EGUARD_BEGIN
    if (!e || member < 0 || member >= (int)e->where.size()) return PS3D_ERR_BADPARAM;
    cudaSetDevice(e->device);
    Ctx& g = *e->groups[e->where[member].first];
    const int m = e->where[member].second;
    { int rc = g.materialize(); if (rc) return rc; }
    e->graph_valid = false;
    double* f[4] = {u, v, w, b};
    for (int q = 0; q < 4; ++q) {
        int rc = g.download_field(g.member_field(q, m), f[q], 0);
        if (rc) return rc;
    }
    return g.download_field((const double*)g.p.p + (size_t)m * g.N, p, 1);
    EGUARD_END
}

PS3D_API int ps3d_ensemble_enqueue(ps3d_ensemble* e, int nsteps) {
    EGUARD_BEGIN
    if (!e || nsteps < 0) return PS3D_ERR_BADPARAM;
    cudaSetDevice(e->device);
    return advance(e, nsteps);
    EGUARD_END
}

PS3D_API int ps3d_ensemble_integrate(ps3d_ensemble* e, int nsteps) {
    EGUARD_BEGIN
    if (!e || nsteps < 0) return PS3D_ERR_BADPARAM;
    cudaSetDevice(e->device);
    int rc = advance(e, nsteps);
    if (rc) return rc;
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return PS3D_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess) return PS3D_ERR_CUDA;
    return PS3D_OK;
    EGUARD_END
}

PS3D_API int ps3d_ensemble_info(ps3d_ensemble* e, int* ngroups, long long* launches, void** stream) {
    if (!e) return PS3D_ERR_BADPARAM;
    if (ngroups) *ngroups = (int)e->groups.size();
    if (launches) {
        long long t = 0;
        for (auto& g : e->groups) t += g->launches;
        *launches = t;
    }
    if (stream) *stream = (void*)e->stream;
    return PS3D_OK;
}

}  // extern "C"
