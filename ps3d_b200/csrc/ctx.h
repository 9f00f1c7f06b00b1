// ctx.h — the device context of one grid (host-side bookkeeping).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <memory>
#include <string>
#include <vector>
#include "engine.h"

// Return PS3D_ERR_CUDA (or PS3D_ERR_OOM) from an int-returning function when a
// CUDA call fails.
#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t ck_e_ = (call);                                                     \
        if (ck_e_ != cudaSuccess) {                                                     \
            ps3d::note_cuda_error(ck_e_, #call, __FILE__, __LINE__);                    \
            return ck_e_ == cudaErrorMemoryAllocation ? PS3D_ERR_OOM : PS3D_ERR_CUDA;   \
        }                                                                               \
    } while (0)

namespace ps3d {

void note_cuda_error(cudaError_t e, const char* what, const char* file, int line);

// owning device (or pinned host) buffer
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool host = false;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    cudaError_t alloc(size_t n) {
        release();
        cudaError_t e = cudaMalloc(&p, n ? n : 1);
        if (e == cudaSuccess) bytes = n; else p = nullptr;
        return e;
    }
    cudaError_t alloc_host(size_t n) {
        release();
        cudaError_t e = cudaMallocHost(&p, n ? n : 1);
        if (e == cudaSuccess) { bytes = n; host = true; } else p = nullptr;
        return e;
    }
    void release() {
        if (p) { if (host) cudaFreeHost(p); else cudaFree(p); }
        p = nullptr; bytes = 0; host = false;
    }
};

struct DevPlan {
    FFTPlan plan{};
    int n = 0;
    DevBuf dtw, dtwf, dpos, dipos;
    cudaError_t build(int len, int policy = 0);
};

bool fft_length_ok(int n);

enum { kSetSave = 10, kSetAve = 11, kSetSave2 = 12, kSetPT0 = 13, kSetComb = 14 };

struct RampGraph;   // a captured ramped integration (engine.cu)

struct Ctx {
    ps3d_params P{};
    int device = 0;
    int nx = 0, ny = 0, nz = 0, nxh = 0;
    long N = 0, M2 = 0, M = 0;
    bool rigid = true, mixed = false;
    bool refine_full = false;   // PS3D_MIXED_REFINED: a full solve + refinement every step
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    // bytes per stored tendency of field f: FP32 history in the mixed path,
    // except w, whose tendency is dominated by the buoyancy term b/dsqr that
    // the pressure gradient nearly cancels (rounding it to FP32 costs ~1e-5
    // relative in w within 100 steps)
    size_t tsz(int f) const { return (hist32 && f != 2) ? sizeof(float) : sizeof(double); }
    // the mixed path's stored history in FP32 (the default); PS3D_MIXED_HISTORY=64
    // keeps it in FP64, a diagnostic that separates the history's rounding
    // from the FP32 transforms' in the mixed path's error budget
    bool hist32 = false;
    int batch = 1;            // instances of this grid stepped together (ensembles)
    int cap = 1;              // instances the buffers hold (batch <= cap; set_active_batch)
    // CUDA graphs of three consecutive steps (tau and the state buffers both
    // cycle with period 3), replayed by advance() for constant parameters: one
    // per phase of the cycle (slot tau - 1), so that calls of any length keep
    // replaying without a new capture
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        int tau = -1, cur = -1;
        long version = -1;
        long long launches = 0;
        bool pend_in = false, pend_out = false;
        const double* pcor_in = nullptr;
        const double* pcor_out = nullptr;
        double dtp_in = 0.0, dtp_out = 0.0;
        bool warm_in = false, warm_out = false;
    };
    GraphSlot gslot[3];
    // the ensemble's capture bookkeeping (ensemble.cu): outputs of its last
    // capture and the inputs it was captured with
    int g_tau = -1, g_cur = -1;
    long version = 0;
    long long g_launches = 0;
    bool g_pend_in = false, g_pend_out = false;
    const double* g_pcor_in = nullptr;
    const double* g_pcor_out = nullptr;
    double g_dtp_in = 0.0, g_dtp_out = 0.0;
    bool g_warm_in = false, g_warm_out = false;
    bool use_graphs = true;
    std::atomic<int>* cancel_flag = nullptr;   // serving: set to abandon a running request
    bool cancelled() const { return cancel_flag && cancel_flag->load(std::memory_order_relaxed) != 0; }
    // state
    DevBuf state[4][3];
    int cur[4] = {0, 0, 0, 0};
    DevBuf p;
    DevBuf tend[4];           // 3 time levels each
    DevBuf FS;                // spectral work array of the Poisson solve
    // projections
    DevBuf spec4[4], g0base, qtmp;
    DevBuf bal[4], base[4], zero[4], save[4], ave[4], save2[4];
    // Warn-et-al. balance: components u1..b3, pTu0..pTb0, combinations,
    // advective tendencies and the spectral work arrays (warn.cu)
    DevBuf first[4], second[4], third[4], pt0[4], comb[4], nl_tend[4];
    DevBuf warn_arr[19];
    // asynchronous snapshots (restart.cu)
    DevBuf snap[5], snap_staging;
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_event = nullptr;
    int warn_filter = -1;
    // ramp graphs of the optimal balance (engine.cu), kept across calls
    std::shared_ptr<std::vector<RampGraph>> ramp_graphs;
    DevBuf saved_p, saved_tend[4];
    // tables
    DevPlan plx, ply, plz;      // radix-16/8 schedules
    DevPlan plx4, ply4;         // radix-4 schedules (autotuner alternative)
    DevPlan plx8, ply8;         // radix-8 schedules (autotuner alternative)
    DevPlan plyh;               // length ny/2 (the y-split solve, k_colsolve)
    int plane_force = -1;       // PS3D_PLANE_IMPL: -1 free, 0 cluster, 1 rows + y-lines
    int force_impl = -1;        // set before init: pins the plane implementation (z-slabs: 1)
    // z-slab of a larger grid (slab.cu): the step kernel advances levels
    // win_kbeg .. win_kbeg+win_kcount-1 whose global level is k + win_kofs of
    // win_nzg, and step() stops after it (the slab driver runs the solve)
    int win_kbeg = 0, win_kcount = 0, win_kofs = 0, win_nzg = 0;
    bool split_solve = false;
    int kchunk = 8;             // z levels per block of the step kernel
    bool tune_timing = true;    // false: the autotuner takes cached choices or the defaults, no timing runs
    std::string tuned;          // description of the autotuned choice
    DevBuf twx;
    DevBuf t_kx, t_ky, t_kz, t_hkx, t_hky, t_hkz, t_ex, t_ey, t_ez, t_px, t_py, t_pz, t_sz, t_cz, t_hkz_ds;
    DevBuf m_phi, m_psi, m_psib;
    DevPlan pl2z;               // rigid lid: length 2 nz, the vertical-mode transforms by FFT
    DevPlan pl1z;               // ... and length nz (phi and psib for even nz)
    DevBuf t_dtw;               // ... and e^{i pi j / 2 nz}, j = 0 .. nz-1
    bool vmode_fft = false;     // the vertical-mode transforms run by FFT (launch_vert_dtt)
    int vmode_transform(const double2* in, double2* out, int f, bool fwd);
    PlaneArgs pa64{}, pa32{};
    // forcing
    int fkind = 0;
    long forcing_gen = 0;     // counts set_forcing calls (keys of the ramp graphs)
    double omega = 0.0;
    DevBuf wr[4], wi[4], ub, bb;
    ps3d_forcing_fn fn = nullptr;
    void* user = nullptr;
    // time levels (main_module.f90:55-59)
    int itt = 0, tau = 3, taum1 = 2, taum2 = 1;
    double time = 0.0;
    // pending pressure-gradient correction (lazy K5): the state arrays hold
    // u'' and the true velocity is u'' - dtp*grad(*pcor); the next step's
    // stencil kernel applies it while loading
    bool pending = false;
    const double* pcor = nullptr;
    double dtp = 0.0;
    bool lazy_correction = true;
    // p holds the pressure of the previous step's projection of this
    // trajectory (set by the time step's solve, cleared whenever the state
    // or p is replaced from outside the time loop): the mixed path then
    // solves only for the FP64 residual against it
    bool p_warm = false;
    bool warm_solve() const { return mixed && !refine_full && p_warm; }
    // per-kernel event timing (ps3d_profile)
    bool prof = false;
    struct ProfRec { int kid; cudaEvent_t e0, e1; };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> prof_pool;
    size_t prof_next = 0;
    long long launches = 0;
    cudaEvent_t prof_event();
    void prof_begin(int kid, cudaEvent_t* e0);
    void prof_end(int kid, cudaEvent_t e0);
    int prof_read(double* ms, long long* count);
    // reductions / staging
    int nred = 0;
    DevBuf red_partials, red_out, staging;
    DevBuf norms;             // a batched optimal balance's per-instance norms (4 doubles each)
    // kernel error word in mapped page-locked memory: kernels whose bounded
    // waits ran out store 1; read after every stream synchronisation
    unsigned* kerr_h = nullptr;
    unsigned* kerr_d = nullptr;

    ~Ctx() {
        for (GraphSlot& s : gslot)
            if (s.exec) cudaGraphExecDestroy(s.exec);
        if (stream) { cudaStreamSynchronize(stream); if (own_stream) cudaStreamDestroy(stream); }
        for (cudaEvent_t e : prof_pool) cudaEventDestroy(e);
        if (snap_stream) { cudaStreamSynchronize(snap_stream); cudaStreamDestroy(snap_stream); }
        if (snap_event) cudaEventDestroy(snap_event);
        if (kerr_h) cudaFreeHost(kerr_h);
    }

    double* field(int f) { return (double*)state[f][cur[f]].p; }
    void rotate() {
        tau = tau % 3 + 1;
        taum1 = taum1 % 3 + 1;
        taum2 = taum2 % 3 + 1;
    }
    int sync() {
        CK(cudaStreamSynchronize(stream));
        CK(cudaGetLastError());
        if (kerr_h && *(volatile unsigned*)kerr_h) {
            *(volatile unsigned*)kerr_h = 0;
            return PS3D_ERR_TIMEOUT;
        }
        return PS3D_OK;
    }

    int init(const ps3d_params& prm, int dev, int nbatch = 1, cudaStream_t use_stream = nullptr);
    int autotune();
    int advance(int nsteps, bool allow_graph);
    bool graphable() const;
    int capture_graph(GraphSlot& slot);
    // parameters changed outside the time loop: captured graphs are stale
    void invalidate_graph() { ++version; }
    // the state or p replaced outside the time loop: graphs are stale, and p
    // no longer holds the previous step's pressure of this trajectory
    void state_replaced() { ++version; p_warm = false; }
    int step(int itt, int tau, int taum1, int taum2);
    // run the first b <= cap instances (a pooled serving context of cap
    // instances taking a smaller group); captured graphs are kept per batch
    int set_active_batch(int b);
    // Grouped step launches (an ensemble's groups in one step-kernel launch):
    // with defer_step set, step() of a fused step does the step kernel's
    // bookkeeping and writes its arguments to *defer_step instead of
    // launching it; the caller launches the kernel, then step_finish() runs
    // the rest of the step (the pressure solve) on this context's stream.
    StepArgs* defer_step = nullptr;
    bool fused_step() const;
    int step_finish() { return pressure_solve(lazy_correction, true); }
    int poisson_once(double* out, double beta, bool lazy = false, const double* pc = nullptr);
    int pressure_solve(bool lazy = false, bool warm = false);
    int materialize();        // apply a pending correction so the state arrays hold the true state
    int forward_transform(const double* const* in);
    int backward_transform(double* const* out);
    int project(int mode);
    int project_spectral(int mode);
    // restart.f90 record layout (restart.cu)
    int write_restart(const char* path);
    int read_restart(const char* path, double* time_out);
    int snapshot_begin(double* const* host);
    int snapshot_wait();
    // Warn-et-al. balance (warn.cu)
    int diag_balance(int order, int filter_width);
    cudaError_t ensure_warn();
    int warn_launch(int mode, double2* o1 = nullptr, double2* o2 = nullptr, double kzcut2 = 0.0);
    int model_nonlin(const double* const* in);
    int model_nonlin_set(int set);
    int warn_comb(int set_a, int set_b, double s, bool divide);
    int backward_to_set(int set);
    int model_run(int in, int out, int max_steps);
    int warn_first();
    int warn_second();
    int warn_third();
    int diagnose(double* ke, double* pe, double* umax, double* wmax, int member = 0);
    int opt_time_ave(int set, int n_end_ave);
    int opt_balance(const ps3d_optbal& O, double* final_norm, int* iters);
    int reset_request();      // back to the just-created state (the serving pool reuses contexts)
    int ramp_run(bool backward, int n_end, double Ro_loc, double dt_loc, double period, void* graphs);
    int set_forcing(const ps3d_forcing* f);

    cudaError_t ensure_spectral4();
    cudaError_t ensure_fieldset(int which);
    cudaError_t ensure_saved_tail();
    cudaError_t ensure_staging();
    DevBuf* fieldset(int which);
    cudaError_t copy_state_to(int set);
    cudaError_t copy_set_to_state(int set);

    int upload_raw(void* dev, const double* h, bool f32);
    int download_raw(const void* dev, double* h, bool pghost, bool f32);
    int upload_field(double* dev, const double* h);
    double* member_field(int f, int m) { return field(f) + (size_t)m * N; }
    int download_field(const double* dev, double* h, int kind);
    int upload_tend(int f, const double* h);
    int download_tend(int f, double* h);
};

}  // namespace ps3d
