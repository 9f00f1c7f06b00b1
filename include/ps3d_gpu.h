/*
 * ps3d_gpu.h — C ABI of the B200 (sm_100a) ps3D time-step engine.
 *
 * The reference model (ceden/ps3D) keeps its state in Fortran module globals
 * (for_src/main_module.f90:3-108) and its hot path is a set of argument-less
 * subroutines: integrate (for_src/integrate.f90:2-115), pressure_solver
 * (for_src/pressure_solver.f90:2-120), the normal-mode projections
 * (for_src/diag_opt_balance.f90:263-335, for_src/diag_balance.f90:109-132),
 * diag_opt_balance (for_src/diag_opt_balance.f90:55-179) and diagnose
 * (for_src/diagnose.F90:2-61).  This header replaces those with entry points
 * on an opaque context that owns the device-resident state.  Every entry point
 * takes plain pointers and sizes, returns an int status (0 = success, negative
 * = error) and never aborts or traps; a Fortran host binds them through
 * ISO_C_BINDING: each entry point is a bind(C) interface with value and
 * reference arguments matching the C types below.
 *
 * Host arrays use the reference's layout: real(8) fields are column-major,
 * x fastest, with two halo points on every side, i.e. Fortran bounds
 * (1-2:nx+2, 1-2:ny+2, 1-2:nz+2) -> (nx+4)*(ny+4)*(nz+4) doubles.  Tendency
 * arrays carry the trailing time-level dimension of 3
 * (for_src/main_module.f90:124-127): 3*(nx+4)*(ny+4)*(nz+4) doubles.
 * Time-level indices tau/taum1/taum2 are 1-based as in Fortran.
 */
#ifndef PS3D_GPU_H
#define PS3D_GPU_H

#include <stddef.h>

#if defined(__GNUC__)
#define PS3D_API __attribute__((visibility("default")))
#else
#define PS3D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PS3D_OK                0
#define PS3D_ERR_CUDA         -1  /* a CUDA runtime call failed                     */
#define PS3D_ERR_NONFINITE    -2  /* NaN/Inf found in the state (diagnose.F90:42-45) */
#define PS3D_ERR_TIMEOUT      -3  /* a bounded device or host wait ran out          */
#define PS3D_ERR_OOM          -4  /* device allocation or admission budget refused  */
#define PS3D_ERR_BADPARAM     -5  /* invalid argument, size or configuration        */
#define PS3D_ERR_UNSUPPORTED  -6  /* valid in the reference, not built here         */
#define PS3D_ERR_CANCELLED    -7  /* a serving request was cancelled                */
#define PS3D_ERR_TOOLARGE     -8  /* grid exceeds a fixed limit: columns too tall for a block's
                                       shared memory, or ps3d_pressure_solve_noalloc's static scratch */

/* ---- parameters (for_src/main_module.f90:16-57) -------------------------- */
typedef struct ps3d_params {
    int nx, ny, nz;                       /* grid points                       */
    double Lx, Ly, Lz;                    /* domain extent (m)                 */
    double dx, dy, dz;                    /* cell size (m)                     */
    double dt;                            /* time step (s)                     */
    double f0, N0;                        /* Coriolis and stability freq.      */
    double Ro, dsqr;                      /* Rossby number, aspect ratio^2     */
    double eps_ab;                        /* AB2 weighting (main_module.f90:56)*/
    double Ah, Av, Kh, Kv;                /* harmonic viscosity / diffusivity  */
    double Ahbi, Avbi, Khbi, Kvbi;        /* biharmonic coefficients           */
    int enable_nonlinear;                 /* main_module.f90:16                */
    int enable_vertical_boundaries;       /* rigid lid (1) or periodic z (0)   */
    int enable_AB_3_order;                /* AB3 (1) or AB2 (0)                */
    int precision;                        /* PS3D_FP64, PS3D_MIXED(_REFINED)   */
} ps3d_params;

#define PS3D_FP64  0   /* every kernel in FP64                                  */
#define PS3D_MIXED 1   /* FP32 stencils/FFTs, FP64 state, tridiagonal, AB and
                          eigen-projection; the Poisson solve is one FP64-residual
                          refinement step per time step, started from the previous
                          step's pressure (a full FP32 solve first after create or
                          an upload): one solve per step, divergence left at the
                          FP32 rounding of the step's change of p              */
#define PS3D_MIXED_REFINED 2   /* as PS3D_MIXED with a full FP32 solve and one
                          FP64-residual refinement at every step: two solves per
                          step, divergence left at FP64 roundoff              */

/* ---- optimal balance knobs (for_src/main_module.f90:24-30) ------------- */
typedef struct ps3d_optbal {
    double period;        /* opt_balance_period: ramp length in s            */
    double average;       /* opt_balance_average (time-averaging variant)    */
    int max_itts;         /* opt_balance_max_Itts                            */
    int average_times;    /* opt_balance_average_times                       */
    double tol;           /* opt_balance_tol                                 */
    int enable_time_ave;  /* enable_diag_opt_time_ave                        */
    int adopt;            /* 1: copy the balanced fields into u,v,w,b at the
                             end, as for_config/test_opt_balance.f90:240-241 */
} ps3d_optbal;

/* ---- user forcing (set_forcing hook, for_src/integrate.f90:82) ---------- */
/* Device view handed to a host forcing callback: interior-only device arrays
 * (x fastest, nx*ny*nz doubles), already friction-updated, and the tendency
 * slot of the current time level.  The callback may launch its own kernels on
 * `stream`; it runs between friction and the Adams-Bashforth update.        */
typedef struct ps3d_device_view {
    int nx, ny, nz;
    double *u, *v, *w, *b;                /* state being stepped             */
    double *du, *dv, *dw, *db;            /* tendencies of time level tau    */
    double dt, Ro;
    int itt;
    void* stream;                         /* cudaStream_t                    */
} ps3d_device_view;

typedef int (*ps3d_forcing_fn)(void* user, const ps3d_device_view* view);

#define PS3D_FORCE_NONE        0
#define PS3D_FORCE_WAVEMAKER   1  /* u += dt*(cos(omega t) u_r + sin(omega t) u_i),
                                     t = dt*itt (for_src/config.f90:224-237)     */
#define PS3D_FORCE_BACKGROUND  2  /* advection by/of a background flow U(x,y,z)
                                     and buoyancy B(x,y,z)
                                     (for_config/lee_wave1.f90:245-312)          */
#define PS3D_FORCE_CALLBACK    4  /* host callback with device pointers          */

typedef struct ps3d_forcing {
    int kind;                             /* bitwise OR of PS3D_FORCE_*      */
    double omega;                         /* wavemaker frequency             */
    /* wavemaker fields, halo layout, NULL = zero field                       */
    const double *u_r, *v_r, *w_r, *b_r, *u_i, *v_i, *w_i, *b_i;
    /* background flow fields, halo layout, NULL = zero field                 */
    const double *u_back, *b_back;
    ps3d_forcing_fn fn;                   /* PS3D_FORCE_CALLBACK             */
    void* user;
} ps3d_forcing;

typedef struct ps3d_ctx ps3d_ctx;

/* Replaces allocate_main_module (main_module.f90:112-144) and
 * wavenumber_initialisation (my_fft.f90:87-156) for one rank on one GPU:
 * allocates the device state, wavenumber and vertical-mode tables.
 * nx, ny must be even (main.f90:45-55) and nz even in periodic mode; every
 * FFT length (nx/2, ny and, periodic, nz) must factor into 2, 3 and 5.     */
PS3D_API int ps3d_create(const ps3d_params* prm, int device, ps3d_ctx** out);
PS3D_API int ps3d_destroy(ps3d_ctx* ctx);

/* Copy the model state in the reference's halo layout to/from the device
 * (u,v,w,b,p: main_module.f90:64-68; du..db with their 3 time levels) and set
 * or read the time-level indices (main_module.f90:55,58).  Any pointer may be
 * NULL on download to skip that field; on upload a NULL tendency pointer
 * zero-fills those time levels.                                             */
PS3D_API int ps3d_upload_state(ps3d_ctx* ctx,
                      const double* u, const double* v, const double* w,
                      const double* b, const double* p,
                      const double* du, const double* dv, const double* dw,
                      const double* db,
                      int itt, int tau, int taum1, int taum2);
PS3D_API int ps3d_download_state(ps3d_ctx* ctx,
                        double* u, double* v, double* w, double* b, double* p,
                        double* du, double* dv, double* dw, double* db,
                        int* itt, int* tau, int* taum1, int* taum2);

/* integrate (integrate.f90:2-115) once, with the caller's time-level indices
 * and step counter; it does not rotate them (the caller does, as main.f90:156-160). */
PS3D_API int ps3d_step(ps3d_ctx* ctx, int itt, int tau, int taum1, int taum2);

/* nsteps iterations of the main loop body (main.f90:139-162 without the
 * diagnostics): integrate, rotate tau/taum1/taum2, time += dt, itt += 1.
 * Device resident; returns after the work is queued and completed.          */
PS3D_API int ps3d_integrate(ps3d_ctx* ctx, int nsteps);

/* Change the per-step parameters the balance drivers ramp
 * (diag_opt_balance.f90:191-198,221-224).                                    */
PS3D_API int ps3d_set_step_params(ps3d_ctx* ctx, double dt, double Ro,
                         double Ahbi, double Avbi, double Khbi, double Kvbi);

/* pressure_solver (pressure_solver.f90:2-120) on the current device state.
 * The mixed paths solve from scratch here (a full FP32 solve and one
 * FP64-residual refinement): only the time step's solve starts from the
 * previous step's pressure.                                                 */
PS3D_API int ps3d_pressure_solve(ps3d_ctx* ctx);

/* Normal-mode projections on the device state:
 *  PS3D_PROJ_NORMAL_MODE   normal_mode_projection   (diag_opt_balance.f90:288-310)
 *  PS3D_PROJ_BASE_POINT    geostrophic_base_point   (diag_opt_balance.f90:263-285):
 *                          stores g0_base and returns the base point in u_base
 *  PS3D_PROJ_EXCHANGE      exchange_geostrophic_base_point (diag_opt_balance.f90:313-335)
 *  PS3D_PROJ_ZERO_ORDER    diag_balance_zero_order  (diag_balance.f90:109-132):
 *                          writes u0..b0, readable with ps3d_get_fields       */
#define PS3D_PROJ_NORMAL_MODE 0
#define PS3D_PROJ_BASE_POINT  1
#define PS3D_PROJ_EXCHANGE    2
#define PS3D_PROJ_ZERO_ORDER  3
PS3D_API int ps3d_project_geostrophic(ps3d_ctx* ctx, int mode);

/* diag_opt_balance (diag_opt_balance.f90:55-179) on the device state.  The
 * model state is restored on return (as :172-176); the balanced fields are
 * kept (u_bal) and copied into the state when opt->adopt is set.            */
PS3D_API int ps3d_opt_balance(ps3d_ctx* ctx, const ps3d_optbal* opt,
                     double* final_norm, int* iters);

/* diag_balance (diag_balance.f90:89-106) without its netCDF output: the
 * Warn-et-al. normal-mode balance of the current state to `order` (0..3):
 * diag_balance_zero_order (:109-132), _first_order (:135-176),
 * _second_order (:180-272) and _third_order (:275-362), with model_nonlin
 * (:500-535) and model_run (:465-497).  The components u0..b0, u1..b1,
 * u2..b2, u3..b3 are read with ps3d_get_fields(PS3D_FIELDS_ZERO .. _THIRD);
 * the balanced state is their sum (for_config/eddy1.f90:111-133).
 * filter_width >= 0 turns on enable_diag_balance_filter with
 * diag_balance_filter_width = filter_width (main_module.f90:22-23); < 0
 * leaves it off.  The model state and time levels are unchanged.         */
PS3D_API int ps3d_diag_balance(ps3d_ctx* ctx, int order, int filter_width);

/* write_restart / read_restart (restart.f90:2-82) for one rank: the file
 * the reference writes as restart_pe=000000000.dta, a Fortran unformatted
 * sequential file with 4-byte record markers holding (nx, ny, nz, itt,
 * time, taum2, taum1, tau), the rank bounds (1, nx, 1, ny, 1, nz) and
 * u, v, w, b, p, du, dv, dw, db in the halo layout.  Records longer than
 * 2147483639 bytes are split into subrecords with negative continuation
 * markers (gfortran's layout for records beyond 2 GiB).  read_restart
 * returns PS3D_ERR_BADPARAM where the reference aborts (grid or bounds
 * mismatch, short or malformed file) and stores the file's time in *time
 * (the reference adds it to runlen); itt, time and the time levels of the
 * context are set from the file.                                            */
PS3D_API int ps3d_write_restart(ps3d_ctx* ctx, const char* path);
PS3D_API int ps3d_read_restart(ps3d_ctx* ctx, const char* path, double* time);

/* Asynchronous snapshot, no counterpart in the reference (whose snapshots,
 * main.f90:144-152, write netCDF synchronously): the state and p as they
 * are at the call are copied on the device, then converted to the halo
 * layout and copied into the host arrays on a second stream while the next
 * steps run.  Any array may be NULL.  The host arrays (page-locked for the
 * copies to overlap) must stay valid until ps3d_snapshot_wait returns; a
 * new ps3d_snapshot_begin first waits for the previous one.                */
PS3D_API int ps3d_snapshot_begin(ps3d_ctx* ctx, double* u, double* v, double* w, double* b, double* p);
PS3D_API int ps3d_snapshot_wait(ps3d_ctx* ctx);

/* Auxiliary field sets in halo layout (u,v,w,b; any may be NULL).          */
#define PS3D_FIELDS_STATE    0   /* u, v, w, b                         */
#define PS3D_FIELDS_BALANCED 1   /* u_bal..b_bal  (diag_opt_balance)   */
#define PS3D_FIELDS_BASE     2   /* u_base..b_base                     */
#define PS3D_FIELDS_ZERO     3   /* u0..b0 (diag_balance_zero_order)   */
#define PS3D_FIELDS_FIRST    4   /* u1..b1 (diag_balance_first_order)  */
#define PS3D_FIELDS_SECOND   5   /* u2..b2 (diag_balance_second_order) */
#define PS3D_FIELDS_THIRD    6   /* u3..b3 (diag_balance_third_order)  */
PS3D_API int ps3d_get_fields(ps3d_ctx* ctx, int which,
                    double* u, double* v, double* w, double* b);

/* diagnose (diagnose.F90:2-61) reductions: mean KE and PE, max horizontal and
 * vertical speed.  Returns PS3D_ERR_NONFINITE when any of u,v,w,b,p holds a
 * NaN or Inf (the reference aborts there, diagnose.F90:42-45).              */
PS3D_API int ps3d_diagnose(ps3d_ctx* ctx, double* ke, double* pe,
                  double* umax, double* wmax);

/* Install the set_forcing hook (integrate.f90:82).  Field arrays are copied
 * to the device during the call.                                            */
PS3D_API int ps3d_set_forcing(ps3d_ctx* ctx, const ps3d_forcing* f);

PS3D_API const char* ps3d_strerror(int status);

/* ---- engine extensions (no counterpart in the reference) ----------------
 * The CUDA stream the context queues its kernels on (a cudaStream_t).      */
PS3D_API int ps3d_get_stream(ps3d_ctx* ctx, void** stream);
/* ps3d_integrate without the final synchronisation: queues nsteps on the
 * context's stream and returns; errors of queued work surface at the next
 * synchronising call.                                                      */
PS3D_API int ps3d_enqueue(ps3d_ctx* ctx, int nsteps);
/* Per-kernel CUDA-event timing.  ps3d_profile(ctx, 1) clears and starts
 * recording an event pair around every launch; ps3d_profile_read waits for
 * the stream and returns, per kernel class (PS3D_K_*), the summed device
 * milliseconds and the number of launches.                                 */
#define PS3D_K_STEP     0   /* fused tendency/friction/AB kernel            */
#define PS3D_K_FFT_FWD  1   /* divergence + forward plane FFT               */
#define PS3D_K_VSOLVE   2   /* vertical Thomas / periodic z solve           */
#define PS3D_K_FFT_INV  3   /* inverse plane FFT                            */
#define PS3D_K_CORRECT  4   /* pressure-gradient correction                 */
#define PS3D_K_OTHER    5   /* friction stages, forcing, projections, ...   */
#define PS3D_K_VMODE    6   /* vertical-mode transforms (rigid-lid projections) */
#define PS3D_K_COUNT    7
PS3D_API int ps3d_profile(ps3d_ctx* ctx, int enable);
/* One-line description of the context's kernel configuration (grid,
 * precision, plane cluster shape, FFT stages, autotuner choice).          */
PS3D_API int ps3d_describe(ps3d_ctx* ctx, char* buf, int len);
PS3D_API int ps3d_profile_read(ps3d_ctx* ctx, double* ms, long long* launches);

/* ---- pressure projection without device allocation -----------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need the projection (they own their device arrays through CUDA
 * Fortran, OpenACC or their own pool, hold a lock their allocator also
 * takes, or must keep a fixed device footprint): the same computation as
 * ps3d_pressure_solve (pressure_solver.f90:2-120, FP64) on the caller's
 * device arrays u, v, w (updated in place) and p (written), each nx*ny*nz
 * doubles, x fastest, interior points only, queued on `stream` (a
 * cudaStream_t, NULL for the default stream) and waited for: the call is
 * synchronous, and cannot be captured in a CUDA graph.  It allocates no
 * device memory: the spectral work array and the FFT tables are file-scope
 * static device arrays (about 16.1 MiB, held on every GPU that loads the
 * library until exit), and the host image of the tables is a static buffer.
 * (nx/2+1)*ny*nz must not exceed 1048576 and nx/2, ny, nz not 1024, and
 * periodic grids nz not about 420 (the z transform's shared memory), else
 * PS3D_ERR_TOOLARGE.  The first call on a device looks up the
 * static arrays with that device current.  Calls from threads of one
 * process are serialised by the library; calls from several processes that
 * overlap on one GPU race on the arrays.                                   */
PS3D_API int ps3d_pressure_solve_noalloc(const ps3d_params* prm, double* u, double* v, double* w, double* p,
                                         void* stream);

/* ---- batched ensembles (no counterpart in the reference) -----------------
 * n independent grids on one GPU.  Members with identical ps3d_params share
 * every kernel launch (the member index is part of the launch grid); all
 * members advance together with the main-loop semantics of ps3d_integrate,
 * and for constant parameters three steps of every member are replayed as
 * one CUDA graph.  Upload/download use the halo layout of each member.     */
typedef struct ps3d_ensemble ps3d_ensemble;
PS3D_API int ps3d_ensemble_create(const ps3d_params* members, int n, int device, ps3d_ensemble** out);
PS3D_API int ps3d_ensemble_destroy(ps3d_ensemble* e);
PS3D_API int ps3d_ensemble_upload(ps3d_ensemble* e, int member, const double* u, const double* v,
                                  const double* w, const double* b);
PS3D_API int ps3d_ensemble_download(ps3d_ensemble* e, int member, double* u, double* v, double* w,
                                    double* b, double* p);
PS3D_API int ps3d_ensemble_integrate(ps3d_ensemble* e, int nsteps);   /* waits for completion */
PS3D_API int ps3d_ensemble_enqueue(ps3d_ensemble* e, int nsteps);     /* queues only         */
PS3D_API int ps3d_ensemble_info(ps3d_ensemble* e, int* ngroups, long long* launches, void** stream);

/* ---- one grid over several GPUs: z-slabs -----------------------------------
 * Replaces the reference's MPI decomposition inside P3DFFT (my_fft.f90,
 * p3dfft_setup; pressure_solver.f90 on its pencils) for the time step: rank r
 * of nranks owns global levels k0 = r*nzl .. k0+nzl-1 (nzl = nz/nranks >= 2).
 * A step is the phases below, in this order, each queued on the slab's
 * stream (ps3d_slab_info); between them the caller moves data between ranks:
 *   TENDENCY, PACK_STATE, [halo exchange], UNPACK_STATE, then `passes` times
 *   (ps3d_slab_info, read before each step: 1 for FP64; for the mixed path 2
 *   on the first step after create or upload, a full solve and its
 *   FP64-residual refinement, then 1, the residual solve against the
 *   previous step's pressure) FORWARD, [all-to-all: xbuf -> colbuf], VSOLVE,
 *   [all-to-all: colbuf -> xbuf], INVERSE, PACK_P, [halo exchange], UNPACK_P;
 *   then END_STEP.
 * Halo exchange: hsend holds [planes for the rank below][planes for the rank
 * above] (state: 4 and 4 planes of nx*ny doubles; p: 2 and 1); hrecv receives
 * [what the rank below sent up][what the rank above sent down]; z is
 * periodic over the ranks.  All-to-all: xbuf is [r][nzl][ccnt[r]] complex
 * (blocks for rank r in rank order), colbuf is [nranks][nzl][ccnt[rank]]
 * (complex double, or complex float in the mixed path).
 * Before the first step after an upload the state halos are exchanged once
 * (PACK_STATE, exchange, UNPACK_STATE).  ps3d_slab_group_step does all of it
 * for the ranks of one process (device copies; one GPU or several).
 * Upload/download take the rank's interior levels, [nzl][ny][nx] doubles,
 * x fastest (no halos).  Rigid lid or triply periodic, the fused step
 * (Laplacian friction, wavemaker and background-flow forcing; not
 * biharmonic friction, a host callback, or background flow together with
 * Laplacian friction: PS3D_ERR_UNSUPPORTED).                               */
#define PS3D_SLAB_TENDENCY     0
#define PS3D_SLAB_PACK_STATE   1
#define PS3D_SLAB_UNPACK_STATE 2
#define PS3D_SLAB_FORWARD      3
#define PS3D_SLAB_VSOLVE       4
#define PS3D_SLAB_INVERSE      5
#define PS3D_SLAB_PACK_P       6
#define PS3D_SLAB_UNPACK_P     7
#define PS3D_SLAB_END_STEP     8
typedef struct ps3d_slab ps3d_slab;
PS3D_API int ps3d_slab_create(const ps3d_params* global, int nranks, int rank, int device, ps3d_slab** out);
PS3D_API int ps3d_slab_destroy(ps3d_slab* s);
PS3D_API int ps3d_slab_info(ps3d_slab* s, int* k0, int* nzl, long long* col0, long long* ncl, void** stream,
                             int* passes);
/* sizes of the exchange buffers and every rank's column count (nranks entries) */
PS3D_API int ps3d_slab_buffers(ps3d_slab* s, size_t* xbytes, size_t* colbytes, size_t* hbytes,
                               long long* col_counts);
/* use caller-owned device buffers (e.g. the tensors a collective library
 * sends from and receives into) instead of the slab's own                 */
PS3D_API int ps3d_slab_bind(ps3d_slab* s, void* xbuf, void* colbuf, void* hsend, void* hrecv);
PS3D_API int ps3d_slab_upload(ps3d_slab* s, const double* u, const double* v, const double* w, const double* b);
/* applies the pending pressure correction first; waits for the stream      */
PS3D_API int ps3d_slab_download(ps3d_slab* s, double* u, double* v, double* w, double* b, double* p);
/* diagnose (diagnose.F90:2-61) over the rank's levels, for a global
 * reduction (global_sum / global_max, parallel_mpi.f90:37-67): the sums of
 * the kinetic and potential energy density over the rank's points (divide
 * the ranks' total by nx ny nz), |u_h| max, |w| max, and 1 where a value is
 * not finite.  Applies the pending pressure correction first; the values
 * are filled whatever the state, so every rank takes part in the reduction. */
PS3D_API int ps3d_slab_diagnose(ps3d_slab* s, double* ke_sum, double* pe_sum, double* umax, double* wmax,
                                int* nonfinite);
/* set_forcing (lee_wave1.f90:232-332; config.f90:224-237) for the rank's
 * levels: kind PS3D_FORCE_WAVEMAKER and/or PS3D_FORCE_BACKGROUND (NONE
 * clears).  Every field pointer of f (NULL = zero field) holds the rank's
 * levels with one halo level each side, [nzl+2][ny][nx] doubles: global
 * levels k0-1 .. k0+nzl, taken periodically in z (the rigid-lid masks never
 * read the wrapped levels).  The callback kind is not supported on slabs.   */
PS3D_API int ps3d_slab_set_forcing(ps3d_slab* s, const ps3d_forcing* f);
PS3D_API int ps3d_slab_phase(ps3d_slab* s, int phase);
PS3D_API int ps3d_slab_sync(ps3d_slab* s);
PS3D_API int ps3d_slab_group_step(ps3d_slab* const* ranks, int n, int nsteps);

/* ---- serving loop for optimal-balance and ensemble requests (no
 * counterpart in the reference) -------------------------------------------
 * Requests (one diag_opt_balance each, on their own grid and state, or one
 * ensemble run) are admitted in arrival order as execution slots and device
 * memory free up:
 * the sum of the admitted requests' footprints (ps3d_server_footprint) stays
 * within hbm_budget_bytes (0: 80% of free memory).  Each admitted request
 * runs on its own CUDA stream, so concurrent requests overlap on the GPU;
 * a request's result does not depend on what else is running.           */
typedef struct ps3d_server ps3d_server;
PS3D_API int ps3d_server_create(int device, size_t hbm_budget_bytes, int max_active, ps3d_server** out);
PS3D_API int ps3d_server_destroy(ps3d_server* s);   /* cancels what is still queued or running */
/* copies the halo-layout inputs; PS3D_ERR_OOM if the request can never fit */
PS3D_API int ps3d_server_submit(ps3d_server* s, const ps3d_params* prm, const ps3d_optbal* opt,
                                const double* u, const double* v, const double* w, const double* b,
                                long long* ticket);
/* waits at most timeout_ms (PS3D_ERR_TIMEOUT otherwise); returns the request's
 * status, copies u_bal..b_bal (NULL to skip) and fills res[6] = {status,
 * final norm, iterations, latency ms, queue ms, run ms}.  A finished request
 * is handed out once.                                                      */
PS3D_API int ps3d_server_wait(ps3d_server* s, long long ticket, int timeout_ms,
                              double* u_bal, double* v_bal, double* w_bal, double* b_bal, double* res);
/* An ensemble run as a request: members[0..n-1] (any grid sizes), each
 * advanced nsteps main-loop steps from its halo-layout u[m], v[m], w[m],
 * b[m] in batched launches (ps3d_ensemble_*); its footprint is the sum of the
 * members'.  ps3d_server_wait_ensemble copies member m's final state to
 * u[m] .. b[m] (any array or entry NULL to skip) and fills res[6] as
 * ps3d_server_wait does (norm 0, iterations = nsteps).                     */
PS3D_API int ps3d_server_submit_ensemble(ps3d_server* s, const ps3d_params* members, int n, int nsteps,
                                         const double* const* u, const double* const* v, const double* const* w,
                                         const double* const* b, long long* ticket);
PS3D_API int ps3d_server_wait_ensemble(ps3d_server* s, long long ticket, int timeout_ms, double* const* u,
                                       double* const* v, double* const* w, double* const* b, double* res);
PS3D_API int ps3d_server_cancel(ps3d_server* s, long long ticket);
/* Shared launches for same-size requests: up to max_batch queued
 * optimal-balance requests whose grid, physics and balance parameters are
 * identical are admitted together and run as instances of one batched
 * context (every kernel launch advances all of them; each keeps its own
 * norm, iteration count and result, bit for bit what it gets alone with the
 * same kernel shapes), as long as their grid points together stay within
 * max_points (0: 2^22; larger grids already fill the GPU alone and run
 * side by side on their own streams instead).  Their footprint is the sum
 * of theirs.  max_batch 1 (the default) runs every request on its own
 * context.  Requests with biharmonic friction always run alone.           */
PS3D_API int ps3d_server_set_batching(ps3d_server* s, int max_batch, long long max_points);
/* stats[6] = {active, queued, bytes in use, peak bytes, peak active, budget} */
PS3D_API int ps3d_server_stats(ps3d_server* s, double* stats);
PS3D_API long long ps3d_server_footprint(const ps3d_params* prm);
/* request contexts created, and taken from the idle pool (a pooled context
 * of k instances serves a group of up to k same-parameter requests)        */
PS3D_API int ps3d_server_context_stats(ps3d_server* s, long long* created, long long* reused);

#ifdef __cplusplus
}
#endif
#endif /* PS3D_GPU_H */
