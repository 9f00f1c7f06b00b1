// engine.h — internal interfaces between the host engine and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include "common.cuh"
#include "ps3d_gpu.h"

namespace ps3d {

// Launch with programmatic stream serialization (see pdl_trigger/pdl_wait):
// only for kernels that call pdl_wait before reading their inputs.  Off by
// default (ordinary full dependencies; griddepcontrol.wait then returns at
// once): measured on a B200 at 256x256x128, the programmatic overlap made
// the step 95 us slower in both precisions, eager or in CUDA graphs.
// PS3D_PDL=1 turns it on.
bool pdl_enabled();
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<A&&>(args)...);
}

// Arguments of one time step for one grid (K1 and the generic-path kernels).
// Tendency slots are untyped: FP64 in the plain path, FP32 in the mixed path.
struct StepArgs {
    int nx, ny, nz;
    int rigid, nonlinear;
    double rdx, rdy, rdz;          // 1/dx, 1/dy, 1/dz
    double dt, dtw;                // dt and dt/dsqr
    double Ro, dsqr, N0sq, f0;
    double Ah, Av, Kh, Kv;
    int harm_uvw, harm_b;          // (Ah>0 .or. Av>0), (Kh>0 .or. Kv>0)
    double ab0, ab1, ab2;          // AB weights of slots tau, taum1, taum2
    int do_ab;                     // 0: stop after friction (generic path)
    const double *u, *v, *w, *b;   // start-of-step state
    const double *ub, *bb;         // background flow (NULL: none)
    double *uo, *vo, *wo, *bo;     // new state
    void* t0[4];                   // tendencies of time level tau (du,dv,dw,db)
    const void* t1[4];             // taum1
    const void* t2[4];             // taum2
    int wm_on;                     // wavemaker active
    double wm_c, wm_s;             // cos(omega t), sin(omega t)
    const double* wr[4];           // wavemaker real parts (NULL = 0)
    const double* wi[4];           // wavemaker imaginary parts
    int batch;                     // instances of the same grid stepped together (>= 1)
    long sN;                       // element stride between instances (fields and tendency slots)
    int kchunk;                    // z levels per block (autotuned)
    // pending pressure correction of the previous step (NULL: state is final):
    // the state arrays hold u'' and the true velocity is u'' - dtp*grad(pc)
    const double* pc;
    double dtp, dtwp;
    // level window of a z-slab (0: the whole local grid): levels
    // kbeg .. kbeg+kcount-1 are stepped; the rigid-lid masks see the global
    // level k + kofs of a grid of nzg levels
    int kbeg, kcount, kofs, nzg;
    // 0.5/dx, 0.5/dy, 0.5/dz, 0.25/dx, 0.25/dy, 0.25/dz, 0.25 f0, 0.5 N0^2 (set by launch_step)
    double hdx, hdy, hdz, qdx, qdy, qdz, qf0, hN0sq;
};

// One step-kernel launch over the grids of several groups (an ensemble's
// members of uneven sizes).  The table is a kernel parameter (sizeof ~11 KB,
// below the 32 KB parameter limit of CUDA 12.1+).
constexpr int kMaxStepGroups = 16;
struct StepGroups {
    StepArgs a[kMaxStepGroups];                    // each group's arguments (launcher-derived fields set)
    int blk0[kMaxStepGroups + 1];                  // first block of each group in the launch
    int gx[kMaxStepGroups], gy[kMaxStepGroups];    // column tiles along x and y of each group's grid
    int n;
};

// Plane-FFT kernels (divergence + forward 2D FFT, inverse 2D FFT) for one grid.
struct PlaneArgs {
    int nx, ny, nz, nxh;
    int C;                         // cluster size (CTAs per z-plane)
    int rows_per_cta, cols_per_cta, row_chunk, ldc, ldr;
    // forward source: mode 0 = divergence of (u,v,w)/dt, mode 1 = real field
    // src, mode 2 = divergence of (u,v,w) - dtp grad(pc), the correction of a
    // pending pressure pc applied on the fly
    int mode;
    const double *u, *v, *w, *src;
    const double* pc;
    double dtp, dtwp;
    int rigid;
    double rdx, rdy, rdz, rdt;
    double scale;                  // dx*dy (forward) or 1/(Lx*Ly[*Lz]) (inverse)
    void* spec;                    // complex spectral array [k][ky][kx]
    double* out;                   // inverse: real output field
    double beta;                   // inverse: out = beta*out + result (0: overwrite)
    FFTPlan px;                    // length nx/2
    FFTPlan py;                    // length ny
    const double2* twx;            // exp(-2 pi i t/nx), t = 0..nx/2
    int batch;                     // instances (>= 1): grid.y = nz*batch
    long sN, sM;                   // instance strides: real fields, spectral elements
    int impl;                      // 0: one cluster per plane (DSMEM), 1: rows pass + y-lines pass,
                                   // 2: as 1 with the forward rows pass pipelined by bulk copies
    int tj;                        // impl 1: rows per CTA of the rows passes
    int ly;                        // impl 1: lines per CTA of the y-lines passes
    FastDiv fd_n2, fd_ny, fd_tj;   // set by the launchers
    unsigned* err;                 // implementation 2: set to 1 when a bounded wait ran out
    // level window of a z-slab (0: the whole local grid; implementation 1
    // only): real-field levels kbeg .. kbeg+kcount-1 map to spectral levels
    // 0 .. kcount-1; the rigid-lid masks see the global level k + kofs of nzg
    int kbeg, kcount, kofs, nzg;
    int l2hint;                    // L2 eviction priorities on (set by the launchers; PS3D_L2HINT=0: off)
    // implementation 1 with the register rows passes only: the rows passes
    // apply the first radix-2 stage of the y transform and the spectra are
    // [k][kx][half][ny/2] (even ky, then odd); the y-lines passes and the
    // vertical solve are then one kernel, k_colsolve (launch_colsolve)
    int ysplit;
    FFTPlan pyh;                   // ysplit: the half-length y plan (length ny/2)
    int zrev;                      // the rows passes walk the planes top down (set by the launchers)
};
// spectral layout of a plane configuration: 0 [k][ky][kx], 1 [k][kx][ky]
inline int spectral_layout(const PlaneArgs& a) { return a.impl != 0; }

struct ColumnArgs {
    int nx, ny, nz, nxh;
    void* spec;                    // complex [k][ky][kx]
    const double* hkx;             // hat_ksqr(kx(i),dx)
    const double* hky;             // hat_ksqr(ky(j),dy)
    const double* hkz;             // hat_ksqr(kz(k),dz)/dsqr  (periodic)
    double fxa;                    // 1/dz^2/dsqr              (rigid lid)
    double dz2dsqr;                // dz**2*dsqr               (rigid lid, (0,0) column)
    double scale;                  // periodic forward z scale (dz)
    FFTPlan pz;                    // length nz (periodic)
    int op;                        // periodic: 0 solve, 1 forward only, 2 inverse only
    int batch;                     // instances (>= 1), spectral stride sM elements
    long sM;
    int layout;                    // spectral layout: 0 [k][ky][kx], 1 [k][kx][ky]
    // column slab (ncl 0: all nxh*ny columns): the array holds ncl columns per
    // level, global columns col0 .. col0+ncl-1 (one instance)
    long col0, ncl;
    FastDiv fd_ncols, fd_ny, fd_nxh;   // set by the launchers
    int l2hint;                        // L2 eviction priorities on (set by the launchers)
    unsigned* err;                     // set to 1 when a bounded wait ran out (NULL: not reported)
};
// the L2 eviction priorities the launchers set: 1 (default) spectra kept in
// L2 across the passes of a solve, 0 off (PS3D_L2HINT=0), 2 also the real
// fields evict_first (PS3D_L2HINT=2)
int l2hint_mode();

cudaError_t launch_step(const StepArgs& a, bool fp32_tendencies, cudaStream_t s);
cudaError_t step_setup();   // opts the step kernels in to their dynamic shared memory
// which fused step kernel a launch of `a` runs (friction, wavemaker,
// background-flow bits); grids of one grouped launch must agree
int step_flavour(const StepArgs& a);
// resident blocks per SM of the step kernel launch_step(a) would run
int step_resident(const StepArgs& a, bool fp32_tendencies);
// one launch of the step kernel over n <= kMaxStepGroups grids, each as
// launch_step(a[g], fp32_tendencies) would step it
cudaError_t launch_step_groups(const StepArgs* a, int n, bool fp32_tendencies, cudaStream_t s);
cudaError_t launch_biharmonic_h(const double* cur, const double* old, double* out, int nx, int ny, int nz,
                                double Hmix, double rdx, double rdy, double dt, cudaStream_t s);
cudaError_t launch_biharmonic_v(const double* cur, const double* old, double* out, int nx, int ny, int nz,
                                int rigid, double Vmix, double rdz, double dt, cudaStream_t s);
cudaError_t launch_forcing_background(const StepArgs& a, cudaStream_t s);
cudaError_t launch_wavemaker_ab(const StepArgs& a, int do_wm, cudaStream_t s);
cudaError_t launch_correct(double* u, double* v, double* w, const double* p, int nx, int ny, int nz, int rigid,
                           double dt, double dtw, double rdx, double rdy, double rdz, cudaStream_t s,
                           int batch = 1, int kbeg = 0, int kcount = 0, int kofs = 0, int nzg = 0);

// poisson.cu
size_t plane_fwd_smem(const PlaneArgs& a, bool fp32);
size_t plane_inv_smem(const PlaneArgs& a, bool fp32);
size_t plane_smem(const PlaneArgs& a, bool fp32);   // largest dynamic shared memory of the configuration
// ny with a register-resident y transform (k_ylines_reg): the y-lines pass
// then has no lines-per-CTA parameter
bool ylines_in_registers(int ny);
// grid with register-resident rows passes (k_rows_fwd_reg / k_rows_inv_reg):
// the rows pass then has no rows-per-CTA parameter
bool rows_in_registers(int nx, int ny);
cudaError_t plane_setup(bool fp32);
// default one-cluster-per-plane shape for element size es (false: no shape
// fits the shared memory of a block)
bool choose_plane_config(int nx, int ny, size_t es, PlaneArgs& a);
cudaError_t launch_plane_fwd(const PlaneArgs& a, bool fp32, cudaStream_t s);
cudaError_t launch_plane_inv(const PlaneArgs& a, bool fp32, cudaStream_t s);
int plane_max_clusters(const PlaneArgs& a, bool fp32, bool fwd);
// rigid-lid vertical solve; cudaErrorInvalidValue when nz is too tall for
// the shared memory of a block (thomas_threads(nz) == 0)
cudaError_t launch_thomas(const ColumnArgs& a, bool fp32, cudaStream_t s);
int thomas_threads(int nz);
// the y transforms and the rigid-lid vertical solve on the y-split layout
// (FP32 spectra); p: the forward plane arguments (scale, half-length plan)
cudaError_t launch_colsolve(const PlaneArgs& p, const ColumnArgs& c, cudaStream_t s);
bool colsolve_fits(int nz, int ny);
bool colsolve2_fits(int nz, int ny);   // the two-CTA cluster form (half the levels per CTA)
// periodic z solve; zsolve_fits(nz, fp32) false: too tall for a block's shared memory
cudaError_t launch_zsolve(const ColumnArgs& a, bool fp32, cudaStream_t s);
bool zsolve_fits(int nz, bool fp32);

// modes.cu: eigen tables for one grid and the projections
struct EigenAxes {
    // per-axis tables, host-computed with libm (my_fft.f90:87-156, eigenvectors.f90:224-268)
    const double* kx;  const double* ky;  const double* kz;
    const double* hkx; const double* hky; const double* hkz;   // hat_ksqr
    const double* ex;  const double* ey;  const double* ez;    // hat_epm
    const double2* px; const double2* py; const double2* pz;   // exp(+i k d)
    const double* sz;  const double* cz;                       // sin/cos(kz/2*dz) (rigid lid)
};
struct ProjArgs {
    int nxh, ny, nz, rigid;
    int layout;                    // spectral layout: 0 [k][ky][kx], 1 [k][kx][ky]
    double dx, dy, dz, f0, N0, dsqr;
    EigenAxes ax;
    double2 *US, *VS, *WS, *BS;
    double2* g0base;
    int mode;                      // PS3D_PROJ_*
};
cudaError_t launch_project(const ProjArgs& a, cudaStream_t s);
// A: nz x nz, read as A[ko + nz*ki] (the forward transform passes the
// transposed mode matrix); cudaErrorInvalidValue when !vert_mode_fits(nz)
cudaError_t launch_vert_mode(const double2* in, double2* out, const double* A, int nz, long ncol, double scale,
                             cudaStream_t s);
bool vert_mode_fits(int nz);
cudaError_t modes_setup();   // per device, before the first launch_vert_mode
// The rigid-lid vertical-mode transforms by FFT of length 2 nz (modes.cu):
// kind 0 = phi (DCT-II / DCT-III), 1 = psi (DST-I), 2 = psib (DST-II / DST-III)
struct VertDttArgs {
    const double2* in;
    double2* out;
    int nz;
    long ncol;          // columns: levels are ncol apart
    double scale;       // forward: dz; backward: 1
    FFTPlan plan;       // length 2 nz, radices <= 8 (radix-8-first plan)
    FFTPlan plan1;      // length nz, radices <= 8 (phi and psib for even nz; n = 0: none)
    const double2* tw;  // e^{i pi j / 2 nz}, j = 0 .. nz-1
    double c0, c1;      // sqrt(1/Lz) (phi's mode 0), sqrt(2/Lz) (every other mode)
    int cols;           // columns per block (set by the launcher)
};
bool fft_length_ok(int n);
bool vert_dtt_fits(int nz);
cudaError_t launch_vert_dtt(const VertDttArgs& a, int kind, bool fwd, cudaStream_t s);

// layout.cu: host halo layout <-> device interior layout (h_dev holds the
// whole host array, (nx+4)*(ny+4)*(nz+4) doubles)
cudaError_t launch_from_halo(const double* h_dev, void* dst, int nx, int ny, int nz, bool f32, cudaStream_t s);
cudaError_t launch_to_halo(const void* src, double* h_dev, int nx, int ny, int nz, bool pghost, bool f32,
                           cudaStream_t s);

// reduce.cu
struct DiagOut { double ke, pe, umax, wmax; unsigned flags; };
cudaError_t launch_diagnose(const double* u, const double* v, const double* w, const double* b, const double* p,
                            int nx, int ny, int nz, double dsqr, double N0, double dz,
                            double* partials, int nblk, DiagOut* out_dev, cudaStream_t s,
                            int kofs = 0);
cudaError_t launch_norm(const double* const* x, const double* const* y, long n, double dsqr, double N0sq,
                        double* partials, int nblk, double* out_dev, cudaStream_t s);
cudaError_t launch_axpby(double* y, const double* x, long n, double a, double b, cudaStream_t s);

}  // namespace ps3d
