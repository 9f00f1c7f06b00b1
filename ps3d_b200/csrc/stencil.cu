// stencil.cu — tendency, friction, forcing, Adams-Bashforth and pressure
// gradient kernels of the ps3D time step on sm_100a.
//
// K1 (k_step) fuses, per grid point, what the reference does in ~40 full
// passes over memory:
//   buoyancy_advection_2nd            advection.f90:2-48
//   N^2 term                          integrate.f90:21-23
//   momentum_advection_2nd            advection.f90:53-184
//   Coriolis and buoyancy force       integrate.f90:37-54
//   harmonic friction (in place)      mixing.f90:225-274, integrate.f90:59-66
//   set_forcing (wavemaker and
//     background-flow advection)      config.f90:224-237, lee_wave1.f90:232-332
//   Adams-Bashforth 2/3               integrate.f90:87-102
// The block owns a 32 x BY column tile and marches up in z; the three planes
// k-1, k, k+1 of u, v, w, b (and of U_back, B_back when present) sit in a
// shared-memory ring with a one-point halo.  Each thread's tile elements and
// their east/north neighbours are located once per block, so a plane load is
// one offset add per field.  Face fluxes are recomputed per
// point instead of being stored, so the kernel reads each state word once
// from HBM and writes tendencies and the new state once.
#include <cstdlib>
#include "engine.h"

namespace ps3d {

constexpr int kTX = 32;

// The ring of state planes, and this level's Adams-Bashforth history of the
// block's points (t1, t2), staged through shared memory so that its loads
// go out with the next plane's before the barrier without holding
// registers through the tendency arithmetic.
template <typename TT, int BY, int NF>
struct StepSmem {
    double pl[NF][3][(BY + 2) * (kTX + 2)];
    TT hu[2][kTX * BY], hv[2][kTX * BY], hb[2][kTX * BY];
    double hw[2][kTX * BY];
};

// The tendency, friction, forcing and Adams-Bashforth update of the point
// (i, j, k) of instance `ioff`: F(f, di, dj, dk) reads field f (0 u, 1 v,
// 2 w, 3 b, 4 U_back, 5 B_back) of the corrected state at the offsets,
// Hh(f, l) the point's stored tendency of field f at history level l
// (0: taum1, 1: taum2).  Shared by the step kernels, which differ only in
// how they stage the state.
template <typename TT, bool HARM, bool WM, bool BG, class FV, class HV>
__device__ __forceinline__ void step_point(const StepArgs& a, const FV& F, const HV& Hh, int i, int j, int k,
                                           long ioff, bool h1, bool h2) {
    using TW = double;   // stored w tendencies stay FP64 in both paths
    const int nx = a.nx, ny = a.ny;
    const long plane = (long)nx * ny;
    const int kofs = a.kofs, nzg = a.nzg ? a.nzg : a.nz;
    const double Ro = a.Ro, rdx = a.rdx, rdy = a.rdy, rdz = a.rdz;
    const bool rigid = a.rigid;
#define U(di, dj, dk) F(0, di, dj, dk)
#define V(di, dj, dk) F(1, di, dj, dk)
#define W(di, dj, dk) F(2, di, dj, dk)
#define B(di, dj, dk) F(3, di, dj, dk)
#define UB(di, dj, dk) F(4, di, dj, dk)
#define BB(di, dj, dk) F(5, di, dj, dk)
    const int kg = k + kofs;                     // global level
    const bool top = rigid && (kg == nzg - 1);   // flux_top(nz) = 0
    const bool bot = rigid && (kg == 0);         // flux_top(0)  = 0
    const long g0 = (long)k * plane + (long)j * nx + i;   // point within the instance
    const long g = g0 + ioff;                              // point within the batch
    double db_, du_, dv_, dw_;
    // ---- buoyancy advection + N^2 (advection.f90:12-47, integrate.f90:21-23)
    // The reference's 0.5 and 0.25 flux factors are powers of two: they
    // are carried in the per-axis factors a.hd* = 0.5/d*, a.qd* = 0.25/d*
    // (and 0.25 f0, 0.5 N0^2, set by the launcher), a multiply saved per
    // flux.  Scaling by a power of two rounds exactly; the results move
    // at round-off level only where the compiler now contracts a flux
    // product into the difference that follows (FMA).
    if (a.nonlinear) {
        const double fe = (B(0, 0, 0) + B(1, 0, 0)) * U(0, 0, 0);
        const double fem = (B(-1, 0, 0) + B(0, 0, 0)) * U(-1, 0, 0);
        const double fn = (B(0, 0, 0) + B(0, 1, 0)) * V(0, 0, 0);
        const double fnm = (B(0, -1, 0) + B(0, 0, 0)) * V(0, -1, 0);
        const double ft = top ? 0.0 : (B(0, 0, 0) + B(0, 0, 1)) * W(0, 0, 0);
        const double ftm = bot ? 0.0 : (B(0, 0, -1) + B(0, 0, 0)) * W(0, 0, -1);
        db_ = -Ro * ((fe - fem) * a.hdx + (fn - fnm) * a.hdy + (ft - ftm) * a.hdz);
        // ---- zonal momentum (advection.f90:65-100)
        {
            const double e = (U(0, 0, 0) + U(1, 0, 0)) * (U(1, 0, 0) + U(0, 0, 0));
            const double em = (U(-1, 0, 0) + U(0, 0, 0)) * (U(0, 0, 0) + U(-1, 0, 0));
            const double n = (U(0, 0, 0) + U(0, 1, 0)) * (V(1, 0, 0) + V(0, 0, 0));
            const double nm = (U(0, -1, 0) + U(0, 0, 0)) * (V(1, -1, 0) + V(0, -1, 0));
            const double t = top ? 0.0 : (U(0, 0, 1) + U(0, 0, 0)) * (W(0, 0, 0) + W(1, 0, 0));
            const double tm = bot ? 0.0 : (U(0, 0, 0) + U(0, 0, -1)) * (W(0, 0, -1) + W(1, 0, -1));
            du_ = -Ro * ((e - em) * a.qdx + (n - nm) * a.qdy + (t - tm) * a.qdz);
        }
        // ---- meridional momentum (advection.f90:104-140)
        {
            const double e = (V(0, 0, 0) + V(1, 0, 0)) * (U(0, 1, 0) + U(0, 0, 0));
            const double em = (V(-1, 0, 0) + V(0, 0, 0)) * (U(-1, 1, 0) + U(-1, 0, 0));
            const double n = (V(0, 0, 0) + V(0, 1, 0)) * (V(0, 1, 0) + V(0, 0, 0));
            const double nm = (V(0, -1, 0) + V(0, 0, 0)) * (V(0, 0, 0) + V(0, -1, 0));
            const double t = top ? 0.0 : (V(0, 0, 1) + V(0, 0, 0)) * (W(0, 0, 0) + W(0, 1, 0));
            const double tm = bot ? 0.0 : (V(0, 0, 0) + V(0, 0, -1)) * (W(0, 0, -1) + W(0, 1, -1));
            dv_ = -Ro * ((e - em) * a.qdx + (n - nm) * a.qdy + (t - tm) * a.qdz);
        }
        // ---- vertical momentum (advection.f90:145-181); rigid lid zeroes
        //      flux_top(nz-1:nz+2) for w (:167-170)
        {
            const bool wtop = rigid && (kg >= nzg - 2);
            const bool wbot = rigid && (kg == 0 || kg >= nzg - 1);
            const double e = (W(0, 0, 0) + W(1, 0, 0)) * (U(0, 0, 0) + U(0, 0, 1));
            const double em = (W(-1, 0, 0) + W(0, 0, 0)) * (U(-1, 0, 0) + U(-1, 0, 1));
            const double n = (W(0, 0, 0) + W(0, 1, 0)) * (V(0, 0, 0) + V(0, 0, 1));
            const double nm = (W(0, -1, 0) + W(0, 0, 0)) * (V(0, -1, 0) + V(0, -1, 1));
            const double t = wtop ? 0.0 : (W(0, 0, 1) + W(0, 0, 0)) * (W(0, 0, 0) + W(0, 0, 1));
            const double tm = wbot ? 0.0 : (W(0, 0, 0) + W(0, 0, -1)) * (W(0, 0, -1) + W(0, 0, 0));
            dw_ = -a.dsqr * Ro * ((e - em) * a.qdx + (n - nm) * a.qdy + (t - tm) * a.qdz);
        }
    } else {
        db_ = du_ = dv_ = dw_ = 0.0;
    }
    db_ = db_ - (W(0, 0, 0) + W(0, 0, -1)) * a.hN0sq;
    // ---- Coriolis, buoyancy force, rigid-lid mask (integrate.f90:37-54)
    du_ = du_ + (V(0, 0, 0) + V(0, -1, 0) + V(1, 0, 0) + V(1, -1, 0)) * a.qf0;
    dv_ = dv_ - (U(-1, 0, 0) + U(0, 0, 0) + U(-1, 1, 0) + U(0, 1, 0)) * a.qf0;
    dw_ = dw_ + 0.5 * (B(0, 0, 0) + B(0, 0, 1));
    if (top) dw_ = 0.0;
    // ---- friction, in place before AB (integrate.f90:59-66)
    double u1 = U(0, 0, 0), v1 = V(0, 0, 0), w1 = W(0, 0, 0), b1 = B(0, 0, 0);
    if constexpr (HARM) {
        const double dt = a.dt;
#define HARMONIC(F, Hm, Vm, out)                                                                   \
    {                                                                                            \
const double e = Hm * (F(1, 0, 0) - F(0, 0, 0)) * rdx;                                   \
const double em = Hm * (F(0, 0, 0) - F(-1, 0, 0)) * rdx;                                 \
const double n = Hm * (F(0, 1, 0) - F(0, 0, 0)) * rdy;                                   \
const double nm = Hm * (F(0, 0, 0) - F(0, -1, 0)) * rdy;                                 \
const double t = top ? 0.0 : Vm * (F(0, 0, 1) - F(0, 0, 0)) * rdz;                       \
const double tm = bot ? 0.0 : Vm * (F(0, 0, 0) - F(0, 0, -1)) * rdz;                     \
out = F(0, 0, 0) + dt * ((e - em) * rdx + (n - nm) * rdy + (t - tm) * rdz);              \
    }
        if (a.harm_uvw) {
            HARMONIC(U, a.Ah, a.Av, u1)
            HARMONIC(V, a.Ah, a.Av, v1)
            HARMONIC(W, a.Ah, a.Av, w1)
            if (top) w1 = 0.0;
        }
        if (a.harm_b) HARMONIC(B, a.Kh, a.Kv, b1)
#undef HARMONIC
    }
    // ---- set_forcing: background-flow advection (lee_wave1.f90:245-312)
    if constexpr (BG) {
        {
            const double e = 2 * 0.25 * (UB(0, 0, 0) + UB(1, 0, 0)) * (U(1, 0, 0) + U(0, 0, 0));
            const double em = 2 * 0.25 * (UB(-1, 0, 0) + UB(0, 0, 0)) * (U(0, 0, 0) + U(-1, 0, 0));
            const double n = 0.25 * (UB(0, 0, 0) + UB(0, 1, 0)) * (V(1, 0, 0) + V(0, 0, 0));
            const double nm = 0.25 * (UB(0, -1, 0) + UB(0, 0, 0)) * (V(1, -1, 0) + V(0, -1, 0));
            const double t = top ? 0.0 : 0.25 * (UB(0, 0, 1) + UB(0, 0, 0)) * (W(0, 0, 0) + W(1, 0, 0));
            const double tm = bot ? 0.0 : 0.25 * (UB(0, 0, 0) + UB(0, 0, -1)) * (W(0, 0, -1) + W(1, 0, -1));
            du_ = du_ - Ro * ((e - em) * rdx + (n - nm) * rdy + (t - tm) * rdz);
        }
        {
            const double e = 0.25 * (V(0, 0, 0) + V(1, 0, 0)) * (UB(0, 1, 0) + UB(0, 0, 0));
            const double em = 0.25 * (V(-1, 0, 0) + V(0, 0, 0)) * (UB(-1, 1, 0) + UB(-1, 0, 0));
            dv_ = dv_ - Ro * (e - em) * rdx;
        }
        {
            const double e = 0.25 * (W(0, 0, 0) + W(1, 0, 0)) * (UB(0, 0, 0) + UB(0, 0, 1));
            const double em = 0.25 * (W(-1, 0, 0) + W(0, 0, 0)) * (UB(-1, 0, 0) + UB(-1, 0, 1));
            dw_ = dw_ - a.dsqr * Ro * (e - em) * rdx;
        }
        {
            const double e = 0.5 * (B(0, 0, 0) + B(1, 0, 0)) * UB(0, 0, 0) + 0.5 * (BB(0, 0, 0) + BB(1, 0, 0)) * U(0, 0, 0);
            const double em = 0.5 * (B(-1, 0, 0) + B(0, 0, 0)) * UB(-1, 0, 0) + 0.5 * (BB(-1, 0, 0) + BB(0, 0, 0)) * U(-1, 0, 0);
            const double n = 0.5 * (BB(0, 0, 0) + BB(0, 1, 0)) * V(0, 0, 0);
            const double nm = 0.5 * (BB(0, -1, 0) + BB(0, 0, 0)) * V(0, -1, 0);
            const double t = top ? 0.0 : 0.5 * (BB(0, 0, 0) + BB(0, 0, 1)) * W(0, 0, 0);
            const double tm = bot ? 0.0 : 0.5 * (BB(0, 0, -1) + BB(0, 0, 0)) * W(0, 0, -1);
            db_ = db_ - Ro * ((e - em) * rdx + (n - nm) * rdy + (t - tm) * rdz);
        }
    }
#undef U
#undef V
#undef W
#undef B
#undef UB
#undef BB
    // ---- set_forcing: wavemaker (config.f90:224-237)
    if constexpr (WM) {
        const double dt = a.dt, c = a.wm_c, s = a.wm_s;
        if (a.wr[0] || a.wi[0]) u1 = u1 + dt * (c * (a.wr[0] ? a.wr[0][g0] : 0.0) + s * (a.wi[0] ? a.wi[0][g0] : 0.0));
        if (a.wr[1] || a.wi[1]) v1 = v1 + dt * (c * (a.wr[1] ? a.wr[1][g0] : 0.0) + s * (a.wi[1] ? a.wi[1][g0] : 0.0));
        if (a.wr[2] || a.wi[2]) w1 = w1 + dt * (c * (a.wr[2] ? a.wr[2][g0] : 0.0) + s * (a.wi[2] ? a.wi[2][g0] : 0.0));
        if (a.wr[3] || a.wi[3]) b1 = b1 + dt * (c * (a.wr[3] ? a.wr[3][g0] : 0.0) + s * (a.wi[3] ? a.wi[3][g0] : 0.0));
    }
    // ---- store tendency of time level tau
    ((TT*)a.t0[0])[g] = (TT)du_;
    ((TT*)a.t0[1])[g] = (TT)dv_;
    ((TW*)a.t0[2])[g] = (TW)dw_;
    ((TT*)a.t0[3])[g] = (TT)db_;
    // ---- Adams-Bashforth (integrate.f90:87-102)
    if (a.do_ab) {
        const double dt = a.dt, dtw = a.dtw;
        const double c0 = a.ab0, c1 = a.ab1, c2 = a.ab2;
        // the current tendency enters at full precision; only the
        // stored history (FP32 in the mixed path) is rounded
        double tu = c0 * du_, tv = c0 * dv_, tw = c0 * dw_, tb = c0 * db_;
        if (h1) {
            tu = tu + c1 * Hh(0, 0); tv = tv + c1 * Hh(1, 0);
            tw = tw + c1 * Hh(2, 0); tb = tb + c1 * Hh(3, 0);
        }
        if (h2) {
            tu = tu + c2 * Hh(0, 1); tv = tv + c2 * Hh(1, 1);
            tw = tw + c2 * Hh(2, 1); tb = tb + c2 * Hh(3, 1);
        }
        u1 = u1 + dt * tu; v1 = v1 + dt * tv; w1 = w1 + dtw * tw; b1 = b1 + dt * tb;
    }
    a.uo[g] = u1; a.vo[g] = v1; a.wo[g] = w1; a.bo[g] = b1;
}

// read field f at offsets (di, dj) in ring slot s
#define SM(fi, s, dj, di) sm.pl[fi][s][(ty + 1 + (dj)) * (kTX + 2) + (tx + 1 + (di))]

// One block's column tile (bx, by) and z chunk / instance bz of the grid
// described by `a`.
template <typename TT, int BY, bool HARM, bool WM, bool BG>
__device__ __forceinline__ void step_tile(const StepArgs& a, int kchunk, int bx, int by, int bz) {
    using TW = double;   // stored w tendencies stay FP64 in both paths
    constexpr int NF = BG ? 6 : 4;
    extern __shared__ __align__(16) unsigned char step_smem_raw[];
    StepSmem<TT, BY, NF>& sm = *reinterpret_cast<StepSmem<TT, BY, NF>*>(step_smem_raw);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int i0 = bx * kTX, j0 = by * BY;
    const int kcnt = a.kcount ? a.kcount : nz;           // levels stepped (a z-slab's interior)
    const int kofs = a.kofs, nzg = a.nzg ? a.nzg : nz;   // global level k + kofs of nzg (rigid-lid masks)
    const int nzc = (kcnt + kchunk - 1) / kchunk;
    const int inst = bz / nzc;
    const int kb = a.kbeg + (bz - inst * nzc) * kchunk;
    const int ke = min(a.kbeg + kcnt, kb + kchunk);
    const long ioff = (long)inst * a.sN;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = (i < nx) && (j < ny);
    const long plane = (long)nx * ny;
    const double* src[6] = {a.u + ioff, a.v + ioff, a.w + ioff, a.b + ioff, a.ub, a.bb};
    const int tid = ty * kTX + tx;
    constexpr int TP = (kTX + 2) * (BY + 2);

    const double* pc = a.pc ? a.pc + ioff : nullptr;
    // per-thread tile elements: plane offsets of the point and of its east and
    // north neighbours, computed once (full modulo: tiles may be wider than the grid)
    constexpr int NT = kTX * BY;
    constexpr int EPT = (TP + NT - 1) / NT;
    int eo[EPT], eoE[EPT], eoN[EPT];
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
        const int t = tid + e * NT;
        const int ti = t % (kTX + 2), tj = t / (kTX + 2);
        const int gi = ((i0 - 1 + ti) % nx + nx) % nx, gj = ((j0 - 1 + tj) % ny + ny) % ny;
        eo[e] = gj * nx + gi;
        eoE[e] = gj * nx + wrap(gi + 1, nx);
        eoN[e] = wrap(gj + 1, ny) * nx + gi;
    }
    auto load_plane = [&](int kk, int slot) {
        const int kw = wrap(kk, nz);
        const long po = (long)kw * plane, pu = (long)wrap(kw + 1, nz) * plane;
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int t = tid + e * NT;
            if (t < TP) {
                double v[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f] = __ldg(src[f] + po + eo[e]);
                if (pc) {
                    // the previous step's pressure-gradient correction
                    // (pressure_solver.f90:98-110), applied where the state is read
                    const double p0 = __ldg(pc + po + eo[e]);
                    const double pe = __ldg(pc + po + eoE[e]);
                    const double pn = __ldg(pc + po + eoN[e]);
                    const double pt = __ldg(pc + pu + eo[e]);
                    v[0] = v[0] - a.dtp * (pe - p0) * a.rdx;
                    v[1] = v[1] - a.dtp * (pn - p0) * a.rdy;
                    v[2] = (a.rigid && wrap(kw + kofs, nzg) == nzg - 1) ? 0.0 : v[2] - a.dtwp * (pt - p0) * a.rdz;
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) sm.pl[f][slot][t] = v[f];
            }
        }
    };

    load_plane(kb - 1, (kb + 2) % 3);
    load_plane(kb, kb % 3);
    const bool h1 = a.do_ab && a.ab1 != 0.0, h2 = a.do_ab && a.ab2 != 0.0;
    for (int k = kb; k < ke; ++k) {
        // history loads first, so they are in flight with the plane's
        TT hu1 = 0, hv1 = 0, hb1 = 0, hu2 = 0, hv2 = 0, hb2 = 0;
        double hw1 = 0.0, hw2 = 0.0;
        const long gh = (long)k * plane + (long)j * nx + i + ioff;
        if (active && h1) {
            const TT* const* h = (const TT* const*)a.t1;
            hu1 = h[0][gh]; hv1 = h[1][gh]; hw1 = ((const TW*)a.t1[2])[gh]; hb1 = h[3][gh];
        }
        if (active && h2) {
            const TT* const* h = (const TT* const*)a.t2;
            hu2 = h[0][gh]; hv2 = h[1][gh]; hw2 = ((const TW*)a.t2[2])[gh]; hb2 = h[3][gh];
        }
        load_plane(k + 1, (k + 1) % 3);
        sm.hu[0][tid] = hu1; sm.hv[0][tid] = hv1; sm.hw[0][tid] = hw1; sm.hb[0][tid] = hb1;
        sm.hu[1][tid] = hu2; sm.hv[1][tid] = hv2; sm.hw[1][tid] = hw2; sm.hb[1][tid] = hb2;
        __syncthreads();
        if (active) {
            const int sm1 = (k + 2) % 3, s0 = k % 3, sp1 = (k + 1) % 3;
            auto F = [&](int f, int di, int dj, int dk) -> double {
                return SM(f, dk < 0 ? sm1 : (dk > 0 ? sp1 : s0), dj, di);
            };
            auto Hh = [&](int f, int l) -> double {
                return f == 0 ? (double)sm.hu[l][tid] : f == 1 ? (double)sm.hv[l][tid]
                     : f == 2 ? sm.hw[l][tid] : (double)sm.hb[l][tid];
            };
            step_point<TT, HARM, WM, BG>(a, F, Hh, i, j, k, ioff, h1, h2);
        }
        __syncthreads();
    }
}

template <typename TT, int BY, bool HARM, bool WM, bool BG>
__global__ void __launch_bounds__(kTX* BY) k_step(const StepArgs a, int kchunk) {
    pdl_trigger();
    pdl_wait();   // the state, p and history were written by the preceding kernels
    step_tile<TT, BY, HARM, WM, BG>(a, kchunk, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One launch over the grids of several groups (an ensemble's members of
// uneven sizes): block b belongs to the group g with blk0[g] <= b <
// blk0[g+1] and runs that group's tile as k_step would.  The table rides in
// the kernel's parameter space (captured by value into a CUDA graph).
template <typename TT, int BY, bool HARM, bool WM, bool BG>
__global__ void __launch_bounds__(kTX* BY, BG ? 2 : 4) k_step_groups(const __grid_constant__ StepGroups m) {
    pdl_trigger();
    pdl_wait();
    int g = 0;
    while (g + 1 < m.n && (int)blockIdx.x >= m.blk0[g + 1]) ++g;
    const int l = blockIdx.x - m.blk0[g];
    const int gx = m.gx[g], gy = m.gy[g];
    step_tile<TT, BY, HARM, WM, BG>(m.a[g], m.a[g].kchunk, l % gx, (l / gx) % gy, l / (gx * gy));
}

// ---------------------------------------------------------------------------
// Generic friction stages with the reference's stale-halo semantics: the
// biharmonic operators of mixing.f90:96-217 run after harmonic() without a
// halo exchange, so any neighbour outside the interior still holds the
// start-of-step value.  `cur` is the field after the previous stage, `old`
// the start-of-step field; out = cur + dt*op(.).
// ---------------------------------------------------------------------------
__global__ void k_biharmonic_h(const double* __restrict__ cur, const double* __restrict__ old,
                               double* __restrict__ out, int nx, int ny, int nz,
                               double Hmix, double rdx, double rdy, double dt) {
    const long N = (long)nx * ny * nz;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
        const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((long)nx * ny));
        const long pk = (long)k * nx * ny;
        auto P = [&](int di, int dj) -> double {
            const int ii = i + di, jj = j + dj;
            const bool in = ii >= 0 && ii < nx && jj >= 0 && jj < ny;
            const long gg = pk + (long)wrap(jj, ny) * nx + wrap(ii, nx);
            return in ? cur[gg] : old[gg];
        };
        auto del2 = [&](int di, int dj) -> double {
            const double fe = -Hmix * (P(di + 1, dj) - P(di, dj)) * rdx;
            const double fem = -Hmix * (P(di, dj) - P(di - 1, dj)) * rdx;
            const double fn = -Hmix * (P(di, dj + 1) - P(di, dj)) * rdy;
            const double fnm = -Hmix * (P(di, dj) - P(di, dj - 1)) * rdy;
            return (fe - fem) * rdx + (fn - fnm) * rdy;
        };
        const double d0 = del2(0, 0);
        const double fe = (del2(1, 0) - d0) * rdx, fem = (d0 - del2(-1, 0)) * rdx;
        const double fn = (del2(0, 1) - d0) * rdy, fnm = (d0 - del2(0, -1)) * rdy;
        out[g] = cur[g] + dt * ((fe - fem) * rdx + (fn - fnm) * rdy);
    }
}

__global__ void k_biharmonic_v(const double* __restrict__ cur, const double* __restrict__ old,
                               double* __restrict__ out, int nx, int ny, int nz, int rigid,
                               double Vmix, double rdz, double dt) {
    const long N = (long)nx * ny * nz;
    const long plane = (long)nx * ny;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
        const int k = (int)(g / plane);
        const long col = g - (long)k * plane;
        // 1-based level kr = k+1; flux_top(kr) lives between levels kr and kr+1
        auto P = [&](int kk) -> double {   // kk: 0-based level, may be outside
            const bool in = kk >= 0 && kk < nz;
            const long gg = (long)wrap(kk, nz) * plane + col;
            return in ? cur[gg] : old[gg];
        };
        auto ft1 = [&](int kr) -> double {  // first-stage flux at 1-based level kr
            if (rigid && (kr <= 0 || kr >= nz)) return 0.0;
            return -Vmix * (P(kr) - P(kr - 1)) * rdz;
        };
        auto del2 = [&](int kr) -> double { return (ft1(kr) - ft1(kr - 1)) * rdz; };
        auto ft2 = [&](int kr) -> double {
            if (rigid && (kr <= 0 || kr >= nz)) return 0.0;
            return (del2(kr + 1) - del2(kr)) * rdz;
        };
        const int kr = k + 1;
        out[g] = cur[g] + dt * ((ft2(kr) - ft2(kr - 1)) * rdz);
    }
}

// background-flow forcing on the friction-updated state (generic path).
// set_forcing runs after the in-place friction with no halo exchange, so a
// neighbour outside the interior still holds its start-of-step value: those
// reads go to the old fields (a.uo..bo hold the start-of-step state here,
// a.u..b the friction-updated one).
__global__ void k_forcing_background(StepArgs a) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long N = (long)nx * ny * nz, plane = (long)nx * ny;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
        const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / plane);
        auto at = [&](const double* f, int di, int dj, int dk) -> double {
            return f[(long)wrap(k + dk, nz) * plane + (long)wrap(j + dj, ny) * nx + wrap(i + di, nx)];
        };
        auto st = [&](int fld, int di, int dj, int dk) -> double {
            const bool in = i + di >= 0 && i + di < nx && j + dj >= 0 && j + dj < ny && k + dk >= 0 && k + dk < nz;
            const double* cur = fld == 0 ? a.u : fld == 1 ? a.v : fld == 2 ? a.w : a.b;
            const double* old = fld == 0 ? a.uo : fld == 1 ? a.vo : fld == 2 ? a.wo : a.bo;
            return at(in ? cur : old, di, dj, dk);
        };
        const double *ub = a.ub, *bb = a.bb;
        const bool top = a.rigid && k == nz - 1, bot = a.rigid && k == 0;
        const double Ro = a.Ro, rdx = a.rdx, rdy = a.rdy, rdz = a.rdz;
        double* const* T0 = (double* const*)a.t0;
        double du_ = T0[0][g], dv_ = T0[1][g], dw_ = T0[2][g], db_ = T0[3][g];
        {
            const double e = 2 * 0.25 * (at(ub, 0, 0, 0) + at(ub, 1, 0, 0)) * (st(0, 1, 0, 0) + st(0, 0, 0, 0));
            const double em = 2 * 0.25 * (at(ub, -1, 0, 0) + at(ub, 0, 0, 0)) * (st(0, 0, 0, 0) + st(0, -1, 0, 0));
            const double n = 0.25 * (at(ub, 0, 0, 0) + at(ub, 0, 1, 0)) * (st(1, 1, 0, 0) + st(1, 0, 0, 0));
            const double nm = 0.25 * (at(ub, 0, -1, 0) + at(ub, 0, 0, 0)) * (st(1, 1, -1, 0) + st(1, 0, -1, 0));
            const double t = top ? 0.0 : 0.25 * (at(ub, 0, 0, 1) + at(ub, 0, 0, 0)) * (st(2, 0, 0, 0) + st(2, 1, 0, 0));
            const double tm = bot ? 0.0 : 0.25 * (at(ub, 0, 0, 0) + at(ub, 0, 0, -1)) * (st(2, 0, 0, -1) + st(2, 1, 0, -1));
            du_ = du_ - Ro * ((e - em) * rdx + (n - nm) * rdy + (t - tm) * rdz);
        }
        {
            const double e = 0.25 * (st(1, 0, 0, 0) + st(1, 1, 0, 0)) * (at(ub, 0, 1, 0) + at(ub, 0, 0, 0));
            const double em = 0.25 * (st(1, -1, 0, 0) + st(1, 0, 0, 0)) * (at(ub, -1, 1, 0) + at(ub, -1, 0, 0));
            dv_ = dv_ - Ro * (e - em) * rdx;
        }
        {
            const double e = 0.25 * (st(2, 0, 0, 0) + st(2, 1, 0, 0)) * (at(ub, 0, 0, 0) + at(ub, 0, 0, 1));
            const double em = 0.25 * (st(2, -1, 0, 0) + st(2, 0, 0, 0)) * (at(ub, -1, 0, 0) + at(ub, -1, 0, 1));
            dw_ = dw_ - a.dsqr * Ro * (e - em) * rdx;
        }
        {
            const double e = 0.5 * (st(3, 0, 0, 0) + st(3, 1, 0, 0)) * at(ub, 0, 0, 0) + 0.5 * (at(bb, 0, 0, 0) + at(bb, 1, 0, 0)) * st(0, 0, 0, 0);
            const double em = 0.5 * (st(3, -1, 0, 0) + st(3, 0, 0, 0)) * at(ub, -1, 0, 0) + 0.5 * (at(bb, -1, 0, 0) + at(bb, 0, 0, 0)) * st(0, -1, 0, 0);
            const double n = 0.5 * (at(bb, 0, 0, 0) + at(bb, 0, 1, 0)) * st(1, 0, 0, 0);
            const double nm = 0.5 * (at(bb, 0, -1, 0) + at(bb, 0, 0, 0)) * st(1, 0, -1, 0);
            const double t = top ? 0.0 : 0.5 * (at(bb, 0, 0, 0) + at(bb, 0, 0, 1)) * st(2, 0, 0, 0);
            const double tm = bot ? 0.0 : 0.5 * (at(bb, 0, 0, -1) + at(bb, 0, 0, 0)) * st(2, 0, 0, -1);
            db_ = db_ - Ro * ((e - em) * rdx + (n - nm) * rdy + (t - tm) * rdz);
        }
        T0[0][g] = du_; T0[1][g] = dv_; T0[2][g] = dw_; T0[3][g] = db_;
    }
}

// wavemaker + Adams-Bashforth, pointwise, in place on the state (generic path)
__global__ void k_wavemaker_ab(StepArgs a, int do_wm) {
    const long N = (long)a.nx * a.ny * a.nz;
    double* fld[4] = {a.uo, a.vo, a.wo, a.bo};
    const double* const* t0 = (const double* const*)a.t0;
    const double* const* t1 = (const double* const*)a.t1;
    const double* const* t2 = (const double* const*)a.t2;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double x = fld[f][g];
            if (do_wm && (a.wr[f] || a.wi[f]))
                x = x + a.dt * (a.wm_c * (a.wr[f] ? a.wr[f][g] : 0.0) + a.wm_s * (a.wi[f] ? a.wi[f][g] : 0.0));
            double t = a.ab0 * t0[f][g];
            if (a.ab1 != 0.0) t = t + a.ab1 * t1[f][g];
            if (a.ab2 != 0.0) t = t + a.ab2 * t2[f][g];
            fld[f][g] = x + (f == 2 ? a.dtw : a.dt) * t;
        }
    }
}

// ---------------------------------------------------------------------------
// pressure gradient correction, pressure_solver.f90:98-110 (and the rigid-lid
// ghost levels :82-93, which make the w correction vanish at level nz)
// ---------------------------------------------------------------------------
// levels kbeg .. kbeg+kcnt-1 of each instance; the rigid lid is global level
// nzg-1 with global level k + kofs
__global__ void k_correct(double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                          const double* __restrict__ p, int nx, int ny, int nz, int rigid,
                          double dt, double dtw, double rdx, double rdy, double rdz, int batch,
                          int kbeg, int kcnt, int kofs, int nzg) {
    const long plane = (long)nx * ny, N = plane * nz, NW = plane * kcnt, NB = NW * batch;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < NB; q += (long)gridDim.x * blockDim.x) {
        const long inst = q / NW, r = q - inst * NW;
        const long g = inst * N + (long)kbeg * plane + r;
        const int i = (int)(r % nx), j = (int)((r / nx) % ny), k = kbeg + (int)(r / plane);
        const double p0 = p[g];
        const double pe = p[g - i + wrap(i + 1, nx)];
        const double pn = p[g + (long)(wrap(j + 1, ny) - j) * nx];
        u[g] = u[g] - dt * (pe - p0) * rdx;
        v[g] = v[g] - dt * (pn - p0) * rdy;
        if (rigid && wrap(k + kofs, nzg) == nzg - 1) {
            w[g] = 0.0;
        } else {
            const double pt = p[g + (long)(wrap(k + 1, nz) - k) * plane];
            w[g] = w[g] - dtw * (pt - p0) * rdz;
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// the launcher-derived fields of a step and its grid of blocks
static dim3 prep_step(StepArgs& a, int by) {
    a.hdx = 0.5 * a.rdx; a.hdy = 0.5 * a.rdy; a.hdz = 0.5 * a.rdz;
    a.qdx = 0.25 * a.rdx; a.qdy = 0.25 * a.rdy; a.qdz = 0.25 * a.rdz;
    a.qf0 = 0.25 * a.f0; a.hN0sq = 0.5 * a.N0sq;
    const int kcnt = a.kcount ? a.kcount : a.nz;
    a.kchunk = a.kchunk > 0 ? std::min(a.kchunk, kcnt) : (kcnt <= 16 ? kcnt : 8);
    return dim3((a.nx + kTX - 1) / kTX, (a.ny + by - 1) / by, ((kcnt + a.kchunk - 1) / a.kchunk) * std::max(1, a.batch));
}

template <typename TT, int BY, bool HARM, bool WM, bool BG>
static cudaError_t launch_step_t(const StepArgs& a0, cudaStream_t s) {
    StepArgs a = a0;
    const dim3 grid = prep_step(a, BY);
    return launch_pdl(k_step<TT, BY, HARM, WM, BG>, grid, dim3(kTX, BY), sizeof(StepSmem<TT, BY, BG ? 6 : 4>), s, a,
                      a.kchunk);
}

template <typename TT, int BY, bool HARM, bool WM, bool BG>
static cudaError_t launch_step_groups_t(const StepArgs* in, int n, cudaStream_t s) {
    static_assert(sizeof(StepGroups) <= 32000, "grouped step table exceeds the kernel parameter space");
    StepGroups m{};
    m.n = n;
    long blocks = 0;
    for (int g = 0; g < n; ++g) {
        m.a[g] = in[g];
        const dim3 gr = prep_step(m.a[g], BY);
        m.gx[g] = (int)gr.x; m.gy[g] = (int)gr.y;
        m.blk0[g] = (int)blocks;
        blocks += (long)gr.x * gr.y * gr.z;
    }
    if (blocks > 0x7fffffffL) return cudaErrorInvalidValue;
    m.blk0[n] = (int)blocks;
    return launch_pdl(k_step_groups<TT, BY, HARM, WM, BG>, dim3((unsigned)blocks), dim3(kTX, BY),
                      sizeof(StepSmem<TT, BY, BG ? 6 : 4>), s, m);
}

int step_flavour(const StepArgs& a) {
    return (a.harm_uvw || a.harm_b ? 1 : 0) | (a.wm_on ? 2 : 0) | (a.ub ? 4 : 0);
}

template <typename TT>
static cudaError_t launch_step_groups_tt(const StepArgs* a, int n, cudaStream_t s) {
    if (n < 1 || n > kMaxStepGroups) return cudaErrorInvalidValue;
    const int fl = step_flavour(a[0]);
    for (int g = 1; g < n; ++g)
        if (step_flavour(a[g]) != fl) return cudaErrorInvalidValue;
#define L(H, W, G) return launch_step_groups_t<TT, 8, H, W, G>(a, n, s)
    switch (fl) {
        case 0: L(false, false, false);
        case 1: L(true, false, false);
        case 2: L(false, true, false);
        case 3: L(true, true, false);
        case 4: L(false, false, true);
        case 5: L(true, false, true);
        case 6: L(false, true, true);
        default: L(true, true, true);
    }
#undef L
}

cudaError_t launch_step_groups(const StepArgs* a, int n, bool fp32_tendencies, cudaStream_t s) {
    return fp32_tendencies ? launch_step_groups_tt<float>(a, n, s) : launch_step_groups_tt<double>(a, n, s);
}

template <typename TT>
static cudaError_t launch_step_tt(const StepArgs& a, cudaStream_t s) {
    const bool harm = a.harm_uvw || a.harm_b;
    const bool wm = a.wm_on != 0;
    const bool bg = a.ub != nullptr;
#define L(H, W, G) return launch_step_t<TT, 8, H, W, G>(a, s)
    if (harm) { if (wm) { if (bg) L(true, true, true); else L(true, true, false); } else { if (bg) L(true, false, true); else L(true, false, false); } }
    else { if (wm) { if (bg) L(false, true, true); else L(false, true, false); } else { if (bg) L(false, false, true); else L(false, false, false); } }
#undef L
}

template <typename TT>
static cudaError_t step_setup_tt() {
    cudaError_t e;
    // PS3D_STEP_CARVEOUT=<percent>: the shared-memory share of the unified
    // L1/shared storage the step kernels ask for (a hint to the driver)
    const char* cv = std::getenv("PS3D_STEP_CARVEOUT");
    const int carve = cv ? std::atoi(cv) : -1;
#define S(H, W, G)                                                                                        \
    if ((e = cudaFuncSetAttribute(k_step<TT, 8, H, W, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                  (int)sizeof(StepSmem<TT, 8, G ? 6 : 4>))))                              \
        return e;                                                                                         \
    if ((e = cudaFuncSetAttribute(k_step_groups<TT, 8, H, W, G>,                                       \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                            \
                                  (int)sizeof(StepSmem<TT, 8, G ? 6 : 4>))))                              \
        return e;                                                                                         \
    if (carve >= 0 &&                                                                                     \
        (e = cudaFuncSetAttribute(k_step<TT, 8, H, W, G>, cudaFuncAttributePreferredSharedMemoryCarveout,  \
                                  carve)))                                                                \
        return e;
    S(true, true, true) S(true, true, false) S(true, false, true) S(true, false, false)
    S(false, true, true) S(false, true, false) S(false, false, true) S(false, false, false)
#undef S
    return cudaSuccess;
}
// opts the step kernels in to their dynamic shared memory (above 48 KB with
// the background fields)
cudaError_t step_setup() {
    cudaError_t e = step_setup_tt<double>();
    return e != cudaSuccess ? e : step_setup_tt<float>();
}

// resident blocks per SM of the fused step kernel that launch_step(a) runs
template <typename TT>
static int step_resident_tt(const StepArgs& a) {
    int n = 0;
    cudaError_t e = cudaSuccess;
#define R(H, W, G)                                                                                            \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<TT, 8, H, W, G>, kTX * 8,                   \
                                                      sizeof(StepSmem<TT, 8, G ? 6 : 4>));
    switch (step_flavour(a)) {
        case 0: R(false, false, false) break;
        case 1: R(true, false, false) break;
        case 2: R(false, true, false) break;
        case 3: R(true, true, false) break;
        case 4: R(false, false, true) break;
        case 5: R(true, false, true) break;
        case 6: R(false, true, true) break;
        default: R(true, true, true) break;
    }
#undef R
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}
int step_resident(const StepArgs& a, bool fp32_tendencies) {
    return fp32_tendencies ? step_resident_tt<float>(a) : step_resident_tt<double>(a);
}

cudaError_t launch_step(const StepArgs& a, bool fp32_tendencies, cudaStream_t s) {
    return fp32_tendencies ? launch_step_tt<float>(a, s) : launch_step_tt<double>(a, s);
}

static inline int grid_for(long n, int threads) {
    long b = (n + threads - 1) / threads;
    return (int)std::min<long>(b, 148L * 16);
}

cudaError_t launch_biharmonic_h(const double* cur, const double* old, double* out, int nx, int ny, int nz,
                                double Hmix, double rdx, double rdy, double dt, cudaStream_t s) {
    const long N = (long)nx * ny * nz;
    k_biharmonic_h<<<grid_for(N, 256), 256, 0, s>>>(cur, old, out, nx, ny, nz, Hmix, rdx, rdy, dt);
    return cudaGetLastError();
}
cudaError_t launch_biharmonic_v(const double* cur, const double* old, double* out, int nx, int ny, int nz,
                                int rigid, double Vmix, double rdz, double dt, cudaStream_t s) {
    const long N = (long)nx * ny * nz;
    k_biharmonic_v<<<grid_for(N, 256), 256, 0, s>>>(cur, old, out, nx, ny, nz, rigid, Vmix, rdz, dt);
    return cudaGetLastError();
}
cudaError_t launch_forcing_background(const StepArgs& a, cudaStream_t s) {
    const long N = (long)a.nx * a.ny * a.nz;
    k_forcing_background<<<grid_for(N, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_wavemaker_ab(const StepArgs& a, int do_wm, cudaStream_t s) {
    const long N = (long)a.nx * a.ny * a.nz;
    k_wavemaker_ab<<<grid_for(N, 256), 256, 0, s>>>(a, do_wm);
    return cudaGetLastError();
}
cudaError_t launch_correct(double* u, double* v, double* w, const double* p, int nx, int ny, int nz, int rigid,
                           double dt, double dtw, double rdx, double rdy, double rdz, cudaStream_t s, int batch,
                           int kbeg, int kcount, int kofs, int nzg) {
    const int kcnt = kcount ? kcount : nz;
    const long N = (long)nx * ny * kcnt * batch;
    k_correct<<<grid_for(N, 256), 256, 0, s>>>(u, v, w, p, nx, ny, nz, rigid, dt, dtw, rdx, rdy, rdz, batch, kbeg, kcnt,
                                              kofs, nzg ? nzg : nz);
    return cudaGetLastError();
}

}  // namespace ps3d
