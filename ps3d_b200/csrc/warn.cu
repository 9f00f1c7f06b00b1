// warn.cu — Warn-et-al. normal-mode balance to third order on the device
// (diag_balance.f90:89-362, model_run :465-497, model_nonlin :500-535).
//
// The balanced state is u0 + u1 + u2 + u3, where u0 is the geostrophic
// (zero-order) projection and the corrections u_n (O(Ro^n)) are built from
// the advective tendencies of lower-order states projected on the two
// inertia-gravity modes s = +-1.  Every spectral step is pointwise, so one
// kernel (k_warn) runs each of the reference's (i,j,k) loops with the
// eigenvectors p(s), q(s) and omega rebuilt per point (eigen.cuh); the
// advective tendencies of model_nonlin come from k_advect, the transforms
// and the 10-step model_run from the engine itself.
#include <cmath>
#include <vector>
#include "ctx.h"
#include "eigen.cuh"

namespace ps3d {

// spectral work arrays of module_diag_balance (diag_balance.f90:3-24)
enum {
    kF1p, kF1m, kI00, kI0p, kI0m, kIf1p, kIf1m, kI0f1p, kI0f1m, kIpT0p, kIpT0m,
    kF2p, kF2m, kIf2p, kIf2m, kI0f2p, kI0f2m, kPTf2p, kPTf2m, kWarnArrays
};
enum { kWarnF1, kWarnPM, kWarnS2b, kWarnS2d, kWarnDiff, kWarnT3, kWarnFilter };

struct WarnArgs {
    int nxh, ny, nz, rigid, layout, mode;
    double dx, dy, dz, f0, N0, dsqr, Ro, dt, kzcut2;
    EigenAxes ax;
    double2 *US, *VS, *WS, *BS;
    double2* A[kWarnArrays];
    double2 *o1, *o2;   // kWarnPM outputs
};

// ---------------------------------------------------------------------------
// model_nonlin's advective tendencies (buoyancy_advection_2nd,
// momentum_advection_2nd; advection.f90:2-184), divided by Ro (w also by
// dsqr), in the reference's operand order.  One thread per point; rigid-lid
// flux zeroing as advection.f90:42-43, 95-96, 134-135, 167-170.
// ---------------------------------------------------------------------------
__global__ void k_advect(const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
                         const double* __restrict__ b, double* __restrict__ du, double* __restrict__ dv,
                         double* __restrict__ dw, double* __restrict__ db, int nx, int ny, int nz, int rigid,
                         double dx, double dy, double dz, double Ro, double dsqr) {
    const long plane = (long)nx * ny, N = plane * nz;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
        const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / plane);
        const int ip = wrap(i + 1, nx), im = wrap(i - 1, nx), jp = wrap(j + 1, ny), jm = wrap(j - 1, ny);
        const int kp = wrap(k + 1, nz), km = wrap(k - 1, nz);
        auto at = [&](const double* f, int ii, int jj, int kk) { return __ldg(f + (long)kk * plane + (long)jj * nx + ii); };
        const bool top = rigid && k == nz - 1, bot = rigid && k == 0;
        const bool wtop = rigid && k >= nz - 2, wbot = rigid && (k == 0 || k >= nz - 1);
        // buoyancy
        {
            const double fe = 0.5 * (at(b, i, j, k) + at(b, ip, j, k)) * at(u, i, j, k);
            const double fem = 0.5 * (at(b, im, j, k) + at(b, i, j, k)) * at(u, im, j, k);
            const double fn = 0.5 * (at(b, i, j, k) + at(b, i, jp, k)) * at(v, i, j, k);
            const double fnm = 0.5 * (at(b, i, jm, k) + at(b, i, j, k)) * at(v, i, jm, k);
            const double ft = top ? 0.0 : 0.5 * (at(b, i, j, k) + at(b, i, j, kp)) * at(w, i, j, k);
            const double ftm = bot ? 0.0 : 0.5 * (at(b, i, j, km) + at(b, i, j, k)) * at(w, i, j, km);
            db[g] = -Ro * ((fe - fem) / dx + (fn - fnm) / dy + (ft - ftm) / dz) / Ro;
        }
        // zonal momentum
        {
            const double e = 0.25 * (at(u, i, j, k) + at(u, ip, j, k)) * (at(u, ip, j, k) + at(u, i, j, k));
            const double em = 0.25 * (at(u, im, j, k) + at(u, i, j, k)) * (at(u, i, j, k) + at(u, im, j, k));
            const double n = 0.25 * (at(u, i, j, k) + at(u, i, jp, k)) * (at(v, ip, j, k) + at(v, i, j, k));
            const double nm = 0.25 * (at(u, i, jm, k) + at(u, i, j, k)) * (at(v, ip, jm, k) + at(v, i, jm, k));
            const double t = top ? 0.0 : 0.25 * (at(u, i, j, kp) + at(u, i, j, k)) * (at(w, i, j, k) + at(w, ip, j, k));
            const double tm = bot ? 0.0 : 0.25 * (at(u, i, j, k) + at(u, i, j, km)) * (at(w, i, j, km) + at(w, ip, j, km));
            du[g] = -Ro * ((e - em) / dx + (n - nm) / dy + (t - tm) / dz) / Ro;
        }
        // meridional momentum
        {
            const double e = 0.25 * (at(v, i, j, k) + at(v, ip, j, k)) * (at(u, i, jp, k) + at(u, i, j, k));
            const double em = 0.25 * (at(v, im, j, k) + at(v, i, j, k)) * (at(u, im, jp, k) + at(u, im, j, k));
            const double n = 0.25 * (at(v, i, j, k) + at(v, i, jp, k)) * (at(v, i, jp, k) + at(v, i, j, k));
            const double nm = 0.25 * (at(v, i, jm, k) + at(v, i, j, k)) * (at(v, i, j, k) + at(v, i, jm, k));
            const double t = top ? 0.0 : 0.25 * (at(v, i, j, kp) + at(v, i, j, k)) * (at(w, i, j, k) + at(w, i, jp, k));
            const double tm = bot ? 0.0 : 0.25 * (at(v, i, j, k) + at(v, i, j, km)) * (at(w, i, j, km) + at(w, i, jp, km));
            dv[g] = -Ro * ((e - em) / dx + (n - nm) / dy + (t - tm) / dz) / Ro;
        }
        // vertical momentum
        {
            const double e = 0.25 * (at(w, i, j, k) + at(w, ip, j, k)) * (at(u, i, j, k) + at(u, i, j, kp));
            const double em = 0.25 * (at(w, im, j, k) + at(w, i, j, k)) * (at(u, im, j, k) + at(u, im, j, kp));
            const double n = 0.25 * (at(w, i, j, k) + at(w, i, jp, k)) * (at(v, i, j, k) + at(v, i, j, kp));
            const double nm = 0.25 * (at(w, i, jm, k) + at(w, i, j, k)) * (at(v, i, jm, k) + at(v, i, jm, kp));
            const double t = wtop ? 0.0 : 0.25 * (at(w, i, j, kp) + at(w, i, j, k)) * (at(w, i, j, k) + at(w, i, j, kp));
            const double tm = wbot ? 0.0 : 0.25 * (at(w, i, j, k) + at(w, i, j, km)) * (at(w, i, j, km) + at(w, i, j, k));
            dw[g] = -dsqr * Ro * ((e - em) / dx + (n - nm) / dy + (t - tm) / dz) / Ro / dsqr;
        }
    }
}

// out = (a ? a : 0) + (divide ? b / s : b * s), four fields
struct Comb4 { const double* a[4]; const double* b[4]; double* out[4]; };
__global__ void k_comb4(Comb4 c, long N, double s, int divide, int has_a) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const double y = divide ? c.b[f][g] / s : c.b[f][g] * s;
            c.out[f][g] = has_a ? c.a[f][g] + y : y;
        }
    }
}

__device__ __forceinline__ cz_t dotp4(const cz_t* p, cz_t U, cz_t V, cz_t W, cz_t B) {
    return p[0] * U + p[1] * V + p[2] * W + p[3] * B;
}

__global__ void k_warn(const WarnArgs a) {
    const long M = (long)a.nxh * a.ny * a.nz;
    const Phys P{a.f0, a.N0, a.dsqr, a.dz};
    const cz_t IM = Cz(0, 1);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < M; t += (long)gridDim.x * blockDim.x) {
        const int i = a.layout ? (int)((t / a.ny) % a.nxh) : (int)(t % a.nxh);
        const int j = a.layout ? (int)(t % a.ny) : (int)((t / a.nxh) % a.ny);
        const int k = (int)(t / ((long)a.nxh * a.ny));
        if (a.mode == kWarnFilter) {   // model_nonlin's kz filter (diag_balance.f90:520-531)
            const double kz = a.ax.kz[k];
            if (kz * kz >= a.kzcut2) {
                st(a.US + t, Cz(0, 0)); st(a.VS + t, Cz(0, 0)); st(a.WS + t, Cz(0, 0)); st(a.BS + t, Cz(0, 0));
            }
            continue;
        }
        if (a.mode == kWarnDiff) {     // pTf2 = (f2 - pTf2)/(10 dt)/Ro (diag_balance.f90:335-336)
            st(a.A[kPTf2p] + t, (ld(a.A[kF2p] + t) - ld(a.A[kPTf2p] + t)) / (10. * a.dt) / a.Ro);
            st(a.A[kPTf2m] + t, (ld(a.A[kF2m] + t) - ld(a.A[kPTf2m] + t)) / (10. * a.dt) / a.Ro);
            continue;
        }
        Ax x{a.ax.kx[i], a.ax.hkx[i], a.ax.ex[i], ld(a.ax.px + i), a.dx};
        Ax y{a.ax.ky[j], a.ax.hky[j], a.ax.ey[j], ld(a.ax.py + j), a.dy};
        Ax z{a.ax.kz[k], a.rigid ? 0.0 : a.ax.hkz[k], a.rigid ? 0.0 : a.ax.ez[k],
             a.rigid ? Cz(1, 0) : ld(a.ax.pz + k), a.dz};
        auto qp = [&](double s, cz_t* q, cz_t* p) {
            if (a.rigid) vec_qp_vbc(x, y, a.ax.kz[k], a.ax.sz[k], a.ax.cz[k], s, P, q, p);
            else vec_qp_discrete(x, y, z, s, P, q, p);
        };
        auto omega = [&]() {
            const double om2 = a.rigid ? omega2_vbc(x, y, a.ax.sz[k], a.ax.cz[k], P) : omega2_discrete(x, y, z, P);
            return sqrt(om2);
        };
        const cz_t US = ld(a.US + t), VS = ld(a.VS + t), WS = ld(a.WS + t), BS = ld(a.BS + t);
        cz_t q0[4], p0[4], qp1[4], pp1[4], qm1[4], pm1[4];
        if (a.mode == kWarnPM) {       // I(+-) = im p(+-1).S
            qp(+1.0, qp1, pp1);
            qp(-1.0, qm1, pm1);
            st(a.o1 + t, IM * dotp4(pp1, US, VS, WS, BS));
            st(a.o2 + t, IM * dotp4(pm1, US, VS, WS, BS));
            continue;
        }
        qp(+1.0, qp1, pp1);
        qp(-1.0, qm1, pm1);
        const double om = omega();
        if (a.mode == kWarnF1) {       // diag_balance.f90:151-171
            qp(0.0, q0, p0);
            const cz_t I00 = IM * dotp4(p0, US, VS, WS, BS);
            const cz_t I0p = IM * dotp4(pp1, US, VS, WS, BS);
            const cz_t I0m = IM * dotp4(pm1, US, VS, WS, BS);
            cz_t f1p = Cz(0, 0), f1m = Cz(0, 0);
            if (om > 0.) { f1p = I0p / om; f1m = -(I0m / om); }
            st(a.A[kI00] + t, I00); st(a.A[kI0p] + t, I0p); st(a.A[kI0m] + t, I0m);
            st(a.A[kF1p] + t, f1p); st(a.A[kF1m] + t, f1m);
            st(a.US + t, a.Ro * (f1p * qp1[0] + f1m * qm1[0]));
            st(a.VS + t, a.Ro * (f1p * qp1[1] + f1m * qm1[1]));
            st(a.WS + t, a.Ro * (f1p * qp1[2] + f1m * qm1[2]));
            st(a.BS + t, a.Ro * (f1p * qp1[3] + f1m * qm1[3]));
        } else if (a.mode == kWarnS2b) {   // diag_balance.f90:203-216
            qp(0.0, q0, p0);
            st(a.A[kI0f1p] + t, IM * dotp4(pp1, US, VS, WS, BS));
            st(a.A[kI0f1m] + t, IM * dotp4(pm1, US, VS, WS, BS));
            const cz_t pTg0 = -(IM * ld(a.A[kI00] + t));
            st(a.US + t, pTg0 * q0[0]); st(a.VS + t, pTg0 * q0[1]);
            st(a.WS + t, pTg0 * q0[2]); st(a.BS + t, pTg0 * q0[3]);
        } else if (a.mode == kWarnS2d) {   // diag_balance.f90:238-266
            const cz_t I0pT0p = IM * dotp4(pp1, US, VS, WS, BS);
            const cz_t I0pT0m = IM * dotp4(pm1, US, VS, WS, BS);
            cz_t f2p = Cz(0, 0), f2m = Cz(0, 0);
            if (om > 0) {
                const cz_t pTf1p = (I0pT0p - ld(a.A[kI0p] + t) - ld(a.A[kIpT0p] + t)) / om;
                const cz_t pTf1m = -((I0pT0m - ld(a.A[kI0m] + t) - ld(a.A[kIpT0m] + t)) / om);
                f2p = (ld(a.A[kI0f1p] + t) - ld(a.A[kI0p] + t) - ld(a.A[kIf1p] + t) - IM * pTf1p) / om;
                f2m = -((ld(a.A[kI0f1m] + t) - ld(a.A[kI0m] + t) - ld(a.A[kIf1m] + t) - IM * pTf1m) / om);
            }
            st(a.A[kF2p] + t, f2p); st(a.A[kF2m] + t, f2m);
            const double Ro2 = a.Ro * a.Ro;
            st(a.US + t, Ro2 * (f2p * qp1[0] + f2m * qm1[0]));
            st(a.VS + t, Ro2 * (f2p * qp1[1] + f2m * qm1[1]));
            st(a.WS + t, Ro2 * (f2p * qp1[2] + f2m * qm1[2]));
            st(a.BS + t, Ro2 * (f2p * qp1[3] + f2m * qm1[3]));
        } else if (a.mode == kWarnT3) {    // diag_balance.f90:342-359
            cz_t f3p = Cz(0, 0), f3m = Cz(0, 0);
            if (om > 0) {
                f3p = (ld(a.A[kI0f2p] + t) + ld(a.A[kIf1p] + t) - ld(a.A[kIf2p] + t) - ld(a.A[kI0p] + t) -
                       IM * ld(a.A[kPTf2p] + t)) / om;
                f3m = -((ld(a.A[kI0f2m] + t) + ld(a.A[kIf1m] + t) - ld(a.A[kIf2m] + t) - ld(a.A[kI0m] + t) -
                         IM * ld(a.A[kPTf2m] + t)) / om);
            }
            const double Ro3 = a.Ro * a.Ro * a.Ro;
            st(a.US + t, Ro3 * (f3p * qp1[0] + f3m * qm1[0]));
            st(a.VS + t, Ro3 * (f3p * qp1[1] + f3m * qm1[1]));
            st(a.WS + t, Ro3 * (f3p * qp1[2] + f3m * qm1[2]));
            st(a.BS + t, Ro3 * (f3p * qp1[3] + f3m * qm1[3]));
        }
    }
}

static int blocks_for(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 16); }

// ---------------------------------------------------------------------------
// host driver (Ctx members)
// ---------------------------------------------------------------------------
cudaError_t Ctx::ensure_warn() {
    if (warn_arr[0].p) return cudaSuccess;
    cudaError_t e;
    for (int q = 0; q < kWarnArrays; ++q) {
        if ((e = warn_arr[q].alloc(M * sizeof(double2)))) return e;
        if ((e = cudaMemsetAsync(warn_arr[q].p, 0, M * sizeof(double2), stream))) return e;
    }
    for (int set : {(int)PS3D_FIELDS_ZERO, (int)PS3D_FIELDS_FIRST, (int)PS3D_FIELDS_SECOND, (int)PS3D_FIELDS_THIRD,
                    (int)kSetPT0, (int)kSetComb, (int)kSetSave})
        if ((e = ensure_fieldset(set))) return e;
    if ((e = ensure_saved_tail())) return e;
    for (int f = 0; f < 4; ++f)
        if ((e = nl_tend[f].alloc(N * sizeof(double)))) return e;
    return ensure_spectral4();
}

int Ctx::warn_launch(int mode, double2* o1, double2* o2, double kzcut2) {
    WarnArgs a{};
    a.nxh = nxh; a.ny = ny; a.nz = nz; a.rigid = rigid; a.layout = spectral_layout(pa64); a.mode = mode;
    a.dx = P.dx; a.dy = P.dy; a.dz = P.dz; a.f0 = P.f0; a.N0 = P.N0; a.dsqr = P.dsqr; a.Ro = P.Ro; a.dt = P.dt;
    a.kzcut2 = kzcut2;
    a.ax.kx = (const double*)t_kx.p; a.ax.ky = (const double*)t_ky.p; a.ax.kz = (const double*)t_kz.p;
    a.ax.hkx = (const double*)t_hkx.p; a.ax.hky = (const double*)t_hky.p; a.ax.hkz = (const double*)t_hkz.p;
    a.ax.ex = (const double*)t_ex.p; a.ax.ey = (const double*)t_ey.p; a.ax.ez = (const double*)t_ez.p;
    a.ax.px = (const double2*)t_px.p; a.ax.py = (const double2*)t_py.p; a.ax.pz = (const double2*)t_pz.p;
    a.ax.sz = (const double*)t_sz.p; a.ax.cz = (const double*)t_cz.p;
    a.US = (double2*)spec4[0].p; a.VS = (double2*)spec4[1].p; a.WS = (double2*)spec4[2].p; a.BS = (double2*)spec4[3].p;
    for (int q = 0; q < kWarnArrays; ++q) a.A[q] = (double2*)warn_arr[q].p;
    a.o1 = o1; a.o2 = o2;
    k_warn<<<blocks_for(M), 256, 0, stream>>>(a);
    CK(cudaGetLastError());
    return PS3D_OK;
}

// model_nonlin (diag_balance.f90:500-535) of the state in `in` into spec4
int Ctx::model_nonlin(const double* const* in) {
    k_advect<<<blocks_for(N), 256, 0, stream>>>(in[0], in[1], in[2], in[3], (double*)nl_tend[0].p,
                                                (double*)nl_tend[1].p, (double*)nl_tend[2].p, (double*)nl_tend[3].p,
                                                nx, ny, nz, rigid, P.dx, P.dy, P.dz, P.Ro, P.dsqr);
    CK(cudaGetLastError());
    const double* t[4] = {(const double*)nl_tend[0].p, (const double*)nl_tend[1].p, (const double*)nl_tend[2].p,
                          (const double*)nl_tend[3].p};
    int rc = forward_transform(t);
    if (rc) return rc;
    if (warn_filter >= 0) {
        std::vector<double> kz(nz);
        CK(cudaMemcpy(kz.data(), t_kz.p, nz * sizeof(double), cudaMemcpyDeviceToHost));
        const double fxa = std::fabs(kz[nz / 2 + warn_filter]);   // kz(nz/2+1+width)
        rc = warn_launch(kWarnFilter, nullptr, nullptr, fxa * fxa);
    }
    return rc;
}

// the combination a + b/s (or b*s) of two field sets into kSetComb
int Ctx::warn_comb(int set_a, int set_b, double s, bool divide) {
    Comb4 c{};
    DevBuf* A = set_a >= 0 ? fieldset(set_a) : nullptr;
    DevBuf* B = fieldset(set_b);
    DevBuf* O = fieldset(kSetComb);
    for (int f = 0; f < 4; ++f) {
        c.a[f] = A ? (const double*)A[f].p : nullptr;
        c.b[f] = (const double*)B[f].p;
        c.out[f] = (double*)O[f].p;
    }
    k_comb4<<<blocks_for(N), 256, 0, stream>>>(c, N, s, divide ? 1 : 0, A ? 1 : 0);
    CK(cudaGetLastError());
    return PS3D_OK;
}
int Ctx::model_nonlin_set(int set) {
    DevBuf* S = fieldset(set);
    const double* in[4] = {(const double*)S[0].p, (const double*)S[1].p, (const double*)S[2].p, (const double*)S[3].p};
    return model_nonlin(in);
}
int Ctx::backward_to_set(int set) {
    DevBuf* S = fieldset(set);
    double* out[4] = {(double*)S[0].p, (double*)S[1].p, (double*)S[2].p, (double*)S[3].p};
    return backward_transform(out);
}

// model_run (diag_balance.f90:465-497): max_steps of integrate from the
// state in set `in` (itt stays 0: forward steps), result into set `out`,
// model state saved and restored
int Ctx::model_run(int in, int out, int max_steps) {
    CK(copy_state_to(kSetSave));
    CK(cudaMemcpyAsync(saved_p.p, p.p, N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    for (int f = 0; f < 4; ++f)
        CK(cudaMemcpyAsync(saved_tend[f].p, tend[f].p, 3 * N * tsz(f), cudaMemcpyDeviceToDevice, stream));
    const int tau_loc = tau, taum1_loc = taum1, taum2_loc = taum2, itt_loc = itt;
    CK(copy_set_to_state(in));
    itt = 0; taum2 = 1; taum1 = 2; tau = 3;
    int rc = PS3D_OK;
    for (int n = 1; n <= max_steps && !rc; ++n) {
        rc = step(itt, tau, taum1, taum2);
        rotate();
    }
    if (!rc) CK(copy_state_to(out));
    CK(copy_set_to_state(kSetSave));
    CK(cudaMemcpyAsync(p.p, saved_p.p, N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    for (int f = 0; f < 4; ++f)
        CK(cudaMemcpyAsync(tend[f].p, saved_tend[f].p, 3 * N * tsz(f), cudaMemcpyDeviceToDevice, stream));
    tau = tau_loc; taum1 = taum1_loc; taum2 = taum2_loc; itt = itt_loc;
    state_replaced();
    return rc;
}

#define WCHK(x)                  \
    do {                         \
        int rc_ = (x);           \
        if (rc_) return rc_;     \
    } while (0)

int Ctx::warn_first() {   // diag_balance.f90:135-176
    WCHK(model_nonlin_set(PS3D_FIELDS_ZERO));
    WCHK(warn_launch(kWarnF1));
    return backward_to_set(PS3D_FIELDS_FIRST);
}
int Ctx::warn_second() {  // diag_balance.f90:180-272
    const double Ro = P.Ro;
    WCHK(warn_comb(-1, PS3D_FIELDS_FIRST, Ro, true));
    WCHK(model_nonlin_set(kSetComb));
    WCHK(warn_launch(kWarnPM, (double2*)warn_arr[kIf1p].p, (double2*)warn_arr[kIf1m].p));
    WCHK(warn_comb(PS3D_FIELDS_ZERO, PS3D_FIELDS_FIRST, Ro, true));
    WCHK(model_nonlin_set(kSetComb));
    WCHK(warn_launch(kWarnS2b));
    WCHK(backward_to_set(kSetPT0));
    WCHK(model_nonlin_set(kSetPT0));
    WCHK(warn_launch(kWarnPM, (double2*)warn_arr[kIpT0p].p, (double2*)warn_arr[kIpT0m].p));
    WCHK(warn_comb(PS3D_FIELDS_ZERO, kSetPT0, 1.0, false));
    WCHK(model_nonlin_set(kSetComb));
    WCHK(warn_launch(kWarnS2d));
    return backward_to_set(PS3D_FIELDS_SECOND);
}
int Ctx::warn_third() {   // diag_balance.f90:275-362
    const double Ro2 = P.Ro * P.Ro;
    WCHK(warn_comb(-1, PS3D_FIELDS_SECOND, Ro2, true));
    WCHK(model_nonlin_set(kSetComb));
    WCHK(warn_launch(kWarnPM, (double2*)warn_arr[kIf2p].p, (double2*)warn_arr[kIf2m].p));
    WCHK(warn_comb(PS3D_FIELDS_ZERO, PS3D_FIELDS_SECOND, Ro2, true));
    WCHK(model_nonlin_set(kSetComb));
    WCHK(warn_launch(kWarnPM, (double2*)warn_arr[kI0f2p].p, (double2*)warn_arr[kI0f2m].p));
    // model_run(u0+u1+u2 -> u3, 10 steps)
    WCHK(warn_comb(PS3D_FIELDS_ZERO, PS3D_FIELDS_FIRST, 1.0, false));
    {
        DevBuf* Cm = fieldset(kSetComb);
        DevBuf* T = fieldset(PS3D_FIELDS_THIRD);
        for (int f = 0; f < 4; ++f)   // the sum so far into THIRD, then THIRD + u2 into kSetComb
            CK(cudaMemcpyAsync(T[f].p, Cm[f].p, N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        WCHK(warn_comb(PS3D_FIELDS_THIRD, PS3D_FIELDS_SECOND, 1.0, false));
    }
    WCHK(model_run(kSetComb, PS3D_FIELDS_THIRD, 10));
    // zero-order projection of u3 into u0
    {
        DevBuf* T = fieldset(PS3D_FIELDS_THIRD);
        const double* in[4] = {(const double*)T[0].p, (const double*)T[1].p, (const double*)T[2].p,
                               (const double*)T[3].p};
        WCHK(forward_transform(in));
        WCHK(project_spectral(PS3D_PROJ_ZERO_ORDER));
        WCHK(backward_to_set(PS3D_FIELDS_ZERO));
    }
    CK(cudaMemcpyAsync(warn_arr[kPTf2p].p, warn_arr[kF2p].p, M * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(warn_arr[kPTf2m].p, warn_arr[kF2m].p, M * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
    WCHK(warn_first());
    WCHK(warn_second());
    WCHK(warn_launch(kWarnDiff));
    WCHK(project(PS3D_PROJ_ZERO_ORDER));
    WCHK(warn_first());
    WCHK(warn_second());
    WCHK(warn_launch(kWarnT3));
    return backward_to_set(PS3D_FIELDS_THIRD);
}

int Ctx::diag_balance(int order, int filter_width) {
    if (order < 0 || order > 3) return PS3D_ERR_BADPARAM;
    if (filter_width >= 0 && nz / 2 + filter_width >= nz) return PS3D_ERR_BADPARAM;
    WCHK(materialize());
    p_warm = false;   // the balanced state replaces the model state
    CK(ensure_warn());
    warn_filter = filter_width;
    WCHK(project(PS3D_PROJ_ZERO_ORDER));   // diag_balance_zero_order
    if (order >= 1) WCHK(warn_first());
    if (order >= 2) WCHK(warn_second());
    if (order >= 3) WCHK(warn_third());
    CK(cudaStreamSynchronize(stream));
    return PS3D_OK;
}

}  // namespace ps3d
