// modes.cu — normal-mode (eigenvector) projection on sm_100a.
//
// Per spectral point the reference evaluates the left/right eigenvectors
// p^0, q^0 of the linear operator (eigenvectors.f90:6-218, dispatched by
// diag_balance.f90:366-418) and projects the state on the geostrophic mode:
//   normal_mode_projection          diag_opt_balance.f90:288-310
//   geostrophic_base_point          diag_opt_balance.f90:263-285
//   exchange_geostrophic_base_point diag_opt_balance.f90:313-335
//   diag_balance_zero_order         diag_balance.f90:109-132
// Storing the eight complex eigenvector components per point would cost
// 128 B of HBM per spectral point; here they are rebuilt in registers from
// 1D per-axis tables (hat_ksqr, hat_epm, exp(i k d), sin/cos(kz dz/2)) that
// the host computes once with libm, so the kernel streams only the four
// spectral fields.  The arithmetic follows eigenvectors.f90 operation for
// operation.
//
// The rigid-lid vertical-mode transforms (my_fft_vert_mode /
// my_ifft_vert_mode, my_fft.f90:211-252) are dense nz x nz real matrices
// applied to every (kx,ky) column; k_vert_mode stages a block of columns in
// shared memory and sums in the reference's order.
#include "engine.h"

namespace ps3d {

struct cz_t { double re, im; };
__device__ __forceinline__ cz_t Cz(double r, double i) { cz_t c; c.re = r; c.im = i; return c; }
__device__ __forceinline__ cz_t operator+(cz_t a, cz_t b) { return Cz(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ cz_t operator-(cz_t a, cz_t b) { return Cz(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ cz_t operator-(cz_t a) { return Cz(-a.re, -a.im); }
__device__ __forceinline__ cz_t operator*(cz_t a, cz_t b) { return Cz(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ __forceinline__ cz_t operator*(cz_t a, double s) { return Cz(a.re * s, a.im * s); }
__device__ __forceinline__ cz_t operator*(double s, cz_t a) { return Cz(s * a.re, s * a.im); }
__device__ __forceinline__ cz_t operator/(cz_t a, double s) { return Cz(a.re / s, a.im / s); }
__device__ __forceinline__ cz_t conjg(cz_t a) { return Cz(a.re, -a.im); }
__device__ __forceinline__ cz_t ld(const double2* p) { double2 v = *p; return Cz(v.x, v.y); }
__device__ __forceinline__ void st(double2* p, cz_t v) { *p = make_double2(v.re, v.im); }

// per-axis quantities of one wavenumber
struct Ax {
    double k;     // wavenumber
    double hk;    // hat_ksqr(k, d)
    double ep;    // hat_epm(k, d)
    cz_t e;       // exp(i k d)
    double d;     // grid spacing
};
__device__ __forceinline__ cz_t hat_kp(const Ax& a) { const cz_t IM = Cz(0, 1); return -(IM * (a.e - Cz(1, 0)) / a.d); }
__device__ __forceinline__ cz_t hat_ep(const Ax& a) { return (a.e + Cz(1, 0)) * 0.5; }
__device__ __forceinline__ cz_t hat_em(const Ax& a) { return (conjg(a.e) + Cz(1, 0)) * 0.5; }

struct Phys { double f0, N0, dsqr, dz; };

// ---- rigid lid, eigenvectors.f90:6-104 (s = 0 only is needed here, but
//      the general form is kept for the balance orders)
__device__ double omega2_vbc(const Ax& x, const Ax& y, double sarg, double carg, const Phys& P) {
    const double k2 = x.hk + y.hk;
    const double m2 = 4 * (sarg * sarg) / (P.dz * P.dz);
    const double N2_hat = (P.N0 * P.N0) * (carg * carg);
    const double f2_hat = (P.f0 * P.f0) * x.ep * y.ep;
    const double Ksqr = P.dsqr * k2 + m2;
    return Ksqr > 0.0 ? (N2_hat * k2 + f2_hat * m2) / Ksqr : 0.0;
}
__device__ void vec_qp_vbc(const Ax& x, const Ax& y, double kz, double sarg, double carg, double s, const Phys& P,
                           cz_t* q, cz_t* p) {
    const cz_t IM = Cz(0, 1);
    const double om2 = omega2_vbc(x, y, sarg, carg, P);
    const double om = sqrt(om2);
    const double f2_hat = (P.f0 * P.f0) * x.ep * y.ep;
    const double N2_hat = (P.N0 * P.N0) * (carg * carg);
    const double lam = 2 * sarg / P.dz;
    cz_t qx, qy, qz, qb;
    if (x.k * x.k + y.k * y.k > 0.0) {
        double fxa = f2_hat - (s * s) * om2;
        qx = (-(IM * P.f0 * hat_ep(x) * hat_em(y) * hat_kp(y)) + s * om * hat_kp(x)) / fxa;
        qy = ((IM * P.f0 * hat_em(x) * hat_ep(y) * hat_kp(x)) + s * om * hat_kp(y)) / fxa;
        if (kz * kz > 0.0) {
            fxa = N2_hat - P.dsqr * (s * s) * om2;
            qz = IM * lam * s * om / fxa;
            qb = Cz(-(lam * carg * (P.N0 * P.N0) / fxa), 0.0);
        } else { qz = Cz(0, 0); qb = Cz(0, 0); }
    } else {
        qx = -(IM * s); qy = Cz(s * s, 0); qz = Cz(0, 0); qb = Cz(0, 0);
    }
    if (s == 0.0 && (f2_hat == 0.0 || N2_hat == 0.0)) { qx = qy = qz = qb = Cz(0, 0); }
    if (s != 0.0 && om2 == 0.0) { qx = qy = qz = qb = Cz(0, 0); }
    q[0] = qx; q[1] = qy; q[2] = qz; q[3] = qb;
    // coeff_p_vbc (eigenvectors.f90:27-47) and vec_p_vbc (:92-104)
    const double k2 = x.hk + y.hk;
    const double m2 = 4 * (sarg * sarg) / (P.dz * P.dz);
    const double dd = k2 * N2_hat + f2_hat * m2;
    double pc;
    if (s == 0.0 && dd > 0.0) pc = f2_hat * N2_hat / dd;
    else if (dd > 0.0) pc = (N2_hat - P.dsqr * om2) * (om2 - f2_hat) / (2 * dd);
    else pc = 0.0;
    p[0] = pc * conjg(qx);
    p[1] = pc * conjg(qy);
    p[2] = pc * conjg(qz) * P.dsqr;
    p[3] = pc * conjg(qb) / (P.N0 * P.N0);
}

// ---- triply periodic, eigenvectors.f90:110-218
__device__ void vec_qp_discrete(const Ax& x, const Ax& y, const Ax& z, double s, const Phys& P, cz_t* q, cz_t* p) {
    const cz_t IM = Cz(0, 1);
    const double k2 = x.hk + y.hk;
    const double Ksqr = P.dsqr * k2 + z.hk;
    const double om2 = Ksqr > 0.0 ? (z.ep * (P.N0 * P.N0) * k2 + (P.f0 * P.f0) * z.hk * x.ep * y.ep) / Ksqr : 0.0;
    const double om = sqrt(om2);
    const double f2_hat = (P.f0 * P.f0) * x.ep * y.ep;
    const double N2_hat = (P.N0 * P.N0) * z.ep;
    cz_t qx, qy, qz, qb;
    if (x.k * x.k + y.k * y.k > 0.0) {
        double fxa = f2_hat - (s * s) * om2;
        qx = (-(IM * P.f0 * hat_ep(x) * hat_em(y) * hat_kp(y)) + s * om * hat_kp(x)) / fxa;
        qy = ((IM * P.f0 * hat_em(x) * hat_ep(y) * hat_kp(x)) + s * om * hat_kp(y)) / fxa;
        if (z.k * z.k > 0.0) {
            fxa = N2_hat - P.dsqr * (s * s) * om2;
            qz = hat_kp(z) * s * om / fxa;
            qb = IM * hat_em(z) * hat_kp(z) * (P.N0 * P.N0) / fxa;
        } else { qz = Cz(0, 0); qb = Cz(0, 0); }
    } else {
        qx = -(IM * s); qy = Cz(s * s, 0); qz = Cz(0, 0); qb = Cz(0, 0);
    }
    if (s == 0.0 && (f2_hat == 0.0 || N2_hat == 0.0)) { qx = qy = qz = qb = Cz(0, 0); }
    if (s != 0.0 && om2 == 0.0) { qx = qy = qz = qb = Cz(0, 0); }
    if ((x.k * x.k + y.k * y.k > 0.0) && (z.k * z.k == 0.0) && (s != 0.0)) {
        qx = Cz(0, 0); qy = Cz(0, 0); qz = IM * s;
        qb = Cz((s * s) * P.N0 * sqrt(P.dsqr), 0.0);
    }
    q[0] = qx; q[1] = qy; q[2] = qz; q[3] = qb;
    const double dd = k2 * N2_hat + f2_hat * z.hk;
    double pc;
    if (s == 0.0 && dd > 0.0) pc = f2_hat * N2_hat / dd;
    else if (dd > 0.0) pc = (N2_hat - P.dsqr * om2) * (om2 - f2_hat) / (2 * dd);
    else pc = 0.0;
    p[0] = pc * conjg(qx);
    p[1] = pc * conjg(qy);
    p[2] = pc * conjg(qz) * P.dsqr;
    p[3] = pc * conjg(qb) / (P.N0 * P.N0);
    if ((x.k * x.k + y.k * y.k == 0.0) && (z.k * z.k > 0.0)) {
        p[0] = IM * s / 2.0; p[1] = Cz((s * s) / 2.0, 0);
    }
    if ((x.k * x.k + y.k * y.k > 0.0) && (z.k * z.k == 0.0) && (s != 0.0)) {
        p[0] = Cz(0, 0); p[1] = Cz(0, 0);
        p[2] = -(IM * s / 2.0);
        p[3] = Cz((s * s) / (2.0 * P.N0 * sqrt(P.dsqr)), 0);
    }
}

__global__ void k_project(const ProjArgs a) {
    const long M = (long)a.nxh * a.ny * a.nz;
    const Phys P{a.f0, a.N0, a.dsqr, a.dz};
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < M; t += (long)gridDim.x * blockDim.x) {
        const int i = a.layout ? (int)((t / a.ny) % a.nxh) : (int)(t % a.nxh);
        const int j = a.layout ? (int)(t % a.ny) : (int)((t / a.nxh) % a.ny);
        const int k = (int)(t / ((long)a.nxh * a.ny));
        Ax x{a.ax.kx[i], a.ax.hkx[i], a.ax.ex[i], ld(a.ax.px + i), a.dx};
        Ax y{a.ax.ky[j], a.ax.hky[j], a.ax.ey[j], ld(a.ax.py + j), a.dy};
        cz_t q[4], p[4];
        if (a.rigid) {
            vec_qp_vbc(x, y, a.ax.kz[k], a.ax.sz[k], a.ax.cz[k], 0.0, P, q, p);
        } else {
            Ax z{a.ax.kz[k], a.ax.hkz[k], a.ax.ez[k], ld(a.ax.pz + k), a.dz};
            vec_qp_discrete(x, y, z, 0.0, P, q, p);
        }
        const cz_t US = ld(a.US + t), VS = ld(a.VS + t), WS = ld(a.WS + t), BS = ld(a.BS + t);
        const cz_t g0 = p[0] * US + p[1] * VS + p[2] * WS + p[3] * BS;
        if (a.mode == PS3D_PROJ_EXCHANGE) {
            const cz_t d = ld(a.g0base + t) - g0;
            st(a.US + t, US + d * q[0]); st(a.VS + t, VS + d * q[1]);
            st(a.WS + t, WS + d * q[2]); st(a.BS + t, BS + d * q[3]);
        } else {
            if (a.mode == PS3D_PROJ_BASE_POINT) st(a.g0base + t, g0);
            st(a.US + t, g0 * q[0]); st(a.VS + t, g0 * q[1]);
            st(a.WS + t, g0 * q[2]); st(a.BS + t, g0 * q[3]);
        }
    }
}

// out[ko][c] = sum_ki in[ki][c] * mode(ki, ko) * scale   (forward, transpose = 0)
// out[ko][c] = sum_ki in[ki][c] * mode(ko, ki) * scale   (inverse, transpose = 1)
// mode is the Fortran column-major nz x nz matrix, mode(a,b) = mode[a + nz*b].
constexpr int kVmCols = 32;
__global__ void __launch_bounds__(256) k_vert_mode(const double2* __restrict__ in, double2* __restrict__ out,
                                                   const double* __restrict__ mode, int nz, long ncol,
                                                   double scale, int transpose) {
    extern __shared__ double2 tile[];   // [nz][kVmCols]
    const long c0 = blockIdx.x * (long)kVmCols;
    const int nl = (int)min((long)kVmCols, ncol - c0);
    for (int t = threadIdx.x; t < nz * kVmCols; t += blockDim.x) {
        const int k = t / kVmCols, l = t - k * kVmCols;
        tile[t] = (l < nl) ? in[(long)k * ncol + c0 + l] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int l = threadIdx.x % kVmCols;
    const int grp = threadIdx.x / kVmCols, ngrp = blockDim.x / kVmCols;
    if (l >= nl) return;
    for (int ko = grp; ko < nz; ko += ngrp) {
        double sr = 0.0, si = 0.0;
        for (int ki = 0; ki < nz; ++ki) {
            const double m = transpose ? __ldg(mode + ko + (long)nz * ki) : __ldg(mode + ki + (long)nz * ko);
            const double2 v = tile[ki * kVmCols + l];
            sr = sr + v.x * m * scale;
            si = si + v.y * m * scale;
        }
        out[(long)ko * ncol + c0 + l] = make_double2(sr, si);
    }
}

cudaError_t launch_project(const ProjArgs& a, cudaStream_t s) {
    const long M = (long)a.nxh * a.ny * a.nz;
    const int blocks = (int)std::min<long>((M + 255) / 256, 148L * 16);
    k_project<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_vert_mode(const double2* in, double2* out, const double* mode, int nz, long ncol,
                             double scale, int transpose, cudaStream_t s) {
    const size_t sm = (size_t)nz * kVmCols * sizeof(double2);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_vert_mode, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_done = true;
    }
    const int blocks = (int)((ncol + kVmCols - 1) / kVmCols);
    k_vert_mode<<<blocks, 256, sm, s>>>(in, out, mode, nz, ncol, scale, transpose);
    return cudaGetLastError();
}

}  // namespace ps3d
