// eigen.cuh — the normal-mode eigenvectors of the linearised operator on the
// device (eigenvectors.f90:6-218, dispatched by diag_balance.f90:366-418),
// rebuilt per spectral point from 1D per-axis tables; shared by the
// projections (modes.cu) and the Warn-et-al. balance (warn.cu).  The
// arithmetic follows eigenvectors.f90 operation for operation.
#pragma once
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
static __device__ double omega2_vbc(const Ax& x, const Ax& y, double sarg, double carg, const Phys& P) {
    const double k2 = x.hk + y.hk;
    const double m2 = 4 * (sarg * sarg) / (P.dz * P.dz);
    const double N2_hat = (P.N0 * P.N0) * (carg * carg);
    const double f2_hat = (P.f0 * P.f0) * x.ep * y.ep;
    const double Ksqr = P.dsqr * k2 + m2;
    return Ksqr > 0.0 ? (N2_hat * k2 + f2_hat * m2) / Ksqr : 0.0;
}
static __device__ void vec_qp_vbc(const Ax& x, const Ax& y, double kz, double sarg, double carg, double s, const Phys& P,
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
static __device__ void vec_qp_discrete(const Ax& x, const Ax& y, const Ax& z, double s, const Phys& P, cz_t* q, cz_t* p) {
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


// omega2_discrete (eigenvectors.f90:110-218 dispatch, triply periodic)
static __device__ double omega2_discrete(const Ax& x, const Ax& y, const Ax& z, const Phys& P) {
    const double k2 = x.hk + y.hk;
    const double Ksqr = P.dsqr * k2 + z.hk;
    return Ksqr > 0.0 ? (z.ep * (P.N0 * P.N0) * k2 + (P.f0 * P.f0) * z.hk * x.ep * y.ep) / Ksqr : 0.0;
}

}  // namespace ps3d
