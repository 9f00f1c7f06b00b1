/*
 * ps3d_oracle.cpp — TEST INFRASTRUCTURE, not the product.
 *
 * A CPU, FP64, loop-for-loop restatement of the ceden/ps3D hot path, used only
 * to check the CUDA engine's results, by tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py.  Nothing in the shipped library links or calls this file.
 *
 * Parity status: the reference itself cannot be built here (Fortran, MPI,
 * P3DFFT, FFTW and netCDF are absent) and ships no tests or golden vectors,
 * so this restatement is checked only against the reference's mathematics
 * (known-answer tests in tests/test_oracle.py) and numpy.fft: parity with
 * the reference binary is UNPINNED.
 *
 * Layout follows for_src/main_module.f90:112-144: every real field carries two
 * halo points on each side, Fortran bounds (1-2:n+2) in each direction, x
 * fastest.  Spectral arrays are (nx/2+1, ny, nz) complex, kx fastest, as the
 * reference indexes FS(i,j,k) with kx(i), ky(j), kz(k) (my_fft.f90:21-23).
 * Expressions keep the reference's operand order so that the arithmetic
 * matches a non-FMA gfortran build term for term (compile with
 * -ffp-contract=off).
 *
 * The FFT is written here (P3DFFT/FFTW are not available): an iterative
 * Stockham autosort FFT with mixed radices 4, 2, 3, 5 (and a direct DFT stage
 * for any other prime factor), unnormalised, forward sign e^{-i}, as FFTW's
 * FFTW_FORWARD which P3DFFT's ftran uses.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <map>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/ps3d_gpu.h"

namespace {

/* ------------------------------------------------------------------------ */
/* complex arithmetic in the form gfortran emits without FMA                */
/* ------------------------------------------------------------------------ */
struct cx { double re, im; };
static inline cx C(double r, double i) { return cx{r, i}; }
static inline cx operator+(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx operator-(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static inline cx operator-(cx a) { return C(-a.re, -a.im); }
static inline cx operator*(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx operator*(cx a, double s) { return C(a.re * s, a.im * s); }
static inline cx operator*(double s, cx a) { return C(s * a.re, s * a.im); }
static inline cx operator/(cx a, double s) { return C(a.re / s, a.im / s); }
/* Smith's division (range-reduced, as -fcx-fortran-rules) */
static inline cx operator/(cx a, cx b) {
    if (std::fabs(b.re) >= std::fabs(b.im)) {
        double r = b.im / b.re, d = b.re + b.im * r;
        return C((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    } else {
        double r = b.re / b.im, d = b.im + b.re * r;
        return C((a.re * r + a.im) / d, (a.im * r - a.re) / d);
    }
}
static inline cx conjg(cx a) { return C(a.re, -a.im); }
static inline cx cexpi(double x) { return C(std::cos(x), std::sin(x)); }
static const cx IM = {0.0, 1.0};

/* ------------------------------------------------------------------------ */
/* FFT                                                                       */
/* ------------------------------------------------------------------------ */
/* exp(sign * 2 pi i t / n) with octant reduction in long double, so that
 * exact values (0, +-1, +-sqrt(1/2)) come out exact.                         */
static cx twiddle(long t, long n, int sign) {
    t %= n; if (t < 0) t += n;
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
    double c, s;
    if ((8 * t) % n == 0) {
        long o = (8 * t) / n;  /* octant multiple of pi/4 */
        static const double r2 = 0.70710678118654752440084436210484904;
        const double cc[8] = {1, r2, 0, -r2, -1, -r2, 0, r2};
        const double ss[8] = {0, r2, 1, r2, 0, -r2, -1, -r2};
        c = cc[o]; s = ss[o];
    } else {
        c = (double)cosl(a); s = (double)sinl(a);
    }
    return C(c, sign < 0 ? -s : s);
}

struct Plan {
    int n = 0;
    std::vector<int> radices;
    std::vector<cx> twf, twb;   /* exp(-+2 pi i t/n), t = 0..n-1 */
};

static std::vector<int> factorise(int n) {
    std::vector<int> r;
    int m = n;
    while (m % 4 == 0) { r.push_back(4); m /= 4; }
    while (m % 2 == 0) { r.push_back(2); m /= 2; }
    while (m % 3 == 0) { r.push_back(3); m /= 3; }
    while (m % 5 == 0) { r.push_back(5); m /= 5; }
    for (int p = 7; m > 1; p += 2) while (m % p == 0) { r.push_back(p); m /= p; }
    return r;
}

static const Plan& get_plan(int n) {
    static std::map<int, Plan> cache;
    const Plan* out = nullptr;
    #pragma omp critical(ps3d_oracle_plan)
    {
        auto it = cache.find(n);
        if (it == cache.end()) {
            Plan p; p.n = n; p.radices = factorise(n);
            p.twf.resize(n); p.twb.resize(n);
            for (int t = 0; t < n; ++t) { p.twf[t] = twiddle(t, n, -1); p.twb[t] = twiddle(t, n, +1); }
            it = cache.emplace(n, std::move(p)).first;
        }
        out = &it->second;
    }
    return *out;
}

/* Stockham autosort, mixed radix: in x (length n), scratch y; result in x. */
static void fft1d(const Plan& P, cx* x, cx* y, int sign) {
    const int n = P.n;
    if (n <= 1) return;
    const cx* tw = sign < 0 ? P.twf.data() : P.twb.data();
    cx* a = x; cx* b = y;
    int Ns = 1;
    cx v[64], o[64];
    for (int R : P.radices) {
        const int stride = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < n / R; ++j) {
            const int jm = j % Ns;
            for (int r = 0; r < R; ++r) {
                cx t = a[j + r * stride];
                v[r] = (r == 0 || jm == 0) ? t : t * tw[((long)r * jm * tstep) % n];
            }
            for (int k = 0; k < R; ++k) {
                cx s = v[0];
                for (int r = 1; r < R; ++r) s = s + v[r] * tw[(long)((r * k) % R) * stride];
                o[k] = s;
            }
            const int idxD = (j / Ns) * Ns * R + jm;
            for (int k = 0; k < R; ++k) b[idxD + k * Ns] = o[k];
        }
        std::swap(a, b);
        Ns *= R;
    }
    if (a != x) std::memcpy(x, a, sizeof(cx) * n);
}

/* ------------------------------------------------------------------------ */
/* the model                                                                 */
/* ------------------------------------------------------------------------ */
struct Model {
    ps3d_params P;
    int nx, ny, nz, nxh;
    long sy, sz, n3;
    bool rigid;
    double pi;
    std::vector<double> u, v, w, b, p;
    std::vector<double> du[3], dv[3], dw[3], db[3];
    std::vector<double> flux_east, flux_north, flux_top;
    int itt = 0, tau = 3, taum1 = 2, taum2 = 1;
    double time = 0.0;
    std::vector<double> kx, ky, kz, ksqr, psi, phi, psib;
    std::vector<cx> FS;
    /* balance work space */
    std::vector<cx> US, VS, WS, BS, g0_base;
    std::vector<double> u_bal, v_bal, w_bal, b_bal, u_base, v_base, w_base, b_base;
    std::vector<double> u0, v0, w0, b0;
    std::vector<double> u_save, v_save, w_save, b_save, u_ave, v_ave, w_ave, b_ave;
    /* Warn-et-al. balance (module_diag_balance, diag_balance.f90:3-24) */
    std::vector<double> u1, v1, w1, b1, u2, v2, w2, b2, u3, v3, w3, b3, pTu0, pTv0, pTw0, pTb0;
    std::vector<cx> f1p, f1m, I_00, I_0p, I_0m, I_f1p, I_f1m, I_0f1p, I_0f1m, I_pT0p, I_pT0m;
    std::vector<cx> f2p, f2m, I_f2p, I_f2m, I_0f2p, I_0f2m, pTf2p, pTf2m;
    bool balance_filter = false;   /* enable_diag_balance_filter (main_module.f90:22) */
    int balance_filter_width = 3;  /* diag_balance_filter_width  (main_module.f90:23) */
    /* forcing */
    int force_kind = 0;
    double omega = 0.0;
    std::vector<double> fr[4], fi[4], u_back, b_back;
    bool has_fr[4] = {false, false, false, false}, has_fi[4] = {false, false, false, false};

    inline long I(int i, int j, int k) const { return (long)(i + 1) + sy * (j + 1) + sz * (k + 1); }
    inline long S(int i, int j, int k) const { return (long)(i - 1) + (long)nxh * ((j - 1) + (long)ny * (k - 1)); }
    long nspec() const { return (long)nxh * ny * nz; }
};

/* ---- parallel_mpi.f90:70-211, single-rank branches ---------------------- */
static void border_exchg_in_x(Model& M, double* a) {
    #pragma omp parallel for
    for (int k = -1; k <= M.nz + 2; ++k)
        for (int j = -1; j <= M.ny + 2; ++j)
            for (int i = 1; i <= 2; ++i) {
                a[M.I(M.nx + i, j, k)] = a[M.I(i, j, k)];
                a[M.I(1 - i, j, k)] = a[M.I(M.nx - i + 1, j, k)];
            }
}
static void border_exchg_in_y(Model& M, double* a) {
    #pragma omp parallel for
    for (int k = -1; k <= M.nz + 2; ++k)
        for (int jj = 1; jj <= 2; ++jj)
            for (int i = -1; i <= M.nx + 2; ++i) {
                a[M.I(i, M.ny + jj, k)] = a[M.I(i, jj, k)];
                a[M.I(i, 1 - jj, k)] = a[M.I(i, M.ny - jj + 1, k)];
            }
}
static void border_exchg_in_z(Model& M, double* a) {
    for (int kk = 1; kk <= 2; ++kk) {
        #pragma omp parallel for
        for (int j = -1; j <= M.ny + 2; ++j)
            for (int i = -1; i <= M.nx + 2; ++i) {
                a[M.I(i, j, M.nz + kk)] = a[M.I(i, j, kk)];
                a[M.I(i, j, 1 - kk)] = a[M.I(i, j, M.nz - kk + 1)];
            }
    }
}
static void border_exchg_3D(Model& M, double* a) {
    border_exchg_in_z(M, a);
    border_exchg_in_y(M, a);
    border_exchg_in_x(M, a);
}

/* ---- FFT wrappers: my_fft.f90:159-205 (P3DFFT 'ffn'/'nff'/'fft') -------- */
/* QP: interior real array nx*ny*nz (x fastest), QS: spectral nxh*ny*nz.     */
static void fft_r2c_x(Model& M, const double* QP, cx* QS) {
    const int nx = M.nx, ny = M.ny, nz = M.nz, nxh = M.nxh;
    const Plan& P = get_plan(nx);
    #pragma omp parallel
    {
        std::vector<cx> row(nx), tmp(nx);
        #pragma omp for collapse(2)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
                for (int i = 0; i < nx; ++i) row[i] = C(QP[i + (long)nx * (j + (long)ny * k)], 0.0);
                fft1d(P, row.data(), tmp.data(), -1);
                for (int i = 0; i < nxh; ++i) QS[i + (long)nxh * (j + (long)ny * k)] = row[i];
            }
    }
}
static void fft_c2r_x(Model& M, const cx* QS, double* QP) {
    const int nx = M.nx, ny = M.ny, nz = M.nz, nxh = M.nxh;
    const Plan& P = get_plan(nx);
    #pragma omp parallel
    {
        std::vector<cx> row(nx), tmp(nx);
        #pragma omp for collapse(2)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
                const cx* h = QS + (long)nxh * (j + (long)ny * k);
                row[0] = C(h[0].re, 0.0);
                if (nx > 1) row[nx / 2] = C(h[nx / 2].re, 0.0);
                for (int i = 1; i < nx / 2; ++i) { row[i] = h[i]; row[nx - i] = conjg(h[i]); }
                fft1d(P, row.data(), tmp.data(), +1);
                for (int i = 0; i < nx; ++i) QP[i + (long)nx * (j + (long)ny * k)] = row[i].re;
            }
    }
}
static void fft_c2c_y(Model& M, cx* QS, int sign) {
    const int ny = M.ny, nz = M.nz, nxh = M.nxh;
    const Plan& P = get_plan(ny);
    #pragma omp parallel
    {
        std::vector<cx> col(ny), tmp(ny);
        #pragma omp for collapse(2)
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nxh; ++i) {
                for (int j = 0; j < ny; ++j) col[j] = QS[i + (long)nxh * (j + (long)ny * k)];
                fft1d(P, col.data(), tmp.data(), sign);
                for (int j = 0; j < ny; ++j) QS[i + (long)nxh * (j + (long)ny * k)] = col[j];
            }
    }
}
static void fft_c2c_z(Model& M, cx* QS, int sign) {
    const int ny = M.ny, nz = M.nz, nxh = M.nxh;
    const long plane = (long)nxh * ny;
    const Plan& P = get_plan(nz);
    #pragma omp parallel
    {
        std::vector<cx> col(nz), tmp(nz);
        #pragma omp for collapse(2)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nxh; ++i) {
                for (int k = 0; k < nz; ++k) col[k] = QS[i + (long)nxh * j + plane * k];
                fft1d(P, col.data(), tmp.data(), sign);
                for (int k = 0; k < nz; ++k) QS[i + (long)nxh * j + plane * k] = col[k];
            }
    }
}
/* my_fft_2D (my_fft.f90:170-178): 'ffn' then QS = QS*dx*dy */
static void my_fft_2D(Model& M, const double* QP, cx* QS) {
    fft_r2c_x(M, QP, QS);
    fft_c2c_y(M, QS, -1);
    const long n = M.nspec();
    for (long t = 0; t < n; ++t) QS[t] = QS[t] * M.P.dx * M.P.dy;
}
/* my_ifft_2D (my_fft.f90:159-167): 'nff' then QP = QP/(Lx*Ly) */
static void my_ifft_2D(Model& M, cx* QS_in, double* QP) {
    std::vector<cx> QS(QS_in, QS_in + M.nspec());  /* P3DFFT btran does not overwrite (overwrite=.false.) */
    fft_c2c_y(M, QS.data(), +1);
    fft_c2r_x(M, QS.data(), QP);
    const long n = (long)M.nx * M.ny * M.nz;
    const double L = M.P.Lx * M.P.Ly;
    for (long t = 0; t < n; ++t) QP[t] = QP[t] / L;
}
/* my_fft_3D (my_fft.f90:197-205): 'fft' then QS = QS*dx*dy*dz */
static void my_fft_3D(Model& M, const double* QP, cx* QS) {
    fft_r2c_x(M, QP, QS);
    fft_c2c_y(M, QS, -1);
    fft_c2c_z(M, QS, -1);
    const long n = M.nspec();
    for (long t = 0; t < n; ++t) QS[t] = QS[t] * M.P.dx * M.P.dy * M.P.dz;
}
/* my_ifft_3D (my_fft.f90:184-192) */
static void my_ifft_3D(Model& M, cx* QS_in, double* QP) {
    std::vector<cx> QS(QS_in, QS_in + M.nspec());
    fft_c2c_z(M, QS.data(), +1);
    fft_c2c_y(M, QS.data(), +1);
    fft_c2r_x(M, QS.data(), QP);
    const long n = (long)M.nx * M.ny * M.nz;
    const double L = M.P.Lx * M.P.Ly * M.P.Lz;
    for (long t = 0; t < n; ++t) QP[t] = QP[t] / L;
}
/* my_fft_vert_mode (my_fft.f90:234-252) */
static void my_fft_vert_mode(Model& M, const double* QP, cx* QS, const std::vector<double>& mode) {
    const int nz = M.nz; const long plane = (long)M.nxh * M.ny;
    std::vector<cx> Qloc(M.nspec());
    fft_r2c_x(M, QP, Qloc.data());
    fft_c2c_y(M, Qloc.data(), -1);
    for (long t = 0; t < M.nspec(); ++t) Qloc[t] = Qloc[t] * M.P.dx * M.P.dy;
    #pragma omp parallel for
    for (long c = 0; c < plane; ++c)
        for (int k1 = 1; k1 <= nz; ++k1) {
            cx s = C(0.0, 0.0);
            for (int k2 = 1; k2 <= nz; ++k2)
                s = s + Qloc[c + plane * (k2 - 1)] * mode[(k2 - 1) + (long)nz * (k1 - 1)] * M.P.dz;
            QS[c + plane * (k1 - 1)] = s;
        }
}
/* my_ifft_vert_mode (my_fft.f90:211-229) */
static void my_ifft_vert_mode(Model& M, const cx* QS, double* QP, const std::vector<double>& mode) {
    const int nz = M.nz; const long plane = (long)M.nxh * M.ny;
    std::vector<cx> Qloc(M.nspec());
    #pragma omp parallel for
    for (long c = 0; c < plane; ++c)
        for (int k2 = 1; k2 <= nz; ++k2) {
            cx s = C(0.0, 0.0);
            for (int k1 = 1; k1 <= nz; ++k1)
                s = s + QS[c + plane * (k1 - 1)] * mode[(k2 - 1) + (long)nz * (k1 - 1)];
            Qloc[c + plane * (k2 - 1)] = s;
        }
    fft_c2c_y(M, Qloc.data(), +1);
    fft_c2r_x(M, Qloc.data(), QP);
    const long n = (long)M.nx * M.ny * M.nz;
    const double L = M.P.Lx * M.P.Ly;
    for (long t = 0; t < n; ++t) QP[t] = QP[t] / L;
}

/* ---- eigenvectors.f90:224-268 helpers ----------------------------------- */
static inline double hat_ksqr(double k, double dx) { return 2.0 * (1.0 - std::cos(k * dx)) / (dx * dx); }
static inline double hat_epm(double k, double dx) { return 0.5 * (1 + std::cos(k * dx)); }
static inline cx hat_kp(double k, double dx) { return -(IM * (cexpi(k * dx) - C(1.0, 0.0)) / dx); }
static inline cx hat_ep(double k, double dx) { return (cexpi(k * dx) + C(1.0, 0.0)) * 0.5; }
static inline cx hat_em(double k, double dx) { return (cexpi(-k * dx) + C(1.0, 0.0)) * 0.5; }

/* ---- eigenvectors.f90:6-104, rigid lid ----------------------------------- */
static double omega2_vbc(double kx, double ky, double kz, const ps3d_params& P) {
    double arg = kz / 2 * P.dz;
    double k2 = hat_ksqr(kx, P.dx) + hat_ksqr(ky, P.dy);
    double s_ = std::sin(arg), c_ = std::cos(arg);
    double m2 = 4 * (s_ * s_) / (P.dz * P.dz);
    double N2_hat = (P.N0 * P.N0) * (c_ * c_);
    double f2_hat = (P.f0 * P.f0) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy);
    double Ksqr = P.dsqr * k2 + m2;
    if (Ksqr > 0.0) return (N2_hat * k2 + f2_hat * m2) / Ksqr;
    return 0.0;
}
static double coeff_p_vbc(double kx, double ky, double kz, double s, const ps3d_params& P) {
    double arg = kz / 2 * P.dz;
    double om2 = omega2_vbc(kx, ky, kz, P);
    double k2 = hat_ksqr(kx, P.dx) + hat_ksqr(ky, P.dy);
    double s_ = std::sin(arg), c_ = std::cos(arg);
    double m2 = 4 * (s_ * s_) / (P.dz * P.dz);
    double f2_hat = (P.f0 * P.f0) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy);
    double N2_hat = (P.N0 * P.N0) * (c_ * c_);
    double d = k2 * N2_hat + f2_hat * m2;
    if (s == 0.0 && d > 0.0) return f2_hat * N2_hat / d;
    if (d > 0.0) return (N2_hat - P.dsqr * om2) * (om2 - f2_hat) / (2 * d);
    return 0.0;
}
static void vec_q_vbc(double kx, double ky, double kz, double s, const ps3d_params& P,
                      cx& qx, cx& qy, cx& qz, cx& qb) {
    double arg = kz / 2 * P.dz;
    double om2 = omega2_vbc(kx, ky, kz, P);
    double om = std::sqrt(om2);
    double f2_hat = (P.f0 * P.f0) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy);
    double c_ = std::cos(arg);
    double N2_hat = (P.N0 * P.N0) * (c_ * c_);
    double lam = 2 * std::sin(arg) / P.dz;
    if (kx * kx + ky * ky > 0.0) {
        double fxa = f2_hat - (s * s) * om2;
        qx = (-(IM * P.f0 * hat_ep(kx, P.dx) * hat_em(ky, P.dy) * hat_kp(ky, P.dy)) + s * om * hat_kp(kx, P.dx)) / fxa;
        qy = ((IM * P.f0 * hat_em(kx, P.dx) * hat_ep(ky, P.dy) * hat_kp(kx, P.dx)) + s * om * hat_kp(ky, P.dy)) / fxa;
        if (kz * kz > 0.0) {
            fxa = N2_hat - P.dsqr * (s * s) * om2;
            qz = IM * lam * s * om / fxa;
            qb = C(-(lam * std::cos(arg) * (P.N0 * P.N0) / fxa), 0.0);
        } else { qz = C(0, 0); qb = C(0, 0); }
    } else {
        qx = -(IM * s);
        qy = C(s * s, 0.0);
        qz = C(0, 0); qb = C(0, 0);
    }
    if (s == 0.0 && (f2_hat == 0.0 || N2_hat == 0.0)) { qx = qy = qz = qb = C(0, 0); }
    if (s != 0.0 && om2 == 0.0) { qx = qy = qz = qb = C(0, 0); }
}
static void vec_p_vbc(double kx, double ky, double kz, double s, const ps3d_params& P,
                      cx& px, cx& py, cx& pz, cx& pb) {
    double p = coeff_p_vbc(kx, ky, kz, s, P);
    vec_q_vbc(kx, ky, kz, s, P, px, py, pz, pb);
    px = p * conjg(px);
    py = p * conjg(py);
    pz = p * conjg(pz) * P.dsqr;
    pb = p * conjg(pb) / (P.N0 * P.N0);
}

/* ---- eigenvectors.f90:110-218, triply periodic --------------------------- */
static double omega2_discrete(double kx, double ky, double kz, const ps3d_params& P) {
    double k2 = hat_ksqr(kx, P.dx) + hat_ksqr(ky, P.dy);
    double Ksqr = P.dsqr * k2 + hat_ksqr(kz, P.dz);
    if (Ksqr > 0.0)
        return (hat_epm(kz, P.dz) * (P.N0 * P.N0) * k2 +
                (P.f0 * P.f0) * hat_ksqr(kz, P.dz) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy)) / Ksqr;
    return 0.0;
}
static double coeff_p_discrete(double kx, double ky, double kz, double s, const ps3d_params& P) {
    double om2 = omega2_discrete(kx, ky, kz, P);
    double k2 = hat_ksqr(kx, P.dx) + hat_ksqr(ky, P.dy);
    double f2_hat = (P.f0 * P.f0) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy);
    double N2_hat = (P.N0 * P.N0) * hat_epm(kz, P.dz);
    double d = k2 * N2_hat + f2_hat * hat_ksqr(kz, P.dz);
    if (s == 0.0 && d > 0.0) return f2_hat * N2_hat / d;
    if (d > 0.0) return (N2_hat - P.dsqr * om2) * (om2 - f2_hat) / (2 * d);
    return 0.0;
}
static void vec_q_discrete(double kx, double ky, double kz, double s, const ps3d_params& P,
                           cx& qx, cx& qy, cx& qz, cx& qb) {
    double om2 = omega2_discrete(kx, ky, kz, P);
    double om = std::sqrt(om2);
    double f2_hat = (P.f0 * P.f0) * hat_epm(kx, P.dx) * hat_epm(ky, P.dy);
    double N2_hat = (P.N0 * P.N0) * hat_epm(kz, P.dz);
    if (kx * kx + ky * ky > 0.0) {
        double fxa = f2_hat - (s * s) * om2;
        qx = (-(IM * P.f0 * hat_ep(kx, P.dx) * hat_em(ky, P.dy) * hat_kp(ky, P.dy)) + s * om * hat_kp(kx, P.dx)) / fxa;
        qy = ((IM * P.f0 * hat_em(kx, P.dx) * hat_ep(ky, P.dy) * hat_kp(kx, P.dx)) + s * om * hat_kp(ky, P.dy)) / fxa;
        if (kz * kz > 0.0) {
            fxa = N2_hat - P.dsqr * (s * s) * om2;
            qz = hat_kp(kz, P.dz) * s * om / fxa;
            qb = IM * hat_em(kz, P.dz) * hat_kp(kz, P.dz) * (P.N0 * P.N0) / fxa;
        } else { qz = C(0, 0); qb = C(0, 0); }
    } else {
        qx = -(IM * s);
        qy = C(s * s, 0.0);
        qz = C(0, 0); qb = C(0, 0);
    }
    if (s == 0.0 && (f2_hat == 0.0 || N2_hat == 0.0)) { qx = qy = qz = qb = C(0, 0); }
    if (s != 0.0 && om2 == 0.0) { qx = qy = qz = qb = C(0, 0); }
    if ((kx * kx + ky * ky > 0.0) && (kz * kz == 0.0) && (s != 0.0)) {
        qx = C(0, 0); qy = C(0, 0);
        qz = IM * s;
        qb = C((s * s) * P.N0 * std::sqrt(P.dsqr), 0.0);
    }
}
static void vec_p_discrete(double kx, double ky, double kz, double s, const ps3d_params& P,
                           cx& px, cx& py, cx& pz, cx& pb) {
    double p = coeff_p_discrete(kx, ky, kz, s, P);
    vec_q_discrete(kx, ky, kz, s, P, px, py, pz, pb);
    px = p * conjg(px);
    py = p * conjg(py);
    pz = p * conjg(pz) * P.dsqr;
    pb = p * conjg(pb) / (P.N0 * P.N0);
    if ((kx * kx + ky * ky == 0.0) && (kz * kz > 0.0)) {
        px = IM * s / 2.0; py = C((s * s) / 2.0, 0.0);
    }
    if ((kx * kx + ky * ky > 0.0) && (kz * kz == 0.0) && (s != 0.0)) {
        px = C(0, 0); py = C(0, 0);
        pz = -(IM * s / 2.0);
        pb = C((s * s) / (2.0 * P.N0 * std::sqrt(P.dsqr)), 0.0);
    }
}
/* dispatchers, diag_balance.f90:366-418 */
static void vec_q(const Model& M, double kx, double ky, double kz, double s, cx& a, cx& b, cx& c, cx& d) {
    if (M.rigid) vec_q_vbc(kx, ky, kz, s, M.P, a, b, c, d); else vec_q_discrete(kx, ky, kz, s, M.P, a, b, c, d);
}
static void vec_p(const Model& M, double kx, double ky, double kz, double s, cx& a, cx& b, cx& c, cx& d) {
    if (M.rigid) vec_p_vbc(kx, ky, kz, s, M.P, a, b, c, d); else vec_p_discrete(kx, ky, kz, s, M.P, a, b, c, d);
}
static double omega2(const Model& M, double kx, double ky, double kz) {
    return M.rigid ? omega2_vbc(kx, ky, kz, M.P) : omega2_discrete(kx, ky, kz, M.P);
}

/* ---- wavenumber_initialisation, my_fft.f90:87-156 ----------------------- */
static void wavenumber_initialisation(Model& M) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    const double pi = M.pi;
    M.kx.assign(nx / 2 + 1, 0.0); M.ky.assign(ny, 0.0); M.kz.assign(nz, 0.0);
    for (int i = 1; i <= nx / 2 + 1; ++i) M.kx[i - 1] = 2 * (i - 1) * pi / M.P.Lx;
    for (int j = 1; j <= (ny + 1) / 2; ++j) M.ky[j - 1] = 2 * (j - 1) * pi / M.P.Ly;
    for (int j = (ny + 1) / 2 + 1; j <= ny; ++j) M.ky[j - 1] = -(2 * (ny - j + 1) * pi / M.P.Ly);
    if (M.rigid) {
        for (int k = 1; k <= nz; ++k) M.kz[k - 1] = (double)(k - 1) * pi / M.P.Lz;
        M.psi.assign((long)nz * nz, 0.0); M.phi.assign((long)nz * nz, 0.0); M.psib.assign((long)nz * nz, 0.0);
        auto A = [nz](std::vector<double>& m, int k, int k2) -> double& { return m[(k - 1) + (long)nz * (k2 - 1)]; };
        for (int k = 1; k <= nz; ++k) { A(M.phi, k, 1) = std::sqrt(1.0 / M.P.Lz); A(M.psi, k, 1) = 0.0; A(M.psib, k, 1) = 0.0; }
        for (int k2 = 2; k2 <= nz; ++k2) {
            for (int k = 1; k <= nz; ++k) A(M.psi, k, k2) = std::sqrt(2.0 / M.P.Lz) * std::sin((k2 - 1) * k * pi / nz);
            const double sd = 2 * std::sin((k2 - 1) * pi / (2 * nz));
            const double cd = 2 * std::cos((k2 - 1) * pi / (2 * nz));
            A(M.phi, 1, k2) = A(M.psi, 1, k2) / sd;
            A(M.psib, 1, k2) = A(M.psi, 1, k2) / cd;
            for (int k = 2; k <= nz; ++k) {
                A(M.phi, k, k2) = (A(M.psi, k, k2) - A(M.psi, k - 1, k2)) / sd;
                A(M.psib, k, k2) = (A(M.psi, k, k2) + A(M.psi, k - 1, k2)) / cd;
            }
        }
        M.ksqr.assign((long)M.nxh * ny, 0.0);
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= M.nxh; ++i)
                M.ksqr[(i - 1) + (long)M.nxh * (j - 1)] = hat_ksqr(M.kx[i - 1], M.P.dx) + hat_ksqr(M.ky[j - 1], M.P.dy);
    } else {
        for (int k = 1; k <= (nz + 1) / 2; ++k) M.kz[k - 1] = 2 * (k - 1) * pi / M.P.Lz;
        for (int k = (nz + 1) / 2 + 1; k <= nz; ++k) M.kz[k - 1] = -(2 * (nz - k + 1) * pi / M.P.Lz);
        M.ksqr.assign(M.nspec(), 0.0);
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= M.nxh; ++i)
                    M.ksqr[M.S(i, j, k)] = hat_ksqr(M.kx[i - 1], M.P.dx) + hat_ksqr(M.ky[j - 1], M.P.dy) +
                                           hat_ksqr(M.kz[k - 1], M.P.dz) / M.P.dsqr;
    }
}

/* ---- advection.f90:2-48 -------------------------------------------------- */
static void buoyancy_advection_2nd(Model& M, double* db_loc) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    const double *u = M.u.data(), *v = M.v.data(), *w = M.w.data(), *b = M.b.data();
    double *fe = M.flux_east.data(), *fn = M.flux_north.data(), *ft = M.flux_top.data();
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i)
                fe[M.I(i, j, k)] = 0.5 * (b[M.I(i, j, k)] + b[M.I(i + 1, j, k)]) * u[M.I(i, j, k)];
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                fn[M.I(i, j, k)] = 0.5 * (b[M.I(i, j, k)] + b[M.I(i, j + 1, k)]) * v[M.I(i, j, k)];
    #pragma omp parallel for
    for (int k = 0; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                ft[M.I(i, j, k)] = 0.5 * (b[M.I(i, j, k)] + b[M.I(i, j, k + 1)]) * w[M.I(i, j, k)];
    if (M.rigid) {
        for (int k = -1; k <= 0; ++k) std::fill(ft + M.I(-1, -1, k), ft + M.I(-1, -1, k) + M.sz, 0.0);
        for (int k = nz; k <= nz + 2; ++k) std::fill(ft + M.I(-1, -1, k), ft + M.I(-1, -1, k) + M.sz, 0.0);
    }
    const double Ro = M.P.Ro, dx = M.P.dx, dy = M.P.dy, dz = M.P.dz;
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                db_loc[M.I(i, j, k)] = -Ro * ((fe[M.I(i, j, k)] - fe[M.I(i - 1, j, k)]) / dx +
                                              (fn[M.I(i, j, k)] - fn[M.I(i, j - 1, k)]) / dy +
                                              (ft[M.I(i, j, k)] - ft[M.I(i, j, k - 1)]) / dz);
}

/* ---- advection.f90:53-184 ------------------------------------------------ */
static void zero_planes(Model& M, double* a, int k0, int k1) {
    for (int k = k0; k <= k1; ++k) std::fill(a + M.I(-1, -1, k), a + M.I(-1, -1, k) + M.sz, 0.0);
}
static void momentum_advection_2nd(Model& M, double* du_loc, double* dv_loc, double* dw_loc) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    const double *u = M.u.data(), *v = M.v.data(), *w = M.w.data();
    double *fe = M.flux_east.data(), *fn = M.flux_north.data(), *ft = M.flux_top.data();
    const double Ro = M.P.Ro, dx = M.P.dx, dy = M.P.dy, dz = M.P.dz, dsqr = M.P.dsqr;
#define U(i, j, k) u[M.I(i, j, k)]
#define V(i, j, k) v[M.I(i, j, k)]
#define W(i, j, k) w[M.I(i, j, k)]
#define FE(i, j, k) fe[M.I(i, j, k)]
#define FN(i, j, k) fn[M.I(i, j, k)]
#define FT(i, j, k) ft[M.I(i, j, k)]
    /* zonal momentum */
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 0; i <= nx; ++i)
        FE(i, j, k) = 0.25 * (U(i, j, k) + U(i + 1, j, k)) * (U(i + 1, j, k) + U(i, j, k));
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 0; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FN(i, j, k) = 0.25 * (U(i, j, k) + U(i, j + 1, k)) * (V(i + 1, j, k) + V(i, j, k));
    #pragma omp parallel for
    for (int k = 0; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FT(i, j, k) = 0.25 * (U(i, j, k + 1) + U(i, j, k)) * (W(i, j, k) + W(i + 1, j, k));
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        du_loc[M.I(i, j, k)] = -Ro * ((FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                      (FT(i, j, k) - FT(i, j, k - 1)) / dz);
    /* meridional momentum */
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 0; i <= nx; ++i)
        FE(i, j, k) = 0.25 * (V(i, j, k) + V(i + 1, j, k)) * (U(i, j + 1, k) + U(i, j, k));
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 0; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FN(i, j, k) = 0.25 * (V(i, j, k) + V(i, j + 1, k)) * (V(i, j + 1, k) + V(i, j, k));
    #pragma omp parallel for
    for (int k = 0; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FT(i, j, k) = 0.25 * (V(i, j, k + 1) + V(i, j, k)) * (W(i, j, k) + W(i, j + 1, k));
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        dv_loc[M.I(i, j, k)] = -Ro * ((FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                      (FT(i, j, k) - FT(i, j, k - 1)) / dz);
    /* vertical momentum */
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 0; i <= nx; ++i)
        FE(i, j, k) = 0.25 * (W(i, j, k) + W(i + 1, j, k)) * (U(i, j, k) + U(i, j, k + 1));
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 0; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FN(i, j, k) = 0.25 * (W(i, j, k) + W(i, j + 1, k)) * (V(i, j, k) + V(i, j, k + 1));
    #pragma omp parallel for
    for (int k = 0; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FT(i, j, k) = 0.25 * (W(i, j, k + 1) + W(i, j, k)) * (W(i, j, k) + W(i, j, k + 1));
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz - 1, nz + 2); }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        dw_loc[M.I(i, j, k)] = -dsqr * Ro * ((FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                             (FT(i, j, k) - FT(i, j, k - 1)) / dz);
}

/* ---- mixing.f90:225-274 (harmonic), in place ----------------------------- */
static void harmonic(Model& M, double* p1, double Hmix, double Vmix) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    double *fe = M.flux_east.data(), *fn = M.flux_north.data(), *ft = M.flux_top.data();
    const double dx = M.P.dx, dy = M.P.dy, dz = M.P.dz, dt = M.P.dt;
#define P1(i, j, k) p1[M.I(i, j, k)]
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = -1; i <= nx + 1; ++i)
        FE(i, j, k) = Hmix * (P1(i + 1, j, k) - P1(i, j, k)) / dx;
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = -1; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        FN(i, j, k) = Hmix * (P1(i, j + 1, k) - P1(i, j, k)) / dy;
    #pragma omp parallel for
    for (int k = -1; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        FT(i, j, k) = Vmix * (P1(i, j, k + 1) - P1(i, j, k)) / dz;
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        P1(i, j, k) = P1(i, j, k) + dt * ((FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                          (FT(i, j, k) - FT(i, j, k - 1)) / dz);
}

/* ---- mixing.f90:96-158 (biharmonic_h), in place -------------------------- */
static void biharmonic_h(Model& M, double* p1, double Hmix) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    double *fe = M.flux_east.data(), *fn = M.flux_north.data();
    const double dx = M.P.dx, dy = M.P.dy, dt = M.P.dt;
    std::vector<double> del2v(M.n3, 0.0);
    double* del2 = del2v.data();
#define D2(i, j, k) del2[M.I(i, j, k)]
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = -1; i <= nx + 1; ++i)
        FE(i, j, k) = -Hmix * (P1(i + 1, j, k) - P1(i, j, k)) / dx;
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = -1; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        FN(i, j, k) = -Hmix * (P1(i, j + 1, k) - P1(i, j, k)) / dy;
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        D2(i, j, k) = (FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy;
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 0; i <= nx; ++i)
        FE(i, j, k) = (D2(i + 1, j, k) - D2(i, j, k)) / dx;
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 0; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FN(i, j, k) = (D2(i, j + 1, k) - D2(i, j, k)) / dy;
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        P1(i, j, k) = P1(i, j, k) + dt * ((FE(i, j, k) - FE(i - 1, j, k)) / dx + (FN(i, j, k) - FN(i, j - 1, k)) / dy);
}

/* ---- mixing.f90:164-217 (biharmonic_v), in place ------------------------- */
static void biharmonic_v(Model& M, double* p1, double Vmix) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    double* ft = M.flux_top.data();
    const double dz = M.P.dz, dt = M.P.dt;
    std::vector<double> del2v(M.n3, 0.0);
    double* del2 = del2v.data();
    #pragma omp parallel for
    for (int k = -1; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        FT(i, j, k) = -Vmix * (P1(i, j, k + 1) - P1(i, j, k)) / dz;
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
    #pragma omp parallel for
    for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i)
        D2(i, j, k) = (FT(i, j, k) - FT(i, j, k - 1)) / dz;
    #pragma omp parallel for
    for (int k = 0; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        FT(i, j, k) = (D2(i, j, k + 1) - D2(i, j, k)) / dz;
    if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        P1(i, j, k) = P1(i, j, k) + dt * ((FT(i, j, k) - FT(i, j, k - 1)) / dz);
}

/* ---- set_forcing: for_src/config.f90:224-237 and lee_wave1.f90:232-332 --- */
static void set_forcing(Model& M) {
    if (!M.force_kind) return;
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    const int tau = M.tau - 1;
    const double Ro = M.P.Ro, dx = M.P.dx, dy = M.P.dy, dz = M.P.dz, dsqr = M.P.dsqr, dt = M.P.dt;
    double *fe = M.flux_east.data(), *fn = M.flux_north.data(), *ft = M.flux_top.data();
    const double *u = M.u.data(), *v = M.v.data(), *w = M.w.data(), *b = M.b.data();
    if (M.force_kind & PS3D_FORCE_BACKGROUND) {
        const double *ub = M.u_back.data(), *bb = M.b_back.data();
#define UB(i, j, k) ub[M.I(i, j, k)]
#define BB(i, j, k) bb[M.I(i, j, k)]
        double *du = M.du[tau].data(), *dv = M.dv[tau].data(), *dw = M.dw[tau].data(), *dbt = M.db[tau].data();
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 0; i <= nx; ++i)
            FE(i, j, k) = 2 * 0.25 * (UB(i, j, k) + UB(i + 1, j, k)) * (U(i + 1, j, k) + U(i, j, k));
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = 0; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            FN(i, j, k) = 0.25 * (UB(i, j, k) + UB(i, j + 1, k)) * (V(i + 1, j, k) + V(i, j, k));
        #pragma omp parallel for
        for (int k = 0; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 1; i <= nx; ++i)
            FT(i, j, k) = 0.25 * (UB(i, j, k + 1) + UB(i, j, k)) * (W(i, j, k) + W(i + 1, j, k));
        if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            du[M.I(i, j, k)] = du[M.I(i, j, k)] - Ro * ((FE(i, j, k) - FE(i - 1, j, k)) / dx +
                                                       (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                                       (FT(i, j, k) - FT(i, j, k - 1)) / dz);
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = 1; j <= ny; ++j) for (int i = 0; i <= nx; ++i)
            FE(i, j, k) = 0.25 * (V(i, j, k) + V(i + 1, j, k)) * (UB(i, j + 1, k) + UB(i, j, k));
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 1; i <= nx; ++i)
            dv[M.I(i, j, k)] = dv[M.I(i, j, k)] - Ro * (FE(i, j, k) - FE(i - 1, j, k)) / dx;
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 0; i <= nx; ++i)
            FE(i, j, k) = 0.25 * (W(i, j, k) + W(i + 1, j, k)) * (UB(i, j, k) + UB(i, j, k + 1));
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 1; i <= nx; ++i)
            dw[M.I(i, j, k)] = dw[M.I(i, j, k)] - dsqr * Ro * (FE(i, j, k) - FE(i - 1, j, k)) / dx;
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = 0; i <= nx; ++i)
            FE(i, j, k) = 0.5 * (b[M.I(i, j, k)] + b[M.I(i + 1, j, k)]) * UB(i, j, k) +
                          0.5 * (BB(i, j, k) + BB(i + 1, j, k)) * U(i, j, k);
        #pragma omp parallel for
        for (int k = -1; k <= nz + 2; ++k) for (int j = 0; j <= ny; ++j) for (int i = -1; i <= nx + 2; ++i)
            FN(i, j, k) = 0.5 * (BB(i, j, k) + BB(i, j + 1, k)) * V(i, j, k);
        #pragma omp parallel for
        for (int k = 0; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = -1; i <= nx + 2; ++i)
            FT(i, j, k) = 0.5 * (BB(i, j, k) + BB(i, j, k + 1)) * W(i, j, k);
        if (M.rigid) { zero_planes(M, ft, -1, 0); zero_planes(M, ft, nz, nz + 2); }
        #pragma omp parallel for
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            dbt[M.I(i, j, k)] = dbt[M.I(i, j, k)] - Ro * ((FE(i, j, k) - FE(i - 1, j, k)) / dx +
                                                        (FN(i, j, k) - FN(i, j - 1, k)) / dy +
                                                        (FT(i, j, k) - FT(i, j, k - 1)) / dz);
    }
    if (M.force_kind & PS3D_FORCE_WAVEMAKER) {
        const double t = dt * M.itt;
        const double c = std::cos(M.omega * t), s = std::sin(M.omega * t);
        double* fld[4] = {M.u.data(), M.v.data(), M.w.data(), M.b.data()};
        for (int f = 0; f < 4; ++f) {
            if (!M.has_fr[f] && !M.has_fi[f]) continue;
            const double* r = M.has_fr[f] ? M.fr[f].data() : nullptr;
            const double* im = M.has_fi[f] ? M.fi[f].data() : nullptr;
            #pragma omp parallel for
            for (long t3 = 0; t3 < M.n3; ++t3)
                fld[f][t3] = fld[f][t3] + dt * (c * (r ? r[t3] : 0.0) + s * (im ? im[t3] : 0.0));
        }
        border_exchg_3D(M, M.u.data()); border_exchg_3D(M, M.v.data());
        border_exchg_3D(M, M.w.data()); border_exchg_3D(M, M.b.data());
    }
}

/* ---- solve_tridiag, pressure_solver.f90:126-162 -------------------------- */
static void solve_tridiag(const double* a, const double* bb, const double* c, const cx* d, cx* x, int n,
                          double* cp, cx* dp) {
    cp[0] = c[0] / bb[0];
    dp[0] = d[0] / bb[0];
    for (int i = 1; i < n; ++i) {
        double m = bb[i] - cp[i - 1] * a[i];
        double fxa = 1.0 / m;
        cp[i] = c[i] * fxa;
        dp[i] = (d[i] - dp[i - 1] * a[i]) * fxa;
    }
    x[n - 1] = dp[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
}

/* ---- pressure_solver.f90:2-120 ------------------------------------------- */
static void pressure_solver(Model& M) {
    const int nx = M.nx, ny = M.ny, nz = M.nz, nxh = M.nxh;
    const double dx = M.P.dx, dy = M.P.dy, dz = M.P.dz, dt = M.P.dt, dsqr = M.P.dsqr;
    double *u = M.u.data(), *v = M.v.data(), *w = M.w.data(), *p = M.p.data();
    std::vector<double> aloc((long)nx * ny * nz);
#define AL(i, j, k) aloc[(long)((i) - 1) + (long)nx * (((j) - 1) + (long)ny * ((k) - 1))]
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        AL(i, j, k) = (U(i, j, k) - U(i - 1, j, k)) / dx + (V(i, j, k) - V(i, j - 1, k)) / dy +
                      (W(i, j, k) - W(i, j, k - 1)) / dz;
    for (auto& a : aloc) a = a / dt;
    cx* FS = M.FS.data();
    const long plane = (long)nxh * ny;
    if (M.rigid) {
        my_fft_2D(M, aloc.data(), FS);
        const double fxa = 1.0 / (dz * dz) / dsqr;
        std::vector<double> a_tri(nz), c_tri(nz);
        for (int k = 2; k <= nz; ++k) a_tri[k - 1] = fxa;
        for (int k = 1; k <= nz - 1; ++k) c_tri[k - 1] = fxa;
        #pragma omp parallel
        {
            std::vector<double> b_tri(nz), cp(nz);
            std::vector<cx> col(nz), dp(nz), bloc(nz);
            #pragma omp for
            for (long c = 0; c < plane; ++c) {
                const double ks = M.ksqr[c];
                for (int k = 0; k < nz; ++k) col[k] = FS[c + plane * k];
                if (ks > 0) {
                    b_tri[0] = -ks - fxa;
                    for (int k = 2; k <= nz - 1; ++k) b_tri[k - 1] = -ks - 2 * fxa;
                    b_tri[nz - 1] = -ks - fxa;
                    solve_tridiag(a_tri.data(), b_tri.data(), c_tri.data(), col.data(), col.data(), nz,
                                  cp.data(), dp.data());
                } else {
                    for (int k = 0; k < nz; ++k) bloc[k] = col[k];
                    col[0] = C(0.0, 0.0);
                    if (nz > 1) col[1] = bloc[0] * (dz * dz) * dsqr;
                    for (int k = 2; k <= nz - 1; ++k)
                        col[k] = 2 * col[k - 1] - col[k - 2] + bloc[k - 1] * (dz * dz) * dsqr;
                }
                for (int k = 0; k < nz; ++k) FS[c + plane * k] = col[k];
            }
        }
        my_ifft_2D(M, FS, aloc.data());
    } else {
        my_fft_3D(M, aloc.data(), FS);
        const long n = M.nspec();
        #pragma omp parallel for
        for (long t = 0; t < n; ++t) {
            if (M.ksqr[t] > 0.0) FS[t] = (-FS[t]) / M.ksqr[t];
            else FS[t] = C(0.0, 0.0);
        }
        my_ifft_3D(M, FS, aloc.data());
    }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
        p[M.I(i, j, k)] = AL(i, j, k);
    border_exchg_3D(M, p);
    if (M.rigid) {
        for (int k = -1; k <= 0; ++k) std::memcpy(p + M.I(-1, -1, k), p + M.I(-1, -1, 1), sizeof(double) * M.sz);
        for (int k = nz + 1; k <= nz + 2; ++k) std::memcpy(p + M.I(-1, -1, k), p + M.I(-1, -1, nz), sizeof(double) * M.sz);
    }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        U(i, j, k) = U(i, j, k) - dt * (p[M.I(i + 1, j, k)] - p[M.I(i, j, k)]) / dx;
        V(i, j, k) = V(i, j, k) - dt * (p[M.I(i, j + 1, k)] - p[M.I(i, j, k)]) / dy;
        W(i, j, k) = W(i, j, k) - dt / dsqr * (p[M.I(i, j, k + 1)] - p[M.I(i, j, k)]) / dz;
    }
    if (M.rigid) { zero_planes(M, w, -1, 0); zero_planes(M, w, nz, nz + 2); }
    border_exchg_3D(M, u); border_exchg_3D(M, v); border_exchg_3D(M, w);
}

/* ---- integrate.f90:2-115 -------------------------------------------------- */
static void integrate(Model& M) {
    const int nx = M.nx, ny = M.ny, nz = M.nz;
    const int t0 = M.tau - 1, t1 = M.taum1 - 1, t2 = M.taum2 - 1;
    double *db = M.db[t0].data(), *du = M.du[t0].data(), *dv = M.dv[t0].data(), *dw = M.dw[t0].data();
    double *u = M.u.data(), *v = M.v.data(), *w = M.w.data(), *b = M.b.data();
    const double N0 = M.P.N0, f0 = M.P.f0;
    if (M.P.enable_nonlinear) buoyancy_advection_2nd(M, db);
    else std::fill(M.db[t0].begin(), M.db[t0].end(), 0.0);
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = -1; i <= nx + 2; ++i)
        db[M.I(i, j, k)] = db[M.I(i, j, k)] - 0.5 * (W(i, j, k) + W(i, j, k - 1)) * (N0 * N0);
    if (M.P.enable_nonlinear) momentum_advection_2nd(M, du, dv, dw);
    else {
        std::fill(M.du[t0].begin(), M.du[t0].end(), 0.0);
        std::fill(M.dv[t0].begin(), M.dv[t0].end(), 0.0);
        std::fill(M.dw[t0].begin(), M.dw[t0].end(), 0.0);
    }
    #pragma omp parallel for
    for (int k = -1; k <= nz + 2; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        du[M.I(i, j, k)] = du[M.I(i, j, k)] + (V(i, j, k) + V(i, j - 1, k) + V(i + 1, j, k) + V(i + 1, j - 1, k)) * 0.25 * f0;
        dv[M.I(i, j, k)] = dv[M.I(i, j, k)] - (U(i - 1, j, k) + U(i, j, k) + U(i - 1, j + 1, k) + U(i, j + 1, k)) * 0.25 * f0;
    }
    #pragma omp parallel for
    for (int k = 1; k <= nz; ++k) for (int j = -1; j <= ny + 2; ++j) for (int i = -1; i <= nx + 2; ++i)
        dw[M.I(i, j, k)] = dw[M.I(i, j, k)] + 0.5 * (b[M.I(i, j, k)] + b[M.I(i, j, k + 1)]);
    if (M.rigid) { zero_planes(M, dw, -1, 0); zero_planes(M, dw, nz, nz + 2); }

    const ps3d_params& P = M.P;
    if (P.Ah > 0. || P.Av > 0.) harmonic(M, u, P.Ah, P.Av);
    if (P.Ah > 0. || P.Av > 0.) harmonic(M, v, P.Ah, P.Av);
    if (P.Ah > 0. || P.Av > 0.) {
        harmonic(M, w, P.Ah, P.Av);
        if (M.rigid) zero_planes(M, w, nz, nz + 2);
    }
    if (P.Kh > 0. || P.Kv > 0.) harmonic(M, b, P.Kh, P.Kv);
    if (P.Ahbi > 0.) biharmonic_h(M, u, P.Ahbi);
    if (P.Ahbi > 0.) biharmonic_h(M, v, P.Ahbi);
    if (P.Ahbi > 0.) biharmonic_h(M, w, P.Ahbi);
    if (P.Avbi > 0.) biharmonic_v(M, u, P.Avbi);
    if (P.Avbi > 0.) biharmonic_v(M, v, P.Avbi);
    if (P.Avbi > 0.) {
        biharmonic_v(M, w, P.Avbi);
        if (M.rigid) zero_planes(M, w, nz, nz + 2);
    }
    if (P.Khbi > 0.) biharmonic_h(M, b, P.Khbi);
    if (P.Kvbi > 0.) biharmonic_v(M, b, P.Kvbi);

    set_forcing(M);

    const double dt = P.dt, dtw = P.dt / P.dsqr;
    double* fld[4] = {u, v, w, b};
    double* tt[4] = {du, dv, dw, db};
    double* t1p[4] = {M.du[t1].data(), M.dv[t1].data(), M.dw[t1].data(), M.db[t1].data()};
    double* t2p[4] = {M.du[t2].data(), M.dv[t2].data(), M.dw[t2].data(), M.db[t2].data()};
    const long n3 = M.n3;
    for (int f = 0; f < 4; ++f) {
        const double h = (f == 2) ? dtw : dt;
        double* x = fld[f]; const double *a0 = tt[f], *a1 = t1p[f], *a2 = t2p[f];
        if (M.itt == 0) {
            #pragma omp parallel for
            for (long t = 0; t < n3; ++t) x[t] = x[t] + h * a0[t];
        } else if (M.itt == 1 || !P.enable_AB_3_order) {
            const double c0 = 1.5 + P.eps_ab, c1 = 0.5 + P.eps_ab;
            #pragma omp parallel for
            for (long t = 0; t < n3; ++t) x[t] = x[t] + h * (c0 * a0[t] - c1 * a1[t]);
        } else {
            const double A = 23.0 / 12.0, B = -16.0 / 12.0, Cc = 5.0 / 12.0;
            #pragma omp parallel for
            for (long t = 0; t < n3; ++t) x[t] = x[t] + h * (A * a0[t] + B * a1[t] + Cc * a2[t]);
        }
    }
    border_exchg_3D(M, u); border_exchg_3D(M, v); border_exchg_3D(M, w); border_exchg_3D(M, b);
    pressure_solver(M);
}

static inline void rotate(Model& M) {
    M.tau = M.tau % 3 + 1;
    M.taum1 = M.taum1 % 3 + 1;
    M.taum2 = M.taum2 % 3 + 1;
}

/* ---- diag_balance.f90:421-462 --------------------------------------------- */
static void interior_copy(const Model& M, const double* h, std::vector<double>& out) {
    out.resize((long)M.nx * M.ny * M.nz);
    for (int k = 1; k <= M.nz; ++k) for (int j = 1; j <= M.ny; ++j) for (int i = 1; i <= M.nx; ++i)
        out[(long)(i - 1) + (long)M.nx * ((j - 1) + (long)M.ny * (k - 1))] = h[M.I(i, j, k)];
}
static void interior_store(const Model& M, const std::vector<double>& in, double* h) {
    for (int k = 1; k <= M.nz; ++k) for (int j = 1; j <= M.ny; ++j) for (int i = 1; i <= M.nx; ++i)
        h[M.I(i, j, k)] = in[(long)(i - 1) + (long)M.nx * ((j - 1) + (long)M.ny * (k - 1))];
}
static void forward_transform(Model& M, const double* u, const double* v, const double* w, const double* b,
                              cx* US, cx* VS, cx* WS, cx* BS) {
    std::vector<double> t;
    const double* in[4] = {u, v, w, b};
    cx* out[4] = {US, VS, WS, BS};
    const std::vector<double>* mode[4] = {&M.phi, &M.phi, &M.psi, &M.psib};
    for (int f = 0; f < 4; ++f) {
        interior_copy(M, in[f], t);
        if (M.rigid) my_fft_vert_mode(M, t.data(), out[f], *mode[f]);
        else my_fft_3D(M, t.data(), out[f]);
    }
}
static void backward_transform(Model& M, cx* US, cx* VS, cx* WS, cx* BS,
                               double* u, double* v, double* w, double* b) {
    std::vector<double> t((long)M.nx * M.ny * M.nz);
    cx* in[4] = {US, VS, WS, BS};
    double* out[4] = {u, v, w, b};
    const std::vector<double>* mode[4] = {&M.phi, &M.phi, &M.psi, &M.psib};
    for (int f = 0; f < 4; ++f) {
        if (M.rigid) my_ifft_vert_mode(M, in[f], t.data(), *mode[f]);
        else my_ifft_3D(M, in[f], t.data());
        interior_store(M, t, out[f]);
    }
    for (int f = 0; f < 4; ++f) border_exchg_3D(M, out[f]);
}

/* projection kinds: 0 normal_mode_projection, 1 geostrophic_base_point,
 * 2 exchange_geostrophic_base_point, 3 diag_balance_zero_order            */
static void project(Model& M, int mode) {
    const long n = M.nspec();
    M.US.resize(n); M.VS.resize(n); M.WS.resize(n); M.BS.resize(n);
    if (mode == 1 || mode == 2) M.g0_base.resize(n);
    forward_transform(M, M.u.data(), M.v.data(), M.w.data(), M.b.data(),
                      M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    #pragma omp parallel for collapse(2)
    for (int k = 1; k <= M.nz; ++k)
        for (int j = 1; j <= M.ny; ++j)
            for (int i = 1; i <= M.nxh; ++i) {
                const long s = M.S(i, j, k);
                cx qx, qy, qz, qb, px, py, pz, pb;
                vec_q(M, M.kx[i - 1], M.ky[j - 1], M.kz[k - 1], 0.0, qx, qy, qz, qb);
                vec_p(M, M.kx[i - 1], M.ky[j - 1], M.kz[k - 1], 0.0, px, py, pz, pb);
                cx g0 = px * M.US[s] + py * M.VS[s] + pz * M.WS[s] + pb * M.BS[s];
                if (mode == 2) {
                    cx d = M.g0_base[s] - g0;
                    M.US[s] = M.US[s] + d * qx; M.VS[s] = M.VS[s] + d * qy;
                    M.WS[s] = M.WS[s] + d * qz; M.BS[s] = M.BS[s] + d * qb;
                } else {
                    if (mode == 1) M.g0_base[s] = g0;
                    M.US[s] = g0 * qx; M.VS[s] = g0 * qy; M.WS[s] = g0 * qz; M.BS[s] = g0 * qb;
                }
            }
    if (mode == 0 || mode == 2) {
        backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(),
                           M.u.data(), M.v.data(), M.w.data(), M.b.data());
    } else if (mode == 1) {
        for (auto* a : {&M.u_base, &M.v_base, &M.w_base, &M.b_base}) a->assign(M.n3, 0.0);
        backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(),
                           M.u_base.data(), M.v_base.data(), M.w_base.data(), M.b_base.data());
    } else {
        for (auto* a : {&M.u0, &M.v0, &M.w0, &M.b0}) a->assign(M.n3, 0.0);
        backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(),
                           M.u0.data(), M.v0.data(), M.w0.data(), M.b0.data());
    }
}

/* ---- diag_balance.f90:500-535: advective tendencies of a given state,
 *      divided by Ro (w also by dsqr), forward transformed; optional kz filter */
static void model_nonlin(Model& M, const double* ui, const double* vi, const double* wi, const double* bi,
                         cx* US, cx* VS, cx* WS, cx* BS) {
    const long n3 = M.n3;
    std::vector<double> u_loc = M.u, v_loc = M.v, w_loc = M.w, b_loc = M.b;
    std::vector<double> du_loc(n3, 0.0), dv_loc(n3, 0.0), dw_loc(n3, 0.0), db_loc(n3, 0.0);
    std::copy(ui, ui + n3, M.u.begin());
    std::copy(vi, vi + n3, M.v.begin());
    std::copy(wi, wi + n3, M.w.begin());
    std::copy(bi, bi + n3, M.b.begin());
    buoyancy_advection_2nd(M, db_loc.data());
    momentum_advection_2nd(M, du_loc.data(), dv_loc.data(), dw_loc.data());
    const double Ro = M.P.Ro, dsqr = M.P.dsqr;
    for (long t = 0; t < n3; ++t) {
        db_loc[t] = db_loc[t] / Ro;
        du_loc[t] = du_loc[t] / Ro;
        dv_loc[t] = dv_loc[t] / Ro;
        dw_loc[t] = dw_loc[t] / Ro / dsqr;
    }
    M.u = u_loc; M.v = v_loc; M.w = w_loc; M.b = b_loc;
    forward_transform(M, du_loc.data(), dv_loc.data(), dw_loc.data(), db_loc.data(), US, VS, WS, BS);
    if (M.balance_filter) {
        const double fxa = std::fabs(M.kz[M.nz / 2 + M.balance_filter_width]);   /* kz(nz/2+1+width) */
        for (int k = 1; k <= M.nz; ++k) {
            if (M.kz[k - 1] * M.kz[k - 1] < fxa * fxa) continue;
            for (int j = 1; j <= M.ny; ++j)
                for (int i = 1; i <= M.nxh; ++i) {
                    const long q = M.S(i, j, k);
                    US[q] = C(0, 0); VS[q] = C(0, 0); WS[q] = C(0, 0); BS[q] = C(0, 0);
                }
        }
    }
}

/* ---- diag_balance.f90:465-497: max_steps of integrate from a given state
 *      (itt stays 0, so every step is a forward step), state saved/restored */
static void model_run(Model& M, const double* ui, const double* vi, const double* wi, const double* bi,
                      double* uo, double* vo, double* wo, double* bo, int max_steps) {
    const long n3 = M.n3;
    std::vector<double> u_loc = M.u, v_loc = M.v, w_loc = M.w, b_loc = M.b, p_loc = M.p;
    std::vector<double> du_loc[3], dv_loc[3], dw_loc[3], db_loc[3];
    for (int s = 0; s < 3; ++s) { du_loc[s] = M.du[s]; dv_loc[s] = M.dv[s]; dw_loc[s] = M.dw[s]; db_loc[s] = M.db[s]; }
    const int tau_loc = M.tau, taum1_loc = M.taum1, taum2_loc = M.taum2, itt_loc = M.itt;
    std::copy(ui, ui + n3, M.u.begin());
    std::copy(vi, vi + n3, M.v.begin());
    std::copy(wi, wi + n3, M.w.begin());
    std::copy(bi, bi + n3, M.b.begin());
    M.itt = 0; M.taum2 = 1; M.taum1 = 2; M.tau = 3;
    for (int n = 1; n <= max_steps; ++n) {
        integrate(M);
        rotate(M);
    }
    std::copy(M.u.begin(), M.u.end(), uo);
    std::copy(M.v.begin(), M.v.end(), vo);
    std::copy(M.w.begin(), M.w.end(), wo);
    std::copy(M.b.begin(), M.b.end(), bo);
    M.u = u_loc; M.v = v_loc; M.w = w_loc; M.b = b_loc; M.p = p_loc;
    for (int s = 0; s < 3; ++s) { M.du[s] = du_loc[s]; M.dv[s] = dv_loc[s]; M.dw[s] = dw_loc[s]; M.db[s] = db_loc[s]; }
    M.tau = tau_loc; M.taum1 = taum1_loc; M.taum2 = taum2_loc; M.itt = itt_loc;
}

/* elementwise a + s*b (s*b alone when a is null) over full halo arrays */
static std::vector<double> comb(const std::vector<double>* a, const std::vector<double>& b, double s, bool divide) {
    std::vector<double> out(b.size());
    for (size_t t = 0; t < b.size(); ++t) {
        const double y = divide ? b[t] / s : b[t] * s;
        out[t] = a ? (*a)[t] + y : y;
    }
    return out;
}

static void warn_alloc(Model& M) {
    const long n = M.nspec();
    for (auto* a : {&M.US, &M.VS, &M.WS, &M.BS, &M.f1p, &M.f1m, &M.I_00, &M.I_0p, &M.I_0m, &M.I_f1p, &M.I_f1m,
                    &M.I_0f1p, &M.I_0f1m, &M.I_pT0p, &M.I_pT0m, &M.f2p, &M.f2m, &M.I_f2p, &M.I_f2m, &M.I_0f2p,
                    &M.I_0f2m, &M.pTf2p, &M.pTf2m})
        if ((long)a->size() != n) a->assign(n, C(0, 0));
    for (auto* a : {&M.u0, &M.v0, &M.w0, &M.b0, &M.u1, &M.v1, &M.w1, &M.b1, &M.u2, &M.v2, &M.w2, &M.b2, &M.u3, &M.v3,
                    &M.w3, &M.b3, &M.pTu0, &M.pTv0, &M.pTw0, &M.pTb0})
        if ((long)a->size() != M.n3) a->assign(M.n3, 0.0);
}

#define WARN_LOOP(...)                                                                                    \
    for (int k = 1; k <= M.nz; ++k)                                                                       \
        for (int j = 1; j <= M.ny; ++j)                                                                   \
            for (int i = 1; i <= M.nxh; ++i) {                                                            \
                const long q = M.S(i, j, k);                                                              \
                const double kxx = M.kx[i - 1], kyy = M.ky[j - 1], kzz = M.kz[k - 1];                     \
                __VA_ARGS__                                                                               \
            }
static inline cx dotp(cx a, cx b, cx c, cx d, cx U, cx V, cx W, cx B) { return a * U + b * V + c * W + d * B; }

/* ---- diag_balance.f90:135-176 -------------------------------------------- */
static void diag_balance_first_order(Model& M) {
    model_nonlin(M, M.u0.data(), M.v0.data(), M.w0.data(), M.b0.data(), M.US.data(), M.VS.data(), M.WS.data(),
                 M.BS.data());
    const double Ro = M.P.Ro;
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx px0, py0, pz0, pb0, pxp, pyp, pzp, pbp, pxm, pym, pzm, pbm, qxp, qyp, qzp, qbp, qxm, qym, qzm, qbm;
        vec_p(M, kxx, kyy, kzz, 0.0, px0, py0, pz0, pb0);
        vec_p(M, kxx, kyy, kzz, +1.0, pxp, pyp, pzp, pbp);
        vec_p(M, kxx, kyy, kzz, -1.0, pxm, pym, pzm, pbm);
        vec_q(M, kxx, kyy, kzz, +1.0, qxp, qyp, qzp, qbp);
        vec_q(M, kxx, kyy, kzz, -1.0, qxm, qym, qzm, qbm);
        const double om = std::sqrt(omega2(M, kxx, kyy, kzz));
        M.I_00[q] = IM * dotp(px0, py0, pz0, pb0, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        M.I_0p[q] = IM * dotp(pxp, pyp, pzp, pbp, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        M.I_0m[q] = IM * dotp(pxm, pym, pzm, pbm, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        if (om > 0.) { M.f1p[q] = M.I_0p[q] / om; M.f1m[q] = -(M.I_0m[q] / om); }
        else { M.f1p[q] = C(0, 0); M.f1m[q] = C(0, 0); }
        M.US[q] = Ro * (M.f1p[q] * qxp + M.f1m[q] * qxm);
        M.VS[q] = Ro * (M.f1p[q] * qyp + M.f1m[q] * qym);
        M.WS[q] = Ro * (M.f1p[q] * qzp + M.f1m[q] * qzm);
        M.BS[q] = Ro * (M.f1p[q] * qbp + M.f1m[q] * qbm);
    })
    backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(), M.u1.data(), M.v1.data(), M.w1.data(),
                       M.b1.data());
}

/* I = im * p(s).S for s = +1 and -1 into (Ip, Im) */
static void warn_pm(Model& M, std::vector<cx>& Ip, std::vector<cx>& Im) {
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx pxp, pyp, pzp, pbp, pxm, pym, pzm, pbm;
        vec_p(M, kxx, kyy, kzz, +1.0, pxp, pyp, pzp, pbp);
        vec_p(M, kxx, kyy, kzz, -1.0, pxm, pym, pzm, pbm);
        Ip[q] = IM * dotp(pxp, pyp, pzp, pbp, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        Im[q] = IM * dotp(pxm, pym, pzm, pbm, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
    })
}

/* ---- diag_balance.f90:180-272 -------------------------------------------- */
static void diag_balance_second_order(Model& M) {
    const double Ro = M.P.Ro;
    {
        auto a = comb(nullptr, M.u1, Ro, true), b = comb(nullptr, M.v1, Ro, true);
        auto c = comb(nullptr, M.w1, Ro, true), d = comb(nullptr, M.b1, Ro, true);
        model_nonlin(M, a.data(), b.data(), c.data(), d.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    }
    warn_pm(M, M.I_f1p, M.I_f1m);
    {
        auto a = comb(&M.u0, M.u1, Ro, true), b = comb(&M.v0, M.v1, Ro, true);
        auto c = comb(&M.w0, M.w1, Ro, true), d = comb(&M.b0, M.b1, Ro, true);
        model_nonlin(M, a.data(), b.data(), c.data(), d.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    }
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx pxp, pyp, pzp, pbp, pxm, pym, pzm, pbm, qx0, qy0, qz0, qb0;
        vec_p(M, kxx, kyy, kzz, +1.0, pxp, pyp, pzp, pbp);
        vec_p(M, kxx, kyy, kzz, -1.0, pxm, pym, pzm, pbm);
        vec_q(M, kxx, kyy, kzz, 0.0, qx0, qy0, qz0, qb0);
        M.I_0f1p[q] = IM * dotp(pxp, pyp, pzp, pbp, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        M.I_0f1m[q] = IM * dotp(pxm, pym, pzm, pbm, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        const cx pTg0 = -(IM * M.I_00[q]);
        M.US[q] = pTg0 * qx0; M.VS[q] = pTg0 * qy0; M.WS[q] = pTg0 * qz0; M.BS[q] = pTg0 * qb0;
    })
    backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(), M.pTu0.data(), M.pTv0.data(),
                       M.pTw0.data(), M.pTb0.data());
    model_nonlin(M, M.pTu0.data(), M.pTv0.data(), M.pTw0.data(), M.pTb0.data(), M.US.data(), M.VS.data(),
                 M.WS.data(), M.BS.data());
    warn_pm(M, M.I_pT0p, M.I_pT0m);
    {
        auto a = comb(&M.u0, M.pTu0, 1.0, false), b = comb(&M.v0, M.pTv0, 1.0, false);
        auto c = comb(&M.w0, M.pTw0, 1.0, false), d = comb(&M.b0, M.pTb0, 1.0, false);
        model_nonlin(M, a.data(), b.data(), c.data(), d.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    }
    const double Ro2 = Ro * Ro;
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx pxp, pyp, pzp, pbp, pxm, pym, pzm, pbm, qxp, qyp, qzp, qbp, qxm, qym, qzm, qbm;
        vec_p(M, kxx, kyy, kzz, +1.0, pxp, pyp, pzp, pbp);
        vec_p(M, kxx, kyy, kzz, -1.0, pxm, pym, pzm, pbm);
        vec_q(M, kxx, kyy, kzz, +1.0, qxp, qyp, qzp, qbp);
        vec_q(M, kxx, kyy, kzz, -1.0, qxm, qym, qzm, qbm);
        const double om = std::sqrt(omega2(M, kxx, kyy, kzz));
        const cx I_0pT0p = IM * dotp(pxp, pyp, pzp, pbp, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        const cx I_0pT0m = IM * dotp(pxm, pym, pzm, pbm, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        if (om > 0) {
            const cx pTf1p = (I_0pT0p - M.I_0p[q] - M.I_pT0p[q]) / om;
            const cx pTf1m = -((I_0pT0m - M.I_0m[q] - M.I_pT0m[q]) / om);
            M.f2p[q] = (M.I_0f1p[q] - M.I_0p[q] - M.I_f1p[q] - IM * pTf1p) / om;
            M.f2m[q] = -((M.I_0f1m[q] - M.I_0m[q] - M.I_f1m[q] - IM * pTf1m) / om);
        } else {
            M.f2p[q] = C(0, 0); M.f2m[q] = C(0, 0);
        }
        M.US[q] = Ro2 * (M.f2p[q] * qxp + M.f2m[q] * qxm);
        M.VS[q] = Ro2 * (M.f2p[q] * qyp + M.f2m[q] * qym);
        M.WS[q] = Ro2 * (M.f2p[q] * qzp + M.f2m[q] * qzm);
        M.BS[q] = Ro2 * (M.f2p[q] * qbp + M.f2m[q] * qbm);
    })
    backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(), M.u2.data(), M.v2.data(), M.w2.data(),
                       M.b2.data());
}

/* ---- diag_balance.f90:275-362 -------------------------------------------- */
static void diag_balance_third_order(Model& M) {
    const double Ro = M.P.Ro, Ro2 = Ro * Ro, Ro3 = Ro * Ro * Ro;
    {
        auto a = comb(nullptr, M.u2, Ro2, true), b = comb(nullptr, M.v2, Ro2, true);
        auto c = comb(nullptr, M.w2, Ro2, true), d = comb(nullptr, M.b2, Ro2, true);
        model_nonlin(M, a.data(), b.data(), c.data(), d.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    }
    warn_pm(M, M.I_f2p, M.I_f2m);
    {
        auto a = comb(&M.u0, M.u2, Ro2, true), b = comb(&M.v0, M.v2, Ro2, true);
        auto c = comb(&M.w0, M.w2, Ro2, true), d = comb(&M.b0, M.b2, Ro2, true);
        model_nonlin(M, a.data(), b.data(), c.data(), d.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
    }
    warn_pm(M, M.I_0f2p, M.I_0f2m);
    {
        auto a = comb(&M.u0, M.u1, 1.0, false), b = comb(&M.v0, M.v1, 1.0, false);
        auto c = comb(&M.w0, M.w1, 1.0, false), d = comb(&M.b0, M.b1, 1.0, false);
        a = comb(&a, M.u2, 1.0, false); b = comb(&b, M.v2, 1.0, false);
        c = comb(&c, M.w2, 1.0, false); d = comb(&d, M.b2, 1.0, false);
        model_run(M, a.data(), b.data(), c.data(), d.data(), M.u3.data(), M.v3.data(), M.w3.data(), M.b3.data(), 10);
    }
    forward_transform(M, M.u3.data(), M.v3.data(), M.w3.data(), M.b3.data(), M.US.data(), M.VS.data(), M.WS.data(),
                      M.BS.data());
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx qx0, qy0, qz0, qb0, px0, py0, pz0, pb0;
        vec_q(M, kxx, kyy, kzz, 0.0, qx0, qy0, qz0, qb0);
        vec_p(M, kxx, kyy, kzz, 0.0, px0, py0, pz0, pb0);
        const cx g0 = dotp(px0, py0, pz0, pb0, M.US[q], M.VS[q], M.WS[q], M.BS[q]);
        M.US[q] = g0 * qx0; M.VS[q] = g0 * qy0; M.WS[q] = g0 * qz0; M.BS[q] = g0 * qb0;
    })
    backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(), M.u0.data(), M.v0.data(), M.w0.data(),
                       M.b0.data());
    M.pTf2p = M.f2p; M.pTf2m = M.f2m;
    diag_balance_first_order(M);
    diag_balance_second_order(M);
    const long n = M.nspec();
    for (long q = 0; q < n; ++q) {
        M.pTf2p[q] = (M.f2p[q] - M.pTf2p[q]) / (10. * M.P.dt) / Ro;
        M.pTf2m[q] = (M.f2m[q] - M.pTf2m[q]) / (10. * M.P.dt) / Ro;
    }
    project(M, 3);   /* diag_balance_zero_order */
    diag_balance_first_order(M);
    diag_balance_second_order(M);
    #pragma omp parallel for collapse(2)
    WARN_LOOP({
        cx qxp, qyp, qzp, qbp, qxm, qym, qzm, qbm;
        vec_q(M, kxx, kyy, kzz, +1.0, qxp, qyp, qzp, qbp);
        vec_q(M, kxx, kyy, kzz, -1.0, qxm, qym, qzm, qbm);
        const double om = std::sqrt(omega2(M, kxx, kyy, kzz));
        cx f3p, f3m;
        if (om > 0) {
            f3p = (M.I_0f2p[q] + M.I_f1p[q] - M.I_f2p[q] - M.I_0p[q] - IM * M.pTf2p[q]) / om;
            f3m = -((M.I_0f2m[q] + M.I_f1m[q] - M.I_f2m[q] - M.I_0m[q] - IM * M.pTf2m[q]) / om);
        } else {
            f3p = C(0, 0); f3m = C(0, 0);
        }
        M.US[q] = Ro3 * (f3p * qxp + f3m * qxm);
        M.VS[q] = Ro3 * (f3p * qyp + f3m * qym);
        M.WS[q] = Ro3 * (f3p * qzp + f3m * qzm);
        M.BS[q] = Ro3 * (f3p * qbp + f3m * qbm);
    })
    backward_transform(M, M.US.data(), M.VS.data(), M.WS.data(), M.BS.data(), M.u3.data(), M.v3.data(), M.w3.data(),
                       M.b3.data());
}

/* diag_balance (diag_balance.f90:89-106) up to `order`, without the output */
static void diag_balance(Model& M, int order) {
    warn_alloc(M);
    project(M, 3);
    if (order >= 1) diag_balance_first_order(M);
    if (order >= 2) diag_balance_second_order(M);
    if (order >= 3) diag_balance_third_order(M);
}

/* ---- diag_opt_balance.f90:367-378 ---------------------------------------- */
static double ramp(double theta) {
    double t1 = 1. / std::max(1e-32, theta);
    double t2 = 1. / std::max(1e-32, 1.0 - theta);
    return std::exp(-t1) / (std::exp(-t1) + std::exp(-t2));
}

/* ---- diag_opt_balance.f90:339-362 ---------------------------------------- */
static double opt_balance_norm(Model& M) {
    double e1 = 0, e2 = 0, d = 0;
    const double dsqr = M.P.dsqr, N2 = M.P.N0 * M.P.N0;
    for (int k = 1; k <= M.nz; ++k) for (int j = 1; j <= M.ny; ++j) for (int i = 1; i <= M.nx; ++i) {
        const long t = M.I(i, j, k);
        const double u = M.u[t], v = M.v[t], w = M.w[t], b = M.b[t];
        const double ub = M.u_bal[t], vb = M.v_bal[t], wb = M.w_bal[t], bb = M.b_bal[t];
        e1 = e1 + u * u + v * v + dsqr * (w * w) + (b * b) / N2;
        e2 = e2 + ub * ub + vb * vb + dsqr * (wb * wb) + (bb * bb) / N2;
        d = d + (u - ub) * (u - ub) + (v - vb) * (v - vb) + dsqr * ((w - wb) * (w - wb)) + ((b - bb) * (b - bb)) / N2;
    }
    return 2.0 * std::sqrt(d) / (std::sqrt(e1) + std::sqrt(e2));
}

/* ---- diag_opt_balance.f90:234-258 ---------------------------------------- */
static void opt_time_ave(Model& M, int n_end_ave, std::vector<double>* loc[4]) {
    M.itt = 0; M.taum2 = 1; M.taum1 = 2; M.tau = 3;
    M.P.dt = std::fabs(M.P.dt);
    M.P.Ro = 0.;
    for (int f = 0; f < 4; ++f) loc[f]->assign(M.n3, 0.0);
    std::vector<double>* fld[4] = {&M.u, &M.v, &M.w, &M.b};
    for (int n = 0; n <= n_end_ave - 1; ++n) {
        integrate(M);
        rotate(M);
        for (int f = 0; f < 4; ++f)
            for (long t = 0; t < M.n3; ++t) (*loc[f])[t] = (*loc[f])[t] + (*fld[f])[t];
    }
    for (int f = 0; f < 4; ++f)
        for (long t = 0; t < M.n3; ++t) (*loc[f])[t] = (*loc[f])[t] / n_end_ave;
}

/* ---- diag_opt_balance.f90:55-231 ------------------------------------------ */
static void diag_opt_balance(Model& M, const ps3d_optbal& O, double* final_norm, int* iters) {
    auto u_loc = M.u, v_loc = M.v, w_loc = M.w, b_loc = M.b, p_loc = M.p;
    std::vector<double> du_loc[3], dv_loc[3], dw_loc[3], db_loc[3];
    for (int s = 0; s < 3; ++s) { du_loc[s] = M.du[s]; dv_loc[s] = M.dv[s]; dw_loc[s] = M.dw[s]; db_loc[s] = M.db[s]; }
    const double Ro_loc = M.P.Ro, dt_loc = M.P.dt;
    const int tau_loc = M.tau, taum1_loc = M.taum1, taum2_loc = M.taum2, itt_loc = M.itt;
    M.u_bal = M.u; M.v_bal = M.v; M.w_bal = M.w; M.b_bal = M.b;
    const int n_end = (int)(O.period / M.P.dt) + 1;
    const int n_end_ave = (int)(O.average / M.P.dt) + 1;
    double norm_diff = 1.0;
    std::vector<double>* base[4] = {&M.u_base, &M.v_base, &M.w_base, &M.b_base};
    std::vector<double>* ave[4] = {&M.u_ave, &M.v_ave, &M.w_ave, &M.b_ave};
    std::vector<double>* fld[4] = {&M.u, &M.v, &M.w, &M.b};
    if (O.enable_time_ave) {
        for (int m = 1; m <= O.average_times; ++m) {
            opt_time_ave(M, n_end_ave, base);
            for (int f = 0; f < 4; ++f) *fld[f] = *base[f];
        }
        M.u = M.u_bal; M.v = M.v_bal; M.w = M.w_bal; M.b = M.b_bal;
    } else {
        project(M, 1);
    }
    int n_done = 0;
    for (int n = 1; n <= O.max_itts; ++n) {
        n_done = n;
        /* opt_backward_integration, :183-209 */
        {
            const double Ahbi_loc = M.P.Ahbi, Avbi_loc = M.P.Avbi, Khbi_loc = M.P.Khbi, Kvbi_loc = M.P.Kvbi;
            M.P.Ahbi = 0; M.P.Avbi = 0; M.P.Khbi = 0; M.P.Kvbi = 0;
            M.itt = 0; M.taum2 = 1; M.taum1 = 2; M.tau = 3;
            M.P.dt = -std::fabs(M.P.dt);
            for (int s = 0; s <= n_end - 1; ++s) {
                const double rho = 1. - ramp(s * dt_loc / O.period);
                M.P.Ro = rho * Ro_loc;
                integrate(M);
                rotate(M);
            }
            M.P.Ahbi = Ahbi_loc; M.P.Avbi = Avbi_loc; M.P.Khbi = Khbi_loc; M.P.Kvbi = Kvbi_loc;
        }
        if (O.enable_time_ave) {
            for (int m = 1; m <= O.average_times; ++m) {
                opt_time_ave(M, n_end_ave, ave);
                for (int f = 0; f < 4; ++f) *fld[f] = *ave[f];
            }
        } else {
            project(M, 0);
        }
        /* opt_forward_integration, :213-231 */
        M.itt = 0; M.taum2 = 1; M.taum1 = 2; M.tau = 3;
        M.P.dt = std::fabs(M.P.dt);
        for (int s = 0; s <= n_end - 1; ++s) {
            const double rho = ramp(s * dt_loc / O.period);
            M.P.Ro = rho * Ro_loc;
            integrate(M);
            rotate(M);
        }
        if (O.enable_time_ave) {
            M.u_save = M.u; M.v_save = M.v; M.w_save = M.w; M.b_save = M.b;
            for (int m = 1; m <= O.average_times; ++m) {
                opt_time_ave(M, n_end_ave, ave);
                for (int f = 0; f < 4; ++f) *fld[f] = *ave[f];
            }
            std::vector<double>* sv[4] = {&M.u_save, &M.v_save, &M.w_save, &M.b_save};
            for (int f = 0; f < 4; ++f)
                for (long t = 0; t < M.n3; ++t) (*fld[f])[t] = (*sv[f])[t] - (*ave[f])[t] + (*base[f])[t];
        } else {
            project(M, 2);
        }
        norm_diff = opt_balance_norm(M);
        M.u_bal = M.u; M.v_bal = M.v; M.w_bal = M.w; M.b_bal = M.b;
        if (n > 1 && norm_diff < O.tol) break;
    }
    M.u = u_loc; M.v = v_loc; M.w = w_loc; M.b = b_loc; M.p = p_loc;
    for (int s = 0; s < 3; ++s) { M.du[s] = du_loc[s]; M.dv[s] = dv_loc[s]; M.dw[s] = dw_loc[s]; M.db[s] = db_loc[s]; }
    M.P.Ro = Ro_loc; M.P.dt = dt_loc;
    M.tau = tau_loc; M.taum1 = taum1_loc; M.taum2 = taum2_loc; M.itt = itt_loc;
    if (O.adopt) { M.u = M.u_bal; M.v = M.v_bal; M.w = M.w_bal; M.b = M.b_bal; }
    if (final_norm) *final_norm = norm_diff;
    if (iters) *iters = n_done;
}

/* ---- diagnose.F90:2-61 (reductions only) ---------------------------------- */
static int diagnose(Model& M, double* ke_o, double* pe_o, double* umax_o, double* wmax_o) {
    double ke = 0, pe = 0, umax = 0, wmax = 0;
    bool nonfinite = false;
    const double dsqr = M.P.dsqr, N0 = M.P.N0, dz = M.P.dz;
    for (int k = 1; k <= M.nz; ++k) for (int j = 1; j <= M.ny; ++j) for (int i = 1; i <= M.nx; ++i) {
        const long t = M.I(i, j, k);
        const double u = M.u[t], v = M.v[t], w = M.w[t], b = M.b[t];
        if (!std::isfinite(u) || !std::isfinite(v) || !std::isfinite(w) || !std::isfinite(b) || !std::isfinite(M.p[t]))
            nonfinite = true;
        umax = std::max(umax, std::sqrt(u * u + v * v));
        wmax = std::max(wmax, std::fabs(w));
        ke = ke + 0.5 * (u * u + v * v + dsqr * (w * w));
        if (N0 > 0.) pe = pe + 0.5 * (b * b) / (N0 * N0);
        else pe = pe + b * (k - 0.5) * dz;
    }
    const double n = (double)M.nx * M.ny * M.nz;
    if (ke_o) *ke_o = ke / n;
    if (pe_o) *pe_o = pe / n;
    if (umax_o) *umax_o = umax;
    if (wmax_o) *wmax_o = wmax;
    return nonfinite ? PS3D_ERR_NONFINITE : PS3D_OK;
}

static std::vector<double>* field_ptr(Model& M, int id) {
    switch (id) {
        case 0: return &M.u; case 1: return &M.v; case 2: return &M.w; case 3: return &M.b; case 4: return &M.p;
        case 5: case 6: case 7: return &M.du[id - 5];
        case 8: case 9: case 10: return &M.dv[id - 8];
        case 11: case 12: case 13: return &M.dw[id - 11];
        case 14: case 15: case 16: return &M.db[id - 14];
        case 20: return &M.u_bal; case 21: return &M.v_bal; case 22: return &M.w_bal; case 23: return &M.b_bal;
        case 24: return &M.u_base; case 25: return &M.v_base; case 26: return &M.w_base; case 27: return &M.b_base;
        case 28: return &M.u0; case 29: return &M.v0; case 30: return &M.w0; case 31: return &M.b0;
        case 32: return &M.u1; case 33: return &M.v1; case 34: return &M.w1; case 35: return &M.b1;
        case 36: return &M.u2; case 37: return &M.v2; case 38: return &M.w2; case 39: return &M.b2;
        case 40: return &M.u3; case 41: return &M.v3; case 42: return &M.w3; case 43: return &M.b3;
        default: return nullptr;
    }
}

}  // namespace

/* ========================================================================= */
/* C ABI for the tests (ctypes)                                              */
/* ========================================================================= */
extern "C" {

void* ps3d_oracle_create(const ps3d_params* prm) {
    Model* M = new Model();
    M->P = *prm;
    M->nx = prm->nx; M->ny = prm->ny; M->nz = prm->nz; M->nxh = prm->nx / 2 + 1;
    M->sy = prm->nx + 4; M->sz = (long)(prm->nx + 4) * (prm->ny + 4);
    M->n3 = M->sz * (prm->nz + 4);
    M->rigid = prm->enable_vertical_boundaries != 0;
    M->pi = std::acos(0.0) * 2.0;
    for (auto* a : {&M->u, &M->v, &M->w, &M->b, &M->p, &M->flux_east, &M->flux_north, &M->flux_top,
                    &M->u_bal, &M->v_bal, &M->w_bal, &M->b_bal, &M->u_base, &M->v_base, &M->w_base, &M->b_base,
                    &M->u0, &M->v0, &M->w0, &M->b0})
        a->assign(M->n3, 0.0);
    for (int s = 0; s < 3; ++s) {
        M->du[s].assign(M->n3, 0.0); M->dv[s].assign(M->n3, 0.0);
        M->dw[s].assign(M->n3, 0.0); M->db[s].assign(M->n3, 0.0);
    }
    M->FS.assign(M->nspec(), C(0, 0));
    wavenumber_initialisation(*M);
    return M;
}
void ps3d_oracle_destroy(void* h) { delete static_cast<Model*>(h); }

/* Pointer to a halo-layout field (ids in field_ptr) for zero-copy numpy views. */
double* ps3d_oracle_field(void* h, int id) {
    Model& M = *static_cast<Model*>(h);
    std::vector<double>* f = field_ptr(M, id);
    if (!f) return nullptr;
    if ((long)f->size() != M.n3) f->assign(M.n3, 0.0);
    return f->data();
}
long ps3d_oracle_field_size(void* h) { return static_cast<Model*>(h)->n3; }

void ps3d_oracle_get_time(void* h, int* itt, int* tau, int* taum1, int* taum2, double* time) {
    Model& M = *static_cast<Model*>(h);
    if (itt) *itt = M.itt;
    if (tau) *tau = M.tau;
    if (taum1) *taum1 = M.taum1;
    if (taum2) *taum2 = M.taum2;
    if (time) *time = M.time;
}
void ps3d_oracle_set_time(void* h, int itt, int tau, int taum1, int taum2, double time) {
    Model& M = *static_cast<Model*>(h);
    M.itt = itt; M.tau = tau; M.taum1 = taum1; M.taum2 = taum2; M.time = time;
}
void ps3d_oracle_set_step_params(void* h, double dt, double Ro, double Ahbi, double Avbi, double Khbi, double Kvbi) {
    Model& M = *static_cast<Model*>(h);
    M.P.dt = dt; M.P.Ro = Ro; M.P.Ahbi = Ahbi; M.P.Avbi = Avbi; M.P.Khbi = Khbi; M.P.Kvbi = Kvbi;
}
void ps3d_oracle_border_exchange(void* h, double* a) { border_exchg_3D(*static_cast<Model*>(h), a); }

/* integrate.f90 once (no rotation) */
void ps3d_oracle_step(void* h) { integrate(*static_cast<Model*>(h)); }
/* main.f90:139-160 loop body, nsteps times (without diagnostics) */
void ps3d_oracle_integrate(void* h, int nsteps) {
    Model& M = *static_cast<Model*>(h);
    for (int n = 0; n < nsteps; ++n) {
        integrate(M);
        rotate(M);
        M.time = M.time + M.P.dt;
        M.itt = M.itt + 1;
    }
}
void ps3d_oracle_pressure_solver(void* h) { pressure_solver(*static_cast<Model*>(h)); }
void ps3d_oracle_project(void* h, int mode) { project(*static_cast<Model*>(h), mode); }
/* diag_balance_zero_order .. third_order up to `order`; filter_width < 0:
 * no enable_diag_balance_filter.  Results in field ids 28-43 (u0..b3). */
void ps3d_oracle_diag_balance(void* h, int order, int filter_width) {
    Model& M = *static_cast<Model*>(h);
    M.balance_filter = filter_width >= 0;
    if (filter_width >= 0) M.balance_filter_width = filter_width;
    diag_balance(M, order);
}
/* forward_transform of the current state into US..BS (diag_balance.f90:421-438) */
void ps3d_oracle_forward_transform(void* h) {
    Model& M = *static_cast<Model*>(h);
    const long n = M.nspec();
    M.US.resize(n); M.VS.resize(n); M.WS.resize(n); M.BS.resize(n);
    forward_transform(M, M.u.data(), M.v.data(), M.w.data(), M.b.data(), M.US.data(), M.VS.data(), M.WS.data(), M.BS.data());
}
void ps3d_oracle_opt_balance(void* h, const ps3d_optbal* o, double* norm, int* iters) {
    diag_opt_balance(*static_cast<Model*>(h), *o, norm, iters);
}
int ps3d_oracle_diagnose(void* h, double* ke, double* pe, double* umax, double* wmax) {
    return diagnose(*static_cast<Model*>(h), ke, pe, umax, wmax);
}
void ps3d_oracle_set_forcing(void* h, const ps3d_forcing* f) {
    Model& M = *static_cast<Model*>(h);
    M.force_kind = f ? f->kind & (PS3D_FORCE_WAVEMAKER | PS3D_FORCE_BACKGROUND) : 0;
    if (!f) return;
    M.omega = f->omega;
    const double* r[4] = {f->u_r, f->v_r, f->w_r, f->b_r};
    const double* im[4] = {f->u_i, f->v_i, f->w_i, f->b_i};
    for (int q = 0; q < 4; ++q) {
        M.has_fr[q] = r[q] != nullptr; M.has_fi[q] = im[q] != nullptr;
        if (r[q]) M.fr[q].assign(r[q], r[q] + M.n3);
        if (im[q]) M.fi[q].assign(im[q], im[q] + M.n3);
    }
    M.u_back.assign(M.n3, 0.0); M.b_back.assign(M.n3, 0.0);
    if (f->u_back) M.u_back.assign(f->u_back, f->u_back + M.n3);
    if (f->b_back) M.b_back.assign(f->b_back, f->b_back + M.n3);
}

/* spectral / table access for known-answer tests */
const double* ps3d_oracle_ksqr(void* h, long* n) {
    Model& M = *static_cast<Model*>(h);
    if (n) *n = (long)M.ksqr.size();
    return M.ksqr.data();
}
const double* ps3d_oracle_modes(void* h, int which) {
    Model& M = *static_cast<Model*>(h);
    return which == 0 ? M.phi.data() : which == 1 ? M.psi.data() : M.psib.data();
}
const double* ps3d_oracle_wavenumbers(void* h, int axis) {
    Model& M = *static_cast<Model*>(h);
    return axis == 0 ? M.kx.data() : axis == 1 ? M.ky.data() : M.kz.data();
}
/* FS after the last pressure solve (complex, nxh*ny*nz interleaved re/im) */
const double* ps3d_oracle_spectral(void* h, int which) {
    Model& M = *static_cast<Model*>(h);
    const std::vector<cx>* v = which == 0 ? &M.FS : which == 1 ? &M.US : which == 2 ? &M.VS :
                               which == 3 ? &M.WS : which == 4 ? &M.BS : &M.g0_base;
    return v->empty() ? nullptr : reinterpret_cast<const double*>(v->data());
}

/* eigenvectors for one wavenumber (s = 0, +1, -1): out = qx,qy,qz,qb,px,py,pz,pb (re,im) + om2 */
void ps3d_oracle_eigen(void* h, double kx, double ky, double kz, double s, double* out) {
    Model& M = *static_cast<Model*>(h);
    cx q[4], p[4];
    vec_q(M, kx, ky, kz, s, q[0], q[1], q[2], q[3]);
    vec_p(M, kx, ky, kz, s, p[0], p[1], p[2], p[3]);
    for (int t = 0; t < 4; ++t) { out[2 * t] = q[t].re; out[2 * t + 1] = q[t].im; }
    for (int t = 0; t < 4; ++t) { out[8 + 2 * t] = p[t].re; out[8 + 2 * t + 1] = p[t].im; }
    out[16] = omega2(M, kx, ky, kz);
}

/* bare complex FFT (n, sign) on interleaved re/im, for checks against numpy */
void ps3d_oracle_fft(double* data, int n, int sign) {
    std::vector<cx> x(n), y(n);
    std::memcpy(x.data(), data, sizeof(cx) * n);
    fft1d(get_plan(n), x.data(), y.data(), sign);
    std::memcpy(data, x.data(), sizeof(cx) * n);
}
/* 2D 'ffn' / 3D 'fft' forward transforms and inverses on interior arrays */
void ps3d_oracle_fft_field(void* h, const double* QP, double* QS, int three_d) {
    Model& M = *static_cast<Model*>(h);
    if (three_d) my_fft_3D(M, QP, reinterpret_cast<cx*>(QS));
    else my_fft_2D(M, QP, reinterpret_cast<cx*>(QS));
}
void ps3d_oracle_ifft_field(void* h, double* QS, double* QP, int three_d) {
    Model& M = *static_cast<Model*>(h);
    if (three_d) my_ifft_3D(M, reinterpret_cast<cx*>(QS), QP);
    else my_ifft_2D(M, reinterpret_cast<cx*>(QS), QP);
}
void ps3d_oracle_tridiag(const double* a, const double* b, const double* c, const double* d, double* x, int n) {
    std::vector<double> cp(n); std::vector<cx> dp(n), xx(n), dd(n);
    std::memcpy(dd.data(), d, sizeof(cx) * n);
    solve_tridiag(a, b, c, dd.data(), xx.data(), n, cp.data(), dp.data());
    std::memcpy(x, xx.data(), sizeof(cx) * n);
}
double ps3d_oracle_ramp(double theta) { return ramp(theta); }
int ps3d_oracle_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

}  /* extern "C" */
