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
#include "eigen.cuh"

namespace ps3d {

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
