// reduce.cu — grid reductions: diagnose (diagnose.F90:14-45), the optimal
// balance energy norm (diag_opt_balance.f90:339-362) and small vector ops.
// Two-stage and deterministic: fixed-shape block partials, then one block
// sums the partials in a fixed order, so repeated calls give identical bits.
#include "engine.h"

namespace ps3d {

constexpr int kRedThreads = 256;

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const bool (&is_max)[NV], double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            x = is_max[q] ? fmax(x, y) : x + y;
        }
        if (lane == 0) sh[wid * NV + q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double x = sh[q];
            for (int w = 1; w < nw; ++w) x = is_max[q] ? fmax(x, sh[w * NV + q]) : x + sh[w * NV + q];
            v[q] = x;
        }
    }
}

__global__ void __launch_bounds__(kRedThreads) k_diag_partial(const double* __restrict__ u, const double* __restrict__ v,
                                                              const double* __restrict__ w, const double* __restrict__ b,
                                                              const double* __restrict__ p, int nx, int ny, int nz,
                                                              double dsqr, double N0, double dz, int kofs,
                                                              double* partials) {
    __shared__ double sh[32 * 5];
    const long N = (long)nx * ny * nz, plane = (long)nx * ny;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};   // ke, pe, umax, wmax, nonfinite
    const bool mx[5] = {false, false, true, true, true};
    const double rN2 = N0 > 0.0 ? 1.0 / (N0 * N0) : 0.0;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
        const double uu = u[g], vv = v[g], ww = w[g], bb = b[g], pp = p[g];
        if (!isfinite(uu) || !isfinite(vv) || !isfinite(ww) || !isfinite(bb) || !isfinite(pp)) acc[4] = 1.0;
        acc[2] = fmax(acc[2], sqrt(uu * uu + vv * vv));
        acc[3] = fmax(acc[3], fabs(ww));
        acc[0] = acc[0] + 0.5 * (uu * uu + vv * vv + dsqr * (ww * ww));
        if (N0 > 0.0) acc[1] = acc[1] + 0.5 * (bb * bb) * rN2;
        else acc[1] = acc[1] + bb * ((double)(g / plane + kofs) + 0.5) * dz;   // level k + kofs of the grid
    }
    block_reduce<5>(acc, mx, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 5; ++q) partials[blockIdx.x * 5 + q] = acc[q];
}

__global__ void __launch_bounds__(kRedThreads) k_diag_final(const double* partials, int nblk, long N, DiagOut* out) {
    __shared__ double sh[32 * 5];
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const bool mx[5] = {false, false, true, true, true};
    for (int t = threadIdx.x; t < nblk; t += blockDim.x) {
        acc[0] += partials[t * 5 + 0]; acc[1] += partials[t * 5 + 1];
        acc[2] = fmax(acc[2], partials[t * 5 + 2]); acc[3] = fmax(acc[3], partials[t * 5 + 3]);
        acc[4] = fmax(acc[4], partials[t * 5 + 4]);
    }
    block_reduce<5>(acc, mx, sh);
    if (threadIdx.x == 0) {
        out->ke = acc[0] / (double)N;
        out->pe = acc[1] / (double)N;
        out->umax = acc[2];
        out->wmax = acc[3];
        out->flags = acc[4] != 0.0 ? kFlagNonFinite : 0u;
    }
}

cudaError_t launch_diagnose(const double* u, const double* v, const double* w, const double* b, const double* p,
                            int nx, int ny, int nz, double dsqr, double N0, double dz,
                            double* partials, int nblk, DiagOut* out_dev, cudaStream_t s, int kofs) {
    k_diag_partial<<<nblk, kRedThreads, 0, s>>>(u, v, w, b, p, nx, ny, nz, dsqr, N0, dz, kofs, partials);
    k_diag_final<<<1, kRedThreads, 0, s>>>(partials, nblk, (long)nx * ny * nz, out_dev);
    return cudaGetLastError();
}

// opt_balance_norm: e1 = |x|^2, e2 = |y|^2, d = |x-y|^2 in the energy metric
struct Ptr8 { const double* p[8]; };
__global__ void __launch_bounds__(kRedThreads) k_norm_partial(Ptr8 xy, long n, double dsqr, double N0sq, double* partials) {
    __shared__ double sh[32 * 3];
    double acc[3] = {0.0, 0.0, 0.0};
    const bool mx[3] = {false, false, false};
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n; g += (long)gridDim.x * blockDim.x) {
        const double u = xy.p[0][g], v = xy.p[1][g], w = xy.p[2][g], b = xy.p[3][g];
        const double ub = xy.p[4][g], vb = xy.p[5][g], wb = xy.p[6][g], bb = xy.p[7][g];
        acc[0] = acc[0] + u * u + v * v + dsqr * (w * w) + (b * b) / N0sq;
        acc[1] = acc[1] + ub * ub + vb * vb + dsqr * (wb * wb) + (bb * bb) / N0sq;
        acc[2] = acc[2] + (u - ub) * (u - ub) + (v - vb) * (v - vb) + dsqr * ((w - wb) * (w - wb)) + ((b - bb) * (b - bb)) / N0sq;
    }
    block_reduce<3>(acc, mx, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) partials[blockIdx.x * 3 + q] = acc[q];
}
__global__ void __launch_bounds__(kRedThreads) k_norm_final(const double* partials, int nblk, double* out) {
    __shared__ double sh[32 * 3];
    double acc[3] = {0.0, 0.0, 0.0};
    const bool mx[3] = {false, false, false};
    for (int t = threadIdx.x; t < nblk; t += blockDim.x) {
        acc[0] += partials[t * 3]; acc[1] += partials[t * 3 + 1]; acc[2] += partials[t * 3 + 2];
    }
    block_reduce<3>(acc, mx, sh);
    if (threadIdx.x == 0) {
        out[0] = acc[0]; out[1] = acc[1]; out[2] = acc[2];
        out[3] = 2.0 * sqrt(acc[2]) / (sqrt(acc[0]) + sqrt(acc[1]));
    }
}
cudaError_t launch_norm(const double* const* x, const double* const* y, long n, double dsqr, double N0sq,
                        double* partials, int nblk, double* out_dev, cudaStream_t s) {
    Ptr8 xy;
    for (int q = 0; q < 4; ++q) { xy.p[q] = x[q]; xy.p[4 + q] = y[q]; }
    k_norm_partial<<<nblk, kRedThreads, 0, s>>>(xy, n, dsqr, N0sq, partials);
    k_norm_final<<<1, kRedThreads, 0, s>>>(partials, nblk, out_dev);
    return cudaGetLastError();
}

// y = a*y + b*x, with a == 0 meaning y = b*x and b == 0 meaning y = a*y
__global__ void k_axpby(double* y, const double* x, long n, double a, double b) {
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n; g += (long)gridDim.x * blockDim.x) {
        const double yy = (a == 0.0) ? 0.0 : a * y[g];
        y[g] = (b == 0.0) ? yy : ((a == 0.0) ? b * x[g] : yy + b * x[g]);
    }
}
cudaError_t launch_axpby(double* y, const double* x, long n, double a, double b, cudaStream_t s) {
    const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
    k_axpby<<<blocks, 256, 0, s>>>(y, x, n, a, b);
    return cudaGetLastError();
}

}  // namespace ps3d
