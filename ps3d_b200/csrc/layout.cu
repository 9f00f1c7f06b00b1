// layout.cu — conversion between the host's halo layout and the device's
// interior-only layout, done on the device so a host array crosses the bus
// in one contiguous copy.
//
// Host layout: Fortran bounds (1-2:nx+2, 1-2:ny+2, 1-2:nz+2), x fastest
// (main_module.f90:124-127).  Interior point (i, j, k) (0-based) sits at
// array index (i+2, j+2, k+2).  On download every halo point is the periodic
// copy of an interior point, as border_exchg_3D leaves it on one rank
// (parallel_mpi.f90:70-211); for p under a rigid lid the z ghost levels copy
// the nearest interior level instead (pressure_solver.f90:82-93).
#include "engine.h"

namespace ps3d {

__global__ void k_from_halo(const double* __restrict__ h, void* __restrict__ dst, int nx, int ny, int nz, int f32) {
    const long N = (long)nx * ny * nz;
    const long sy = nx + 4, sz = sy * (ny + 4);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < N; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx);
        const long r = t / nx;
        const int j = (int)(r % ny), k = (int)(r / ny);
        const double v = h[(i + 2) + sy * (j + 2) + sz * (k + 2)];
        if (f32) reinterpret_cast<float*>(dst)[t] = (float)v;
        else reinterpret_cast<double*>(dst)[t] = v;
    }
}

__global__ void k_to_halo(const void* __restrict__ src, double* __restrict__ h, int nx, int ny, int nz, int pghost,
                          int f32) {
    const long sy = nx + 4, sz = sy * (ny + 4), n3 = sz * (nz + 4);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n3; t += (long)gridDim.x * blockDim.x) {
        const int xx = (int)(t % sy);
        const long r = t / sy;
        const int yy = (int)(r % (ny + 4)), zz = (int)(r / (ny + 4));
        const int i = ((xx - 2) % nx + nx) % nx;
        const int j = ((yy - 2) % ny + ny) % ny;
        const int k = pghost ? min(max(zz - 2, 0), nz - 1) : ((zz - 2) % nz + nz) % nz;
        const long g = ((long)k * ny + j) * nx + i;
        h[t] = f32 ? (double)reinterpret_cast<const float*>(src)[g] : reinterpret_cast<const double*>(src)[g];
    }
}

static int grid_of(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 16); }

cudaError_t launch_from_halo(const double* h_dev, void* dst, int nx, int ny, int nz, bool f32, cudaStream_t s) {
    k_from_halo<<<grid_of((long)nx * ny * nz), 256, 0, s>>>(h_dev, dst, nx, ny, nz, f32 ? 1 : 0);
    return cudaGetLastError();
}
cudaError_t launch_to_halo(const void* src, double* h_dev, int nx, int ny, int nz, bool pghost, bool f32,
                           cudaStream_t s) {
    k_to_halo<<<grid_of((long)(nx + 4) * (ny + 4) * (nz + 4)), 256, 0, s>>>(src, h_dev, nx, ny, nz, pghost ? 1 : 0,
                                                                           f32 ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace ps3d
