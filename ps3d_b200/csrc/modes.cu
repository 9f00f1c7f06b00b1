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
#include <cstdlib>
#include "eigen.cuh"
#include "fft.cuh"

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

// Vertical-mode transforms (my_fft_vert_mode, my_fft.f90:234-252;
// my_ifft_vert_mode, my_fft.f90:211-229) over the columns of a plane-FFT'd
// field:
//   out[ko][c] = scale * sum_ki in[ki][c] * A[ko + nz*ki]
// with A = mode(ki, ko) (forward: the transpose of the Fortran column-major
// mode matrix) or A = mode(ko, ki) (inverse: the matrix itself); the forward
// scale dz multiplies the sum instead of every term.  A dense FP64 product,
// nz^2 multiply-adds per complex column: bound by the FP64 pipe, not HBM.
// A block stages 32 columns (one per lane) x nz levels in shared memory;
// each warp accumulates kVmKo output levels of its lane's column per pass in
// FP64 registers, reading each 16-byte pair of matrix entries once per warp
// (a warp-uniform load, broadcast from L1), so a shared-memory load of one
// complex input feeds 2*kVmKo fused multiply-adds.
constexpr int kVmCols = 32;
constexpr int kVmKo = 8;
constexpr int kVmThreads = 256;

size_t vert_mode_smem(int nz) { return (size_t)nz * kVmCols * sizeof(double2); }
bool vert_mode_fits(int nz) { return vert_mode_smem(nz) <= 227 * 1024; }

template <bool VEC>
__global__ void __launch_bounds__(kVmThreads) k_vert_mode(const double2* __restrict__ in, double2* __restrict__ out,
                                                          const double* __restrict__ A, int nz, long ncol,
                                                          double scale) {
    extern __shared__ double2 tile[];   // [nz][kVmCols]
    const long c0 = blockIdx.x * (long)kVmCols;
    const int nl = (int)min((long)kVmCols, ncol - c0);
    for (int t = threadIdx.x; t < nz * kVmCols; t += blockDim.x) {
        const int k = t / kVmCols, l = t - k * kVmCols;
        tile[t] = (l < nl) ? in[(long)k * ncol + c0 + l] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int l = threadIdx.x % kVmCols;
    const int wid = threadIdx.x / kVmCols, nw = blockDim.x / kVmCols;
    if (l >= nl) return;   // no block barrier below
    const int nch = (nz + kVmKo - 1) / kVmKo;
    for (int ch = wid; ch < nch; ch += nw) {
        const int ko0 = ch * kVmKo;
        double ar[kVmKo], ai[kVmKo];
#pragma unroll
        for (int q = 0; q < kVmKo; ++q) { ar[q] = 0.0; ai[q] = 0.0; }
        if (VEC && ko0 + kVmKo <= nz) {
            // nz even and ko0 a multiple of kVmKo: the pairs are 16-byte aligned
#pragma unroll 2
            for (int ki = 0; ki < nz; ++ki) {
                const double2 v = tile[ki * kVmCols + l];
                const double2* row = reinterpret_cast<const double2*>(A + ko0 + (long)nz * ki);
#pragma unroll
                for (int q = 0; q < kVmKo / 2; ++q) {
                    const double2 m = __ldg(row + q);
                    ar[2 * q] = fma(v.x, m.x, ar[2 * q]);
                    ai[2 * q] = fma(v.y, m.x, ai[2 * q]);
                    ar[2 * q + 1] = fma(v.x, m.y, ar[2 * q + 1]);
                    ai[2 * q + 1] = fma(v.y, m.y, ai[2 * q + 1]);
                }
            }
        } else {
            for (int ki = 0; ki < nz; ++ki) {
                const double2 v = tile[ki * kVmCols + l];
#pragma unroll
                for (int q = 0; q < kVmKo; ++q) {
                    if (ko0 + q < nz) {
                        const double m = __ldg(A + ko0 + q + (long)nz * ki);
                        ar[q] = fma(v.x, m, ar[q]);
                        ai[q] = fma(v.y, m, ai[q]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kVmKo; ++q)
            if (ko0 + q < nz) out[(long)(ko0 + q) * ncol + c0 + l] = make_double2(ar[q] * scale, ai[q] * scale);
    }
}

cudaError_t launch_project(const ProjArgs& a, cudaStream_t s) {
    const long M = (long)a.nxh * a.ny * a.nz;
    const int blocks = (int)std::min<long>((M + 255) / 256, 148L * 16);
    k_project<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// The same product with the matrix staged in shared memory as well (nz^2
// doubles beside the tile; nz <= 104 keeps two blocks per SM): the matrix
// pairs are then warp-uniform shared-memory loads instead of L1 loads.  The
// grid is as many blocks as are resident at once, each copying the matrix
// once and walking the column tiles with the grid's stride, so the copy is
// amortised and no SM idles in a partial last wave.
size_t vert_mode_smem_staged(int nz) { return (size_t)nz * kVmCols * sizeof(double2) + (size_t)nz * nz * sizeof(double); }

__global__ void __launch_bounds__(kVmThreads) k_vert_mode_staged(const double2* __restrict__ in,
                                                                 double2* __restrict__ out,
                                                                 const double* __restrict__ A, int nz, long ncol,
                                                                 double scale) {
    extern __shared__ double2 tile[];   // [nz][kVmCols], then the matrix [ki][ko]
    double* Am = reinterpret_cast<double*>(tile + (size_t)nz * kVmCols);
    for (int t = threadIdx.x; t < nz * nz; t += blockDim.x) Am[t] = __ldg(A + t);
    const int l = threadIdx.x % kVmCols;
    const int wid = threadIdx.x / kVmCols, nw = blockDim.x / kVmCols;
    const int nch = (nz + kVmKo - 1) / kVmKo;
    const long ntiles = (ncol + kVmCols - 1) / kVmCols;
    for (long tile_i = blockIdx.x; tile_i < ntiles; tile_i += gridDim.x) {
        const long c0 = tile_i * kVmCols;
        const int nl = (int)min((long)kVmCols, ncol - c0);
        __syncthreads();   // the previous tile is read (and, the first time, nothing)
        for (int t = threadIdx.x; t < nz * kVmCols; t += blockDim.x) {
            const int k = t / kVmCols, ll = t - k * kVmCols;
            tile[t] = (ll < nl) ? in[(long)k * ncol + c0 + ll] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (l < nl) {
            for (int ch = wid; ch < nch; ch += nw) {
                const int ko0 = ch * kVmKo;
                double ar[kVmKo], ai[kVmKo];
#pragma unroll
                for (int q = 0; q < kVmKo; ++q) { ar[q] = 0.0; ai[q] = 0.0; }
                if (ko0 + kVmKo <= nz) {
#pragma unroll 2
                    for (int ki = 0; ki < nz; ++ki) {
                        const double2 v = tile[ki * kVmCols + l];
                        const double2* row = reinterpret_cast<const double2*>(Am + ko0 + nz * ki);
#pragma unroll
                        for (int q = 0; q < kVmKo / 2; ++q) {
                            const double2 m = row[q];
                            ar[2 * q] = fma(v.x, m.x, ar[2 * q]);
                            ai[2 * q] = fma(v.y, m.x, ai[2 * q]);
                            ar[2 * q + 1] = fma(v.x, m.y, ar[2 * q + 1]);
                            ai[2 * q + 1] = fma(v.y, m.y, ai[2 * q + 1]);
                        }
                    }
                } else {
                    for (int ki = 0; ki < nz; ++ki) {
                        const double2 v = tile[ki * kVmCols + l];
#pragma unroll
                        for (int q = 0; q < kVmKo; ++q) {
                            if (ko0 + q < nz) {
                                const double m = Am[ko0 + q + nz * ki];
                                ar[q] = fma(v.x, m, ar[q]);
                                ai[q] = fma(v.y, m, ai[q]);
                            }
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kVmKo; ++q)
                    if (ko0 + q < nz) out[(long)(ko0 + q) * ncol + c0 + l] = make_double2(ar[q] * scale, ai[q] * scale);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same transforms by FFT.  The rigid-lid mode matrices (my_fft.f90:
// 112-127) are sampled sines and cosines, for levels k = 1..N and modes
// j = m-1 = 0..N-1:
//   psi(k, j)  = c sin(pi j k / N)                      (DST-I)
//   phi(k, j)  = c_j cos(pi j (k - 1/2) / N)            (DCT-II; c_0 = sqrt(1/Lz))
//   psib(k, j) = c sin(pi j (k - 1/2) / N), j >= 1      (DST-II; mode 0 is zero)
// with c = sqrt(2/Lz) (phi and psib are the differences and sums of psi's
// neighbouring levels, divided by 2 sin and 2 cos of pi j / 2N).  Each
// column's analysis (forward: out_j = dz sum_k in_k mode(k, j)) and
// synthesis (backward: out_k = sum_j in_j mode(k, j)) is then one complex
// FFT of length 2N of the column's even or odd extension, with a twiddle
// e^{+-i pi j / 2N} before or after (the data are complex; the transforms
// act on both parts alike):
//   DCT-II   X_j = 1/2 e^{-i pi j/2N} Y_j,   y = [x, reversed x]
//   DST-II   X_j = i/2 e^{-i pi j/2N} Y_j,   y = [x, -reversed x]
//   DST-I    X_j = i/2 Y_j,                  y = [0, x_1..x_{N-1}, 0, -reversed]
// and for the synthesis the spectrum V of length 2N whose inverse FFT is the
// column: V_j, V_{2N-j} = the weighted input times e^{+-i pi j/2N}/2
// (DCT-III, V_0 = the mode-0 term), times e^{+-i pi j/2N}/(+-2i) (DST-III),
// or /(+-2i) (DST-I).  O(N log N) per column instead of N^2 multiply-adds.
// The results differ from the dense sums at round-off (the parity tests
// hold both to the oracle).  A block takes kDttCols columns, buf[e][column]
// as fft_batch lays lines out (its radix-8 build: 80 registers, three
// blocks per SM), and walks the column tiles with the grid's stride.
// Measured per transform with every field at length 2 nz: 52 us against 49
// us for the dense product at 256x256x64, 90 against 202 us at
// 256x256x128, 162 against 1012 us at 256x128x256; k_vert_dttn below
// halves the length for phi and psib.
constexpr int kDttCols = 16;
constexpr int kDttThreads = 256;

size_t vert_dtt_smem(int nz, int cols) {
    return align16((size_t)2 * nz * (cols | 1) * sizeof(double2)) + plan_tables_bytes(2 * nz, sizeof(double2));
}

template <int KIND, bool FWD>
__global__ void __launch_bounds__(kDttThreads, 3) k_vert_dtt(const VertDttArgs a) {
    using T = double2;
    extern __shared__ __align__(16) unsigned char dtt_raw[];
    const int N = a.nz, N2 = 2 * a.nz, C = a.cols, ld = a.cols | 1;
    T* buf = reinterpret_cast<T*>(dtt_raw);
    const PlanTables<double> tp = stage_plan<double>(a.plan, dtt_raw + align16((size_t)N2 * ld * sizeof(T)));
    const long ncol = a.ncol;
    const long ntiles = (ncol + C - 1) / C;
    // weight of mode j and the twiddle e^{i pi j / 2N}
    auto weight = [&](int j) { return j == 0 ? (KIND == 0 ? a.c0 : 0.0) : a.c1; };
    for (long ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const long c0 = ti * C;
        const int nl = (int)min((long)C, ncol - c0);
        __syncthreads();   // the previous tile is stored (and the tables staged)
        for (int t = threadIdx.x; t < N2 * C; t += blockDim.x) {
            const int e = t / C, l = t - e * C;
            T v = make_double2(0.0, 0.0);
            if (l < nl) {
                const T* col = a.in + c0 + l;
                if (FWD) {
                    if (KIND == 1) {   // [0, x_1..x_{N-1}, 0, -x_{N-1}..-x_1], x_k = level k (index k-1)
                        if (e >= 1 && e < N) v = col[(long)(e - 1) * ncol];
                        else if (e > N) v = cscale(col[(long)(N2 - e - 1) * ncol], -1.0);
                    } else {           // [x, +-reversed x]
                        if (e < N) v = col[(long)e * ncol];
                        else v = cscale(col[(long)(N2 - 1 - e) * ncol], KIND == 0 ? 1.0 : -1.0);
                    }
                } else if (e != N) {
                    const int j = e < N ? e : N2 - e;
                    const T z = cscale(col[(long)j * ncol], weight(j));
                    if (KIND == 0) {
                        // V_0 = Z_0; V_j = Z_j w_j / 2; V_{2N-j} = Z_j conj(w_j) / 2
                        v = j == 0 ? z : cscale(cmul(z, e < N ? a.tw[j] : cconj(a.tw[j])), 0.5);
                    } else if (j != 0) {
                        // / (2i) = * (-i/2); the mirrored half with the opposite sign
                        const T zw = KIND == 2 ? cmul(z, e < N ? a.tw[j] : cconj(a.tw[j])) : z;
                        v = cscale(cmul_si(zw, -1), e < N ? 0.5 : -0.5);
                    }
                }
            }
            buf[e * ld + l] = v;
        }
        fft_batch<false, double, 8>(buf, ld, C, a.plan, FWD ? -1 : +1, tp.tw);   // synchronises
        for (int t = threadIdx.x; t < N * C; t += blockDim.x) {
            const int j = t / C, l = t - j * C;
            if (l >= nl) continue;
            // element j of the transform (DIF: digit-reversed slots); the
            // psi synthesis's level k = j+1 is element j+1
            const T y = buf[tp.pos[(!FWD && KIND == 1) ? j + 1 : j] * ld + l];
            T o;
            if (FWD) {
                if (KIND == 1) o = cmul_si(y, 1);                         // i Y_j
                else o = KIND == 0 ? cmul(y, cconj(a.tw[j])) : cmul_si(cmul(y, cconj(a.tw[j])), 1);
                o = cscale(o, 0.5 * a.scale * weight(j));
            } else {
                o = cscale(y, a.scale);
            }
            a.out[(long)j * ncol + c0 + l] = o;
        }
    }
}

// phi and psib (kinds 0 and 2) for even nz by FFTs of length nz (Makhoul
// 1980, "A fast cosine transform in one and multiple dimensions", its
// even/odd reordering, carried over to complex data): half the transform
// length of the extension form.
//   DCT-II   v = [x_0, x_2, .., x_{N-2}, x_{N-1}, .., x_3, x_1], V = FFT_N(v),
//            X_j = ((P.x + Q.x) + i (P.y - Q.y)) / 2 with P = e^{-i pi j/2N} V_j,
//            Q = e^{-i pi j/2N} conj(V_{N-j}) (the real and imaginary parts
//            of the data separated through V_j and V_{N-j})
//   DST-II   X_j = DCT-II((-1)^k x_k)_{N-j}
//   DCT-III  V_0 = 2 Z_0, V_j = e^{i pi j/2N} (Z_j - i Z_{N-j}), v = IFFT_N(V)/2,
//            x_{2n} = v_n, x_{2n+1} = v_{N-1-n}
//   DST-III  x_k = (-1)^k DCT-III(Z')_k with Z'_j = Z_{N-j}, Z'_0 = 0
size_t vert_dttn_smem(int nz, int cols) {
    return align16((size_t)nz * (cols | 1) * sizeof(double2)) + plan_tables_bytes(nz, sizeof(double2));
}

template <int KIND, bool FWD>
__global__ void __launch_bounds__(kDttThreads, 3) k_vert_dttn(const VertDttArgs a) {
    static_assert(KIND == 0 || KIND == 2, "phi and psib");
    using T = double2;
    extern __shared__ __align__(16) unsigned char dttn_raw[];
    const int N = a.nz, H = a.nz / 2, C = a.cols, ld = a.cols | 1;
    T* buf = reinterpret_cast<T*>(dttn_raw);
    const PlanTables<double> tp = stage_plan<double>(a.plan1, dttn_raw + align16((size_t)N * ld * sizeof(T)));
    const long ncol = a.ncol;
    const long ntiles = (ncol + C - 1) / C;
    for (long ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const long c0 = ti * C;
        const int nl = (int)min((long)C, ncol - c0);
        __syncthreads();   // the previous tile is stored (and the tables staged)
        for (int t = threadIdx.x; t < N * C; t += blockDim.x) {
            const int e = t / C, l = t - e * C;
            T v = make_double2(0.0, 0.0);
            if (l < nl) {
                const T* col = a.in + c0 + l;
                if (FWD) {
                    // v_e = x_{2e} (e < N/2), x_{2(N-1-e)+1} (e >= N/2); DST-II's (-1)^k on the odd ones
                    if (e < H) v = col[(long)(2 * e) * ncol];
                    else v = cscale(col[(long)(2 * (N - 1 - e) + 1) * ncol], KIND == 0 ? 1.0 : -1.0);
                } else {
                    // Z_j (phi: the weighted input; psib: Z'_j = c1 in_{N-j}, Z'_0 = 0) and Z_{N-j}
                    auto z = [&](int j) -> T {
                        if (j <= 0 || j >= N) return (KIND == 0 && j == 0) ? cscale(col[0], a.c0) : make_double2(0.0, 0.0);
                        return cscale(col[(long)(KIND == 0 ? j : N - j) * ncol], a.c1);
                    };
                    if (e == 0) v = cscale(z(0), 2.0);
                    else {
                        const T d = csub(z(e), cmul_si(z(N - e), 1));   // Z_j - i Z_{N-j}
                        v = cmul(d, a.tw[e]);
                    }
                }
            }
            buf[e * ld + l] = v;
        }
        fft_batch<false, double, 8>(buf, ld, C, a.plan1, FWD ? -1 : +1, tp.tw);   // synchronises
        for (int t = threadIdx.x; t < N * C; t += blockDim.x) {
            const int j = t / C, l = t - j * C;
            if (l >= nl) continue;
            T o;
            if (FWD) {
                // element jp of the DCT-II (phi: jp = j; psib: jp = N - j, and mode 0 is zero)
                const int jp = KIND == 0 ? j : N - j;
                if (KIND == 2 && j == 0) {
                    o = make_double2(0.0, 0.0);
                } else {
                    const T w = cconj(a.tw[jp]);
                    const T P = cmul(buf[tp.pos[jp] * ld + l], w);
                    const T Q = cmul(cconj(buf[tp.pos[(N - jp) % N] * ld + l]), w);
                    const double wt = (KIND == 0 && j == 0) ? a.c0 : a.c1;
                    o = cscale(make_double2(P.x + Q.x, P.y - Q.y), 0.5 * a.scale * wt);
                }
            } else {
                // x_{2n} = v_n, x_{2n+1} = v_{N-1-n}; DST-III's (-1)^k
                const int n = (j & 1) ? N - 1 - (j >> 1) : (j >> 1);
                o = cscale(buf[tp.pos[n] * ld + l], (KIND == 2 && (j & 1) ? -0.5 : 0.5) * a.scale);
            }
            a.out[(long)j * ncol + c0 + l] = o;
        }
    }
}

// opts the transform in to its dynamic shared memory on the current device
cudaError_t modes_setup() {
    cudaError_t e = cudaFuncSetAttribute(k_vert_mode<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_vert_mode_staged, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
#define DTT_ATTR(K, F)                                                                                        \
    if ((e = cudaFuncSetAttribute(k_vert_dtt<K, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024))) \
        return e;
    DTT_ATTR(0, true) DTT_ATTR(1, true) DTT_ATTR(2, true) DTT_ATTR(0, false) DTT_ATTR(1, false) DTT_ATTR(2, false)
#undef DTT_ATTR
#define DTTN_ATTR(K, F)                                                                                        \
    if ((e = cudaFuncSetAttribute(k_vert_dttn<K, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024))) \
        return e;
    DTTN_ATTR(0, true) DTTN_ATTR(2, true) DTTN_ATTR(0, false) DTTN_ATTR(2, false)
#undef DTTN_ATTR
    return cudaFuncSetAttribute(k_vert_mode<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

cudaError_t launch_vert_mode(const double2* in, double2* out, const double* A, int nz, long ncol, double scale,
                             cudaStream_t s) {
    if (!vert_mode_fits(nz)) return cudaErrorInvalidValue;
    // the staged form where two blocks fit an SM and nz is even (16-byte
    // matrix pairs); PS3D_VMODE_FORM=0|1 pins the form
    int form = (nz % 2 == 0 && vert_mode_smem_staged(nz) <= 113 * 1024) ? 1 : 0;
    if (const char* f = std::getenv("PS3D_VMODE_FORM"))
        if ((f[0] == '0' || f[0] == '1') && (f[0] == '0' || (nz % 2 == 0 && vert_mode_smem_staged(nz) <= 227 * 1024)))
            form = f[0] - '0';
    if (form == 1) {
        const size_t sm = vert_mode_smem_staged(nz);
        int dev = 0, nsm = 148, per = 1;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_vert_mode_staged, kVmThreads, sm) != cudaSuccess ||
            per < 1) {
            cudaGetLastError();
            per = 1;
        }
        const long ntiles = (ncol + kVmCols - 1) / kVmCols;
        const int blocks = (int)std::min<long>(ntiles, (long)nsm * per);
        k_vert_mode_staged<<<blocks, kVmThreads, sm, s>>>(in, out, A, nz, ncol, scale);
        return cudaGetLastError();
    }
    const size_t sm = vert_mode_smem(nz);
    const int blocks = (int)((ncol + kVmCols - 1) / kVmCols);
    if (nz % 2 == 0) k_vert_mode<true><<<blocks, kVmThreads, sm, s>>>(in, out, A, nz, ncol, scale);
    else k_vert_mode<false><<<blocks, kVmThreads, sm, s>>>(in, out, A, nz, ncol, scale);
    return cudaGetLastError();
}

bool vert_dtt_fits(int nz) { return fft_length_ok(2 * nz) && vert_dtt_smem(nz, kDttCols) <= 227 * 1024; }

cudaError_t launch_vert_dtt(const VertDttArgs& a0, int kind, bool fwd, cudaStream_t s) {
    VertDttArgs a = a0;
    // columns per block: kDttCols, or PS3D_DTT_COLS (a multiple of 8, up to 64) where it fits
    a.cols = kDttCols;
    if (const char* c = std::getenv("PS3D_DTT_COLS")) {
        const int v = std::atoi(c);
        if (v >= 8 && v <= 64 && v % 8 == 0 && vert_dtt_smem(a.nz, v) <= 227 * 1024) a.cols = v;
    }
    if (!vert_dtt_fits(a.nz) || a.plan.n != 2 * a.nz || kind < 0 || kind > 2) return cudaErrorInvalidValue;
    for (int q = 0; q < a.plan.nst; ++q)
        if (a.plan.r[q] > 8) return cudaErrorInvalidValue;   // the radix-8 build
    // phi and psib by FFTs of length nz where nz is even and that plan is set
    const bool half = kind != 1 && a.nz % 2 == 0 && a.plan1.n == a.nz && vert_dttn_smem(a.nz, a.cols) <= 227 * 1024;
    if (half)
        for (int q = 0; q < a.plan1.nst; ++q)
            if (a.plan1.r[q] > 8) return cudaErrorInvalidValue;
    const size_t sm = half ? vert_dttn_smem(a.nz, a.cols) : vert_dtt_smem(a.nz, a.cols);
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long ntiles = (a.ncol + a.cols - 1) / a.cols;
    const int per = std::max(1, (int)((227 * 1024) / (sm + 1024)));
    const int blocks = (int)std::min<long>(ntiles, (long)nsm * std::min(per, 8));
    if (half) {
        if (kind == 0) {
            if (fwd) k_vert_dttn<0, true><<<blocks, kDttThreads, sm, s>>>(a);
            else k_vert_dttn<0, false><<<blocks, kDttThreads, sm, s>>>(a);
        } else {
            if (fwd) k_vert_dttn<2, true><<<blocks, kDttThreads, sm, s>>>(a);
            else k_vert_dttn<2, false><<<blocks, kDttThreads, sm, s>>>(a);
        }
        return cudaGetLastError();
    }
#define DTT_L(K)                                                                                   \
    if (kind == K) {                                                                               \
        if (fwd) k_vert_dtt<K, true><<<blocks, kDttThreads, sm, s>>>(a);                          \
        else k_vert_dtt<K, false><<<blocks, kDttThreads, sm, s>>>(a);                             \
    }
    DTT_L(0) DTT_L(1) DTT_L(2)
#undef DTT_L
    return cudaGetLastError();
}

}  // namespace ps3d
