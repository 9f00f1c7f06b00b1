// poisson.cu — the FFT Poisson projection of pressure_solver.f90:2-120 on
// sm_100a, replacing P3DFFT's distributed transposes by one thread-block
// cluster per z-plane.
//
// K2 k_plane_fwd  : divergence (pressure_solver.f90:16-24) fused with the
//                   real-to-complex x FFT and the complex y FFT of one plane
//                   (my_fft_2D, my_fft.f90:170-178; P3DFFT op 'ffn').
//                   CTA r of the cluster transforms rows [r*R, (r+1)*R) along
//                   x and scatters each kx straight into the shared memory of
//                   the CTA that owns that kx column (distributed shared
//                   memory), which then transforms along y.  The plane never
//                   round-trips through HBM between the two directions.
// K3 k_thomas     : the vertical tridiagonal solves and the (0,0)-mode
//                   recurrence (pressure_solver.f90:33-53,126-162); one thread
//                   per (kx,ky) column, coefficients rebuilt from ksqr on the
//                   fly, the c' sweep checkpointed every 8 levels in shared
//                   memory and recomputed on the way back.
//    k_zsolve     : periodic branch (pressure_solver.f90:58-70): z FFT,
//                   -f/ksqr and inverse z FFT of a batch of columns in one pass.
// K4 k_plane_inv  : inverse y FFT, DSMEM gather, complex-to-real x FFT and the
//                   1/(Lx*Ly) scaling (my_ifft_2D, my_fft.f90:159-167).
// The real FFTs pack even/odd samples into a half-length complex FFT.
#include <cooperative_groups.h>
#include "engine.h"
#include "fft.cuh"

namespace cg = cooperative_groups;

namespace ps3d {

constexpr int kPlaneThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kPlaneThreads, 2) k_plane_fwd(const PlaneArgs a) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    T* colbuf = reinterpret_cast<T*>(smem_raw);
    T* rowbuf = colbuf + (size_t)a.ny * a.ldc;
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const long ioff = (long)inst * a.sN;
    const int rank = (int)cluster.block_rank();
    const long plane = (long)nx * ny;
    const int ldr = a.ldr, ldc = a.ldc, cpc = a.cols_per_cta;
    const double* au = a.u + ioff;
    const double* av = a.v + ioff;
    const double* aw = a.w + ioff;
    const double* asrc = a.src ? a.src + ioff : nullptr;
    cluster.sync();   // every CTA of the cluster is running before DSMEM stores
    const int jb = rank * a.rows_per_cta;
    for (int jc = 0; jc < a.rows_per_cta; jc += a.row_chunk) {
        const int nr = min(a.row_chunk, a.rows_per_cta - jc);
        for (int t = threadIdx.x; t < nr * n2; t += blockDim.x) {
            const int rr = t / n2, m = t - rr * n2;
            const int j = jb + jc + rr;
            const long g = (long)k * plane + (long)j * nx + 2 * m;
            double d0, d1;
            if (a.mode == 0) {
                const double2 uu = *reinterpret_cast<const double2*>(au + g);
                const double um = au[g - 2 * m + wrap(2 * m - 1, nx)];
                const long gv = g + (long)(wrap(j - 1, ny) - j) * nx;
                const long gw = g + (long)(wrap(k - 1, nz) - k) * plane;
                const double2 vv = *reinterpret_cast<const double2*>(av + g);
                const double2 vm = *reinterpret_cast<const double2*>(av + gv);
                const double2 ww = *reinterpret_cast<const double2*>(aw + g);
                const double2 wm = *reinterpret_cast<const double2*>(aw + gw);
                d0 = ((uu.x - um) * a.rdx + (vv.x - vm.x) * a.rdy + (ww.x - wm.x) * a.rdz) * a.rdt;
                d1 = ((uu.y - uu.x) * a.rdx + (vv.y - vm.y) * a.rdy + (ww.y - wm.y) * a.rdz) * a.rdt;
            } else {
                const double2 s = *reinterpret_cast<const double2*>(asrc + g);
                d0 = s.x; d1 = s.y;
            }
            rowbuf[m * ldr + rr] = mk<R>((R)d0, (R)d1);
        }
        fft_batch<false, R>(rowbuf, ldr, nr, a.px, -1);
        // unpack the half-length transform: X_k = E_k + W^k O_k
        for (int t = threadIdx.x; t < nr * (n2 + 1); t += blockDim.x) {
            const int kx = t / nr, rr = t - kx * nr;
            const int k1 = (kx == n2) ? 0 : kx;
            const int k2 = (kx == 0) ? 0 : n2 - kx;
            const T Zk = rowbuf[a.px.pos[k1] * ldr + rr];
            const T Zc = cconj(rowbuf[a.px.pos[k2] * ldr + rr]);
            const T E = cscale(cadd(Zk, Zc), (R)0.5);
            const T H = cscale(cmul_si(csub(Zk, Zc), -1), (R)0.5);   // O_k = -i (Zk - Zc)/2
            const double2 wd = __ldg(a.twx + kx);
            const T X = cadd(E, cmul(mk<R>((R)wd.x, (R)wd.y), H));
            const int owner = kx / cpc, c = kx - owner * cpc;
            T* dst = cluster.map_shared_rank(colbuf, owner);
            dst[(jb + jc + rr) * ldc + c] = X;
        }
        __syncthreads();
    }
    cluster.sync();   // all rows delivered
    const int c0 = rank * cpc;
    const int ncol = max(0, min(cpc, nxh - c0));
    if (ncol > 0) fft_batch<false, R>(colbuf, ldc, ncol, a.py, -1);
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM;
    const R sc = (R)a.scale;
    for (int t = threadIdx.x; t < ny * ncol; t += blockDim.x) {
        const int ky = t / ncol, c = t - ky * ncol;
        spec[((long)k * ny + ky) * nxh + c0 + c] = cscale(colbuf[a.py.pos[ky] * ldc + c], sc);
    }
}

template <typename R>
__global__ void __launch_bounds__(kPlaneThreads, 2) k_plane_inv(const PlaneArgs a) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    T* colbuf = reinterpret_cast<T*>(smem_raw);
    T* rowbuf = colbuf + (size_t)a.ny * a.ldc;
    const int nx = a.nx, ny = a.ny, nxh = a.nxh, n2 = nx / 2;
    const int inst = blockIdx.y / a.nz;
    const int k = blockIdx.y - inst * a.nz;
    double* out = a.out + (long)inst * a.sN;
    const int rank = (int)cluster.block_rank();
    const long plane = (long)nx * ny;
    const int ldr = a.ldr, ldc = a.ldc, cpc = a.cols_per_cta;
    const int c0 = rank * cpc;
    const int ncol = max(0, min(cpc, nxh - c0));
    const T* spec = reinterpret_cast<const T*>(a.spec) + (long)inst * a.sM;
    for (int t = threadIdx.x; t < ny * ncol; t += blockDim.x) {
        const int ky = t / ncol, c = t - ky * ncol;
        colbuf[ky * ldc + c] = spec[((long)k * ny + ky) * nxh + c0 + c];
    }
    if (ncol > 0) fft_batch<false, R>(colbuf, ldc, ncol, a.py, +1);
    cluster.sync();   // every column transformed; gather rows from the owners
    const int jb = rank * a.rows_per_cta;
    for (int jc = 0; jc < a.rows_per_cta; jc += a.row_chunk) {
        const int nr = min(a.row_chunk, a.rows_per_cta - jc);
        for (int t = threadIdx.x; t < nr * n2; t += blockDim.x) {
            const int kk = t / nr, rr = t - kk * nr;
            const int prow = a.py.pos[jb + jc + rr];
            const int kc = n2 - kk;
            const int o1 = kk / cpc, o2 = kc / cpc;
            const T* s1 = cluster.map_shared_rank(colbuf, o1);
            const T* s2 = cluster.map_shared_rank(colbuf, o2);
            T Xk = s1[prow * ldc + (kk - o1 * cpc)];
            T Xc = s2[prow * ldc + (kc - o2 * cpc)];
            if (kk == 0) { Xk.y = (R)0; Xc.y = (R)0; }   // c2r ignores Im of DC and Nyquist
            Xc = cconj(Xc);
            const double2 wd = __ldg(a.twx + kk);
            const T wb = mk<R>((R)wd.x, (R)-wd.y);      // W^{-k}
            const T Z = cadd(cadd(Xk, Xc), cmul_si(cmul(wb, csub(Xk, Xc)), +1));
            rowbuf[kk * ldr + rr] = Z;
        }
        fft_batch<false, R>(rowbuf, ldr, nr, a.px, +1);
        const double sc = a.scale;
        for (int t = threadIdx.x; t < nr * n2; t += blockDim.x) {
            const int rr = t / n2, m = t - rr * n2;
            const int j = jb + jc + rr;
            const T z = rowbuf[a.px.pos[m] * ldr + rr];
            const long g = (long)k * plane + (long)j * nx + 2 * m;
            double2 o = make_double2((double)z.x * sc, (double)z.y * sc);
            if (a.beta != 0.0) {
                const double2 prev = *reinterpret_cast<const double2*>(out + g);
                o.x = o.x + a.beta * prev.x; o.y = o.y + a.beta * prev.y;
            }
            *reinterpret_cast<double2*>(out + g) = o;
        }
        __syncthreads();
    }
    cluster.sync();   // keep this CTA's columns alive until every reader is done
}

// ---------------------------------------------------------------------------
// K3, rigid lid: batched Thomas along z (pressure_solver.f90:33-53, 126-162)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(128) k_thomas(const ColumnArgs a) {
    using T = cpx<R>;
    extern __shared__ double cps[];   // [nz/8 + 1][blockDim.x] checkpoints of c'
    const long ncols = (long)a.nxh * a.ny;
    const long cg_ = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (cg_ >= ncols * a.batch) return;
    const long inst = cg_ / ncols;
    const long c = cg_ - inst * ncols;
    T* spec = reinterpret_cast<T*>(a.spec) + inst * a.sM;
    const int nz = a.nz;
    const int i = a.layout ? (int)(c / a.ny) : (int)(c % a.nxh);
    const int j = a.layout ? (int)(c % a.ny) : (int)(c / a.nxh);
    const double ks = a.hkx[i] + a.hky[j];
    const double fxa = a.fxa;
    if (ks > 0) {
        // levels are processed in chunks of 8: the 8 loads of a chunk are
        // issued together, then the serial recurrence runs on registers
        const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
        double cp = 0.0, dpx = 0.0, dpy = 0.0;
        for (int kb = 0; kb < nz; kb += 8) {
            T d[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (kb + q < nz) d[q] = spec[c + (long)(kb + q) * ncols];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = kb + q;
                if (k < nz) {
                    const double bk = (k == 0 || k == nz - 1) ? bend : bmid;
                    if (k == 0) {
                        cp = fxa / bk;                       // cp(1) = c(1)/b(1)
                        dpx = (double)d[q].x / bk;           // dp(1) = d(1)/b(1)
                        dpy = (double)d[q].y / bk;
                    } else {
                        const double r = 1.0 / (bk - cp * fxa);
                        cp = fxa * r;
                        dpx = ((double)d[q].x - dpx * fxa) * r;
                        dpy = ((double)d[q].y - dpy * fxa) * r;
                    }
                    if (q == 0) cps[(kb >> 3) * blockDim.x + threadIdx.x] = cp;
                    d[q] = mk<R>((R)dpx, (R)dpy);
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (kb + q < nz) spec[c + (long)(kb + q) * ncols] = d[q];
        }
        double xx = dpx, xy = dpy;   // x(nz) = dp(nz)
        for (int sg = (nz - 1) >> 3; sg >= 0; --sg) {
            const int kb = sg * 8;
            T d[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (kb + q < nz - 1) d[q] = spec[c + (long)(kb + q) * ncols];
            double cpl[8];
            cpl[0] = cps[sg * blockDim.x + threadIdx.x];
#pragma unroll
            for (int q = 1; q < 8; ++q) {
                const int k = kb + q;
                if (k < nz) {
                    const double bk = (k == nz - 1) ? bend : bmid;
                    cpl[q] = fxa * (1.0 / (bk - cpl[q - 1] * fxa));
                } else {
                    cpl[q] = 0.0;
                }
            }
#pragma unroll
            for (int q = 7; q >= 0; --q) {
                if (kb + q >= nz - 1) continue;
                xx = (double)d[q].x - cpl[q] * xx;
                xy = (double)d[q].y - cpl[q] * xy;
                d[q] = mk<R>((R)xx, (R)xy);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (kb + q < nz - 1) spec[c + (long)(kb + q) * ncols] = d[q];
        }
    } else {
        // (0,0) mode: p(1) = 0, p(2) = f(1) dz^2 dsqr, p(k+1) = 2p(k) - p(k-1) + f(k) dz^2 dsqr
        const double h = a.dz2dsqr;
        T prev_orig = spec[c];
        spec[c] = mk<R>((R)0, (R)0);
        if (nz > 1) {
            double x0x = 0.0, x0y = 0.0;
            const T o1 = spec[c + ncols];
            double x1x = (double)prev_orig.x * h, x1y = (double)prev_orig.y * h;
            spec[c + ncols] = mk<R>((R)x1x, (R)x1y);
            T orig_km1 = o1;
            for (int k = 2; k < nz; ++k) {
                const T ok = spec[c + (long)k * ncols];
                const double xkx = 2 * x1x - x0x + (double)orig_km1.x * h;
                const double xky = 2 * x1y - x0y + (double)orig_km1.y * h;
                spec[c + (long)k * ncols] = mk<R>((R)xkx, (R)xky);
                x0x = x1x; x0y = x1y; x1x = xkx; x1y = xky;
                orig_km1 = ok;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// K3, triply periodic: z FFT, spectral division, inverse z FFT
// (pressure_solver.f90:58-70; my_fft_3D/my_ifft_3D z leg)
// ---------------------------------------------------------------------------
constexpr int kZLines = 32;

template <typename R>
__global__ void __launch_bounds__(256) k_zsolve(const ColumnArgs a) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int ld = kZLines + 1;
    const long ncols = (long)a.nxh * a.ny;
    const long bpi = (ncols + kZLines - 1) / kZLines;   // blocks per instance
    const long inst = blockIdx.x / bpi;
    const long c0 = (blockIdx.x - inst * bpi) * (long)kZLines;
    const int nl = (int)min((long)kZLines, ncols - c0);
    const int nz = a.nz;
    T* spec = reinterpret_cast<T*>(a.spec) + inst * a.sM;
    for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
        const int k = t / nl, l = t - k * nl;
        const int slot = (a.op == 2) ? a.pz.pos[k] : k;
        buf[slot * ld + l] = spec[c0 + l + (long)k * ncols];
    }
    if (a.op == 2) {
        fft_batch<true, R>(buf, ld, nl, a.pz, +1);
    } else {
        fft_batch<false, R>(buf, ld, nl, a.pz, -1);
        const R sc = (R)a.scale;
        for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
            const int p = t / nl, l = t - p * nl;
            T v = cscale(buf[p * ld + l], sc);
            if (a.op == 0) {
                const long c = c0 + l;
                const int i = a.layout ? (int)(c / a.ny) : (int)(c % a.nxh);
                const int j = a.layout ? (int)(c % a.ny) : (int)(c / a.nxh);
                const int k = a.pz.ipos[p];
                const double ks = a.hkx[i] + a.hky[j] + a.hkz[k];
                if (ks > 0.0) { v.x = (R)(-(double)v.x / ks); v.y = (R)(-(double)v.y / ks); }
                else { v.x = (R)0; v.y = (R)0; }
            }
            buf[p * ld + l] = v;
        }
        if (a.op == 0) fft_batch<true, R>(buf, ld, nl, a.pz, +1);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
        const int k = t / nl, l = t - k * nl;
        const int slot = (a.op == 1) ? a.pz.pos[k] : k;
        spec[c0 + l + (long)k * ncols] = buf[slot * ld + l];
    }
}

// ---------------------------------------------------------------------------
// Plane transforms, second implementation: a rows pass and a y-lines pass.
// The spectral array is [k][kx][ky], so every kx line is contiguous in ky:
// the rows pass writes each kx as one coalesced run of tj rows, the y-lines
// pass loads and stores whole lines, and the vertical solves read columns
// with consecutive threads on consecutive ky.  The intermediate makes one
// extra trip through memory (largely L2-resident), in exchange for
// independent CTAs with small shared memory and no cluster barriers.
// Digit-reversed data are always read in shared-memory order and scattered
// to global memory instead, which keeps the shared-memory accesses free of
// bank conflicts.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256, 2) k_rows_fwd(const PlaneArgs a) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int tj = a.tj, ld = tj | 1;
    const int jb = blockIdx.x * tj;
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const long ioff = (long)inst * a.sN;
    const long plane = (long)nx * ny;
    const double* au = a.u + ioff;
    const double* av = a.v + ioff;
    const double* aw = a.w + ioff;
    const double* asrc = a.src ? a.src + ioff : nullptr;
    for (int t = threadIdx.x; t < tj * n2; t += blockDim.x) {
        const int rr = t / n2, m = t - rr * n2;
        const int j = jb + rr;
        const long g = (long)k * plane + (long)j * nx + 2 * m;
        double d0, d1;
        if (a.mode == 0) {
            const double2 uu = *reinterpret_cast<const double2*>(au + g);
            const double um = au[g - 2 * m + wrap(2 * m - 1, nx)];
            const long gv = g + (long)(wrap(j - 1, ny) - j) * nx;
            const long gw = g + (long)(wrap(k - 1, nz) - k) * plane;
            const double2 vv = *reinterpret_cast<const double2*>(av + g);
            const double2 vm = *reinterpret_cast<const double2*>(av + gv);
            const double2 ww = *reinterpret_cast<const double2*>(aw + g);
            const double2 wm = *reinterpret_cast<const double2*>(aw + gw);
            d0 = ((uu.x - um) * a.rdx + (vv.x - vm.x) * a.rdy + (ww.x - wm.x) * a.rdz) * a.rdt;
            d1 = ((uu.y - uu.x) * a.rdx + (vv.y - vm.y) * a.rdy + (ww.y - wm.y) * a.rdz) * a.rdt;
        } else {
            const double2 sv = *reinterpret_cast<const double2*>(asrc + g);
            d0 = sv.x; d1 = sv.y;
        }
        buf[m * ld + rr] = mk<R>((R)d0, (R)d1);
    }
    fft_batch<false, R>(buf, ld, tj, a.px, -1);
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)k * nxh * ny;
    for (int t = threadIdx.x; t < tj * (n2 + 1); t += blockDim.x) {
        const int kx = t / tj, rr = t - kx * tj;
        const int k1 = (kx == n2) ? 0 : kx;
        const int k2 = (kx == 0) ? 0 : n2 - kx;
        const T Zk = buf[a.px.pos[k1] * ld + rr];
        const T Zc = cconj(buf[a.px.pos[k2] * ld + rr]);
        const T E = cscale(cadd(Zk, Zc), (R)0.5);
        const T H = cscale(cmul_si(csub(Zk, Zc), -1), (R)0.5);
        const double2 wd = __ldg(a.twx + kx);
        spec[(long)kx * ny + jb + rr] = cadd(E, cmul(mk<R>((R)wd.x, (R)wd.y), H));
    }
}

// one y transform of every kx line of a plane, in place on [k][kx][ky]
template <typename R>
__global__ void __launch_bounds__(256, 2) k_ylines(const PlaneArgs a, int sign, double scale) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int ny = a.ny, nz = a.nz, nxh = a.nxh;
    const int ly = a.ly, ld = ly | 1;
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const int l0 = blockIdx.x * ly;
    const int nl = min(ly, nxh - l0);
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + ((long)k * nxh + l0) * ny;
    for (int t = threadIdx.x; t < nl * ny; t += blockDim.x) {
        const int line = t / ny, e = t - line * ny;
        buf[e * ld + line] = spec[(long)line * ny + e];
    }
    fft_batch<false, R>(buf, ld, nl, a.py, sign);
    const R sc = (R)scale;
    for (int t = threadIdx.x; t < nl * ny; t += blockDim.x) {
        const int line = t / ny, q = t - line * ny;   // q: position in shared memory
        spec[(long)line * ny + a.py.ipos[q]] = cscale(buf[q * ld + line], sc);
    }
}

template <typename R>
__global__ void __launch_bounds__(256, 2) k_rows_inv(const PlaneArgs a) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int tj = a.tj, ld = tj | 1;
    const int jb = blockIdx.x * tj;
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const long plane = (long)nx * ny;
    const T* spec = reinterpret_cast<const T*>(a.spec) + (long)inst * a.sM + (long)k * nxh * ny;
    double* out = a.out + (long)inst * a.sN;
    for (int t = threadIdx.x; t < tj * n2; t += blockDim.x) {
        const int kk = t / tj, rr = t - kk * tj;
        T Xk = spec[(long)kk * ny + jb + rr];
        T Xc = spec[(long)(n2 - kk) * ny + jb + rr];
        if (kk == 0) { Xk.y = (R)0; Xc.y = (R)0; }   // c2r ignores Im of DC and Nyquist
        Xc = cconj(Xc);
        const double2 wd = __ldg(a.twx + kk);
        const T wb = mk<R>((R)wd.x, (R)-wd.y);
        buf[kk * ld + rr] = cadd(cadd(Xk, Xc), cmul_si(cmul(wb, csub(Xk, Xc)), +1));
    }
    fft_batch<false, R>(buf, ld, tj, a.px, +1);
    const double sc = a.scale;
    for (int t = threadIdx.x; t < tj * n2; t += blockDim.x) {
        const int rr = t / n2, q = t - rr * n2;
        const int m = a.px.ipos[q];
        const T z = buf[q * ld + rr];
        const long g = (long)k * plane + (long)(jb + rr) * nx + 2 * m;
        double2 o = make_double2((double)z.x * sc, (double)z.y * sc);
        if (a.beta != 0.0) {
            const double2 prev = *reinterpret_cast<const double2*>(out + g);
            o.x = o.x + a.beta * prev.x; o.y = o.y + a.beta * prev.y;
        }
        *reinterpret_cast<double2*>(out + g) = o;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
size_t rows_smem(const PlaneArgs& a, bool fp32) {
    return (size_t)(a.nx / 2) * (a.tj | 1) * (fp32 ? sizeof(float2) : sizeof(double2));
}
size_t ylines_smem(const PlaneArgs& a, bool fp32) {
    return (size_t)a.ny * (a.ly | 1) * (fp32 ? sizeof(float2) : sizeof(double2));
}

template <typename R>
static cudaError_t launch_split_t(const PlaneArgs& a, bool fwd, cudaStream_t s) {
    const int nb = std::max(1, a.batch);
    const dim3 grows(a.ny / a.tj, a.nz * nb), glines((a.nxh + a.ly - 1) / a.ly, a.nz * nb);
    const size_t smr = rows_smem(a, sizeof(R) == 4), sml = ylines_smem(a, sizeof(R) == 4);
    if (fwd) {
        k_rows_fwd<R><<<grows, 256, smr, s>>>(a);
        k_ylines<R><<<glines, 256, sml, s>>>(a, -1, a.scale);
    } else {
        k_ylines<R><<<glines, 256, sml, s>>>(a, +1, 1.0);
        k_rows_inv<R><<<grows, 256, smr, s>>>(a);
    }
    return cudaGetLastError();
}

size_t plane_fwd_smem(const PlaneArgs& a, bool fp32) {
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    return ((size_t)a.ny * a.ldc + (size_t)(a.nx / 2) * a.ldr) * es;
}
size_t plane_inv_smem(const PlaneArgs& a, bool fp32) { return plane_fwd_smem(a, fp32); }

template <typename R>
static cudaError_t setup_t() {
    cudaError_t e;
    const int maxsm = 227 * 1024;
    if ((e = cudaFuncSetAttribute(k_plane_fwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_inv<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_fwd<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_inv<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
    if ((e = cudaFuncSetAttribute(k_zsolve<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_fwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_inv<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_ylines<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    return cudaSuccess;
}
cudaError_t plane_setup(bool fp32) { return fp32 ? setup_t<float>() : setup_t<double>(); }

template <typename R, bool FWD>
static cudaError_t launch_plane_t(const PlaneArgs& a, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.C, a.nz * std::max(1, a.batch), 1);
    cfg.blockDim = dim3(kPlaneThreads, 1, 1);
    cfg.dynamicSmemBytes = plane_fwd_smem(a, sizeof(R) == 4);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (FWD) return cudaLaunchKernelEx(&cfg, k_plane_fwd<R>, a);
    return cudaLaunchKernelEx(&cfg, k_plane_inv<R>, a);
}
template <typename R, bool FWD>
static int max_clusters_t(const PlaneArgs& a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.C, a.nz * std::max(1, a.batch), 1);
    cfg.blockDim = dim3(kPlaneThreads, 1, 1);
    cfg.dynamicSmemBytes = plane_fwd_smem(a, sizeof(R) == 4);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    cudaError_t e = FWD ? cudaOccupancyMaxActiveClusters(&n, k_plane_fwd<R>, &cfg)
                        : cudaOccupancyMaxActiveClusters(&n, k_plane_inv<R>, &cfg);
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}
int plane_max_clusters(const PlaneArgs& a, bool fp32, bool fwd) {
    if (fp32) return fwd ? max_clusters_t<float, true>(a) : max_clusters_t<float, false>(a);
    return fwd ? max_clusters_t<double, true>(a) : max_clusters_t<double, false>(a);
}

cudaError_t launch_plane_fwd(const PlaneArgs& a, bool fp32, cudaStream_t s) {
    if (a.impl == 1) return fp32 ? launch_split_t<float>(a, true, s) : launch_split_t<double>(a, true, s);
    return fp32 ? launch_plane_t<float, true>(a, s) : launch_plane_t<double, true>(a, s);
}
cudaError_t launch_plane_inv(const PlaneArgs& a, bool fp32, cudaStream_t s) {
    if (a.impl == 1) return fp32 ? launch_split_t<float>(a, false, s) : launch_split_t<double>(a, false, s);
    return fp32 ? launch_plane_t<float, false>(a, s) : launch_plane_t<double, false>(a, s);
}

cudaError_t launch_thomas(const ColumnArgs& a, bool fp32, cudaStream_t s) {
    const long ncols = (long)a.nxh * a.ny * std::max(1, a.batch);
    const int threads = 128;
    const int blocks = (int)((ncols + threads - 1) / threads);
    const size_t sm = (size_t)((a.nz + 7) / 8 + 1) * threads * sizeof(double);
    if (fp32) k_thomas<float><<<blocks, threads, sm, s>>>(a);
    else k_thomas<double><<<blocks, threads, sm, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_zsolve(const ColumnArgs& a, bool fp32, cudaStream_t s) {
    const long ncols = (long)a.nxh * a.ny;
    const int blocks = (int)(((ncols + kZLines - 1) / kZLines) * std::max(1, a.batch));
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    const size_t sm = (size_t)a.nz * (kZLines + 1) * es;
    if (fp32) k_zsolve<float><<<blocks, 256, sm, s>>>(a);
    else k_zsolve<double><<<blocks, 256, sm, s>>>(a);
    return cudaGetLastError();
}

}  // namespace ps3d
