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
//                   per (kx,ky) column and part, FP64 recurrences checkpointed
//                   every 8 levels in shared memory, the pivots formed on the fly.
//    k_zsolve     : periodic branch (pressure_solver.f90:58-70): z FFT,
//                   -f/ksqr and inverse z FFT of a batch of columns in one pass.
// K4 k_plane_inv  : inverse y FFT, DSMEM gather, complex-to-real x FFT and the
//                   1/(Lx*Ly) scaling (my_ifft_2D, my_fft.f90:159-167).
// The real FFTs pack even/odd samples into a half-length complex FFT.
#include <cooperative_groups.h>
#include <cstdlib>
#include "engine.h"
#include "async.cuh"
#include "fft.cuh"

namespace cg = cooperative_groups;

namespace ps3d {

constexpr int kPlaneThreads = 256;

// blocks per SM the plane kernels are built for: the radix-16 instantiation
// needs ~128 FP64 registers, the radix-8 one fits in 80
template <int MAXR> constexpr int plane_min_blocks() { return MAXR >= 16 ? 2 : 3; }
template <typename R, int MAXR> constexpr int lines_min_blocks() { return MAXR >= 16 ? 2 : 4; }

// the L2 policies of a kernel (PlaneArgs/ColumnArgs::l2hint): the spectra
// evict_last while later passes read them, evict_first at their last read;
// the real fields default priority (evict_first with l2hint == 2)
__device__ __forceinline__ unsigned long long pol_keep(int h) { return l2_policy(h ? kL2Keep : kL2Normal); }
__device__ __forceinline__ unsigned long long pol_last(int h) { return l2_policy(h ? kL2Stream : kL2Normal); }
__device__ __forceinline__ unsigned long long pol_field(int h) { return l2_policy(h == 2 ? kL2Stream : kL2Normal); }

// Divergence of the pair of points (2m, 2m+1) of row j in plane k, divided by
// dt (pressure_solver.f90:16-24), or the pair of source values (mode 1).
__device__ __forceinline__ double2 plane_source_pair(const PlaneArgs& a, const double* au, const double* av,
                                                     const double* aw, const double* asrc, int k, int j, int m,
                                                     unsigned long long pol) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long plane = (long)nx * ny;
    const long g = (long)k * plane + (long)j * nx + 2 * m;
    if (a.mode == 1) return ldg_l2(reinterpret_cast<const double2*>(asrc + g), pol);
    const long gum = g - 2 * m + wrap(2 * m - 1, nx);
    const long gv = g + (long)(wrap(j - 1, ny) - j) * nx;
    const long gw = g + (long)(wrap(k - 1, nz) - k) * plane;
    double2 uu = ldg_l2(reinterpret_cast<const double2*>(au + g), pol);
    double um = ldg_l2(au + gum, pol);
    double2 vv = ldg_l2(reinterpret_cast<const double2*>(av + g), pol);
    double2 vm = ldg_l2(reinterpret_cast<const double2*>(av + gv), pol);
    double2 ww = ldg_l2(reinterpret_cast<const double2*>(aw + g), pol);
    double2 wm = ldg_l2(reinterpret_cast<const double2*>(aw + gw), pol);
    if (a.mode == 2) {
        // u - dt grad p at the points the divergence reads (pressure_solver.f90:98-110)
        const double* pc = a.pc + (au - a.u);   // same instance offset as the fields
        const long gpe = g - 2 * m + wrap(2 * m + 2, nx);
        const long gpn = g + (long)(wrap(j + 1, ny) - j) * nx;
        const long gpu = g + (long)(wrap(k + 1, nz) - k) * plane;
        const double2 p0 = ldg_l2(reinterpret_cast<const double2*>(pc + g), pol);
        const double pw = ldg_l2(pc + gum, pol), pe = ldg_l2(pc + gpe, pol);
        const double2 ps = ldg_l2(reinterpret_cast<const double2*>(pc + gv), pol);
        const double2 pn = ldg_l2(reinterpret_cast<const double2*>(pc + gpn), pol);
        const double2 pd = ldg_l2(reinterpret_cast<const double2*>(pc + gw), pol);
        const double2 pu = ldg_l2(reinterpret_cast<const double2*>(pc + gpu), pol);
        const double dt = a.dtp, dtw = a.dtwp;
        um = um - dt * (p0.x - pw) * a.rdx;
        uu.x = uu.x - dt * (p0.y - p0.x) * a.rdx;
        uu.y = uu.y - dt * (pe - p0.y) * a.rdx;
        vv.x = vv.x - dt * (pn.x - p0.x) * a.rdy;
        vv.y = vv.y - dt * (pn.y - p0.y) * a.rdy;
        vm.x = vm.x - dt * (p0.x - ps.x) * a.rdy;
        vm.y = vm.y - dt * (p0.y - ps.y) * a.rdy;
        const int kg = k + a.kofs, nzg = a.nzg ? a.nzg : nz;   // global level (z-slabs)
        if (a.rigid && kg == nzg - 1) {
            ww.x = 0.0; ww.y = 0.0;
        } else {
            ww.x = ww.x - dtw * (pu.x - p0.x) * a.rdz;
            ww.y = ww.y - dtw * (pu.y - p0.y) * a.rdz;
        }
        if (a.rigid && kg == 0) {   // the level below is the (global) top
            wm.x = 0.0; wm.y = 0.0;
        } else {
            wm.x = wm.x - dtw * (p0.x - pd.x) * a.rdz;
            wm.y = wm.y - dtw * (p0.y - pd.y) * a.rdz;
        }
    }
    double2 d;
    d.x = ((uu.x - um) * a.rdx + (vv.x - vm.x) * a.rdy + (ww.x - wm.x) * a.rdz) * a.rdt;
    d.y = ((uu.y - uu.x) * a.rdx + (vv.y - vm.y) * a.rdy + (ww.y - wm.y) * a.rdz) * a.rdt;
    return d;
}

// exp(-2 pi i t / nx), t = 0..nx/2, staged in the working precision
template <typename R>
__device__ cpx<R>* stage_twx(const PlaneArgs& a, unsigned char* dst) {
    cpx<R>* t = reinterpret_cast<cpx<R>*>(dst);
    for (int e = threadIdx.x; e < a.nxh; e += blockDim.x) {
        const double2 w = __ldg(a.twx + e);
        t[e] = mk<R>((R)w.x, (R)w.y);
    }
    return t;
}

// bytes of shared memory after the work buffers: tables of x, of y, twx
PS3D_HD size_t tables_x_bytes(const PlaneArgs& a, size_t es) {
    return plan_tables_bytes(a.nx / 2, es) + align16((size_t)a.nxh * es);
}
PS3D_HD size_t tables_y_bytes(const PlaneArgs& a, size_t es) { return plan_tables_bytes(a.ny, es); }

// X_k = E_k + W^k O_k from the half-length transform Z (r2c unpack)
template <typename R>
__device__ __forceinline__ cpx<R> r2c_unpack(cpx<R> Zk, cpx<R> Zc, cpx<R> w) {
    using T = cpx<R>;
    Zc = cconj(Zc);
    const T E = cscale(cadd(Zk, Zc), (R)0.5);
    const T H = cscale(cmul_si(csub(Zk, Zc), -1), (R)0.5);   // O_k = -i (Zk - Zc)/2
    return cadd(E, cmul(w, H));
}
// Z_k = (X_k + conj X_{n2-k}) + i W^{-k} (X_k - conj X_{n2-k}) (c2r pack; the
// factor 1/2 is in the caller's scale)
template <typename R>
__device__ __forceinline__ cpx<R> c2r_pack(cpx<R> Xk, cpx<R> Xc, cpx<R> w, bool dc) {
    using T = cpx<R>;
    if (dc) { Xk.y = (R)0; Xc.y = (R)0; }   // c2r ignores Im of DC and Nyquist
    Xc = cconj(Xc);
    const T wb = mk<R>(w.x, -w.y);           // W^{-k}
    return cadd(cadd(Xk, Xc), cmul_si(cmul(wb, csub(Xk, Xc)), +1));
}

// ---------------------------------------------------------------------------
// K2/K4, first implementation: one thread-block cluster per z-plane
// ---------------------------------------------------------------------------
template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_blocks<MAXR>()) k_plane_fwd(const PlaneArgs a) {
    const unsigned long long pfield = pol_field(a.l2hint), pkeep = pol_keep(a.l2hint);
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    T* colbuf = reinterpret_cast<T*>(smem_raw);
    T* rowbuf = colbuf + (size_t)a.ny * a.ldc;
    unsigned char* tail = smem_raw + align16(((size_t)a.ny * a.ldc + (size_t)(a.nx / 2) * a.ldr) * sizeof(T));
    const PlanTables<R> tx = stage_plan<R>(a.px, tail);
    const T* twx = stage_twx<R>(a, tail + plan_tables_bytes(a.nx / 2, sizeof(T)));
    const PlanTables<R> ty = stage_plan<R>(a.py, tail + tables_x_bytes(a, sizeof(T)));
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const long ioff = (long)inst * a.sN;
    const int rank = (int)cluster.block_rank();
    const int ldr = a.ldr, ldc = a.ldc, cpc = a.cols_per_cta;
    const double* au = a.u + ioff;
    const double* av = a.v + ioff;
    const double* aw = a.w + ioff;
    const double* asrc = a.src ? a.src + ioff : nullptr;
    cluster.sync();   // every CTA of the cluster is running before DSMEM stores; tables staged
    const int jb = rank * a.rows_per_cta;
    constexpr int LB = 2;
    for (int jc = 0; jc < a.rows_per_cta; jc += a.row_chunk) {
        const int nr = min(a.row_chunk, a.rows_per_cta - jc);
        const int total = nr * n2;
        for (int t0 = threadIdx.x; t0 < total; t0 += LB * blockDim.x) {
            double2 d[LB];
#pragma unroll
            for (int q = 0; q < LB; ++q) {
                const int t = t0 + q * blockDim.x;
                if (t < total) {
                    const int rr = t / n2, m = t - rr * n2;
                    d[q] = plane_source_pair(a, au, av, aw, asrc, k, jb + jc + rr, m, pfield);
                }
            }
#pragma unroll
            for (int q = 0; q < LB; ++q) {
                const int t = t0 + q * blockDim.x;
                if (t < total) {
                    const int rr = t / n2, m = t - rr * n2;
                    rowbuf[m * ldr + rr] = mk<R>((R)d[q].x, (R)d[q].y);
                }
            }
        }
        fft_batch<false, R, MAXR>(rowbuf, ldr, nr, a.px, -1, tx.tw);
        for (int t = threadIdx.x; t < nr * (n2 + 1); t += blockDim.x) {
            const int kx = t / nr, rr = t - kx * nr;
            const int k1 = (kx == n2) ? 0 : kx;
            const int k2 = (kx == 0) ? 0 : n2 - kx;
            const T X = r2c_unpack<R>(rowbuf[tx.pos[k1] * ldr + rr], rowbuf[tx.pos[k2] * ldr + rr], twx[kx]);
            const int owner = kx / cpc, c = kx - owner * cpc;
            T* dst = cluster.map_shared_rank(colbuf, owner);
            dst[(jb + jc + rr) * ldc + c] = X;
        }
        __syncthreads();
    }
    cluster.sync();   // all rows delivered
    const int c0 = rank * cpc;
    const int ncol = max(0, min(cpc, nxh - c0));
    fft_batch<false, R, MAXR>(colbuf, ldc, ncol, a.py, -1, ty.tw);
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM;
    const R sc = (R)a.scale;
    for (int t = threadIdx.x; t < ny * ncol; t += blockDim.x) {
        const int ky = t / ncol, c = t - ky * ncol;
        st_l2(&spec[((long)k * ny + ky) * nxh + c0 + c], cscale(colbuf[ty.pos[ky] * ldc + c], sc), pkeep);
    }
}

template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_blocks<MAXR>()) k_plane_inv(const PlaneArgs a) {
    const unsigned long long plast = pol_last(a.l2hint);
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    T* colbuf = reinterpret_cast<T*>(smem_raw);
    T* rowbuf = colbuf + (size_t)a.ny * a.ldc;
    unsigned char* tail = smem_raw + align16(((size_t)a.ny * a.ldc + (size_t)(a.nx / 2) * a.ldr) * sizeof(T));
    const PlanTables<R> tx = stage_plan<R>(a.px, tail);
    const T* twx = stage_twx<R>(a, tail + plan_tables_bytes(a.nx / 2, sizeof(T)));
    const PlanTables<R> ty = stage_plan<R>(a.py, tail + tables_x_bytes(a, sizeof(T)));
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
    constexpr int LB = sizeof(R) == 8 ? 4 : 8;
    const int total = ny * ncol;
    for (int t0 = threadIdx.x; t0 < total; t0 += LB * blockDim.x) {
        T v[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int ky = t / ncol, c = t - ky * ncol;
                v[q] = ld_l2(&spec[((long)k * ny + ky) * nxh + c0 + c], plast);
            }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int ky = t / ncol, c = t - ky * ncol;
                colbuf[ky * ldc + c] = v[q];
            }
        }
    }
    fft_batch<false, R, MAXR>(colbuf, ldc, ncol, a.py, +1, ty.tw);   // also orders the staged tables
    cluster.sync();   // every column transformed; gather rows from the owners
    const int jb = rank * a.rows_per_cta;
    for (int jc = 0; jc < a.rows_per_cta; jc += a.row_chunk) {
        const int nr = min(a.row_chunk, a.rows_per_cta - jc);
        for (int t = threadIdx.x; t < nr * n2; t += blockDim.x) {
            const int kk = t / nr, rr = t - kk * nr;
            const int prow = ty.pos[jb + jc + rr];
            const int kc = n2 - kk;
            const int o1 = kk / cpc, o2 = kc / cpc;
            const T* s1 = cluster.map_shared_rank(colbuf, o1);
            const T* s2 = cluster.map_shared_rank(colbuf, o2);
            rowbuf[kk * ldr + rr] = c2r_pack<R>(s1[prow * ldc + (kk - o1 * cpc)], s2[prow * ldc + (kc - o2 * cpc)],
                                                twx[kk], kk == 0);
        }
        fft_batch<false, R, MAXR>(rowbuf, ldr, nr, a.px, +1, tx.tw);
        const double sc = a.scale;
        for (int t = threadIdx.x; t < nr * n2; t += blockDim.x) {
            const int rr = t / n2, m = t - rr * n2;
            const int j = jb + jc + rr;
            const T z = rowbuf[tx.pos[m] * ldr + rr];
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
// K3, rigid lid: batched Thomas along z (pressure_solver.f90:33-53;
// solve_tridiag, pressure_solver.f90:126-162) and the (0,0)-mode recurrence.
// The coefficients are real, so the real and imaginary parts of a column are
// independent recurrences: one thread per (column, part), every column in
// one wave.  Levels move in chunks of KC, and the loads of the next chunk
// are issued before the recurrence runs over the current one, so memory
// latency overlaps the serial arithmetic.  The elimination runs in FP64 and
// is never rounded to the storage precision: the forward sweep writes
// nothing to the array, it keeps (c', d') of the level before every chunk in
// shared memory; the backward sweep re-reads a chunk's right-hand side,
// recomputes its pivots and d' from those two values with the same
// operations (so the same values), substitutes back and overwrites the
// chunk with x.  The pivots are formed from ksqr on the fly (rcp_newton):
// no factor table and no d' array in HBM.
// ---------------------------------------------------------------------------
// The FP64 reciprocal of a pivot by Newton-Raphson from the hardware
// approximation (PTX rcp.approx.ftz.f64): each iteration y += y (1 - x y)
// squares the relative error, two take it far below the FP64 rounding unit,
// and a third, with the residual 1 - x y formed exactly by an FMA, rounds
// the result correctly (Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990); on a
// B200 it agreed bit for bit with the correctly rounded 1.0 / x on 2^30
// random inputs over 81 binades, in fewer instructions.  The pivots are
// normal numbers bounded away from zero (the matrix is strictly diagonally
// dominant), so the flush-to-zero approximation never sees a subnormal.
__device__ __forceinline__ double rcp_newton(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

constexpr int kThomasChunk = 8;
constexpr int kThomasThreads = 128;

PS3D_HD size_t thomas_smem(int nz, int threads) {
    return (size_t)((nz + kThomasChunk - 1) / kThomasChunk + 1) * threads * sizeof(double2);
}

template <typename R, bool FULL>
__global__ void __launch_bounds__(kThomasThreads, 4) k_thomas(const ColumnArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pk = pol_keep(a.l2hint);   // the inverse y lines read the solution
    constexpr int KC = kThomasChunk;
    // FULL: nz is a multiple of KC, so only the chunk ends need tests
#define IN(cond) (FULL || (cond))
    extern __shared__ double2 ckp[];   // [chunk][thread]: (c', d') of the level before the chunk
    const long ncols = a.ncl ? a.ncl : (long)a.nxh * a.ny;   // columns held (a column slab: ncl)
    const long gid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (gid >= 2 * ncols * a.batch) return;
    const int part = (int)(gid & 1);
    const unsigned cb = (unsigned)(gid >> 1);
    const unsigned inst = fdiv(cb, a.fd_ncols);
    const unsigned c = cb - inst * (unsigned)ncols;
    R* col = reinterpret_cast<R*>(a.spec) + 2 * ((long)inst * a.sM + c) + part;
    const long ls = 2 * ncols;   // level stride in R
    const int nz = a.nz;
    const unsigned cg = c + (unsigned)a.col0;   // global column: its wavenumbers
    const unsigned q0 = fdiv(cg, a.layout ? a.fd_ny : a.fd_nxh);
    const int i = a.layout ? (int)q0 : (int)(cg - q0 * (unsigned)a.nxh);
    const int j = a.layout ? (int)(cg - q0 * (unsigned)a.ny) : (int)q0;
    const double ks = a.hkx[i] + a.hky[j];
    const double fxa = a.fxa;
    double2* ck = ckp + threadIdx.x;
    const int cs = blockDim.x;   // checkpoint stride
    if (ks > 0) {
        const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
        // one level of the forward elimination: cp(1) = c/b(1), dp(1) = d(1)/b(1);
        // r = 1/(b(k) - cp(k-1) a), cp(k) = c r, dp(k) = (d(k) - dp(k-1) a) r
        auto elim = [&](int k, double d, double& cp, double& dp) {
            const double bk = (k == 0 || k == nz - 1) ? bend : bmid;
            if (k == 0) {
                cp = fxa / bk;
                dp = d / bk;
            } else {
                const double r = rcp_newton(bk - cp * fxa);
                cp = fxa * r;
                dp = (d - dp * fxa) * r;
            }
        };
        double cp = 0.0, dp = 0.0;
        R nxt[KC];
#pragma unroll
        for (int q = 0; q < KC; ++q)
            if (IN(q < nz)) nxt[q] = ld_l2(&col[(long)q * ls], pk);
        for (int kb = 0; kb < nz; kb += KC) {
            R d[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) d[q] = nxt[q];
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (FULL ? (kb + KC < nz) : (kb + KC + q < nz)) nxt[q] = ld_l2(&col[(long)(kb + KC + q) * ls], pk);
            ck[(kb / KC) * cs] = make_double2(cp, dp);   // (cp, dp) of level kb-1
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (IN(kb + q < nz)) elim(kb + q, (double)d[q], cp, dp);
        }
        // back substitution, chunk by chunk from the top: x(nz) = dp(nz),
        // x(k) = dp(k) - cp(k) x(k+1)
        double x = 0.0;
        const int last = (nz - 1) / KC;
#pragma unroll
        for (int q = 0; q < KC; ++q)
            if (IN(last * KC + q < nz)) nxt[q] = ld_l2(&col[(long)(last * KC + q) * ls], pk);
        for (int sg = last; sg >= 0; --sg) {
            const int kb = sg * KC;
            R d[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) d[q] = nxt[q];
            if (sg > 0) {
#pragma unroll
                for (int q = 0; q < KC; ++q) nxt[q] = ld_l2(&col[(long)(kb - KC + q) * ls], pk);
            }
            double cpl[KC], dpl[KC];
            {
                const double2 c0 = ck[sg * cs];
                double cpv = c0.x, dpv = c0.y;
#pragma unroll
                for (int q = 0; q < KC; ++q) {
                    if (IN(kb + q < nz)) elim(kb + q, (double)d[q], cpv, dpv);
                    cpl[q] = cpv;
                    dpl[q] = dpv;
                }
            }
#pragma unroll
            for (int q = KC - 1; q >= 0; --q) {
                const int k = kb + q;
                if (IN(k < nz)) {
                    x = (k == nz - 1) ? dpl[q] : dpl[q] - cpl[q] * x;
                    d[q] = (R)x;
                }
            }
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (IN(kb + q < nz)) st_l2(&col[(long)(kb + q) * ls], d[q], pk);
        }
    } else {
        // (0,0) mode: p(1) = 0, p(2) = f(1) dz^2 dsqr, p(k+1) = 2p(k) - p(k-1) + f(k) dz^2 dsqr,
        // in chunks with the next chunk's loads in flight like the sweeps above
        const double h = a.dz2dsqr;
        double x0 = 0.0, x1 = 0.0, fprev = 0.0;   // p(k-2), p(k-1), f(k-1)
        R nxt[KC];
#pragma unroll
        for (int q = 0; q < KC; ++q)
            if (IN(q < nz)) nxt[q] = ld_l2(&col[(long)q * ls], pk);
        for (int kb = 0; kb < nz; kb += KC) {
            R d[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) d[q] = nxt[q];
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (FULL ? (kb + KC < nz) : (kb + KC + q < nz)) nxt[q] = ld_l2(&col[(long)(kb + KC + q) * ls], pk);
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const int k = kb + q;
                if (IN(k < nz)) {
                    const double xk = k == 0 ? 0.0 : 2 * x1 - x0 + fprev * h;
                    fprev = (double)d[q];
                    x0 = x1; x1 = xk;
                    d[q] = (R)xk;
                }
            }
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (IN(kb + q < nz)) st_l2(&col[(long)(kb + q) * ls], d[q], pk);
        }
    }
}
#undef IN


// The same solve eliminated from both ends at once (a twisted
// factorisation): the matrix is persymmetric (constant a = c = fxa, the same
// end coefficient at the top and the bottom level), so the elimination from
// the bottom up runs through exactly the pivots of the elimination from the
// top down, cp(j) for level j from the top and level nz-1-j from the bottom.
// One pivot chain of ceil(nz/2) levels therefore serves two d' chains, the
// two halves meet in a 2x2 solve at the middle,
//   x(m) = (dp(m) - cp(m) dq(jb)) / (1 - cp(m) cp(jb)),  x(m+1) = dq(jb) - cp(jb) x(m),
// and two back substitutions run outward.  The serial FP64 chain (divide,
// then multiply-add, per level) is half as long as a one-ended sweep, where
// it bounds the kernel.  Checkpoints (cp, dp, dq) before every chunk of 8
// pivot levels in shared memory; each chunk's values recomputed on the way
// back as in k_thomas.
//
// Two instantiation switches, neither of which changes an operation or its
// order (every form gives the same bits):
//   FULL  nz is even and nz/2 a multiple of the chunk: both halves end on a
//         chunk boundary, so no level needs a bounds test, and the first
//         pivot level and the meeting level sit at fixed positions of the
//         first and the last chunk;
//   RTAB  the forward sweep parks every level's reciprocal pivot r in shared
//         memory ([level][complex column]: the two parts of a column form the
//         same r), and the backward sweep takes it from there (cp = fxa r)
//         instead of forming it again; the checkpoints then hold (dp, dq).
//         Blocks of kThomas2RThreads threads, so that the table, H x 32
//         doubles, leaves eight blocks an SM.
// Level offsets are 32-bit (the launcher checks nz x level stride < 2^32).
constexpr int kThomas2RThreads = 64;

PS3D_HD size_t thomas2_smem(int nz, int threads) {
    const int h = (nz + 1) / 2;
    return (size_t)((h + kThomasChunk - 1) / kThomasChunk + 1) * threads * (sizeof(double2) + sizeof(double));
}
PS3D_HD size_t thomas2r_smem(int nz, int threads) {
    const int h = (nz + 1) / 2;
    return (size_t)((h + kThomasChunk - 1) / kThomasChunk + 1) * threads * sizeof(double2) +
           (size_t)h * (threads / 2) * sizeof(double);
}

template <typename R, bool FULL, bool RTAB>
__global__ void __launch_bounds__(RTAB ? kThomas2RThreads : kThomasThreads, RTAB ? 8 : 4) k_thomas2(const ColumnArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pk = pol_keep(a.l2hint);   // the inverse y lines read the solution
    constexpr int KC = kThomasChunk;
#define IN(cond) (FULL || (cond))
    // checkpoints [chunk][thread]: (cp, dp) and, after them, dq (RTAB: (dp, dq));
    // RTAB: then the reciprocal pivots [level][complex column]
    extern __shared__ double2 ck2[];
    const int nz = a.nz;
    const int H = (nz + 1) / 2;   // pivot levels: top 0 .. H-1, bottom nz-1 .. nz-Bc
    const int Bc = nz - H;
    const int m = H - 1, jb = Bc - 1;
    const int nch = (H + KC - 1) / KC;
    const int T = blockDim.x, tid = threadIdx.x;
    double* ckq = reinterpret_cast<double*>(ck2 + (size_t)(nch + 1) * T);
    double* rt = ckq + (tid >> 1);   // RTAB: level jj's r at rt[jj * (T / 2)]
    const int rts = T >> 1;
    const long ncols = a.ncl ? a.ncl : (long)a.nxh * a.ny;   // columns held (a column slab: ncl)
    const long gid = blockIdx.x * (long)T + tid;
    if (gid >= 2 * ncols * a.batch) return;
    const int part = (int)(gid & 1);
    const unsigned cb = (unsigned)(gid >> 1);
    const unsigned inst = fdiv(cb, a.fd_ncols);
    const unsigned c = cb - inst * (unsigned)ncols;
    R* col = reinterpret_cast<R*>(a.spec) + 2 * ((long)inst * a.sM + c) + part;
    const unsigned ls = (unsigned)(2 * ncols);   // level stride in R
    R* const bot0 = col + (size_t)(nz - 1) * ls;
    const unsigned cg = c + (unsigned)a.col0;   // global column: its wavenumbers
    const unsigned q0 = fdiv(cg, a.layout ? a.fd_ny : a.fd_nxh);
    const int i = a.layout ? (int)q0 : (int)(cg - q0 * (unsigned)a.nxh);
    const int j = a.layout ? (int)(cg - q0 * (unsigned)a.ny) : (int)q0;
    const double ks = a.hkx[i] + a.hky[j];
    const double fxa = a.fxa;
    if (!(ks > 0)) {
        // (0,0) mode: p(1) = 0, p(2) = f(1) dz^2 dsqr, p(k+1) = 2p(k) - p(k-1) + f(k) dz^2 dsqr
        const double h = a.dz2dsqr;
        double x0 = 0.0, x1 = 0.0, fprev = 0.0;   // p(k-2), p(k-1), f(k-1)
        R nxt[KC];
#pragma unroll
        for (int q = 0; q < KC; ++q)
            if (q < nz) nxt[q] = ld_l2(&col[(unsigned)q * ls], pk);
        for (int kb = 0; kb < nz; kb += KC) {
            R d[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) d[q] = nxt[q];
#pragma unroll
            for (int q = 0; q < KC; ++q)
                if (kb + KC + q < nz) nxt[q] = ld_l2(&col[(unsigned)(kb + KC + q) * ls], pk);
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const int k = kb + q;
                if (k < nz) {
                    const double xk = k == 0 ? 0.0 : 2 * x1 - x0 + fprev * h;
                    fprev = (double)d[q];
                    x0 = x1; x1 = xk;
                    st_l2(&col[(unsigned)k * ls], (R)xk, pk);
                }
            }
        }
        return;
    }
    const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
    // pivot level jj (first: jj == 0) with the top value dt and the bottom
    // value db: cp(1) = c/b(1), dp(1) = d(1)/b(1); r = 1/(b - cp a),
    // cp = c r, dp = (d - dp a) r (the bottom chain the same with its own d;
    // both: level jj has a bottom partner)
    auto elim = [&](bool first, bool both, double dt, double db, double& cp, double& dp, double& dq, double& r) {
        if (first) {
            cp = fxa / bend;
            dp = dt / bend;
            dq = db / bend;
        } else {
            r = rcp_newton(bmid - cp * fxa);
            cp = fxa * r;
            dp = (dt - dp * fxa) * r;
            if (both) dq = (db - dq * fxa) * r;
        }
    };
    // the chunk of pivot levels jc .. jc+KC-1: top levels jc.., bottom levels nz-1-jc..
    auto load = [&](int jc, R* top, R* bot) {
#pragma unroll
        for (int q = 0; q < KC; ++q) {
            const int jj = jc + q;
            const unsigned o = (unsigned)jj * ls;
            if (IN(jj < H)) top[q] = ld_l2(col + o, pk);
            if (IN(jj < Bc)) bot[q] = ld_l2(bot0 - o, pk);
        }
    };
    double cp = 0.0, dp = 0.0, dq = 0.0, cp_jb = 0.0, dq_jb = 0.0;
    R nt[KC], nb[KC];
#pragma unroll
    for (int q = 0; q < KC; ++q) { nt[q] = (R)0; nb[q] = (R)0; }
    load(0, nt, nb);
    for (int ch = 0; ch < nch; ++ch) {
        const int jc = ch * KC;
        R dt[KC], db[KC];
#pragma unroll
        for (int q = 0; q < KC; ++q) { dt[q] = nt[q]; db[q] = nb[q]; }
        if (ch + 1 < nch) load(jc + KC, nt, nb);
        if constexpr (RTAB) {
            ck2[ch * T + tid] = make_double2(dp, dq);   // before pivot level jc
        } else {
            ck2[ch * T + tid] = make_double2(cp, dp);
            ckq[ch * T + tid] = dq;
        }
#pragma unroll
        for (int q = 0; q < KC; ++q) {
            const int jj = jc + q;
            if (IN(jj < H)) {
                const bool first = q == 0 && ch == 0;
                double r = 0.0;
                elim(first, IN(jj < Bc), (double)dt[q], (double)db[q], cp, dp, dq, r);
                if (RTAB && !first) rt[jj * rts] = r;
                if (FULL ? (q == KC - 1 && ch == nch - 1) : (jj == jb)) { cp_jb = cp; dq_jb = dq; }
            }
        }
    }
    // the two halves meet: x(m) and x(m+1)
    double xt = (dp - cp * dq_jb) / (1.0 - cp * cp_jb);
    double xb = dq_jb - cp_jb * xt;
    // back substitution outward, chunk by chunk from the middle
    load((nch - 1) * KC, nt, nb);
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int jc = ch * KC;
        R dt[KC], db[KC];
#pragma unroll
        for (int q = 0; q < KC; ++q) { dt[q] = nt[q]; db[q] = nb[q]; }
        if (ch > 0) load(jc - KC, nt, nb);
        double cpl[KC], dpl[KC], dql[KC];
        {
            const double2 c0 = ck2[ch * T + tid];
            double cpv = RTAB ? 0.0 : c0.x, dpv = RTAB ? c0.x : c0.y, dqv = RTAB ? c0.y : ckq[ch * T + tid];
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const int jj = jc + q;
                if (IN(jj < H)) {
                    const bool first = q == 0 && ch == 0;
                    if (RTAB && !first) {
                        const double r = rt[jj * rts];
                        cpv = fxa * r;
                        dpv = ((double)dt[q] - dpv * fxa) * r;
                        if (IN(jj < Bc)) dqv = ((double)db[q] - dqv * fxa) * r;
                    } else {
                        double r;
                        elim(first, IN(jj < Bc), (double)dt[q], (double)db[q], cpv, dpv, dqv, r);
                    }
                }
                cpl[q] = cpv;
                dpl[q] = dpv;
                dql[q] = dqv;
            }
        }
#pragma unroll
        for (int q = KC - 1; q >= 0; --q) {
            const int jj = jc + q;
            if (IN(jj < H)) {
                const unsigned o = (unsigned)jj * ls;
                const bool mid = FULL ? (q == KC - 1 && ch == nch - 1) : (jj >= m);   // the meeting level
                if (!mid) xt = dpl[q] - cpl[q] * xt;
                st_l2(col + o, (R)xt, pk);
                if (IN(jj <= jb)) {
                    if (FULL ? !mid : (jj < jb)) xb = dql[q] - cpl[q] * xb;
                    st_l2(bot0 - o, (R)xb, pk);
                }
            }
        }
    }
#undef IN
}

// ---------------------------------------------------------------------------
// K3 with the y transforms, on the y-split layout (PlaneArgs::ysplit): one
// block per (instance, kx, half) holds that half-line's nz x ny/2 spectra
// in shared memory, as [j][k] with an odd pitch, and runs
//   the forward half-length y transforms of its nz levels (DIF, staying in
//     digit-reversed order, scaled by dx dy as the y-lines pass scales),
//   the rigid-lid vertical solves of its ny/2 columns — the two-ended FP64
//     elimination of k_thomas2, one thread per (column, part), (c', d', d'')
//     checkpointed every kT2KC levels, each chunk re-formed on the way back —
//     and the (0,0) recurrence,
//   the inverse half-length y transforms (DIT, back to natural order),
// so the spectral array crosses memory once in and once out instead of six
// times, and three kernels become one.  Column j of a half sits at ky =
// 2 j + half.
// ---------------------------------------------------------------------------
constexpr int kCsThreads = 256;
constexpr int kCsKC = 8;

struct ColSolveArgs {
    int nz, ny, nxh;
    void* spec;                    // [inst][k][kx][half][ny/2], float2
    long sM;                       // instance stride (elements)
    int batch;
    FFTPlan ph;                    // length ny/2
    double scale;                  // forward y-transform scale (dx dy)
    const double* hkx;             // hat_ksqr(kx)
    const double* hky;             // hat_ksqr(ky)
    double fxa, dz2dsqr;           // 1/dz^2/dsqr, dz^2 dsqr
    int l2hint;
};

PS3D_HD size_t colsolve_smem(int nz, int ny) {
    const int ny2 = ny / 2, H = (nz + 1) / 2, nch = (H + kCsKC - 1) / kCsKC;
    return align16((size_t)ny2 * (nz | 1) * sizeof(float2)) +
           align16((size_t)nch * 3 * kCsThreads * sizeof(double)) + plan_tables_bytes(ny2, sizeof(float2));
}

__global__ void __launch_bounds__(kCsThreads) k_colsolve(const ColSolveArgs a) {
    using T = float2;
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    extern __shared__ __align__(16) unsigned char cs_raw[];
    const int nz = a.nz, ny = a.ny, ny2 = ny / 2, nxh = a.nxh;
    const int ld = nz | 1;
    const int H = (nz + 1) / 2, Bc = nz - H, m = H - 1, jb = Bc - 1;
    const int nch = (H + kCsKC - 1) / kCsKC;
    T* buf = reinterpret_cast<T*>(cs_raw);                                        // [j][k], pitch ld
    double* ck = reinterpret_cast<double*>(cs_raw + align16((size_t)ny2 * ld * sizeof(T)));   // [chunk][3][thread]
    const PlanTables<float> ty = stage_plan<float>(
        a.ph, cs_raw + align16((size_t)ny2 * ld * sizeof(T)) + align16((size_t)nch * 3 * kCsThreads * sizeof(double)));
    const int units = nxh * 2;
    const int inst = blockIdx.x / units, u = blockIdx.x - inst * units;
    const int kx = u >> 1, half = u & 1;
    T* g = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)kx * ny + half * ny2;
    const long ls = (long)nxh * ny;   // level stride
    const unsigned long long pk = pol_keep(a.l2hint), pl = pol_last(a.l2hint);
    const float sc = (float)a.scale;
    for (int t = threadIdx.x; t < nz * ny2; t += kCsThreads) {
        const int k = t / ny2, j = t - k * ny2;
        buf[j * ld + k] = cscale(ld_l2(&g[(long)k * ls + j], pl), sc);
    }
    fft_batch<false, float, 16>(buf, ld, nz, a.ph, -1, ty.tw);   // synchronises before and after
    // ---- vertical solves: thread (column p, part)
    const int tid = threadIdx.x;
    float* bf = reinterpret_cast<float*>(buf);
    for (int p0 = 0; p0 < ny2; p0 += kCsThreads / 2) {
        const int p = p0 + (tid >> 1), part = tid & 1;
        if (p < ny2) {
            float* col = bf + (size_t)p * ld * 2 + part;   // level k at col[2 k]
            const int ky = 2 * ty.ipos[p] + half;
            const double ks = a.hkx[kx] + a.hky[ky];
            const double fxa = a.fxa;
            if (!(ks > 0)) {
                // (0,0): p(1) = 0, p(2) = f(1) dz^2 dsqr, p(k+1) = 2p(k) - p(k-1) + f(k) dz^2 dsqr
                double x0 = 0.0, x1 = 0.0, fprev = 0.0;
                for (int k = 0; k < nz; ++k) {
                    const double xk = k == 0 ? 0.0 : 2 * x1 - x0 + fprev * a.dz2dsqr;
                    fprev = (double)col[2 * k];
                    x0 = x1; x1 = xk;
                    col[2 * k] = (float)xk;
                }
            } else {
                const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
                auto elim = [&](int jj, double dt, double db, double& cp, double& dp, double& dq) {
                    if (jj == 0) {
                        cp = fxa / bend;
                        dp = dt / bend;
                        dq = db / bend;
                    } else {
                        const double r = rcp_newton(bmid - cp * fxa);
                        cp = fxa * r;
                        dp = (dt - dp * fxa) * r;
                        if (jj < Bc) dq = (db - dq * fxa) * r;
                    }
                };
                double cp = 0.0, dp = 0.0, dq = 0.0, cp_jb = 0.0, dq_jb = 0.0;
                for (int ch = 0; ch < nch; ++ch) {
                    double* c = ck + (size_t)ch * 3 * kCsThreads + tid;
                    c[0] = cp; c[kCsThreads] = dp; c[2 * kCsThreads] = dq;
#pragma unroll
                    for (int q = 0; q < kCsKC; ++q) {
                        const int jj = ch * kCsKC + q;
                        if (jj < H) {
                            elim(jj, (double)col[2 * jj], jj < Bc ? (double)col[2 * (nz - 1 - jj)] : 0.0, cp, dp, dq);
                            if (jj == jb) { cp_jb = cp; dq_jb = dq; }
                        }
                    }
                }
                double xt = (dp - cp * dq_jb) / (1.0 - cp * cp_jb);
                double xb = dq_jb - cp_jb * xt;
                for (int ch = nch - 1; ch >= 0; --ch) {
                    const int jc = ch * kCsKC;
                    const double* c = ck + (size_t)ch * 3 * kCsThreads + tid;
                    double cpv = c[0], dpv = c[kCsThreads], dqv = c[2 * kCsThreads];
                    double cpl[kCsKC], dpl[kCsKC], dql[kCsKC];
#pragma unroll
                    for (int q = 0; q < kCsKC; ++q) {
                        const int jj = jc + q;
                        if (jj < H)
                            elim(jj, (double)col[2 * jj], jj < Bc ? (double)col[2 * (nz - 1 - jj)] : 0.0, cpv, dpv, dqv);
                        cpl[q] = cpv; dpl[q] = dpv; dql[q] = dqv;
                    }
#pragma unroll
                    for (int q = kCsKC - 1; q >= 0; --q) {
                        const int jj = jc + q;
                        if (jj < H) {
                            if (jj < m) xt = dpl[q] - cpl[q] * xt;
                            col[2 * jj] = (float)xt;
                            if (jj <= jb) {
                                if (jj < jb) xb = dql[q] - cpl[q] * xb;
                                col[2 * (nz - 1 - jj)] = (float)xb;
                            }
                        }
                    }
                }
            }
        }
    }
    fft_batch<true, float, 16>(buf, ld, nz, a.ph, +1, ty.tw);
    for (int t = threadIdx.x; t < nz * ny2; t += kCsThreads) {
        const int k = t / ny2, j = t - k * ny2;
        st_l2(&g[(long)k * ls + j], buf[j * ld + k], pk);
    }
}

// The same solve split over a cluster of two CTAs by levels: CTA 0 holds
// levels 0 .. H-1, CTA 1 levels nz-1 down to H (its local level q is level
// nz-1-q), so each runs the y transforms of half the levels, and each
// eliminates one end of the two-ended factorisation over its own levels:
// the top-down chain (c', d') in CTA 0 and the bottom-up chain (c', d'') in
// CTA 1, through the same pivots (the matrix is persymmetric).  The halves
// meet through distributed shared memory: each CTA writes its end value
// d'(m) or d''(jb) into the other's shared memory, one cluster barrier, and
// both form the middle 2x2 solve from the same operands, so x(m) and
// x(m+1) come out as in k_colsolve and k_thomas2, bit for bit.  The (0,0)
// recurrence runs through CTA 0's levels, passes (p(H-2), p(H-1), f(H-1))
// across, and CTA 1 continues after the barrier.  Half the shared memory of
// k_colsolve per CTA: two clusters' CTAs fit an SM.
constexpr int kCs2KC = 16;

PS3D_HD size_t colsolve2_smem(int nz, int ny) {
    const int ny2 = ny / 2, H = (nz + 1) / 2, nch = (H + kCs2KC - 1) / kCs2KC;
    return align16((size_t)ny2 * (H | 1) * sizeof(float2)) +         // spectra [j][q]
           align16((size_t)nch * 2 * 2 * ny2 * sizeof(double)) +      // checkpoints [chunk][2][column part]
           align16((size_t)6 * 2 * ny2 * sizeof(double)) +            // own end values, pivots, exchange
           plan_tables_bytes(ny2, sizeof(float2));
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kCsThreads, 2) k_colsolve2(const ColSolveArgs a) {
    using T = float2;
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    extern __shared__ __align__(16) unsigned char cs2_raw[];
    const int nz = a.nz, ny = a.ny, ny2 = ny / 2, nxh = a.nxh;
    const int H = (nz + 1) / 2, Bc = nz - H, m = H - 1, jb = Bc - 1;
    const int L = rank == 0 ? H : Bc;   // levels held; chain index jj = local level q
    const int ld = H | 1;
    const int nch = (L + kCs2KC - 1) / kCs2KC;
    const int ncp = 2 * ny2;            // column parts
    unsigned char* base = cs2_raw;
    T* buf = reinterpret_cast<T*>(base);                                   // [j][q], pitch ld
    base += align16((size_t)ny2 * ld * sizeof(T));
    double* ck = reinterpret_cast<double*>(base);                          // [chunk][2][cp]
    base += align16((size_t)((H + kCs2KC - 1) / kCs2KC) * 2 * ncp * sizeof(double));
    double* own = reinterpret_cast<double*>(base);                         // [0] end value, [1] c'(m), [2] c'(jb)
    double* xch = own + 3 * ncp;                                           // [3][cp]: written by the other CTA
    base += align16((size_t)6 * ncp * sizeof(double));
    const PlanTables<float> ty = stage_plan<float>(a.ph, base);
    const int units = nxh * 2;
    const int pair = blockIdx.x >> 1;
    const int inst = pair / units, u = pair - inst * units;
    const int kx = u >> 1, half = u & 1;
    T* g = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)kx * ny + half * ny2;
    const long ls = (long)nxh * ny;   // level stride
    const unsigned long long pk = pol_keep(a.l2hint), pl = pol_last(a.l2hint);
    const float sc = (float)a.scale;
    for (int t = threadIdx.x; t < L * ny2; t += kCsThreads) {
        const int q = t / ny2, j = t - q * ny2;
        const int k = rank == 0 ? q : nz - 1 - q;
        buf[j * ld + q] = cscale(ld_l2(&g[(long)k * ls + j], pl), sc);
    }
    fft_batch<false, float, 16>(buf, ld, L, a.ph, -1, ty.tw);   // synchronises before and after
    cluster.sync();   // the other CTA is running before its shared memory is written
    const int tid = threadIdx.x;
    float* bf = reinterpret_cast<float*>(buf);
    double* peer = cluster.map_shared_rank(xch, rank ^ 1);
    const double fxa = a.fxa;
    // pivot level jj: cp(0) = c/b_end, cp(jj) = c / (b_mid - cp(jj-1) a); d the chain's own value
    // (d' from the top in CTA 0, d'' from the bottom in CTA 1)
    auto elim = [&](int jj, double dv, double bend, double bmid, double& cp, double& d) {
        if (jj == 0) {
            cp = fxa / bend;
            d = dv / bend;
        } else {
            const double r = rcp_newton(bmid - cp * fxa);
            cp = fxa * r;
            d = (dv - d * fxa) * r;
        }
    };
    // ---- forward eliminations over this CTA's levels
    for (int p0 = 0; p0 < ny2; p0 += kCsThreads / 2) {
        const int p = p0 + (tid >> 1), part = tid & 1, c = 2 * p + part;
        if (p < ny2) {
            float* col = bf + (size_t)p * ld * 2 + part;   // local level q at col[2 q]
            const int ky = 2 * ty.ipos[p] + half;
            const double ks = a.hkx[kx] + a.hky[ky];
            if (!(ks > 0)) {
                if (rank == 0) {
                    // (0,0): p(1) = 0, p(2) = f(1) dz^2 dsqr, p(k+1) = 2p(k) - p(k-1) + f(k) dz^2 dsqr
                    double x0 = 0.0, x1 = 0.0, fprev = 0.0;
                    for (int q = 0; q < H; ++q) {
                        const double xk = q == 0 ? 0.0 : 2 * x1 - x0 + fprev * a.dz2dsqr;
                        fprev = (double)col[2 * q];
                        x0 = x1; x1 = xk;
                        col[2 * q] = (float)xk;
                    }
                    peer[c] = x0; peer[ncp + c] = x1; peer[2 * ncp + c] = fprev;
                }
            } else {
                const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
                double cp = 0.0, d = 0.0, cp_jb = 0.0;
                for (int ch = 0; ch < nch; ++ch) {
                    ck[(size_t)(ch * 2) * ncp + c] = cp;
                    ck[(size_t)(ch * 2 + 1) * ncp + c] = d;
#pragma unroll
                    for (int q = 0; q < kCs2KC; ++q) {
                        const int jj = ch * kCs2KC + q;
                        if (jj < L) {
                            elim(jj, (double)col[2 * jj], bend, bmid, cp, d);
                            if (jj == jb) cp_jb = cp;
                        }
                    }
                }
                // c'(m): CTA 1 ends at jb, one level short of m when nz is odd
                double cp_m = cp;
                if (rank == 1 && m > jb) {
                    double dd = 0.0;
                    elim(m, 0.0, bend, bmid, cp_m, dd);
                }
                own[c] = d; own[ncp + c] = cp_m; own[2 * ncp + c] = cp_jb;
                peer[c] = d;
            }
        }
    }
    cluster.sync();   // both ends' values delivered
    for (int p0 = 0; p0 < ny2; p0 += kCsThreads / 2) {
        const int p = p0 + (tid >> 1), part = tid & 1, c = 2 * p + part;
        if (p < ny2) {
            float* col = bf + (size_t)p * ld * 2 + part;
            const int ky = 2 * ty.ipos[p] + half;
            const double ks = a.hkx[kx] + a.hky[ky];
            if (!(ks > 0)) {
                if (rank == 1) {
                    double x0 = xch[c], x1 = xch[ncp + c], fprev = xch[2 * ncp + c];
                    for (int k = H; k < nz; ++k) {
                        const int q = nz - 1 - k;
                        const double xk = 2 * x1 - x0 + fprev * a.dz2dsqr;
                        fprev = (double)col[2 * q];
                        x0 = x1; x1 = xk;
                        col[2 * q] = (float)xk;
                    }
                }
            } else {
                const double bend = -ks - fxa, bmid = -ks - 2 * fxa;
                const double dp_m = rank == 0 ? own[c] : xch[c];
                const double dq_jb = rank == 0 ? xch[c] : own[c];
                const double cp_m = own[ncp + c], cp_jb = own[2 * ncp + c];
                const double xt = (dp_m - cp_m * dq_jb) / (1.0 - cp_m * cp_jb);   // x(m)
                double x = rank == 0 ? xt : dq_jb - cp_jb * xt;                     // CTA 1: x(m+1)
                const int top = rank == 0 ? m : jb;   // the chain's last level holds x as formed
                for (int ch = nch - 1; ch >= 0; --ch) {
                    const int jc = ch * kCs2KC;
                    double cpv = ck[(size_t)(ch * 2) * ncp + c], dv = ck[(size_t)(ch * 2 + 1) * ncp + c];
                    double cpl[kCs2KC], dl[kCs2KC];
#pragma unroll
                    for (int q = 0; q < kCs2KC; ++q) {
                        const int jj = jc + q;
                        if (jj < L) elim(jj, (double)col[2 * jj], bend, bmid, cpv, dv);
                        cpl[q] = cpv; dl[q] = dv;
                    }
#pragma unroll
                    for (int q = kCs2KC - 1; q >= 0; --q) {
                        const int jj = jc + q;
                        if (jj < L) {
                            if (jj < top) x = dl[q] - cpl[q] * x;
                            col[2 * jj] = (float)x;
                        }
                    }
                }
            }
        }
    }
    fft_batch<true, float, 16>(buf, ld, L, a.ph, +1, ty.tw);
    for (int t = threadIdx.x; t < L * ny2; t += kCsThreads) {
        const int q = t / ny2, j = t - q * ny2;
        const int k = rank == 0 ? q : nz - 1 - q;
        st_l2(&g[(long)k * ls + j], buf[j * ld + q], pk);
    }
}

bool colsolve_fits(int nz, int ny) {
    return ny % 16 == 0 && colsolve_smem(nz, ny) <= 227 * 1024 - 64;
}

bool colsolve2_fits(int nz, int ny) {
    return ny % 16 == 0 && colsolve2_smem(nz, ny) <= 227 * 1024 - 64;
}

cudaError_t launch_colsolve(const PlaneArgs& p, const ColumnArgs& c, cudaStream_t s) {
    // the two-CTA form where it fits, unless PS3D_COLSOLVE=1 pins the one-CTA form
    const char* fv = std::getenv("PS3D_COLSOLVE");
    const int form = fv ? std::atoi(fv) : 2;
    const bool two = form != 1 && colsolve2_fits(c.nz, c.ny);
    if (!two && !colsolve_fits(c.nz, c.ny)) return cudaErrorInvalidValue;
    if (plan_max_radix(p.pyh) > 16) return cudaErrorInvalidValue;
    ColSolveArgs a{};
    a.nz = c.nz; a.ny = c.ny; a.nxh = c.nxh;
    a.spec = c.spec; a.sM = c.sM; a.batch = std::max(1, c.batch);
    a.ph = p.pyh;
    a.scale = p.scale;
    a.hkx = c.hkx; a.hky = c.hky;
    a.fxa = c.fxa; a.dz2dsqr = c.dz2dsqr;
    a.l2hint = l2hint_mode();
    const dim3 g((unsigned)(c.nxh * 2 * a.batch)), b(kCsThreads);
    if (two) return launch_pdl(k_colsolve2, dim3(2 * g.x), b, colsolve2_smem(c.nz, c.ny), s, a);
    return launch_pdl(k_colsolve, g, b, colsolve_smem(c.nz, c.ny), s, a);
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
    const int nz = a.nz;
    const PlanTables<R> tz = stage_plan<R>(a.pz, smem_raw + align16((size_t)nz * ld * sizeof(T)));
    const long ncols = a.ncl ? a.ncl : (long)a.nxh * a.ny;   // columns held (a column slab: ncl)
    const long bpi = (ncols + kZLines - 1) / kZLines;   // blocks per instance
    const long inst = blockIdx.x / bpi;
    const long c0 = (blockIdx.x - inst * bpi) * (long)kZLines;
    const int nl = (int)min((long)kZLines, ncols - c0);
    T* spec = reinterpret_cast<T*>(a.spec) + inst * a.sM;
    __syncthreads();
    for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
        const int k = t / nl, l = t - k * nl;
        const int slot = (a.op == 2) ? tz.pos[k] : k;
        buf[slot * ld + l] = spec[c0 + l + (long)k * ncols];
    }
    if (a.op == 2) {
        fft_batch<true, R>(buf, ld, nl, a.pz, +1, tz.tw);
    } else {
        fft_batch<false, R>(buf, ld, nl, a.pz, -1, tz.tw);
        const R sc = (R)a.scale;
        for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
            const int p = t / nl, l = t - p * nl;
            T v = cscale(buf[p * ld + l], sc);
            if (a.op == 0) {
                const long c = c0 + l + a.col0;   // global column: its wavenumbers
                const int i = a.layout ? (int)(c / a.ny) : (int)(c % a.nxh);
                const int j = a.layout ? (int)(c % a.ny) : (int)(c / a.nxh);
                const int k = tz.ipos[p];
                const double ks = a.hkx[i] + a.hky[j] + a.hkz[k];
                if (ks > 0.0) { v.x = (R)(-(double)v.x / ks); v.y = (R)(-(double)v.y / ks); }
                else { v.x = (R)0; v.y = (R)0; }
            }
            buf[p * ld + l] = v;
        }
        if (a.op == 0) fft_batch<true, R>(buf, ld, nl, a.pz, +1, tz.tw);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nz * nl; t += blockDim.x) {
        const int k = t / nl, l = t - k * nl;
        const int slot = (a.op == 1) ? tz.pos[k] : k;
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
// bank conflicts.  Global loads are issued in batches (LB per thread)
// before their shared-memory stores, so each thread keeps several loads in
// flight.
// ---------------------------------------------------------------------------
template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_blocks<MAXR>()) k_rows_fwd(const PlaneArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pfield = pol_field(a.l2hint), pkeep = pol_keep(a.l2hint);
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int tj = a.tj, ld = tj | 1;
    unsigned char* tail = smem_raw + align16((size_t)n2 * ld * sizeof(T));
    const PlanTables<R> tx = stage_plan<R>(a.px, tail);
    const T* twx = stage_twx<R>(a, tail + plan_tables_bytes(n2, sizeof(T)));
    const int jb = blockIdx.x * tj;
    const int kcnt = a.kcount ? a.kcount : nz;   // levels of the window (z-slab)
    const int inst = blockIdx.y / kcnt;
    // spectral level; zrev walks the planes top down (the step kernel before
    // the forward pass wrote the top levels last, so some are still in L2)
    const int kl = a.zrev ? kcnt - 1 - (int)(blockIdx.y - inst * kcnt) : (int)(blockIdx.y - inst * kcnt);
    const int k = a.kbeg + kl;                    // real-field level
    const long ioff = (long)inst * a.sN;
    const double* au = a.u + ioff;
    const double* av = a.v + ioff;
    const double* aw = a.w + ioff;
    const double* asrc = a.src ? a.src + ioff : nullptr;
    constexpr int LB = 2;
    const int total = tj * n2;
    for (int t0 = threadIdx.x; t0 < total; t0 += LB * blockDim.x) {
        double2 d[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int rr = (int)fdiv(t, a.fd_n2), m = t - rr * n2;
                d[q] = plane_source_pair(a, au, av, aw, asrc, k, jb + rr, m, pfield);
            }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int rr = (int)fdiv(t, a.fd_n2), m = t - rr * n2;
                buf[m * ld + rr] = mk<R>((R)d[q].x, (R)d[q].y);
            }
        }
    }
    fft_batch<false, R, MAXR, true>(buf, ld, tj, a.px, -1, tx.tw, tj);   // its first barrier also orders the tables
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)kl * nxh * ny;
    for (int t = threadIdx.x; t < tj * (n2 + 1); t += blockDim.x) {
        const int kx = (int)fdiv(t, a.fd_tj), rr = t - kx * tj;
        const int k1 = (kx == n2) ? 0 : kx;
        const int k2 = (kx == 0) ? 0 : n2 - kx;
        st_l2(&spec[(long)kx * ny + jb + rr], r2c_unpack<R>(buf[tx.pos[k1] * ld + rr], buf[tx.pos[k2] * ld + rr], twx[kx]),
              pkeep);
    }
}

// ---------------------------------------------------------------------------
// Rows pass, pipelined (implementation 2, divergence and source modes): a
// persistent grid walks the (plane, row-block) tiles; the whole input rows
// of a tile (u, v with the row below, w at k and k-1, or the source field)
// arrive by bulk copies on the TMA engine into one of two shared-memory
// stages while the previous tile is transformed, so the HBM stream never
// waits on the FFT.  The arithmetic is that of k_rows_fwd.
// ---------------------------------------------------------------------------
__host__ __device__ inline int pipe_rows(const PlaneArgs& a) { return a.mode == 0 ? 4 * a.tj + 1 : a.tj; }
__host__ __device__ inline size_t pipe_stage_bytes(const PlaneArgs& a) {
    return (size_t)(4 * a.tj + 1) * a.nx * sizeof(double);
}

template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, 2) k_rows_fwd_pipe(const PlaneArgs a, int ntiles) {
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int tj = a.tj, ld = tj | 1;
    const size_t sb = pipe_stage_bytes(a);
    auto stage = [&](int s) { return reinterpret_cast<double*>(smem_raw + (size_t)s * sb); };
    T* buf = reinterpret_cast<T*>(smem_raw + 2 * sb);
    unsigned char* tail = smem_raw + 2 * sb + align16((size_t)n2 * ld * sizeof(T));
    const PlanTables<R> tx = stage_plan<R>(a.px, tail);
    const T* twx = stage_twx<R>(a, tail + plan_tables_bytes(n2, sizeof(T)));
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(tail + tables_x_bytes(a, sizeof(T)));
    __shared__ int abort_flag;
    const int tpp = ny / tj;                 // tiles per plane
    const long plane = (long)nx * ny;
    const int nrows = pipe_rows(a);
    const unsigned bytes = (unsigned)((size_t)nrows * nx * sizeof(double));
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async();
    }
    __syncthreads();
    auto tile_of = [&](int t, int& inst, int& k, int& jb) {
        inst = t / (tpp * nz);
        const int r = t - inst * tpp * nz;
        k = r / tpp;
        jb = (r - k * tpp) * tj;
    };
    // warp 0 issues every row of tile t into stage s
    auto issue = [&](int t, int s) {
        if (threadIdx.x >= 32) return;
        int inst, k, jb;
        tile_of(t, inst, k, jb);
        const long ioff = (long)inst * a.sN;
        if (threadIdx.x == 0) {
            fence_proxy_async();
            mbar_expect(&bars[s], bytes);
        }
        __syncwarp();
        const int km = wrap(k - 1, nz);
        for (int r = threadIdx.x; r < nrows; r += 32) {
            const double* row;
            if (a.mode != 0) row = a.src + ioff + (long)k * plane + (long)(jb + r) * nx;
            else if (r < tj) row = a.u + ioff + (long)k * plane + (long)(jb + r) * nx;
            else if (r < 2 * tj + 1) row = a.v + ioff + (long)k * plane + (long)wrap(jb - 1 + (r - tj), ny) * nx;
            else if (r < 3 * tj + 1) row = a.w + ioff + (long)k * plane + (long)(jb + (r - 2 * tj - 1)) * nx;
            else row = a.w + ioff + (long)km * plane + (long)(jb + (r - 3 * tj - 1)) * nx;
            bulk_copy_g2s(stage(s) + (size_t)r * nx, row, (unsigned)(nx * sizeof(double)), &bars[s]);
        }
    };
    const int G = gridDim.x;
    int n = 0, t = blockIdx.x;
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + G < ntiles) issue(blockIdx.x + G, 1);
    for (; t < ntiles; t += G, ++n) {
        const int s = n & 1;
        if (!mbar_wait(&bars[s], (unsigned)(n >> 1) & 1u)) {
            abort_flag = 1;
            if (a.err) *(volatile unsigned*)a.err = 1u;
        }
        __syncthreads();
        if (abort_flag) break;
        int inst, k, jb;
        tile_of(t, inst, k, jb);
        const double* st = stage(s);
        const int total = tj * n2;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int rr = (int)fdiv(e, a.fd_n2), m = e - rr * n2;
            double d0, d1;
            if (a.mode == 0) {
                const double* U = st + (size_t)rr * nx;
                const double* Vm = st + (size_t)(tj + rr) * nx;
                const double* Vc = Vm + nx;
                const double* Wc = st + (size_t)(2 * tj + 1 + rr) * nx;
                const double* Wm = st + (size_t)(3 * tj + 1 + rr) * nx;
                const double2 uu = *reinterpret_cast<const double2*>(U + 2 * m);
                const double um = U[wrap(2 * m - 1, nx)];
                const double2 vv = *reinterpret_cast<const double2*>(Vc + 2 * m);
                const double2 vm = *reinterpret_cast<const double2*>(Vm + 2 * m);
                const double2 ww = *reinterpret_cast<const double2*>(Wc + 2 * m);
                const double2 wm = *reinterpret_cast<const double2*>(Wm + 2 * m);
                d0 = ((uu.x - um) * a.rdx + (vv.x - vm.x) * a.rdy + (ww.x - wm.x) * a.rdz) * a.rdt;
                d1 = ((uu.y - uu.x) * a.rdx + (vv.y - vm.y) * a.rdy + (ww.y - wm.y) * a.rdz) * a.rdt;
            } else {
                const double2 sv = *reinterpret_cast<const double2*>(st + (size_t)rr * nx + 2 * m);
                d0 = sv.x; d1 = sv.y;
            }
            buf[m * ld + rr] = mk<R>((R)d0, (R)d1);
        }
        __syncthreads();   // stage s consumed: refill it with tile t + 2G
        if (t + 2 * G < ntiles) issue(t + 2 * G, s);
        fft_batch<false, R, MAXR, true>(buf, ld, tj, a.px, -1, tx.tw, tj);
        T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)k * nxh * ny;
        for (int e = threadIdx.x; e < tj * (n2 + 1); e += blockDim.x) {
            const int kx = (int)fdiv(e, a.fd_tj), rr = e - kx * tj;
            const int k1 = (kx == n2) ? 0 : kx;
            const int k2 = (kx == 0) ? 0 : n2 - kx;
            spec[(long)kx * ny + jb + rr] = r2c_unpack<R>(buf[tx.pos[k1] * ld + rr], buf[tx.pos[k2] * ld + rr], twx[kx]);
        }
        __syncthreads();   // buf free for the next tile
    }
    if (abort_flag && threadIdx.x == 0) {
        // let copies already in flight (tiles t and t + G) land before the
        // block's shared memory is released
        mbar_wait(&bars[n & 1], (unsigned)(n >> 1) & 1u);
        if (t + G < ntiles) mbar_wait(&bars[(n + 1) & 1], (unsigned)((n + 1) >> 1) & 1u);
    }
}

// one y transform of every kx line of a plane, in place on [k][kx][ky]
template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, lines_min_blocks<R, MAXR>()) k_ylines(const PlaneArgs a, int sign,
                                                                                  double scale) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pkeep = pol_keep(a.l2hint);
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int ny = a.ny, nz = a.nz, nxh = a.nxh;
    const int ly = a.ly, ld = ly | 1;
    const PlanTables<R> ty = stage_plan<R>(a.py, smem_raw + align16((size_t)ny * ld * sizeof(T)));
    const int inst = blockIdx.y / nz;
    const int k = blockIdx.y - inst * nz;
    const int l0 = blockIdx.x * ly;
    const int nl = min(ly, nxh - l0);
    T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + ((long)k * nxh + l0) * ny;
    constexpr int LB = sizeof(R) == 8 ? 4 : 8;
    const int total = nl * ny;
    for (int t0 = threadIdx.x; t0 < total; t0 += LB * blockDim.x) {
        T v[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) v[q] = ld_l2(&spec[t], pkeep);
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int line = (int)fdiv(t, a.fd_ny), e = t - line * ny;
                buf[e * ld + line] = v[q];
            }
        }
    }
    fft_batch<false, R, MAXR, true>(buf, ld, nl, a.py, sign, ty.tw, ly);
    const R sc = (R)scale;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int line = (int)fdiv(t, a.fd_ny), q = t - line * ny;   // q: position in shared memory
        st_l2(&spec[(long)line * ny + ty.ipos[q]], cscale(buf[q * ld + line], sc), pkeep);
    }
}

// ---------------------------------------------------------------------------
// y transforms held in registers, for ny = N1 N2 (64, 128, 256): the
// four-step split of one DFT of length N,
//   X[k1 + N1 k2] = sum_n2 w_N2^(n2 k2) w_N^(n2 k1) sum_n1 x[N2 n1 + n2] w_N1^(n1 k1),
// with w_M = exp(sign 2 pi i / M).  A line is N2 adjacent lanes of one warp:
// lane n2 loads x[N2 n1 + n2] straight from HBM (consecutive lanes,
// consecutive addresses), runs the length-N1 DFT in registers, applies
// w_N^(n2 k1) and writes its N1 values to the line's shared-memory tile;
// after a warp barrier lane t takes the N1/N2 rows k1 = t + N2 r, runs the
// length-N2 DFTs and stores X in natural order, again consecutive lanes on
// consecutive addresses.  One shared-memory round trip per element (the
// staged radix stages of k_ylines make one per stage plus the staging), no
// block barrier, no permutation.  Lines run over all planes and instances
// of the [k][kx][ky] array, so partial blocks occur only at the very end.
// ---------------------------------------------------------------------------
template <int N1, int N2>
struct YReg {
    static constexpr int N = N1 * N2;
    static constexpr int LPB = kPlaneThreads / N2;            // lines per block
    static constexpr int LS = N1 * (N2 + 1) + 1;              // tile stride of a line (elements)
};

// four resident blocks in FP32 (64 registers, no spills; 80 and three
// blocks without the bound), two in FP64 (128 registers; capping them spills)
template <typename R, int N1, int N2>
__global__ void __launch_bounds__(kPlaneThreads, sizeof(R) == 4 ? 4 : 2) k_ylines_reg(const PlaneArgs a, long nlines, int sign,
                                                                 double scale) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pkeep = pol_keep(a.l2hint);
    using T = cpx<R>;
    using Y = YReg<N1, N2>;
    static_assert(N1 >= N2 && N1 % N2 == 0, "split");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tl = threadIdx.x % N2;
    const int li = threadIdx.x / N2;
    T* tile = reinterpret_cast<T*>(smem_raw) + li * Y::LS;
    const long g = (long)blockIdx.x * Y::LPB + li;
    const bool valid = g < nlines;
    T* line = reinterpret_cast<T*>(a.spec) + (valid ? g : 0) * Y::N;
    const T* tw = reinterpret_cast<const T*>(sizeof(R) == 8 ? (const void*)a.py.tw : (const void*)a.py.twf);
    T v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = valid ? ld_l2(&line[N2 * n1 + tl], pkeep) : mk<R>((R)0, (R)0);
    small_dft<N1>(v, sign);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
        T w = __ldg(tw + tl * k1);
        if (sign > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) tile[k1 * (N2 + 1) + tl] = v[k1];
    __syncwarp();
    const R sc = (R)scale;
#pragma unroll
    for (int r = 0; r < N1 / N2; ++r) {
        const int k1 = tl + N2 * r;
        T u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = tile[k1 * (N2 + 1) + n2];
        small_dft<N2>(u, sign);
        if (valid) {
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) st_l2(&line[k1 + N1 * k2], cscale(u[k2], sc), pkeep);
        }
    }
}

// ---------------------------------------------------------------------------
// Rows passes held in registers, for nx/2 = N1 N2 (64, 128, 256): the
// half-length complex transform of each row (z_m = s(2m) + i s(2m+1)) by
// the same four-step split as k_ylines_reg.  A block takes kRowsRegTJ
// consecutive rows of one plane, N2 lanes per row.
//   forward: all lanes form z from u, v, w (or the source field) with m
//            fastest into the rows' tiles; lane n2 of a row takes
//            m = N2 n1 + n2, DFT N1, twiddle, warp-local transpose, DFT N2;
//            Z goes to a block tile [m][row] (a barrier, aliasing the row
//            tiles) from which the r2c unpack reads Z_kx and Z_{N-kx} and
//            writes each kx as a run of kRowsRegTJ rows.
//   inverse: the c2r pack reads X_kx and X_{N-kx} in runs of rows into the
//            block tile, lanes take their stride-N2 elements from it, DFT
//            N1, twiddle, transpose, DFT N2, and each lane stores its pairs
//            (2m, 2m+1) straight to p.
// Three (forward) and two (inverse) shared-memory round trips per element
// against the staged kernels' one per radix stage plus staging and the
// unpack gather.
// ---------------------------------------------------------------------------
constexpr int kRowsRegTJ = 16;

template <int N1, int N2, typename R = float>
struct RowReg {
    static constexpr int N = N1 * N2;
    static constexpr int TJ = kRowsRegTJ;
    static constexpr int NT = TJ * N2;                    // threads per block
    // Tile pitches chosen against shared-memory bank conflicts.  FP32
    // complex elements take two 4-byte banks and a half-warp's 16 lanes are
    // served together: with N2 = 8 a half-warp spans two rows, so the rows'
    // transpose tiles start 16 banks apart (LS = 8 mod 16 elements), and in
    // the block tile [m][row], where the lanes of a row step through m, the
    // pitch is TJ + 2 (4 banks per step of m, the two rows 2 banks apart).
    // FP64 complex elements take four banks and a quarter-warp of 8 lanes
    // (one row) is served together: the block tile's pitch is TJ + 1 (4
    // banks per step of m), and the row tiles need no spacing.
    static constexpr bool F32 = sizeof(R) == 4;
    static constexpr int LS0 = N1 * (N2 + 1);
    static constexpr int LS = (F32 && N2 == 8) ? LS0 + (24 - LS0 % 16) % 16 : LS0 + 1;   // transpose tile stride of a row
    static constexpr int LD = F32 ? TJ + 2 : TJ + 1;      // block tile [m][row] pitch
    static constexpr size_t T1 = (size_t)TJ * LS, T2 = (size_t)N * LD;
    static constexpr size_t elems = T1 > T2 ? T1 : T2;
};

// YS (the y-split layout, PlaneArgs::ysplit): a block takes rows jb .. jb+7
// and jb+ny/2 .. jb+ny/2+7 (jb = 8 blockIdx.x) and applies the first radix-2
// stage of the forward y transform to each row pair before the store:
//   E_j = X_j + X_{j+ny/2},  O_j = (X_j - X_{j+ny/2}) w_ny^j   (j < ny/2),
// so that the y transform of every kx line splits into two independent
// half-length transforms, E to the even and O to the odd ky, written as
// [k][kx][half][j] (k_colsolve runs them with the vertical solve).
template <int TJ, bool YS>
__device__ __forceinline__ int rowreg_row(int jb_block, int r, int ny) {
    if constexpr (!YS) return jb_block * TJ + r;
    return jb_block * (TJ / 2) + (r < TJ / 2 ? r : ny / 2 + r - TJ / 2);
}

template <typename R, int N1, int N2, bool YS>
__global__ void __launch_bounds__(RowReg<N1, N2, R>::NT) k_rows_fwd_reg(const PlaneArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long pfield = pol_field(a.l2hint), pkeep = pol_keep(a.l2hint);
    using T = cpx<R>;
    using G = RowReg<N1, N2, R>;
    constexpr int N = G::N, TJ = G::TJ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* tb = reinterpret_cast<T*>(smem_raw);
    const int nz = a.nz, ny = a.ny;
    const int tl = threadIdx.x % N2;
    const int row = threadIdx.x / N2;
    const int jb = blockIdx.x * TJ;
    const int kcnt = a.kcount ? a.kcount : nz;   // levels of the window (z-slab)
    const int inst = blockIdx.y / kcnt;
    // spectral level; zrev walks the planes top down (the step kernel before
    // the forward pass wrote the top levels last, so some are still in L2)
    const int kl = a.zrev ? kcnt - 1 - (int)(blockIdx.y - inst * kcnt) : (int)(blockIdx.y - inst * kcnt);
    const int k = a.kbeg + kl;                    // real-field level
    const long ioff = (long)inst * a.sN;
    const double* asrc = a.src ? a.src + ioff : nullptr;
    const T* tw = reinterpret_cast<const T*>(sizeof(R) == 8 ? (const void*)a.px.tw : (const void*)a.px.twf);
    // z = s(2m) + i s(2m+1) of the block's rows, formed by all lanes with m
    // fastest (coalesced, LB points in flight per lane) into each row's tile
    constexpr int LB = 4;
    static_assert((N * TJ) % (LB * G::NT) == 0, "source batches");
    for (int t0 = threadIdx.x; t0 < N * TJ; t0 += LB * G::NT) {
        double2 d[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * G::NT;
            d[q] = plane_source_pair(a, a.u + ioff, a.v + ioff, a.w + ioff, asrc, k,
                                     rowreg_row<TJ, YS>(blockIdx.x, t / N, ny), t % N, pfield);
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * G::NT;
            tb[(t / N) * G::LS + t % N] = mk<R>((R)d[q].x, (R)d[q].y);
        }
    }
    __syncthreads();
    T* t1 = tb + row * G::LS;   // this row's tile: the source, then the transpose
    T v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = t1[N2 * n1 + tl];
    __syncwarp();
    small_dft<N1>(v, -1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], __ldg(tw + tl * k1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) t1[k1 * (N2 + 1) + tl] = v[k1];
    __syncwarp();
    T z[N1];   // z[r N2 + k2] = Z[k1 + N1 k2], k1 = tl + N2 r
#pragma unroll
    for (int r = 0; r < N1 / N2; ++r) {
        const int k1 = tl + N2 * r;
        T u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = t1[k1 * (N2 + 1) + n2];
        small_dft<N2>(u, -1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) z[r * N2 + k2] = u[k2];
    }
    __syncthreads();   // the transpose tiles are read; the block tile reuses them
#pragma unroll
    for (int r = 0; r < N1 / N2; ++r)
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) tb[(tl + N2 * r + N1 * k2) * G::LD + row] = z[r * N2 + k2];
    __syncthreads();
    if constexpr (YS) {
        constexpr int TH = TJ / 2;
        const int ny2 = ny / 2, j0 = blockIdx.x * TH;
        T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)kl * a.nxh * ny + j0;
        const T* twy = reinterpret_cast<const T*>(sizeof(R) == 8 ? (const void*)a.py.tw : (const void*)a.py.twf);
        for (int t = threadIdx.x; t < (N + 1) * TH; t += G::NT) {
            const int kx = t / TH, rr = t - kx * TH;
            const int k1 = (kx == N) ? 0 : kx;
            const int k2 = (kx == 0) ? 0 : N - kx;
            const double2 w = __ldg(a.twx + kx);
            const T wx = mk<R>((R)w.x, (R)w.y);
            const T xa = r2c_unpack<R>(tb[k1 * G::LD + rr], tb[k2 * G::LD + rr], wx);
            const T xb = r2c_unpack<R>(tb[k1 * G::LD + rr + TH], tb[k2 * G::LD + rr + TH], wx);
            const T wy = __ldg(twy + j0 + rr);   // w_ny^j
            st_l2(&spec[(long)kx * ny + rr], cadd(xa, xb), pkeep);
            st_l2(&spec[(long)kx * ny + ny2 + rr], cmul(csub(xa, xb), wy), pkeep);
        }
    } else {
        T* spec = reinterpret_cast<T*>(a.spec) + (long)inst * a.sM + (long)kl * a.nxh * ny + jb;
        for (int t = threadIdx.x; t < (N + 1) * TJ; t += G::NT) {
            const int kx = t / TJ, rr = t - kx * TJ;
            const int k1 = (kx == N) ? 0 : kx;
            const int k2 = (kx == 0) ? 0 : N - kx;
            const double2 w = __ldg(a.twx + kx);
            st_l2(&spec[(long)kx * ny + rr], r2c_unpack<R>(tb[k1 * G::LD + rr], tb[k2 * G::LD + rr], mk<R>((R)w.x, (R)w.y)),
                  pkeep);
        }
    }
}

// YS: the inverse of the split above: from the half-length inverse
// transforms E' (even ky) and O' (odd ky) of [k][kx][half][j], rows j and
// j+ny/2 of the inverse y transform are E'_j + w_ny^-j O'_j and
// E'_j - w_ny^-j O'_j.
template <typename R, int N1, int N2, bool YS>
__global__ void __launch_bounds__(RowReg<N1, N2, R>::NT) k_rows_inv_reg(const PlaneArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long plast = pol_last(a.l2hint);
    using T = cpx<R>;
    using G = RowReg<N1, N2, R>;
    constexpr int N = G::N, TJ = G::TJ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* tb = reinterpret_cast<T*>(smem_raw);
    const int nz = a.nz, ny = a.ny, nx = a.nx;
    const int tl = threadIdx.x % N2;
    const int row = threadIdx.x / N2;
    const int jb = blockIdx.x * TJ;
    const int kcnt = a.kcount ? a.kcount : nz;   // levels of the window (z-slab)
    const int inst = blockIdx.y / kcnt;
    // spectral level; zrev walks the planes top down (the step kernel before
    // the forward pass wrote the top levels last, so some are still in L2)
    const int kl = a.zrev ? kcnt - 1 - (int)(blockIdx.y - inst * kcnt) : (int)(blockIdx.y - inst * kcnt);
    const int k = a.kbeg + kl;                    // real-field level
    const T* spec = reinterpret_cast<const T*>(a.spec) + (long)inst * a.sM + (long)kl * a.nxh * ny + jb;
    const T* tw = reinterpret_cast<const T*>(sizeof(R) == 8 ? (const void*)a.px.tw : (const void*)a.px.twf);
    // c2r pack into the block tile [m][row], loads batched per thread
    if constexpr (YS) {
        constexpr int TH = TJ / 2, LB2 = 2;
        static_assert((N * TH) % (LB2 * G::NT) == 0, "pack batches");
        const int ny2 = ny / 2, j0 = blockIdx.x * TH;
        const T* sp = reinterpret_cast<const T*>(a.spec) + (long)inst * a.sM + (long)kl * a.nxh * ny + j0;
        const T* twy = reinterpret_cast<const T*>(sizeof(R) == 8 ? (const void*)a.py.tw : (const void*)a.py.twf);
        for (int t0 = threadIdx.x; t0 < N * TH; t0 += LB2 * G::NT) {
            T ek[LB2], ok[LB2], ec[LB2], oc[LB2];
#pragma unroll
            for (int q = 0; q < LB2; ++q) {
                const int t = t0 + q * G::NT;
                const int kk = t / TH, rr = t - kk * TH;
                ek[q] = ld_l2(&sp[(long)kk * ny + rr], plast);
                ok[q] = ld_l2(&sp[(long)kk * ny + ny2 + rr], plast);
                ec[q] = ld_l2(&sp[(long)(N - kk) * ny + rr], plast);
                oc[q] = ld_l2(&sp[(long)(N - kk) * ny + ny2 + rr], plast);
            }
#pragma unroll
            for (int q = 0; q < LB2; ++q) {
                const int t = t0 + q * G::NT;
                const int kk = t / TH, rr = t - kk * TH;
                const double2 w = __ldg(a.twx + kk);
                const T wx = mk<R>((R)w.x, (R)w.y);
                T wy = __ldg(twy + j0 + rr);
                wy.y = -wy.y;   // w_ny^-j
                const T ok2 = cmul(ok[q], wy), oc2 = cmul(oc[q], wy);
                tb[kk * G::LD + rr] = c2r_pack<R>(cadd(ek[q], ok2), cadd(ec[q], oc2), wx, kk == 0);
                tb[kk * G::LD + rr + TH] = c2r_pack<R>(csub(ek[q], ok2), csub(ec[q], oc2), wx, kk == 0);
            }
        }
    } else {
    constexpr int LB = 4;
    static_assert((N * TJ) % (LB * G::NT) == 0, "pack batches");
    for (int t0 = threadIdx.x; t0 < N * TJ; t0 += LB * G::NT) {
        T xk[LB], xc[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * G::NT;
            const int kk = t / TJ, rr = t - kk * TJ;
            xk[q] = ld_l2(&spec[(long)kk * ny + rr], plast);
            xc[q] = ld_l2(&spec[(long)(N - kk) * ny + rr], plast);
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * G::NT;
            const int kk = t / TJ, rr = t - kk * TJ;
            const double2 w = __ldg(a.twx + kk);
            tb[kk * G::LD + rr] = c2r_pack<R>(xk[q], xc[q], mk<R>((R)w.x, (R)w.y), kk == 0);
        }
    }
    }
    __syncthreads();
    T v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = tb[(N2 * n1 + tl) * G::LD + row];
    __syncthreads();   // the block tile is read; the transpose tiles reuse it
    small_dft<N1>(v, +1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
        T w = __ldg(tw + tl * k1);
        w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    T* t1 = tb + row * G::LS;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) t1[k1 * (N2 + 1) + tl] = v[k1];
    __syncwarp();
    const double sc = a.scale;
    double* out = a.out + (long)inst * a.sN + (long)k * nx * ny + (long)rowreg_row<TJ, YS>(blockIdx.x, row, ny) * nx;
#pragma unroll
    for (int r = 0; r < N1 / N2; ++r) {
        const int k1 = tl + N2 * r;
        T u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = t1[k1 * (N2 + 1) + n2];
        small_dft<N2>(u, +1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            const int m = k1 + N1 * k2;
            double2 o = make_double2((double)u[k2].x * sc, (double)u[k2].y * sc);
            double2* g = reinterpret_cast<double2*>(out + 2 * m);
            if (a.beta != 0.0) {
                const double2 prev = *g;
                o.x = o.x + a.beta * prev.x; o.y = o.y + a.beta * prev.y;
            }
            *g = o;
        }
    }
}

template <typename R, int MAXR>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_blocks<MAXR>()) k_rows_inv(const PlaneArgs a) {
    pdl_trigger();
    pdl_wait();   // inputs written by the preceding kernels
    const unsigned long long plast = pol_last(a.l2hint);
    using T = cpx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = a.nxh, n2 = nx / 2;
    const int tj = a.tj, ld = tj | 1;
    unsigned char* tail = smem_raw + align16((size_t)n2 * ld * sizeof(T));
    const PlanTables<R> tx = stage_plan<R>(a.px, tail);
    const T* twx = stage_twx<R>(a, tail + plan_tables_bytes(n2, sizeof(T)));
    const int jb = blockIdx.x * tj;
    const int kcnt = a.kcount ? a.kcount : nz;   // levels of the window (z-slab)
    const int inst = blockIdx.y / kcnt;
    // spectral level; zrev walks the planes top down (the step kernel before
    // the forward pass wrote the top levels last, so some are still in L2)
    const int kl = a.zrev ? kcnt - 1 - (int)(blockIdx.y - inst * kcnt) : (int)(blockIdx.y - inst * kcnt);
    const int k = a.kbeg + kl;                    // real-field level
    const long plane = (long)nx * ny;
    const T* spec = reinterpret_cast<const T*>(a.spec) + (long)inst * a.sM + (long)kl * nxh * ny;
    double* out = a.out + (long)inst * a.sN;
    __syncthreads();   // twx staged
    constexpr int LB = sizeof(R) == 8 ? 2 : 4;
    const int total = tj * n2;
    for (int t0 = threadIdx.x; t0 < total; t0 += LB * blockDim.x) {
        T xk[LB], xc[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int kk = (int)fdiv(t, a.fd_tj), rr = t - kk * tj;
                xk[q] = ld_l2(&spec[(long)kk * ny + jb + rr], plast);
                xc[q] = ld_l2(&spec[(long)(n2 - kk) * ny + jb + rr], plast);
            }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int t = t0 + q * blockDim.x;
            if (t < total) {
                const int kk = (int)fdiv(t, a.fd_tj), rr = t - kk * tj;
                buf[kk * ld + rr] = c2r_pack<R>(xk[q], xc[q], twx[kk], kk == 0);
            }
        }
    }
    fft_batch<false, R, MAXR, true>(buf, ld, tj, a.px, +1, tx.tw, tj);
    const double sc = a.scale;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int rr = (int)fdiv(t, a.fd_n2), q = t - rr * n2;
        const int m = tx.ipos[q];
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
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    return align16((size_t)(a.nx / 2) * (a.tj | 1) * es) + tables_x_bytes(a, es);
}
size_t ylines_smem(const PlaneArgs& a, bool fp32) {
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    return align16((size_t)a.ny * (a.ly | 1) * es) + tables_y_bytes(a, es);
}
size_t plane_fwd_smem(const PlaneArgs& a, bool fp32) {
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    return align16(((size_t)a.ny * a.ldc + (size_t)(a.nx / 2) * a.ldr) * es) + tables_x_bytes(a, es) +
           tables_y_bytes(a, es);
}
size_t plane_inv_smem(const PlaneArgs& a, bool fp32) { return plane_fwd_smem(a, fp32); }
size_t pipe_smem(const PlaneArgs& a, bool fp32);
size_t plane_smem(const PlaneArgs& a, bool fp32) {
    if (a.impl == 2) return std::max(pipe_smem(a, fp32), std::max(rows_smem(a, fp32), ylines_smem(a, fp32)));
    if (a.impl == 1) return std::max(rows_smem(a, fp32), ylines_smem(a, fp32));
    return plane_fwd_smem(a, fp32);
}

static int maxr_x(const PlaneArgs& a) { return plan_max_radix(a.px) >= 16 ? 16 : 8; }
static int maxr_y(const PlaneArgs& a) { return plan_max_radix(a.py) >= 16 ? 16 : 8; }

size_t pipe_smem(const PlaneArgs& a, bool fp32) {
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    return 2 * pipe_stage_bytes(a) + align16((size_t)(a.nx / 2) * (a.tj | 1) * es) + tables_x_bytes(a, es) +
           2 * sizeof(unsigned long long);
}

template <typename R, int MX>
static cudaError_t launch_pipe(const PlaneArgs& a, cudaStream_t s) {
    const size_t sm = pipe_smem(a, sizeof(R) == 4);
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rows_fwd_pipe<R, MX>, kPlaneThreads, sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int ntiles = (a.ny / a.tj) * a.nz * std::max(1, a.batch);
    const int grid = std::min(ntiles, per_sm * sms);
    k_rows_fwd_pipe<R, MX><<<grid, kPlaneThreads, sm, s>>>(a, ntiles);
    return cudaGetLastError();
}

template <typename R, int N1, int N2>
static cudaError_t launch_ylines_reg_t(const PlaneArgs& a, int sign, double scale, cudaStream_t s) {
    using Y = YReg<N1, N2>;
    const long nlines = (long)a.nxh * a.nz * std::max(1, a.batch);
    const size_t sm = (size_t)Y::LPB * Y::LS * sizeof(cpx<R>);
    return launch_pdl(k_ylines_reg<R, N1, N2>, dim3((unsigned)((nlines + Y::LPB - 1) / Y::LPB)), dim3(kPlaneThreads), sm, s,
                      a, nlines, sign, scale);
}
// the register y transform when ny has a two-factor split, else false
bool ylines_in_registers(int ny) { return ny == 64 || ny == 128 || ny == 256; }

template <typename R>
static bool ylines_reg(const PlaneArgs& a, int sign, double scale, cudaStream_t s, cudaError_t* e) {
    switch (a.ny) {
        case 64: *e = launch_ylines_reg_t<R, 8, 8>(a, sign, scale, s); return true;
        case 128: *e = launch_ylines_reg_t<R, 16, 8>(a, sign, scale, s); return true;
        case 256: *e = launch_ylines_reg_t<R, 16, 16>(a, sign, scale, s); return true;
        default: return false;
    }
}

bool rows_in_registers(int nx, int ny) {
    return (nx == 128 || nx == 256 || nx == 512) && ny % kRowsRegTJ == 0;
}
template <typename R, int N1, int N2>
static cudaError_t launch_rows_reg_t(const PlaneArgs& a, bool fwd, cudaStream_t s) {
    using G = RowReg<N1, N2, R>;
    const dim3 g(a.ny / G::TJ, (a.kcount ? a.kcount : a.nz) * std::max(1, a.batch));
    const size_t sm = G::elems * sizeof(cpx<R>);
    if (a.ysplit) {
        if (fwd) return launch_pdl(k_rows_fwd_reg<R, N1, N2, true>, g, dim3(G::NT), sm, s, a);
        return launch_pdl(k_rows_inv_reg<R, N1, N2, true>, g, dim3(G::NT), sm, s, a);
    }
    if (fwd) return launch_pdl(k_rows_fwd_reg<R, N1, N2, false>, g, dim3(G::NT), sm, s, a);
    return launch_pdl(k_rows_inv_reg<R, N1, N2, false>, g, dim3(G::NT), sm, s, a);
    return cudaGetLastError();
}
// The register rows pass when nx/2 has a two-factor split, else false.  The
// FP64 forward pass keeps the staged kernel: its register form needs ~92
// registers for the 16 source points of a lane and runs 5 blocks per SM,
// too few to cover the six loads per point (112.8 vs 105.4 us for the
// forward transform at 256x256x128); in FP32 it runs 7 (87 vs 100 us).
template <typename R>
static bool rows_reg(const PlaneArgs& a, bool fwd, cudaStream_t s, cudaError_t* e) {
    if (fwd && sizeof(R) == 8) return false;
    if (!rows_in_registers(a.nx, a.ny)) return false;
    switch (a.nx) {
        case 128: *e = launch_rows_reg_t<R, 8, 8>(a, fwd, s); return true;
        case 256: *e = launch_rows_reg_t<R, 16, 8>(a, fwd, s); return true;
        case 512: *e = launch_rows_reg_t<R, 16, 16>(a, fwd, s); return true;
        default: return false;
    }
}

template <typename R, int MX, int MY>
static cudaError_t launch_split_m(const PlaneArgs& a, bool fwd, cudaStream_t s) {
    const int nb = std::max(1, a.batch);
    const int kcnt = a.kcount ? a.kcount : a.nz;
    const dim3 grows(a.ny / a.tj, kcnt * nb), glines((a.nxh + a.ly - 1) / a.ly, kcnt * nb);
    // the y-lines passes see only the spectral array: kcnt levels
    PlaneArgs ay = a;
    ay.nz = kcnt; ay.kbeg = 0; ay.kcount = 0;
    const size_t smr = rows_smem(a, sizeof(R) == 4), sml = ylines_smem(a, sizeof(R) == 4);
    cudaError_t e = cudaSuccess;
    if (fwd && a.impl == 2 && a.mode != 2) {
        e = launch_pipe<R, MX>(a, s);
        if (e != cudaSuccess) return e;
        if (!ylines_reg<R>(ay, -1, a.scale, s, &e))
            e = launch_pdl(k_ylines<R, MY>, glines, dim3(kPlaneThreads), sml, s, ay, -1, a.scale);
    } else if (fwd && a.ysplit) {   // the y transforms run inside k_colsolve
        if (!rows_reg<R>(a, true, s, &e)) return cudaErrorInvalidValue;
    } else if (a.ysplit) {
        if (!rows_reg<R>(a, false, s, &e)) return cudaErrorInvalidValue;
    } else if (fwd) {
        if (!rows_reg<R>(a, true, s, &e)) e = launch_pdl(k_rows_fwd<R, MX>, grows, dim3(kPlaneThreads), smr, s, a);
        if (e != cudaSuccess) return e;
        if (!ylines_reg<R>(ay, -1, a.scale, s, &e))
            e = launch_pdl(k_ylines<R, MY>, glines, dim3(kPlaneThreads), sml, s, ay, -1, a.scale);
    } else {
        if (!ylines_reg<R>(ay, +1, 1.0, s, &e))
            e = launch_pdl(k_ylines<R, MY>, glines, dim3(kPlaneThreads), sml, s, ay, +1, 1.0);
        if (e != cudaSuccess) return e;
        if (!rows_reg<R>(a, false, s, &e)) e = launch_pdl(k_rows_inv<R, MX>, grows, dim3(kPlaneThreads), smr, s, a);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}
int l2hint_mode() {
    static const int m = [] {
        const char* e = std::getenv("PS3D_L2HINT");
        return e ? std::atoi(e) : 1;
    }();
    return m;
}

template <typename R>
static cudaError_t launch_split_t(const PlaneArgs& a0, bool fwd, cudaStream_t s) {
    PlaneArgs a = a0;
    a.l2hint = l2hint_mode();
    // the forward rows pass walks the planes top down (PS3D_ZREV=0: bottom
    // up): the step kernel wrote the top levels last, so some are still in
    // L2 (FP64 forward transform 109 -> 103 us at 256x256x128; the inverse
    // pass top down measured slower, 58 -> 62 us, and keeps the bottom-up order)
    static const int zrev = [] {
        const char* e = std::getenv("PS3D_ZREV");
        return e && e[0] == '0' ? 0 : 1;
    }();
    a.zrev = fwd ? zrev : 0;
    a.fd_n2 = make_fastdiv(a.nx / 2);
    a.fd_ny = make_fastdiv(a.ny);
    a.fd_tj = make_fastdiv(a.tj);
    const int mx = maxr_x(a), my = maxr_y(a);
    if (mx == 16 && my == 16) return launch_split_m<R, 16, 16>(a, fwd, s);
    if (mx == 16) return launch_split_m<R, 16, 8>(a, fwd, s);
    if (my == 16) return launch_split_m<R, 8, 16>(a, fwd, s);
    return launch_split_m<R, 8, 8>(a, fwd, s);
}

// opt a kernel in to the largest dynamic shared memory its static shared
// memory leaves within the 227 KB a block may use
template <typename K>
static cudaError_t max_dynamic_smem(K kernel) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                227 * 1024 - (int)fa.sharedSizeBytes);
}

template <typename R, int MAXR>
static cudaError_t setup_m() {
    cudaError_t e;
    const int maxsm = 227 * 1024;
    if ((e = cudaFuncSetAttribute(k_plane_fwd<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_inv<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_fwd<R, MAXR>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
    if ((e = cudaFuncSetAttribute(k_plane_inv<R, MAXR>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_fwd<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_rows_inv<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_ylines<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = max_dynamic_smem(k_rows_fwd_pipe<R, MAXR>))) return e;
    return cudaSuccess;
}
template <typename R>
static cudaError_t setup_t() {
    cudaError_t e;
    if ((e = max_dynamic_smem(k_ylines_reg<R, 8, 8>))) return e;
    if ((e = max_dynamic_smem(k_ylines_reg<R, 16, 8>))) return e;
    if ((e = max_dynamic_smem(k_ylines_reg<R, 16, 16>))) return e;
#define PS3D_ROWS_SETUP(YS)                                                   \
    if ((e = max_dynamic_smem(k_rows_fwd_reg<R, 8, 8, YS>))) return e;       \
    if ((e = max_dynamic_smem(k_rows_fwd_reg<R, 16, 8, YS>))) return e;      \
    if ((e = max_dynamic_smem(k_rows_fwd_reg<R, 16, 16, YS>))) return e;     \
    if ((e = max_dynamic_smem(k_rows_inv_reg<R, 8, 8, YS>))) return e;       \
    if ((e = max_dynamic_smem(k_rows_inv_reg<R, 16, 8, YS>))) return e;      \
    if ((e = max_dynamic_smem(k_rows_inv_reg<R, 16, 16, YS>))) return e;
    PS3D_ROWS_SETUP(false)
    PS3D_ROWS_SETUP(true)
#undef PS3D_ROWS_SETUP
    if ((e = cudaFuncSetAttribute(k_zsolve<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024))) return e;
    if ((e = max_dynamic_smem(k_thomas2<R, false, false>))) return e;
    if ((e = max_dynamic_smem(k_thomas2<R, true, false>))) return e;
    if ((e = max_dynamic_smem(k_thomas2<R, false, true>))) return e;
    if ((e = max_dynamic_smem(k_thomas2<R, true, true>))) return e;
    if ((e = max_dynamic_smem(k_colsolve))) return e;
    if ((e = max_dynamic_smem(k_colsolve2))) return e;
    if ((e = max_dynamic_smem(k_thomas<R, true>))) return e;
    if ((e = max_dynamic_smem(k_thomas<R, false>))) return e;
    if ((e = setup_m<R, 16>())) return e;
    return setup_m<R, 8>();
}
cudaError_t plane_setup(bool fp32) { return fp32 ? setup_t<float>() : setup_t<double>(); }

static cudaLaunchConfig_t plane_cfg(const PlaneArgs& a, bool fp32, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.C, a.nz * std::max(1, a.batch), 1);
    cfg.blockDim = dim3(kPlaneThreads, 1, 1);
    cfg.dynamicSmemBytes = plane_fwd_smem(a, fp32);
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <typename R, bool FWD, int MAXR>
static cudaError_t launch_plane_m(const PlaneArgs& a, cudaStream_t s) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_cfg(a, sizeof(R) == 4, attr);
    cfg.stream = s;
    if (FWD) return cudaLaunchKernelEx(&cfg, k_plane_fwd<R, MAXR>, a);
    return cudaLaunchKernelEx(&cfg, k_plane_inv<R, MAXR>, a);
}
template <typename R, bool FWD>
static cudaError_t launch_plane_t(const PlaneArgs& a0, cudaStream_t s) {
    PlaneArgs a = a0;
    a.l2hint = l2hint_mode();
    if (std::max(maxr_x(a), maxr_y(a)) >= 16) return launch_plane_m<R, FWD, 16>(a, s);
    return launch_plane_m<R, FWD, 8>(a, s);
}
template <typename R, bool FWD, int MAXR>
static int max_clusters_m(const PlaneArgs& a) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_cfg(a, sizeof(R) == 4, attr);
    int n = 0;
    cudaError_t e = FWD ? cudaOccupancyMaxActiveClusters(&n, k_plane_fwd<R, MAXR>, &cfg)
                        : cudaOccupancyMaxActiveClusters(&n, k_plane_inv<R, MAXR>, &cfg);
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}
template <typename R, bool FWD>
static int max_clusters_t(const PlaneArgs& a) {
    if (std::max(maxr_x(a), maxr_y(a)) >= 16) return max_clusters_m<R, FWD, 16>(a);
    return max_clusters_m<R, FWD, 8>(a);
}
int plane_max_clusters(const PlaneArgs& a, bool fp32, bool fwd) {
    if (fp32) return fwd ? max_clusters_t<float, true>(a) : max_clusters_t<float, false>(a);
    return fwd ? max_clusters_t<double, true>(a) : max_clusters_t<double, false>(a);
}

cudaError_t launch_plane_fwd(const PlaneArgs& a, bool fp32, cudaStream_t s) {
    if ((a.kcount || a.kbeg) && a.impl != 1) return cudaErrorInvalidValue;   // level windows: implementation 1 only
    if (a.impl >= 1) return fp32 ? launch_split_t<float>(a, true, s) : launch_split_t<double>(a, true, s);
    return fp32 ? launch_plane_t<float, true>(a, s) : launch_plane_t<double, true>(a, s);
}
cudaError_t launch_plane_inv(const PlaneArgs& a, bool fp32, cudaStream_t s) {
    if ((a.kcount || a.kbeg) && a.impl != 1) return cudaErrorInvalidValue;
    if (a.impl >= 1) return fp32 ? launch_split_t<float>(a, false, s) : launch_split_t<double>(a, false, s);
    return fp32 ? launch_plane_t<float, false>(a, s) : launch_plane_t<double, false>(a, s);
}

// threads per block of the vertical solve: 128 while its checkpoints fit
// in a block's shared memory, fewer for tall columns; 0 when not even 32 fit
int thomas_threads(int nz) {
    for (int t = kThomasThreads; t >= 32; t /= 2)
        if (thomas_smem(nz, t) <= 227 * 1024 - 64) return t;
    return 0;
}

cudaError_t launch_thomas(const ColumnArgs& a0, bool fp32, cudaStream_t s) {
    ColumnArgs a = a0;
    a.l2hint = l2hint_mode();
    const long ncols = a.ncl ? a.ncl : (long)a.nxh * a.ny;
    a.fd_ncols = make_fastdiv((unsigned)ncols);
    a.fd_ny = make_fastdiv(a.ny);
    a.fd_nxh = make_fastdiv(a.nxh);
    // the two-ended form with two threads per column where 4 blocks of 128
    // fit an SM, else the one-ended form with as many threads per block as
    // its checkpoints allow; PS3D_THOMAS_FORM=0|2|3 pins one (3: the
    // two-ended form with its pivot table); PS3D_THOMAS_FULL=0 keeps the
    // bounds-tested instantiation of the two-ended form on every grid
    const char* pin = std::getenv("PS3D_THOMAS_FORM");
    const char* fe = std::getenv("PS3D_THOMAS_FULL");
    const int form = pin ? pin[0] - '0' : (thomas2_smem(a.nz, kThomasThreads) <= 56 * 1024 ? 2 : 0);
    const bool off32 = (long)a.nz * 2 * ncols < (1L << 32);   // 32-bit level offsets
    const bool full = a.nz % (2 * kThomasChunk) == 0 && !(fe && fe[0] == '0');
    const long n2 = 2 * ncols * std::max(1, a.batch);
    if (form == 3 && off32 && thomas2r_smem(a.nz, kThomas2RThreads) <= 227 * 1024 - 64) {
        const dim3 g((unsigned)((n2 + kThomas2RThreads - 1) / kThomas2RThreads)), b(kThomas2RThreads);
        const size_t sm = thomas2r_smem(a.nz, kThomas2RThreads);
        if (full) return fp32 ? launch_pdl(k_thomas2<float, true, true>, g, b, sm, s, a)
                              : launch_pdl(k_thomas2<double, true, true>, g, b, sm, s, a);
        return fp32 ? launch_pdl(k_thomas2<float, false, true>, g, b, sm, s, a)
                    : launch_pdl(k_thomas2<double, false, true>, g, b, sm, s, a);
    }
    if (form == 2 && off32 && thomas2_smem(a.nz, kThomasThreads) <= 227 * 1024 - 64) {
        const dim3 g((unsigned)((n2 + kThomasThreads - 1) / kThomasThreads)), b(kThomasThreads);
        const size_t sm = thomas2_smem(a.nz, kThomasThreads);
        if (full) return fp32 ? launch_pdl(k_thomas2<float, true, false>, g, b, sm, s, a)
                              : launch_pdl(k_thomas2<double, true, false>, g, b, sm, s, a);
        return fp32 ? launch_pdl(k_thomas2<float, false, false>, g, b, sm, s, a)
                    : launch_pdl(k_thomas2<double, false, false>, g, b, sm, s, a);
    }
    const int nt = thomas_threads(a.nz);
    if (nt == 0 || ncols < 1) return cudaErrorInvalidValue;
    const long nthreads = 2 * ncols * std::max(1, a.batch);
    const int blocks = (int)((nthreads + nt - 1) / nt);
    const size_t sm = thomas_smem(a.nz, nt);
    const dim3 g(blocks), b(nt);
    if (a.nz % kThomasChunk == 0) {
        if (fp32) return launch_pdl(k_thomas<float, true>, g, b, sm, s, a);
        return launch_pdl(k_thomas<double, true>, g, b, sm, s, a);
    }
    if (fp32) return launch_pdl(k_thomas<float, false>, g, b, sm, s, a);
    return launch_pdl(k_thomas<double, false>, g, b, sm, s, a);
}

static size_t zsolve_smem(int nz, size_t es) {
    return align16((size_t)nz * (kZLines + 1) * es) + plan_tables_bytes(nz, es);
}
bool zsolve_fits(int nz, bool fp32) {
    return zsolve_smem(nz, fp32 ? sizeof(float2) : sizeof(double2)) <= 227 * 1024;
}

cudaError_t launch_zsolve(const ColumnArgs& a, bool fp32, cudaStream_t s) {
    const long ncols = a.ncl ? a.ncl : (long)a.nxh * a.ny;
    const int blocks = (int)(((ncols + kZLines - 1) / kZLines) * std::max(1, a.batch));
    const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
    const size_t sm = zsolve_smem(a.nz, es);
    if (sm > 227 * 1024) return cudaErrorInvalidValue;
    if (fp32) k_zsolve<float><<<blocks, 256, sm, s>>>(a);
    else k_zsolve<double><<<blocks, 256, sm, s>>>(a);
    return cudaGetLastError();
}

}  // namespace ps3d
