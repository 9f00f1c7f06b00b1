// fft.cuh — batched in-place mixed-radix FFTs in shared memory.
//
// Replaces the 1D FFTW kernels inside P3DFFT (call sites my_fft.f90:165-244).
// A batch of `nlines` complex lines of length P.n is stored interleaved,
// element e of line l at buf[e * ld + l] (ld >= nlines, odd ld avoids bank
// conflicts), so a warp works on the same butterfly of consecutive lines and
// shares one twiddle.  Two in-place variants share one index scheme:
//   fft_dit: input in digit-reversed order (P.pos), output natural;
//   fft_dif: input natural, output digit-reversed.
// DIF is the transpose of DIT (the DFT matrix is symmetric), so a forward DIF
// followed by an inverse DIT needs no permutation pass.  Both are
// unnormalised; sign = -1 is FFTW_FORWARD (e^{-i}), +1 backward.
#pragma once
#include "common.cuh"

namespace ps3d {

// Shared-memory copy of one plan's tables: the twiddles in the working
// precision, the digit-reversal permutation and its inverse.  Staging them
// once per block keeps the butterflies off the L1/L2 load path.
template <typename R>
struct PlanTables {
    const cpx<R>* tw;
    const int* pos;
    const int* ipos;
};

PS3D_HD constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
PS3D_HD size_t plan_tables_bytes(int n, size_t es) {
    return align16((size_t)n * es) + 2 * align16((size_t)n * sizeof(int));
}

// Block-cooperative copy into dst (16-byte aligned, plan_tables_bytes long).
// The caller synchronises the block before the tables are read.
template <typename R>
__device__ PlanTables<R> stage_plan(const FFTPlan& P, unsigned char* dst) {
    cpx<R>* t = reinterpret_cast<cpx<R>*>(dst);
    int* p = reinterpret_cast<int*>(dst + align16((size_t)P.n * sizeof(cpx<R>)));
    int* q = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(p) + align16((size_t)P.n * sizeof(int)));
    for (int e = threadIdx.x; e < P.n; e += blockDim.x) {
        if constexpr (sizeof(R) == 8) t[e] = __ldg(P.tw + e);
        else t[e] = __ldg(P.twf + e);
        p[e] = __ldg(P.pos + e);
        q[e] = __ldg(P.ipos + e);
    }
    return {t, p, q};
}

// radix-RAD DFT in registers: y_m = sum_q v_q exp(sign 2 pi i q m / RAD)
template <int RAD, typename T>
PS3D_HD void small_dft(T* v, int sign) {
    using R = decltype(v[0].x);
    if constexpr (RAD == 2) {
        T a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if constexpr (RAD == 4) {
        T a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        T c = cadd(v[1], v[3]), d = cmul_si(csub(v[1], v[3]), sign);
        v[0] = cadd(a, c); v[2] = csub(a, c);
        v[1] = cadd(b, d); v[3] = csub(b, d);
    } else if constexpr (RAD == 3) {
        const R h = (R)0.86602540378443864676;  // sqrt(3)/2
        T c = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        T m = csub(v[0], cscale(c, (R)0.5));
        T e = cscale(cmul_si(d, sign), h);
        v[0] = cadd(v[0], c);
        v[1] = cadd(m, e); v[2] = csub(m, e);
    } else if constexpr (RAD == 8) {
        // radix 2 x 4: y_m = E_m + W8^m O_m, y_{m+4} = E_m - W8^m O_m
        const R h = (R)0.70710678118654752440;   // sqrt(1/2)
        T e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        small_dft<4>(e, sign);
        small_dft<4>(o, sign);
        const T o1 = mk<R>(h * (o[1].x - sign * o[1].y), h * (o[1].y + sign * o[1].x));   // W8^1
        const T o2 = cmul_si(o[2], sign);                                                // W8^2 = s i
        const T o3 = mk<R>(h * (-o[3].x - sign * o[3].y), h * (sign * o[3].x - o[3].y)); // W8^3
        v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
    } else if constexpr (RAD == 16) {
        // radix 4 x 4: A[q2][m1] = DFT4_q1(v[4 q1 + q2]) W16^{q2 m1}; y[m1 + 4 m2] = DFT4_q2(A[q2][m1])
        const R cs[10] = {(R)1.0, (R)0.92387953251128675613, (R)0.70710678118654752440, (R)0.38268343236508977173,
                          (R)0.0, (R)-0.38268343236508977173, (R)-0.70710678118654752440, (R)-0.92387953251128675613,
                          (R)-1.0, (R)-0.92387953251128675613};
        const R sn[10] = {(R)0.0, (R)0.38268343236508977173, (R)0.70710678118654752440, (R)0.92387953251128675613,
                          (R)1.0, (R)0.92387953251128675613, (R)0.70710678118654752440, (R)0.38268343236508977173,
                          (R)0.0, (R)-0.38268343236508977173};
        T A[4][4];
#pragma unroll
        for (int q2 = 0; q2 < 4; ++q2) {
            T t[4] = {v[q2], v[4 + q2], v[8 + q2], v[12 + q2]};
            small_dft<4>(t, sign);
#pragma unroll
            for (int m1 = 0; m1 < 4; ++m1) {
                const int e = q2 * m1;
                A[q2][m1] = e == 0 ? t[m1] : cmul(t[m1], mk<R>(cs[e], sign * sn[e]));
            }
        }
#pragma unroll
        for (int m1 = 0; m1 < 4; ++m1) {
            T t[4] = {A[0][m1], A[1][m1], A[2][m1], A[3][m1]};
            small_dft<4>(t, sign);
#pragma unroll
            for (int m2 = 0; m2 < 4; ++m2) v[m1 + 4 * m2] = t[m2];
        }
    } else if constexpr (RAD == 5) {
        const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
        const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
        T a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        T a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        T t0 = v[0];
        T m1 = cadd(t0, cadd(cscale(a1, c1), cscale(a2, c2)));
        T m2 = cadd(t0, cadd(cscale(a1, c2), cscale(a2, c1)));
        T e1 = cmul_si(cadd(cscale(b1, s1), cscale(b2, s2)), sign);
        T e2 = cmul_si(csub(cscale(b1, s2), cscale(b2, s1)), sign);
        v[0] = cadd(t0, cadd(a1, a2));
        v[1] = cadd(m1, e1); v[4] = csub(m1, e1);
        v[2] = cadd(m2, e2); v[3] = csub(m2, e2);
    }
}

// Work split of one batched stage in fixed-line mode: every thread keeps one
// line slot (nslots divides the block size) and steps through butterflies,
// so no per-item division is needed; slots beyond the active lines idle.
struct StageSplit {
    int line0, bfly0, bstep;
};
__device__ __forceinline__ StageSplit stage_split(int nslots) {
    StageSplit s;
    s.line0 = threadIdx.x % nslots;
    s.bfly0 = threadIdx.x / nslots;
    s.bstep = blockDim.x / nslots;
    return s;
}

template <int RAD, bool DIT, typename R>
__device__ __forceinline__ void fft_butterfly(cpx<R>* buf, int ld, int line, int base, int Lp, int j, int tstride,
                                              int sign, const cpx<R>* tw) {
    using T = cpx<R>;
    T v[RAD];
#pragma unroll
    for (int q = 0; q < RAD; ++q) v[q] = buf[(base + q * Lp) * ld + line];
    if (DIT && j) {
#pragma unroll
        for (int q = 1; q < RAD; ++q) {
            T w = tw[q * j * tstride];
            if (sign > 0) w.y = -w.y;
            v[q] = cmul(v[q], w);
        }
    }
    small_dft<RAD>(v, sign);
    if (!DIT && j) {
#pragma unroll
        for (int q = 1; q < RAD; ++q) {
            T w = tw[q * j * tstride];
            if (sign > 0) w.y = -w.y;
            v[q] = cmul(v[q], w);
        }
    }
#pragma unroll
    for (int q = 0; q < RAD; ++q) buf[(base + q * Lp) * ld + line] = v[q];
}

template <int RAD, bool DIT, bool FIXED, typename R>
__device__ __forceinline__ void fft_stage(cpx<R>* buf, int ld, int nlines, const FFTPlan& P,
                                          int Lp, int sign, const cpx<R>* tw, const StageSplit& sp) {
    const int n = P.n;
    const int L = Lp * RAD;
    const int tstride = n / L;
    const int nb = n / RAD;
    if constexpr (FIXED) {
        if (sp.line0 >= nlines) return;
        const bool p2 = (Lp & (Lp - 1)) == 0;
        const int lg = __ffs(Lp) - 1;
        for (int bfly = sp.bfly0; bfly < nb; bfly += sp.bstep) {
            const int blk = p2 ? (bfly >> lg) : bfly / Lp;
            const int j = bfly - blk * Lp;
            fft_butterfly<RAD, DIT, R>(buf, ld, sp.line0, blk * L + j, Lp, j, tstride, sign, tw);
        }
    } else {
        const int total = nb * nlines;
        for (int item = threadIdx.x; item < total; item += blockDim.x) {
            const int bfly = item / nlines;
            const int line = item - bfly * nlines;
            const int blk = bfly / Lp;
            const int j = bfly - blk * Lp;
            fft_butterfly<RAD, DIT, R>(buf, ld, line, blk * L + j, Lp, j, tstride, sign, tw);
        }
    }
}

// Whole-block batched FFT.  Must be called by every thread of the block; it
// synchronises the block before returning.  tw: the plan's twiddles staged
// in shared memory (stage_plan).  MAXR is the largest radix instantiated:
// kernels built with MAXR = 8 hold fewer registers and run more blocks per
// SM, and only take plans without radix-16 stages.  NSLOTS > 0 selects the
// fixed-line split (NSLOTS must divide the block size, nlines <= NSLOTS is
// passed at run time); 0 splits (butterfly, line) items.
template <bool DIT, typename R, int MAXR = 16, bool FIXED = false>
__device__ void fft_batch(cpx<R>* buf, int ld, int nlines, const FFTPlan& P, int sign, const cpx<R>* tw,
                          int nslots = 0) {
    __syncthreads();
    const StageSplit sp = stage_split(FIXED ? nslots : 1);
    for (int s0 = 0; s0 < P.nst; ++s0) {
        const int st = DIT ? s0 : P.nst - 1 - s0;
        const int Lp = P.lp[st];
        switch (P.r[st]) {
            case 2: fft_stage<2, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp); break;
            case 3: fft_stage<3, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp); break;
            case 4: fft_stage<4, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp); break;
            case 5: fft_stage<5, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp); break;
            case 8: fft_stage<8, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp); break;
            case 16:
                if constexpr (MAXR >= 16) fft_stage<16, DIT, FIXED, R>(buf, ld, nlines, P, Lp, sign, tw, sp);
                break;
            default: break;
        }
        __syncthreads();
    }
}

// largest radix of a plan (host side): selects the MAXR instantiation
inline int plan_max_radix(const FFTPlan& P) {
    int m = 1;
    for (int s = 0; s < P.nst; ++s) m = P.r[s] > m ? P.r[s] : m;
    return m;
}

}  // namespace ps3d
