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

template <typename R>
__device__ __forceinline__ cpx<R> twiddle(const FFTPlan& P, int t, int sign);
template <>
__device__ __forceinline__ double2 twiddle<double>(const FFTPlan& P, int t, int sign) {
    double2 w = __ldg(P.tw + t);
    if (sign > 0) w.y = -w.y;
    return w;
}
template <>
__device__ __forceinline__ float2 twiddle<float>(const FFTPlan& P, int t, int sign) {
    float2 w = __ldg(P.twf + t);
    if (sign > 0) w.y = -w.y;
    return w;
}

// radix-RAD DFT in registers: y_m = sum_q v_q exp(sign 2 pi i q m / RAD)
template <int RAD, typename T>
__device__ __forceinline__ void small_dft(T* v, int sign) {
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

template <int RAD, bool DIT, typename R>
__device__ __forceinline__ void fft_stage(cpx<R>* buf, int ld, int nlines, const FFTPlan& P,
                                          int Lp, int sign) {
    using T = cpx<R>;
    const int n = P.n;
    const int L = Lp * RAD;
    const int tstride = n / L;
    const int nb = n / RAD;
    const int total = nb * nlines;
    for (int item = threadIdx.x; item < total; item += blockDim.x) {
        const int bfly = item / nlines;
        const int line = item - bfly * nlines;
        const int blk = bfly / Lp;
        const int j = bfly - blk * Lp;
        const int base = blk * L + j;
        T v[RAD];
#pragma unroll
        for (int q = 0; q < RAD; ++q) v[q] = buf[(base + q * Lp) * ld + line];
        if (DIT && j) {
#pragma unroll
            for (int q = 1; q < RAD; ++q) v[q] = cmul(v[q], twiddle<R>(P, q * j * tstride, sign));
        }
        small_dft<RAD>(v, sign);
        if (!DIT && j) {
#pragma unroll
            for (int q = 1; q < RAD; ++q) v[q] = cmul(v[q], twiddle<R>(P, q * j * tstride, sign));
        }
#pragma unroll
        for (int q = 0; q < RAD; ++q) buf[(base + q * Lp) * ld + line] = v[q];
    }
}

// Whole-block batched FFT.  Must be called by every thread of the block; it
// synchronises the block before returning.
template <bool DIT, typename R>
__device__ void fft_batch(cpx<R>* buf, int ld, int nlines, const FFTPlan& P, int sign) {
    __syncthreads();
    int Lps[kMaxStages];
    int acc = 1;
    for (int s = 0; s < P.nst; ++s) { Lps[s] = acc; acc *= P.r[s]; }
    for (int s0 = 0; s0 < P.nst; ++s0) {
        const int st = DIT ? s0 : P.nst - 1 - s0;
        const int Lp = Lps[st];
        switch (P.r[st]) {
            case 2: fft_stage<2, DIT, R>(buf, ld, nlines, P, Lp, sign); break;
            case 3: fft_stage<3, DIT, R>(buf, ld, nlines, P, Lp, sign); break;
            case 4: fft_stage<4, DIT, R>(buf, ld, nlines, P, Lp, sign); break;
            case 5: fft_stage<5, DIT, R>(buf, ld, nlines, P, Lp, sign); break;
            default: break;
        }
        __syncthreads();
    }
}

}  // namespace ps3d
