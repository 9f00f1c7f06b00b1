// common.cuh — shared device definitions of the ps3D B200 engine.
//
// Device layout (differs from the host's halo layout on purpose): every real
// field is stored interior-only, x fastest, nx*ny*nz elements, and stencils
// wrap their indices periodically.  On one rank the reference's halo
// exchange (for_src/parallel_mpi.f90:70-211) makes every halo point an exact
// periodic copy of an interior point, so the halo carries no extra state;
// the one place where halos differ from the wrapped interior (friction
// stages reading pre-friction halos, for_src/integrate.f90:59-78) is
// reproduced explicitly by the friction kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#define PS3D_HD __host__ __device__ __forceinline__

namespace ps3d {

// ---------------------------------------------------------------------------
// complex helpers (interleaved re/im, double2/float2 compatible with the
// reference's complex(8) storage)
// ---------------------------------------------------------------------------
template <typename R> struct cpx_t;
template <> struct cpx_t<double> { using type = double2; };
template <> struct cpx_t<float> { using type = float2; };
template <typename R> using cpx = typename cpx_t<R>::type;

template <typename R> PS3D_HD cpx<R> mk(R a, R b) { cpx<R> c; c.x = a; c.y = b; return c; }
template <typename T> PS3D_HD T cadd(T a, T b) { a.x += b.x; a.y += b.y; return a; }
template <typename T> PS3D_HD T csub(T a, T b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename T> PS3D_HD T cmul(T a, T b) {
    T c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
template <typename T> PS3D_HD T cconj(T a) { a.y = -a.y; return a; }
template <typename T, typename S> PS3D_HD T cscale(T a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by s*i  (s = +-1)
template <typename T> PS3D_HD T cmul_si(T a, int s) {
    T c; c.x = -s * a.y; c.y = s * a.x; return c;
}

// ---------------------------------------------------------------------------
// FFT plan for one transform length, device side
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 16;

struct FFTPlan {
    int n;                    // transform length
    int nst;                  // number of stages
    int r[kMaxStages];        // radices in DIT stage order (product = n)
    int lp[kMaxStages];       // product of the radices before each stage
    const double2* tw;        // exp(-2 pi i t / n), t = 0..n-1
    const float2* twf;        // the same, rounded to FP32
    const int* pos;           // digit-reversal: natural index t -> position
    const int* ipos;          // inverse of pos
};

// ---------------------------------------------------------------------------
// Division by a run-time invariant divisor 1 <= d < 2^31, for numerators
// 0 <= n < 2^31, by one multiply-high, one add and one shift: the round-up
// method of Granlund & Montgomery, "Division by invariant integers using
// multiplication" (PLDI 1994).  With l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, n / d = (mulhi(m, n) + n) >> l.
// ---------------------------------------------------------------------------
struct FastDiv {
    unsigned d, m;
    int l;
};
inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d ? d : 1;
    f.l = 0;
    while ((1ull << f.l) < f.d) ++f.l;
    f.m = (unsigned)((((1ull << 32) * ((1ull << f.l) - f.d)) / f.d) + 1);
    return f;
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) { return (__umulhi(n, f.m) + n) >> f.l; }

// ---------------------------------------------------------------------------
// periodic index helpers
// ---------------------------------------------------------------------------
PS3D_HD int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// ---------------------------------------------------------------------------
// Programmatic dependent launch (sm_90+): a kernel launched with
// launch_pdl lets the next kernel of the stream be scheduled once all of its
// own blocks are resident (pdl_trigger at block start), so the successor's
// launch and prologue overlap this kernel's tail; every such kernel calls
// pdl_wait before it reads anything an earlier kernel wrote (it returns when
// the preceding grids have completed and their memory is visible).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------------------
// L2 eviction priorities (createpolicy + .L2::cache_hint).  A pressure solve
// writes its spectral array in the forward rows pass and every later pass
// reads it (y lines, vertical solve, y lines, inverse rows), while the real
// fields stream through L2 at several times its bytes: the spectra are
// accessed with evict_last and the streamed fields with evict_first, so the
// spectra stay resident in the 126 MB L2 between the kernels of a solve
// instead of being pushed out by the fields.  kL2Normal gives the default
// priority (the hints off).
// ---------------------------------------------------------------------------
enum : int { kL2Normal = 0, kL2Keep = 1, kL2Stream = 2 };
__device__ __forceinline__ unsigned long long l2_policy(int kind) {
    unsigned long long p;
    if (kind == kL2Keep)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else if (kind == kL2Stream)
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    else
        asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// coherent loads and stores with a policy (data the kernel may also write)
__device__ __forceinline__ float2 ld_l2(const float2* a, unsigned long long pol) {
    float2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ double2 ld_l2(const double2* a, unsigned long long pol) {
    double2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ void st_l2(float2* a, float2 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_l2(double2* a, double2 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ float ld_l2(const float* a, unsigned long long pol) {
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ double ld_l2(const double* a, unsigned long long pol) {
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ void st_l2(float* a, float v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_l2(double* a, double v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
// read-only (non-coherent) loads with a policy: fields the kernel does not write
__device__ __forceinline__ double ldg_l2(const double* a, unsigned long long pol) {
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ldg_l2(const double2* a, unsigned long long pol) {
    double2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
    return v;
}

// status flags written by kernels (bit mask, OR-ed)
enum : unsigned {
    kFlagNonFinite = 1u,
    kFlagBounds = 2u,
};

}  // namespace ps3d
