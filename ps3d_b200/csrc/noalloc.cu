// noalloc.cu — a pressure projection that allocates no device memory.
//
// Some hosts cannot call cudaMalloc at the point where they want the
// projection: a Fortran or C code that hands over device arrays it owns
// (CUDA Fortran, OpenACC or a memory pool managed by the host program), a
// caller inside a region where allocation is forbidden or would deadlock
// (e.g. while its own allocator holds a lock), or a code that must keep its
// device footprint fixed after start-up.  ps3d_pressure_solve_noalloc serves
// them: the caller passes its own device arrays u, v, w (updated in place)
// and p (written), and the engine works in two file-scope static __device__
// arrays instead of allocating:
//   g_spectral  the spectral work array, kMaxSpectral complex doubles
//               (16 MiB): grids with (nx/2+1)*ny*nz <= 1048576 points;
//   g_tables    FFT twiddles, digit-reversal permutations and wavenumber
//               symbols for transform lengths up to kMaxLen.
// Every GPU that loads the library holds both arrays (about 16.1 MiB) until
// the process exits.  Nothing in them has to start at zero: each call
// rewrites the tables and every spectral element it later reads.  All calls
// share the arrays, so calls that overlap on the GPU race: calls from host
// threads of one process are serialised here (one lock around the call),
// calls from other processes must be serialised by the caller.  The call is
// synchronous (it waits for its stream) and cannot be captured in a CUDA
// graph; it allocates no device memory, and its host staging image is a
// static per-device buffer.
#include <cmath>
#include <cstring>
#include <mutex>
#include "ctx.h"

namespace ps3d {

constexpr long kMaxSpectral = 1L << 20;     // complex doubles in the spectral scratch
constexpr int kMaxLen = 1024;               // longest FFT / axis the tables cover

// table layout inside g_tables (in doubles)
constexpr long kTwX = 0;                          // tw (length nx/2), double2
constexpr long kTwY = kTwX + 2L * kMaxLen;        // tw (length ny), double2
constexpr long kTwZ = kTwY + 2L * kMaxLen;        // tw (length nz), double2
constexpr long kTwR = kTwZ + 2L * kMaxLen;        // exp(-2 pi i t/nx), t = 0..nx/2, double2
constexpr long kHkx = kTwR + 2L * (kMaxLen + 1);  // hat_ksqr(kx)
constexpr long kHky = kHkx + kMaxLen + 1;         // hat_ksqr(ky)
constexpr long kHkz = kHky + kMaxLen;             // hat_ksqr(kz)/dsqr
constexpr long kPos = kHkz + kMaxLen;             // int tables start here (6 x kMaxLen ints)
constexpr long kTableDoubles = kPos + 3L * kMaxLen;

static __device__ __align__(256) double2 g_spectral[kMaxSpectral];
static __device__ __align__(256) double g_tables[kTableDoubles];

// device addresses of the static arrays, looked up once per device, and the
// host image of the tables (static, so a call allocates no host memory either)
struct StaticArrays {
    double2* spectral = nullptr;
    double* tables = nullptr;
    bool ready = false;
    double img[kTableDoubles];
};
static std::mutex g_mu;   // held for a whole call
static StaticArrays g_dev[16];

// with g_mu held
static int static_arrays(int dev, StaticArrays*& out) {
    if (dev < 0 || dev >= 16) return PS3D_ERR_BADPARAM;
    StaticArrays& s = g_dev[dev];
    if (!s.ready) {
        void* a = nullptr;
        void* b = nullptr;
        if (cudaGetSymbolAddress(&a, g_spectral) != cudaSuccess) return PS3D_ERR_CUDA;
        if (cudaGetSymbolAddress(&b, g_tables) != cudaSuccess) return PS3D_ERR_CUDA;
        s.spectral = (double2*)a;
        s.tables = (double*)b;
        if (plane_setup(false) != cudaSuccess) return PS3D_ERR_CUDA;
        s.ready = true;
    }
    out = &s;
    return PS3D_OK;
}

// host construction of one FFT plan's tables into the staging image
static bool plan_into(int n, double* img, long tw_off, long pos_off, long ipos_off, FFTPlan& P,
                      const double* dev_tables) {
    int r[64];
    int nr = 0;
    int m = n;
    while (m % 16 == 0) { r[nr++] = 16; m /= 16; }
    if (m % 8 == 0) { r[nr++] = 8; m /= 8; }
    while (m % 4 == 0) { r[nr++] = 4; m /= 4; }
    while (m % 2 == 0) { r[nr++] = 2; m /= 2; }
    while (m % 3 == 0) { r[nr++] = 3; m /= 3; }
    while (m % 5 == 0) { r[nr++] = 5; m /= 5; }
    if (m != 1 || n > kMaxLen || nr > kMaxStages) return false;
    int* ip = reinterpret_cast<int*>(img + kPos);
    for (int t = 0; t < n; ++t) {
        long tt = t;
        double c, s;
        if ((8 * tt) % n == 0) {
            static const double r2 = 0.70710678118654752440084436210484904;
            const double cc[8] = {1, r2, 0, -r2, -1, -r2, 0, r2};
            const double ss[8] = {0, r2, 1, r2, 0, -r2, -1, -r2};
            c = cc[(8 * tt) / n]; s = ss[(8 * tt) / n];
        } else {
            const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)tt / (long double)n;
            c = (double)cosl(a); s = (double)sinl(a);
        }
        img[tw_off + 2 * t] = c;
        img[tw_off + 2 * t + 1] = -s;
    }
    int* pos = ip + ipos_off;   // scratch: overwritten by the inverse table below
    int* ipos = ip + ipos_off;
    for (int t = 0; t < n; ++t) {
        int v = t, len = n, p = 0;
        for (int st = nr - 1; st >= 0; --st) {
            const int R = r[st];
            p += (v % R) * (len / R);
            v /= R;
            len /= R;
        }
        pos[t] = p;
    }
    for (int t = 0; t < n; ++t) ip[pos_off + t] = pos[t];
    for (int t = 0; t < n; ++t) ipos[ip[pos_off + t]] = t;
    P.n = n;
    P.nst = nr;
    int acc = 1;
    for (int st = 0; st < kMaxStages; ++st) {
        P.r[st] = st < nr ? r[st] : 1;
        P.lp[st] = acc;
        acc *= P.r[st];
    }
    P.tw = reinterpret_cast<const double2*>(dev_tables + tw_off);
    P.twf = nullptr;
    const int* dev_int = reinterpret_cast<const int*>(dev_tables + kPos);
    P.pos = dev_int + pos_off;
    P.ipos = dev_int + ipos_off;
    return true;
}

}  // namespace ps3d

extern "C" {

// pressure_solver (for_src/pressure_solver.f90:2-120) on caller-owned device
// arrays, FP64, allocating nothing.  u, v, w, p: nx*ny*nz doubles each, x
// fastest, interior points only.  The first call on a device looks up the
// static arrays' device addresses (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture.  Synchronous.
PS3D_API int ps3d_pressure_solve_noalloc(const ps3d_params* prm, double* u, double* v, double* w, double* p,
                                         void* stream) {
    using namespace ps3d;
    if (!prm) return PS3D_ERR_BADPARAM;
    const ps3d_params& P = *prm;
    const bool rigid = P.enable_vertical_boundaries != 0;
    const int nx = P.nx, ny = P.ny, nz = P.nz, nxh = nx / 2 + 1;
    if (nx < 2 || ny < 2 || nz < 2 || nx % 2 || ny % 2 || (!rigid && nz % 2)) return PS3D_ERR_BADPARAM;
    // the static arrays and the column kernels' shared memory bound the grid;
    // checked before the field pointers so that a caller can probe a size
    // with null pointers
    if ((long)nxh * ny * nz > kMaxSpectral || nx / 2 > kMaxLen || ny > kMaxLen || nz > kMaxLen)
        return PS3D_ERR_TOOLARGE;
    if (rigid ? thomas_threads(nz) == 0 : !zsolve_fits(nz, false)) return PS3D_ERR_TOOLARGE;
    if (!u || !v || !w || !p) return PS3D_ERR_BADPARAM;
    if (!(P.dx > 0 && P.dy > 0 && P.dz > 0 && P.Lx > 0 && P.Ly > 0 && P.Lz > 0 && P.dsqr > 0 && P.dt != 0))
        return PS3D_ERR_BADPARAM;
    // a failing CUDA call: its error is taken off the thread's error state so
    // that it is not reported again by a later call
    auto fail = [](cudaError_t e) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? PS3D_ERR_OOM : PS3D_ERR_CUDA;
    };
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(e);
    std::lock_guard<std::mutex> lk(g_mu);
    StaticArrays* sa = nullptr;
    int rc = static_arrays(dev, sa);
    if (rc) { cudaGetLastError(); return rc; }
    cudaStream_t s = (cudaStream_t)stream;
    // tables: built on the host into the static image, copied into g_tables
    double* img = sa->img;
    std::memset(img, 0, sizeof(sa->img));
    FFTPlan px{}, py{}, pz{};
    if (!plan_into(nx / 2, img, kTwX, 0, kMaxLen, px, sa->tables)) return PS3D_ERR_BADPARAM;
    if (!plan_into(ny, img, kTwY, 2 * kMaxLen, 3 * kMaxLen, py, sa->tables)) return PS3D_ERR_BADPARAM;
    if (!rigid && !plan_into(nz, img, kTwZ, 4 * kMaxLen, 5 * kMaxLen, pz, sa->tables)) return PS3D_ERR_BADPARAM;
    const double pi = std::acos(0.0) * 2.0;
    for (int t = 0; t < nxh; ++t) {
        long tt = t;
        double c, sn;
        if ((8 * tt) % nx == 0) {
            static const double r2 = 0.70710678118654752440084436210484904;
            const double cc[8] = {1, r2, 0, -r2, -1, -r2, 0, r2};
            const double ss[8] = {0, r2, 1, r2, 0, -r2, -1, -r2};
            c = cc[(8 * tt) / nx]; sn = ss[(8 * tt) / nx];
        } else {
            const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)tt / (long double)nx;
            c = (double)cosl(a); sn = (double)sinl(a);
        }
        img[kTwR + 2 * t] = c;
        img[kTwR + 2 * t + 1] = -sn;
    }
    auto hat = [](double k, double d) { return 2.0 * (1.0 - std::cos(k * d)) / (d * d); };
    for (int i = 1; i <= nxh; ++i) img[kHkx + i - 1] = hat(2 * (i - 1) * pi / P.Lx, P.dx);
    for (int j = 1; j <= ny; ++j) {
        const double ky = j <= (ny + 1) / 2 ? 2 * (j - 1) * pi / P.Ly : -(2 * (ny - j + 1) * pi / P.Ly);
        img[kHky + j - 1] = hat(ky, P.dy);
    }
    if (!rigid)
        for (int k = 1; k <= nz; ++k) {
            const double kz = k <= (nz + 1) / 2 ? 2 * (k - 1) * pi / P.Lz : -(2 * (nz - k + 1) * pi / P.Lz);
            img[kHkz + k - 1] = hat(kz, P.dz) / P.dsqr;
        }
    // plane-kernel shape: the engine's default one-cluster-per-plane shape
    PlaneArgs a{};
    a.nx = nx; a.ny = ny; a.nz = nz; a.nxh = nxh;
    a.px = px; a.py = py;
    a.twx = reinterpret_cast<const double2*>(sa->tables + kTwR);
    a.rdx = 1.0 / P.dx; a.rdy = 1.0 / P.dy; a.rdz = 1.0 / P.dz;
    a.batch = 1; a.sN = (long)nx * ny * nz; a.sM = (long)nxh * ny * nz;
    if (!choose_plane_config(nx, ny, sizeof(double2), a)) return PS3D_ERR_TOOLARGE;
    a.impl = 0;
    if ((e = cudaMemcpyAsync(sa->tables, img, sizeof(sa->img), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail(e);
    PlaneArgs f = a;
    f.mode = 0; f.u = u; f.v = v; f.w = w;
    f.rdt = 1.0 / P.dt;
    f.scale = P.dx * P.dy;
    f.spec = sa->spectral;
    if ((e = launch_plane_fwd(f, false, s)) != cudaSuccess) return fail(e);
    ColumnArgs c{};
    c.nx = nx; c.ny = ny; c.nz = nz; c.nxh = nxh; c.spec = sa->spectral;
    c.batch = 1; c.sM = a.sM;
    c.hkx = sa->tables + kHkx; c.hky = sa->tables + kHky; c.hkz = sa->tables + kHkz;
    c.layout = spectral_layout(a);
    if (rigid) {
        c.fxa = 1.0 / (P.dz * P.dz) / P.dsqr;
        c.dz2dsqr = P.dz * P.dz * P.dsqr;
        if ((e = launch_thomas(c, false, s)) != cudaSuccess) return fail(e);
    } else {
        c.pz = pz; c.scale = P.dz; c.op = 0;
        if ((e = launch_zsolve(c, false, s)) != cudaSuccess) return fail(e);
    }
    PlaneArgs b = a;
    b.spec = sa->spectral;
    b.out = p;
    b.beta = 0.0;
    b.scale = rigid ? 1.0 / (P.Lx * P.Ly) : 1.0 / (P.Lx * P.Ly * P.Lz);
    if ((e = launch_plane_inv(b, false, s)) != cudaSuccess) return fail(e);
    if ((e = launch_correct(u, v, w, p, nx, ny, nz, rigid, P.dt, P.dt / P.dsqr, 1.0 / P.dx, 1.0 / P.dy, 1.0 / P.dz,
                            s)) != cudaSuccess)
        return fail(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e);
    return PS3D_OK;
}

}  // extern "C"
