// slab.cu — one grid cut into z-slabs over several contexts (GPUs).
//
// The reference decomposes its grid over MPI ranks inside P3DFFT; here a
// rank owns the levels k0 .. k0+nzl-1 of the global grid (nz = nranks * nzl)
// and the step runs in phases between which the ranks exchange data:
//
//   tendency    K1 (k_step) on the interior levels, the previous step's
//               pressure correction applied while loading
//   state halo  the new u, v, w, b: the interior bottom plane goes to the
//               rank below, the top plane to the rank above (z periodic, as
//               border_exchg_3D, parallel_mpi.f90:70-211; the rigid-lid masks
//               see global levels)
//   forward     divergence + per-level 2D transforms of the interior planes
//               into a compact spectral array [nzl][kx][ky], then packed by
//               destination rank: columns cbeg[r] .. cbeg[r]+ccnt[r]-1
//   transpose   all-to-all: each rank receives every rank's levels of its own
//               columns, i.e. whole columns [nz][ccnt] (pressure_solver.f90
//               needs the full column for the tridiagonal solve)
//   vsolve      the vertical solves of those columns: the Thomas solves
//               (rigid lid) or the z transform, division and inverse z
//               transform (triply periodic, pressure_solver.f90:58-70) on a
//               column slab
//   transpose   all-to-all back, unpacked into [nzl][kx][ky]
//   inverse     per-level inverse 2D transforms into p (pending correction)
//   p halo      p one level below and two above (the step kernel's lazy
//               correction reads p at the plane it loads and the one above)
//
// The mixed path (FP32 transforms) solves for the divergence of
// u - dt grad p in FP64 and adds that pressure to p (pressure_solve in
// engine.cu): once per step from the previous step's p (warm), and on a cold
// start (after create or upload) after a first full solve, so forward ..
// p halo run twice on that step.
//
// Local arrays hold nzl + 3 levels: halo 0, interior 1 .. nzl, halos nzl+1
// and nzl+2 (the second only for p).  The transport between ranks is the
// caller's: NCCL all-to-all and send/receive between processes (the Python
// driver, ps3d_b200/slab.py), or ps3d_slab_group_step for contexts in one
// process, which copies device to device.  Supported: rigid lid or triply
// periodic, FP64 and mixed, the fused step (Laplacian friction, the
// wavemaker and background-flow forcing of set_forcing on the rank's levels
// and one halo level each side; no biharmonic friction, no host callback).
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>
#include "ctx.h"

using ps3d::Ctx;
using ps3d::DevBuf;

struct ps3d_slab {
    std::unique_ptr<Ctx> ctx;
    int nranks = 1, rank = 0, nzg = 0, nzl = 0, k0 = 0;
    long ncols = 0, plane = 0;
    std::vector<long> cbeg, ccnt;   // column split over ranks
    DevBuf own_x, own_col, own_hs, own_hr;
    void* xbuf = nullptr;           // [r][nzl][ccnt[r]] complex: forward send / backward receive
    void* colbuf = nullptr;         // [nz][ccnt[rank]] complex: forward receive / backward send
    void* hsend = nullptr;          // halo planes to send: [down][up]
    void* hrecv = nullptr;          // halo planes received: [from below][from above]
    bool need_halo = true;          // state halos not yet exchanged (after an upload)
    bool mixed = false;             // FP32 spectra, residual solves
    bool rigid = true;
    double Lz = 0.0;                // the global grid's depth
    ps3d::DevPlan plz;              // triply periodic: the global z transform
    DevBuf hkz;                     // ... and hat_ksqr(kz)/dsqr of the global levels
    int pass = 0;                   // solve pass: 0 full solve, 1 residual solve (mixed path)
    cudaEvent_t ev = nullptr;       // ps3d_slab_group_step: marks this rank's stream for the others
    ~ps3d_slab() {
        if (ev) cudaEventDestroy(ev);
    }

    // solve passes of the next step: 1 in FP64; in the mixed path 2 on a cold
    // start (full solve, then the residual one), else 1 (the residual solve
    // against the previous step's p)
    int passes() const { return mixed && !ctx->warm_solve() ? 2 : 1; }
    size_t es() const { return mixed ? sizeof(float2) : sizeof(double2); }
    size_t xbytes() const { return (size_t)nzl * ncols * es(); }
    size_t colbytes() const { return (size_t)nzg * ccnt[rank] * es(); }
    size_t hbytes() const { return (size_t)8 * plane * sizeof(double); }
    double* lvl(double* f, int L) const { return f + (size_t)L * plane; }
};

namespace {

// planes sent down (to the rank below) and up: state u, v, w, b; p two down, one up
constexpr int kDown[2] = {4, 2}, kUp[2] = {4, 1};

int slab_tendency(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    s->pass = c.warm_solve() ? 1 : 0;
    return c.step(c.itt, c.tau, c.taum1, c.taum2);
}

int halo_pack(ps3d_slab* s, int which) {
    Ctx& c = *s->ctx;
    const size_t pb = (size_t)s->plane * sizeof(double);
    char* out = (char*)s->hsend;
    auto cp = [&](void* dst, const void* src) { return cudaMemcpyAsync(dst, src, pb, cudaMemcpyDeviceToDevice, c.stream); };
    if (which == 0) {
        for (int f = 0; f < 4; ++f) CK(cp(out + f * pb, s->lvl(c.field(f), 1)));
        for (int f = 0; f < 4; ++f) CK(cp(out + (4 + f) * pb, s->lvl(c.field(f), s->nzl)));
    } else {
        double* p = (double*)c.p.p;
        CK(cp(out, s->lvl(p, 1)));
        CK(cp(out + pb, s->lvl(p, 2)));
        CK(cp(out + 2 * pb, s->lvl(p, s->nzl)));
    }
    return PS3D_OK;
}

int halo_unpack(ps3d_slab* s, int which) {
    Ctx& c = *s->ctx;
    const size_t pb = (size_t)s->plane * sizeof(double);
    const char* in = (const char*)s->hrecv;
    auto cp = [&](void* dst, const void* src) { return cudaMemcpyAsync(dst, src, pb, cudaMemcpyDeviceToDevice, c.stream); };
    const int nzl = s->nzl;
    if (which == 0) {
        // from below: its top interior plane; from above: its bottom one
        for (int f = 0; f < 4; ++f) CK(cp(s->lvl(c.field(f), 0), in + f * pb));
        for (int f = 0; f < 4; ++f) CK(cp(s->lvl(c.field(f), nzl + 1), in + (4 + f) * pb));
        s->need_halo = false;
    } else {
        double* p = (double*)c.p.p;
        CK(cp(s->lvl(p, 0), in));
        CK(cp(s->lvl(p, nzl + 1), in + pb));
        CK(cp(s->lvl(p, nzl + 2), in + 2 * pb));
    }
    return PS3D_OK;
}

ps3d::PlaneArgs window(ps3d_slab* s, const ps3d::PlaneArgs& base) {
    ps3d::PlaneArgs a = base;
    a.batch = 1;
    a.kbeg = 1; a.kcount = s->nzl; a.kofs = s->k0 - 1; a.nzg = s->nzg;
    a.sM = (long)s->nzl * s->ncols;
    return a;
}

int slab_forward(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    ps3d::PlaneArgs a = window(s, s->mixed ? c.pa32 : c.pa64);
    // pass 1 (mixed): the divergence of u - dt grad p, p from pass 0 or from the
    // previous step, with its halos
    a.mode = s->pass ? 2 : 0;
    a.u = c.field(0); a.v = c.field(1); a.w = c.field(2);
    a.pc = s->pass ? (const double*)c.p.p : nullptr;
    a.dtp = c.P.dt; a.dtwp = c.P.dt / c.P.dsqr;
    a.rigid = s->rigid;
    a.rdt = 1.0 / c.P.dt;
    a.scale = c.P.dx * c.P.dy;
    a.spec = c.FS.p;
    CK(ps3d::launch_plane_fwd(a, s->mixed, c.stream));
    const size_t es = s->es();
    for (int r = 0; r < s->nranks; ++r)
        CK(cudaMemcpy2DAsync((char*)s->xbuf + (size_t)s->nzl * s->cbeg[r] * es, s->ccnt[r] * es,
                             (const char*)c.FS.p + s->cbeg[r] * es, s->ncols * es, s->ccnt[r] * es, s->nzl,
                             cudaMemcpyDeviceToDevice, c.stream));
    return PS3D_OK;
}

int slab_vsolve(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    ps3d::ColumnArgs a{};
    a.nx = c.nx; a.ny = c.ny; a.nz = s->nzg; a.nxh = c.nxh;
    a.spec = s->colbuf;
    a.batch = 1; a.sM = (long)s->nzg * s->ccnt[s->rank];
    a.layout = ps3d::spectral_layout(s->mixed ? c.pa32 : c.pa64);
    a.hkx = (const double*)c.t_hkx.p; a.hky = (const double*)c.t_hky.p;
    a.col0 = s->cbeg[s->rank]; a.ncl = s->ccnt[s->rank];
    a.err = c.kerr_d;
    if (!s->rigid) {
        a.hkz = (const double*)s->hkz.p;
        a.pz = s->plz.plan; a.scale = c.P.dz; a.op = 0;
        CK(ps3d::launch_zsolve(a, s->mixed, c.stream));
        return PS3D_OK;
    }
    a.fxa = 1.0 / (c.P.dz * c.P.dz) / c.P.dsqr;
    a.dz2dsqr = c.P.dz * c.P.dz * c.P.dsqr;
    CK(ps3d::launch_thomas(a, s->mixed, c.stream));
    return PS3D_OK;
}

int slab_inverse(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    const size_t es = s->es();
    for (int r = 0; r < s->nranks; ++r)
        CK(cudaMemcpy2DAsync((char*)c.FS.p + s->cbeg[r] * es, s->ncols * es,
                             (const char*)s->xbuf + (size_t)s->nzl * s->cbeg[r] * es, s->ccnt[r] * es,
                             s->ccnt[r] * es, s->nzl, cudaMemcpyDeviceToDevice, c.stream));
    ps3d::PlaneArgs b = window(s, s->mixed ? c.pa32 : c.pa64);
    b.spec = c.FS.p;
    b.out = (double*)c.p.p;
    b.beta = s->pass ? 1.0 : 0.0;   // the residual pass adds its pressure
    b.scale = s->rigid ? 1.0 / (c.P.Lx * c.P.Ly) : 1.0 / (c.P.Lx * c.P.Ly * s->Lz);
    CK(ps3d::launch_plane_inv(b, s->mixed, c.stream));
    if (++s->pass >= (s->mixed ? 2 : 1)) {
        c.pending = true;
        c.pcor = (const double*)c.p.p;
        c.dtp = c.P.dt;
        c.p_warm = true;
    }
    return PS3D_OK;
}

int slab_end_step(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    c.rotate();
    c.time = c.time + c.P.dt;
    ++c.itt;
    return PS3D_OK;
}

// host waits for every rank's stream (the end of ps3d_slab_group_step)
int sync_all(ps3d_slab* const* r, int n) {
    for (int q = 0; q < n; ++q) {
        cudaSetDevice(r[q]->ctx->device);
        int rc = r[q]->ctx->sync();
        if (rc) return rc;
    }
    return PS3D_OK;
}

// The group driver orders the ranks' streams with events, without host
// synchronisation: mark(q) records rank q's event on its stream, after(q, p)
// makes rank q's stream wait for rank p's last mark.  Every wait on a mark is
// issued (host order) before that event is recorded again.
cudaError_t mark(const ps3d_slab* s) { return cudaEventRecord(s->ev, s->ctx->stream); }
cudaError_t after(const ps3d_slab* s, const ps3d_slab* p) { return cudaStreamWaitEvent(s->ctx->stream, p->ev, 0); }

int transport_halo(ps3d_slab* const* r, int n, int which) {
    const size_t pb = (size_t)r[0]->plane * sizeof(double);
    const int nd = kDown[which], nu = kUp[which];
    for (int q = 0; q < n; ++q) { cudaSetDevice(r[q]->ctx->device); CK(mark(r[q])); }   // packed
    for (int q = 0; q < n; ++q) {
        const ps3d_slab* below = r[(q + n - 1) % n];
        const ps3d_slab* above = r[(q + 1) % n];
        char* in = (char*)r[q]->hrecv;
        cudaSetDevice(r[q]->ctx->device);
        CK(after(r[q], below));
        CK(after(r[q], above));
        // from below: what it sent up; from above: what it sent down
        CK(cudaMemcpyAsync(in, (const char*)below->hsend + nd * pb, nu * pb, cudaMemcpyDefault, r[q]->ctx->stream));
        CK(cudaMemcpyAsync(in + nu * pb, above->hsend, nd * pb, cudaMemcpyDefault, r[q]->ctx->stream));
    }
    // a rank's send planes are read by its neighbours' copies: it packs
    // again only after those
    for (int q = 0; q < n; ++q) { cudaSetDevice(r[q]->ctx->device); CK(mark(r[q])); }
    for (int q = 0; q < n; ++q) {
        cudaSetDevice(r[q]->ctx->device);
        CK(after(r[q], r[(q + n - 1) % n]));
        CK(after(r[q], r[(q + 1) % n]));
    }
    return PS3D_OK;
}

int transport_columns(ps3d_slab* const* r, int n, bool forward) {
    const size_t es = r[0]->es();
    if (forward)
        for (int q = 0; q < n; ++q) { cudaSetDevice(r[q]->ctx->device); CK(mark(r[q])); }   // packed
    for (int d = 0; d < n; ++d) {
        cudaSetDevice(r[d]->ctx->device);
        if (forward)
            for (int q = 0; q < n; ++q)
                if (q != d) CK(after(r[d], r[q]));
        for (int q = 0; q < n; ++q) {
            // the block of rank q's levels and rank d's columns, moved on rank d's stream
            const size_t bytes = (size_t)r[q]->nzl * r[d]->ccnt[d] * es;
            if (forward)
                CK(cudaMemcpyAsync((char*)r[d]->colbuf + (size_t)q * r[q]->nzl * r[d]->ccnt[d] * es,
                                   (const char*)r[q]->xbuf + (size_t)r[q]->nzl * r[q]->cbeg[d] * es, bytes,
                                   cudaMemcpyDefault, r[d]->ctx->stream));
            else
                CK(cudaMemcpyAsync((char*)r[q]->xbuf + (size_t)r[q]->nzl * r[q]->cbeg[d] * es,
                                   (const char*)r[d]->colbuf + (size_t)q * r[q]->nzl * r[d]->ccnt[d] * es, bytes,
                                   cudaMemcpyDefault, r[d]->ctx->stream));
        }
    }
    if (!forward) {
        // every rank unpacks only after every rank's blocks have landed in its xbuf
        for (int d = 0; d < n; ++d) { cudaSetDevice(r[d]->ctx->device); CK(mark(r[d])); }
        for (int q = 0; q < n; ++q) {
            cudaSetDevice(r[q]->ctx->device);
            for (int d = 0; d < n; ++d)
                if (d != q) CK(after(r[q], r[d]));
        }
    }
    return PS3D_OK;
}

int group_halo(ps3d_slab* const* r, int n, int which) {
    for (int q = 0; q < n; ++q) {
        cudaSetDevice(r[q]->ctx->device);
        int rc = halo_pack(r[q], which);
        if (rc) return rc;
    }
    int rc = transport_halo(r, n, which);
    if (rc) return rc;
    for (int q = 0; q < n; ++q) {
        cudaSetDevice(r[q]->ctx->device);
        rc = halo_unpack(r[q], which);
        if (rc) return rc;
    }
    return PS3D_OK;
}

#define FOR_RANKS(call)                                 \
    for (int q = 0; q < n; ++q) {                       \
        cudaSetDevice(r[q]->ctx->device);               \
        int rc_ = call;                                 \
        if (rc_) return rc_;                            \
    }

int group_step(ps3d_slab* const* r, int n) {
    int rc;
    if (r[0]->need_halo && (rc = group_halo(r, n, 0))) return rc;
    FOR_RANKS(slab_tendency(r[q]))
    if ((rc = group_halo(r, n, 0))) return rc;
    const int np = r[0]->passes();
    for (int pass = 0; pass < np; ++pass) {
        FOR_RANKS(slab_forward(r[q]))
        if ((rc = transport_columns(r, n, true))) return rc;
        FOR_RANKS(slab_vsolve(r[q]))
        if ((rc = transport_columns(r, n, false))) return rc;
        FOR_RANKS(slab_inverse(r[q]))
        if ((rc = group_halo(r, n, 1))) return rc;
    }
    FOR_RANKS(slab_end_step(r[q]))
    return PS3D_OK;
}

}  // namespace

#define SGUARD_BEGIN try {
#define SGUARD_END                                         \
    }                                                      \
    catch (const std::bad_alloc&) { return PS3D_ERR_OOM; } \
    catch (...) { return PS3D_ERR_CUDA; }

extern "C" {

PS3D_API int ps3d_slab_create(const ps3d_params* global, int nranks, int rank, int device, ps3d_slab** out) {
    SGUARD_BEGIN
    if (!global || !out || nranks < 1 || rank < 0 || rank >= nranks) return PS3D_ERR_BADPARAM;
    *out = nullptr;
    if (global->nz % nranks || global->nz / nranks < 2) return PS3D_ERR_BADPARAM;
    const bool rigid = global->enable_vertical_boundaries != 0;
    if (!rigid && (global->nz % 2 || !ps3d::fft_length_ok(global->nz) || !ps3d::zsolve_fits(global->nz, false)))
        return PS3D_ERR_BADPARAM;
    std::unique_ptr<ps3d_slab> s(new ps3d_slab());
    s->nranks = nranks; s->rank = rank;
    s->mixed = global->precision == PS3D_MIXED || global->precision == PS3D_MIXED_REFINED;
    s->nzg = global->nz; s->nzl = global->nz / nranks; s->k0 = rank * s->nzl;
    s->rigid = rigid;
    s->Lz = global->Lz;
    ps3d_params lp = *global;
    lp.nz = s->nzl + 3;
    lp.Lz = global->dz * lp.nz;   // keeps dz; the local grid's own Lz is not used by the slab phases
    s->ctx.reset(new Ctx());
    Ctx& c = *s->ctx;
    c.force_impl = 1;
    c.split_solve = true;
    c.win_kbeg = 1; c.win_kcount = s->nzl; c.win_kofs = s->k0 - 1; c.win_nzg = s->nzg;
    int rc = c.init(lp, device);
    if (rc) return rc;
    if ((s->mixed ? c.pa32 : c.pa64).impl != 1) return PS3D_ERR_UNSUPPORTED;   // grid the rows + y-lines kernels cannot take
    c.use_graphs = false;
    if (!rigid) {
        // the global z transform and its wavenumbers (my_fft.f90:87-156)
        CK(s->plz.build(s->nzg, 0));
        const double pi = std::acos(0.0) * 2.0, dz = global->dz, Lz = global->Lz;
        std::vector<double> hk(s->nzg);
        for (int k = 1; k <= s->nzg; ++k) {
            const double kz = k <= (s->nzg + 1) / 2 ? 2 * (k - 1) * pi / Lz : -(2 * (s->nzg - k + 1) * pi / Lz);
            hk[k - 1] = 2.0 * (1.0 - std::cos(kz * dz)) / (dz * dz) / global->dsqr;
        }
        CK(s->hkz.alloc(hk.size() * sizeof(double)));
        CK(cudaMemcpy(s->hkz.p, hk.data(), hk.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    s->ncols = (long)c.nxh * c.ny;
    s->plane = (long)c.nx * c.ny;
    for (int r = 0; r < nranks; ++r) {
        const long b = s->ncols * r / nranks, e = s->ncols * (r + 1) / nranks;
        s->cbeg.push_back(b);
        s->ccnt.push_back(e - b);
    }
    CK(s->own_x.alloc(s->xbytes()));
    CK(s->own_col.alloc(s->colbytes()));
    CK(s->own_hs.alloc(s->hbytes()));
    CK(s->own_hr.alloc(s->hbytes()));
    s->xbuf = s->own_x.p; s->colbuf = s->own_col.p; s->hsend = s->own_hs.p; s->hrecv = s->own_hr.p;
    CK(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming));
    *out = s.release();
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_destroy(ps3d_slab* s) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    cudaSetDevice(s->ctx->device);
    delete s;
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_info(ps3d_slab* s, int* k0, int* nzl, long long* col0, long long* ncl, void** stream,
                             int* passes) {
    if (!s) return PS3D_ERR_BADPARAM;
    if (passes) *passes = s->passes();
    if (k0) *k0 = s->k0;
    if (nzl) *nzl = s->nzl;
    if (col0) *col0 = s->cbeg[s->rank];
    if (ncl) *ncl = s->ccnt[s->rank];
    if (stream) *stream = (void*)s->ctx->stream;
    return PS3D_OK;
}

PS3D_API int ps3d_slab_buffers(ps3d_slab* s, size_t* xbytes, size_t* colbytes, size_t* hbytes,
                               long long* col_counts) {
    if (!s) return PS3D_ERR_BADPARAM;
    if (xbytes) *xbytes = s->xbytes();
    if (colbytes) *colbytes = s->colbytes();
    if (hbytes) *hbytes = s->hbytes();
    if (col_counts)
        for (int r = 0; r < s->nranks; ++r) col_counts[r] = s->ccnt[r];
    return PS3D_OK;
}

PS3D_API int ps3d_slab_bind(ps3d_slab* s, void* xbuf, void* colbuf, void* hsend, void* hrecv) {
    SGUARD_BEGIN
    if (!s || !xbuf || !colbuf || !hsend || !hrecv) return PS3D_ERR_BADPARAM;
    cudaSetDevice(s->ctx->device);
    CK(cudaStreamSynchronize(s->ctx->stream));
    s->xbuf = xbuf; s->colbuf = colbuf; s->hsend = hsend; s->hrecv = hrecv;
    s->own_x.release(); s->own_col.release(); s->own_hs.release(); s->own_hr.release();
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_upload(ps3d_slab* s, const double* u, const double* v, const double* w, const double* b) {
    SGUARD_BEGIN
    if (!s || !u || !v || !w || !b) return PS3D_ERR_BADPARAM;
    Ctx& c = *s->ctx;
    cudaSetDevice(c.device);
    CK(cudaStreamSynchronize(c.stream));
    const double* f[4] = {u, v, w, b};
    const size_t bytes = (size_t)s->nzl * s->plane * sizeof(double);
    for (int q = 0; q < 4; ++q) CK(cudaMemcpy(s->lvl(c.field(q), 1), f[q], bytes, cudaMemcpyHostToDevice));
    c.pending = false;
    c.p_warm = false;
    c.itt = 0; c.tau = 3; c.taum1 = 2; c.taum2 = 1; c.time = 0.0;
    for (int q = 0; q < 4; ++q) CK(cudaMemset(c.tend[q].p, 0, c.tend[q].bytes));
    s->need_halo = true;
    return PS3D_OK;
    SGUARD_END
}

// the pending correction of the interior and of both state halo planes (p is
// valid one level below and two above), so the halos stay consistent
static int apply_pending(ps3d_slab* s) {
    Ctx& c = *s->ctx;
    if (c.pending) {
        CK(ps3d::launch_correct(c.field(0), c.field(1), c.field(2), c.pcor, c.nx, c.ny, c.nz, 1, c.dtp,
                                c.dtp / c.P.dsqr, 1.0 / c.P.dx, 1.0 / c.P.dy, 1.0 / c.P.dz, c.stream, 1, 0, s->nzl + 2,
                                s->k0 - 1, s->nzg));
        c.pending = false;
    }
    return PS3D_OK;
}

PS3D_API int ps3d_slab_diagnose(ps3d_slab* s, double* ke_sum, double* pe_sum, double* umax, double* wmax,
                                int* nonfinite) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    Ctx& c = *s->ctx;
    cudaSetDevice(c.device);
    int rc = apply_pending(s);
    if (rc) return rc;
    // the interior levels 1 .. nzl; the potential energy of the N0 = 0 form
    // weighs b by the global level k0 + k
    ps3d::DiagOut* d = (ps3d::DiagOut*)c.red_out.p;
    CK(ps3d::launch_diagnose(s->lvl(c.field(0), 1), s->lvl(c.field(1), 1), s->lvl(c.field(2), 1),
                             s->lvl(c.field(3), 1), s->lvl((double*)c.p.p, 1), c.nx, c.ny, s->nzl, c.P.dsqr, c.P.N0,
                             c.P.dz, (double*)c.red_partials.p, c.nred, d, c.stream, s->k0));
    ps3d::DiagOut h{};
    CK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    if ((rc = c.sync())) return rc;
    const double n = (double)s->nzl * (double)s->plane;   // the kernel returned means over these points
    if (ke_sum) *ke_sum = h.ke * n;
    if (pe_sum) *pe_sum = h.pe * n;
    if (umax) *umax = h.umax;
    if (wmax) *wmax = h.wmax;
    if (nonfinite) *nonfinite = h.flags ? 1 : 0;
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_download(ps3d_slab* s, double* u, double* v, double* w, double* b, double* p) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    Ctx& c = *s->ctx;
    cudaSetDevice(c.device);
    {
        int rc0 = apply_pending(s);
        if (rc0) return rc0;
    }
    int rc = c.sync();
    if (rc) return rc;
    double* f[5] = {u, v, w, b, p};
    const size_t bytes = (size_t)s->nzl * s->plane * sizeof(double);
    for (int q = 0; q < 5; ++q)
        if (f[q]) CK(cudaMemcpy(f[q], s->lvl(q < 4 ? c.field(q) : (double*)c.p.p, 1), bytes, cudaMemcpyDeviceToHost));
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_set_forcing(ps3d_slab* s, const ps3d_forcing* f) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    Ctx& c = *s->ctx;
    cudaSetDevice(c.device);
    CK(cudaStreamSynchronize(c.stream));
    for (int q = 0; q < 4; ++q) { c.wr[q].release(); c.wi[q].release(); }
    c.ub.release(); c.bb.release();
    c.invalidate_graph();
    ++c.forcing_gen;
    c.fkind = 0; c.fn = nullptr; c.user = nullptr;
    if (!f || f->kind == PS3D_FORCE_NONE) return PS3D_OK;
    if (f->kind & ~(PS3D_FORCE_WAVEMAKER | PS3D_FORCE_BACKGROUND | PS3D_FORCE_CALLBACK)) return PS3D_ERR_BADPARAM;
    if (f->kind & PS3D_FORCE_CALLBACK) return PS3D_ERR_UNSUPPORTED;
    // local arrays: levels 0 .. nzl+2 as the state's (halo 0, interior 1 .. nzl, halo nzl+1; the
    // second upper halo, which only p uses, stays zero)
    const size_t nloc = (size_t)(s->nzl + 3) * s->plane * sizeof(double);
    const size_t nin = (size_t)(s->nzl + 2) * s->plane * sizeof(double);
    auto put = [&](DevBuf& d, const double* h) -> cudaError_t {
        cudaError_t e = d.alloc(nloc);
        if (e) return e;
        if ((e = cudaMemset(d.p, 0, nloc))) return e;
        return h ? cudaMemcpy(d.p, h, nin, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    c.omega = f->omega;
    if (f->kind & PS3D_FORCE_WAVEMAKER) {
        const double* r[4] = {f->u_r, f->v_r, f->w_r, f->b_r};
        const double* im[4] = {f->u_i, f->v_i, f->w_i, f->b_i};
        for (int q = 0; q < 4; ++q) {
            if (r[q]) CK(put(c.wr[q], r[q]));
            if (im[q]) CK(put(c.wi[q], im[q]));
        }
    }
    if (f->kind & PS3D_FORCE_BACKGROUND) {
        CK(put(c.ub, f->u_back));
        CK(put(c.bb, f->b_back));
    }
    c.fkind = f->kind;
    if (!c.fused_step()) {   // background flow with Laplacian friction: the generic step
        for (int q = 0; q < 4; ++q) { c.wr[q].release(); c.wi[q].release(); }
        c.ub.release(); c.bb.release();
        c.fkind = 0;
        return PS3D_ERR_UNSUPPORTED;
    }
    return PS3D_OK;
    SGUARD_END
}

PS3D_API int ps3d_slab_phase(ps3d_slab* s, int phase) {
    SGUARD_BEGIN
    if (!s) return PS3D_ERR_BADPARAM;
    cudaSetDevice(s->ctx->device);
    switch (phase) {
        case PS3D_SLAB_TENDENCY: return slab_tendency(s);
        case PS3D_SLAB_PACK_STATE: return halo_pack(s, 0);
        case PS3D_SLAB_UNPACK_STATE: return halo_unpack(s, 0);
        case PS3D_SLAB_FORWARD: return slab_forward(s);
        case PS3D_SLAB_VSOLVE: return slab_vsolve(s);
        case PS3D_SLAB_INVERSE: return slab_inverse(s);
        case PS3D_SLAB_PACK_P: return halo_pack(s, 1);
        case PS3D_SLAB_UNPACK_P: return halo_unpack(s, 1);
        case PS3D_SLAB_END_STEP: return slab_end_step(s);
        default: return PS3D_ERR_BADPARAM;
    }
    SGUARD_END
}

PS3D_API int ps3d_slab_sync(ps3d_slab* s) {
    if (!s) return PS3D_ERR_BADPARAM;
    cudaSetDevice(s->ctx->device);
    return s->ctx->sync();
}

PS3D_API int ps3d_slab_group_step(ps3d_slab* const* ranks, int n, int nsteps) {
    SGUARD_BEGIN
    if (!ranks || n < 1 || nsteps < 0) return PS3D_ERR_BADPARAM;
    for (int q = 0; q < n; ++q)
        if (!ranks[q] || ranks[q]->nranks != n || ranks[q]->rank != q) return PS3D_ERR_BADPARAM;
    for (int t = 0; t < nsteps; ++t) {
        int rc = group_step(ranks, n);
        if (rc) return rc;
    }
    return sync_all(ranks, n);
    SGUARD_END
}

}  // extern "C"
