// restart.cu — the reference's restart file for one rank (restart.f90:2-82).
//
// A Fortran unformatted sequential file as gfortran writes it: every record
// is framed by 4-byte little-endian length markers.  Three records:
//   1. nx, ny, nz, itt (int32), time (real*8), taum2, taum1, tau (int32)
//   2. is_pe, ie_pe, js_pe, je_pe, ks_pe, ke_pe (int32; 1, nx, 1, ny, 1, nz)
//   3. u, v, w, b, p, du, dv, dw, db (real*8, halo layout, du..db with the
//      trailing time-level dimension 3)
// A record longer than 2147483639 bytes is split into subrecords of at most
// that length; the leading marker of a subrecord that is continued and the
// trailing marker of a subrecord that continues another carry the negative
// length (gfortran's convention for records beyond 2 GiB).
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#include "ctx.h"

namespace {

constexpr long long kMaxSub = 2147483639LL;

struct File {
    std::FILE* f = nullptr;
    ~File() { if (f) std::fclose(f); }
};

bool put_marker(std::FILE* f, long long v) {
    const int m = (int)v;
    return std::fwrite(&m, 4, 1, f) == 1;
}

// one record made of `parts` (pointer, bytes) written back to back
bool write_record(std::FILE* f, const std::vector<std::pair<const void*, size_t>>& parts) {
    long long total = 0;
    for (auto& p : parts) total += (long long)p.second;
    size_t pi = 0, off = 0;
    long long left = total;
    bool first = true;
    do {
        const long long n = left > kMaxSub ? kMaxSub : left;
        const bool more = left > kMaxSub;
        if (!put_marker(f, more ? -n : n)) return false;
        long long todo = n;
        while (todo > 0) {
            const size_t avail = parts[pi].second - off;
            const size_t k = (size_t)std::min<long long>(todo, (long long)avail);
            if (k && std::fwrite((const char*)parts[pi].first + off, 1, k, f) != k) return false;
            off += k;
            todo -= (long long)k;
            if (off == parts[pi].second) { ++pi; off = 0; }
        }
        if (!put_marker(f, first ? n : -n)) return false;
        first = false;
        left -= n;
    } while (left > 0);
    return true;
}

// reads one record into the given parts; false if its length differs
bool read_record(std::FILE* f, const std::vector<std::pair<void*, size_t>>& parts) {
    long long want = 0;
    for (auto& p : parts) want += (long long)p.second;
    size_t pi = 0, off = 0;
    long long got = 0;
    for (;;) {
        int lead = 0, trail = 0;
        if (std::fread(&lead, 4, 1, f) != 1) return false;
        const long long n = lead < 0 ? -(long long)lead : lead;
        if (got + n > want) return false;
        long long todo = n;
        while (todo > 0) {
            const size_t avail = parts[pi].second - off;
            const size_t k = (size_t)std::min<long long>(todo, (long long)avail);
            if (k && std::fread((char*)parts[pi].first + off, 1, k, f) != k) return false;
            off += k;
            todo -= (long long)k;
            if (off == parts[pi].second) { ++pi; off = 0; }
        }
        got += n;
        if (std::fread(&trail, 4, 1, f) != 1) return false;
        if ((trail < 0 ? -(long long)trail : trail) != n) return false;
        if (lead >= 0) break;
    }
    return got == want;
}

}  // namespace

namespace ps3d {

int Ctx::write_restart(const char* path) {
    if (!path || batch != 1) return PS3D_ERR_BADPARAM;
    int rc = materialize();
    if (rc) return rc;
    const size_t n3 = (size_t)(nx + 4) * (ny + 4) * (nz + 4);
    std::vector<double> h(17 * n3);
    double* f[5] = {h.data(), h.data() + n3, h.data() + 2 * n3, h.data() + 3 * n3, h.data() + 4 * n3};
    for (int q = 0; q < 4; ++q) if ((rc = download_field(field(q), f[q], 0))) return rc;
    if ((rc = download_field((const double*)p.p, f[4], 1))) return rc;
    for (int q = 0; q < 4; ++q) if ((rc = download_tend(q, h.data() + (5 + 3 * q) * n3))) return rc;
    File F;
    F.f = std::fopen(path, "wb");
    if (!F.f) return PS3D_ERR_BADPARAM;
    const int hdr_i[4] = {nx, ny, nz, itt}, hdr_t[3] = {taum2, taum1, tau};
    const double t = time;
    const int bounds[6] = {1, nx, 1, ny, 1, nz};
    bool ok = write_record(F.f, {{hdr_i, sizeof hdr_i}, {&t, sizeof t}, {hdr_t, sizeof hdr_t}}) &&
              write_record(F.f, {{bounds, sizeof bounds}}) &&
              write_record(F.f, {{h.data(), h.size() * sizeof(double)}});
    return ok ? PS3D_OK : PS3D_ERR_BADPARAM;
}

int Ctx::read_restart(const char* path, double* time_out) {
    if (!path || batch != 1) return PS3D_ERR_BADPARAM;
    File F;
    F.f = std::fopen(path, "rb");
    if (!F.f) return PS3D_ERR_BADPARAM;
    int hdr_i[4], hdr_t[3], bounds[6];
    double t = 0.0;
    if (!read_record(F.f, {{hdr_i, sizeof hdr_i}, {&t, sizeof t}, {hdr_t, sizeof hdr_t}})) return PS3D_ERR_BADPARAM;
    if (hdr_i[0] != nx || hdr_i[1] != ny || hdr_i[2] != nz) return PS3D_ERR_BADPARAM;   // restart.f90:57-64
    if (!read_record(F.f, {{bounds, sizeof bounds}})) return PS3D_ERR_BADPARAM;
    if (bounds[0] != 1 || bounds[1] != nx || bounds[2] != 1 || bounds[3] != ny || bounds[4] != 1 || bounds[5] != nz)
        return PS3D_ERR_BADPARAM;                                                        // restart.f90:68-75
    for (int v : hdr_t) if (v < 1 || v > 3) return PS3D_ERR_BADPARAM;
    const size_t n3 = (size_t)(nx + 4) * (ny + 4) * (nz + 4);
    std::vector<double> h(17 * n3);
    if (!read_record(F.f, {{h.data(), h.size() * sizeof(double)}})) return PS3D_ERR_BADPARAM;
    int rc = materialize();
    if (rc) return rc;
    state_replaced();
    pending = false;
    for (int q = 0; q < 4; ++q) if ((rc = upload_field(field(q), h.data() + q * n3))) return rc;
    if ((rc = upload_field((double*)p.p, h.data() + 4 * n3))) return rc;
    for (int q = 0; q < 4; ++q) if ((rc = upload_tend(q, h.data() + (5 + 3 * q) * n3))) return rc;
    itt = hdr_i[3];
    taum2 = hdr_t[0]; taum1 = hdr_t[1]; tau = hdr_t[2];
    time = t;
    if (time_out) *time_out = t;
    return PS3D_OK;
}

// ---------------------------------------------------------------------------
// Asynchronous snapshot (the snapshot cadence of main.f90:144-152 without the
// netCDF writer): the state and p are copied on the device at the point of
// the call, then converted to the halo layout and copied to the host on a
// second stream while the main stream keeps stepping.
// ---------------------------------------------------------------------------
int Ctx::snapshot_begin(double* const* host) {
    if (batch != 1) return PS3D_ERR_BADPARAM;
    int rc = materialize();
    if (rc) return rc;
    if (!snap_stream) CK(cudaStreamCreateWithFlags(&snap_stream, cudaStreamNonBlocking));
    if (!snap_event) CK(cudaEventCreateWithFlags(&snap_event, cudaEventDisableTiming));
    CK(cudaStreamSynchronize(snap_stream));   // the previous snapshot's buffers are free
    const size_t n3 = (size_t)(nx + 4) * (ny + 4) * (nz + 4);
    if (!snap[0].p) {
        for (int q = 0; q < 5; ++q) CK(snap[q].alloc(N * sizeof(double)));
        CK(snap_staging.alloc(n3 * sizeof(double)));
    }
    const double* src[5] = {field(0), field(1), field(2), field(3), (const double*)p.p};
    for (int q = 0; q < 5; ++q)
        CK(cudaMemcpyAsync(snap[q].p, src[q], N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaEventRecord(snap_event, stream));
    CK(cudaStreamWaitEvent(snap_stream, snap_event, 0));
    for (int q = 0; q < 5; ++q) {
        if (!host[q]) continue;
        CK(launch_to_halo(snap[q].p, (double*)snap_staging.p, nx, ny, nz, q == 4 && rigid, false, snap_stream));
        CK(cudaMemcpyAsync(host[q], snap_staging.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, snap_stream));
    }
    return PS3D_OK;
}

int Ctx::snapshot_wait() {
    if (!snap_stream) return PS3D_OK;
    CK(cudaStreamSynchronize(snap_stream));
    CK(cudaGetLastError());
    return PS3D_OK;
}

}  // namespace ps3d
