// ps3d_main.cpp — the reference's main program (for_src/main.f90:1-208) as a
// C++ host over the C ABI of include/ps3d_gpu.h, for hosts without a Fortran
// compiler.  It uses nothing but that header: no CUDA headers, no torch.
//
//   ps3d_main [--dry-run] [parameter file] [key=value ...]
//   ps3d_main --help        the accepted keys
//
// set_parameter        a parameter file of `key = value` lines ('!' and '#'
//                      start comments; Fortran 1d-3 exponents and .true. /
//                      .false. accepted) and key=value arguments after it,
//                      with main_module.f90's defaults (keys below)
// set_initial_conditions
//                      init = rest (all zero) or the path of a raw file of
//                      u, v, w, b (optionally p) in the halo layout, float64
//                      little-endian, x fastest; w is then zeroed on the
//                      rigid-lid levels as main.f90:119-122
// set_forcing          the hook integrate.f90:82 calls, through ps3d_set_forcing:
//                      forcing_wavemaker = path of u_r, v_r, w_r, b_r, u_i, v_i,
//                      w_i, b_i (halo layout) with omega_forc (config.f90:224-237);
//                      forcing_background = path of u_back, b_back
//                      (lee_wave1.f90:245-312); forcing_plugin = lib.so:symbol,
//                      a ps3d_forcing_fn for any other forcing, loaded with
//                      dlopen in place of a compiled-in set_forcing
// read_restart         restart = path (default restart_pe=000000000.dta, the
//                      reference's one-rank file name): read when it exists,
//                      runlen += its time (restart.f90:27-82)
// main loop            main.f90:139-162: integrate; diagnose every
//                      max(1, int(tsmonint/dt)) steps and at itt = 0;
//                      snapshot / diag_balance / diag_opt_balance every
//                      max(1, int(snapint/dt)) steps and at itt = 0; tau
//                      rotation, time += dt, itt += 1.  The steps between two
//                      such events go to the library as one ps3d_integrate
//                      call (n loop bodies, replayed as CUDA graphs).
// write_restart, the timing summary (main.f90:166-187) and the `ritt` file.
//
// Snapshots (diag_snap) and the balance outputs are raw files instead of
// netCDF (no library here): a 64-byte header ("PS3DSNAP", int32 nx, ny, nz,
// nfields, itt, float64 time, zero padding) followed by the fields in the
// halo layout.  Errors print the library's message and exit with status 99,
// the reference's MPI_ABORT code.  --dry-run runs the loop schedule without a
// GPU and prints every event.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "ps3d_gpu.h"

namespace {

struct Run {
    ps3d_params p{};
    bool dx_set = false, dy_set = false, dz_set = false;
    double runlen = 0.0, tsmonint = 0.0, snapint = 0.0;   // main_module.f90:59,107
    bool diag_snap = false;                                // main_module.f90:106
    bool diag_balance = false, diag_balance_filter = false;
    int diag_balance_filter_width = 3;                     // main_module.f90:19-22
    bool diag_opt_balance = false;
    ps3d_optbal opt{1.0, 1.0, 100, 1, 1e-9, 0, 0};         // main_module.f90:23-29
    std::string init = "rest";
    std::string forcing_wavemaker, forcing_background, forcing_plugin;
    double omega_forc = 0.0;
    std::string restart = "restart_pe=000000000.dta";
    bool write_restart = true;
    std::string outdir = ".";
    int device = 0;
    bool profile = false;
    bool dry_run = false;
};

[[noreturn]] void halt(const std::string& msg) {
    std::fprintf(stderr, " ERROR: %s\n", msg.c_str());
    std::fflush(stdout);
    std::exit(99);
}

void check(int rc, const char* what) {
    if (rc != PS3D_OK) halt(std::string(what) + ": " + ps3d_strerror(rc));
}

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

double to_double(const std::string& key, std::string v) {
    for (char& c : v)
        if (c == 'd' || c == 'D') c = 'e';   // Fortran double-precision exponent
    char* end = nullptr;
    const double x = std::strtod(v.c_str(), &end);
    if (v.empty() || *end) halt("bad number for " + key + ": " + v);
    return x;
}

int to_int(const std::string& key, const std::string& v) {
    char* end = nullptr;
    const long x = std::strtol(v.c_str(), &end, 10);
    if (v.empty() || *end || x < -2147483647L || x > 2147483647L) halt("bad integer for " + key + ": " + v);
    return (int)x;
}

bool to_bool(const std::string& key, const std::string& v) {
    const std::string s = lower(v);
    if (s == ".true." || s == "true" || s == "t" || s == "1") return true;
    if (s == ".false." || s == "false" || s == "f" || s == "0") return false;
    halt("bad logical for " + key + ": " + v);
}

using Setter = std::function<void(Run&, const std::string&, const std::string&)>;

const std::map<std::string, Setter>& setters() {
    static const std::map<std::string, Setter> m = [] {
        std::map<std::string, Setter> s;
        auto dbl = [&](const char* k, double ps3d_params::*f) {
            s[k] = [f](Run& r, const std::string& key, const std::string& v) { r.p.*f = to_double(key, v); };
        };
        auto in = [&](const char* k, int ps3d_params::*f) {
            s[k] = [f](Run& r, const std::string& key, const std::string& v) { r.p.*f = to_int(key, v); };
        };
        auto lg = [&](const char* k, int ps3d_params::*f) {
            s[k] = [f](Run& r, const std::string& key, const std::string& v) { r.p.*f = to_bool(key, v) ? 1 : 0; };
        };
        in("nx", &ps3d_params::nx); in("ny", &ps3d_params::ny); in("nz", &ps3d_params::nz);
        dbl("lx", &ps3d_params::Lx); dbl("ly", &ps3d_params::Ly); dbl("lz", &ps3d_params::Lz);
        s["dx"] = [](Run& r, const std::string& k, const std::string& v) { r.p.dx = to_double(k, v); r.dx_set = true; };
        s["dy"] = [](Run& r, const std::string& k, const std::string& v) { r.p.dy = to_double(k, v); r.dy_set = true; };
        s["dz"] = [](Run& r, const std::string& k, const std::string& v) { r.p.dz = to_double(k, v); r.dz_set = true; };
        dbl("dt", &ps3d_params::dt); dbl("f0", &ps3d_params::f0); dbl("n0", &ps3d_params::N0);
        dbl("ro", &ps3d_params::Ro); dbl("dsqr", &ps3d_params::dsqr); dbl("eps_ab", &ps3d_params::eps_ab);
        dbl("ah", &ps3d_params::Ah); dbl("av", &ps3d_params::Av); dbl("kh", &ps3d_params::Kh);
        dbl("kv", &ps3d_params::Kv); dbl("ahbi", &ps3d_params::Ahbi); dbl("avbi", &ps3d_params::Avbi);
        dbl("khbi", &ps3d_params::Khbi); dbl("kvbi", &ps3d_params::Kvbi);
        lg("enable_nonlinear", &ps3d_params::enable_nonlinear);
        lg("enable_vertical_boundaries", &ps3d_params::enable_vertical_boundaries);
        lg("enable_ab_3_order", &ps3d_params::enable_AB_3_order);
        s["precision"] = [](Run& r, const std::string& k, const std::string& v) {
            const std::string x = lower(v);
            if (x == "fp64" || x == "0") r.p.precision = PS3D_FP64;
            else if (x == "mixed" || x == "1") r.p.precision = PS3D_MIXED;
            else if (x == "mixed_refined" || x == "2") r.p.precision = PS3D_MIXED_REFINED;
            else halt("bad value for " + k + ": " + v + " (fp64, mixed or mixed_refined)");
        };
        s["runlen"] = [](Run& r, const std::string& k, const std::string& v) { r.runlen = to_double(k, v); };
        s["tsmonint"] = [](Run& r, const std::string& k, const std::string& v) { r.tsmonint = to_double(k, v); };
        s["snapint"] = [](Run& r, const std::string& k, const std::string& v) { r.snapint = to_double(k, v); };
        s["enable_diag_snap"] = [](Run& r, const std::string& k, const std::string& v) { r.diag_snap = to_bool(k, v); };
        s["enable_diag_balance"] = [](Run& r, const std::string& k, const std::string& v) {
            r.diag_balance = r.diag_balance || to_bool(k, v);
        };
        s["enable_diag_balance_chunks"] = s["enable_diag_balance"];
        s["enable_diag_balance_filter"] = [](Run& r, const std::string& k, const std::string& v) {
            r.diag_balance_filter = to_bool(k, v);
        };
        s["diag_balance_filter_width"] = [](Run& r, const std::string& k, const std::string& v) {
            r.diag_balance_filter_width = to_int(k, v);
        };
        s["enable_diag_opt_balance"] = [](Run& r, const std::string& k, const std::string& v) {
            r.diag_opt_balance = to_bool(k, v);
        };
        s["enable_diag_opt_time_ave"] = [](Run& r, const std::string& k, const std::string& v) {
            r.opt.enable_time_ave = to_bool(k, v) ? 1 : 0;
        };
        s["opt_balance_period"] = [](Run& r, const std::string& k, const std::string& v) { r.opt.period = to_double(k, v); };
        s["opt_balance_average"] = [](Run& r, const std::string& k, const std::string& v) { r.opt.average = to_double(k, v); };
        s["opt_balance_max_itts"] = [](Run& r, const std::string& k, const std::string& v) { r.opt.max_itts = to_int(k, v); };
        s["opt_balance_average_times"] = [](Run& r, const std::string& k, const std::string& v) {
            r.opt.average_times = to_int(k, v);
        };
        s["opt_balance_tol"] = [](Run& r, const std::string& k, const std::string& v) { r.opt.tol = to_double(k, v); };
        s["init"] = [](Run& r, const std::string&, const std::string& v) { r.init = v; };
        s["forcing_wavemaker"] = [](Run& r, const std::string&, const std::string& v) { r.forcing_wavemaker = v; };
        s["forcing_background"] = [](Run& r, const std::string&, const std::string& v) { r.forcing_background = v; };
        s["forcing_plugin"] = [](Run& r, const std::string&, const std::string& v) { r.forcing_plugin = v; };
        s["omega_forc"] = [](Run& r, const std::string& k, const std::string& v) { r.omega_forc = to_double(k, v); };
        s["restart"] = [](Run& r, const std::string&, const std::string& v) { r.restart = v; };
        s["write_restart"] = [](Run& r, const std::string& k, const std::string& v) { r.write_restart = to_bool(k, v); };
        s["outdir"] = [](Run& r, const std::string&, const std::string& v) { r.outdir = v; };
        s["device"] = [](Run& r, const std::string& k, const std::string& v) { r.device = to_int(k, v); };
        s["profile"] = [](Run& r, const std::string& k, const std::string& v) { r.profile = to_bool(k, v); };
        return s;
    }();
    return m;
}

void set_one(Run& r, const std::string& line, const std::string& where) {
    const size_t eq = line.find('=');
    if (eq == std::string::npos) halt("expected key = value at " + where + ": " + line);
    const std::string key = lower(trim(line.substr(0, eq)));
    std::string val = trim(line.substr(eq + 1));
    if (val.size() >= 2 && (val.front() == '\'' || val.front() == '"') && val.back() == val.front())
        val = val.substr(1, val.size() - 2);
    auto it = setters().find(key);
    if (it == setters().end()) halt("unknown parameter " + key + " at " + where);
    it->second(r, key, val);
}

void read_parameter_file(Run& r, const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) halt(std::string("cannot open parameter file ") + path);
    char buf[4096];
    int ln = 0;
    while (std::fgets(buf, sizeof buf, f)) {
        ++ln;
        std::string s(buf);
        const size_t c = s.find_first_of("!#");
        if (c != std::string::npos) s = s.substr(0, c);
        s = trim(s);
        if (!s.empty()) set_one(r, s, std::string(path) + ":" + std::to_string(ln));
    }
    std::fclose(f);
}

// set_parameter (config.f90) from the command line; main_module.f90:16-57 defaults
Run set_parameter(int argc, char** argv) {
    Run r;
    r.p.Ro = 1.0; r.p.dsqr = 1.0; r.p.eps_ab = 0.0;
    r.p.enable_nonlinear = 1; r.p.enable_vertical_boundaries = 0; r.p.enable_AB_3_order = 0;
    r.p.precision = PS3D_FP64;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--help" || s == "-h") {
            std::printf("usage: %s [--dry-run] [parameter file] [key=value ...]\nkeys:", argv[0]);
            int col = 0;
            for (const auto& kv : setters()) {
                if (col % 4 == 0) std::printf("\n ");
                std::printf(" %-28s", kv.first.c_str());
                ++col;
            }
            std::printf("\n");
            std::exit(0);
        }
        if (s == "--dry-run") r.dry_run = true;
        else if (s.find('=') != std::string::npos) set_one(r, s, "argument " + std::to_string(a));
        else read_parameter_file(r, argv[a]);
    }
    if (r.p.nx < 1 || r.p.ny < 1 || r.p.nz < 1) halt("nx, ny, nz must be set");
    if (!r.dx_set) r.p.dx = r.p.Lx / r.p.nx;
    if (!r.dy_set) r.p.dy = r.p.Ly / r.p.ny;
    if (!r.dz_set) r.p.dz = r.p.Lz / r.p.nz;
    if (!(r.p.dt > 0.0)) halt("dt must be positive");
    return r;
}

// main.f90:45-57
void check_grid(const Run& r) {
    const ps3d_params& p = r.p;
    auto bad = [](int n) { return n % 2 != 0 && n > 1; };
    if (p.enable_vertical_boundaries) {
        if (bad(p.nx) || bad(p.ny)) halt("nx,ny need to be even or one");
    } else if (bad(p.nx) || bad(p.ny) || bad(p.nz)) {
        halt("nx,ny,nz need to be even or one");
    }
}

// main.f90:84-108
void print_parameters(const Run& r) {
    const ps3d_params& p = r.p;
    std::printf(" \n nx x ny x nz = %4d x %4d x %4d\n", p.nx, p.ny, p.nz);
    std::printf(" Lx x Ly x Lz = %8.2f x %8.2f x %8.2f m\n", p.Lx, p.Ly, p.Lz);
    std::printf(" Ro      = %8.2f\n delta   = %8.2f\n", p.Ro, std::sqrt(p.dsqr));
    std::printf(" Delta t = %8.2f s\n Delta x = %8.2f m\n Delta y = %8.2f m\n Delta z = %8.2f m\n", p.dt, p.dx, p.dy,
                p.dz);
    std::printf(" Ah      = %12.6e m**2/s\n Kh      = %12.6e m**2/s\n", p.Ah, p.Kh);
    std::printf(" Av      = %12.6e m**2/s\n Kv      = %12.6e m**2/s\n", p.Av, p.Kv);
    std::printf(" Ahbi    = %12.6e m**4/s\n Khbi    = %12.6e m**4/s\n", p.Ahbi, p.Khbi);
    std::printf(" Avbi    = %12.6e m**4/s\n Kvbi    = %12.6e m**4/s\n", p.Avbi, p.Kvbi);
    std::printf(" f0      = %12.6e 1/s\n N0      = %12.6e 1/s\n", p.f0, p.N0);
    std::printf(" runlen  = %8.2f s\n eps_ab  = %12.6e\n", r.runlen, p.eps_ab);
    std::printf(" enable_vertical_boundaries  = %s\n enable_AB_3_order           = %s\n",
                p.enable_vertical_boundaries ? "T" : "F", p.enable_AB_3_order ? "T" : "F");
    std::printf(" precision                   = %s\n \n",
                p.precision == PS3D_FP64 ? "fp64" : p.precision == PS3D_MIXED ? "mixed" : "mixed_refined");
}

// max(1, int(interval/dt)) of main.f90:144-145, without overflowing the int
int every(double interval, double dt) {
    const double q = std::trunc(interval / dt);
    if (!(q >= 1.0)) return 1;
    return q > 2147483647.0 ? 2147483647 : (int)q;
}

size_t halo_points(const ps3d_params& p) { return (size_t)(p.nx + 4) * (p.ny + 4) * (p.nz + 4); }

std::string out_path(const Run& r, const std::string& name) {
    if (name.empty() || name[0] == '/' || r.outdir.empty() || r.outdir == ".") return name;
    return r.outdir + "/" + name;
}

void write_fields(const Run& r, const char* stem, int itt, double time, const std::vector<const double*>& fields) {
    char name[96];
    std::snprintf(name, sizeof name, "%s_%09d.bin", stem, itt);
    const std::string path = out_path(r, name);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) halt("cannot write " + path);
    unsigned char hdr[64] = {0};
    std::memcpy(hdr, "PS3DSNAP", 8);
    const int32_t ints[5] = {r.p.nx, r.p.ny, r.p.nz, (int32_t)fields.size(), itt};
    std::memcpy(hdr + 8, ints, sizeof ints);
    std::memcpy(hdr + 32, &time, sizeof time);
    bool ok = std::fwrite(hdr, 1, sizeof hdr, f) == sizeof hdr;
    const size_t n = halo_points(r.p);
    for (const double* a : fields) ok = ok && std::fwrite(a, sizeof(double), n, f) == n;
    if (std::fclose(f) != 0 || !ok) halt("error writing " + path);
}

// fields in the halo layout from a raw file holding one of `counts` fields;
// returns how many it held
int read_fields(const Run& r, const std::string& path, const char* what, std::initializer_list<int> counts,
                std::vector<std::vector<double>>& f) {
    const size_t n = halo_points(r.p);
    FILE* fh = std::fopen(path.c_str(), "rb");
    if (!fh) halt(std::string("cannot open ") + what + " " + path);
    std::fseek(fh, 0, SEEK_END);
    const long bytes = std::ftell(fh);
    std::fseek(fh, 0, SEEK_SET);
    int nf = 0;
    std::string want;
    for (int c : counts) {
        if (bytes == (long)(c * n * sizeof(double))) nf = c;
        want += (want.empty() ? "" : " or ") + std::to_string(c * n * sizeof(double));
    }
    if (!nf) halt(std::string(what) + " " + path + ": " + std::to_string(bytes) + " bytes, expected " + want);
    if ((int)f.size() < nf) f.resize(nf, std::vector<double>(n, 0.0));
    for (int q = 0; q < nf; ++q)
        if (std::fread(f[q].data(), sizeof(double), n, fh) != n) halt("short read of " + path);
    std::fclose(fh);
    return nf;
}

// set_forcing (integrate.f90:82) through ps3d_set_forcing; the host arrays
// are copied to the device during the call
void set_forcing(const Run& r, ps3d_ctx* ctx) {
    ps3d_forcing fc{};
    std::vector<std::vector<double>> wm, bg;
    if (!r.forcing_wavemaker.empty()) {
        read_fields(r, r.forcing_wavemaker, "wavemaker forcing (u_r, v_r, w_r, b_r, u_i, v_i, w_i, b_i)", {8}, wm);
        fc.kind |= PS3D_FORCE_WAVEMAKER;
        fc.omega = r.omega_forc;
        fc.u_r = wm[0].data(); fc.v_r = wm[1].data(); fc.w_r = wm[2].data(); fc.b_r = wm[3].data();
        fc.u_i = wm[4].data(); fc.v_i = wm[5].data(); fc.w_i = wm[6].data(); fc.b_i = wm[7].data();
    }
    if (!r.forcing_background.empty()) {
        read_fields(r, r.forcing_background, "background flow (u_back, b_back)", {2}, bg);
        fc.kind |= PS3D_FORCE_BACKGROUND;
        fc.u_back = bg[0].data(); fc.b_back = bg[1].data();
    }
    if (!r.forcing_plugin.empty()) {
        const size_t c = r.forcing_plugin.rfind(':');
        if (c == std::string::npos || c == 0 || c + 1 == r.forcing_plugin.size())
            halt("forcing_plugin wants library:symbol, got " + r.forcing_plugin);
        const std::string lib = r.forcing_plugin.substr(0, c), sym = r.forcing_plugin.substr(c + 1);
        void* h = dlopen(lib.c_str(), RTLD_NOW | RTLD_LOCAL);   // kept open for the run
        if (!h) halt("cannot load forcing plugin " + lib + ": " + dlerror());
        void* fn = dlsym(h, sym.c_str());
        if (!fn) halt("forcing plugin " + lib + " has no symbol " + sym);
        fc.kind |= PS3D_FORCE_CALLBACK;
        fc.fn = reinterpret_cast<ps3d_forcing_fn>(fn);
        fc.user = nullptr;
    }
    if (fc.kind) check(ps3d_set_forcing(ctx, &fc), "ps3d_set_forcing");
}

// set_initial_conditions: a rest state or the fields of a file
void initial_conditions(const Run& r, std::vector<std::vector<double>>& f, bool& have_p) {
    const size_t n = halo_points(r.p);
    f.assign(5, std::vector<double>(n, 0.0));
    have_p = false;
    if (lower(r.init) != "rest") have_p = read_fields(r, r.init, "initial conditions (u, v, w, b[, p])", {4, 5}, f) == 5;
    if (r.p.enable_vertical_boundaries) {   // main.f90:119-122: w(:,:,1-onx:0) = 0, w(:,:,nz:nz+onx) = 0
        const size_t plane = (size_t)(r.p.nx + 4) * (r.p.ny + 4);
        std::vector<double>& w = f[2];
        for (int L : {0, 1, r.p.nz + 1, r.p.nz + 2, r.p.nz + 3})   // k = -1, 0, nz, nz+1, nz+2
            std::fill(w.begin() + (size_t)L * plane, w.begin() + (size_t)(L + 1) * plane, 0.0);
    }
}

bool file_exists(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
}

double now() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// diagnose (diagnose.F90:2-61): the library's reductions, the reference's output
void diagnose(const Run& r, ps3d_ctx* ctx, int itt, double time) {
    std::printf(" diagnosing at t=%8.2f itt=%10d\n", time, itt);
    double ke = 0, pe = 0, umax = 0, wmax = 0;
    const int rc = ps3d_diagnose(ctx, &ke, &pe, &umax, &wmax);
    if (rc == PS3D_ERR_NONFINITE) {
        std::printf(" ERROR: in diagnose detected NaN, aborting at t=%g itt=%d\n", time, itt);
        halt("in diagnose");
    }
    check(rc, "ps3d_diagnose");
    const ps3d_params& p = r.p;
    const double cfl_h = umax * p.dt / p.dx, cfl_v = wmax * p.dt / p.dz;
    const double um = std::max(umax, wmax);
    const double pecl_h = std::min(um * p.dx / (1e-32 + p.Ah), um * p.dx * p.dx * p.dx / (1e-32 + p.Ahbi));
    const double pecl_v = std::min(um * p.dz / (1e-32 + p.Av), um * p.dz * p.dz * p.dz / (1e-32 + p.Avbi));
    std::printf(" max hor. CFL = %8.2f hor. PECL = %8.2e\n", cfl_h, pecl_h);
    std::printf(" max ver. CFL = %8.2f ver. PECL = %8.2e\n", cfl_v, pecl_v);
    std::printf(" KE = %10.4e m^2/s^2, PE = %10.4e m^2/s^2, sum %20.14e m^2/s^2\n", ke, pe, ke + pe);
}

struct Snap {
    std::vector<std::vector<double>> f;
    bool pending = false;
    int itt = 0;
    double time = 0.0;
};

void finish_snapshot(const Run& r, ps3d_ctx* ctx, Snap& s) {
    if (!s.pending) return;
    check(ps3d_snapshot_wait(ctx), "ps3d_snapshot_wait");
    write_fields(r, "snap", s.itt, s.time, {s.f[0].data(), s.f[1].data(), s.f[2].data(), s.f[3].data(), s.f[4].data()});
    s.pending = false;
}

}  // namespace

int main(int argc, char** argv) {
    const double t_setup = now();
    Run r = set_parameter(argc, argv);
    std::printf(" setting parameters \n");
    check_grid(r);
    print_parameters(r);
    ps3d_params& p = r.p;
    const int nmon = every(r.tsmonint, p.dt), nsnap = every(r.snapint, p.dt);
    const bool snap_work = r.diag_snap || r.diag_balance || r.diag_opt_balance;
    auto due_diag = [&](int itt) { return itt % nmon == 0 || itt == 0; };
    auto due_snap = [&](int itt) { return snap_work && (itt % nsnap == 0 || itt == 0); };

    double time = 0.0;
    int itt = 0;
    ps3d_ctx* ctx = nullptr;
    if (!r.dry_run) {
        check(ps3d_create(&p, r.device, &ctx), "ps3d_create");   // allocate_main_module, wavenumber_initialisation
        set_forcing(r, ctx);
        std::printf(" setting initial conditions \n");
        std::vector<std::vector<double>> f;
        bool have_p = false;
        initial_conditions(r, f, have_p);
        check(ps3d_upload_state(ctx, f[0].data(), f[1].data(), f[2].data(), f[3].data(), have_p ? f[4].data() : nullptr,
                                nullptr, nullptr, nullptr, nullptr, 0, 3, 2, 1),
              "ps3d_upload_state");
        std::printf(" done setting initial conditions \n");
    }
    const double setup_s = now() - t_setup;
    std::printf(" starting main loop \n");

    // read_restart (restart.f90:27-82)
    const std::string rpath = out_path(r, r.restart);
    if (!r.dry_run && file_exists(rpath)) {
        std::printf(" reading restart file %s\n", rpath.c_str());
        double t0 = 0.0;
        const int rc = ps3d_read_restart(ctx, rpath.c_str(), &t0);
        if (rc != PS3D_OK) {
            std::printf(" Warning: error reading restart file\n");
            halt(std::string("ps3d_read_restart: ") + ps3d_strerror(rc));
        }
        int tau = 0, t1 = 0, t2 = 0;
        check(ps3d_download_state(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  &itt, &tau, &t1, &t2),
              "ps3d_download_state");
        time = t0;
        std::printf(" time = %g itt = %d\n", time, itt);
        r.runlen += time;
        std::printf(" adjusting run length to = %g\n", r.runlen);
    } else if (!r.dry_run) {
        std::printf(" found no restart file %s\n proceeding with initial conditions\n", rpath.c_str());
    }
    if (!r.dry_run && r.profile) check(ps3d_profile(ctx, 1), "ps3d_profile");

    Snap snap;
    if (r.diag_snap) snap.f.assign(5, std::vector<double>(halo_points(p)));
    std::vector<std::vector<double>> bal;
    double integrate_s = 0.0, diag_s = 0.0;
    long long steps = 0, calls = 0;
    const double t_loop = now();
    while (time < r.runlen) {
        // the loop bodies up to and including the next one with an event
        int k = 0, ev_itt = -1;
        double ev_time = 0.0;
        bool ev_diag = false, ev_snap = false;
        while (time < r.runlen) {
            ++k;
            ev_diag = due_diag(itt);
            ev_snap = due_snap(itt);
            if (ev_diag || ev_snap) { ev_itt = itt; ev_time = time; }
            time = time + p.dt;   // main.f90:156-160, after the diagnostics of this itt
            ++itt;
            if (ev_itt >= 0) break;
        }
        steps += k;
        ++calls;
        if (r.dry_run) {
            std::printf("integrate %d\n", k);
        } else {
            const double t0 = now();
            check(ps3d_integrate(ctx, k), "ps3d_integrate");
            integrate_s += now() - t0;
        }
        if (ev_itt < 0) continue;
        const double t0 = now();
        if (r.dry_run) {
            if (ev_diag) std::printf("diagnose itt=%d time=%.17g\n", ev_itt, ev_time);
            if (ev_snap) std::printf("snapshot itt=%d time=%.17g\n", ev_itt, ev_time);
            continue;
        }
        if (ev_diag) diagnose(r, ctx, ev_itt, ev_time);
        if (ev_snap) {
            if (r.diag_snap) {
                finish_snapshot(r, ctx, snap);
                check(ps3d_snapshot_begin(ctx, snap.f[0].data(), snap.f[1].data(), snap.f[2].data(), snap.f[3].data(),
                                          snap.f[4].data()),
                      "ps3d_snapshot_begin");
                snap.pending = true; snap.itt = ev_itt; snap.time = ev_time;
            }
            if ((r.diag_balance || r.diag_opt_balance) && bal.empty())
                bal.assign(4, std::vector<double>(halo_points(p)));
            if (r.diag_balance) {
                // diag_balance (diag_balance.f90:89-106): orders 0..3; the balanced state is their sum
                check(ps3d_diag_balance(ctx, 3, r.diag_balance_filter ? r.diag_balance_filter_width : -1),
                      "ps3d_diag_balance");
                std::vector<std::vector<double>> sum(4, std::vector<double>(halo_points(p), 0.0));
                for (int which = PS3D_FIELDS_ZERO; which <= PS3D_FIELDS_THIRD; ++which) {
                    check(ps3d_get_fields(ctx, which, bal[0].data(), bal[1].data(), bal[2].data(), bal[3].data()),
                          "ps3d_get_fields");
                    for (int q = 0; q < 4; ++q)
                        for (size_t i = 0; i < sum[q].size(); ++i) sum[q][i] += bal[q][i];
                }
                write_fields(r, "balance", ev_itt, ev_time, {sum[0].data(), sum[1].data(), sum[2].data(), sum[3].data()});
            }
            if (r.diag_opt_balance) {
                // diag_opt_balance + write_diag_opt_balance (diag_opt_balance.f90:55-258)
                double norm = 0.0;
                int iters = 0;
                check(ps3d_opt_balance(ctx, &r.opt, &norm, &iters), "ps3d_opt_balance");
                std::printf(" optimal balance: %d iterations, norm of last change %e\n", iters, norm);
                check(ps3d_get_fields(ctx, PS3D_FIELDS_BALANCED, bal[0].data(), bal[1].data(), bal[2].data(),
                                      bal[3].data()),
                      "ps3d_get_fields");
                write_fields(r, "opt_balance", ev_itt, ev_time, {bal[0].data(), bal[1].data(), bal[2].data(), bal[3].data()});
            }
        }
        diag_s += now() - t0;
    }
    const double loop_s = now() - t_loop;

    if (r.dry_run) {
        std::printf("final itt=%d time=%.17g steps=%lld calls=%lld\n", itt, time, steps, calls);
        return 0;
    }
    finish_snapshot(r, ctx, snap);
    if (r.write_restart) {   // write_restart (restart.f90:2-22)
        std::printf(" writing to restart file %s\n at itt = %12d\n", rpath.c_str(), itt);
        const int rc = ps3d_write_restart(ctx, rpath.c_str());
        if (rc != PS3D_OK) std::printf(" Warning: error writing restart file\n");
    }
    // timing summary (main.f90:166-180)
    std::printf("\nTiming summary for PE #   0\n");
    std::printf(" setup time summary       = %15.2f s\n", setup_s);
    std::printf(" loop                     = %15.2f s\n", loop_s);
    std::printf(" integrate                = %15.2f s\n", integrate_s);
    if (r.profile) {
        double ms[PS3D_K_COUNT] = {0};
        long long n[PS3D_K_COUNT] = {0};
        check(ps3d_profile_read(ctx, ms, n), "ps3d_profile_read");
        std::printf(" stencils (device)        = %15.4f s\n", ms[PS3D_K_STEP] * 1e-3);
        std::printf(" pressure (device)        = %15.4f s\n",
                    (ms[PS3D_K_FFT_FWD] + ms[PS3D_K_VSOLVE] + ms[PS3D_K_FFT_INV] + ms[PS3D_K_CORRECT]) * 1e-3);
    }
    std::printf(" diagnostics              = %15.2f s\n", diag_s);
    std::printf(" steps %lld in %lld library calls\n", steps, calls);
    // main.f90:190-195
    const std::string ritt = out_path(r, "ritt");
    if (FILE* f = std::fopen(ritt.c_str(), "w")) {
        std::fprintf(f, "%12d\n", itt);
        std::fclose(f);
    }
    check(ps3d_destroy(ctx), "ps3d_destroy");
    std::printf("\n");
    return 0;
}
