// lsb_run -- the reference's time loop (src/main.f90:62-111) as a native driver over the C
// ABI of include/lsbgpu.h: read the run's set-up and a restart file, advance the resident
// state with lsb_step, write a q snapshot every iomod steps (and after the last step when
// NSTEPS is not a multiple of IOMOD) and a restart file at the end, in the reference's
// float32 layouts (src/mpi_io.f90:9-161 restart, :339-497 snapshot).
//
//   lsb_run SETUP START NSTEPS IOMOD OUTDIR [--no-ref-bug]
//   lsb_run --check-setup SETUP            counts and sums of the set-up arrays (no device)
//   lsb_run --io-selftest START OUTDIR     restart round trip and q layout (no device)
//
// SETUP is written by lsbflow_b200.lib.write_setup_file: the lsb_config struct and the
// lsb_create arrays, the eigendecomposition of the Chebyshev Helmholtz operator included
// (an input, as diag/smat/simat are inputs of solve_helmholtz, src/helmholtz.f90:130).
// Like the reference, the driver stops with a message on the first error.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lsbgpu.h"

namespace {

[[noreturn]] void die(const std::string& m) {
    std::fprintf(stderr, "lsb_run: %s\n", m.c_str());
    std::exit(1);
}

void ck(int rc, const char* what) {
    if (rc != LSB_OK) die(std::string(what) + " failed (" + std::to_string(rc) + "): " + lsb_last_error());
}

std::vector<char> read_file(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) die("cannot open " + path);
    std::vector<char> buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    std::fclose(f);
    return buf;
}

void write_file(const std::string& path, const std::vector<float>& data) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) die("cannot create " + path);
    if (std::fwrite(data.data(), sizeof(float), data.size(), f) != data.size()) die("short write to " + path);
    std::fclose(f);
}

// ------------------------------------------------------------------ set-up file
const char* const kArrayNames[18] = {"xpts", "ypts", "zpts", "wavx", "wavy", "dz1", "dz2", "lam", "e",
                                     "ei", "ubar", "ubarp", "ubarpp", "hbot", "htop", "d2hbot", "d2htop",
                                     "lamx"};

struct Setup {
    lsb_config cfg{};
    double dx = 0, dy = 0;
    std::vector<std::vector<double>> a;  // in kArrayNames order
};

Setup read_setup(const std::string& path) {
    const std::vector<char> b = read_file(path);
    size_t off = 0;
    auto take = [&](void* dst, size_t n) {
        if (off + n > b.size()) die(path + ": truncated set-up file");
        std::memcpy(dst, b.data() + off, n);
        off += n;
    };
    char magic[8];
    take(magic, 8);
    if (std::memcmp(magic, "LSBSETUP", 8) != 0) die(path + ": not a set-up file");
    int32_t version = 0, csize = 0;
    take(&version, 4);
    take(&csize, 4);
    if (version != 1) die(path + ": set-up file version " + std::to_string(version) + " (expected 1)");
    if (csize != (int32_t)sizeof(lsb_config)) die(path + ": lsb_config size differs from this build's");
    Setup s;
    take(&s.cfg, sizeof(lsb_config));
    take(&s.dx, 8);
    take(&s.dy, 8);
    const long long nx = s.cfg.nx, ny = s.cfg.ny, nzp = s.cfg.nz + 1, nzm = s.cfg.nz - 1;
    const long long want[18] = {nx, ny, nzp, nx, ny, nzp * nzp, nzp * nzp, nzm, nzm * nzm, nzm * nzm,
                                nzp, nzp, nzp, nzp, nzp, nzp, nzp, nx};
    for (int i = 0; i < 18; ++i) {
        int64_t n = 0;
        take(&n, 8);
        if (n != want[i])
            die(path + ": array " + kArrayNames[i] + " has " + std::to_string(n) + " values, expected " +
                std::to_string(want[i]));
        std::vector<double> v((size_t)n);
        take(v.data(), (size_t)n * 8);
        s.a.push_back(std::move(v));
    }
    if (off != b.size()) die(path + ": trailing bytes in the set-up file");
    return s;
}

lsb_setup setup_struct(const Setup& s) {
    lsb_setup su{};
    const double* p[18];
    for (int i = 0; i < 18; ++i) p[i] = s.a[i].data();
    su.xpts = p[0]; su.ypts = p[1]; su.zpts = p[2]; su.wavx = p[3]; su.wavy = p[4];
    su.dx = s.dx; su.dy = s.dy;
    su.dz1 = p[5]; su.dz2 = p[6]; su.lam = p[7]; su.e = p[8]; su.ei = p[9];
    su.ubar = p[10]; su.ubarp = p[11]; su.ubarpp = p[12];
    su.hbot = p[13]; su.htop = p[14]; su.d2hbot = p[15]; su.d2htop = p[16]; su.lamx = p[17];
    return su;
}

}  // namespace

namespace {

// ------------------------------------------------------------------ restart and q files
// restart: 9 float32 [isum, t, dt, dt2, dt3, nx, ny, nzp, nxpl], then 20 variables (u, v, w,
// T, uni(1:3), unmi(1:3), nlni(1:3), nlnmi(1:3), tn, tnm, nltn, nltnm) of nx*ny*nzp values
// in (i, j, k) order, k fastest.  Fields here are in the device layout [nzp][ny][nx].
constexpr int kRestartVars = 20;

struct Restart {
    float head[9] = {};
    int nx = 0, ny = 0, nzp = 0;
    std::vector<std::vector<double>> v;  // 20 fields, [nzp][ny][nx]
};

Restart read_restart(const std::string& path, int nx, int ny, int nzp) {
    const std::vector<char> b = read_file(path);
    if (b.size() < 9 * sizeof(float)) die(path + ": no restart header");
    Restart r;
    std::memcpy(r.head, b.data(), sizeof(r.head));
    r.nx = (int)std::lround(r.head[5]);
    r.ny = (int)std::lround(r.head[6]);
    r.nzp = (int)std::lround(r.head[7]);
    if (nx > 0 && (r.nx != nx || r.ny != ny || r.nzp != nzp))  // src/mpi_io.f90:233-242 stops here too
        die(path + ": restart dimensions (" + std::to_string(r.nx) + " " + std::to_string(r.ny) + " " +
            std::to_string(r.nzp) + ") differ from the run's");
    const size_t res = (size_t)r.nx * r.ny * r.nzp;
    if (b.size() < (9 + kRestartVars * res) * sizeof(float)) die(path + ": truncated restart file");
    const float* f = reinterpret_cast<const float*>(b.data()) + 9;
    for (int var = 0; var < kRestartVars; ++var, f += res) {
        std::vector<double> a(res);
        for (int i = 0; i < r.nx; ++i)
            for (int j = 0; j < r.ny; ++j)
                for (int k = 0; k < r.nzp; ++k)
                    a[((size_t)k * r.ny + j) * r.nx + i] = f[((size_t)i * r.ny + j) * r.nzp + k];
        r.v.push_back(std::move(a));
    }
    return r;
}

// the reference's writer stores nlni again in variables 14-16 (src/mpi_io.f90:62); with
// ref_bug that is reproduced, so the file reads back as the reference's files do
void write_restart(const std::string& path, const Restart& r, bool ref_bug) {
    const size_t res = (size_t)r.nx * r.ny * r.nzp;
    std::vector<float> out(9 + kRestartVars * res);
    std::memcpy(out.data(), r.head, sizeof(r.head));
    float* f = out.data() + 9;
    for (int var = 0; var < kRestartVars; ++var, f += res) {
        const std::vector<double>& a = r.v[(ref_bug && var >= 13 && var <= 15) ? var - 3 : var];
        for (int i = 0; i < r.nx; ++i)
            for (int j = 0; j < r.ny; ++j)
                for (int k = 0; k < r.nzp; ++k)
                    f[((size_t)i * r.ny + j) * r.nzp + k] = (float)a[((size_t)k * r.ny + j) * r.nx + i];
    }
    write_file(path, out);
}

// q snapshot: 7 float32 [isum, t, dt, nx, ny, nzp, nypl], then u + ubar, v, w, T + Tbar, p
// of nx*ny*nzp values in (y, z, x) order, x fastest; q holds u + ubar, v, w, p as
// [4][nzp][ny][nx] (lsb_snapshot_async's layout) and T is zero
void write_q(const std::string& path, int isum, double t, double dt, int nx, int ny, int nzp,
             const std::vector<double>& q) {
    const size_t res = (size_t)nx * ny * nzp;
    std::vector<float> out(7 + 5 * res, 0.0f);
    const float head[7] = {(float)isum, (float)t, (float)dt, (float)nx, (float)ny, (float)nzp, (float)ny};
    std::memcpy(out.data(), head, sizeof(head));
    const int src[5] = {0, 1, 2, -1, 3};
    for (int var = 0; var < 5; ++var) {
        if (src[var] < 0) continue;
        const double* a = q.data() + (size_t)src[var] * res;
        float* f = out.data() + 7 + (size_t)var * res;
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nzp; ++k)
                for (int i = 0; i < nx; ++i) f[((size_t)j * nzp + k) * nx + i] = (float)a[((size_t)k * ny + j) * nx + i];
    }
    write_file(path, out);
}

std::string qname(const std::string& dir, int isum) {
    char b[32];
    std::snprintf(b, sizeof(b), "q%05d.dat", isum);
    return dir + "/" + b;
}

}  // namespace

namespace {

int check_setup(const std::string& path) {
    const Setup s = read_setup(path);
    std::printf("nx %d ny %d nz %d precision %d sgsflag %d sgsmodel %d dx %.17g dy %.17g\n", s.cfg.nx, s.cfg.ny,
                s.cfg.nz, s.cfg.precision, s.cfg.sgsflag, s.cfg.sgsmodel, s.dx, s.dy);
    for (int i = 0; i < 18; ++i) {
        double sum = 0.0;
        for (double x : s.a[i]) sum += x;
        std::printf("%s %zu %.17g\n", kArrayNames[i], s.a[i].size(), sum);
    }
    return 0;
}

// restart round trip and a q file whose u, v, w, p are the restart's u, v, w, T fields
int io_selftest(const std::string& start, const std::string& dir) {
    const Restart r = read_restart(start, 0, 0, 0);
    write_restart(dir + "/roundtrip.dat", r, false);
    const size_t res = (size_t)r.nx * r.ny * r.nzp;
    std::vector<double> q(4 * res);
    for (int f = 0; f < 4; ++f) std::copy(r.v[f].begin(), r.v[f].end(), q.begin() + f * res);
    write_q(qname(dir, (int)std::lround(r.head[0])), (int)std::lround(r.head[0]), r.head[1], r.head[2], r.nx, r.ny,
            r.nzp, q);
    return 0;
}

int run(const std::string& setup_path, const std::string& start, int nsteps, int iomod, const std::string& dir,
        bool ref_bug) {
    if (nsteps < 0 || iomod < 1) die("NSTEPS must be >= 0 and IOMOD >= 1");
    const Setup s = read_setup(setup_path);
    const int nx = s.cfg.nx, ny = s.cfg.ny, nzp = s.cfg.nz + 1;
    Restart r = read_restart(start, nx, ny, nzp);
    const lsb_setup su = setup_struct(s);
    lsb_handle* h = nullptr;
    ck(lsb_create(&s.cfg, &su, &h), "lsb_create");
    // the velocity histories come from the file; p and p^(n-1) are not in it and start at
    // zero, as after mpi_read_restart_file
    const size_t res = (size_t)nx * ny * nzp;
    std::vector<double> zero(res, 0.0), hist[4];
    for (int g = 0; g < 4; ++g)
        for (int l = 0; l < 3; ++l) hist[g].insert(hist[g].end(), r.v[4 + 3 * g + l].begin(), r.v[4 + 3 * g + l].end());
    ck(lsb_upload_state(h, r.v[0].data(), r.v[1].data(), r.v[2].data(), zero.data(), zero.data(), hist[0].data(),
                        hist[1].data(), hist[2].data(), hist[3].data(), r.head[1], r.head[2], r.head[3], r.head[4], 0),
       "lsb_upload_state");
    int isum = (int)std::lround(r.head[0]);
    std::vector<double> q(4 * res);
    for (int done = 0; done < nsteps;) {
        const int k = std::min(iomod, nsteps - done);
        ck(lsb_step(h, k), "lsb_step");
        done += k;
        isum += k;
        ck(lsb_snapshot_async(h, q.data()), "lsb_snapshot_async");
        ck(lsb_synchronize(h), "lsb_synchronize");
        lsb_diagnostics dg{};
        ck(lsb_diag(h, &dg), "lsb_diag");
        if (dg.nonfinite) die("NaN in the velocity at step " + std::to_string(isum));
        write_q(qname(dir, isum), isum, dg.t, dg.dt, nx, ny, nzp, q);
        std::printf("step %d t %.6f dt %.6g div %.3e cfl %.3f %.3f %.3f\n", isum, dg.t, dg.dt, dg.divergence,
                    dg.cflx, dg.cfly, dg.cflz);
    }
    // the final state as a restart file (src/main.f90:109-111)
    std::vector<double> u(res), v(res), w(res), p(res), pn(res), st[4];
    for (auto& x : st) x.resize(3 * res);
    double t = 0, dt = 0, dt2 = 0, dt3 = 0;
    int istep = 0;
    ck(lsb_download_state(h, u.data(), v.data(), w.data(), p.data(), pn.data(), st[0].data(), st[1].data(),
                          st[2].data(), st[3].data(), &t, &dt, &dt2, &dt3, &istep),
       "lsb_download_state");
    ck(lsb_destroy(h), "lsb_destroy");
    r.v[0] = u;
    r.v[1] = v;
    r.v[2] = w;
    for (int g = 0; g < 4; ++g)
        for (int l = 0; l < 3; ++l) r.v[4 + 3 * g + l].assign(st[g].begin() + l * res, st[g].begin() + (l + 1) * res);
    r.head[0] = (float)isum;
    r.head[1] = (float)t;
    r.head[2] = (float)dt;
    r.head[3] = (float)dt2;
    r.head[4] = (float)dt3;
    r.head[8] = (float)nx;
    write_restart(dir + "/end.dat", r, ref_bug);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    const std::vector<std::string> a(argv + 1, argv + argc);
    if (a.size() == 2 && a[0] == "--check-setup") return check_setup(a[1]);
    if (a.size() == 3 && a[0] == "--io-selftest") return io_selftest(a[1], a[2]);
    if (a.size() == 5 || (a.size() == 6 && a[5] == "--no-ref-bug"))
        return run(a[0], a[1], std::atoi(a[2].c_str()), std::atoi(a[3].c_str()), a[4], a.size() == 5);
    std::fprintf(stderr,
                 "usage: lsb_run SETUP START NSTEPS IOMOD OUTDIR [--no-ref-bug]\n"
                 "       lsb_run --check-setup SETUP\n"
                 "       lsb_run --io-selftest START OUTDIR\n");
    return 2;
}
