// C++/OpenMP restatement of the reference's time step on the host cores: the timed CPU
// baseline of the benchmark (test infrastructure, not the product: nothing in the library
// links it; the product path is the CUDA library).
//
// It restates, in compiled code with OpenMP threads, the FP64 step that oracle/lsb_oracle.py
// states in NumPy: timestep / navierstokes_update (src/navierstokes.f90:10-90, 1157-1496),
// nlterm_skewsym (:658-855) with the 3/2-rule products of dealiasing_2d_fftw
// (src/dealiasing.f90:262-447; each field padded once, the products summed on the padded
// grid, which the linearity of the map makes the same result), force (:92-211), the ceiling
// dipole of the benchmark's bctype 3, horfft (src/horfft.f90:61-150), norm (:153-224), the
// z derivatives as their dense matrices (src/derivatives.f90:112-188), solve_helmholtz /
// solve_nhom_helmholtz (src/helmholtz.f90:130-358) and the dynamic Smagorinsky model with
// its 3-point test filter (src/sgsterm.f90:123-280, src/filters.f90:363-613).  Scope: the
// configurations of the benchmark's workloads -- dealiasflag 0 or 1 (textbook 3/2 layout),
// sgsflag 0 or 1 with sgsmodel 1, forcing 0/1, bctype 0 or 3, fixed dt, nstart 0.
//
//   cpu_step <setup file> <nx_lg> <ny_lg> <state in> <nsteps> <threads> [state out]
//
// The set-up file is the library's (lsbflow_b200.lib.write_setup_file); the state file holds
// u, v, w spectral [nzp][ny][nx] (float64) and the dt.  It prints one line per run:
// "steps <n> seconds <s> threads <t>" (seconds of the stepping alone).
#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "lsbgpu.h"

namespace {

struct cx {
    double re, im;
};
inline cx operator+(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
inline cx operator-(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
inline cx operator*(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cx operator*(double s, cx a) { return {s * a.re, s * a.im}; }
inline cx conj(cx a) { return {a.re, -a.im}; }

const double PI = 4.0 * std::atan(1.0);

// complex DFT of length n (a product of 2, 3, 4), X[k] = sum_j x[j] exp(sign 2 pi i jk / n),
// by Stockham radix-r decimation in frequency (out of place, natural order at the end)
struct Fft {
    int n = 0;
    std::vector<int> rad;
    std::vector<std::vector<cx>> tw[2];  // per sign, per stage: exp(sign 2 pi i p k / n_s)
    explicit Fft(int n_ = 1) : n(n_) {
        int m = n;
        while (m > 1) {
            if (m % 4 == 0) rad.push_back(4), m /= 4;
            else if (m % 2 == 0) rad.push_back(2), m /= 2;
            else if (m % 3 == 0) rad.push_back(3), m /= 3;
            else throw std::runtime_error("FFT length " + std::to_string(n) + " is not a product of 2 and 3");
        }
        for (int sg = 0; sg < 2; ++sg) {
            const double sign = sg ? 1.0 : -1.0;
            int ns = n;
            for (int r : rad) {
                const int ms = ns / r;
                std::vector<cx> t((size_t)ms * r);
                for (int p = 0; p < ms; ++p)
                    for (int k = 0; k < r; ++k) {
                        const double a = sign * 2.0 * PI * (double)p * k / ns;
                        t[(size_t)p * r + k] = {std::cos(a), std::sin(a)};
                    }
                tw[sg].push_back(std::move(t));
                ns = ms;
            }
        }
    }
    // x: input (overwritten), y: work of n; result in x
    void exec(cx* x, cx* y, int sign) const {
        const int sg = sign > 0 ? 1 : 0;
        int ns = n, s = 1;
        cx* a = x;
        cx* b = y;
        for (size_t st = 0; st < rad.size(); ++st) {
            const int r = rad[st], ms = ns / r;
            const cx* t = tw[sg][st].data();
            if (r == 2) {
                for (int p = 0; p < ms; ++p) {
                    const cx w1 = t[2 * p + 1];
                    for (int q = 0; q < s; ++q) {
                        const cx u0 = a[q + s * p], u1 = a[q + s * (p + ms)];
                        b[q + s * (2 * p)] = u0 + u1;
                        b[q + s * (2 * p + 1)] = (u0 - u1) * w1;
                    }
                }
            } else if (r == 4) {
                const cx jj = {0.0, sign > 0 ? 1.0 : -1.0};  // exp(sign i pi / 2)
                for (int p = 0; p < ms; ++p) {
                    const cx w1 = t[4 * p + 1], w2 = t[4 * p + 2], w3 = t[4 * p + 3];
                    for (int q = 0; q < s; ++q) {
                        const cx u0 = a[q + s * p], u1 = a[q + s * (p + ms)], u2 = a[q + s * (p + 2 * ms)],
                                 u3 = a[q + s * (p + 3 * ms)];
                        const cx s02 = u0 + u2, d02 = u0 - u2, s13 = u1 + u3, d13 = (u1 - u3) * jj;
                        b[q + s * (4 * p)] = s02 + s13;
                        b[q + s * (4 * p + 1)] = (d02 + d13) * w1;
                        b[q + s * (4 * p + 2)] = (s02 - s13) * w2;
                        b[q + s * (4 * p + 3)] = (d02 - d13) * w3;
                    }
                }
            } else {  // 3
                const double c3 = -0.5, s3 = (sign > 0 ? 1.0 : -1.0) * std::sqrt(3.0) / 2.0;
                for (int p = 0; p < ms; ++p) {
                    const cx w1 = t[3 * p + 1], w2 = t[3 * p + 2];
                    for (int q = 0; q < s; ++q) {
                        const cx u0 = a[q + s * p], u1 = a[q + s * (p + ms)], u2 = a[q + s * (p + 2 * ms)];
                        const cx sm = u1 + u2, df = u1 - u2;
                        const cx m1 = u0 + c3 * sm;
                        const cx m2 = {-s3 * df.im, s3 * df.re};
                        b[q + s * (3 * p)] = u0 + sm;
                        b[q + s * (3 * p + 1)] = (m1 + m2) * w1;
                        b[q + s * (3 * p + 2)] = (m1 - m2) * w2;
                    }
                }
            }
            std::swap(a, b);
            ns = ms;
            s *= r;
        }
        if (a != x) std::memcpy(x, a, sizeof(cx) * n);
    }
};

// real transforms of even length nr through a complex FFT of nr / 2
struct RealFft {
    int nr = 0;
    Fft half;
    std::vector<cx> w;  // exp(-2 pi i k / nr)
    explicit RealFft(int nr_ = 2) : nr(nr_), half(nr_ / 2) {
        w.resize(nr / 2 + 1);
        for (int k = 0; k <= nr / 2; ++k) w[k] = {std::cos(-2.0 * PI * k / nr), std::sin(-2.0 * PI * k / nr)};
    }
    // x[nr] real -> X[0 .. nr/2 - 1] (the Nyquist mode dropped), unnormalised; z, y: work of nr/2
    void r2c(const double* x, cx* X, cx* z, cx* y) const {
        const int h = nr / 2;
        for (int m = 0; m < h; ++m) z[m] = {x[2 * m], x[2 * m + 1]};
        half.exec(z, y, -1);
        for (int k = 0; k < h; ++k) {
            const cx zk = z[k], zc = conj(z[(h - k) % h]);
            const cx e = 0.5 * (zk + zc), o = 0.5 * (zk - zc);
            const cx t = w[k] * o;  // -i w o added: X = e - i w o
            X[k] = {e.re + t.im, e.im - t.re};
        }
    }
    // X[0 .. nr/2 - 1] (Nyquist 0; the imaginary part of X[0] ignored) -> x[nr], unnormalised
    void c2r(const cx* X, double* x, cx* z, cx* y) const {
        const int h = nr / 2;
        for (int k = 0; k < h; ++k) {
            cx a = X[k];
            if (k == 0) a.im = 0.0;
            const cx b = (k == 0) ? cx{0.0, 0.0} : conj(X[h - k]);  // conj(X[nr/2 - k]) (Nyquist 0 at k = 0)
            const cx e = a + b, o = (a - b) * conj(w[k]);
            z[k] = {e.re - o.im, e.im + o.re};  // e + i o
        }
        half.exec(z, y, +1);
        for (int m = 0; m < h; ++m) {
            x[2 * m] = z[m].re;
            x[2 * m + 1] = z[m].im;
        }
    }
};

struct Setup {
    lsb_config c{};
    double dx = 0, dy = 0;
    std::vector<double> xpts, ypts, zpts, wavx, wavy, dz1, dz2, lam, e, ei, ubar, ubarp, ubarpp, hbot, htop, d2hbot,
        d2htop, lamx;
};

std::vector<double> read_arr(FILE* f) {
    int64_t n = 0;
    if (std::fread(&n, 8, 1, f) != 1) throw std::runtime_error("set-up file truncated");
    std::vector<double> a((size_t)n);
    if (n && std::fread(a.data(), 8, (size_t)n, f) != (size_t)n) throw std::runtime_error("set-up file truncated");
    return a;
}

Setup read_setup(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    char magic[8];
    int32_t ver = 0, csize = 0;
    Setup s;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "LSBSETUP", 8) != 0) throw std::runtime_error("not a set-up file");
    if (std::fread(&ver, 4, 1, f) != 1 || std::fread(&csize, 4, 1, f) != 1 || csize != (int32_t)sizeof(lsb_config))
        throw std::runtime_error("set-up file: lsb_config size differs");
    if (std::fread(&s.c, sizeof(lsb_config), 1, f) != 1 || std::fread(&s.dx, 8, 1, f) != 1 || std::fread(&s.dy, 8, 1, f) != 1)
        throw std::runtime_error("set-up file truncated");
    std::vector<double>* arrs[] = {&s.xpts, &s.ypts, &s.zpts, &s.wavx, &s.wavy, &s.dz1, &s.dz2, &s.lam, &s.e,
                                   &s.ei, &s.ubar, &s.ubarp, &s.ubarpp, &s.hbot, &s.htop, &s.d2hbot, &s.d2htop,
                                   &s.lamx};
    for (auto* a : arrs) *a = read_arr(f);
    std::fclose(f);
    return s;
}

using Field = std::vector<double>;

struct Solver {
    Setup su;
    int nx, ny, nzp, nzm, nxl, nyl, kx;
    long long S, C, P, Pl;
    RealFft rx, rxl;
    Fft fy, fyl;
    // state
    Field u[3], un[3], unm[3], nl[3], nln[3], nlnm[3], p, pn;
    double t = 0, dt = 0, dt2 = 0, dt3 = 0;
    int istep = 0;
    std::vector<double> delta;  // dynamic model: delta(z) (src/sgsterm.f90:159-164)
    // scratch fields by name, allocated on first use and kept: no allocation inside a step
    mutable std::map<std::string, Field> wsp;
    double* ws(const std::string& name, long long n) const {
        Field& f = wsp[name];
        if ((long long)f.size() != n) f.assign((size_t)n, 0.0);
        return f.data();
    }

    Solver(const Setup& s, int nxl_, int nyl_)
        : su(s), nx(s.c.nx), ny(s.c.ny), nzp(s.c.nz + 1), nzm(s.c.nz - 1), nxl(nxl_), nyl(nyl_), kx(s.c.nx / 2),
          rx(s.c.nx), rxl(nxl_), fy(s.c.ny), fyl(nyl_) {
        S = (long long)nx * ny * nzp;
        C = (long long)nx * ny;
        P = S;
        Pl = (long long)nxl * nyl * nzp;
        for (int l = 0; l < 3; ++l) {
            u[l].assign(S, 0.0), un[l].assign(S, 0.0), unm[l].assign(S, 0.0);
            nl[l].assign(S, 0.0), nln[l].assign(S, 0.0), nlnm[l].assign(S, 0.0);
        }
        p.assign(S, 0.0);
        pn.assign(S, 0.0);
        // delta of the dynamic model (src/sgsterm.f90:159-164)
        const auto& zp = su.zpts;
        delta.resize(nzp);
        for (int k = 0; k < nzp; ++k) {
            double dz = (k == 0) ? zp[0] - zp[1] : (k == nzp - 1) ? zp[nzp - 2] - zp[nzp - 1] : 0.5 * (zp[k - 1] - zp[k + 1]);
            delta[k] = std::pow(su.dx * su.dy * dz, 1.0 / 3.0);
        }
    }

    double w2(long long c) const {
        const int i = (int)(c % nx), j = (int)(c / nx);
        return su.wavx[i] * su.wavx[i] + su.wavy[j] * su.wavy[j];
    }

    // ---------------------------------------------------------------- horfft
    // spectral (padded or not) -> physical [nzp][nyl][nxl]: y c2c backward of every kx column
    // (negative ky to the top rows when padded), x c2r; mode: 0 copy, 1 i kx, 2 i ky; mean added
    void to_phys(const double* spec, double* phys, bool padded, int mode, const double* mean, double scale = 1.0) const {
        const int NX = padded ? nxl : nx, NY = padded ? nyl : ny;
        const RealFft& RX = padded ? rxl : rx;
        const Fft& FY = padded ? fyl : fy;
#pragma omp parallel
        {
            std::vector<cx> plane((size_t)NY * kx), col(NY), wk(NY > NX ? NY : NX), row(NX / 2), z(NX / 2);
#pragma omp for schedule(static)
            for (int k = 0; k < nzp; ++k) {
                const double* sp = spec + (long long)k * C;
                for (int i = 0; i < kx; ++i) {
                    for (int jl = 0; jl < NY; ++jl) col[jl] = {0.0, 0.0};
                    for (int j = 0; j < ny; ++j) {
                        int jl = j;
                        if (padded && j >= ny / 2) jl = NY - ny + j;
                        cx v = {sp[(long long)j * nx + 2 * i], sp[(long long)j * nx + 2 * i + 1]};
                        if (mode == 1) v = {-su.wavx[2 * i] * v.im, su.wavx[2 * i] * v.re};
                        if (mode == 2) v = {-su.wavy[j] * v.im, su.wavy[j] * v.re};
                        col[jl] = v;
                    }
                    FY.exec(col.data(), wk.data(), +1);
                    for (int jl = 0; jl < NY; ++jl) plane[(size_t)jl * kx + i] = col[jl];
                }
                for (int jl = 0; jl < NY; ++jl) {
                    for (int i = 0; i < NX / 2; ++i) row[i] = (i < kx) ? plane[(size_t)jl * kx + i] : cx{0.0, 0.0};
                    double* out = phys + ((long long)k * NY + jl) * NX;
                    RX.c2r(row.data(), out, z.data(), wk.data());
                    const double m = mean ? mean[k] : 0.0;
                    if (scale != 1.0 || mean)
                        for (int i = 0; i < NX; ++i) out[i] = scale * out[i] + m;
                }
            }
        }
    }
    // physical [nzp][NY][NX] -> spectral: x r2c, y c2c forward, / (NX NY), truncated to ny rows
    // and kx modes; out = alpha * T + beta * out
    void to_spec(const double* phys, double* spec, bool padded, double alpha, double beta) const {
        const int NX = padded ? nxl : nx, NY = padded ? nyl : ny;
        const RealFft& RX = padded ? rxl : rx;
        const Fft& FY = padded ? fyl : fy;
        const double sc = 1.0 / ((double)NX * (double)NY);
#pragma omp parallel
        {
            std::vector<cx> plane((size_t)NY * kx), col(NY), wk(NY > NX ? NY : NX), X(NX / 2), z(NX / 2);
#pragma omp for schedule(static)
            for (int k = 0; k < nzp; ++k) {
                for (int jl = 0; jl < NY; ++jl) {
                    RX.r2c(phys + ((long long)k * NY + jl) * NX, X.data(), z.data(), wk.data());
                    for (int i = 0; i < kx; ++i) plane[(size_t)jl * kx + i] = X[i];
                }
                double* sp = spec + (long long)k * C;
                std::vector<cx> tr(ny);
                for (int i = 0; i < kx; ++i) {
                    for (int jl = 0; jl < NY; ++jl) col[jl] = plane[(size_t)jl * kx + i];
                    FY.exec(col.data(), wk.data(), -1);
                    for (int j = 0; j < ny; ++j) {
                        const int jl = (padded && j >= ny / 2) ? NY - ny + j : j;
                        tr[j] = {col[jl].re * sc, col[jl].im * sc};
                    }
                    if (padded && i == 0) {
                        // the truncated kx = 0 column as the reference's round trip through the
                        // unpadded physical grid leaves it: 1/2 (X(ky) + conj X(-ky)) (the ky = -ny/2
                        // row has no partner left after the truncation)
                        std::vector<cx> h(tr);
                        for (int j = 0; j < ny; ++j) tr[j] = 0.5 * (h[j] + conj(h[(ny - j) % ny]));
                    }
                    for (int j = 0; j < ny; ++j) {
                        const long long o = (long long)j * nx + 2 * i;
                        sp[o] = alpha * tr[j].re + (beta != 0.0 ? beta * sp[o] : 0.0);
                        sp[o + 1] = alpha * tr[j].im + (beta != 0.0 ? beta * sp[o + 1] : 0.0);
                    }
                }
            }
        }
    }

    // ---------------------------------------------------------------- z contractions
    // out[r][c] = sum_k A[r][k] in[k + koff][c], r < M (A is M x K row-major)
    void zmat(const double* A, int M, int K, const double* in, int koff, double* out) const {
        const long long CB = 256;
#pragma omp parallel for schedule(static)
        for (long long c0 = 0; c0 < C; c0 += CB) {
            const long long cn = (C - c0 < CB) ? C - c0 : CB;
            for (int r = 0; r < M; ++r) {
                double acc[256];
                for (long long c = 0; c < cn; ++c) acc[c] = 0.0;
                for (int k = 0; k < K; ++k) {
                    const double a = A[(size_t)r * K + k];
                    const double* x = in + (long long)(k + koff) * C + c0;
                    for (long long c = 0; c < cn; ++c) acc[c] += a * x[c];
                }
                double* o = out + (long long)r * C + c0;
                for (long long c = 0; c < cn; ++c) o[c] = acc[c];
            }
        }
    }
    void dfdz(const double* in, double* out) const { zmat(su.dz1.data(), nzp, nzp, in, 0, out); }

    // solve_nhom_helmholtz (bc null: solve_helmholtz) in place on rhs
    void helmholtz(double* rhs, const double* bc, double dtnui) const {
        const double *hb = su.hbot.data(), *ht = su.htop.data(), *d2hb = su.d2hbot.data(), *d2ht = su.d2htop.data();
        if (bc) {
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nzp; ++k)
                for (long long c = 0; c < C; ++c) {
                    const double f = -w2(c) - dtnui;
                    const double abot = d2hb[k] + f * hb[k];
                    double v = rhs[(long long)k * C + c] - abot * bc[(long long)(nzp - 1) * C + c];
                    const double atop = d2ht[k] + f * ht[k];
                    rhs[(long long)k * C + c] = v - atop * bc[c];
                }
        }
        double* tq = ws("helm_t", (long long)nzm * C);
        zmat(su.ei.data(), nzm, nzm, rhs, 1, tq);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < nzm; ++r)
            for (long long c = 0; c < C; ++c) {
                const double dfac = -w2(c) - dtnui;
                tq[(long long)r * C + c] = tq[(long long)r * C + c] / (su.lam[r] + dfac);
            }
        zmat(su.e.data(), nzm, nzm, tq, 0, rhs + C);
#pragma omp parallel for schedule(static)
        for (long long c = 0; c < C; ++c) {
            rhs[c] = 0.0;
            rhs[(long long)(nzp - 1) * C + c] = 0.0;
        }
        if (bc) {
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nzp; ++k)
                for (long long c = 0; c < C; ++c)
                    rhs[(long long)k * C + c] =
                        rhs[(long long)k * C + c] + hb[k] * bc[(long long)(nzp - 1) * C + c] + ht[k] * bc[c];
        }
    }

    // ---------------------------------------------------------------- SGS: dynamic Smagorinsky
    // filter_q_3pt (x, y periodic; z interior planes with the interpolating weights of
    // src/filters.f90:398-443), in -> out
    void filter3(const double* in, double* out, double a, double b, bool interp_z) const {
        const double s = 2.0 * a + b;
        double* qy = ws("filter_y", P);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nzp; ++k)
            for (int j = 0; j < ny; ++j) {
                const double* rowm = in + ((long long)k * ny + (j + ny - 1) % ny) * nx;
                const double* row0 = in + ((long long)k * ny + j) * nx;
                const double* rowp = in + ((long long)k * ny + (j + 1) % ny) * nx;
                double* o = qy + ((long long)k * ny + j) * nx;
                for (int i = 0; i < nx; ++i) {
                    const int im = (i + nx - 1) % nx, ip = (i + 1) % nx;
                    const double hm = (a * rowm[im] + b * rowm[i] + a * rowm[ip]) / s;
                    const double h0 = (a * row0[im] + b * row0[i] + a * row0[ip]) / s;
                    const double hp = (a * rowp[im] + b * rowp[i] + a * rowp[ip]) / s;
                    o[i] = (a * hm + b * h0 + a * hp) / s;
                }
            }
        // z weights of this (a, b): interpolating on the mapped grid (mapping 1 / 2)
        std::vector<double> za(nzp, 0.0), zb(nzp, 0.0), zc(nzp, 0.0);
        const auto& zp = su.zpts;
        for (int k = 1; k < nzp - 1; ++k) {
            const double dltm = zp[k] - zp[k - 1], dltp = zp[k + 1] - zp[k];
            za[k] = a * 2.0 * dltm / (dltp + dltm);
            zb[k] = a * 2.0 * (1.0 - dltm / dltp) + b;
            zc[k] = a * 2.0 * dltm * dltm / (dltp * (dltp + dltm));
        }
        if (su.c.mapping == 1) za[1] = 0.0, zb[1] = 2.0 * a + b, zc[1] = 0.0;
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nzp; ++k) {
            const long long o = (long long)k * C;
            if (k == 0 || k == nzp - 1) {
                for (long long c = 0; c < C; ++c) out[o + c] = qy[o + c];
            } else {
                const double A_ = interp_z ? za[k] : a, B_ = interp_z ? zb[k] : b, C_ = interp_z ? zc[k] : a;
                for (long long c = 0; c < C; ++c)
                    out[o + c] = (A_ * qy[o - C + c] + B_ * qy[o + c] + C_ * qy[o + C + c]) / s;
            }
        }
    }

    // tau_ij (9 fields, [3 l + m]) of the dynamic model from u_i, u_i u_j (6, symmetric order
    // 11 12 13 22 23 33) and du_l/dx_m (9)
    void dynamic(double* const* ui, double* const* uu6, double* const* g9, double* const* tau) const {
        static const int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        const double a = su.c.a, b = su.c.b;
        double *sij[6], *lij[6], *sh[6], *mh[6], *uh[3], *lh[6];
        for (int q = 0; q < 6; ++q) {
            const std::string i = std::to_string(q);
            sij[q] = ws("dyn_s" + i, P), lij[q] = ws("dyn_l" + i, P), sh[q] = ws("dyn_sh" + i, P);
            mh[q] = ws("dyn_mh" + i, P), lh[q] = ws("dyn_lh" + i, P);
        }
        for (int l = 0; l < 3; ++l) uh[l] = ws("dyn_uh" + std::to_string(l), P);
        double *snorm = ws("dyn_sn", P), *num = ws("dyn_num", P), *den = ws("dyn_den", P), *ctot = ws("dyn_ct", P),
               *cdd = ws("dyn_cdd", P);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < P; ++e) {
            const int k = (int)(e / C);
            double s6[6];
            for (int l = 0; l < 3; ++l)
                for (int m = l; m < 3; ++m) s6[sym[l][m]] = 0.5 * (g9[3 * l + m][e] + g9[3 * m + l][e]);
            double sn = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) sn = sn + 2.0 * s6[sym[l][m]] * s6[sym[l][m]];
            sn = std::sqrt(sn);
            snorm[e] = sn;
            for (int q = 0; q < 6; ++q) {
                sij[q][e] = s6[q];
                lij[q][e] = delta[k] * delta[k] * sn * s6[q];
            }
        }
        for (int q = 0; q < 6; ++q) {
            filter3(sij[q], sh[q], a, b, true);
            filter3(lij[q], mh[q], a, b, true);
            filter3(uu6[q], lh[q], a, b, true);
        }
        for (int l = 0; l < 3; ++l) filter3(ui[l], uh[l], a, b, true);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < P; ++e) {
            const int k = (int)(e / C);
            const double cd = 2.0 * delta[k];
            double shn = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) shn = shn + 2.0 * sh[sym[l][m]][e] * sh[sym[l][m]][e];
            shn = std::sqrt(shn);
            double nu_ = 0.0, de = 0.0;
            for (int m = 0; m < 3; ++m)
                for (int l = 0; l < 3; ++l) {
                    const int q = sym[l][m];
                    const double mij = 2.0 * (mh[q][e] - cd * cd * shn * sh[q][e]);
                    const double lv = lh[q][e] - uh[l][e] * uh[m][e];
                    nu_ = nu_ + mij * lv;
                    de = de + mij * mij;
                }
            num[e] = nu_;
            den[e] = de;
        }
        filter3(num, ctot, 1.0, 1.0, true);
        filter3(den, cdd, 1.0, 1.0, true);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < P; ++e) {
            const int k = (int)(e / C);
            double c = ctot[e] / cdd[e];
            if (c < 0.0 || std::isnan(c)) c = 0.0;
            if (c > 0.2 * 0.2) c = 0.2 * 0.2;
            const double nu = c * delta[k] * delta[k] * snorm[e];
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) tau[3 * l + m][e] = -2.0 * nu * sij[sym[l][m]][e];
        }
    }

    // ---------------------------------------------------------------- nlterm_skewsym
    void nlterm(const Field* uin, Field* Nout) {
        const auto& c = su.c;
        const bool dl = c.dealiasflag == 1;
        double* dz[3];
        for (int l = 0; l < 3; ++l) dz[l] = ws("nl_dz" + std::to_string(l), S), dfdz(uin[l].data(), dz[l]);
        // the 12 fields on the (padded) product grid: u_l (+ ubar), du_l/dx, du_l/dy, du_l/dz (+ ubar')
        const long long Q = dl ? Pl : P;
        double *U[3], *D[3][3];
        for (int l = 0; l < 3; ++l) {
            const std::string i = std::to_string(l);
            U[l] = ws("nl_U" + i, Q), to_phys(uin[l].data(), U[l], dl, 0, l == 0 ? su.ubar.data() : nullptr);
            D[l][0] = ws("nl_Dx" + i, Q), to_phys(uin[l].data(), D[l][0], dl, 1, nullptr);
            D[l][1] = ws("nl_Dy" + i, Q), to_phys(uin[l].data(), D[l][1], dl, 2, nullptr);
            D[l][2] = ws("nl_Dz" + i, Q), to_phys(dz[l], D[l][2], dl, 0, l == 0 ? su.ubarp.data() : nullptr);
        }
        // products: N_l = -1/2 u_m d_m u_l, h_lm = 1/2 u_l u_m (6), on that grid
        static const int pl[6] = {0, 0, 0, 1, 1, 2}, pm[6] = {0, 1, 2, 1, 2, 2};
        double *Np[3], *Hp[6];
        for (int l = 0; l < 3; ++l) Np[l] = ws("nl_Np" + std::to_string(l), Q);
        for (int q = 0; q < 6; ++q) Hp[q] = ws("nl_Hp" + std::to_string(q), Q);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < Q; ++e) {
            for (int l = 0; l < 3; ++l)
                Np[l][e] = ((0.0 - 0.5 * (U[0][e] * D[l][0][e])) - 0.5 * (U[1][e] * D[l][1][e])) - 0.5 * (U[2][e] * D[l][2][e]);
            for (int q = 0; q < 6; ++q) Hp[q][e] = 0.5 * (U[pl[q]][e] * U[pm[q]][e]);
        }
        double* H[6];
        for (int l = 0; l < 3; ++l) to_spec(Np[l], Nout[l].data(), dl, 1.0, 0.0);
        for (int q = 0; q < 6; ++q) H[q] = ws("nl_H" + std::to_string(q), S), to_spec(Hp[q], H[q], dl, 1.0, 0.0);
        const bool phys = c.forcing == 1 || c.sgsflag == 1;
        double* ui[3] = {nullptr, nullptr, nullptr};
        if (phys) {
            for (int l = 0; l < 3; ++l)
                ui[l] = ws("nl_ui" + std::to_string(l), P), to_phys(uin[l].data(), ui[l], false, 0, l == 0 ? su.ubar.data() : nullptr);
        }
        if (c.forcing == 1) {  // lambda(x) (ubar - u), -lambda v, -lambda w added to N
            double* f = ws("nl_f", P);
            for (int l = 0; l < 3; ++l) {
                const double* q = ui[l];
#pragma omp parallel for schedule(static)
                for (long long e = 0; e < P; ++e) {
                    const int k = (int)(e / C), i = (int)(e % nx);
                    const double ub = (l == 0) ? su.ubar[k] : 0.0;
                    f[e] = su.lamx[i] * (ub - q[e]);
                }
                to_spec(f, Nout[l].data(), false, 1.0, 1.0);
            }
        }
        if (c.sgsflag == 1) {
            double *g9[9], *uu6[6], *tau[9];
            for (int l = 0; l < 3; ++l) {
                const std::string i = std::to_string(l);
                g9[3 * l + 0] = ws("nl_g0" + i, P), to_phys(uin[l].data(), g9[3 * l + 0], false, 1, nullptr);
                g9[3 * l + 1] = ws("nl_g1" + i, P), to_phys(uin[l].data(), g9[3 * l + 1], false, 2, nullptr);
                g9[3 * l + 2] = ws("nl_g2" + i, P), to_phys(dz[l], g9[3 * l + 2], false, 0, l == 0 ? su.ubarp.data() : nullptr);
            }
            for (int q = 0; q < 6; ++q) uu6[q] = ws("nl_uu" + std::to_string(q), P);
            if (dl) {  // the dealiased products on the unpadded grid: u_i u_j = 2 h_ij
                for (int q = 0; q < 6; ++q) to_phys(H[q], uu6[q], false, 0, nullptr, 2.0);
            } else {   // the plain products of the unpadded fields
                for (int q = 0; q < 6; ++q) {
                    double* o = uu6[q];
                    const double *a = ui[pl[q]], *b = ui[pm[q]];
#pragma omp parallel for schedule(static)
                    for (long long e = 0; e < P; ++e) o[e] = a[e] * b[e];
                }
            }
            for (int q = 0; q < 9; ++q) tau[q] = ws("nl_tau" + std::to_string(q), P);
            dynamic(ui, uu6, g9, tau);
            for (int q = 0; q < 6; ++q) to_spec(tau[3 * pl[q] + pm[q]], H[q], false, 1.0, 1.0);
        }
        // N_l -= d h_l1/dx + d h_l2/dy + d h_l3/dz
        static const int hq[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        double* dzh = ws("nl_dzh", S);
        for (int l = 0; l < 3; ++l) {
            dfdz(H[hq[l][2]], dzh);
            const double* hx = H[hq[l][0]];
            const double* hy = H[hq[l][1]];
            double* N = Nout[l].data();
#pragma omp parallel for schedule(static)
            for (long long e = 0; e < S / 2; ++e) {
                const long long c_ = (2 * e) % C;
                const int i = (int)(c_ % nx), j = (int)(c_ / nx);
                const double wx = su.wavx[i], wy = su.wavy[j];
                const long long re = 2 * e, im = 2 * e + 1;
                const double dxr = -wx * hx[im], dxi = wx * hx[re];
                const double dyr = -wy * hy[im], dyi = wy * hy[re];
                N[re] = ((N[re] - dxr) - dyr) - dzh[re];
                N[im] = ((N[im] - dxi) - dyi) - dzh[im];
            }
        }
    }

    // ---------------------------------------------------------------- bound (bctype 3)
    Field bshape;  // spectral ceiling plane of the dipole (C)
    void make_bshape() {
        const auto& c = su.c;
        bshape.assign(C, 0.0);
        if (c.bctype != 3) return;
        Field ph((size_t)P, 0.0);
        const double xc = su.xpts[0] + c.bc3_xc;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double e = (su.xpts[i] - xc) / c.bc3_s;
                ph[(long long)j * nx + i] = c.bc3_amp * e * std::exp(-e * e);
            }
        Field sp((size_t)S, 0.0);
        to_spec(ph.data(), sp.data(), false, 1.0, 0.0);
        std::copy(sp.begin(), sp.begin() + C, bshape.begin());
    }

    void norm(double* f) const {
        const int nyh = ny / 2;
        for (int k = 0; k < nzp; ++k) {
            double* q = f + (long long)k * C;
            q[1] = 0.0;
            if (ny > 2) {
                for (int j = 2; j <= nyh; ++j) {
                    const int jp = ny + 2 - j;
                    q[(j - 1) * nx + 0] = 0.5 * (q[(j - 1) * nx + 0] + q[(jp - 1) * nx + 0]);
                    q[(j - 1) * nx + 1] = 0.5 * (q[(j - 1) * nx + 1] - q[(jp - 1) * nx + 1]);
                }
                for (int j = 2; j <= nyh; ++j) {
                    const int jp = ny + 2 - j;
                    q[(jp - 1) * nx + 0] = q[(j - 1) * nx + 0];
                    q[(jp - 1) * nx + 1] = -q[(j - 1) * nx + 1];
                }
                for (int i = 0; i < nx; ++i) q[nyh * nx + i] = 0.0;
            }
        }
    }

    // ---------------------------------------------------------------- the step
    void step() {
        const auto& c = su.c;
        istep += 1;
        double ab[3], bdf[3], bdfv;
        if (istep == 1) ab[0] = 1, ab[1] = 0, ab[2] = 0, bdf[0] = 1, bdf[1] = 0, bdf[2] = 0, bdfv = 1.0;
        else if (istep == 2) ab[0] = 2, ab[1] = -1, ab[2] = 0, bdf[0] = 2, bdf[1] = -0.5, bdf[2] = 0, bdfv = 2.0 / 3.0;
        else ab[0] = 3, ab[1] = -3, ab[2] = 1, bdf[0] = 3, bdf[1] = -1.5, bdf[2] = 1.0 / 3.0, bdfv = 6.0 / 11.0;
        Field* N = nl;  // the new nonlinear term (rotated into the history below)
        nlterm(u, N);
        const double dtnui = 1.0 / (c.xnu * dt);
        double* rhs[3];
        for (int l = 0; l < 3; ++l) {
            rhs[l] = ws("st_rhs" + std::to_string(l), S);
#pragma omp parallel for schedule(static)
            for (long long e = 0; e < S; ++e) {
                const double nlt = ab[0] * N[l][e] + ab[1] * nln[l][e] + ab[2] * nlnm[l][e];
                rhs[l][e] = -dtnui * (dt * nlt + bdf[0] * u[l][e] + bdf[1] * un[l][e] + bdf[2] * unm[l][e]);
            }
        }
        // the mean-flow diffusion term: - horfft(ubar'') in the (0, 0) mode
        {
            double any = 0.0;
            for (int k = 0; k < nzp; ++k) any += std::fabs(su.ubarpp[k]);
            if (any > 0.0)
                for (int k = 0; k < nzp; ++k) rhs[0][(long long)k * C] -= su.ubarpp[k];
        }
        for (int l = 0; l < 3; ++l) {  // N^{n-2} <- N^{n-1} <- N^n, u^{n-2} <- u^{n-1} <- u^n
            nlnm[l].swap(nln[l]);
            nln[l].swap(nl[l]);
            unm[l].swap(un[l]);
            un[l].swap(u[l]);
        }
        double pf0 = 2.0, pf1 = -1.0;
        if (istep == 1) pf0 = 0.0, pf1 = 0.0;
        else if (istep == 2) pf0 = 1.0, pf1 = 0.0;
        // boundary fields: bc[l] holds the ceiling (plane 0) and wall (plane nzp - 1) values
        double* bc[3];
        double* d2w = ws("st_d2w", 2 * C);
        for (int l = 0; l < 3; ++l) {
            bc[l] = ws("st_bc" + std::to_string(l), S);
            std::fill(bc[l], bc[l] + S, 0.0);
        }
        {
            const double* w = un[2].data();
#pragma omp parallel for schedule(static)
            for (long long cc = 0; cc < C; ++cc) {
                double t0 = 0.0, t1 = 0.0;
                for (int k = 0; k < nzp; ++k) {
                    t0 += su.dz2[k] * w[(long long)k * C + cc];
                    t1 += su.dz2[(size_t)(nzp - 1) * nzp + k] * w[(long long)k * C + cc];
                }
                d2w[cc] = t0;
                d2w[C + cc] = t1;
            }
        }
        const bool active = c.bctype > 0 && t >= c.istartbound;
        const long long W = (long long)(nzp - 1) * C;
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < C / 2; ++e) {
            const long long re = 2 * e, im = 2 * e + 1;
            const double wx = su.wavx[re % nx], wy = su.wavy[re / nx];
            const double wsq = wx * wx + wy * wy;
            const double psr = pf0 * p[W + re] + pf1 * pn[W + re], psi = pf0 * p[W + im] + pf1 * pn[W + im];
            const double dtb = dt * bdfv;
            bc[0][W + re] = dtb * (-wx * psi), bc[0][W + im] = dtb * (wx * psr);
            bc[1][W + re] = dtb * (-wy * psi), bc[1][W + im] = dtb * (wy * psr);
            if (c.bctype == 3 && c.bc3_top == 1) {
                bc[0][re] = bc[0][im] = bc[1][re] = bc[1][im] = 0.0;
            } else {
                bc[0][re] = -rhs[0][re] / (wsq + dtnui / bdfv), bc[0][im] = -rhs[0][im] / (wsq + dtnui / bdfv);
                bc[1][re] = -rhs[1][re] / (wsq + dtnui / bdfv), bc[1][im] = -rhs[1][im] / (wsq + dtnui / bdfv);
            }
            const double zh = c.xnu * dt * bdfv;
            if (active) {
                bc[2][re] = bshape[re] + zh * d2w[re], bc[2][im] = bshape[im] + zh * d2w[im];
            } else {
                bc[2][re] = zh * d2w[re], bc[2][im] = zh * d2w[im];
                bc[2][W + re] = zh * d2w[C + re], bc[2][W + im] = zh * d2w[C + im];
            }
        }
        for (int l = 0; l < 3; ++l) helmholtz(rhs[l], (active || c.forcing == 1) ? bc[l] : nullptr, dtnui / bdfv);
        // pressure: Poisson for w, then phi = -(Dw + div)/(k^2 dt bdfv) and the projection
        double *du = ws("st_du", S), *dv = ws("st_dv", S), *divdz = ws("st_divdz", S), *divf = ws("st_divf", S),
               *r3 = ws("st_r3", S), *bcp = ws("st_bcp", S);
        std::fill(bcp, bcp + S, 0.0);
        dfdz(rhs[0], du);
        dfdz(rhs[1], dv);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < S / 2; ++e) {
            const long long re = 2 * e, im = 2 * e + 1, c_ = re % C;
            const double wx = su.wavx[c_ % nx], wy = su.wavy[c_ / nx];
            divdz[re] = -wx * du[im] - wy * dv[im], divdz[im] = wx * du[re] + wy * dv[re];
            divf[re] = -wx * rhs[0][im] - wy * rhs[1][im], divf[im] = wx * rhs[0][re] + wy * rhs[1][re];
            r3[re] = -divdz[re] - (wx * wx + wy * wy) * rhs[2][re];
            r3[im] = -divdz[im] - (wx * wx + wy * wy) * rhs[2][im];
        }
        if (active)
            for (long long cc = 0; cc < C; ++cc) bcp[cc] = bshape[cc];
        helmholtz(r3, bcp, 0.0);
        double* dw = ws("st_dw", S);
        dfdz(r3, dw);
        pn.swap(p);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < S / 2; ++e) {
            const long long re = 2 * e, im = 2 * e + 1, c_ = re % C;
            const double wx = su.wavx[c_ % nx], wy = su.wavy[c_ / nx];
            const double k2 = wx * wx + wy * wy;
            double pr = 0.0, pi = 0.0;
            if (k2 != 0.0) {
                pr = -(dw[re] + divf[re]) / (k2 * dt * bdfv);
                pi = -(dw[im] + divf[im]) / (k2 * dt * bdfv);
            }
            p[re] = pr, p[im] = pi;
            u[0][re] = rhs[0][re] - dt * bdfv * (-wx * pi), u[0][im] = rhs[0][im] - dt * bdfv * (wx * pr);
            u[1][re] = rhs[1][re] - dt * bdfv * (-wy * pi), u[1][im] = rhs[1][im] - dt * bdfv * (wy * pr);
            u[2][re] = r3[re], u[2][im] = r3[im];
        }
        for (int l = 0; l < 3; ++l) norm(u[l].data());
        t = t + dt;
        dt3 = dt2;
        dt2 = dt;
    }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 7) {
        std::fprintf(stderr, "usage: cpu_step <setup> <nx_lg> <ny_lg> <state in> <nsteps> <threads> [state out]\n");
        return 2;
    }
    try {
        const Setup su = read_setup(argv[1]);
        omp_set_num_threads(std::atoi(argv[6]));
        Solver s(su, std::atoi(argv[2]), std::atoi(argv[3]));
        FILE* f = std::fopen(argv[4], "rb");
        if (!f) throw std::runtime_error("cannot open the state file");
        for (int l = 0; l < 3; ++l)
            if (std::fread(s.u[l].data(), 8, (size_t)s.S, f) != (size_t)s.S) throw std::runtime_error("state file truncated");
        if (std::fread(&s.dt, 8, 1, f) != 1) throw std::runtime_error("state file truncated");
        std::fclose(f);
        s.dt2 = s.dt3 = s.dt;
        s.make_bshape();
        const int nsteps = std::atoi(argv[5]);
        const auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < nsteps; ++i) s.step();
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("steps %d seconds %.6f threads %d\n", nsteps, sec, omp_get_max_threads());
        if (argc > 7) {
            FILE* o = std::fopen(argv[7], "wb");
            if (!o) throw std::runtime_error("cannot write the state file");
            for (int l = 0; l < 3; ++l) std::fwrite(s.u[l].data(), 8, (size_t)s.S, o);
            std::fwrite(s.p.data(), 8, (size_t)s.S, o);
            std::fclose(o);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "cpu_step: %s\n", e.what());
        return 1;
    }
    return 0;
}
