// C ABI and step orchestration of the LSBFLOW B200 library (include/lsbgpu.h).
//
// lsb_step() is timestep() / navierstokes_update() (src/navierstokes.f90:10-90, 1157-1496)
// as a fixed sequence of kernels on one stream, with the histories (u^{n-1}, u^{n-2},
// N^{n-1}, N^{n-2}, p^{n-1}) kept resident as rotating buffers: no copies between steps.
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "lsb_internal.cuh"
#include "lsb_spectral.cuh"
#include "lsb_handle.cuh"

using namespace lsb;

namespace {

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
    try {
        f();
        return LSB_OK;
    } catch (const LsbError& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return LSB_ERR_STATE;
    }
}

void fail(int code, const std::string& m) { throw LsbError{code, m}; }

bool factor(int n, std::vector<int>& rad) {
    rad.clear();
    while (n % 4 == 0 && n > 1) { rad.push_back(4); n /= 4; }
    while (n % 2 == 0 && n > 1) { rad.push_back(2); n /= 2; }
    for (int r : {3, 5, 7}) while (n % r == 0 && n > 1) { rad.push_back(r); n /= r; }
    return n == 1;
}

}  // namespace

namespace {

// single-precision copy of a table (the mixed-precision kernels read their twiddles in FP32)
const float2* upload_f32(lsb_handle* h, const std::vector<double>& v) {
    std::vector<float> f(v.size() + 1);  // +1 keeps the byte count a whole number of doubles
    for (size_t i = 0; i < v.size(); ++i) f[i] = (float)v[i];
    return (const float2*)h->upload((const double*)f.data(), (f.size() * sizeof(float) + 7) / 8);
}

// max_g: the widest lane group the warp-group split may use (fewer lanes and more registers
// per lane mean fewer shuffle stages per element; the register product rows need 32; the
// spanwise passes use 16, which fills their 16-column tiles in one round of 8 warps)
void make_plan(lsb_handle* h, int n, FftPlan& P, int max_g = 32) {
    std::vector<int> rad;
    if (!factor(n, rad) || (int)rad.size() > kMaxStages)
        fail(LSB_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " is not a product of 2,3,5,7");
    P.n = n;
    P.nst = (int)rad.size();
    auto fd = [](uint32_t d) {
        FastDiv f;
        f.d = d;
        if (d > 1) {
            uint32_t s = 0;
            while ((1ull << s) < d) ++s;
            f.s = s;
            f.m = (uint32_t)((((1ull << s) - d) << 32) / d + 1);
        }
        return f;
    };
    int pp = 1;
    for (int i = 0; i < P.nst; ++i) {
        P.radix[i] = rad[i];
        P.p[i] = pp;
        P.fdT[i] = fd((uint32_t)(n / rad[i]));
        P.fdP[i] = fd((uint32_t)pp);
        pp *= rad[i];
    }
    std::vector<double> tw(2 * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < n; ++m) {
        const long double a = 2.0L * pi * (long double)m / (long double)n;
        tw[2 * m] = (double)cosl(a);
        tw[2 * m + 1] = (double)-sinl(a);
    }
    P.tw = (const double2*)h->upload(tw.data(), tw.size());
    P.twf = upload_f32(h, tw);
    // register two-pass split: n = n1 * n2 with both factors in {1,2,3,4,6,8,12,16}
    static const int pairs[][2] = {{2, 1},  {3, 1},  {4, 1},  {6, 1},  {8, 1},   {12, 1},  {16, 1},
                                   {3, 3},  {6, 3},  {8, 3},  {8, 4},  {12, 3},  {8, 6},   {16, 3},
                                   {8, 8},  {12, 6}, {12, 8}, {16, 6}, {12, 12}, {16, 8},  {16, 12},
                                   {16, 16}};
    P.n1 = P.n2 = 0;
    for (auto& pr : pairs)
        if (pr[0] * pr[1] == n) {
            P.n1 = pr[0];
            P.n2 = pr[1];
            break;
        }
    int ls = n + 1;
    if (P.n1 > 0 && P.n2 > 1) {
        const int pb = (P.n2 % 2 == 0) ? P.n2 + 1 : P.n2;
        ls = std::max(ls, P.n1 * pb);
    }
    if (ls % 2 == 0) ++ls;
    P.ls = ls;
    // warp-group split: g = the largest power of two <= max_g dividing n, widened (up to 32)
    // until r = n / g is in {1,2,3,4,6,8}
    P.g = P.r = P.lgg = 0;
    {
        int gg = 1;
        while (gg < max_g && n % (gg * 2) == 0) gg *= 2;
        auto ok = [](int r) { return r == 1 || r == 2 || r == 3 || r == 4 || r == 6 || r == 8; };
        while (!ok(n / gg) && gg < 32 && n % (gg * 2) == 0) gg *= 2;
        const int rr = n / gg;
        if (n % gg == 0 && ok(rr)) {
            P.g = gg;
            P.r = rr;
            int lg = 0;
            while ((1 << lg) < gg) ++lg;
            P.lgg = lg;
        }
    }
}

void make_real_plan(lsb_handle* h, int nr, RealPlan& R, int max_g = 32) {
    if (nr % 2) fail(LSB_ERR_UNSUPPORTED, "real transform length must be even");
    R.nr = nr;
    make_plan(h, nr / 2, R.half, max_g);
    std::vector<double> tw(2 * (size_t)nr);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < nr; ++m) {
        const long double a = 2.0L * pi * (long double)m / (long double)nr;
        tw[2 * m] = (double)cosl(a);
        tw[2 * m + 1] = (double)-sinl(a);
    }
    R.twr = (const double2*)h->upload(tw.data(), tw.size());
    R.twrf = upload_f32(h, tw);
}

Mat make_mat(lsb_handle* h, const double* A, int M, int K, int row0 = 0, int nrows = -1, int zero_pad_rows_top = 0,
             int total_rows = -1) {
    // builds a zero-padded [Mp][Kp] copy of rows row0..row0+nrows-1 of A (M x K, row-major),
    // optionally placed starting at output row zero_pad_rows_top inside total_rows rows
    if (nrows < 0) nrows = M;
    if (total_rows < 0) total_rows = nrows;
    Mat m;
    m.M = total_rows;
    m.K = K;
    m.Mp = ((total_rows + 15) / 16) * 16;  // m16 row tiles of the FP64 MMA
    m.Kp = ((K + 15) / 16) * 16;
    if (m.Mp > 144) fail(LSB_ERR_UNSUPPORTED, "nz too large (nzp <= 144 supported)");
    std::vector<double> buf((size_t)m.Mp * m.Kp, 0.0);
    for (int r = 0; r < nrows; ++r)
        for (int k = 0; k < K; ++k) buf[(size_t)(r + zero_pad_rows_top) * m.Kp + k] = A[(size_t)(row0 + r) * K + k];
    m.p = h->upload(buf.data(), buf.size());
    return m;
}

GemmArgs gemm_base(lsb_handle* h, const Mat& m) {
    GemmArgs g{};
    g.A = m.p;
    g.M = m.M;
    g.K = m.K;
    g.Mp = m.Mp;
    g.Kp = m.Kp;
    g.C = h->d.C();
    g.nfields = 1;
    g.wavx = h->wavx;
    g.wavy = h->wavy;
    g.nx = h->d.nx;
    g.in_fstride = g.out_fstride = h->d.S();
    g.alpha = 1.0;
    g.hb = h->hb;
    g.ht = h->ht;
    g.d2hb = h->d2hb;
    g.d2ht = h->d2ht;
    g.nw = h->sched.gemm_warps;
    return g;
}

// a matrix's int8 digits for the mixed form's tensor-core contractions, on the device (an
// empty OzMat when the sizes do not apply: those contractions stay FP64)
OzMat upload_ozaki(lsb_handle* h, const double* A, int M, int K, int S) {
    OzHost oh;
    if (!make_ozaki_mat(A, M, K, S, oh)) return OzMat{};
    OzMat om = oh.mat;
    om.img = reinterpret_cast<const uint8_t*>(
        h->upload(reinterpret_cast<const double*>(oh.img.data()), (oh.img.size() + 7) / 8));
    om.rscale = h->upload(oh.rscale.data(), oh.rscale.size());
    if (!oh.arow.empty()) om.arow = h->upload(oh.arow.data(), oh.arow.size());
    if (!oh.acol.empty()) om.acol = h->upload(oh.acol.data(), oh.acol.size());
    return om;
}

// a z contraction: on the int8 tensor cores in the mixed form when the matrix has digits
// there, else the FP64 tensor-core MMA
void contract(lsb_handle* h, const GemmArgs& g, const OzMat& om) {
    if (h->cfg.precision == 1 && om.img && launch_ozaki(g, om, h->uerr, h->stream)) return;
    launch_gemm(g, h->stream);
}

}  // namespace

namespace lsb {
// out = Mz . in   (dfdz when mz = dz1, d2fdz2 when dz2), nf fields of stride S
void zgemm(lsb_handle* h, const Mat& m, const double* in, double* out, int nf, int epi, double alpha, double beta,
           const double* aux) {
    GemmArgs g = gemm_base(h, m);
    g.in = in;
    g.out = out;
    g.nfields = nf;
    g.epi = epi;
    g.alpha = alpha;
    g.beta = beta;
    g.aux = aux;
    launch_gemm(g, h->stream);
}
}  // namespace lsb

namespace {
void zgemm1(lsb_handle* h, const Mat& m, const double* in, double* out, int nf) {
    zgemm(h, m, in, out, nf, EPI_STORE, 1.0, 0.0, nullptr);
}

// Helmholtz / Poisson solve of nf fields (stride S): out = solve(rhs, sigma) with the
// lifting functions of solve_nhom_helmholtz when bc != null (bc: [nf][2][C], ceiling first).
// tc: the mixed form's int8 tensor-core contractions where the handle has them (the
// velocity solves); the Poisson solve keeps FP64 contractions in both forms, because the
// pressure -(Dw + div)/(k^2 dt bdfv) is a near-cancellation that turns their error into
// pressure error a thousandfold and more.
void helmholtz(lsb_handle* h, const double* rhs, double* out, int nf, double sigma, const double* bc,
               bool tc = true) {
    const long long C = h->d.C();
    GemmArgs g1 = gemm_base(h, h->m_ei);
    g1.in = rhs;
    g1.koff = 1;
    g1.out = h->T;
    g1.nfields = nf;
    g1.epi = EPI_HELM_SCALE;
    g1.sigma = sigma;
    g1.lam = h->lam;
    if (bc) {
        g1.bcb = bc + C;
        g1.bct = bc;
        g1.bc_fstride = 2 * C;
        g1.lift_sigma = sigma;
    }
    GemmArgs g2 = gemm_base(h, h->m_eext);
    g2.in = h->T;
    g2.out = out;
    g2.nfields = nf;
    g2.epi = EPI_LIFT_ADD;
    if (bc) {
        g2.bcb = bc + C;
        g2.bct = bc;
        g2.bc_fstride = 2 * C;
    }
    // both contractions on the FP64 tensor cores: one launch, the intermediate in registers
    const bool fp64 = !(h->cfg.precision == 1 && tc);
    if (fp64 && launch_helm_fused(g1, g2, h->stream)) return;
    contract(h, g1, tc ? h->oz_ei : OzMat{});
    contract(h, g2, tc ? h->oz_eext : OzMat{});
}

// the built-in staging of the FP64 spanwise passes (y_staging 0): TMA tile loads on the padded
// grid (measured at 256x64x129: forward 128.5 -> 117.0 us, inverse 125 -> 122 us for 9
// fields), cp.async on the unpadded one (no gain measured: its transform's write-back meets
// 4-way bank conflicts under the TMA's swizzle)

YPassArgs ypass(lsb_handle* h, bool padded, int nzp) {
    YPassArgs a{};
    a.ny = h->d.ny;
    a.nyl = padded ? h->d.nyl : h->d.ny;
    a.kxc = h->d.kx;
    a.nzp = nzp;
    a.nx = h->d.nx;
    a.layout = h->cfg.dealias_layout;
    a.scale = 1.0 / ((double)(padded ? h->d.nxl : h->d.nx) * (double)(padded ? h->d.nyl : h->d.ny));
    a.wavy = h->wavy;
    a.wavx = h->wavx;
    a.plan = padded ? h->pyl : h->py;
    a.y_tma = (h->sched.y_staging == 2 || (h->sched.y_staging == 0 && padded && a.nyl != a.ny)) ? 1 : 0;
    a.err = h->uerr;
    return a;
}

RowArgs rowargs(lsb_handle* h, bool padded, int nzp) {
    RowArgs r{};
    r.kxc = h->d.kx;
    r.nxl = padded ? h->d.nxl : h->d.nx;
    r.nyl = padded ? h->d.nyl : h->d.ny;
    r.nzp = nzp;
    r.row_pitch = r.nxl;
    r.wavx = h->wavx;
    r.rp = padded ? h->rxl : h->rx;
    return r;
}

}  // namespace

namespace lsb {
// horfft(-1): physical (unpadded, [nzp][ny][nx]) -> spectral, nf fields
void phys_to_spec(lsb_handle* h, const double* const* phys, double* const* spec, int nf, int nzp, double alpha,
                  double beta, double* const* ybuf, bool f32, const double* lam, const double* const* lmeans,
                  int nlam, const TauRowArgs* tau) {
    if (tau && (nf > kMaxJobs || nf < 6)) fail(LSB_ERR_STATE, "fused stress pass: 6..12 fields in one batch");
    for (int f0 = 0; f0 < nf; f0 += kMaxJobs) {
        const int n = std::min(kMaxJobs, nf - f0);
        RowJobList rj{};
        YFwdJobList yj{};
        rj.n = yj.n = n;
        for (int i = 0; i < n; ++i) {
            double* y = ybuf ? ybuf[f0 + i] : h->Yu + (long long)i * h->Yu1;
            rj.j[i] = RowIO{phys[f0 + i], y, YM_COPY, 0.0, nullptr, 1.0, nullptr};
            if (f0 + i < nlam) {
                const double* m = lmeans ? lmeans[f0 + i] : nullptr;
                rj.j[i].lam = lam;
                rj.j[i].mean = m;
                rj.j[i].add_mean = m ? 1.0 : 0.0;
            }
            yj.j[i] = YFwdJob{y, spec[f0 + i], alpha, beta, 0};
        }
        RowArgs ra = rowargs(h, false, nzp);
        YPassArgs ya = ypass(h, false, nzp);
        ra.f32 = ya.f32 = f32 ? 1 : 0;
        if (tau) {
            // the plain rows first, then the stresses from S_ij and the filtered contractions
            rj.n = n - 6;
            if (rj.n > 0) launch_row_r2c(rj, ra, h->stream);
            TauRowArgs t = *tau;
            t.r = ra;
            for (int q = 0; q < 6; ++q) t.out[q] = const_cast<double*>(yj.j[n - 6 + q].in);
            launch_row_r2c_tau(t, h->stream);
        } else {
            launch_row_r2c(rj, ra, h->stream);
        }
        launch_yfwd(yj, ya, h->stream);
    }
}

// horfft(+1): spectral -> physical (unpadded), optional mean added to field 0
void spec_to_phys(lsb_handle* h, const double* const* spec, double* const* phys, int nf, int nzp,
                  const double* const* means, const int* modes, bool f32, double scale) {
    for (int f0 = 0; f0 < nf; f0 += kMaxJobs) {
        const int n = std::min(kMaxJobs, nf - f0);
        YInvJobList yj{};
        RowJobList rj{};
        yj.n = 0;
        rj.n = n;
        for (int i = 0; i < n; ++i) {
            const int mode = modes ? modes[f0 + i] : YM_COPY;
            const int ymode = mode == YM_IKY ? YM_IKY : YM_COPY;
            // u and du/dx share one spanwise transform (ikx is applied in the row pass)
            int yi = -1;
            for (int j = 0; j < yj.n; ++j)
                if (yj.j[j].in == spec[f0 + i] && yj.j[j].mode == ymode) yi = j;
            if (yi < 0) {
                yi = yj.n++;
                yj.j[yi] = YInvJob{spec[f0 + i], h->Yu + (long long)yi * h->Yu1, ymode};
            }
            const double* mean = means ? means[f0 + i] : nullptr;
            rj.j[i] = RowIO{yj.j[yi].out, phys[f0 + i], mode == YM_IKX ? YM_IKX : YM_COPY, mean ? 1.0 : 0.0, mean, scale};
        }
        RowArgs ra = rowargs(h, false, nzp);
        YPassArgs ya = ypass(h, false, nzp);
        ra.f32 = ya.f32 = f32 ? 1 : 0;
        launch_yinv(yj, ya, h->stream);
        launch_row_c2r(rj, ra, h->stream);
    }
}

}  // namespace lsb

namespace {
double* Hsym(lsb_handle* h, int l, int m) {
    static const int idx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    return h->H + (long long)idx[l][m] * h->d.S();
}

// nlterm_skewsym (src/navierstokes.f90:658-855), velocity part: uin (3S) -> Nout (3S)
void nlterm(lsb_handle* h, const double* uin, double* Nout) {
    const Dims& d = h->d;
    const long long S = d.S();
    const bool dealias = h->cfg.dealiasflag == 1;
    // du_l/dz
    {
        TimerScope ts(h, "gemm_dz");
        GemmArgs g = gemm_base(h, h->m_dz1);
        g.in = uin;
        g.out = h->dz;
        g.nfields = 3;
        g.epi = EPI_STORE;
        contract(h, g, h->oz_dz1);
    }
    // spanwise inverse: u_l, du_l/dy, du_l/dz  -> Y[0..8]
    YInvJobList yj{};
    yj.n = 9;
    for (int l = 0; l < 3; ++l) {
        yj.j[l] = YInvJob{uin + l * S, h->Y + (long long)l * h->Yl, YM_COPY};
        yj.j[3 + l] = YInvJob{uin + l * S, h->Y + (long long)(3 + l) * h->Yl, YM_IKY};
        yj.j[6 + l] = YInvJob{h->dz + l * S, h->Y + (long long)(6 + l) * h->Yl, YM_COPY};
    }
    const int f32 = h->cfg.precision == 1 ? 1 : 0;  // the physical (unpadded) fields
    const int f32nl = (f32 && h->nl_f32) ? 1 : 0;     // the padded product passes
    YPassArgs ya = ypass(h, dealias, d.nzp);
    ya.f32 = f32nl;
    { TimerScope ts(h, "yinv_nl"); launch_yinv(yj, ya, h->stream); }
    NlRowArgs na{};
    na.r = rowargs(h, dealias, d.nzp);
    na.r.f32 = f32nl;
    for (int l = 0; l < 3; ++l) {
        na.U[l] = h->Y + (long long)l * h->Yl;
        na.DY[l] = h->Y + (long long)(3 + l) * h->Yl;
        na.DZ[l] = h->Y + (long long)(6 + l) * h->Yl;
        na.N[l] = h->Y + (long long)(9 + l) * h->Yl;
    }
    for (int m = 0; m < 6; ++m) na.H[m] = h->Y + (long long)(12 + m) * h->Yl;
    na.ubar = h->ubar;
    na.ubarp = h->ubarp;
    na.lamx = (!dealias && h->cfg.forcing == 1) ? h->lamx : nullptr;
    { TimerScope ts(h, "row_nl"); launch_row_nl(na, h->stream); }
    YFwdJobList yf{};
    yf.n = 9;
    for (int l = 0; l < 3; ++l) yf.j[l] = YFwdJob{na.N[l], Nout + l * S, 1.0, 0.0, dealias ? 1 : 0};
    for (int m = 0; m < 6; ++m) yf.j[3 + m] = YFwdJob{na.H[m], h->H + m * S, 1.0, 0.0, dealias ? 1 : 0};
    { TimerScope ts(h, "yfwd_nl"); launch_yfwd(yf, ya, h->stream); }
    if (f32nl) launch_add_half_sq(h->H, h->ubar, d.C(), d.nzp, h->stream);

    const bool need_phys = (dealias && h->cfg.forcing == 1) || h->cfg.sgsflag == 1;
    if (need_phys) {
        // unpadded physical u_l (+ubar), du_l/dx_m (+ubarp on du/dz); FP32 fields in the
        // mixed form (field i at float offset i * P)
        const long long P = h->P;
        auto PH = [&](long long i) {
            return f32 ? reinterpret_cast<double*>(reinterpret_cast<float*>(h->phys) + i * P) : h->phys + i * P;
        };
        double* ph[12];
        for (int i = 0; i < 12; ++i) ph[i] = PH(i);
        const double* spec[12];
        int modes[12];
        const double* means[12] = {nullptr};
        for (int l = 0; l < 3; ++l) {
            spec[l] = uin + l * S;  // u_l
            modes[l] = YM_COPY;
            spec[3 + 3 * l + 0] = uin + l * S;  // du_l/dx
            modes[3 + 3 * l + 0] = YM_IKX;
            spec[3 + 3 * l + 1] = uin + l * S;  // du_l/dy
            modes[3 + 3 * l + 1] = YM_IKY;
            spec[3 + 3 * l + 2] = h->dz + l * S;  // du_l/dz
            modes[3 + 3 * l + 2] = YM_COPY;
        }
        means[0] = h->ubar;
        means[3 + 2] = h->ubarp;
        const int nphys = (h->cfg.sgsflag == 1) ? 12 : 3;
        // the dynamic model takes only S_ij and delta^2 |S| S_ij from the gradients: its row
        // pass forms them in registers (k_row_c2r_dyn) and the nine gradient rows are not stored
        RowArgs ra = rowargs(h, false, d.nzp);
        ra.f32 = f32;
        const bool dynfuse = h->cfg.sgsflag == 1 && h->cfg.sgsmodel == 1 && row_c2r_dyn_plan(ra);
        {
            TimerScope ts(h, "phys_fields");
            if (dynfuse) {
                YInvJobList yj{};
                DynRowArgs da{};
                da.r = ra;
                yj.n = 9;
                for (int l = 0; l < 3; ++l) {
                    double* yu = h->Yu + (long long)l * h->Yu1;
                    double* ydy = h->Yu + (long long)(3 + l) * h->Yu1;
                    double* ydz = h->Yu + (long long)(6 + l) * h->Yu1;
                    yj.j[l] = YInvJob{uin + l * S, yu, YM_COPY};
                    yj.j[3 + l] = YInvJob{uin + l * S, ydy, YM_IKY};
                    yj.j[6 + l] = YInvJob{h->dz + l * S, ydz, YM_COPY};
                    da.yu[l] = yu;
                    da.ydy[l] = ydy;
                    da.ydz[l] = ydz;
                    da.u[l] = ph[l];
                }
                for (int q = 0; q < 6; ++q) {
                    da.sij[q] = sgs_dyn_field(h, q);
                    da.lij[q] = sgs_dyn_field(h, 6 + q);
                }
                da.ubar = h->ubar;
                da.ubarp = h->ubarp;
                da.delta = h->sgs.delta;
                // the mixed form's forcing reads an FP32 u' without the mean (scratch field 21)
                if (f32 && dealias && h->cfg.forcing == 1) da.uprime = PH(21);
                YPassArgs ya = ypass(h, false, d.nzp);
                ya.f32 = f32;
                launch_yinv(yj, ya, h->stream);
                launch_row_c2r_dyn(da, h->stream);
            } else {
                spec_to_phys(h, spec, ph, nphys, d.nzp, means, modes, f32);
            }
        }
        h->sgs.dyn1_fused = dynfuse;
        // with SGS the forcing goes to spectral space in the same launches as the stresses
        // (scratch field 21 holds the FP32 u' of the mixed form; the SGS model uses 12..17)
        double* no[3] = {Nout, Nout + S, Nout + 2 * S};
        // the fringe forcing lambda(x) (ubar - u) (src/navierstokes.f90:191-204) is formed by the
        // forward row transform as it reads u, v, w (k_row_r2c_*: RowIO::lam)
        const bool forcing = dealias && h->cfg.forcing == 1;
        const double* fin[3] = {ph[0], ph[1], ph[2]};
        const double* fmean[3] = {h->ubar, nullptr, nullptr};  // ph[0] holds u + ubar
        if (forcing) {
            TimerScope ts(h, "forcing");
            if (f32) {
                // lambda (ubar - u) = -lambda u' from an FP32 u' without the mean (no cancellation;
                // the dynamic model's fused row pass has written it already)
                double* up = PH(21);
                const double* sp1[1] = {uin};
                double* pp1[1] = {up};
                if (!dynfuse) spec_to_phys(h, sp1, pp1, 1, d.nzp, nullptr, nullptr, true);
                fin[0] = up;
                fmean[0] = nullptr;
            }
            if (h->cfg.sgsflag != 1) phys_to_spec(h, fin, no, 3, d.nzp, 1.0, 1.0, nullptr, f32, h->lamx, fmean, 3);
        }
        if (h->cfg.sgsflag == 1) {
            TimerScope ts(h, "sgs_total");
            sgs_add_tau(h, ph, dealias, forcing ? fin : nullptr, forcing ? no : nullptr, forcing ? 3 : 0,
                        forcing ? h->lamx : nullptr, fmean);
        }
        h->sgs.dyn1_fused = false;
    }
    // N_l -= d h_l1/dx + d h_l2/dy + d h_l3/dz
    NlDivArgs nd{};
    const bool full9 = h->cfg.sgsflag == 1 && h->sgs.nonsym;
    for (int l = 0; l < 3; ++l) {
        nd.N[l] = Nout + l * S;
        nd.hx[l] = full9 ? h->sgs.H9 + (l * 3 + 0) * S : Hsym(h, l, 0);
        nd.hy[l] = full9 ? h->sgs.H9 + (l * 3 + 1) * S : Hsym(h, l, 1);
    }
    TimerScope ts(h, "nl_divergence");
    // d h_l3 / dz for the three components in one FP64 contraction whose epilogue applies the
    // whole divergence (d h_l3/dz is not stored).  The mixed form uses it too: its int8
    // contraction followed by an elementwise divergence pass took longer (73 + 44 us against
    // 111 us at 256x64x129), and this derivative is then exact
    GemmArgs gz = gemm_base(h, h->m_dz1);
    for (int l = 0; l < 3; ++l) gz.inf[l] = full9 ? h->sgs.H9 + (l * 3 + 2) * S : Hsym(h, l, 2);
    gz.in = gz.inf[0];
    gz.out = h->dz;  // not written
    gz.nfields = 3;
    gz.epi = EPI_NLDIV;
    for (int l = 0; l < 3; ++l) {
        gz.nd_N[l] = nd.N[l];
        gz.nd_hx[l] = nd.hx[l];
        gz.nd_hy[l] = nd.hy[l];
    }
    launch_gemm(gz, h->stream);
}

void coefficients(lsb_handle* h) {
    const int istep = h->istep;
    const int nstart = h->cfg.nstart;
    if (istep <= 3 || h->dt != h->dt2 || h->dt2 != h->dt3) {
        if (nstart == 0 && istep == 1) { h->abfac[0] = 1; h->abfac[1] = 0; h->abfac[2] = 0; }
        else if (nstart == 0 && istep == 2) { h->abfac[0] = 2; h->abfac[1] = -1; h->abfac[2] = 0; }
        else { h->abfac[0] = 3; h->abfac[1] = -3; h->abfac[2] = 1; }
        const double dt1 = h->dt, dt2 = h->dt2, dt3 = h->dt3;
        if (nstart == 0 && istep == 1) {
            h->bdfv = 1.0; h->bdf[0] = 1.0; h->bdf[1] = 0.0; h->bdf[2] = 0.0;
        } else if (nstart == 0 && istep == 2) {
            h->bdfv = 2. / 3.; h->bdf[0] = 2.0; h->bdf[1] = -0.5; h->bdf[2] = 0.0;
        } else if (dt1 != dt2 || dt2 != dt3) {
            const double d12 = dt1 + dt2, d23 = dt2 + dt3, d123 = dt1 + dt2 + dt3;
            const double v = 1. + dt1 / d12 + dt1 / d123;
            h->bdfv = 1. / v;
            h->bdf[0] = -(-1. - dt1 / dt2 - dt1 / d123 - dt1 * dt1 / (d123 * dt2) - dt1 * dt1 * d12 / (d123 * d23 * dt2));
            h->bdf[1] = -(dt1 * dt1 / (d12 * dt2) + dt1 * dt1 / (dt2 * d123) + dt1 * dt1 * d12 / (dt2 * d23 * d123) +
                          dt1 * dt1 * d12 / (dt3 * d23 * d123));
            h->bdf[2] = -(-dt1 * dt1 * d12 / (dt3 * d23 * d123));
        } else {
            h->bdfv = 6. / 11.; h->bdf[0] = 3.0; h->bdf[1] = -1.5; h->bdf[2] = 1. / 3.;
        }
    }
}

// time coefficients of bound(): ceiling shape, wall shapes a and b (src/navierstokes.f90:214-355)
void bound_coeffs(lsb_handle* h, double t, double& ctop, double& cwa, double& cwb) {
    const lsb_config& c = h->cfg;
    const double pi = 4.0 * std::atan(1.0);
    ctop = cwa = cwb = 0.0;
    if (c.bctype == 1) {
        double amp = c.samp * c.u0 / (0.24 * std::sqrt(pi));
        double bamp = c.samp / 2.25;
        const double ref_time = c.xlen / c.u0;
        if (t - c.istartbound <= ref_time) {
            const double s = std::pow(std::sin(0.5 * pi * (t - c.istartbound) / ref_time), 2.0);
            amp *= s;
            bamp *= s;
        } else if (!(t - c.istartbound > ref_time)) {
            amp = bamp = 0.0;
        }
        ctop = amp;
        // bfac = bcf(1,1,1)/bcf(1,1,nzp) makes the wall flux balance the ceiling flux
        const double b00 = bamp * h->bshape_norm;  // bamp * S_wall(0,0) relative to S_top(0,0)
        cwa = (b00 != 0.0) ? amp / h->bshape_norm : 0.0;
        (void)b00;
    } else if (c.bctype == 2) {
        const double A = 0.002 * c.u0, A_half = 0.0001 * c.u0, phi = 0.0;
        const double omega = 1.24e-4 * (c.x0 / c.u0);
        const double theta = t - c.istartbound;
        cwa = A * std::sin(omega * theta);
        cwb = A_half * std::cos(omega / 2.0 * theta + phi);
    } else if (c.bctype == 3) {
        ctop = 1.0;
    }
}

void build_bound_shapes(lsb_handle* h) {
    const lsb_config& c = h->cfg;
    const Dims& d = h->d;
    if (c.bctype == 0) return;
    const double pi = 4.0 * std::atan(1.0);
    const int nx = d.nx, ny = d.ny;
    std::vector<double> top((size_t)nx * ny, 0.0), wa((size_t)nx * ny, 0.0), wb((size_t)nx * ny, 0.0);
    const std::vector<double>& x = h->h_xpts;
    if (c.bctype == 1) {
        const double hh = h->h_zpts[0];
        double xloc = 1.0e5 * c.xnu / c.u0;
        if (x[nx / 2 - 1] < xloc) xloc = c.x0 + 3. / 7. * c.xlen;
        const double xwidth = 0.24 * hh;
        const double bwidth = xwidth * 2.25;
        const double x1 = x[nx - 1] - 2. * bwidth;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double eta = (x[i] - xloc) / xwidth;
                top[(size_t)j * nx + i] = std::exp(-std::pow(eta, 2.0));
                const double eta0 = (x[i] - x1) / bwidth;
                wa[(size_t)j * nx + i] = std::exp(-std::pow(eta0, 4.0));
            }
    } else if (c.bctype == 2) {
        const double x1 = 1.655e5 * c.xnu / c.u0, x2 = 1.81e5 * c.xnu / c.u0, xm = (x1 + x2) / 2.0;
        const double lambda_y = 0.151367188 * c.x0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double eta = 0.0;
                if (x[i] >= x1 && x[i] <= xm) eta = (x[i] - x1) / (xm - x1);
                if (x[i] >= xm && x[i] <= x2) eta = (x2 - x[i]) / (x2 - xm);
                if (x[i] >= x1 && x[i] <= x2) {
                    double f = 15.1875 * std::pow(eta, 5) - 35.4375 * std::pow(eta, 4) + 20.25 * std::pow(eta, 3);
                    if (x[i] > xm) f = -f;
                    const double g = std::cos(2.0 * pi * h->h_ypts[j] / lambda_y);
                    wa[(size_t)j * nx + i] = f;
                    wb[(size_t)j * nx + i] = f * g;
                }
            }
    } else if (c.bctype == 3) {
        const double xc = x[0] + c.bc3_xc;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double e = (x[i] - xc) / c.bc3_s;
                top[(size_t)j * nx + i] = c.bc3_amp * e * std::exp(-e * e);
            }
    } else {
        fail(LSB_ERR_UNSUPPORTED, "bctype must be 0..3");
    }
    const long long C = d.C();
    double* tmp = h->phys;
    CK(cudaMemcpyAsync(tmp, top.data(), C * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(tmp + C, wa.data(), C * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(tmp + 2 * C, wb.data(), C * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const double* ph[3] = {tmp, tmp + C, tmp + 2 * C};
    double* sp[3] = {h->bshape, h->bshape + C, h->bshape + 2 * C};
    phys_to_spec(h, ph, sp, 3, 1, 1.0, 0.0, nullptr);
    if (c.bctype == 1) {
        double s00[2];
        CK(cudaMemcpyAsync(&s00[0], h->bshape, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(&s00[1], h->bshape + C, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        // wall coefficient = bfac*bamp = amp*S_top00/S_wall00 (0 when S_wall00 = 0)
        h->bshape_norm = (s00[1] != 0.0) ? s00[1] / s00[0] : 0.0;
    }
}

void step_one(lsb_handle* h) {
    const Dims& d = h->d;
    const lsb_config& c = h->cfg;
    const long long S = d.S(), C = d.C();
    cudaStream_t st = h->stream;
    h->istep += 1;
    if (c.ifilt >= 1 && c.modfilt > 0 && h->istep % c.modfilt == 0) filter_hook(h);
    coefficients(h);
    const double dt = h->dt;
    // 1-2. nonlinear term (from spectrally filtered velocities when dealiasflag >= 2)
    const double* uin = h->vel;
    if (c.dealiasflag >= 2) {
        const double pi = 4.0 * std::atan(1.0);
        const double alpha = 2.0 * pi / c.xlen, beta = 2.0 * pi / c.ylen;
        SpecFilterArgs fa{};
        for (int l = 0; l < 3; ++l) {
            fa.in[l] = h->vel + l * S;
            fa.out[l] = h->filt + l * S;
        }
        fa.S = S;
        fa.C = C;
        fa.nx = d.nx;
        fa.wavx = h->wavx;
        fa.wavy = h->wavy;
        fa.akmax = std::sqrt(std::pow((d.nx / 2) * alpha, 2) + std::pow((d.ny / 2) * beta, 2));
        fa.akc = fa.akmax * c.kc;
        fa.amp = c.filt_amp;
        fa.order = c.filt_order;
        { TimerScope ts(h, "specfilter"); launch_specfilter(fa, st); }
        uin = h->filt;
    }
    nlterm(h, uin, h->nlc);
    const double* uif = (c.dealiasflag >= 3) ? h->filt : h->vel;
    // 3. velocity right-hand sides
    const double dtnui = 1.0 / (c.xnu * dt);
    RhsArgs ra{};
    for (int l = 0; l < 3; ++l) {
        ra.rhs[l] = h->rhs + l * S;
        ra.N[l] = h->nlc + l * S;
        ra.nln[l] = h->nln + l * S;
        ra.nlnm[l] = h->nlnm + l * S;
        ra.u[l] = uif + l * S;
        ra.un[l] = h->veln + l * S;
        ra.unm[l] = h->velnm + l * S;
        ra.ab[l] = h->abfac[l];
        ra.bdf[l] = h->bdf[l];
    }
    ra.dt = dt;
    ra.dtnui = dtnui;
    ra.ubarpp = h->ubarpp;
    ra.S = S;
    ra.C = C;
    { TimerScope ts(h, "rhs"); launch_rhs(ra, st); }
    // 4. rotate the histories: N^{n-2} <- N^{n-1} <- N^n, u^{n-2} <- u^{n-1} <- u^n
    {
        double* t1 = h->nlnm;
        h->nlnm = h->nln;
        h->nln = h->nlc;
        h->nlc = t1;
        double* t2 = h->velnm;
        h->velnm = h->veln;
        h->veln = h->vel;
        h->vel = t2;
        if (c.dealiasflag >= 3) CK(cudaMemcpyAsync(h->veln, h->filt, 3 * S * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    // 5. boundary planes (Zang-Hussaini)
    double pfac0 = 2.0, pfac1 = -1.0;
    if (h->istep == 1) { pfac0 = 0.0; pfac1 = 0.0; }
    else if (h->istep == 2) { pfac0 = 1.0; pfac1 = 0.0; }
    const bool active = c.bctype > 0 && h->t >= c.istartbound;
    BcArgs ba{};
    for (int l = 0; l < 3; ++l) {
        ba.bc[l] = h->bc + l * 2 * C;
        ba.rtop[l] = h->rhs + l * S;
    }
    ba.bcp = h->bcp;
    ba.pwall = h->p + (long long)(d.nzp - 1) * C;
    ba.pnwall = h->pn + (long long)(d.nzp - 1) * C;
    ba.top_free = (c.bctype == 3 && c.bc3_top == 1) ? 1 : 0;
    ba.w = h->veln + 2 * S;  // rows 1 and nzp of d2fdz2(w^n), formed by the kernel
    ba.d2rows = h->m_dz2rows.p;
    ba.d2ld = h->m_dz2rows.Kp;
    ba.nzp = d.nzp;
    ba.btop = h->bshape;
    ba.bwa = h->bshape + C;
    ba.bwb = h->bshape + 2 * C;
    bound_coeffs(h, h->t, ba.ctop, ba.cwa, ba.cwb);
    ba.pfac0 = pfac0;
    ba.pfac1 = pfac1;
    ba.dt = dt;
    ba.bdfv = h->bdfv;
    ba.dtnui = dtnui;
    ba.xnu = c.xnu;
    ba.active = active ? 1 : 0;
    ba.wavx = h->wavx;
    ba.wavy = h->wavy;
    ba.nx = d.nx;
    ba.C = C;
    { TimerScope ts(h, "bc_planes"); launch_bc_planes(ba, st); }
    // 6. three Helmholtz solves (non-homogeneous when bctype>0 or forcing, src/navierstokes.f90:1388-1394)
    const bool nhom = active || c.forcing == 1;
    { TimerScope ts(h, "helmholtz_uvw"); helmholtz(h, h->rhs, h->vel, 3, dtnui / h->bdfv, nhom ? h->bc : nullptr); }
    // 7. Poisson right-hand side: -D(ikx u + iky v) - k^2 w
    {
        TimerScope ts(h, "poisson");
        launch_divuv(h->vel, h->vel + S, h->divf, h->wavx, h->wavy, d.nx, S, C, st);
        // (FP64 contractions in both forms: see helmholtz())
        zgemm(h, h->m_dz1, h->divf, h->rhs, 1, EPI_POISSON_RHS, 1.0, 0.0, h->vel + 2 * S);
        // 8-9. Poisson solve for w^{n+1}
        helmholtz(h, h->rhs, h->vel + 2 * S, 1, 0.0, h->bcp, false);
    }
    // 10-11. Dw^{n+1}, the pressure phi = -(Dw + div)/(k^2 dt bdfv) into pn (then swapped into
    // p) and the projection of u, v: one contraction whose epilogue does the last two
    {
        TimerScope ts(h, "pressure");
        GemmArgs g = gemm_base(h, h->m_dz1);
        g.in = h->vel + 2 * S;
        g.out = h->T;  // not written
        g.nfields = 1;
        g.epi = EPI_PRESSURE;
        g.pp_u = h->vel;
        g.pp_v = h->vel + S;
        g.pp_p = h->pn;
        g.pp_div = h->divf;
        g.pp_dt = dt;
        g.pp_bdfv = h->bdfv;
        launch_gemm(g, st);
    }
    // norm; ifrz
    TimerScope ts(h, "projection_norm");
    std::swap(h->p, h->pn);
    launch_norm(h->vel, h->vel + S, h->vel + 2 * S, d.nx, d.ny, d.nzp, c.ifrz, st);
    // 12. time
    h->t = h->t + dt;
    h->dt3 = h->dt2;
    h->dt2 = dt;
}

// a kernel raises h->uerr when one of its bounded waits ran out (the int8 tensor-core
// contractions, the TMA-staged spanwise passes and SGS filter)
void check_uerr(lsb_handle* h) {
    if (!h->uerr) return;
    int e = 0;
    CK(cudaMemcpy(&e, h->uerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (e != 0) {
        CK(cudaMemset(h->uerr, 0, sizeof(int)));
        fail(LSB_ERR_CUDA, "a bounded completion wait timed out (tensor-core contraction or TMA staging)");
    }
}

void check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(LSB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- step graphs
// A step whose launches carry the same arguments as an earlier one can be replayed from a
// CUDA graph: after the start-up steps, with a constant dt, no timers, no dt adaptation or
// filter hook, a boundary forcing whose amplitude no longer depends on t, and the time-
// average switch settled.  The graph key adds the history pointers (their rotation has
// period 6, so at most 6 graphs) and the scalars passed by value.
bool graph_eligible(lsb_handle* h) {
    const lsb_config& c = h->cfg;
    if (!h->graphs_on || h->timing || c.dtadapt == 1) return false;
    if (c.ifilt >= 1 && c.modfilt > 0) return false;
    if (h->istep < 3) return false;  // start-up coefficients and boundary-row factors
    if (h->dt != h->dt2 || h->dt2 != h->dt3) return false;
    if (c.otfavg == 1 && h->istep < c.istartavg) return false;
    if (c.bctype == 2) return false;
    if (c.bctype > 0 && h->t < c.istartbound) return false;
    if (c.bctype == 1 && !(h->t - c.istartbound > c.xlen / c.u0)) return false;  // amplitude ramp
    return true;
}

struct HostStep {
    double t, dt, dt2, dt3, abfac[3], bdf[3], bdfv;
    int istep;
    double *vel, *veln, *velnm, *nlc, *nln, *nlnm, *p, *pn;
};
HostStep save_host(const lsb_handle* h) {
    HostStep s{h->t, h->dt, h->dt2, h->dt3, {h->abfac[0], h->abfac[1], h->abfac[2]}, {h->bdf[0], h->bdf[1], h->bdf[2]},
               h->bdfv, h->istep, h->vel, h->veln, h->velnm, h->nlc, h->nln, h->nlnm, h->p, h->pn};
    return s;
}
void restore_host(lsb_handle* h, const HostStep& s) {
    h->t = s.t; h->dt = s.dt; h->dt2 = s.dt2; h->dt3 = s.dt3;
    for (int k = 0; k < 3; ++k) { h->abfac[k] = s.abfac[k]; h->bdf[k] = s.bdf[k]; }
    h->bdfv = s.bdfv; h->istep = s.istep;
    h->vel = s.vel; h->veln = s.veln; h->velnm = s.velnm; h->nlc = s.nlc; h->nln = s.nln; h->nlnm = s.nlnm;
    h->p = s.p; h->pn = s.pn;
}

// the host side of one step, as step_one leaves it (the replayed graph does the device side)
void replay_advance(lsb_handle* h) {
    h->istep += 1;
    coefficients(h);
    double* t1 = h->nlnm;
    h->nlnm = h->nln;
    h->nln = h->nlc;
    h->nlc = t1;
    double* t2 = h->velnm;
    h->velnm = h->veln;
    h->veln = h->vel;
    h->vel = t2;
    std::swap(h->p, h->pn);
    h->t = h->t + h->dt;
    h->dt3 = h->dt2;
    h->dt2 = h->dt;
}

// runs one step from a graph (replayed, or captured now and launched); false: not eligible
// or capture unavailable, and the caller runs the step with ordinary launches
template <class Body>
bool graph_step(lsb_handle* h, Body&& body) {
    if (!graph_eligible(h)) return false;
    double ctop = 0, cwa = 0, cwb = 0;
    bound_coeffs(h, h->t, ctop, cwa, cwb);
    const void* key[8] = {h->vel, h->veln, h->velnm, h->nlc, h->nln, h->nlnm, h->p, h->pn};
    for (auto& g : h->graphs) {
        if (std::memcmp(g.key, key, sizeof(key)) != 0 || g.dt != h->dt || g.ctop != ctop || g.cwa != cwa || g.cwb != cwb)
            continue;
        CK(cudaGraphLaunch(g.exec, h->stream));
        lsb::note_launches((long long)g.kernels);
        replay_advance(h);
        return true;
    }
    if (h->graphs.size() >= 6) return false;
    const HostStep snap = save_host(h);
    const unsigned long long k0 = lsb::launches_so_far();
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        h->graphs_on = false;
        return false;
    }
    bool ok = true;
    try {
        body();
    } catch (...) {
        ok = false;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (ok && e == cudaSuccess && graph != nullptr && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        lsb_handle::StepGraph g;
        std::memcpy(g.key, key, sizeof(key));
        g.dt = snap.dt;
        g.ctop = ctop;
        g.cwa = cwa;
        g.cwb = cwb;
        g.kernels = lsb::launches_so_far() - k0;
        g.exec = exec;
        h->graphs.push_back(g);
        CK(cudaGraphLaunch(exec, h->stream));  // the captured step has not run yet
        return true;
    }
    // capture did not work here: undo the host side of the captured step, run it plainly
    cudaGetLastError();
    if (graph) cudaGraphDestroy(graph);
    restore_host(h, snap);
    lsb::note_launches(-(long long)(lsb::launches_so_far() - k0));
    h->graphs_on = false;
    return false;
}

// one timestep() on the handle's stream with ordinary launches: the update, then dt
// adaptation (src/navierstokes.f90:78-87) and the on-the-fly averages (src/main.f90:70-76)
void run_step(lsb_handle* h) {
    const lsb_config& c = h->cfg;
    const long long S = h->d.S();
    step_one(h);
    check_launch();
    // adaptive dt: NaN check + maxcalc every 5 steps and every iomod steps
    if (c.dtadapt == 1 && (h->istep % c.iomod == 0 || h->istep % 5 == 0)) {
        lsb_diagnostics dg;
        diag_compute(h, &dg);
        if (dg.nonfinite) fail(LSB_ERR_NONFINITE, "NaN detected at step " + std::to_string(h->istep));
        const bool exceed = dg.cflz > 0.45 || dg.cflx > 0.25 || dg.cfly > 0.25;
        const bool below = dg.cflz < 0.25 && dg.cflx < 0.10 && dg.cfly < 0.12 && h->dt < 1.0;
        if (exceed || below) {
            const double cdt = exceed ? 1.25 : 1.0 / 1.25;
            h->dt2 = h->dt;
            h->dt = h->dt / cdt;
        }
    }
    // on-the-fly averages: q_tavg += q / iomod
    if (c.otfavg == 1 && h->istep > c.istartavg) {
        const double* q[4] = {h->vel, h->vel + S, h->vel + 2 * S, h->p};
        for (int k = 0; k < 4; ++k) launch_tavg_add(h->tavg + k * S, q[k], (double)c.iomod, S, h->stream);
    }
}

// one step of one handle: from its step graphs when steady, else ordinary launches
void step_once(lsb_handle* h) {
    NvtxRange r("timestep");
    if (graph_step(h, [h] { run_step(h); })) return;
    run_step(h);
}

}  // namespace

// ---------------------------------------------------------------- ensembles
// Runs stepped together (lsb_batch_*): every batch step advances each member by one
// timestep().  When every member's step is steady (graph_eligible), the members' steps are
// captured as parallel branches of ONE CUDA graph (fork from the batch stream onto each
// member's stream, join back) and replayed with one graph launch per ensemble step, so the
// members' kernels overlap on the device and the host issues one launch instead of one per
// member kernel.  The ensemble key is every member's step-graph key; the members advance in
// lockstep, so their history rotations stay in phase and at most 6 ensemble graphs exist.
struct lsb_batch {
    std::vector<lsb_handle*> m;
    cudaStream_t own = nullptr;      // the batch's own stream
    cudaStream_t stream = nullptr;   // ensemble graphs are launched here (own or the caller's)
    cudaEvent_t fork = nullptr;      // batch stream -> member streams
    std::vector<cudaEvent_t> join;   // member stream i -> batch stream
    struct EnsGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<const void*> key;
        std::vector<double> sc;      // per member: dt, ctop, cwa, cwb
        unsigned long long kernels = 0;
    };
    std::vector<EnsGraph> graphs;
    bool graphs_on = true;
    bool on_batch = false;  // the members' latest work is on the batch stream
    void drop_graphs() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    ~lsb_batch() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (auto e : join)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (own) cudaStreamDestroy(own);
    }
};

namespace {

// member streams wait for the batch stream (after ensemble replays)
void batch_to_members(lsb_batch* b) {
    if (!b->on_batch) return;
    CK(cudaEventRecord(b->fork, b->stream));
    for (lsb_handle* h : b->m) CK(cudaStreamWaitEvent(h->stream, b->fork, 0));
    b->on_batch = false;
}

// the batch stream waits for every member stream (before ensemble replays)
void members_to_batch(lsb_batch* b) {
    if (b->on_batch) return;
    for (size_t i = 0; i < b->m.size(); ++i) {
        CK(cudaEventRecord(b->join[i], b->m[i]->stream));
        CK(cudaStreamWaitEvent(b->stream, b->join[i], 0));
    }
    b->on_batch = true;
}

// one ensemble step from an ensemble graph (replayed, or captured now); false: some member
// is not steady, or capture is unavailable, and the caller steps the members one by one
bool batch_graph_step(lsb_batch* b) {
    if (!b->graphs_on) return false;
    const size_t n = b->m.size();
    std::vector<const void*> key;
    std::vector<double> sc;
    key.reserve(8 * n);
    sc.reserve(5 * n);
    for (lsb_handle* h : b->m) {
        if (!graph_eligible(h)) return false;
        double ctop = 0, cwa = 0, cwb = 0;
        bound_coeffs(h, h->t, ctop, cwa, cwb);
        const void* k[8] = {h->vel, h->veln, h->velnm, h->nlc, h->nln, h->nlnm, h->p, h->pn};
        key.insert(key.end(), k, k + 8);
        // the member's graph generation: a schedule set on it since makes a new capture
        const double s[5] = {h->dt, ctop, cwa, cwb, (double)h->graph_gen};
        sc.insert(sc.end(), s, s + 5);
    }
    members_to_batch(b);
    for (auto& g : b->graphs) {
        if (g.key != key || g.sc != sc) continue;
        CK(cudaGraphLaunch(g.exec, b->stream));
        lsb::note_launches((long long)g.kernels);
        for (lsb_handle* h : b->m) replay_advance(h);
        return true;
    }
    if (b->graphs.size() >= 6) b->drop_graphs();  // a member's scalars changed
    std::vector<HostStep> snap;
    snap.reserve(n);
    for (lsb_handle* h : b->m) snap.push_back(save_host(h));
    const unsigned long long k0 = lsb::launches_so_far();
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        b->graphs_on = false;
        return false;
    }
    bool ok = cudaEventRecord(b->fork, b->stream) == cudaSuccess;
    for (size_t i = 0; ok && i < n; ++i) {
        lsb_handle* h = b->m[i];
        if (cudaStreamWaitEvent(h->stream, b->fork, 0) != cudaSuccess) {
            ok = false;
            break;
        }
        try {
            run_step(h);
        } catch (...) {
            ok = false;
        }
        // join this member back even after a failure, so that the capture can end
        if (cudaEventRecord(b->join[i], h->stream) != cudaSuccess ||
            cudaStreamWaitEvent(b->stream, b->join[i], 0) != cudaSuccess)
            ok = false;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (ok && e == cudaSuccess && graph != nullptr && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        lsb_batch::EnsGraph g;
        g.key = std::move(key);
        g.sc = std::move(sc);
        g.kernels = lsb::launches_so_far() - k0;
        g.exec = exec;
        b->graphs.push_back(std::move(g));
        CK(cudaGraphLaunch(exec, b->stream));  // the captured step has not run yet
        return true;
    }
    // capture did not work: undo the members' host side, step them one by one
    cudaGetLastError();
    if (graph) cudaGraphDestroy(graph);
    for (size_t i = 0; i < n; ++i) restore_host(b->m[i], snap[i]);
    lsb::note_launches(-(long long)(lsb::launches_so_far() - k0));
    b->graphs_on = false;
    return false;
}

}  // namespace

namespace lsb {
void set_last_error(const std::string& m) { g_err = m; }

// kernels launched by this library since it was loaded (all handles, all threads)
static std::atomic<unsigned long long> g_kernel_launches{0};
void note_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long n) { g_kernel_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launches_so_far() { return g_kernel_launches.load(); }

static std::mutex g_occ_mu;
static std::map<std::tuple<int, const void*, int, size_t>, int> g_occ;
static std::map<int, int> g_nsm;

int sm_count() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = g_nsm.find(dev);
    if (it != g_nsm.end()) return it->second;
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
    g_nsm[dev] = n;
    return n;
}

size_t smem_optin() {
    static std::map<int, size_t> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cache[dev] = (size_t)(v > 0 ? v : 48 * 1024);
    return cache[dev];
}

bool allow_smem(const void* kern, size_t smem) {
    // the limit is a property of the kernel, not of a launch: keep the largest value set so
    // far per (device, kernel) and only ever raise it
    static std::map<std::pair<int, const void*>, size_t> cur;
    if (smem <= 48 * 1024) return true;
    if (smem > smem_optin()) return false;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_pair(dev, kern);
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = cur.find(key);
    if (it != cur.end() && it->second >= smem) return true;
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        cudaGetLastError();  // clear it: the caller falls back to another kernel
        if (std::getenv("LSB_DEBUG"))
            std::fprintf(stderr, "lsbgpu: dynamic shared memory %zu refused: %s\n", smem, cudaGetErrorString(e));
        return false;
    }
    cur[key] = smem;
    return true;
}

int resident_blocks(const void* kern, int threads, size_t smem) {
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, kern, threads, smem);
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(key);
        if (it != g_occ.end()) return it->second;
    }
    size_t lim = smem > 200 * 1024 ? smem : 200 * 1024;
    if (lim > smem_optin()) lim = smem_optin();
    allow_smem(kern, lim);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
    if (occ < 1) occ = 1;
    std::lock_guard<std::mutex> lk(g_occ_mu);
    g_occ[key] = occ;
    return occ;
}
}  // namespace lsb

// ====================================================================================== C ABI
extern "C" {

const char* lsb_last_error(void) { return g_err.c_str(); }
int lsb_version(void) { return 1; }
unsigned long long lsb_kernel_launches(void) { return lsb::g_kernel_launches.load(); }

int lsb_device_bytes(lsb_handle* h, unsigned long long* bytes) {
    return guard([&] {
        if (!h || !bytes) fail(LSB_ERR_ARG, "null argument");
        *bytes = h->device_bytes;
    });
}

int lsb_create(const lsb_config* cfg, const lsb_setup* su, lsb_handle** out) {
    return guard([&] {
        if (!cfg || !su || !out) fail(LSB_ERR_ARG, "null argument");
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(LSB_ERR_CUDA, "no CUDA device");
        std::unique_ptr<lsb_handle> h(new lsb_handle());
        h->cfg = *cfg;
        Dims& d = h->d;
        d.nx = cfg->nx;
        d.ny = cfg->ny;
        d.nz = cfg->nz;
        d.nzp = cfg->nz + 1;
        d.nzm = cfg->nz - 1;
        d.kx = cfg->nx / 2;
        if (d.nx < 4 || d.nx % 2 || d.ny < 1 || d.nz < 3) fail(LSB_ERR_ARG, "bad grid size");
        if ((long long)d.nx * d.ny * (d.nz + 1) >= (1LL << 31)) fail(LSB_ERR_ARG, "grid too large (2^31 points or more)");
        if (cfg->dealiasflag == 1) {
            // setup_dealiasing, nproch = 1 (src/dealiasing.f90:133-154)
            if (d.nx % 2 == 0 && d.nx % 4 == 0) d.nxl = 3 * d.nx / 2;
            else if (d.nx % 3 == 0) d.nxl = 5 * d.nx / 3;
            else if (d.nx % 5 == 0) d.nxl = 8 * d.nx / 5;
            else d.nxl = 2 * d.nx;
            if (d.ny % 2 == 0) d.nyl = 3 * d.ny / 2;
            else if (d.ny % 3 == 0) d.nyl = 5 * d.ny / 3;
            else if (d.ny % 5 == 0) d.nyl = 8 * d.ny / 5;
            else d.nyl = 2 * d.ny;
        } else {
            d.nxl = d.nx;
            d.nyl = d.ny;
        }
        if (cfg->sgsflag == 1 && (cfg->sgsmodel < 0 || cfg->sgsmodel > 4)) fail(LSB_ERR_ARG, "sgsmodel must be 0..4");
        CK(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        h->stream = h->own;
        const int nx = d.nx, ny = d.ny, nzp = d.nzp, nzm = d.nzm;
        h->h_xpts.assign(su->xpts, su->xpts + nx);
        h->h_ypts.assign(su->ypts, su->ypts + ny);
        h->h_zpts.assign(su->zpts, su->zpts + nzp);
        h->h_ubar.assign(su->ubar, su->ubar + nzp);
        h->dx = su->dx;
        h->dy = su->dy;
        h->wavx = h->upload(su->wavx, nx);
        h->wavy = h->upload(su->wavy, ny);
        h->zpts = h->upload(su->zpts, nzp);
        h->ubar = h->upload(su->ubar, nzp);
        h->ubarp = h->upload(su->ubarp, nzp);
        h->ubarpp = h->upload(su->ubarpp, nzp);
        h->hb = h->upload(su->hbot, nzp);
        h->ht = h->upload(su->htop, nzp);
        h->d2hb = h->upload(su->d2hbot, nzp);
        h->d2ht = h->upload(su->d2htop, nzp);
        h->lam = h->upload(su->lam, nzm);
        h->lamx = h->upload(su->lamx, nx);
        h->m_dz1 = make_mat(h.get(), su->dz1, nzp, nzp);
        h->uerr = reinterpret_cast<int*>(h->alloc(1));
        h->m_dz2 = make_mat(h.get(), su->dz2, nzp, nzp);
        {
            std::vector<double> rows(2 * (size_t)nzp);
            for (int k = 0; k < nzp; ++k) {
                rows[k] = su->dz2[k];
                rows[nzp + k] = su->dz2[(size_t)(nzp - 1) * nzp + k];
            }
            h->m_dz2rows = make_mat(h.get(), rows.data(), 2, nzp);
        }
        h->m_ei = make_mat(h.get(), su->ei, nzm, nzm);
        h->m_eext = make_mat(h.get(), su->e, nzm, nzm, 0, nzm, 1, nzp);  // zero ceiling / wall rows
        if (cfg->precision == 1) {
            // the mixed form's contractions on the int8 tensor cores: D, E^-1 and E (the latter
            // with its zero ceiling and wall rows, as m_eext)
            std::vector<double> eext((size_t)nzp * nzm, 0.0);
            for (int r = 0; r < nzm; ++r)
                for (int k = 0; k < nzm; ++k) eext[(size_t)(r + 1) * nzm + k] = su->e[(size_t)r * nzm + k];
            h->oz_dz1 = upload_ozaki(h.get(), su->dz1, nzp, nzp, 5);
            h->oz_ei = upload_ozaki(h.get(), su->ei, nzm, nzm, 5);
            h->oz_eext = upload_ozaki(h.get(), eext.data(), nzp, nzm, 5);
        }
        make_plan(h.get(), ny, h->py, 16);
        make_plan(h.get(), d.nyl, h->pyl, 16);
        make_real_plan(h.get(), nx, h->rx);
        make_real_plan(h.get(), d.nxl, h->rxl);
        if (cfg->precision != 0 && cfg->precision != 1) fail(LSB_ERR_ARG, "precision must be 0 (FP64) or 1 (mixed)");
        if (cfg->precision == 1) {
            const bool dl = cfg->dealiasflag == 1;
            const bool phys = cfg->sgsflag == 1 || (dl && cfg->forcing == 1);
            // the nonlinear term's (padded) passes in FP32 where their lengths have full-warp
            // register plans, else in FP64 (the 3/2-rule x length 48 of a 64-point grid)
            h->nl_f32 = (dl ? h->pyl : h->py).g != 0 && (dl ? h->rxl : h->rx).half.g == 32;
            if ((!dl && !h->nl_f32) || (phys && (h->py.g == 0 || h->rx.half.g == 0)))
                fail(LSB_ERR_ARG, "mixed precision needs transform lengths with register plans: x/2 a multiple of "
                                  "32 (32 R, R in 1,2,3,4,6,8) and y a power of two times 1,2,3,4,6,8");
        }
        const long long S = d.S(), C = d.C();
        h->Yl = (long long)nzp * d.nyl * nx;
        h->Yu1 = (long long)nzp * ny * nx;
        h->P = (long long)nzp * ny * nx;
        h->vel = h->alloc(3 * S);
        h->veln = h->alloc(3 * S);
        h->velnm = h->alloc(3 * S);
        h->nlc = h->alloc(3 * S);
        h->nln = h->alloc(3 * S);
        h->nlnm = h->alloc(3 * S);
        h->p = h->alloc(S);
        h->pn = h->alloc(S);
        h->filt = h->alloc(3 * S);
        h->dz = h->alloc(3 * S);
        h->H = h->alloc(6 * S);
        h->rhs = h->alloc(3 * S);
        h->T = h->alloc(3 * S);
        h->divf = h->alloc(S);
        h->Y = h->alloc(18 * h->Yl);
        h->Yu = h->alloc(kMaxJobs * h->Yu1);
        h->phys = h->alloc((long long)lsb_handle::kPhys * h->P);
        h->bc = h->alloc(6 * C);
        h->bcp = h->alloc(2 * C);
        h->bshape = h->alloc(3 * C);
        h->io = h->alloc(12 * S);
        h->red = h->alloc(512);
        filters_init(h.get());
        if (cfg->sgsflag == 1) sgs_init(h.get());
        if (cfg->otfavg == 1) h->tavg = h->alloc(4 * S);
        if (cfg->ifilt >= 1 && cfg->modfilt <= 0) fail(LSB_ERR_ARG, "ifilt needs modfilt > 0");
        if (cfg->dtadapt == 1 && cfg->iomod <= 0) fail(LSB_ERR_ARG, "dtadapt needs iomod > 0");
        build_bound_shapes(h.get());
        CK(cudaStreamSynchronize(h->stream));
        check_launch();
        *out = h.release();
    });
}

int lsb_destroy(lsb_handle* h) {
    return guard([&] { delete h; });
}

int lsb_set_stream(lsb_handle* h, void* stream) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        CK(cudaStreamSynchronize(h->stream));
        h->stream = stream ? (cudaStream_t)stream : h->own;
    });
}

int lsb_synchronize(lsb_handle* h) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        CK(cudaStreamSynchronize(h->stream));
        check_launch();
        check_uerr(h);
    });
}

int lsb_upload_state(lsb_handle* h, const double* uf, const double* vf, const double* wf, const double* pf,
                     const double* pnf, const double* unif, const double* unmif, const double* nlnif,
                     const double* nlnmif, double t, double dt, double dt2, double dt3, int istep) {
    return guard([&] {
        if (!h || !uf || !vf || !wf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        const size_t B = S * sizeof(double);
        auto up = [&](double* dst, const double* src, size_t bytes) {
            if (src) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
            else CK(cudaMemsetAsync(dst, 0, bytes, h->stream));
        };
        up(h->vel, uf, B);
        up(h->vel + S, vf, B);
        up(h->vel + 2 * S, wf, B);
        up(h->p, pf, B);
        up(h->pn, pnf, B);
        up(h->veln, unif, 3 * B);
        up(h->velnm, unmif, 3 * B);
        up(h->nln, nlnif, 3 * B);
        up(h->nlnm, nlnmif, 3 * B);
        h->t = t;
        h->dt = dt;
        h->dt2 = dt2;
        h->dt3 = dt3;
        h->istep = istep;
        CK(cudaStreamSynchronize(h->stream));
    });
}

int lsb_download_state(lsb_handle* h, double* uf, double* vf, double* wf, double* pf, double* pnf, double* unif,
                       double* unmif, double* nlnif, double* nlnmif, double* t, double* dt, double* dt2, double* dt3,
                       int* istep) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        const long long S = h->d.S();
        const size_t B = S * sizeof(double);
        auto dn = [&](double* dst, const double* src, size_t bytes) {
            if (dst) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
        };
        dn(uf, h->vel, B);
        dn(vf, h->vel + S, B);
        dn(wf, h->vel + 2 * S, B);
        dn(pf, h->p, B);
        dn(pnf, h->pn, B);
        dn(unif, h->veln, 3 * B);
        dn(unmif, h->velnm, 3 * B);
        dn(nlnif, h->nln, 3 * B);
        dn(nlnmif, h->nlnm, 3 * B);
        CK(cudaStreamSynchronize(h->stream));
        check_uerr(h);
        if (t) *t = h->t;
        if (dt) *dt = h->dt;
        if (dt2) *dt2 = h->dt2;
        if (dt3) *dt3 = h->dt3;
        if (istep) *istep = h->istep;
    });
}

int lsb_upload_state_device(lsb_handle* h, const double* uf, const double* vf, const double* wf) {
    return guard([&] {
        if (!h || !uf || !vf || !wf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        CK(cudaMemcpyAsync(h->vel, uf, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->vel + S, vf, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->vel + 2 * S, wf, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    });
}

int lsb_download_velocity_device(lsb_handle* h, double* uf, double* vf, double* wf) {
    return guard([&] {
        if (!h || !uf || !vf || !wf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        CK(cudaMemcpyAsync(uf, h->vel, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(vf, h->vel + S, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(wf, h->vel + 2 * S, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    });
}

int lsb_step(lsb_handle* h, int nsteps) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        if (nsteps < 0) fail(LSB_ERR_ARG, "nsteps < 0");
        if (!(h->dt > 0.0) || !std::isfinite(h->dt)) fail(LSB_ERR_STATE, "dt must be finite and > 0");
        for (int i = 0; i < nsteps; ++i) step_once(h);
    });
}

// ---------------------------------------------------------------- ensembles (lsb_batch_*)
int lsb_batch_create(lsb_handle* const* members, int nmembers, lsb_batch** out) {
    return guard([&] {
        if (!members || !out || nmembers < 1) fail(LSB_ERR_ARG, "need an array of at least one member handle");
        *out = nullptr;
        for (int i = 0; i < nmembers; ++i) {
            if (!members[i]) fail(LSB_ERR_ARG, "null member handle " + std::to_string(i));
            for (int j = 0; j < i; ++j)
                if (members[j] == members[i]) fail(LSB_ERR_ARG, "member " + std::to_string(i) + " appears twice");
        }
        std::unique_ptr<lsb_batch> b(new lsb_batch);
        b->m.assign(members, members + nmembers);
        CK(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
        b->stream = b->own;
        CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        b->join.assign(nmembers, nullptr);
        for (int i = 0; i < nmembers; ++i) CK(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming));
        *out = b.release();
    });
}

int lsb_batch_destroy(lsb_batch* b) {
    return guard([&] { delete b; });
}

int lsb_batch_step(lsb_batch* b, int nsteps) {
    return guard([&] {
        if (!b) fail(LSB_ERR_ARG, "null batch");
        if (nsteps < 0) fail(LSB_ERR_ARG, "nsteps < 0");
        for (size_t i = 0; i < b->m.size(); ++i) {
            const double dt = b->m[i]->dt;
            if (!(dt > 0.0) || !std::isfinite(dt))
                fail(LSB_ERR_STATE, "member " + std::to_string(i) + ": dt must be finite and > 0");
        }
        try {
            for (int s = 0; s < nsteps; ++s) {
                NvtxRange r("ensemble_step");
                if (batch_graph_step(b)) continue;
                batch_to_members(b);
                for (lsb_handle* h : b->m) step_once(h);
            }
            // both ways: an event recorded on the batch stream now follows every member's
            // steps, and work queued on a member's stream follows the ensemble replays
            members_to_batch(b);
            batch_to_members(b);
        } catch (...) {
            if (b->on_batch) {  // keep the members ordered after the batch's launches
                cudaEventRecord(b->fork, b->stream);
                for (lsb_handle* h : b->m) cudaStreamWaitEvent(h->stream, b->fork, 0);
                b->on_batch = false;
            }
            throw;
        }
    });
}

int lsb_batch_set_stream(lsb_batch* b, void* stream) {
    return guard([&] {
        if (!b) fail(LSB_ERR_ARG, "null batch");
        CK(cudaStreamSynchronize(b->stream));
        b->stream = stream ? (cudaStream_t)stream : b->own;
    });
}

int lsb_batch_synchronize(lsb_batch* b) {
    return guard([&] {
        if (!b) fail(LSB_ERR_ARG, "null batch");
        CK(cudaStreamSynchronize(b->stream));
        for (lsb_handle* h : b->m) CK(cudaStreamSynchronize(h->stream));
        check_launch();
        for (lsb_handle* h : b->m) check_uerr(h);
    });
}

int lsb_batch_graphs(lsb_batch* b, int enable) {
    return guard([&] {
        if (!b) fail(LSB_ERR_ARG, "null batch");
        CK(cudaStreamSynchronize(b->stream));
        b->drop_graphs();
        b->graphs_on = enable != 0;
    });
}

int lsb_set_schedule(lsb_handle* h, const lsb_schedule* s) {
    return guard([&] {
        if (!h || !s) fail(LSB_ERR_ARG, "null argument");
        if (s->gemm_warps != 0 && (s->gemm_warps < 4 || s->gemm_warps > 8))
            fail(LSB_ERR_ARG, "gemm_warps must be 0 or 4..8");
        const int zmax = std::max(1, (h->d.nzp + 3) / 4);
        if (s->filter_zchunks < 0 || s->filter_zchunks > zmax)
            fail(LSB_ERR_ARG, "filter_zchunks must be 0.." + std::to_string(zmax));
        if (s->y_staging < 0 || s->y_staging > 2) fail(LSB_ERR_ARG, "y_staging must be 0, 1 or 2");
        if (s->filter_staging < 0 || s->filter_staging > 2) fail(LSB_ERR_ARG, "filter_staging must be 0, 1 or 2");
        if (s->filter_staging == 2 && (h->d.nx * (h->cfg.precision == 1 ? 4 : 8)) % 128 != 0)
            fail(LSB_ERR_ARG, "filter_staging 2 needs rows of a multiple of 128 bytes");
        CK(cudaStreamSynchronize(h->stream));
        h->drop_graphs();
        h->sched = *s;
    });
}

int lsb_get_schedule(lsb_handle* h, lsb_schedule* s) {
    return guard([&] {
        if (!h || !s) fail(LSB_ERR_ARG, "null argument");
        *s = h->sched;
    });
}

int lsb_graphs(lsb_handle* h, int enable) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        CK(cudaStreamSynchronize(h->stream));
        h->drop_graphs();
        h->graphs_on = enable != 0;
    });
}

// ---------------------------------------------------------------- tier 1
namespace {
void to_dev_phys(lsb_handle* h, const double* src, double* dst, int nf) {
    // host (nx+2, ny, nzp) -> device [nzp][ny][nx]
    const Dims& d = h->d;
    const size_t rows = (size_t)d.ny * d.nzp;
    for (int f = 0; f < nf; ++f)
        CK(cudaMemcpy2DAsync(dst + f * h->P, d.nx * sizeof(double), src + f * rows * (d.nx + 2),
                             (d.nx + 2) * sizeof(double), d.nx * sizeof(double), rows, cudaMemcpyHostToDevice,
                             h->stream));
}
void from_dev_phys(lsb_handle* h, const double* src, double* dst, int nf) {
    const Dims& d = h->d;
    const size_t rows = (size_t)d.ny * d.nzp;
    for (int f = 0; f < nf; ++f) {
        std::memset(dst + f * rows * (d.nx + 2), 0, rows * (d.nx + 2) * sizeof(double));
        CK(cudaMemcpy2DAsync(dst + f * rows * (d.nx + 2), (d.nx + 2) * sizeof(double), src + f * h->P,
                             d.nx * sizeof(double), d.nx * sizeof(double), rows, cudaMemcpyDeviceToHost, h->stream));
    }
}
void to_dev(lsb_handle* h, const double* src, double* dst, long long n) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
}
void from_dev(lsb_handle* h, const double* src, double* dst, long long n) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    check_launch();
    check_uerr(h);
}
}  // namespace

int lsb_horfft(lsb_handle* h, double* ain, double* ainf, int is) {
    return guard([&] {
        if (!h || !ain || !ainf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        double* ph = h->phys;
        double* sp = h->io;
        if (is == -1) {
            to_dev_phys(h, ain, ph, 1);
            const double* pp[1] = {ph};
            double* ss[1] = {sp};
            phys_to_spec(h, pp, ss, 1, h->d.nzp, 1.0, 0.0, nullptr);
            from_dev(h, sp, ainf, S);
        } else if (is == 1) {
            to_dev(h, ainf, sp, S);
            const double* ss[1] = {sp};
            double* pp[1] = {ph};
            spec_to_phys(h, ss, pp, 1, h->d.nzp, nullptr, nullptr);
            from_dev_phys(h, ph, ain, 1);
            CK(cudaStreamSynchronize(h->stream));
            check_launch();
        } else {
            fail(LSB_ERR_ARG, "is must be -1 or +1");
        }
    });
}

int lsb_dfdx(lsb_handle* h, const double* uf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        launch_dxy(h->io, h->io + S, h->wavx, h->wavy, h->d.nx, S, h->d.C(), 0, h->stream);
        from_dev(h, h->io + S, out, S);
    });
}

int lsb_dfdy(lsb_handle* h, const double* uf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        launch_dxy(h->io, h->io + S, h->wavx, h->wavy, h->d.nx, S, h->d.C(), 1, h->stream);
        from_dev(h, h->io + S, out, S);
    });
}

int lsb_dfdz(lsb_handle* h, const double* uf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        // the contraction of the handle's form (int8 tensor cores in the mixed form)
        GemmArgs g = gemm_base(h, h->m_dz1);
        g.in = h->io;
        g.out = h->io + S;
        g.epi = EPI_STORE;
        contract(h, g, h->oz_dz1);
        from_dev(h, h->io + S, out, S);
    });
}

int lsb_d2fdz2(lsb_handle* h, const double* uf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        zgemm1(h, h->m_dz2, h->io, h->io + S, 1);
        from_dev(h, h->io + S, out, S);
    });
}

int lsb_lapl(lsb_handle* h, const double* uf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        zgemm1(h, h->m_dz2, h->io, h->io + S, 1);
        launch_lapl_xy(h->io, h->io + S, h->wavx, h->wavy, h->d.nx, S, h->d.C(), h->stream);
        from_dev(h, h->io + S, out, S);
    });
}

int lsb_divuv(lsb_handle* h, const double* uf, const double* vf, double* out) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uf, h->io, S);
        to_dev(h, vf, h->io + S, S);
        launch_divuv(h->io, h->io + S, h->io + 2 * S, h->wavx, h->wavy, h->d.nx, S, h->d.C(), h->stream);
        from_dev(h, h->io + 2 * S, out, S);
    });
}

int lsb_solve_helmholtz(lsb_handle* h, double* rhs, double dtnui) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, rhs, h->io, S);
        helmholtz(h, h->io, h->io + S, 1, dtnui, nullptr);
        from_dev(h, h->io + S, rhs, S);
    });
}

int lsb_solve_nhom_helmholtz(lsb_handle* h, double* rhs, const double* bc, double dtnui) {
    return guard([&] {
        const Dims& d = h->d;
        const long long S = d.S(), C = d.C();
        to_dev(h, rhs, h->io, S);
        // boundary field: only its planes k = 1 (ceiling) and k = nzp (wall) are read
        to_dev(h, bc, h->io + 2 * S, C);
        to_dev(h, bc + (long long)(d.nzp - 1) * C, h->io + 2 * S + C, C);
        helmholtz(h, h->io, h->io + S, 1, dtnui, h->io + 2 * S);
        from_dev(h, h->io + S, rhs, S);
    });
}

int lsb_dealias_product(lsb_handle* h, const double* a, const double* b, double* ab) {
    return guard([&] {
        const Dims& d = h->d;
        if (h->cfg.dealiasflag != 1) fail(LSB_ERR_STATE, "handle was created without dealiasflag = 1");
        const long long S = d.S();
        to_dev_phys(h, a, h->phys, 1);
        to_dev_phys(h, b, h->phys + h->P, 1);
        const double* pp[2] = {h->phys, h->phys + h->P};
        double* ss[2] = {h->io, h->io + S};
        phys_to_spec(h, pp, ss, 2, d.nzp, 1.0, 0.0, nullptr);
        // pad, inverse, product, forward, truncate: reuse the spanwise / row passes on the padded grid
        YInvJobList yj{};
        yj.n = 2;
        yj.j[0] = YInvJob{h->io, h->Y, YM_COPY};
        yj.j[1] = YInvJob{h->io + S, h->Y + h->Yl, YM_COPY};
        launch_yinv(yj, ypass(h, true, d.nzp), h->stream);
        RowJobList rj{};
        rj.n = 2;
        const long long PL = (long long)d.nxl * d.nyl * d.nzp;
        double* pl = h->Y + 2 * h->Yl;  // padded physical rows live after the two y-intermediates
        if (2 * h->Yl + 3 * PL > 18 * h->Yl) fail(LSB_ERR_STATE, "scratch too small");
        rj.j[0] = RowIO{h->Y, pl, YM_COPY, 0.0, nullptr, 1.0};
        rj.j[1] = RowIO{h->Y + h->Yl, pl + PL, YM_COPY, 0.0, nullptr, 1.0};
        launch_row_c2r(rj, rowargs(h, true, d.nzp), h->stream);
        launch_axpby(pl + 2 * PL, pl, 1.0, 0.0, PL, h->stream);
        sgs_mul(pl + 2 * PL, pl + PL, PL, h->stream);
        RowJobList rf{};
        rf.n = 1;
        rf.j[0] = RowIO{pl + 2 * PL, h->Y, YM_COPY, 0.0, nullptr, 1.0};
        launch_row_r2c(rf, rowargs(h, true, d.nzp), h->stream);
        YFwdJobList yf{};
        yf.n = 1;
        yf.j[0] = YFwdJob{h->Y, h->io + 2 * S, 1.0, 0.0, 0};
        launch_yfwd(yf, ypass(h, true, d.nzp), h->stream);
        const double* ss2[1] = {h->io + 2 * S};
        double* pp2[1] = {h->phys + 2 * h->P};
        spec_to_phys(h, ss2, pp2, 1, d.nzp, nullptr, nullptr);
        from_dev_phys(h, h->phys + 2 * h->P, ab, 1);
        CK(cudaStreamSynchronize(h->stream));
        check_launch();
    });
}

int lsb_nlterm(lsb_handle* h, const double* uif, double* nltermif) {
    return guard([&] {
        const long long S = h->d.S();
        to_dev(h, uif, h->io, 3 * S);
        nlterm(h, h->io, h->io + 3 * S);
        from_dev(h, h->io + 3 * S, nltermif, 3 * S);
    });
}

int lsb_tau_sgs(lsb_handle* h, const double* ui, const double* uiuj, const double* duidxj, double* tauij) {
    return guard([&] {
        if (h->cfg.sgsflag != 1) fail(LSB_ERR_STATE, "handle was created without sgsflag = 1");
        const long long P = h->P;
        const size_t F = (size_t)(h->d.nx + 2) * h->d.ny * h->d.nzp;  // host field size
        // ui: 3 fields; uiuj, duidxj, tauij: 9 fields in Fortran order (..., l, m), l fastest;
        // on the device tensor component (l, m) is field 3*l + m
        to_dev_phys(h, ui, h->phys, 3);
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m) {
                to_dev_phys(h, duidxj + (l + 3 * m) * F, h->phys + (3 + 3 * l + m) * P, 1);
                to_dev_phys(h, uiuj + (l + 3 * m) * F, h->phys + (12 + 3 * l + m) * P, 1);
            }
        sgs_tau_phys(h, h->phys, h->phys + 3 * P, h->phys + 12 * P, h->sgs.tau);
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m) from_dev_phys(h, h->sgs.tau + (3 * l + m) * P, tauij + (l + 3 * m) * F, 1);
        CK(cudaStreamSynchronize(h->stream));
        check_launch();
    });
}

int lsb_tavg(lsb_handle* h, double* uf, double* vf, double* wf, double* pf, int reset) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        if (!h->tavg) fail(LSB_ERR_STATE, "handle was created without otfavg = 1");
        const long long S = h->d.S();
        double* outs[4] = {uf, vf, wf, pf};
        for (int k = 0; k < 4; ++k)
            if (outs[k]) CK(cudaMemcpyAsync(outs[k], h->tavg + k * S, S * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (reset) CK(cudaMemsetAsync(h->tavg, 0, 4 * S * sizeof(double), h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

int lsb_spanwise_stats(lsb_handle* h, double* mean, double* rms) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        if (!mean || !rms) fail(LSB_ERR_ARG, "null output");
        const Dims& d = h->d;
        const long long S = d.S(), P = h->P, n = 4LL * d.nzp * d.nx;
        // u + ubar, v, w, p on the physical grid in the first four scratch fields (FP64 in
        // both precisions), the profiles after them
        double* ph[4] = {h->phys, h->phys + P, h->phys + 2 * P, h->phys + 3 * P};
        const double* spec[4] = {h->vel, h->vel + S, h->vel + 2 * S, h->p};
        const double* means[4] = {h->ubar, nullptr, nullptr, nullptr};
        spec_to_phys(h, spec, ph, 4, d.nzp, means, nullptr, false);
        double* dm = h->phys + 4 * P;
        double* dr = dm + n;
        launch_spanwise_stats(h->phys, dm, dr, 4, d.nx, d.ny, d.nzp, P, h->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(mean, dm, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(rms, dr, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

int lsb_snapshot_async(lsb_handle* h, double* q) {
    return guard([&] {
        if (!h || !q) fail(LSB_ERR_ARG, "null argument");
        const Dims& d = h->d;
        const long long S = d.S(), P = h->P;
        // the fields of spanwise_stats: u + ubar, v, w, p on the physical grid (FP64 in both
        // precisions) in the first four scratch fields, then copied out without waiting
        double* ph[4] = {h->phys, h->phys + P, h->phys + 2 * P, h->phys + 3 * P};
        const double* spec[4] = {h->vel, h->vel + S, h->vel + 2 * S, h->p};
        const double* means[4] = {h->ubar, nullptr, nullptr, nullptr};
        spec_to_phys(h, spec, ph, 4, d.nzp, means, nullptr, false);
        check_launch();
        const long long n = (long long)d.nzp * d.ny * d.nx;
        for (int k = 0; k < 4; ++k)
            CK(cudaMemcpyAsync(q + k * n, ph[k], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    });
}

int lsb_timers(lsb_handle* h, int enable) {
    return guard([&] {
        if (!h) fail(LSB_ERR_ARG, "null handle");
        CK(cudaStreamSynchronize(h->stream));
        if (enable) {
            for (auto& kv : h->timers)
                for (auto& ev : kv.second) {
                    cudaEventDestroy(ev.first);
                    cudaEventDestroy(ev.second);
                }
            h->timers.clear();
        }
        h->timing = enable != 0;
    });
}

int lsb_timer_report(lsb_handle* h, char* buf, int buflen) {
    return guard([&] {
        if (!h || !buf || buflen <= 0) fail(LSB_ERR_ARG, "null argument");
        CK(cudaStreamSynchronize(h->stream));
        std::string s;
        for (auto& kv : h->timers) {
            double tot = 0.0;
            for (auto& ev : kv.second) {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, ev.first, ev.second));
                tot += ms;
            }
            s += kv.first + " " + std::to_string(kv.second.size()) + " " + std::to_string(tot) + "\n";
        }
        std::strncpy(buf, s.c_str(), (size_t)buflen - 1);
        buf[buflen - 1] = 0;
    });
}

int lsb_upload_velocity(lsb_handle* h, const double* uf, const double* vf, const double* wf) {
    return guard([&] {
        if (!h || !uf || !vf || !wf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        CK(cudaMemcpyAsync(h->vel, uf, S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->vel + S, vf, S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->vel + 2 * S, wf, S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    });
}

int lsb_download_velocity(lsb_handle* h, double* uf, double* vf, double* wf) {
    return guard([&] {
        if (!h || !uf || !vf || !wf) fail(LSB_ERR_ARG, "null argument");
        const long long S = h->d.S();
        CK(cudaMemcpyAsync(uf, h->vel, S * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(vf, h->vel + S, S * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(wf, h->vel + 2 * S, S * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    });
}

int lsb_diag(lsb_handle* h, lsb_diagnostics* out) {
    return guard([&] {
        if (!h || !out) fail(LSB_ERR_ARG, "null argument");
        diag_compute(h, out);
    });
}

}  // extern "C"
