// Internal declarations of the LSBFLOW B200 time-step library.
//
// Device data layout (all FP64, reference ordering, i fastest):
//   spectral field  : [nzp][ny][nx]       nx reals = nx/2 complex kx modes (Re, Im interleaved),
//                                          ky in FFT order, k = 0 the ceiling, k = nzp-1 the wall
//   y-intermediate  : [nzp][nyl][nx]      after the spanwise transform: kx modes per physical y row
//   physical field  : [nzp][ny][nx]       no pad columns on the device (the reference's two pad
//                                          columns hold nothing any result depends on)
// nyl / nxl are the 3/2-rule padded sizes when dealiasflag == 1, else ny / nx.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace lsb {

// counts every kernel launch of the library (lsb_kernel_launches)
void note_launch();
void note_launches(long long n);       // n kernels run by a replayed graph (n < 0: a capture undone)
unsigned long long launches_so_far();

// resident blocks of a kernel on one SM for a block size and dynamic shared memory,
// queried once per (device, kernel, threads, shared memory) and cached; the first query
// also raises the kernel's dynamic shared memory limit to 200 KB
int resident_blocks(const void* kern, int threads, size_t smem);
// SMs of the current device (cached per device)
int sm_count();
// opt-in maximum of dynamic shared memory per block on the current device (cached)
size_t smem_optin();
// raises a kernel's dynamic shared memory limit to smem (once per device, kernel and size);
// false, with the CUDA error cleared, when the device refuses it
bool allow_smem(const void* kern, size_t smem);

constexpr int kMaxStages = 16;

// exact unsigned division by a constant: q = (umulhi(n, m) + n) >> s  (d > 1), valid for
// the n < 2^31 used here
struct FastDiv {
    uint32_t d = 1, m = 0, s = 0;
};

// One complex FFT length: radix schedule + twiddle table tw[m] = exp(-2 pi i m / n).
// Per stage st: p = product of the radices before it, T = n / R, stride = n / (p R).
struct FftPlan {
    int n = 0;
    int nst = 0;
    int radix[kMaxStages] = {0};
    int p[kMaxStages] = {0};
    FastDiv fdT[kMaxStages];
    FastDiv fdP[kMaxStages];
    const double2* tw = nullptr;   // device, n entries
    const float2* twf = nullptr;   // the same in FP32
    int n1 = 0, n2 = 0;            // register two-pass split n = n1*n2 (n1 = 0: Stockham stages)
    int g = 0, r = 0, lgg = 0;     // warp-group split n = g*r (g lanes, r registers; g = 0: none)
    int ls = 0;                    // shared-memory line stride (complex) a kernel must use
};

// A real transform of length nr (even) done through a complex FFT of length nr/2.
struct RealPlan {
    int nr = 0;                    // real length
    FftPlan half;                  // complex plan of length nr/2
    const double2* twr = nullptr;  // device, nr entries: exp(-2 pi i m / nr)
    const float2* twrf = nullptr;  // the same in FP32
};

struct Dims {
    int nx = 0, ny = 0, nz = 0, nzp = 0, nzm = 0;
    int kx = 0;            // nx/2 stored complex kx modes
    int nxl = 0, nyl = 0;  // transform grid (padded when dealiasing)
    long long S() const { return (long long)nx * ny * nzp; }
    long long C() const { return (long long)nx * ny; }
};

// ---------------------------------------------------------------- FFT passes (fft_kernels.cu)
// multiplier applied to a spectral column before the y inverse transform
enum YMode { YM_COPY = 0, YM_IKY = 1, YM_IKX = 2 };

struct YInvJob {
    const double* in;   // spectral [nzp][ny][nx]
    double* out;        // y-intermediate [nzp][nyl][nx]
    int mode;
};
struct YFwdJob {
    const double* in;   // y-intermediate [nzp][nyl][nx]
    double* out;        // spectral [nzp][ny][nx]
    double alpha;       // out = alpha * T(in) + beta * out
    double beta;
    int sym;            // apply the kx = 0 Hermitian symmetrisation of the horfft round trip
};

struct YPassArgs {
    int ny, nyl, kxc, nzp, nx;  // kxc = number of complex kx columns
    int layout;                 // 0 = reference layout, 1 = correct 3/2 layout
    double scale;               // forward only: 1/(nxl*nyl)
    const double* wavy;         // [ny] device
    const double* wavx;         // [nx] device
    FftPlan plan;               // length nyl
    int f32 = 0;                // 1: y-intermediates in FP32, transforms in FP32 (mixed form)
    int y_tma = 0;              // FP64 tiles staged by TMA tile loads (1) or by cp.async (0)
    int* err = nullptr;         // raised when a bounded wait of a TMA-staged pass timed out
};

constexpr int kMaxJobs = 12;
struct YInvJobList { int n; YInvJob j[kMaxJobs]; };
struct YFwdJobList { int n; YFwdJob j[kMaxJobs]; };
void launch_yinv(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s);
void launch_yfwd(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s);

// row transforms between y-intermediate rows (kxc complex modes) and physical rows (nxl reals)
struct RowIO {
    const double* yin;  // y-intermediate source (c2r) or physical source (r2c)
    double* out;
    int mode;           // YM_COPY or YM_IKX (c2r only)
    double add_mean;    // c2r only: 0 or 1 -> add mean[k] to the physical row (u + ubar)
    const double* mean; // [nzp] or nullptr
    double scale;       // c2r only: the physical row is scale * c2r (+ mean)
    const double* lam;  // r2c only: fringe lambda(x) [nxl] or nullptr; the row read is then
                        // lambda(x) (m - q(x)), m = mean[z] * add_mean (or 0), before the transform
};
struct RowArgs {
    int f32 = 0;                // 1: y-intermediate and physical rows in FP32 (mixed form)
    int kxc, nxl, nyl, nzp;
    long long row_pitch;        // physical row pitch in doubles (nxl)
    const double* wavx;
    RealPlan rp;
};
struct RowJobList { int n; RowIO j[kMaxJobs]; };
void launch_row_c2r(const RowJobList& jobs, const RowArgs& a, cudaStream_t s);
void launch_row_r2c(const RowJobList& jobs, const RowArgs& a, cudaStream_t s);

// the unpadded row pass of the dynamic SGS model's physical fields, with the model's first
// pointwise pass fused in: u_l, S_ij and delta^2 |S| S_ij from the y-intermediates
struct DynRowArgs {
    RowArgs r;
    const double* yu[3];   // y-intermediates of u_l (also the source of du_l/dx, with ikx)
    const double* ydy[3];  // of du_l/dy
    const double* ydz[3];  // of du_l/dz
    double* u[3];          // physical u_l (u_1 + ubar)
    double* uprime;        // or null: u_1 without the mean as well (the mixed form's forcing)
    double* sij[6];        // S_ij for (11, 12, 13, 22, 23, 33)
    double* lij[6];        // delta^2 |S| S_ij
    const double* ubar;    // [nzp], added to u_1
    const double* ubarp;   // [nzp], added to du_1/dz
    const double* delta;   // [nzp], the model's filter width
};
// whether the unpadded row plan has the fused form (full-warp groups, even R)
bool row_c2r_dyn_plan(const RowArgs& r);
void launch_row_c2r_dyn(const DynRowArgs& a, cudaStream_t s);

// the forward row pass of the dynamic model's stresses with its last pointwise pass fused in:
// tau_ij = -2 nu S_ij, nu = C delta^2 |S| with C the clipped ratio of the filtered
// contractions, transformed straight from S_ij into the y-intermediates
struct TauRowArgs {
    RowArgs r;
    const double* sij[6];  // S_ij for (11, 12, 13, 22, 23, 33)
    const double* ctot;    // filtered <L M>
    const double* cdd;     // filtered <M M>
    const double* delta;   // [nzp]
    double* out[6];        // y-intermediate rows of tau_ij
};
bool row_r2c_tau_plan(const RowArgs& r);
void launch_row_r2c_tau(const TauRowArgs& a, cudaStream_t s);

// the fused nonlinear-product row kernel
struct NlRowArgs {
    RowArgs r;
    const double* U[3];   // y-intermediate velocities
    const double* DY[3];  // y-intermediate d/dy
    const double* DZ[3];  // y-intermediate d/dz
    double* N[3];         // y-intermediate outputs: -0.5 u_m d_m u_l (+ forcing)
    double* H[6];         // y-intermediate outputs: 0.5 u_l u_m for (11,12,13,22,23,33)
    const double* ubar;   // [nzp]
    const double* ubarp;  // [nzp]
    const double* lamx;   // [nxl] fringe lambda(x) or nullptr (only on the unpadded grid)
};
void launch_row_nl(const NlRowArgs& a, cudaStream_t s);

// warp-group register FFT variants (fft_warp.cu); they return false when the plan has no
// warp split, in which case the block-batched kernels of fft_kernels.cu run instead
bool launch_yinv_warp(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s);
bool launch_yfwd_warp(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s);
bool launch_row_c2r_warp(const RowJobList& jobs, const RowArgs& a, cudaStream_t s);
bool launch_row_r2c_warp(const RowJobList& jobs, const RowArgs& a, cudaStream_t s);
bool launch_row_nl_warp(const NlRowArgs& a, cudaStream_t s);

// ---------------------------------------------------------------- z contractions (gemm_kernels.cu)
// out[f][r][c] = epi( sum_k A[r][k] * in[f][k + koff][c] ) for r < M (rows written at r + roff)
enum GemmEpi {
    EPI_STORE = 0,          // out = acc
    EPI_AXPBY = 1,          // out = alpha*acc + beta*out
    EPI_HELM_SCALE = 2,     // out = acc / (lam[r] - w2(c) - sigma)
    EPI_POISSON_RHS = 4,    // out = -acc - w2(c)*aux
    EPI_LIFT_ADD = 5,       // out = acc + hb[row]*bcb(c) + ht[row]*bct(c)   (bcb may be null)
    EPI_NLDIV = 6,          // acc = d h_l3/dz is not stored: N_l -= d h_l1/dx + d h_l2/dy + acc
                            // (field f = l; nd_N, nd_hx, nd_hy; the elementwise divergence pass)
    EPI_PRESSURE = 7,       // acc = Dw is not stored: pressure phi = -(acc + div)/(k^2 dt bdfv)
                            // into pp_p, u -= dt bdfv dphi/dx, v -= dt bdfv dphi/dy (one field)
};
struct GemmArgs {
    const double* A;        // device, [Mp][Kp] zero padded
    int M, K, Mp, Kp;
    const double* in;       // field base
    long long in_fstride;
    int koff;               // first input row
    double* out;
    long long out_fstride;
    int roff;               // first output row
    long long C;            // columns per plane (nx*ny)
    int nfields;
    int epi;
    double alpha, beta, sigma, coef;
    const double* lam;      // EPI_HELM_SCALE
    const double* aux;      // EPI_POISSON_RHS: aux field (same layout as out)
    const double* wavx;     // [nx]
    const double* wavy;     // [ny]
    int nx;
    // lift prologue (solve_nhom_helmholtz): in' = in - abot(k,c)*bcb(c) - atop(k,c)*bct(c)
    const double* bcb;      // wall plane of the boundary field, or nullptr
    const double* bct;      // ceiling plane
    long long bc_fstride;
    const double* hb; const double* ht; const double* d2hb; const double* d2ht;
    double lift_sigma;
    // optional per-field pointers (fields that are not a fixed stride apart); used when set
    const double* inf[4];
    double* outf[4];
    int nw;                 // CTA width in warps, 4..8, set by the handle's schedule; 0: wave model
    // EPI_NLDIV: per field l, the nonlinear term updated in place and the fluxes h_l1, h_l2
    double* nd_N[3];
    const double* nd_hx[3];
    const double* nd_hy[3];
    // EPI_PRESSURE: the velocity updated in place, the pressure written, the divergence read
    double* pp_u;
    double* pp_v;
    double* pp_p;
    const double* pp_div;
    double pp_dt, pp_bdfv;
};
void launch_gemm(const GemmArgs& g, cudaStream_t s);
// the FP64 Helmholtz solve in one launch: g1 = E^-1 with the lifted right-hand side and the
// Helmholtz scale (EPI_HELM_SCALE), g2 = E with the boundary rows and the lift (EPI_LIFT_ADD,
// its input is g1's output); the intermediate stays in registers.  false when the shapes
// have no fused form (the caller then launches the two contractions)
bool launch_helm_fused(const GemmArgs& g1, const GemmArgs& g2, cudaStream_t s);
void launch_spanwise_stats(const double* ph, double* mean, double* rms, int nf, int nx, int ny, int nzp, long long P,
                           cudaStream_t s);

// mixed form: z contractions on the int8 tensor cores, operands split into int8 digits with
// power-of-two scales (ozaki_kernels.cu)
struct OzMat {
    const uint8_t* img = nullptr;   // device: matrix digits in the shared-memory image
    const double* rscale = nullptr; // device [nmma]: 2^e_r per row
    const double* arow = nullptr;   // device [K]: FP64 row 128 (M == 129), or null
    const double* acol = nullptr;   // device [128]: FP64 column 128 (K == 129), or null
    unsigned img_bytes = 0;
    int M = 0, K = 0, nmma = 0, kin = 0, ksteps = 0;
    int digits = 0;                 // int8 digits per operand (5)
};
struct OzHost {                     // the host side of an OzMat, before upload
    OzMat mat;
    std::vector<uint8_t> img;
    std::vector<double> rscale, arow, acol;
};
// false when M or K is above 129 or S is not 5
bool make_ozaki_mat(const double* A, int M, int K, int S, OzHost& out);
// false when it does not apply (matrix sizes, shared memory refused)
bool launch_ozaki(const GemmArgs& g, const OzMat& om, int* err, cudaStream_t s);

}  // namespace lsb
