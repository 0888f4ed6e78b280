// Argument blocks of the elementwise kernels (spectral_kernels.cu).
#pragma once
#include "lsb_internal.cuh"

namespace lsb {

struct SpecFilterArgs {
    const double* in[3];
    double* out[3];
    long long S, C;
    int nx;
    const double* wavx;
    const double* wavy;
    double akc, akmax, amp, order;
};

struct RhsArgs {
    double* rhs[3];
    const double* N[3];
    const double* nln[3];
    const double* nlnm[3];
    const double* u[3];
    const double* un[3];
    const double* unm[3];
    double ab[3], bdf[3];
    double dt, dtnui;
    const double* ubarpp;
    long long S, C;
};

struct BcArgs {
    double* bc[3];            // [2][C] each: ceiling plane, wall plane
    double* bcp;              // [2][C] w boundary field of the pressure step
    const double* rtop[3];    // ceiling planes of the velocity right-hand sides
    const double* pwall;      // wall plane of p^n
    const double* pnwall;     // wall plane of p^(n-1)
    int top_free;             // 1: u' = v = 0 on the ceiling (bctype 3, bc3_top = 1)
    const double* w;          // w^n ([nzp][C]): rows 1 and nzp of its d2fdz2 are formed in the kernel
    const double* d2rows;     // the two rows of the Chebyshev second derivative, row stride d2ld
    int d2ld, nzp;
    const double* btop;       // spectral shape planes of bound(), or null
    const double* bwa;
    const double* bwb;
    double ctop, cwa, cwb;
    double pfac0, pfac1, dt, bdfv, dtnui, xnu;
    int active;
    const double* wavx;
    const double* wavy;
    int nx;
    long long C;
};

// the nonlinear term's divergence operands: N_l and the fluxes h_l1, h_l2 (d h_l3/dz is
// formed and subtracted by the contraction's EPI_NLDIV epilogue)
struct NlDivArgs {
    double* N[3];
    const double* hx[3];
    const double* hy[3];
};

void launch_specfilter(const SpecFilterArgs& a, cudaStream_t s);
void launch_rhs(const RhsArgs& a, cudaStream_t s);
void launch_bc_planes(const BcArgs& a, cudaStream_t s);
void launch_divuv(const double* u, const double* v, double* out, const double* wavx, const double* wavy, int nx,
                  long long S, long long C, cudaStream_t s);
void launch_dxy(const double* in, double* out, const double* wavx, const double* wavy, int nx, long long S,
                long long C, int mode, cudaStream_t s);
void launch_lapl_xy(const double* u, double* d2, const double* wavx, const double* wavy, int nx, long long S,
                    long long C, cudaStream_t s);
void launch_norm(double* f0, double* f1, double* f2, int nx, int ny, int nzp, int ifrz, cudaStream_t s);
void launch_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t s);
void launch_tavg_add(double* a, const double* q, double iomod, long long n, cudaStream_t s);
void launch_add_half_sq(double* h11, const double* ubar, long long C, int nzp, cudaStream_t s);

}  // namespace lsb
