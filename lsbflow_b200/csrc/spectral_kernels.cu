// Elementwise spectral / physical kernels of navierstokes_update and timestep
// (src/navierstokes.f90:10-90, 1157-1496), the spectral filter of filterqspec
// (src/filters.f90:164-192, 281-360) and norm (src/horfft.f90:153-224).
// Floating-point expressions keep the reference's evaluation order.
#include "lsb_spectral.cuh"

namespace lsb {

__device__ __forceinline__ void ij_of(long long c2, int nx, int& i, int& j) {
    // c2 = complex index within a plane: (j, ic) with ic < nx/2
    const int kxc = nx / 2;
    j = (int)(c2 / kxc);
    i = 2 * (int)(c2 % kxc);
}

// ---------------------------------------------------------------- spectral filter
__global__ void k_specfilter(SpecFilterArgs a) {
    const long long n2 = a.S / 2;  // complex elements per field
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3 * n2; e += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(e / n2);
        const long long ce = e % n2;
        const long long cplane = ce % (a.C / 2);
        int i, j;
        ij_of(cplane, a.nx, i, j);
        const double fr = a.in[f][2 * ce], fi = a.in[f][2 * ce + 1];
        const double fmag = sqrt(fr * fr + fi * fi);
        double orr = 0.0, oi = 0.0;
        if (fmag != 0.0) {
            double cosc = fr / fmag;
            const double sinc = fi / fmag;
            cosc = fmin(1.0, fmax(-1.0, cosc));
            const double phase = (sinc >= 0.0) ? acos(cosc) : -acos(cosc);
            const double wx = a.wavx[i], wy = a.wavy[j];
            const double ak = sqrt(wx * wx + wy * wy);
            double filt = 1.0;
            if (fabs(ak) >= a.akc) {
                const double theta = (fabs(ak) - a.akc) / (a.akmax - a.akc);
                filt = exp(-a.amp * pow(theta, 2.0 * a.order));
            }
            const double fmagf = fmag * filt;
            orr = fmagf * cos(phase);
            oi = fmagf * sin(phase);
        }
        a.out[f][2 * ce] = orr;
        a.out[f][2 * ce + 1] = oi;
    }
}

// ---------------------------------------------------------------- velocity RHS
// rhs_l = -dtnui*(dt*(ab0 N + ab1 nln + ab2 nlnm) + bdf0 u + bdf1 un + bdf2 unm) ;
// rhs_1 -= horfft(ubarpp) (the (0,0) mode)      src/navierstokes.f90:1239,1282-1296
__global__ void k_rhs(RhsArgs a) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3 * a.S; e += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(e / a.S);
        const long long x = e % a.S;
        const double nlt = a.ab[0] * a.N[l][x] + a.ab[1] * a.nln[l][x] + a.ab[2] * a.nlnm[l][x];
        double r = -a.dtnui * (a.dt * nlt + a.bdf[0] * a.u[l][x] + a.bdf[1] * a.un[l][x] + a.bdf[2] * a.unm[l][x]);
        if (l == 0 && (x % a.C) == 0) r = r - a.ubarpp[x / a.C];
        a.rhs[l][x] = r;
    }
}

// ---------------------------------------------------------------- boundary planes
// Zang-Hussaini BCs of src/navierstokes.f90:1320-1373; bc[f][0] = ceiling (k=1),
// bc[f][1] = wall (k=nzp).  Bound planes = c_top*btop, c_wa*bwa + c_wb*bwb.
// The ceiling and wall rows of d2fdz2(w^n) (src/navierstokes.f90:1340-1345) are formed here:
// a block owns BC_MODES (kx, ky) modes, warp s sums the z points k = s, s + 16, ... of both
// rows for its lane's mode (each z row of the field read as contiguous 16-byte modes), the
// sixteen partial sums meet in shared memory and warp 0 writes the planes.
constexpr int BC_MODES = 32, BC_SLICES = 16;
__global__ void __launch_bounds__(BC_MODES * BC_SLICES) k_bc_planes(BcArgs a) {
    __shared__ double2 part[BC_SLICES][2][BC_MODES];
    const int lane = threadIdx.x & (BC_MODES - 1), sl = threadIdx.x / BC_MODES;
    const long long n2 = a.C / 2;
    const long long e = (long long)blockIdx.x * BC_MODES + lane;
    double2 p0 = make_double2(0.0, 0.0), p1 = make_double2(0.0, 0.0);
    if (e < n2) {
        const double2* w = reinterpret_cast<const double2*>(a.w);
#pragma unroll 8
        for (int k = sl; k < a.nzp; k += BC_SLICES) {
            const double2 wk = w[(long long)k * n2 + e];
            const double d0 = a.d2rows[k], d1 = a.d2rows[a.d2ld + k];
            p0.x = fma(d0, wk.x, p0.x);
            p0.y = fma(d0, wk.y, p0.y);
            p1.x = fma(d1, wk.x, p1.x);
            p1.y = fma(d1, wk.y, p1.y);
        }
    }
    part[sl][0][lane] = p0;
    part[sl][1][lane] = p1;
    __syncthreads();
    if (sl == 0 && e < n2) {
        double2 d2t = part[0][0][lane], d2b = part[0][1][lane];  // ceiling and wall rows
#pragma unroll
        for (int t = 1; t < BC_SLICES; ++t) {
            d2t.x += part[t][0][lane].x;
            d2t.y += part[t][0][lane].y;
            d2b.x += part[t][1][lane].x;
            d2b.y += part[t][1][lane].y;
        }
        int i, j;
        ij_of(e, a.nx, i, j);
        const double wx = a.wavx[i], wy = a.wavy[j];
        const double w2 = wx * wx + wy * wy;
        const long long re = 2 * e, im = 2 * e + 1;
        const double den = w2 + a.dtnui / a.bdfv;
        const double psr = a.pfac0 * a.pwall[re] + a.pfac1 * a.pnwall[re];
        const double psi = a.pfac0 * a.pwall[im] + a.pfac1 * a.pnwall[im];
        const double dtb = a.dt * a.bdfv;
        // u, v: the ceiling row of the momentum equation without z diffusion (the reference),
        // or the free stream (u' = v = 0 in the velocity solves)
        if (a.top_free) {
            a.bc[0][re] = a.bc[0][im] = 0.0;
            a.bc[1][re] = a.bc[1][im] = 0.0;
        } else {
            a.bc[0][re] = -a.rtop[0][re] / den;
            a.bc[0][im] = -a.rtop[0][im] / den;
            a.bc[1][re] = -a.rtop[1][re] / den;
            a.bc[1][im] = -a.rtop[1][im] / den;
        }
        a.bc[0][a.C + re] = dtb * (-wx * psi);
        a.bc[0][a.C + im] = dtb * (wx * psr);
        a.bc[1][a.C + re] = dtb * (-wy * psi);
        a.bc[1][a.C + im] = dtb * (wy * psr);
        // w
        const double zh = a.xnu * a.dt * a.bdfv;
        if (a.active) {
            double tr = 0.0, ti = 0.0, wr = 0.0, wi = 0.0;
            if (a.btop) { tr = a.ctop * a.btop[re]; ti = a.ctop * a.btop[im]; }
            if (a.bwa) { wr = a.cwa * a.bwa[re]; wi = a.cwa * a.bwa[im]; }
            if (a.bwb) { wr += a.cwb * a.bwb[re]; wi += a.cwb * a.bwb[im]; }
            a.bc[2][re] = tr + zh * d2t.x;
            a.bc[2][im] = ti + zh * d2t.y;
            a.bc[2][a.C + re] = wr;
            a.bc[2][a.C + im] = wi;
            // the pressure step's w BC (bound() again, src/navierstokes.f90:1432-1433)
            a.bcp[re] = tr;
            a.bcp[im] = ti;
            a.bcp[a.C + re] = wr;
            a.bcp[a.C + im] = wi;
        } else {
            a.bc[2][re] = zh * d2t.x;
            a.bc[2][im] = zh * d2t.y;
            a.bc[2][a.C + re] = zh * d2b.x;
            a.bc[2][a.C + im] = zh * d2b.y;
            a.bcp[re] = 0.0;
            a.bcp[im] = 0.0;
            a.bcp[a.C + re] = 0.0;
            a.bcp[a.C + im] = 0.0;
        }
    }
}

// ---------------------------------------------------------------- small spectral ops
__global__ void k_divuv(const double* __restrict__ u, const double* __restrict__ v, double* __restrict__ out,
                        const double* __restrict__ wavx, const double* __restrict__ wavy, int nx, long long S,
                        long long C) {
    const long long n2 = S / 2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n2; e += (long long)gridDim.x * blockDim.x) {
        int i, j;
        ij_of(e % (C / 2), nx, i, j);
        const double wx = wavx[i], wy = wavy[j];
        const double ur = u[2 * e], ui = u[2 * e + 1], vr = v[2 * e], vi = v[2 * e + 1];
        out[2 * e] = -wx * ui - wy * vi;
        out[2 * e + 1] = wx * ur + wy * vr;
    }
}

// out = d/dx (mode 0), d/dy (mode 1) of in; lapl uses k_lapl_xy
__global__ void k_dxy(const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ wavx,
                      const double* __restrict__ wavy, int nx, long long S, long long C, int mode) {
    const long long n2 = S / 2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n2; e += (long long)gridDim.x * blockDim.x) {
        int i, j;
        ij_of(e % (C / 2), nx, i, j);
        const double w = (mode == 0) ? wavx[i] : wavy[j];
        const double r = in[2 * e], im = in[2 * e + 1];
        out[2 * e] = -w * im;
        out[2 * e + 1] = w * r;
    }
}

// lapl: out = d2 - (wavxx + wavyy)*u  (src/derivatives.f90:319-323)
__global__ void k_lapl_xy(const double* __restrict__ u, double* __restrict__ d2, const double* __restrict__ wavx,
                          const double* __restrict__ wavy, int nx, long long S, long long C) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S; e += (long long)gridDim.x * blockDim.x) {
        const long long c = e % C;
        const int i = (int)(c % nx), j = (int)(c / nx);
        const double wx = wavx[i], wy = wavy[j];
        d2[e] = d2[e] - (wx * wx + wy * wy) * u[e];
    }
}

// norm (src/horfft.f90:153-224) on 3 fields + the ifrz mean removal (src/navierstokes.f90:53-59)
__global__ void k_norm(double* f0, double* f1, double* f2, int nx, int ny, int nzp, int ifrz) {
    const int k = blockIdx.x;
    double* f = (blockIdx.y == 0) ? f0 : (blockIdx.y == 1 ? f1 : f2);
    double* pl = f + (long long)k * nx * ny;
    const int nyh = ny / 2;
    if (threadIdx.x == 0) pl[1] = 0.0;
    if (ny > 2) {
        // the pairs (ky, -ky) of the kx = 0 column are disjoint (rows 1..nyh-1 and
        // nyh+1..ny-1): one thread per pair, the reference's two loops in that order
        for (int jj = 1 + threadIdx.x; jj <= nyh - 1; jj += blockDim.x) {
            const int jp = ny - jj;
            const double re = 0.5 * (pl[jj * nx + 0] + pl[jp * nx + 0]);
            const double im = 0.5 * (pl[jj * nx + 1] - pl[jp * nx + 1]);
            pl[jj * nx + 0] = re;
            pl[jj * nx + 1] = im;
            pl[jp * nx + 0] = re;
            pl[jp * nx + 1] = -im;
        }
        for (int i = threadIdx.x; i < nx; i += blockDim.x) pl[nyh * nx + i] = 0.0;
    }
    __syncthreads();
    if (ifrz && threadIdx.x == 0) {
        pl[0] = 0.0;
        pl[1] = 0.0;
    }
}

__global__ void k_tavg_add(double* __restrict__ a, const double* __restrict__ q, double iomod, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        a[e] = a[e] + q[e] / iomod;
}

__global__ void k_axpby(double* __restrict__ y, const double* __restrict__ x, double a, double b, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = a * x[e] + (b != 0.0 ? b * y[e] : 0.0);
}

// spanwise mean and rms over y of nf physical fields [nzp][ny][nx] -> [nf][nzp][nx] each;
// one thread per (field, z, x), consecutive x coalesced; rms about the mean (two passes)
__global__ void k_spanwise_stats(const double* __restrict__ ph, double* __restrict__ mean, double* __restrict__ rms,
                                 int nf, int nx, int ny, int nzp, long long P) {
    const long long n = (long long)nf * nzp * nx;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % nx);
        const long long fz = e / nx;
        const int z = (int)(fz % nzp), f = (int)(fz / nzp);
        const double* col = ph + f * P + (long long)z * ny * nx + x;
        double s = 0.0;
        for (int y = 0; y < ny; ++y) s += col[(long long)y * nx];
        const double m = s / ny;
        double s2 = 0.0;
        for (int y = 0; y < ny; ++y) {
            const double d = col[(long long)y * nx] - m;
            s2 += d * d;
        }
        mean[e] = m;
        rms[e] = sqrt(s2 / ny);
    }
}

// ---------------------------------------------------------------- launchers
static inline int nblk(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 16) b = 148LL * 16;
    if (b < 1) b = 1;
    return (int)b;
}

void launch_specfilter(const SpecFilterArgs& a, cudaStream_t s) { lsb::note_launch(); k_specfilter<<<nblk(3 * a.S / 2), 256, 0, s>>>(a); }
void launch_rhs(const RhsArgs& a, cudaStream_t s) { lsb::note_launch(); k_rhs<<<nblk(3 * a.S), 256, 0, s>>>(a); }
void launch_bc_planes(const BcArgs& a, cudaStream_t s) {
    lsb::note_launch();
    k_bc_planes<<<(unsigned)((a.C / 2 + BC_MODES - 1) / BC_MODES), BC_MODES * BC_SLICES, 0, s>>>(a);
}
void launch_divuv(const double* u, const double* v, double* out, const double* wavx, const double* wavy, int nx,
                  long long S, long long C, cudaStream_t s) {
    { lsb::note_launch(); k_divuv<<<nblk(S / 2), 256, 0, s>>>(u, v, out, wavx, wavy, nx, S, C); }
}
void launch_dxy(const double* in, double* out, const double* wavx, const double* wavy, int nx, long long S,
                long long C, int mode, cudaStream_t s) {
    { lsb::note_launch(); k_dxy<<<nblk(S / 2), 256, 0, s>>>(in, out, wavx, wavy, nx, S, C, mode); }
}
void launch_lapl_xy(const double* u, double* d2, const double* wavx, const double* wavy, int nx, long long S,
                    long long C, cudaStream_t s) {
    { lsb::note_launch(); k_lapl_xy<<<nblk(S), 256, 0, s>>>(u, d2, wavx, wavy, nx, S, C); }
}
void launch_norm(double* f0, double* f1, double* f2, int nx, int ny, int nzp, int ifrz, cudaStream_t s) {
    { lsb::note_launch(); k_norm<<<dim3(nzp, 3), 128, 0, s>>>(f0, f1, f2, nx, ny, nzp, ifrz); }
}

// mixed form: the FP32 product kernel leaves 0.5 ubar(z)^2 out of h_11; its (kx, ky) = (0, 0)
// coefficient is restored here in FP64 (the dynamic model filters u_1 u_1 in physical space)
__global__ void k_add_half_sq(double* h11, const double* ubar, long long C, int nzp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nzp) h11[(long long)k * C] += 0.5 * (ubar[k] * ubar[k]);
}
void launch_add_half_sq(double* h11, const double* ubar, long long C, int nzp, cudaStream_t s) {
    { lsb::note_launch(); k_add_half_sq<<<(nzp + 127) / 128, 128, 0, s>>>(h11, ubar, C, nzp); }
}

void launch_tavg_add(double* a, const double* q, double iomod, long long n, cudaStream_t s) {
    { lsb::note_launch(); k_tavg_add<<<nblk(n), 256, 0, s>>>(a, q, iomod, n); }
}
void launch_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t s) {
    { lsb::note_launch(); k_axpby<<<nblk(n), 256, 0, s>>>(y, x, a, b, n); }
}

void launch_spanwise_stats(const double* ph, double* mean, double* rms, int nf, int nx, int ny, int nzp, long long P,
                           cudaStream_t s) {
    lsb::note_launch();
    k_spanwise_stats<<<nblk((long long)nf * nzp * nx), 256, 0, s>>>(ph, mean, rms, nf, nx, ny, nzp, P);
}

}  // namespace lsb
