// Batched FP64 FFT passes of the horizontal transforms (the reference's horfft,
// src/horfft.f90:61-150, and the padded passes of dealiasing_2d_fftw,
// src/dealiasing.f90:262-447), written as three kinds of kernels:
//
//   k_yinv  : spanwise inverse transform of kx columns, with the 3/2 zero pad placed
//             in the reference ("ref") or the textbook ("correct") layout and an optional
//             i*ky / i*kx multiplier (dfdy / dfdx fused into the transform);
//   row     : streamwise c2r / r2c of one (z, y) row through a half-length complex FFT,
//             with the pointwise nonlinear products of nlterm_skewsym between them;
//   k_yfwd  : spanwise forward transform, truncation to ny, the 1/(nxl*nyl) scale and the
//             kx = 0 Hermitian symmetrisation of the reference's horfft(+1)/horfft(-1)
//             round trip, accumulated into the output as alpha*T + beta*out.
//
// The complex FFT of a line is a mixed-radix (2,3,4,5,7,8) Stockham autosort transform in
// shared memory owned by one warp.  FFTW's c2r semantics are kept: the imaginary parts of
// the DC and Nyquist inputs are ignored and the kx Nyquist mode is dropped / zero.
#include "lsb_internal.cuh"

namespace lsb {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// R-point DFT of u in registers, U[s] = sum_q u[q] exp(SIGN 2 pi i q s / R)
template <int R, int SIGN>
__device__ __forceinline__ void dft_small(double2 (&u)[R], const double2* __restrict__ tw, int n) {
    if constexpr (R == 2) {
        double2 a = u[0], b = u[1];
        u[0] = cadd(a, b);
        u[1] = csub(a, b);
    } else if constexpr (R == 4) {
        double2 a = cadd(u[0], u[2]), b = csub(u[0], u[2]);
        double2 c = cadd(u[1], u[3]), d = csub(u[1], u[3]);
        u[0] = cadd(a, c);
        u[2] = csub(a, c);
        if (SIGN < 0) {  // -i * d = (d.y, -d.x)
            u[1] = make_double2(b.x + d.y, b.y - d.x);
            u[3] = make_double2(b.x - d.y, b.y + d.x);
        } else {
            u[1] = make_double2(b.x - d.y, b.y + d.x);
            u[3] = make_double2(b.x + d.y, b.y - d.x);
        }
    } else {
        double2 U[R];
        const int step = n / R;
#pragma unroll
        for (int s = 0; s < R; ++s) {
            double2 acc = u[0];
#pragma unroll
            for (int q = 1; q < R; ++q) {
                double2 w = __ldg(&tw[((q * s) % R) * step]);
                if (SIGN > 0) w.y = -w.y;
                acc = cadd(acc, cmul(u[q], w));
            }
            U[s] = acc;
        }
#pragma unroll
        for (int s = 0; s < R; ++s) u[s] = U[s];
    }
}

template <int R, int SIGN>
__device__ __forceinline__ void fft_stage(const double2* __restrict__ src, double2* __restrict__ dst, int n, int p,
                                          const double2* __restrict__ tw, int lane) {
    const int T = n / R;
    const int stride = n / (p * R);
    for (int i = lane; i < T; i += 32) {
        const int k = i % p;
        double2 u[R];
#pragma unroll
        for (int q = 0; q < R; ++q) u[q] = src[i + q * T];
        if (k != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                double2 w = __ldg(&tw[q * k * stride]);
                if (SIGN > 0) w.y = -w.y;
                u[q] = cmul(u[q], w);
            }
        }
        dft_small<R, SIGN>(u, tw, n);
        const int j = (i - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) dst[j + q * p] = u[q];
    }
}

// Complex FFT of one line a[0..n) by one warp; b is scratch of the same size.
// Returns the buffer holding the result (a if the stage count is even, else b).
template <int SIGN>
__device__ double2* fft_line(double2* a, double2* b, const FftPlan& P, int lane) {
    double2* src = a;
    double2* dst = b;
    int p = 1;
    for (int s = 0; s < P.nst; ++s) {
        const int R = P.radix[s];
        switch (R) {
            case 2: fft_stage<2, SIGN>(src, dst, P.n, p, P.tw, lane); break;
            case 3: fft_stage<3, SIGN>(src, dst, P.n, p, P.tw, lane); break;
            case 4: fft_stage<4, SIGN>(src, dst, P.n, p, P.tw, lane); break;
            case 5: fft_stage<5, SIGN>(src, dst, P.n, p, P.tw, lane); break;
            case 7: fft_stage<7, SIGN>(src, dst, P.n, p, P.tw, lane); break;
            default: fft_stage<8, SIGN>(src, dst, P.n, p, P.tw, lane); break;
        }
        __syncwarp();
        double2* t = src;
        src = dst;
        dst = t;
        p *= R;
    }
    return src;
}

__device__ __forceinline__ int pad_row(int j, int ny, int nyl, int layout) {
    if (layout == 0 || nyl == ny) return j;
    return (j < ny / 2) ? j : j + (nyl - ny);
}

constexpr int KC = 16;  // kx columns per spanwise block

// ----------------------------------------------------------------------------- k_yinv
__global__ void __launch_bounds__(256) k_yinv(YInvJobList jobs, YPassArgs a) {
    extern __shared__ double2 smem[];
    const YInvJob job = jobs.j[blockIdx.z];
    const int z = blockIdx.y;
    const int c0 = blockIdx.x * KC;
    const int nyl = a.nyl, ny = a.ny;
    double2* A = smem;
    double2* B = smem + KC * nyl;
    const int tid = threadIdx.x;
    for (int i = tid; i < KC * nyl; i += blockDim.x) A[i] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int idx = tid; idx < ny * KC; idx += blockDim.x) {
        const int j = idx / KC, cc = idx % KC, c = c0 + cc;
        if (c >= a.kxc) continue;
        const double2 v = *reinterpret_cast<const double2*>(job.in + ((long long)z * ny + j) * a.nx + 2 * c);
        double2 r = v;
        if (job.mode == YM_IKY) {
            const double k = a.wavy[j];
            r = make_double2(-k * v.y, k * v.x);
        } else if (job.mode == YM_IKX) {
            const double k = a.wavx[2 * c];
            r = make_double2(-k * v.y, k * v.x);
        }
        A[cc * nyl + pad_row(j, ny, nyl, a.layout)] = r;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int cc = warp; cc < KC; cc += blockDim.x >> 5) fft_line<+1>(A + cc * nyl, B + cc * nyl, a.plan, lane);
    const bool inA = (a.plan.nst % 2) == 0;
    __syncthreads();
    const double2* R = inA ? A : B;
    for (int idx = tid; idx < nyl * KC; idx += blockDim.x) {
        const int jl = idx / KC, cc = idx % KC, c = c0 + cc;
        if (c >= a.kxc) continue;
        *reinterpret_cast<double2*>(job.out + ((long long)z * nyl + jl) * a.nx + 2 * c) = R[cc * nyl + jl];
    }
}

// ----------------------------------------------------------------------------- k_yfwd
__global__ void __launch_bounds__(256) k_yfwd(YFwdJobList jobs, YPassArgs a) {
    extern __shared__ double2 smem[];
    const YFwdJob job = jobs.j[blockIdx.z];
    const int z = blockIdx.y;
    const int c0 = blockIdx.x * KC;
    const int nyl = a.nyl, ny = a.ny;
    double2* A = smem;
    double2* B = smem + KC * nyl;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nyl * KC; idx += blockDim.x) {
        const int jl = idx / KC, cc = idx % KC, c = c0 + cc;
        double2 v = make_double2(0.0, 0.0);
        if (c < a.kxc) v = *reinterpret_cast<const double2*>(job.in + ((long long)z * nyl + jl) * a.nx + 2 * c);
        A[cc * nyl + jl] = v;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int cc = warp; cc < KC; cc += blockDim.x >> 5) fft_line<-1>(A + cc * nyl, B + cc * nyl, a.plan, lane);
    const bool inA = (a.plan.nst % 2) == 0;
    __syncthreads();
    const double2* R = inA ? A : B;
    for (int idx = tid; idx < ny * KC; idx += blockDim.x) {
        const int j = idx / KC, cc = idx % KC, c = c0 + cc;
        if (c >= a.kxc) continue;
        double2 v = R[cc * nyl + pad_row(j, ny, nyl, a.layout)];
        if (job.sym && c == 0) {
            const int jm = (ny - j) % ny;
            const double2 w = R[cc * nyl + pad_row(jm, ny, nyl, a.layout)];
            v = make_double2(0.5 * (v.x + w.x), 0.5 * (v.y - w.y));
        }
        v.x *= a.scale;
        v.y *= a.scale;
        double2* o = reinterpret_cast<double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c);
        double2 r;
        if (job.beta != 0.0) {
            const double2 old = *o;
            r = make_double2(fma(job.alpha, v.x, job.beta * old.x), fma(job.alpha, v.y, job.beta * old.y));
        } else {
            r = make_double2(job.alpha * v.x, job.alpha * v.y);
        }
        *o = r;
    }
}

static size_t ypass_smem(const YPassArgs& a) { return (size_t)2 * KC * a.nyl * sizeof(double2); }

void launch_yinv(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    dim3 grid((a.kxc + KC - 1) / KC, a.nzp, jobs.n);
    size_t sm = ypass_smem(a);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_yinv, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    k_yinv<<<grid, 256, sm, s>>>(jobs, a);
}

void launch_yfwd(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    dim3 grid((a.kxc + KC - 1) / KC, a.nzp, jobs.n);
    size_t sm = ypass_smem(a);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_yfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    k_yfwd<<<grid, 256, sm, s>>>(jobs, a);
}

// ----------------------------------------------------------------------------- rows
// c2r of one y-intermediate row into Z (N = nxl/2 double2 = the nxl physical reals).
// X is scratch of N+1 entries (it doubles as the FFT ping-pong buffer).
__device__ void row_c2r_warp(const double* __restrict__ yrow, int mode, const double* __restrict__ wavx, int kxc,
                             double meanv, const RealPlan& rp, double2* X, double2* Z, int lane) {
    const int N = rp.nr / 2;
    for (int k = lane; k <= N; k += 32) {
        double2 v = make_double2(0.0, 0.0);
        if (k < kxc) {
            v = *reinterpret_cast<const double2*>(yrow + 2 * k);
            if (mode == YM_IKX) {
                const double kk = wavx[2 * k];
                v = make_double2(-kk * v.y, kk * v.x);
            }
        }
        if (k == 0) v = make_double2(v.x, 0.0);  // FFTW c2r ignores Im of the DC input
        X[k] = v;
    }
    __syncwarp();
    for (int k = lane; k < N; k += 32) {
        const double2 xa = X[k];
        const double2 xb = cconj(X[N - k]);
        const double2 e = cadd(xa, xb);
        const double2 o = cmul(csub(xa, xb), cconj(__ldg(&rp.twr[k])));
        Z[k] = make_double2(e.x - o.y, e.y + o.x);
    }
    __syncwarp();
    double2* r = fft_line<+1>(Z, X, rp.half, lane);
    if (r != Z) {
        for (int k = lane; k < N; k += 32) Z[k] = r[k];
        __syncwarp();
    }
    if (meanv != 0.0) {
        for (int k = lane; k < N; k += 32) {
            Z[k].x += meanv;
            Z[k].y += meanv;
        }
        __syncwarp();
    }
}

// r2c of the physical row held in Z (destroyed); writes kx modes 0..kxc-1 to yrow.
__device__ void row_r2c_warp(double2* Z, double2* X, const RealPlan& rp, int kxc, double* __restrict__ yrow,
                             int lane) {
    const int N = rp.nr / 2;
    const double2* r = fft_line<-1>(Z, X, rp.half, lane);
    for (int k = lane; k < kxc; k += 32) {
        const double2 za = r[k];
        const double2 zb = cconj(r[(N - k) % N]);
        const double2 e = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y + zb.y));
        const double2 o = make_double2(0.5 * (za.x - zb.x), 0.5 * (za.y - zb.y));
        const double2 t = cmul(__ldg(&rp.twr[k]), o);
        *reinterpret_cast<double2*>(yrow + 2 * k) = make_double2(e.x + t.y, e.y - t.x);
    }
    __syncwarp();
}

constexpr int ROW_WARPS = 4;

__global__ void __launch_bounds__(ROW_WARPS * 32) k_row_c2r(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * ROW_WARPS + warp;
    if (row >= a.nyl * a.nzp) return;
    const RowIO job = jobs.j[blockIdx.y];
    const int N = a.nxl / 2;
    double2* X = smem + warp * (2 * N + 1);
    double2* Z = X + N + 1;
    const int z = row / a.nyl;
    const double meanv = (job.mean != nullptr && job.add_mean != 0.0) ? job.mean[z] * job.add_mean : 0.0;
    row_c2r_warp(job.yin + (long long)row * 2 * a.kxc, job.mode, a.wavx, a.kxc, meanv, a.rp, X, Z, lane);
    double2* o = reinterpret_cast<double2*>(job.out + (long long)row * a.row_pitch);
    for (int k = lane; k < N; k += 32) o[k] = Z[k];
}

__global__ void __launch_bounds__(ROW_WARPS * 32) k_row_r2c(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * ROW_WARPS + warp;
    if (row >= a.nyl * a.nzp) return;
    const RowIO job = jobs.j[blockIdx.y];
    const int N = a.nxl / 2;
    double2* X = smem + warp * (2 * N + 1);
    double2* Z = X + N + 1;
    const double2* in = reinterpret_cast<const double2*>(job.yin + (long long)row * a.row_pitch);
    for (int k = lane; k < N; k += 32) Z[k] = in[k];
    __syncwarp();
    row_r2c_warp(Z, X, a.rp, a.kxc, job.out + (long long)row * 2 * a.kxc, lane);
}

void launch_row_c2r(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    const int rows = a.nyl * a.nzp;
    dim3 grid((rows + ROW_WARPS - 1) / ROW_WARPS, jobs.n);
    size_t sm = (size_t)ROW_WARPS * (a.nxl + 1) * sizeof(double2);
    k_row_c2r<<<grid, ROW_WARPS * 32, sm, s>>>(jobs, a);
}

void launch_row_r2c(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    const int rows = a.nyl * a.nzp;
    dim3 grid((rows + ROW_WARPS - 1) / ROW_WARPS, jobs.n);
    size_t sm = (size_t)ROW_WARPS * (a.nxl + 1) * sizeof(double2);
    k_row_r2c<<<grid, ROW_WARPS * 32, sm, s>>>(jobs, a);
}

// ----------------------------------------------------------------------------- NL row
// One (z, y) row per block: 12 c2r (u, du/dx, du/dy, du/dz for 3 components), the
// skew-symmetric products of nlterm_skewsym (src/navierstokes.f90:725-769), and 9 r2c.
constexpr int NL_WARPS = 8;

__global__ void __launch_bounds__(NL_WARPS * 32) k_row_nl(NlRowArgs a) {
    extern __shared__ double2 smem[];
    const RowArgs& r = a.r;
    const int N = r.nxl / 2;
    const int yl = blockIdx.x, z = blockIdx.y;
    const long long row = (long long)z * r.nyl + yl;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2* P = smem;                          // 12 rows of N double2
    double2* X = smem + 12 * N + warp * (N + 1);
    // inputs: 0..2 u_l, 3..5 du_l/dx, 6..8 du_l/dy, 9..11 du_l/dz
    for (int f = warp; f < 12; f += NL_WARPS) {
        const int l = f % 3, kind = f / 3;
        const double* src;
        int mode = YM_COPY;
        double meanv = 0.0;
        if (kind == 0) {
            src = a.U[l];
            if (l == 0) meanv = a.ubar[z];
        } else if (kind == 1) {
            src = a.U[l];
            mode = YM_IKX;
        } else if (kind == 2) {
            src = a.DY[l];
        } else {
            src = a.DZ[l];
            if (l == 0) meanv = a.ubarp[z];
        }
        row_c2r_warp(src + row * 2 * r.kxc, mode, r.wavx, r.kxc, meanv, r.rp, X, P + f * N, lane);
    }
    __syncthreads();
    const double* p = reinterpret_cast<const double*>(P);
    double* q = reinterpret_cast<double*>(P);
    const int n = r.nxl;
    const double ub = a.ubar[z];
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        double u[3], g[3][3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            u[l] = p[(0 + l) * 2 * N + x];
            g[l][0] = p[(3 + l) * 2 * N + x];
            g[l][1] = p[(6 + l) * 2 * N + x];
            g[l][2] = p[(9 + l) * 2 * N + x];
        }
        double nl[3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            double acc = 0.0;
            acc = acc - 0.5 * (u[0] * g[l][0]);
            acc = acc - 0.5 * (u[1] * g[l][1]);
            acc = acc - 0.5 * (u[2] * g[l][2]);
            nl[l] = acc;
        }
        if (a.lamx != nullptr) {
            const double lx = a.lamx[x];
            nl[0] = nl[0] + lx * (ub - u[0]);
            nl[1] = nl[1] + lx * (0.0 - u[1]);
            nl[2] = nl[2] + lx * (0.0 - u[2]);
        }
        const double h11 = 0.5 * (u[0] * u[0]), h12 = 0.5 * (u[0] * u[1]), h13 = 0.5 * (u[0] * u[2]);
        const double h22 = 0.5 * (u[1] * u[1]), h23 = 0.5 * (u[1] * u[2]), h33 = 0.5 * (u[2] * u[2]);
        q[0 * 2 * N + x] = nl[0];
        q[1 * 2 * N + x] = nl[1];
        q[2 * 2 * N + x] = nl[2];
        q[3 * 2 * N + x] = h11;
        q[4 * 2 * N + x] = h12;
        q[5 * 2 * N + x] = h13;
        q[6 * 2 * N + x] = h22;
        q[7 * 2 * N + x] = h23;
        q[8 * 2 * N + x] = h33;
    }
    __syncthreads();
    for (int f = warp; f < 9; f += NL_WARPS) {
        double* dst = (f < 3) ? a.N[f] : a.H[f - 3];
        row_r2c_warp(P + f * N, X, r.rp, r.kxc, dst + row * 2 * r.kxc, lane);
    }
}

void launch_row_nl(const NlRowArgs& a, cudaStream_t s) {
    const int N = a.r.nxl / 2;
    size_t sm = (size_t)(12 * N + NL_WARPS * (N + 1)) * sizeof(double2);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_row_nl, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    dim3 grid(a.r.nyl, a.r.nzp);
    k_row_nl<<<grid, NL_WARPS * 32, sm, s>>>(a);
}

}  // namespace lsb
