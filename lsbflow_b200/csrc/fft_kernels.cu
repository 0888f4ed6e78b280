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
// The complex FFTs are mixed-radix (2,3,4,5,7) Stockham autosort transforms in shared
// memory; every stage runs over all lines a block holds, with all its threads.  FFTW's c2r semantics are kept: the imaginary parts of
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

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    return f.d == 1 ? n : ((__umulhi(n, f.m) + n) >> f.s);
}

// One radix-R Stockham stage over nlines lines (line stride ls) done by the whole block.
template <int R, int SIGN>
__device__ __forceinline__ void bstage(const double2* __restrict__ src, double2* __restrict__ dst, int nlines, int ls,
                                       int n, int p, const FastDiv& fdT, const FastDiv& fdP,
                                       const double2* __restrict__ tw, int tid, int nthr) {
    const int T = n / R;
    const int stride = n / (p * R);
    const int total = nlines * T;
    for (int idx = tid; idx < total; idx += nthr) {
        const int line = (int)fdiv((uint32_t)idx, fdT);
        const int i = idx - line * T;
        const int mq = (int)fdiv((uint32_t)i, fdP);
        const int k = i - mq * p;
        const double2* sl = src + line * ls;
        double2* dl = dst + line * ls;
        double2 u[R];
#pragma unroll
        for (int q = 0; q < R; ++q) u[q] = sl[i + q * T];
        if (k != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                double2 w = __ldg(&tw[q * k * stride]);
                if (SIGN > 0) w.y = -w.y;
                u[q] = cmul(u[q], w);
            }
        }
        dft_small<R, SIGN>(u, tw, n);
        const int j = mq * p * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) dl[j + q * p] = u[q];
    }
}

// Complex FFT of nlines lines held in A (stride ls) by the whole block; B is scratch of
// the same shape.  Returns true when the result is in A (even number of stages).
// WIDE kernels also carry the radix-5 and radix-7 stages (lengths with factors 5 or 7);
// the others only 2, 3, 4, which keeps their register footprint small.
template <int SIGN, bool WIDE>
__device__ bool fft_batch(double2* A, double2* B, int nlines, int ls, const FftPlan& P, int tid, int nthr) {
    double2* src = A;
    double2* dst = B;
    for (int s = 0; s < P.nst; ++s) {
        switch (P.radix[s]) {
            case 2: bstage<2, SIGN>(src, dst, nlines, ls, P.n, P.p[s], P.fdT[s], P.fdP[s], P.tw, tid, nthr); break;
            case 3: bstage<3, SIGN>(src, dst, nlines, ls, P.n, P.p[s], P.fdT[s], P.fdP[s], P.tw, tid, nthr); break;
            case 4: bstage<4, SIGN>(src, dst, nlines, ls, P.n, P.p[s], P.fdT[s], P.fdP[s], P.tw, tid, nthr); break;
            default:
                if constexpr (WIDE) {
                    if (P.radix[s] == 5)
                        bstage<5, SIGN>(src, dst, nlines, ls, P.n, P.p[s], P.fdT[s], P.fdP[s], P.tw, tid, nthr);
                    else
                        bstage<7, SIGN>(src, dst, nlines, ls, P.n, P.p[s], P.fdT[s], P.fdP[s], P.tw, tid, nthr);
                }
                break;
        }
        __syncthreads();
        double2* t = src;
        src = dst;
        dst = t;
    }
    return src == A;
}

__device__ __forceinline__ int pad_row(int j, int ny, int nyl, int layout) {
    if (layout == 0 || nyl == ny) return j;
    return (j < ny / 2) ? j : j + (nyl - ny);
}

constexpr int KC = 16;  // kx columns per spanwise block

// ----------------------------------------------------------------------------- k_yinv
template <bool WIDE>
__global__ void __launch_bounds__(256, WIDE ? 2 : 3) k_yinv(YInvJobList jobs, YPassArgs a) {
    extern __shared__ double2 smem[];
    const YInvJob job = jobs.j[blockIdx.z];
    const int z = blockIdx.y;
    const int c0 = blockIdx.x * KC;
    const int nyl = a.nyl, ny = a.ny;
    const int LS = nyl + 1;  // odd line stride: conflict-free column writes
    double2* A = smem;
    double2* B = smem + KC * LS;
    const int tid = threadIdx.x;
    for (int i = tid; i < KC * LS; i += blockDim.x) A[i] = make_double2(0.0, 0.0);
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
        A[cc * LS + pad_row(j, ny, nyl, a.layout)] = r;
    }
    __syncthreads();
    const bool inA = fft_batch<+1, WIDE>(A, B, KC, LS, a.plan, tid, blockDim.x);
    const double2* R = inA ? A : B;
    for (int idx = tid; idx < nyl * KC; idx += blockDim.x) {
        const int jl = idx / KC, cc = idx % KC, c = c0 + cc;
        if (c >= a.kxc) continue;
        *reinterpret_cast<double2*>(job.out + ((long long)z * nyl + jl) * a.nx + 2 * c) = R[cc * LS + jl];
    }
}

// ----------------------------------------------------------------------------- k_yfwd
template <bool WIDE>
__global__ void __launch_bounds__(256, WIDE ? 2 : 3) k_yfwd(YFwdJobList jobs, YPassArgs a) {
    extern __shared__ double2 smem[];
    const YFwdJob job = jobs.j[blockIdx.z];
    const int z = blockIdx.y;
    const int c0 = blockIdx.x * KC;
    const int nyl = a.nyl, ny = a.ny;
    const int LS = nyl + 1;
    double2* A = smem;
    double2* B = smem + KC * LS;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nyl * KC; idx += blockDim.x) {
        const int jl = idx / KC, cc = idx % KC, c = c0 + cc;
        double2 v = make_double2(0.0, 0.0);
        if (c < a.kxc) v = *reinterpret_cast<const double2*>(job.in + ((long long)z * nyl + jl) * a.nx + 2 * c);
        A[cc * LS + jl] = v;
    }
    __syncthreads();
    const bool inA = fft_batch<-1, WIDE>(A, B, KC, LS, a.plan, tid, blockDim.x);
    const double2* R = inA ? A : B;
    for (int idx = tid; idx < ny * KC; idx += blockDim.x) {
        const int j = idx / KC, cc = idx % KC, c = c0 + cc;
        if (c >= a.kxc) continue;
        double2 v = R[cc * LS + pad_row(j, ny, nyl, a.layout)];
        if (job.sym && c == 0) {
            const int jm = (ny - j) % ny;
            const double2 w = R[cc * LS + pad_row(jm, ny, nyl, a.layout)];
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

static size_t ypass_smem(const YPassArgs& a) { return (size_t)2 * KC * (a.nyl + 1) * sizeof(double2); }

static bool wide(const FftPlan& P) {
    for (int i = 0; i < P.nst; ++i)
        if (P.radix[i] > 4) return true;
    return false;
}

template <class K>
static void smem_attr(K kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void launch_yinv(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    dim3 grid((a.kxc + KC - 1) / KC, a.nzp, jobs.n);
    size_t sm = ypass_smem(a);
    static bool attr = false;
    if (!attr) {
        smem_attr(k_yinv<true>);
        smem_attr(k_yinv<false>);
        attr = true;
    }
    if (wide(a.plan)) k_yinv<true><<<grid, 256, sm, s>>>(jobs, a);
    else k_yinv<false><<<grid, 256, sm, s>>>(jobs, a);
}

void launch_yfwd(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    dim3 grid((a.kxc + KC - 1) / KC, a.nzp, jobs.n);
    size_t sm = ypass_smem(a);
    static bool attr = false;
    if (!attr) {
        smem_attr(k_yfwd<true>);
        smem_attr(k_yfwd<false>);
        attr = true;
    }
    if (wide(a.plan)) k_yfwd<true><<<grid, 256, sm, s>>>(jobs, a);
    else k_yfwd<false><<<grid, 256, sm, s>>>(jobs, a);
}

// ----------------------------------------------------------------------------- rows
// Batched c2r of L lines.  On entry X[l][0..N] holds the kx modes (zero beyond kxc, DC
// imaginary part already dropped); Z is scratch.  Returns the buffer holding the N double2
// (= 2N physical reals) of each line (stride N+1).
template <bool WIDE>
__device__ double2* rows_c2r(double2* X, double2* Z, int L, const RealPlan& rp, int tid, int nthr) {
    const int N = rp.nr / 2, LS = N + 1;
    for (int idx = tid; idx < L * N; idx += nthr) {
        const int l = idx / N, k = idx - l * N;
        const double2* xl = X + l * LS;
        const double2 xa = xl[k];
        const double2 xb = cconj(xl[N - k]);
        const double2 e = cadd(xa, xb);
        const double2 o = cmul(csub(xa, xb), cconj(__ldg(&rp.twr[k])));
        Z[l * LS + k] = make_double2(e.x - o.y, e.y + o.x);
    }
    __syncthreads();
    const bool inZ = fft_batch<+1, WIDE>(Z, X, L, LS, rp.half, tid, nthr);
    return inZ ? Z : X;
}

// Batched r2c of L physical lines held in Z (N double2 each, stride N+1; destroyed); X is
// scratch.  Returns the buffer holding the half-length spectra; the kx mode k < kxc of
// line l is then made by r2c_mode().
template <bool WIDE>
__device__ double2* rows_r2c(double2* Z, double2* X, int L, const RealPlan& rp, int tid, int nthr) {
    const int N = rp.nr / 2;
    const bool inZ = fft_batch<-1, WIDE>(Z, X, L, N + 1, rp.half, tid, nthr);
    return inZ ? Z : X;
}

__device__ __forceinline__ double2 r2c_mode(const double2* Rl, int k, int N, const double2* __restrict__ twr) {
    const double2 za = Rl[k];
    const double2 zb = cconj(Rl[(N - k) % N]);
    const double2 e = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y + zb.y));
    const double2 o = make_double2(0.5 * (za.x - zb.x), 0.5 * (za.y - zb.y));
    const double2 t = cmul(__ldg(&twr[k]), o);
    return make_double2(e.x + t.y, e.y - t.x);
}

constexpr int RB = 8;  // rows per block of the generic row kernels

template <bool WIDE>
__global__ void __launch_bounds__(256, WIDE ? 2 : 3) k_row_c2r(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const RowIO job = jobs.j[blockIdx.y];
    const int N = a.nxl / 2, LS = N + 1;
    const int nrows = a.nyl * a.nzp;
    const int row0 = blockIdx.x * RB;
    const int L = min(RB, nrows - row0);
    double2* X = smem;
    double2* Z = smem + RB * LS;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < L * LS; idx += blockDim.x) {
        const int l = idx / LS, k = idx - l * LS;
        double2 v = make_double2(0.0, 0.0);
        if (k < a.kxc) {
            v = *reinterpret_cast<const double2*>(job.yin + (long long)(row0 + l) * 2 * a.kxc + 2 * k);
            if (job.mode == YM_IKX) {
                const double kk = a.wavx[2 * k];
                v = make_double2(-kk * v.y, kk * v.x);
            }
        }
        if (k == 0) v.y = 0.0;  // FFTW c2r ignores Im of the DC input
        X[idx] = v;
    }
    __syncthreads();
    const double2* R = rows_c2r<WIDE>(X, Z, L, a.rp, tid, blockDim.x);
    for (int idx = tid; idx < L * N; idx += blockDim.x) {
        const int l = idx / N, k = idx - l * N;
        double2 v = R[l * LS + k];
        if (job.mean != nullptr && job.add_mean != 0.0) {
            const double m = job.mean[(row0 + l) / a.nyl] * job.add_mean;
            v.x += m;
            v.y += m;
        }
        reinterpret_cast<double2*>(job.out + (long long)(row0 + l) * a.row_pitch)[k] = v;
    }
}

template <bool WIDE>
__global__ void __launch_bounds__(256, WIDE ? 2 : 3) k_row_r2c(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const RowIO job = jobs.j[blockIdx.y];
    const int N = a.nxl / 2, LS = N + 1;
    const int nrows = a.nyl * a.nzp;
    const int row0 = blockIdx.x * RB;
    const int L = min(RB, nrows - row0);
    double2* Z = smem;
    double2* X = smem + RB * LS;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < L * N; idx += blockDim.x) {
        const int l = idx / N, k = idx - l * N;
        Z[l * LS + k] = reinterpret_cast<const double2*>(job.yin + (long long)(row0 + l) * a.row_pitch)[k];
    }
    __syncthreads();
    const double2* R = rows_r2c<WIDE>(Z, X, L, a.rp, tid, blockDim.x);
    for (int idx = tid; idx < L * a.kxc; idx += blockDim.x) {
        const int l = idx / a.kxc, k = idx - l * a.kxc;
        *reinterpret_cast<double2*>(job.out + (long long)(row0 + l) * 2 * a.kxc + 2 * k) =
            r2c_mode(R + l * LS, k, N, a.rp.twr);
    }
}

static size_t rows_smem(int nxl) { return (size_t)2 * RB * (nxl / 2 + 1) * sizeof(double2); }

void launch_row_c2r(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    const int rows = a.nyl * a.nzp;
    dim3 grid((rows + RB - 1) / RB, jobs.n);
    static bool attr = false;
    if (!attr) {
        smem_attr(k_row_c2r<true>);
        smem_attr(k_row_c2r<false>);
        attr = true;
    }
    if (wide(a.rp.half)) k_row_c2r<true><<<grid, 256, rows_smem(a.nxl), s>>>(jobs, a);
    else k_row_c2r<false><<<grid, 256, rows_smem(a.nxl), s>>>(jobs, a);
}

void launch_row_r2c(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    const int rows = a.nyl * a.nzp;
    dim3 grid((rows + RB - 1) / RB, jobs.n);
    static bool attr = false;
    if (!attr) {
        smem_attr(k_row_r2c<true>);
        smem_attr(k_row_r2c<false>);
        attr = true;
    }
    if (wide(a.rp.half)) k_row_r2c<true><<<grid, 256, rows_smem(a.nxl), s>>>(jobs, a);
    else k_row_r2c<false><<<grid, 256, rows_smem(a.nxl), s>>>(jobs, a);
}

// ----------------------------------------------------------------------------- NL row
// One (z, y) row per block: 12 c2r (u, du/dx, du/dy, du/dz for 3 components), the
// skew-symmetric products of nlterm_skewsym (src/navierstokes.f90:725-769), and 9 r2c.
template <bool WIDE>
__global__ void __launch_bounds__(256, WIDE ? 2 : 3) k_row_nl(NlRowArgs a) {
    extern __shared__ double2 smem[];
    const RowArgs& r = a.r;
    const int N = r.nxl / 2, LS = N + 1;
    const int yl = blockIdx.x, z = blockIdx.y;
    const long long row = (long long)z * r.nyl + yl;
    const int tid = threadIdx.x;
    double2* X = smem;            // 12 lines
    double2* Z = smem + 12 * LS;  // 12 lines
    // inputs: 0..2 u_l, 3..5 du_l/dx, 6..8 du_l/dy, 9..11 du_l/dz
    for (int idx = tid; idx < 12 * LS; idx += blockDim.x) {
        const int f = idx / LS, k = idx - f * LS;
        const int l = f % 3, kind = f / 3;
        double2 v = make_double2(0.0, 0.0);
        if (k < r.kxc) {
            const double* src = (kind == 0 || kind == 1) ? a.U[l] : (kind == 2 ? a.DY[l] : a.DZ[l]);
            v = *reinterpret_cast<const double2*>(src + row * 2 * r.kxc + 2 * k);
            if (kind == 1) {
                const double kk = r.wavx[2 * k];
                v = make_double2(-kk * v.y, kk * v.x);
            }
        }
        if (k == 0) v.y = 0.0;
        X[idx] = v;
    }
    __syncthreads();
    double2* R = rows_c2r<WIDE>(X, Z, 12, r.rp, tid, blockDim.x);
    double2* O = (R == Z) ? X : Z;
    const double* p = reinterpret_cast<const double*>(R);
    double* q = reinterpret_cast<double*>(O);
    const int n = r.nxl, L2 = 2 * LS;
    const double ub = a.ubar[z], ubp = a.ubarp[z];
    for (int x = tid; x < n; x += blockDim.x) {
        double u[3], g[3][3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            u[l] = p[(0 + l) * L2 + x];
            g[l][0] = p[(3 + l) * L2 + x];
            g[l][1] = p[(6 + l) * L2 + x];
            g[l][2] = p[(9 + l) * L2 + x];
        }
        u[0] += ub;
        g[0][2] += ubp;
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
        q[0 * L2 + x] = nl[0];
        q[1 * L2 + x] = nl[1];
        q[2 * L2 + x] = nl[2];
        q[3 * L2 + x] = 0.5 * (u[0] * u[0]);
        q[4 * L2 + x] = 0.5 * (u[0] * u[1]);
        q[5 * L2 + x] = 0.5 * (u[0] * u[2]);
        q[6 * L2 + x] = 0.5 * (u[1] * u[1]);
        q[7 * L2 + x] = 0.5 * (u[1] * u[2]);
        q[8 * L2 + x] = 0.5 * (u[2] * u[2]);
    }
    __syncthreads();
    const double2* R2 = rows_r2c<WIDE>(O, R, 9, r.rp, tid, blockDim.x);
    for (int idx = tid; idx < 9 * r.kxc; idx += blockDim.x) {
        const int f = idx / r.kxc, k = idx - f * r.kxc;
        double* dst = (f < 3) ? a.N[f] : a.H[f - 3];
        *reinterpret_cast<double2*>(dst + row * 2 * r.kxc + 2 * k) = r2c_mode(R2 + f * LS, k, N, r.rp.twr);
    }
}

void launch_row_nl(const NlRowArgs& a, cudaStream_t s) {
    const int N = a.r.nxl / 2;
    size_t sm = (size_t)24 * (N + 1) * sizeof(double2);
    static bool attr = false;
    if (!attr) {
        smem_attr(k_row_nl<true>);
        smem_attr(k_row_nl<false>);
        attr = true;
    }
    dim3 grid(a.r.nyl, a.r.nzp);
    if (wide(a.r.rp.half)) k_row_nl<true><<<grid, 256, sm, s>>>(a);
    else k_row_nl<false><<<grid, 256, sm, s>>>(a);
}

}  // namespace lsb
