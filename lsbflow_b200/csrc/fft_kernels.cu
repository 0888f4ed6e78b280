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
#include <stdexcept>

#include "lsb_internal.cuh"
#include "lsb_fftdev.cuh"

namespace lsb {

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

// Complex FFT of L lines (stride ls) of length N = N1*N2 by the whole block, result in A:
// pass 1 does the N1-point DFTs of the stride-N2 subsequences in registers and the
// twiddles exp(SIGN 2 pi i n2 k1 / N) (table tw), into B with padded rows; pass 2 the
// N2-point DFTs, back into A in natural order.
template <int N1, int N2, int SIGN>
__device__ void fft2p(double2* A, double2* B, int L, int ls, const double2* __restrict__ tw, int tid, int nthr) {
    if constexpr (N2 == 1) {
        for (int line = tid; line < L; line += nthr) {
            double2* a = A + line * ls;
            double2 v[N1];
#pragma unroll
            for (int k = 0; k < N1; ++k) v[k] = a[k];
            dft_reg<N1, SIGN>(v);
#pragma unroll
            for (int k = 0; k < N1; ++k) a[k] = v[k];
        }
        __syncthreads();
    } else {
        constexpr int PB = (N2 % 2 == 0) ? N2 + 1 : N2;
        for (int idx = tid; idx < L * N2; idx += nthr) {
            const int line = idx / N2, n2 = idx - line * N2;
            const double2* a = A + line * ls;
            double2 v[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) v[n1] = a[N2 * n1 + n2];
            dft_reg<N1, SIGN>(v);
            if (n2 != 0) {
#pragma unroll
                for (int k1 = 1; k1 < N1; ++k1) {
                    double2 w = __ldg(&tw[n2 * k1]);
                    if (SIGN > 0) w.y = -w.y;
                    v[k1] = cmul(v[k1], w);
                }
            }
            double2* b = B + line * ls;
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) b[k1 * PB + n2] = v[k1];
        }
        __syncthreads();
        for (int idx = tid; idx < L * N1; idx += nthr) {
            const int line = idx / N1, k1 = idx - line * N1;
            const double2* b = B + line * ls;
            double2 v[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) v[n2] = b[k1 * PB + n2];
            dft_reg<N2, SIGN>(v);
            double2* a = A + line * ls;
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) a[k1 + N1 * k2] = v[k2];
        }
        __syncthreads();
    }
}

// returns true (result in A) when the plan has a register two-pass split
template <int SIGN>
__device__ __forceinline__ bool fft_twopass(double2* A, double2* B, int L, int ls, const FftPlan& P, int tid,
                                            int nthr) {
#define LSB_2P(a_, b_)                                                   \
    if (P.n1 == a_ && P.n2 == b_) {                                     \
        fft2p<a_, b_, SIGN>(A, B, L, ls, P.tw, tid, nthr);              \
        return true;                                                    \
    }
    LSB_2P(2, 1) LSB_2P(3, 1) LSB_2P(4, 1) LSB_2P(6, 1) LSB_2P(8, 1) LSB_2P(12, 1) LSB_2P(16, 1)
    LSB_2P(3, 3) LSB_2P(6, 3) LSB_2P(8, 3) LSB_2P(8, 4) LSB_2P(12, 3) LSB_2P(8, 6) LSB_2P(16, 3)
    LSB_2P(8, 8) LSB_2P(12, 6) LSB_2P(12, 8) LSB_2P(16, 6) LSB_2P(12, 12) LSB_2P(16, 8) LSB_2P(16, 12)
    LSB_2P(16, 16)
#undef LSB_2P
    return false;
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
    if constexpr (!WIDE) {
        if (fft_twopass<SIGN>(A, B, nlines, ls, P, tid, nthr)) return true;
    }
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

constexpr int KC = 16;  // kx columns per spanwise work item
constexpr int RB = 8;   // rows per work item of the generic row kernels

// ---------------------------------------------------------------- pipelining helpers
// Every FFT kernel below is persistent: a block loops over work items and stages the
// next item's input with cp.async while it transforms the current one (two input
// buffers used alternately, one scratch buffer for the FFT ping-pong).
__device__ __forceinline__ void cpa16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// ----------------------------------------------------------------------------- k_yinv
// item = (job, z, kx chunk); input rows go straight into line layout (pad rows zeroed)
template <bool WIDE>
__global__ void __launch_bounds__(256, 2) k_yinv(YInvJobList jobs, YPassArgs a, int nch) {
    extern __shared__ double2 smem[];
    const int ny = a.ny, nyl = a.nyl, LS = a.plan.ls;
    double2* Buf[2] = {smem, smem + KC * LS};
    double2* Scr = smem + 2 * KC * LS;
    const int tid = threadIdx.x;
    const int nitems = jobs.n * a.nzp * nch;
    const int npad = nyl - ny;
    auto issue = [&](int item, double2* A) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const double* in = jobs.j[jb].in;
        const int c0 = ch * KC;
        for (int idx = tid; idx < ny * KC; idx += 256) {
            const int j = idx / KC, cc = idx - j * KC, c = c0 + cc;
            double2* d = &A[cc * LS + pad_row(j, ny, nyl, a.layout)];
            if (c < a.kxc) cpa16(d, in + ((long long)z * ny + j) * a.nx + 2 * c);
            else *d = make_double2(0.0, 0.0);
        }
        for (int idx = tid; idx < npad * KC; idx += 256) {
            const int r = idx / KC, cc = idx - r * KC;
            const int jl = (a.layout == 0) ? ny + r : ny / 2 + r;
            A[cc * LS + jl] = make_double2(0.0, 0.0);
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, Buf[0]);
    for (; item < nitems; item += gridDim.x) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const YInvJob job = jobs.j[jb];
        const int c0 = ch * KC;
        double2* A = Buf[cur];
        cpa_wait_all();
        __syncthreads();
        if (job.mode != YM_COPY) {
            for (int idx = tid; idx < ny * KC; idx += 256) {
                const int j = idx / KC, cc = idx - j * KC, c = c0 + cc;
                double2* d = &A[cc * LS + pad_row(j, ny, nyl, a.layout)];
                const double k = (job.mode == YM_IKY) ? a.wavy[j] : a.wavx[2 * min(c, a.kxc - 1)];
                const double2 v = *d;
                *d = make_double2(-k * v.y, k * v.x);
            }
            __syncthreads();
        }
        const int next = item + gridDim.x;
        if (next < nitems) issue(next, Buf[cur ^ 1]);
        const bool inA = fft_batch<+1, WIDE>(A, Scr, KC, LS, a.plan, tid, 256);
        const double2* R = inA ? A : Scr;
        for (int idx = tid; idx < nyl * KC; idx += 256) {
            const int jl = idx / KC, cc = idx - jl * KC, c = c0 + cc;
            if (c >= a.kxc) continue;
            *reinterpret_cast<double2*>(job.out + ((long long)z * nyl + jl) * a.nx + 2 * c) = R[cc * LS + jl];
        }
        __syncthreads();
        cur ^= 1;
    }
}

// ----------------------------------------------------------------------------- k_yfwd
template <bool WIDE>
__global__ void __launch_bounds__(256, 2) k_yfwd(YFwdJobList jobs, YPassArgs a, int nch) {
    extern __shared__ double2 smem[];
    const int ny = a.ny, nyl = a.nyl, LS = a.plan.ls;
    double2* Buf[2] = {smem, smem + KC * LS};
    double2* Scr = smem + 2 * KC * LS;
    const int tid = threadIdx.x;
    const int nitems = jobs.n * a.nzp * nch;
    auto issue = [&](int item, double2* A) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const double* in = jobs.j[jb].in;
        const int c0 = ch * KC;
        for (int idx = tid; idx < nyl * KC; idx += 256) {
            const int jl = idx / KC, cc = idx - jl * KC, c = c0 + cc;
            double2* d = &A[cc * LS + jl];
            if (c < a.kxc) cpa16(d, in + ((long long)z * nyl + jl) * a.nx + 2 * c);
            else *d = make_double2(0.0, 0.0);
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, Buf[0]);
    for (; item < nitems; item += gridDim.x) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const YFwdJob job = jobs.j[jb];
        const int c0 = ch * KC;
        double2* A = Buf[cur];
        cpa_wait_all();
        __syncthreads();
        const int next = item + gridDim.x;
        if (next < nitems) issue(next, Buf[cur ^ 1]);
        const bool inA = fft_batch<-1, WIDE>(A, Scr, KC, LS, a.plan, tid, 256);
        const double2* R = inA ? A : Scr;
        for (int idx = tid; idx < ny * KC; idx += 256) {
            const int j = idx / KC, cc = idx - j * KC, c = c0 + cc;
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
        __syncthreads();
        cur ^= 1;
    }
}

static bool wide(const FftPlan& P) {
    for (int i = 0; i < P.nst; ++i)
        if (P.radix[i] > 4) return true;
    return false;
}

// persistent grid: resident blocks per SM x SMs, capped by the number of work items
template <class K>
static int persistent_grid(K kern, size_t smem, int nitems) {
    const int g = resident_blocks((const void*)kern, 256, smem) * sm_count();
    return g < nitems ? g : nitems;
}

void launch_yinv(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    if (launch_yinv_warp(jobs, a, s)) return;
    if (a.f32) throw std::runtime_error("mixed precision: y transform length has no warp plan");
    const int nch = (a.kxc + KC - 1) / KC;
    const int nitems = jobs.n * a.nzp * nch;
    const size_t sm = (size_t)3 * KC * a.plan.ls * sizeof(double2);
    if (wide(a.plan)) { lsb::note_launch(); k_yinv<true><<<persistent_grid(k_yinv<true>, sm, nitems), 256, sm, s>>>(jobs, a, nch); }
    else { lsb::note_launch(); k_yinv<false><<<persistent_grid(k_yinv<false>, sm, nitems), 256, sm, s>>>(jobs, a, nch); }
}

void launch_yfwd(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    if (launch_yfwd_warp(jobs, a, s)) return;
    if (a.f32) throw std::runtime_error("mixed precision: y transform length has no warp plan");
    const int nch = (a.kxc + KC - 1) / KC;
    const int nitems = jobs.n * a.nzp * nch;
    const size_t sm = (size_t)3 * KC * a.plan.ls * sizeof(double2);
    if (wide(a.plan)) { lsb::note_launch(); k_yfwd<true><<<persistent_grid(k_yfwd<true>, sm, nitems), 256, sm, s>>>(jobs, a, nch); }
    else { lsb::note_launch(); k_yfwd<false><<<persistent_grid(k_yfwd<false>, sm, nitems), 256, sm, s>>>(jobs, a, nch); }
}

// ----------------------------------------------------------------------------- rows
// Batched c2r of L lines.  On entry X[l][0..N] holds the kx modes (zero beyond kxc, DC
// imaginary part already dropped); Z is scratch.  Returns the buffer holding the N double2
// (= 2N physical reals) of each line (stride N+1).
template <bool WIDE>
__device__ double2* rows_c2r(double2* X, double2* Z, int L, const RealPlan& rp, int tid, int nthr) {
    const int N = rp.nr / 2, LS = rp.half.ls;
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
    const bool inZ = fft_batch<-1, WIDE>(Z, X, L, rp.half.ls, rp.half, tid, nthr);
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


// item = (job, chunk of RB rows)
template <bool WIDE>
__global__ void __launch_bounds__(256, 2) k_row_c2r(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const int N = a.nxl / 2, LS = a.rp.half.ls;
    const int nrows = a.nyl * a.nzp;
    const int nrc = (nrows + RB - 1) / RB;
    const int nitems = jobs.n * nrc;
    double2* Buf[2] = {smem, smem + RB * LS};
    double2* Z = smem + 2 * RB * LS;
    const int tid = threadIdx.x;
    auto issue = [&](int item, double2* X) {
        const int rc = item % nrc, jb = item / nrc;
        const int row0 = rc * RB, L = min(RB, nrows - row0);
        const double* yin = jobs.j[jb].yin;
        for (int idx = tid; idx < L * (N + 1); idx += 256) {
            const int l = idx / (N + 1), k = idx - l * (N + 1);
            double2* d = &X[l * LS + k];
            if (k < a.kxc) cpa16(d, yin + (long long)(row0 + l) * 2 * a.kxc + 2 * k);
            else *d = make_double2(0.0, 0.0);
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, Buf[0]);
    for (; item < nitems; item += gridDim.x) {
        const int rc = item % nrc, jb = item / nrc;
        const RowIO job = jobs.j[jb];
        const int row0 = rc * RB, L = min(RB, nrows - row0);
        double2* X = Buf[cur];
        cpa_wait_all();
        __syncthreads();
        for (int idx = tid; idx < L * a.kxc; idx += 256) {
            const int l = idx / a.kxc, k = idx - l * a.kxc;
            double2 v = X[l * LS + k];
            if (job.mode == YM_IKX) {
                const double kk = a.wavx[2 * k];
                v = make_double2(-kk * v.y, kk * v.x);
            }
            if (k == 0) v.y = 0.0;  // FFTW c2r ignores Im of the DC input
            X[l * LS + k] = v;
        }
        __syncthreads();
        const int next = item + gridDim.x;
        if (next < nitems) issue(next, Buf[cur ^ 1]);
        const double2* R = rows_c2r<WIDE>(X, Z, L, a.rp, tid, 256);
        for (int idx = tid; idx < L * N; idx += 256) {
            const int l = idx / N, k = idx - l * N;
            double2 v = R[l * LS + k];
            v.x *= job.scale;
            v.y *= job.scale;
            if (job.mean != nullptr && job.add_mean != 0.0) {
                const double m = job.mean[(row0 + l) / a.nyl] * job.add_mean;
                v.x += m;
                v.y += m;
            }
            reinterpret_cast<double2*>(job.out + (long long)(row0 + l) * a.row_pitch)[k] = v;
        }
        __syncthreads();
        cur ^= 1;
    }
}

template <bool WIDE>
__global__ void __launch_bounds__(256, 2) k_row_r2c(RowJobList jobs, RowArgs a) {
    extern __shared__ double2 smem[];
    const int N = a.nxl / 2, LS = a.rp.half.ls;
    const int nrows = a.nyl * a.nzp;
    const int nrc = (nrows + RB - 1) / RB;
    const int nitems = jobs.n * nrc;
    double2* Buf[2] = {smem, smem + RB * LS};
    double2* X = smem + 2 * RB * LS;
    const int tid = threadIdx.x;
    auto issue = [&](int item, double2* Z) {
        const int rc = item % nrc, jb = item / nrc;
        const int row0 = rc * RB, L = min(RB, nrows - row0);
        const double* in = jobs.j[jb].yin;
        for (int idx = tid; idx < L * N; idx += 256) {
            const int l = idx / N, k = idx - l * N;
            cpa16(&Z[l * LS + k], in + (long long)(row0 + l) * a.row_pitch + 2 * k);
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, Buf[0]);
    for (; item < nitems; item += gridDim.x) {
        const int rc = item % nrc, jb = item / nrc;
        const RowIO job = jobs.j[jb];
        const int row0 = rc * RB, L = min(RB, nrows - row0);
        double2* Z = Buf[cur];
        cpa_wait_all();
        __syncthreads();
        const int next = item + gridDim.x;
        if (next < nitems) issue(next, Buf[cur ^ 1]);
        const double2* R = rows_r2c<WIDE>(Z, X, L, a.rp, tid, 256);
        for (int idx = tid; idx < L * a.kxc; idx += 256) {
            const int l = idx / a.kxc, k = idx - l * a.kxc;
            *reinterpret_cast<double2*>(job.out + (long long)(row0 + l) * 2 * a.kxc + 2 * k) =
                r2c_mode(R + l * LS, k, N, a.rp.twr);
        }
        __syncthreads();
        cur ^= 1;
    }
}

void launch_row_c2r(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    if (launch_row_c2r_warp(jobs, a, s)) return;
    if (a.f32) throw std::runtime_error("mixed precision: x transform length has no warp plan");
    const int nitems = jobs.n * ((a.nyl * a.nzp + RB - 1) / RB);
    const size_t sm = (size_t)3 * RB * a.rp.half.ls * sizeof(double2);
    if (wide(a.rp.half)) { lsb::note_launch(); k_row_c2r<true><<<persistent_grid(k_row_c2r<true>, sm, nitems), 256, sm, s>>>(jobs, a); }
    else { lsb::note_launch(); k_row_c2r<false><<<persistent_grid(k_row_c2r<false>, sm, nitems), 256, sm, s>>>(jobs, a); }
}

void launch_row_r2c(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (jobs.n <= 0) return;
    if (launch_row_r2c_warp(jobs, a, s)) return;
    if (a.f32) throw std::runtime_error("mixed precision: x transform length has no warp plan");
    const int nitems = jobs.n * ((a.nyl * a.nzp + RB - 1) / RB);
    const size_t sm = (size_t)3 * RB * a.rp.half.ls * sizeof(double2);
    if (wide(a.rp.half)) { lsb::note_launch(); k_row_r2c<true><<<persistent_grid(k_row_r2c<true>, sm, nitems), 256, sm, s>>>(jobs, a); }
    else { lsb::note_launch(); k_row_r2c<false><<<persistent_grid(k_row_r2c<false>, sm, nitems), 256, sm, s>>>(jobs, a); }
}

// ----------------------------------------------------------------------------- NL row
// One (z, y) row per work item: 12 c2r (u, du/dx, du/dy, du/dz for 3 components), the
// skew-symmetric products of nlterm_skewsym (src/navierstokes.f90:725-769), and 9 r2c.
template <bool WIDE>
__global__ void __launch_bounds__(256, 2) k_row_nl(NlRowArgs a) {
    extern __shared__ double2 smem[];
    const RowArgs& r = a.r;
    const int N = r.nxl / 2, LS = r.rp.half.ls;
    const int nitems = r.nyl * r.nzp;
    double2* Buf[2] = {smem, smem + 12 * LS};
    double2* Z = smem + 24 * LS;
    const int tid = threadIdx.x;
    // lines: 0..2 u_l, 3..5 u_l (-> du_l/dx), 6..8 du_l/dy, 9..11 du_l/dz
    auto issue = [&](int row, double2* X) {
        for (int idx = tid; idx < 12 * (N + 1); idx += 256) {
            const int f = idx / (N + 1), k = idx - f * (N + 1);
            const int l = f % 3, kind = f / 3;
            double2* d = &X[f * LS + k];
            if (k < r.kxc) {
                const double* src = (kind <= 1) ? a.U[l] : (kind == 2 ? a.DY[l] : a.DZ[l]);
                cpa16(d, src + (long long)row * 2 * r.kxc + 2 * k);
            } else {
                *d = make_double2(0.0, 0.0);
            }
        }
        cpa_commit();
    };
    int cur = 0;
    int row = blockIdx.x;
    if (row < nitems) issue(row, Buf[0]);
    for (; row < nitems; row += gridDim.x) {
        const int z = row / r.nyl;
        double2* X = Buf[cur];
        cpa_wait_all();
        __syncthreads();
        for (int idx = tid; idx < 12 * r.kxc; idx += 256) {
            const int f = idx / r.kxc, k = idx - f * r.kxc;
            double2 v = X[f * LS + k];
            if (f >= 3 && f < 6) {
                const double kk = r.wavx[2 * k];
                v = make_double2(-kk * v.y, kk * v.x);
            }
            if (k == 0) v.y = 0.0;
            X[f * LS + k] = v;
        }
        __syncthreads();
        const int next = row + gridDim.x;
        if (next < nitems) issue(next, Buf[cur ^ 1]);
        double2* R = rows_c2r<WIDE>(X, Z, 12, r.rp, tid, 256);
        double2* O = (R == Z) ? X : Z;
        const double* p = reinterpret_cast<const double*>(R);
        double* q = reinterpret_cast<double*>(O);
        const int n = r.nxl, L2 = 2 * LS;
        const double ub = a.ubar[z], ubp = a.ubarp[z];
        for (int x = tid; x < n; x += 256) {
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
        const double2* R2 = rows_r2c<WIDE>(O, R, 9, r.rp, tid, 256);
        for (int idx = tid; idx < 9 * r.kxc; idx += 256) {
            const int f = idx / r.kxc, k = idx - f * r.kxc;
            double* dst = (f < 3) ? a.N[f] : a.H[f - 3];
            *reinterpret_cast<double2*>(dst + (long long)row * 2 * r.kxc + 2 * k) =
                r2c_mode(R2 + f * LS, k, N, r.rp.twr);
        }
        __syncthreads();
        cur ^= 1;
    }
}

void launch_row_nl(const NlRowArgs& a, cudaStream_t s) {
    if (launch_row_nl_warp(a, s)) return;
    if (a.r.f32) throw std::runtime_error("mixed precision: x transform length has no warp plan");
    const size_t sm = (size_t)36 * a.r.rp.half.ls * sizeof(double2);
    const int nitems = a.r.nyl * a.r.nzp;
    if (wide(a.r.rp.half)) { lsb::note_launch(); k_row_nl<true><<<persistent_grid(k_row_nl<true>, sm, nitems), 256, sm, s>>>(a); }
    else { lsb::note_launch(); k_row_nl<false><<<persistent_grid(k_row_nl<false>, sm, nitems), 256, sm, s>>>(a); }
}

}  // namespace lsb
