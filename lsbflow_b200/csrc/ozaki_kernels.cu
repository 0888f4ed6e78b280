// z contractions of the mixed-precision form on the int8 tensor cores (tcgen05 kind::i8).
//
// The Chebyshev derivatives (dfdz, src/derivatives.f90:112-188) and the two eigenbasis
// products of the Helmholtz and Poisson solves (solve_helmholtz, src/helmholtz.f90:130-208,
// with the lifting of solve_nhom_helmholtz, :211-358) are out = A . x over every (kx, ky)
// column.  Both operands are split into int8 digits after the error-free splitting of
// Ozaki, Ogita, Oishi and Rump ("Error-free transformations of matrix multiplication by
// using fast routines of matrix multiplication and its applications", Numer. Algorithms
// 59, 2012), in the integer form of Ootomo, Ozaki and Yokota (DGEMM emulation on integer
// tensor cores, IJHPCA 2024):
//
//   x[k][c] = 2^e_c  sum_{i=1..S} d_i[k][c] 2^(-6-7(i-1))     |d_i| <= 64
//   A[r][k] = 2^e_r  sum_{j=1..S} a_j[r][k] 2^(-6-7(j-1))     |a_j| <= 64
//   (A x)[r][c] ~ 2^(e_r+e_c) sum_{L=0..S-1} 2^(-12-7L) sum_{i+j=L+2} (a_j . d_i)[r][c]
//
// with 2^e_c just above the column's largest |x| and 2^e_r above the row's largest |A|.
// Each int8 product a_j . d_i over K <= 128 is exact in an int32 tensor-memory accumulator
// (|.| <= 128 * 64 * 64, at most S products per level), the S level sums are combined in
// FP64; the products of levels above S - 1 are dropped.  With S = 5 the error of an output
// is of the order 2^-35 K max_k|A[r][k]| max_k|x[k][c]| (measured 3e-10 .. 4e-9 relative on
// the Chebyshev D and the eigenbasis matrices, whose rows span four decades, against 2e-8 ..
// 6e-8 for FP32 operands): better than FP32, with exact accumulation.
//
// A CTA (16 warps, one per SM) walks tiles of 128 columns.  Thread (m, part) loads a quarter of
// its column's K into registers (32 independent loads), applying the lifting prologue; the
// quarters' maxima give e_c; the digits go to the shared-memory image of the MMA's A operand
// (K-major, no swizzle); the matrix rows go in passes of 64 (the five level accumulators take
// 5 x 64 tensor-memory columns), one thread issuing the 15 digit products per K step of 32;
// the epilogue reads the five level accumulators, combines them exactly and applies the
// store, Helmholtz-scale, Poisson or lifting epilogue.  Rows and K are 128 at most on the tensor cores; the 129th row (the wall
// row of D, a zero row of the lifted E) and the 129th input row are FP64 dot products on
// the CUDA cores.  Every wait is bounded: on time-out the kernel raises the handle's error
// word, frees its tensor memory and returns.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "lsb_internal.cuh"
#include "lsb_tcgen05.cuh"

namespace lsb {

namespace {

constexpr int OZ_M = 128;       // columns per tile (the MMA's M)
constexpr int OZ_PARTS = 4;     // threads per column: quarters of K (32 rows each) and of the row chunks
constexpr int OZ_T = OZ_PARTS * 128;  // threads
constexpr int OZ_NP = 64;       // matrix rows per pass (the MMA's N): S levels x 64 columns of tensor memory
constexpr int OZ_TCOLS = 512;   // tensor-memory columns allocated (S x 64 <= 512)
constexpr int OZ_HDR = 12288;   // shared-memory header: barrier at 0, column data 1024..11264

struct OzArgs {
    GemmArgs g;
    const uint4* img;        // matrix digits, shared-memory image [S][ksteps][nmma / 8][256 B]
    unsigned img_bytes;
    const double* rscale;    // [nmma] 2^e_r
    const double* arow;      // [K] FP64 row 128 of the matrix (M == 129), or null
    const double* acol;      // [128] FP64 column 128 of the matrix (K == 129), or null
    int nmma;                // rows on the tensor cores, padded to 16
    int ksteps;              // K steps of 32 on the tensor cores
    int kin;                 // rows of K on the tensor cores (<= 128)
    int* err;
};

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ double oz_w2(const GemmArgs& g, long long c) {
    const int i = (int)((unsigned)c % (unsigned)g.nx);
    const int j = (int)((unsigned)c / (unsigned)g.nx);
    const double wx = g.wavx[i], wy = g.wavy[j];
    return wx * wx + wy * wy;
}

// a 32-bit two's-complement integer as an FP64 value: its bits below those of 2^52 + 2^31
__device__ __forceinline__ double i2d(uint32_t x) {
    return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 0x1.00000800000p52;
}

// weight 2^(-12 - 7 L) of level L (digit pairs i + j = L, digits counted from 0)
__host__ __device__ constexpr double level_weight(int L) {
    double w = 1.0 / 4096.0;
    for (int i = 0; i < L; ++i) w *= 1.0 / 128.0;
    return w;
}

template <int S>
__global__ void __launch_bounds__(OZ_T, 1) k_ozaki(OzArgs o) {
    extern __shared__ __align__(1024) unsigned char osm[];
    const GemmArgs& g = o.g;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m = tid & (OZ_M - 1), part = tid >> 7;  // column m of the tile, quarter of K (and of the rows)
    uint64_t* mbar = reinterpret_cast<uint64_t*>(osm);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(osm + 16);
    int* sabort = reinterpret_cast<int*>(osm + 32);
    double* cmax = reinterpret_cast<double*>(osm + 1024);  // [4][128] column maxima of the quarters
    double* rfix = cmax + OZ_PARTS * OZ_M;                  // [4][128] partial sums of row 128
    double* xk = rfix + OZ_PARTS * OZ_M;                    // [128] x'[128][c]
    double* cscale = xk + OZ_M;                             // [128] 2^e_c
    unsigned char* bimg = osm + OZ_HDR;
    unsigned char* aop = bimg + ((o.img_bytes + 1023u) & ~1023u);

    if (tid == 0) {
        tc::mbar_init(mbar);
        *sabort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::smem_u32(tslot)),
                     "r"(OZ_TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    // the matrix digits, once per CTA
    for (unsigned i = tid; i < o.img_bytes / 16u; i += OZ_T) {
        const uint32_t sa = tc::smem_u32(bimg + 16u * i);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(o.img + i));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    // this thread's groups of 16 K rows: part * 2, part * 2 + 1 (ksteps <= 4: 8 groups)
    const int ngroups = 2 * o.ksteps;
    const int npass = (o.nmma + OZ_NP - 1) / OZ_NP;
    const long long ntc = (g.C + OZ_M - 1) / OZ_M;
    const long long ntiles = ntc * g.nfields;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const int mrows = g.M < OZ_M ? g.M : OZ_M;
    uint32_t phase = 0;

    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int f = (int)(tile / ntc);
        const long long c = (tile - (long long)f * ntc) * OZ_M + m;
        const bool cok = c < g.C;
        const double* in = (f < 4 && g.inf[f]) ? g.inf[f] : g.in + f * g.in_fstride;
        const double* bcb = g.bcb ? g.bcb + f * g.bc_fstride : nullptr;
        const double* bct = g.bct ? g.bct + f * g.bc_fstride : nullptr;
        const bool lift = (g.epi != EPI_LIFT_ADD) && (bcb != nullptr);
        double w2 = 0.0, lbcb = 0.0, lbct = 0.0, lfac = 0.0;
        if (cok && (lift || g.epi == EPI_HELM_SCALE || g.epi == EPI_POISSON_RHS)) w2 = oz_w2(g, c);
        if (cok && lift) {
            lbcb = bcb[c];
            lbct = bct[c];
            lfac = (-w2) - g.lift_sigma;
        }
        // this thread's quarter of the column in registers: the 32 loads first, all independent
        double xr[32];
        const double* src = in + (long long)g.koff * g.C + c;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int k = part * 32 + i;
            xr[i] = (cok && k < o.kin) ? __ldg(src + (long long)k * g.C) : 0.0;
        }
        // x'[k][c]: the input row less the lifting functions' part (solve_nhom_helmholtz)
        auto unlift = [&](int k, double v) {
            const int kin = k + g.koff;
            const double abot = __ldg(&g.d2hb[kin]) + lfac * __ldg(&g.hb[kin]);
            v = v - abot * lbcb;
            const double atop = __ldg(&g.d2ht[kin]) + lfac * __ldg(&g.ht[kin]);
            return v - atop * lbct;
        };
        if (lift && cok) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (part * 32 + i < o.kin) xr[i] = unlift(part * 32 + i, xr[i]);
        }
        double amax = 0.0;
#pragma unroll
        for (int i = 0; i < 32; ++i) amax = fmax(amax, fabs(xr[i]));
        double x128 = 0.0;
        if (o.acol && part == OZ_PARTS - 1 && cok) {
            x128 = __ldg(src + (long long)128 * g.C);
            if (lift) x128 = unlift(128, x128);
        }
        // row 128 of the matrix (M == 129) in FP64 over all K
        double rpart = 0.0;
        if (o.arow && cok) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (part * 32 + i < o.kin) rpart = fma(__ldg(&o.arow[part * 32 + i]), xr[i], rpart);
            if (o.acol && part == OZ_PARTS - 1) rpart = fma(__ldg(&o.arow[128]), x128, rpart);
        }
        cmax[part * OZ_M + m] = amax;
        __syncthreads();  // (also orders the previous tile's epilogue reads before the writes below)
        const double cm = fmax(fmax(cmax[m], cmax[OZ_M + m]), fmax(cmax[2 * OZ_M + m], cmax[3 * OZ_M + m]));
        int ec = (cm > 0.0) ? ilogb(cm) + 1 : 0;  // cm < 2^ec
        if (ec < -1000) ec = -1000;
        // X = rint(x' 2^(34 - e_c)), |X| < 2^34, as Xh 2^14 + Xl with Xh = rint(X 2^-14) and
        // |Xl| <= 2^13, each rounded by the round-to-integer constant 1.5 2^52 (its low 32 bits
        // are then the integer); X = D0 2^28 + D1 2^21 + D2 2^14 + D3 2^7 + D4 with balanced
        // digits: Xl + 64 holds D4 + 64 in bits 0..6 and D3 above; Xh + 64 (128 + 1) holds
        // D2 + 64, D1 + 64 in two 7-bit fields and D0 above
        static_assert(S == 5, "the digit split below is written for five digits");
        const double inv = ldexp(1.0, 34 - ec);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int gi = part * 2 + q;
            if (gi >= ngroups) continue;
            uint32_t w[S][4];
#pragma unroll
            for (int k4 = 0; k4 < 4; ++k4) {
                uint32_t fd[S][4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const double t = xr[q * 16 + 4 * k4 + e] * inv;
                    const double yh = fma(t, 0x1p-14, 0x1.8p52);
                    const int xh = __double2loint(yh);
                    const double r = fma(yh - 0x1.8p52, -16384.0, t);  // t - Xh 2^14, exact
                    const int xl = __double2loint(r + 0x1.8p52);
                    const int yl = xl + 64;
                    const int yhb = xh + 64 * 128 + 64;
                    fd[4][e] = (uint32_t)yl & 127u;
                    fd[3][e] = (uint32_t)((yl >> 7) + 64);
                    fd[2][e] = (uint32_t)yhb & 127u;
                    fd[1][e] = ((uint32_t)yhb >> 7) & 127u;
                    fd[0][e] = (uint32_t)((yhb >> 14) + 64);
                }
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    // bytes hold digit + 64 in [0, 128]: (b + 64) ^ 0x80 is the digit as a signed byte
                    const uint32_t packed = fd[i][0] | (fd[i][1] << 8) | (fd[i][2] << 16) | (fd[i][3] << 24);
                    w[i][k4] = (packed + 0x40404040u) ^ 0x80808080u;
                }
            }
            const int ks = gi >> 1;
#pragma unroll
            for (int i = 0; i < S; ++i)
                *reinterpret_cast<uint4*>(aop + ((i * o.ksteps + ks) * (OZ_M / 8) + (m >> 3)) * 256 + (gi & 1) * 128 +
                                          (m & 7) * 16) = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
        }
        rfix[part * OZ_M + m] = rpart;
        if (part == OZ_PARTS - 1) xk[m] = x128;
        if (part == 0) cscale[m] = ldexp(1.0, ec);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();

        double* out = (f < 4 && g.outf[f]) ? g.outf[f] : g.out + f * g.out_fstride;
        const double* aux = g.aux ? g.aux + f * g.out_fstride : nullptr;
        const double sc = cscale[m];
        const double xkc = xk[m];
        auto store = [&](double v, int r) {
            const long long oo = (long long)(r + g.roff) * g.C + c;
            switch (g.epi) {
                case EPI_STORE: break;
                case EPI_AXPBY: v = g.alpha * v + (g.beta != 0.0 ? g.beta * out[oo] : 0.0); break;
                case EPI_HELM_SCALE: v = v / (g.lam[r] + ((-w2) - g.sigma)); break;
                case EPI_POISSON_RHS: v = -v - w2 * aux[oo]; break;
                default:  // EPI_LIFT_ADD: acc + hb*bcb + ht*bct
                    if (bcb != nullptr) v = v + g.hb[r + g.roff] * bcb[c] + g.ht[r + g.roff] * bct[c];
                    break;
            }
            out[oo] = v;
        };
        // the matrix rows in passes of 64: the S(S+1)/2 digit products per K step into S level
        // accumulators, then the epilogue of those rows (16-row chunk j by quarter j % 4)
        for (int p = 0; p < npass; ++p) {
            const int r0 = p * OZ_NP;
            const int np = (o.nmma - r0) < OZ_NP ? (o.nmma - r0) : OZ_NP;
            if (tid == 0 && *sabort == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                // M = 128 columns, N = np rows, s8 x s8 -> s32, both K-major
                const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(np >> 3) << 17) |
                                       ((uint32_t)(OZ_M >> 4) << 24);
                uint32_t started = 0u;  // levels whose accumulator holds this pass's first product
                for (int ks = 0; ks < o.ksteps; ++ks)
                    for (int i = 0; i < S; ++i)
                        for (int j = 0; i + j < S; ++j) {
                            const int L = i + j;
                            const uint64_t ad =
                                tc::kmajor_desc(tc::smem_u32(aop + (i * o.ksteps + ks) * (OZ_M / 8) * 256), 128, 256);
                            const uint64_t bd = tc::kmajor_desc(
                                tc::smem_u32(bimg + ((j * o.ksteps + ks) * (o.nmma / 8) + r0 / 8) * 256), 128, 256);
                            mma_i8(tmem + (uint32_t)(L * OZ_NP), ad, bd, idesc, (started >> L) & 1u);
                            started |= 1u << L;
                        }
                tc::commit_to(mbar);
            }
            const bool ok = tc::mbar_wait(tc::smem_u32(mbar), phase);
            phase ^= 1u;
            if (!ok) *sabort = 1;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            __syncthreads();
            if (*sabort != 0) break;
            for (int j = part; j < np / 16; j += OZ_PARTS) {
                uint32_t v[S][16];
#pragma unroll
                for (int L = 0; L < S; ++L) tc::tmem_ld16(tmem + lane_base + (uint32_t)(L * OZ_NP + j * 16), v[L]);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (!cok) continue;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int r = r0 + j * 16 + e;
                    if (r >= mrows) continue;
                    // the five levels' integer sum T = A0 2^28 + (A1 2^7 + A2) 2^14 + (A3 2^7 + A4)
                    // (|A_L| < 2^22: the pairs fit 32 bits, T < 2^51 is exact in FP64); int32 to
                    // FP64 by the constant 2^52 + 2^31 (exact, on the FP64 pipe)
                    const int p1 = (int)v[1][e] * 128 + (int)v[2][e];
                    const int p2 = (int)v[3][e] * 128 + (int)v[4][e];
                    const double sum = fma(i2d(v[0][e]), 0x1p28, fma(i2d((uint32_t)p1), 0x1p14, i2d((uint32_t)p2))) *
                                       level_weight(S - 1);
                    double val = sum * (sc * __ldg(&o.rscale[r]));
                    if (o.acol) val = fma(__ldg(&o.acol[r]), xkc, val);
                    store(val, r);
                }
            }
            // the next pass's products overwrite the accumulators: every read must be done
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncthreads();
        }
        if (*sabort != 0) break;
        if (g.M > OZ_M && part == 0 && cok)
            store((rfix[m] + rfix[OZ_M + m]) + (rfix[2 * OZ_M + m] + rfix[3 * OZ_M + m]), OZ_M);
    }
    if (*sabort != 0 && tid == 0) atomicExch(o.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(OZ_TCOLS));
}

// the S int8 digits of t (|t| < 64), most significant first: d0 = rint(t), t <- 128 (t - d0), ...
void digits_of(double t, int S, int8_t* d) {
    for (int i = 0; i < S; ++i) {
        const double r = std::nearbyint(t);
        t = (t - r) * 128.0;
        d[i] = (int8_t)(int)r;
    }
}

size_t ozaki_smem_bytes(const OzMat& om) {
    const size_t aop = (size_t)om.digits * om.ksteps * (OZ_M / 8) * 256;
    return OZ_HDR + ((om.img_bytes + 1023u) & ~1023u) + aop;
}

template <int S>
bool launch_s(const OzArgs& o, size_t sm, int grid, cudaStream_t s) {
    if (!allow_smem((const void*)k_ozaki<S>, sm)) return false;
    note_launch();
    k_ozaki<S><<<grid, OZ_T, sm, s>>>(o);
    return true;
}

}  // namespace

// The matrix A (M x K, row-major, FP64; M, K <= 129) as S int8 digits per entry with a
// power-of-two scale per row, in the shared-memory image of the MMA's B operand:
// B[n][k] = A[n][k], K-major, core matrices of 8 rows x 16 bytes, [digit][K step of 32][8-row
// group][2 x 128 B]; rows 0..127 and columns 0..127 of A on the tensor cores, row 128 and
// column 128 (when present) kept in FP64.
bool make_ozaki_mat(const double* A, int M, int K, int S, OzHost& out) {
    if (M < 1 || K < 1 || M > OZ_M + 1 || K > OZ_M + 1 || S != 5) return false;
    OzMat& om = out.mat;
    om.M = M;
    om.K = K;
    om.digits = S;
    const int mr = M < OZ_M ? M : OZ_M, kin = K < OZ_M ? K : OZ_M;
    om.nmma = ((mr + 15) / 16) * 16;
    om.kin = kin;
    om.ksteps = (kin + 31) / 32;
    const size_t per_digit = (size_t)om.ksteps * (om.nmma / 8) * 256;
    out.img.assign((size_t)S * per_digit, 0);
    out.rscale.assign(om.nmma, 1.0);
    std::vector<int8_t> d(S);
    for (int n = 0; n < mr; ++n) {
        double amax = 0.0;
        for (int k = 0; k < kin; ++k) amax = std::fmax(amax, std::fabs(A[(size_t)n * K + k]));
        int er = (amax > 0.0) ? std::ilogb(amax) + 1 : 0;
        if (er < -1000) er = -1000;
        out.rscale[n] = std::ldexp(1.0, er);
        const double inv = std::ldexp(1.0, 6 - er);
        for (int k = 0; k < kin; ++k) {
            digits_of(A[(size_t)n * K + k] * inv, S, d.data());
            const int st = k / 32, hf = (k % 32) / 16, kk = k % 16;
            const size_t off = ((size_t)st * (om.nmma / 8) + n / 8) * 256 + hf * 128 + (n % 8) * 16 + kk;
            for (int i = 0; i < S; ++i) out.img[i * per_digit + off] = (uint8_t)d[i];
        }
    }
    out.arow.clear();
    out.acol.clear();
    if (M > OZ_M) {
        // row 128 on the CUDA cores; none when it is a zero row (the lifted E's wall row)
        bool any = false;
        for (int k = 0; k < K; ++k) any = any || A[(size_t)OZ_M * K + k] != 0.0;
        if (any) out.arow.assign(A + (size_t)OZ_M * K, A + (size_t)OZ_M * K + K);
    }
    if (K > OZ_M) {
        out.acol.assign(OZ_M, 0.0);
        for (int n = 0; n < mr; ++n) out.acol[n] = A[(size_t)n * K + OZ_M];
    }
    om.img_bytes = (unsigned)(S * per_digit);
    return true;
}

bool launch_ozaki(const GemmArgs& g, const OzMat& om, int* err, cudaStream_t s) {
    if (om.img == nullptr || g.M != om.M || g.K != om.K) return false;
    const size_t sm = ozaki_smem_bytes(om);
    if (sm > smem_optin()) return false;
    OzArgs o{};
    o.g = g;
    o.img = reinterpret_cast<const uint4*>(om.img);
    o.img_bytes = om.img_bytes;
    o.rscale = om.rscale;
    o.arow = om.arow;
    o.acol = om.acol;
    o.nmma = om.nmma;
    o.ksteps = om.ksteps;
    o.kin = om.kin;
    o.err = err;
    const long long ntiles = ((g.C + OZ_M - 1) / OZ_M) * g.nfields;
    const int grid = (int)(ntiles < sm_count() ? ntiles : sm_count());
    return launch_s<5>(o, sm, grid, s);
}

}  // namespace lsb
