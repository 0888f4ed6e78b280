// z derivatives of the mixed-precision form on the fifth-generation tensor cores (tcgen05).
//
// In the mixed form the Chebyshev derivatives of the nonlinear term (dfdz of u, v, w and
// of the fluxes h_l3, src/navierstokes.f90:735-741, 796-804) feed FP32 transforms, so they
// need FP32 accuracy, not FP64.  They run as BF16 tcgen05 MMAs with FP32 accumulation in
// tensor memory, each FP64 operand split into three BF16 parts (hi + mid + lo carries the
// 24 bits of its FP32 value) and the six products hi.hi, hi.mid, mid.hi, hi.lo, mid.mid,
// lo.hi accumulated: an FP32-accurate contraction at a sixth of the BF16 rate.
//
// A CTA (4 warps, one per SM) walks tiles of 128 (kx, ky) columns: D[c][r] = sum_k in[k][c] A[r][k]
// with M = 128 columns, N = nzp padded to 16, K = nzp in steps of 16.  Both operands are
// K-major in the canonical no-swizzle layout (8 x 16-byte core matrices: leading byte offset
// 128 between the two K halves of a step, stride byte offset 256 between 8-row groups).  The
// split matrix is prepared on the host in exactly that layout and copied in once per CTA; the input
// columns arrive by cp.async in FP64 chunks of two K steps, double-buffered, so the next chunk
// loads while the CTA's threads split the current one into BF16 and one thread issues its MMAs,
// committed to an mbarrier that frees the split buffer for the next chunk.  Every wait is bounded: on time-out the kernel raises the handle's error word,
// frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "lsb_internal.cuh"

namespace lsb {

namespace {

constexpr int UM_M = 128;      // columns per CTA (MMA M)
constexpr int UM_CH = 2;       // K steps of 16 per producer chunk
constexpr int UM_TCOLS = 256;  // tensor-memory columns allocated (>= N, a power of two)
constexpr unsigned UM_ABUF = 3u * UM_CH * (UM_M / 8) * 256u;  // bytes of one split input chunk (3 splits)
constexpr unsigned UM_RAW = (unsigned)UM_M * UM_CH * 16u * 8u;    // bytes of one FP64 input chunk

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no swizzle, version 1 (sm_100): start >> 4, LBO >> 4 at bit 16, SBO >> 4 at bit 32
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// waits for the phase of the given parity with a time limit (about 0.2 s); false on time-out
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > 400000000LL) return false;
    }
}

struct UmmaArgs {
    GemmArgs g;             // fields, K, M, C, koff, roff, epilogue (EPI_STORE or EPI_AXPBY)
    const uint4* img;       // split matrix in the shared-memory image (3 splits x nsteps steps)
    unsigned img_bytes;
    int npad, nsteps, nchunks;
    int* err;               // raised to 1 when a wait times out
};

__global__ void __launch_bounds__(128, 1) k_umma_dz(UmmaArgs u) {
    extern __shared__ __align__(1024) unsigned char usm[];
    const GemmArgs& g = u.g;
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(usm);            // MMA completion
    uint32_t* tslot = reinterpret_cast<uint32_t*>(usm + 16);      // tensor-memory base address
    int* sabort = reinterpret_cast<int*>(usm + 32);
    unsigned char* bimg = usm + 1024;
    unsigned char* A = bimg + ((u.img_bytes + 1023u) & ~1023u);  // split chunk (MMA operand)
    double* raw[2];                                                // FP64 chunks [k][128 columns]
    raw[0] = reinterpret_cast<double*>(A + UM_ABUF);
    raw[1] = raw[0] + UM_RAW / 8;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
        *sabort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(UM_TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    const long long ntc = (g.C + UM_M - 1) / UM_M;
    const long long ntiles = ntc * g.nfields;
    const long long my_tiles = (blockIdx.x < ntiles) ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long long nseq = my_tiles * u.nchunks;
    // FP64 input chunk s (tile, chunk) -> raw[s & 1] by 16-byte cp.async, zero-filled past K and C
    auto issue = [&](long long s) {
        if (s < nseq) {
            const long long tile = blockIdx.x + (s / u.nchunks) * gridDim.x;
            const int q = (int)(s % u.nchunks);
            const int f = (int)(tile / ntc);
            const long long c0 = (tile - (long long)f * ntc) * UM_M;
            const double* in = (f < 4 && g.inf[f]) ? g.inf[f] : g.in + f * g.in_fstride;
            double* dst = raw[s & 1];
            for (int idx = tid; idx < UM_CH * 16 * (UM_M / 2); idx += 128) {
                const int kk = idx / (UM_M / 2), c2 = idx - kk * (UM_M / 2);
                const int k = q * UM_CH * 16 + kk;
                const long long c = c0 + 2 * c2;
                const bool ok = k < g.K && c < g.C;  // C is even
                const uint32_t sa = smem_u32(dst + kk * UM_M + 2 * c2);
                const double* src = ok ? in + (long long)(k + g.koff) * g.C + c : in;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 16 : 0));
            }
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    issue(0);
    // the split matrix, once per CTA (the CTA then walks its column tiles)
    for (unsigned i = tid; i < u.img_bytes / 16u; i += 128) {
        const uint32_t sa = smem_u32(bimg + 16u * i);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(u.img + i));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    // M = 128, N = npad, BF16 x BF16 -> F32, both K-major
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(u.npad >> 3) << 17) | ((uint32_t)(UM_M >> 4) << 24);
    const unsigned bstep = (unsigned)(u.npad / 8) * 256u;  // bytes of one K step of one split
    const int m = tid;
    for (long long s = 0; s < nseq; ++s) {
        const int q = (int)(s % u.nchunks);
        issue(s + 1);
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();
        // the split buffer still feeds chunk s - 1's MMAs until they complete
        if (s >= 1 && *sabort == 0 && !mbar_wait(smem_u32(mbar), (uint32_t)((s - 1) & 1))) *sabort = 1;
        const double* x = raw[s & 1];
#pragma unroll
        for (int sl = 0; sl < UM_CH; ++sl) {
            uint32_t hw[3][8];
#pragma unroll
            for (int k2 = 0; k2 < 8; ++k2) {
                uint32_t h[3][2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const float xf = (float)x[(sl * 16 + 2 * k2 + e) * UM_M + m];
                    const __nv_bfloat16 h0 = __float2bfloat16_rn(xf);
                    const float r1 = xf - __bfloat162float(h0);
                    const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
                    const float r2 = r1 - __bfloat162float(h1);
                    h[0][e] = __bfloat16_as_ushort(h0);
                    h[1][e] = __bfloat16_as_ushort(h1);
                    h[2][e] = __bfloat16_as_ushort(__float2bfloat16_rn(r2));
                }
#pragma unroll
                for (int p = 0; p < 3; ++p) hw[p][k2] = h[p][0] | (h[p][1] << 16);
            }
#pragma unroll
            for (int p = 0; p < 3; ++p)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                    *reinterpret_cast<uint4*>(A + ((p * UM_CH + sl) * (UM_M / 8) + (m >> 3)) * 256 + j * 128 + (m & 7) * 16) =
                        make_uint4(hw[p][4 * j], hw[p][4 * j + 1], hw[p][4 * j + 2], hw[p][4 * j + 3]);
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0 && *sabort == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // the six products of the three-way splits, largest first
            const int pa[6] = {0, 0, 1, 0, 1, 2};
            const int pb[6] = {0, 1, 0, 2, 1, 0};
            for (int sl = 0; sl < UM_CH; ++sl) {
                const int step = q * UM_CH + sl;
                if (step >= u.nsteps) break;
                for (int t = 0; t < 6; ++t) {
                    const uint64_t ad = umma_desc(smem_u32(A + (pa[t] * UM_CH + sl) * (UM_M / 8) * 256), 128, 256);
                    const uint64_t bd = umma_desc(smem_u32(bimg + (pb[t] * u.nsteps + step) * bstep), 128, 256);
                    umma_bf16(tmem, ad, bd, idesc, (q | sl | t) != 0 ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(mbar)));
        }
        if (q != u.nchunks - 1) continue;
        // the tile's last commit covers all its MMAs: read the accumulator out
        if (*sabort == 0 && !mbar_wait(smem_u32(mbar), (uint32_t)(s & 1))) *sabort = 1;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        __syncthreads();
        if (*sabort != 0) break;
        const long long tile = blockIdx.x + (s / u.nchunks) * gridDim.x;
        const int f = (int)(tile / ntc);
        const long long c = (tile - (long long)f * ntc) * UM_M + m;
        const bool cok = c < g.C;
        double* out = (f < 4 && g.outf[f]) ? g.outf[f] : g.out + f * g.out_fstride;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        for (int j = 0; j < u.npad / 16; ++j) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + lane_base + (uint32_t)(j * 16)));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (!cok) continue;
            double old[16];
            if (g.epi == EPI_AXPBY && g.beta != 0.0) {
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int r = j * 16 + e;
                    old[e] = (r < g.M) ? out[(long long)(r + g.roff) * g.C + c] : 0.0;
                }
            }
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int r = j * 16 + e;
                if (r >= g.M) continue;
                double val = (double)__uint_as_float(v[e]);
                if (g.epi == EPI_AXPBY) val = g.alpha * val + (g.beta != 0.0 ? g.beta * old[e] : 0.0);
                out[(long long)(r + g.roff) * g.C + c] = val;
            }
        }
        // the next tile's first MMA overwrites the accumulator: all reads must be done
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    if (*sabort != 0 && tid == 0) atomicExch(u.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(UM_TCOLS));
}

uint16_t bf16_bits_rn(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan: not produced here
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
float bf16_to_float(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace

// three-way BF16 split of the matrix A (M x K, row-major, FP64) in the shared-memory image of
// the B operand: B[k][n] = A[n][k], K-major, steps of 16 in K, 8-row groups in N
UmmaMat make_umma_mat(const double* A, int M, int K, std::vector<uint16_t>& img) {
    UmmaMat um;
    um.M = M;
    um.K = K;
    um.npad = ((M + 15) / 16) * 16;
    um.nsteps = (K + 15) / 16;
    const size_t per_split = (size_t)um.nsteps * um.npad * 16;  // elements
    img.assign(3 * per_split, 0);
    for (int n = 0; n < M; ++n)
        for (int k = 0; k < K; ++k) {
            const float xf = (float)A[(size_t)n * K + k];
            const uint16_t h0 = bf16_bits_rn(xf);
            const float r1 = xf - bf16_to_float(h0);
            const uint16_t h1 = bf16_bits_rn(r1);
            const float r2 = r1 - bf16_to_float(h1);
            const uint16_t h2 = bf16_bits_rn(r2);
            const int s = k / 16, j = (k % 16) / 8, kk = k % 8, i = n / 8, rr = n % 8;
            const size_t off = (((size_t)s * (um.npad / 8) + i) * 256 + j * 128 + rr * 16 + kk * 2) / 2;
            img[0 * per_split + off] = h0;
            img[1 * per_split + off] = h1;
            img[2 * per_split + off] = h2;
        }
    um.img_bytes = (unsigned)(3 * per_split * 2);
    return um;
}

size_t umma_smem_bytes(const UmmaMat& um) {
    return 1024 + ((um.img_bytes + 1023u) & ~1023u) + (size_t)UM_ABUF + 2 * (size_t)UM_RAW;
}

bool launch_umma_dz(const GemmArgs& g, const UmmaMat& um, int* err, cudaStream_t s) {
    if (um.img == nullptr || g.epi > EPI_AXPBY || um.npad > UM_TCOLS || g.K != um.K || g.M != um.M) return false;
    const size_t sm = umma_smem_bytes(um);
    if (!allow_smem((const void*)k_umma_dz, sm)) return false;
    UmmaArgs u{};
    u.g = g;
    u.img = reinterpret_cast<const uint4*>(um.img);
    u.img_bytes = um.img_bytes;
    u.npad = um.npad;
    u.nsteps = um.nsteps;
    u.nchunks = (um.nsteps + UM_CH - 1) / UM_CH;
    u.err = err;
    const long long ntiles = ((g.C + UM_M - 1) / UM_M) * g.nfields;
    const int grid = (int)(ntiles < sm_count() ? ntiles : sm_count());
    note_launch();
    k_umma_dz<<<grid, 128, sm, s>>>(u);
    return true;
}

}  // namespace lsb
