// lsb_solve_helmholtz_noalloc: the Helmholtz / Poisson solve of solve_helmholtz for
// callers that are not allowed to allocate GPU memory.
//
// Who needs it: a host program whose device memory is owned by someone else -- a
// pool allocator or framework that hands out every byte and forbids direct
// cudaMalloc -- or a time-stepping loop that cannot afford cudaMalloc / cudaFree,
// which synchronize the whole device.  Such a caller can pass device pointers it
// already holds, but cannot let the library create a handle (lsb_create allocates).
//
// How: all working memory of this entry point (the zero-padded eigenvector
// matrices and the intermediate E^-1 . rhs tile) lives in one file-scope
// __device__ array of LSB_NOALLOC_SCRATCH_BYTES.  Every GPU that loads the library
// keeps that array for the life of the process.  The columns are solved in chunks
// that fit the array, so the grid size is limited only through nz (nzp <= 129).
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current and caches it; make that first
// call outside any stream capture.  Calls share the array and it keeps the last
// call's contents: calls that overlap on the GPU (two streams, or two host threads
// on one device) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "lsbgpu.h"

namespace lsb {
void set_last_error(const std::string& m);  // lsbgpu.cu
void note_launch();                         // lsbgpu.cu
}

namespace {

constexpr long long kScratchDoubles = LSB_NOALLOC_SCRATCH_BYTES / 8;
constexpr int kMaxNzp = 129;
constexpr int kBN = 64, kBK = 16, kLDA = 20, kLDB = 68;
constexpr int kMaxMp = 136;               // rows of the padded eigenvector matrices
constexpr int kMaxKp = 128;               // padded nzm
constexpr long long kMatDoubles = 2LL * kMaxMp * kMaxKp;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_ptr[64] = {nullptr};    // device address per device ordinal

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Zero-padded copies [Mp][Kp] of Ei (nzm x nzm) and of E extended with zero ceiling /
// wall rows ((nzm+2) x nzm), written into the scratch (every entry, each call).
__global__ void k_pad_mats(const double* __restrict__ e, const double* __restrict__ ei, int nzm, int mp1, int mp2,
                           int kp, double* __restrict__ a1, double* __restrict__ a2) {
    const long long n1 = (long long)mp1 * kp, n2 = (long long)mp2 * kp;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n1 + n2; x += (long long)gridDim.x * blockDim.x) {
        if (x < n1) {
            const int r = (int)(x / kp), k = (int)(x % kp);
            a1[x] = (r < nzm && k < nzm) ? ei[(long long)r * nzm + k] : 0.0;
        } else {
            const long long y = x - n1;
            const int r = (int)(y / kp), k = (int)(y % kp);
            a2[y] = (r >= 1 && r <= nzm && k < nzm) ? e[(long long)(r - 1) * nzm + k] : 0.0;
        }
    }
}

// out[r][c] = sum_k A[r][k] in[k + koff][c] for columns c0 <= c < c0 + ncols of a field
// whose rows have ld doubles; phase 1 scales by 1/(lam[r] - kx^2 - ky^2 - sigma).
template <int MT, bool SCALE>
__global__ void __launch_bounds__(256) k_helm_chunk(const double* __restrict__ A, int M, int K, int kp,
                                                    const double* __restrict__ in, long long in_ld, int koff,
                                                    double* __restrict__ out, long long out_ld, long long c0,
                                                    long long ncols, long long in_c0, long long out_c0,
                                                    const double* __restrict__ lam, const double* __restrict__ wavx,
                                                    const double* __restrict__ wavy, int nx, double sigma) {
    __shared__ double As[MT * 8][kLDA];
    __shared__ double Bs[kBK][kLDB];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long cb0 = (long long)blockIdx.x * kBN;
    double acc[MT][2];
#pragma unroll
    for (int t = 0; t < MT; ++t) acc[t][0] = acc[t][1] = 0.0;
    for (int kc = 0; kc < kp; kc += kBK) {
        for (int idx = tid; idx < MT * 8 * kBK; idx += 256) {
            const int r = idx / kBK, cc = idx % kBK;
            As[r][cc] = A[(long long)r * kp + kc + cc];
        }
        for (int idx = tid; idx < kBK * kBN; idx += 256) {
            const int kk = idx / kBN, n = idx % kBN;
            const int k = kc + kk;
            const long long cl = cb0 + n;
            Bs[kk][n] = (k < K && cl < ncols) ? in[(long long)(k + koff) * in_ld + in_c0 + cl] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < kBK / 4; ++k4) {
            const double b = Bs[k4 * 4 + (lane & 3)][warp * 8 + (lane >> 2)];
#pragma unroll
            for (int t = 0; t < MT; ++t) dmma884(acc[t], As[t * 8 + (lane >> 2)][k4 * 4 + (lane & 3)], b);
        }
        __syncthreads();
    }
#pragma unroll
    for (int t = 0; t < MT; ++t) {
        const int r = t * 8 + (lane >> 2);
        if (r >= M) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const long long cl = cb0 + warp * 8 + (lane & 3) * 2 + e;
            if (cl >= ncols) continue;
            double v = acc[t][e];
            if (SCALE) {
                const long long c = c0 + cl;  // column within the (kx, ky) plane
                const double wx = wavx[c % nx], wy = wavy[c / nx];
                const double dfac = (-(wx * wx + wy * wy)) - sigma;
                v = v / (lam[r] + dfac);
            }
            out[(long long)r * out_ld + out_c0 + cl] = v;
        }
    }
}

template <bool SCALE>
void launch_chunk(int mt, dim3 grid, cudaStream_t s, const double* A, int M, int K, int kp, const double* in,
                  long long in_ld, int koff, double* out, long long out_ld, long long c0, long long ncols,
                  long long in_c0, long long out_c0, const double* lam, const double* wavx, const double* wavy,
                  int nx, double sigma) {
    switch (mt) {
#define LSB_NA(n)                                                                                          \
    case n:                                                                                                \
        { lsb::note_launch(); k_helm_chunk<n, SCALE><<<grid, 256, 0, s>>>(A, M, K, kp, in, in_ld, koff, out, out_ld, c0, ncols, \
                                                    in_c0, out_c0, lam, wavx, wavy, nx, sigma); }            \
        break;
        LSB_NA(1) LSB_NA(2) LSB_NA(3) LSB_NA(4) LSB_NA(5) LSB_NA(6) LSB_NA(7) LSB_NA(8) LSB_NA(9)
        LSB_NA(10) LSB_NA(11) LSB_NA(12) LSB_NA(13) LSB_NA(14) LSB_NA(15) LSB_NA(16) LSB_NA(17)
#undef LSB_NA
        default: break;
    }
}

int fail(int code, const std::string& m) {
    lsb::set_last_error(m);  // reported by lsb_last_error()
    return code;
}

}  // namespace

extern "C" int lsb_solve_helmholtz_noalloc(int nx, int ny, int nz, const double* rhs, double* out, const double* lam,
                                           const double* e, const double* ei, const double* wavx,
                                           const double* wavy, double dtnui, void* stream) {
    if (!rhs || !out || !lam || !e || !ei || !wavx || !wavy) return fail(LSB_ERR_ARG, "null pointer argument");
    if (rhs == out) return fail(LSB_ERR_ARG, "rhs and out must not alias");
    if (nx < 2 || nx % 2 || ny < 1 || nz < 3) return fail(LSB_ERR_ARG, "bad grid size");
    const int nzp = nz + 1, nzm = nz - 1;
    if (nzp > kMaxNzp)
        return fail(LSB_ERR_UNSUPPORTED, "nz = " + std::to_string(nz) + " exceeds the no-allocation limit nzp <= " +
                                             std::to_string(kMaxNzp));
    const int kp = ((nzm + 15) / 16) * 16;
    const int mp1 = ((nzm + 7) / 8) * 8, mp2 = ((nzp + 7) / 8) * 8;
    const long long C = (long long)nx * ny;
    const long long avail = kScratchDoubles - kMatDoubles;
    long long chunk = (avail / nzm) / kBN * kBN;  // columns per pass, a multiple of the tile
    if (chunk < kBN) return fail(LSB_ERR_UNSUPPORTED, "scratch too small for nzm = " + std::to_string(nzm));
    if (chunk > C) chunk = C;

    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(LSB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (dev < 0 || dev >= 64) return fail(LSB_ERR_UNSUPPORTED, "device ordinal out of range");
    double* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_scratch_ptr[dev] == nullptr) {
            // once per device, with that device current: the device address of the array
            void* p = nullptr;
            ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (ce != cudaSuccess)
                return fail(LSB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
            g_scratch_ptr[dev] = (double*)p;
        }
        base = g_scratch_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (s != nullptr) {
        // the scratch address above belongs to the current device: the stream must too
        int sdev = -1;
        ce = cudaStreamGetDevice(s, &sdev);
        if (ce != cudaSuccess) return fail(LSB_ERR_CUDA, std::string("cudaStreamGetDevice: ") + cudaGetErrorString(ce));
        if (sdev != dev)
            return fail(LSB_ERR_ARG, "the stream belongs to device " + std::to_string(sdev) + ", not the current device " +
                                         std::to_string(dev));
    }
    double* a1 = base;                        // padded E^-1
    double* a2 = base + (long long)kMaxMp * kMaxKp;  // padded E with zero ceiling / wall rows
    double* tmp = base + kMatDoubles;         // nzm x chunk intermediate
    { lsb::note_launch(); k_pad_mats<<<64, 256, 0, s>>>(e, ei, nzm, mp1, mp2, kp, a1, a2); }
    for (long long c0 = 0; c0 < C; c0 += chunk) {
        const long long nc = (C - c0 < chunk) ? C - c0 : chunk;
        dim3 grid((unsigned)((nc + kBN - 1) / kBN));
        // phase 1: tmp = (E^-1 . rhs[1..nz-1]) / (lam - k^2 - sigma)
        launch_chunk<true>(mp1 / 8, grid, s, a1, nzm, nzm, kp, rhs, C, 1, tmp, nc, c0, nc, c0, 0, lam, wavx, wavy,
                           nx, dtnui);
        // phase 2: out[0..nzp-1] = E_ext . tmp  (rows 0 and nzp-1 are exactly 0)
        launch_chunk<false>(mp2 / 8, grid, s, a2, nzp, nzm, kp, tmp, nc, 0, out, C, c0, nc, 0, c0, lam, wavx, wavy,
                            nx, 0.0);
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(LSB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(ce));
    return LSB_OK;
}
