// Subgrid-scale stresses in physical space (src/sgsterm.f90:10-467) with the
// 3-point x/y/z test filter of filter_q_3pt (src/filters.f90:363-613), and the
// reductions of the diagnostics (maxcalc, divcheck, ener).
//
// Fields live on the unpadded physical grid [nzp][ny][nx] (one GPU: the spanwise
// halo exchange of filtery_q_3pt becomes a periodic wrap).  Tensor fields are stored
// as 9 components with index 3*l + m (du_l/dx_m), symmetric ones as 6 components
// (11, 12, 13, 22, 23, 33).  Floating-point expressions keep the reference's order.
#include <cmath>
#include <cstring>
#include <vector>

#include "lsb_handle.cuh"
#include "lsb_sgs.cuh"
#include "lsb_spectral.cuh"
#include "lsb_tma.cuh"

namespace lsb {

namespace {
void sfail(int code, const std::string& m) { throw LsbError{code, m}; }


inline int nblk(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148LL * 16) b = 148LL * 16;
    if (b < 1) b = 1;
    return (int)b;
}

constexpr int kFilterFields = 24;  // fields per filter launch
struct FieldList {
    const double* in[kFilterFields];
    double* out[kFilterFields];
    int n;
};
struct P9 {
    const double* p[9];
};
struct W9 {
    double* p[9];
};

// filter_q_3pt: x (periodic) then y (periodic) then z (interior planes, non-uniform
// weights; the ceiling and wall planes are xy-filtered only, src/filters.f90:450).
// A block owns a JB x IB tile of (y, x) columns and marches a chunk of ZC planes in z:
// each plane is read once into shared memory with a one-point periodic halo, filtered in
// x and y, and the last three y-filtered planes are kept in registers for the z stencil.
constexpr int FIB = 32, FJB = 8, FZC = 16;

__global__ void __launch_bounds__(256) k_filter3(FieldList fl, int nx, int ny, int nzp, double a, double b,
                                                 const double* __restrict__ az, const double* __restrict__ bz,
                                                 const double* __restrict__ cz, int nzc) {
    __shared__ double tile[FJB + 2][FIB + 2];
    __shared__ double X[FJB + 2][FIB];
    const int f = blockIdx.z / nzc, zc = blockIdx.z % nzc;
    const double* q = fl.in[f];
    double* out = fl.out[f];
    const int i0 = blockIdx.x * FIB, j0 = blockIdx.y * FJB;
    const int k0 = zc * FZC, k1 = min(nzp, k0 + FZC);  // output planes [k0, k1)
    const int ks = max(0, k0 - 1), ke = min(nzp - 1, k1);
    const double rs = 1.0 / (2.0 * a + b);  // the reference divides by 2a+b; one rounding apart
    const int tid = threadIdx.x;
    const int jj = tid / FIB, ii = tid % FIB;  // this thread's output column (256 = FJB * FIB)
    const int jo = j0 + jj, io = i0 + ii;
    const bool mine = (jo < ny) && (io < nx);
    // periodic source indices of the two tile elements this thread loads per plane
    long long off[2];
    bool ld[2];
    for (int r = 0; r < 2; ++r) {
        const int idx = tid + 256 * r;
        ld[r] = idx < (FJB + 2) * (FIB + 2);
        const int jr = idx / (FIB + 2), ir = idx % (FIB + 2);
        int j = j0 + jr - 1, i = i0 + ir - 1;
        j = ((j % ny) + ny) % ny;
        i = ((i % nx) + nx) % nx;
        off[r] = (long long)j * nx + i;
    }
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;  // y-filtered planes kk-2, kk-1, kk
    double* tflat = &tile[0][0];
    for (int kk = ks; kk <= ke; ++kk) {
        const double* pl = q + (long long)kk * ny * nx;
        if (ld[0]) tflat[tid] = __ldg(pl + off[0]);
        if (ld[1]) tflat[tid + 256] = __ldg(pl + off[1]);
        __syncthreads();
        for (int idx = tid; idx < (FJB + 2) * FIB; idx += 256) {
            const int jr = idx / FIB, ir = idx % FIB;
            X[jr][ir] = (a * tile[jr][ir] + b * tile[jr][ir + 1] + a * tile[jr][ir + 2]) * rs;
        }
        __syncthreads();
        const double yn = (a * X[jj][ii] + b * X[jj + 1][ii] + a * X[jj + 2][ii]) * rs;
        y0 = y1;
        y1 = y2;
        y2 = yn;
        if (mine) {
            const int ko = kk - 1;  // plane whose z stencil is now complete
            if (ko >= k0 && ko < k1) {
                double v;
                if (ko == 0) v = y1;
                else v = (az[ko] * y0 + bz[ko] * y1 + cz[ko] * y2) * rs;
                out[((long long)ko * ny + jo) * nx + io] = v;
            }
            if (kk == nzp - 1 && kk >= k0 && kk < k1) out[((long long)kk * ny + jo) * nx + io] = yn;
        }
        __syncthreads();
    }
}

// Row-tile version of the same filter (nx a power of two, 4..512): a block owns FJ
// full x rows (FJ * nx = 2048) and marches a chunk of zch planes.  Each plane with its
// periodic y halo rows is copied into shared memory by cp.async, three planes deep, so
// two planes are in flight while one is filtered; the x halo is the row itself (periodic).
// The only re-reads are the two y halo rows and the two z halo planes of the chunk.
constexpr int RT_NX = 512, RT_ST = 3;

__device__ __forceinline__ void cpa16s(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cpa_commit_s() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cpa_wait_s() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Thread -> an x pair (2p, 2p+1) and FR consecutive output rows of the block's FJ rows
// (FJ = FR * 512 / nx), so the x filter reads one vector and two neighbours per row straight
// from the plane tile and the y and z filters run in registers: one barrier per plane.
constexpr int FR = 4;

// the input fields' row maps ([nzp * ny][nx], box of min(nx, 256) x 1) for TMA staging
struct alignas(64) FiltMaps {
    CUtensorMap m[kFilterFields];
};

// three blocks per SM fit the FP32 form in 80 registers; the FP64 form would spill there.
// TMA = true: each plane of the ring (the block's rows and their two periodic y halo rows)
// is brought in by TMA row loads, one per lane of warp 0 (issued from one thread they
// serialised and ran slower than cp.async), completing on an mbarrier per ring slot
// (bounded waits: a time-out raises *err and ends the block after its loads in flight have
// landed); TMA = false: cp.async by all threads.
template <class T, bool TMA>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) k_filter3p(FieldList fl, int lgx, int ny, int nzp, int FJ, int zch, T a, T b,
                                                     const double* __restrict__ az, const double* __restrict__ bz,
                                                     const double* __restrict__ cz,
                                                     const __grid_constant__ FiltMaps tm, int* err) {
    using V2 = typename Vec2<T>::type;
    const int nx = 1 << lgx, NP = nx >> 1;
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    // TMA destinations are 128-byte aligned: the tiles start on a 128-byte boundary and a
    // row is a multiple of 128 bytes (checked by the host)
    unsigned char* sbase = TMA ? fsm_raw + ((128u - (unsigned)(__cvta_generic_to_shared(fsm_raw) & 127u)) & 127u)
                               : fsm_raw;
    const int tsz = (FJ + 2) * nx;
    T* tiles = reinterpret_cast<T*>(sbase);  // RT_ST tiles of (FJ + 2) rows
    uint64_t* bar = reinterpret_cast<uint64_t*>(tiles + RT_ST * tsz);  // [RT_ST] (TMA)
    int* sabort = reinterpret_cast<int*>(bar + RT_ST);
    // FP64: the z filter's row coefficients, staged once (their loads had been waited for at
    // every plane: 163 -> 159 us per step at 256x64x129; the FP32 form measured slower with
    // them staged, 112 -> 117 us); the first plane's barrier orders these stores before their
    // reads
    constexpr bool ZS = sizeof(T) == 8;
    double* zco = reinterpret_cast<double*>(bar + RT_ST + 1);  // [3][nzp]: az, bz, cz
    if (ZS)
        for (int i = threadIdx.x; i < 3 * nzp; i += blockDim.x)
            zco[i] = (i < nzp) ? az[i] : (i < 2 * nzp ? bz[i - nzp] : cz[i - 2 * nzp]);
    const double* zaa = ZS ? zco : az;
    const double* zbb = ZS ? zco + nzp : bz;
    const double* zcc = ZS ? zco + 2 * nzp : cz;
    const int f = blockIdx.z, zc = blockIdx.y;
    const T* q = reinterpret_cast<const T*>(fl.in[f]);
    T* out = reinterpret_cast<T*>(fl.out[f]);
    const int j0 = blockIdx.x * FJ;
    const int rows = min(FJ, ny - j0);
    const int k0 = zc * zch, k1 = min(nzp, k0 + zch);
    const int ks = max(0, k0 - 1), ke = min(nzp - 1, k1);
    const T rs = (T)(1.0 / (2.0 * (double)a + (double)b));
    const int tid = threadIdx.x;
    const int p = tid & (NP - 1), r0 = (tid >> (lgx - 1)) * FR;
    const int xl = (2 * p - 1) & (nx - 1), xr = (2 * p + 2) & (nx - 1);
    constexpr int V = 16 / sizeof(T);          // elements per 16-byte copy
    constexpr int LGV = (V == 2) ? 1 : 2;
    const int lgrv = lgx - LGV;                // log2 of the copies per row
    const int nld_v = (rows + 2) << lgrv;
    const long long plane = (long long)ny * nx;
    const int bx = nx < 256 ? nx : 256;        // TMA box width
    // per ring slot i: bit i of phm is the mbarrier phase to wait for, bit i of infm marks a
    // load in flight (bits of a register: indexed arrays of these went to local memory)
    uint32_t phm = 0u, infm = 0u;
    if (TMA) {
        if (tid == 0) {
            for (int i = 0; i < RT_ST; ++i) tma::mbar_init(&bar[i], 1);
            tma::fence_init();
            *sabort = 0;
        }
        __syncthreads();
    }
    auto issue = [&](int kk) {
        if (TMA) {
            if (kk > ke) return;
            const int sl = kk % RT_ST;
            if (tid < 32) {
                // warp 0 issues the plane's row loads, one per lane (lane 0 first announces
                // their bytes); the block's reads of this slot, ordered before this call by a
                // barrier, come before the TMA's writes
                T* dst = tiles + sl * tsz;
                tma::fence_proxy_async();
                if (tid == 0) tma::mbar_expect_tx(&bar[sl], (uint32_t)((rows + 2) * nx * (int)sizeof(T)));
                __syncwarp();
                const int nb = nx / bx;
                for (int i = tid; i < (rows + 2) * nb; i += 32) {
                    const int r = i / nb, x0 = (i - r * nb) * bx;
                    int j = j0 + r - 1;
                    j = (j < 0) ? j + ny : (j >= ny ? j - ny : j);
                    tma::load_2d(dst + (r << lgx) + x0, &tm.m[f], x0, kk * ny + j, &bar[sl]);
                }
            }
            infm |= 1u << sl;
            return;
        }
        if (kk <= ke) {
            T* dst = tiles + (kk % RT_ST) * tsz;
            const T* src = q + (long long)kk * plane;
            for (int c = tid; c < nld_v; c += 256) {
                const int r = c >> lgrv, cv = c & ((1 << lgrv) - 1);
                int j = j0 + r - 1;
                j = (j < 0) ? j + ny : (j >= ny ? j - ny : j);
                cpa16s(dst + (r << lgx) + cv * V, src + ((long long)j << lgx) + cv * V);
            }
        }
        cpa_commit_s();  // one group per plane slot, empty past the end
    };
    issue(ks);
    issue(ks + 1);
    T y0[FR][2], y1[FR][2], y2[FR][2];
#pragma unroll
    for (int i = 0; i < FR; ++i) y0[i][0] = y0[i][1] = y1[i][0] = y1[i][1] = y2[i][0] = y2[i][1] = (T)0;
    for (int kk = ks; kk <= ke; ++kk) {
        if (TMA) {
            const int sl = kk % RT_ST;
            if (tma::mbar_wait(&bar[sl], (phm >> sl) & 1u)) {
                phm ^= 1u << sl;
                infm &= ~(1u << sl);
            } else {
                *sabort = 1;  // the slot stays in flight for the clean-up below
            }
        } else {
            cpa_wait_s<1>();
        }
        __syncthreads();  // plane kk has landed; every thread is done with plane kk - 1's slot
        if (TMA && *sabort != 0) break;
        issue(kk + 2);
        const T* tile = tiles + (kk % RT_ST) * tsz;
        // x filter of tile rows r0 .. r0 + FR + 1 (grid rows j0 + r0 - 1 ..), then y filter
        T xf[FR + 2][2];
#pragma unroll
        for (int i = 0; i < FR + 2; ++i) {
            const T* row = tile + (r0 + i) * nx;
            const V2 c = *reinterpret_cast<const V2*>(row + 2 * p);
            const T l = row[xl], rr = row[xr];
            xf[i][0] = (a * l + b * c.x + a * c.y) * rs;
            xf[i][1] = (a * c.x + b * c.y + a * rr) * rs;
        }
        const int ko = kk - 1;
        const T za = (ko >= 1) ? (T)zaa[ko] : (T)0, zb = (ko >= 1) ? (T)zbb[ko] : (T)0,
                zcf = (ko >= 1) ? (T)zcc[ko] : (T)0;
#pragma unroll
        for (int i = 0; i < FR; ++i) {
            T yn[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                yn[e] = (a * xf[i][e] + b * xf[i + 1][e] + a * xf[i + 2][e]) * rs;
                y0[i][e] = y1[i][e];
                y1[i][e] = y2[i][e];
                y2[i][e] = yn[e];
            }
            if (r0 + i >= rows) continue;
            const long long ob = (long long)(j0 + r0 + i) * nx + 2 * p;
            if (ko >= k0 && ko < k1) {
                V2 v;
                if (ko == 0) {
                    v.x = y1[i][0];
                    v.y = y1[i][1];
                } else {
                    v.x = (za * y0[i][0] + zb * y1[i][0] + zcf * y2[i][0]) * rs;
                    v.y = (za * y0[i][1] + zb * y1[i][1] + zcf * y2[i][1]) * rs;
                }
                *reinterpret_cast<V2*>(out + (long long)ko * plane + ob) = v;
            }
            if (kk == nzp - 1 && kk >= k0 && kk < k1) {
                V2 v;
                v.x = yn[0];
                v.y = yn[1];
                *reinterpret_cast<V2*>(out + (long long)kk * plane + ob) = v;
            }
        }
    }
    if (TMA) {
        // after a time-out: the loads still in flight land before the block exits (bounded
        // waits again), and the launch's error word is raised
        if (*sabort != 0) {
            for (int i = 0; i < RT_ST; ++i)
                if ((infm >> i) & 1u) tma::mbar_wait(&bar[i], (phm >> i) & 1u);
            if (tid == 0 && err) atomicExch(err, 1);
        }
    } else {
        cpa_wait_s<0>();
    }
}

void filter3_any(lsb_handle* h, const void* const* in, void* const* out, int n, double a, double b, int which,
                 bool f32) {
    const Dims& d = h->d;
    const double* zf = h->sgs.zf + (long long)which * 3 * d.nzp;  // which: 0 (a,b) 1 (1,1) 2 (1,6) 3 (1,2)
    int lgx = 0;
    while ((1 << lgx) < d.nx) ++lgx;
    const bool rowtile = d.nx <= RT_NX && d.nx >= 4 && (1 << lgx) == d.nx;
    if (!rowtile && f32) sfail(LSB_ERR_UNSUPPORTED, "mixed precision: the SGS filter needs nx a power of two, 4..512");
    for (int f0 = 0; f0 < n; f0 += kFilterFields) {
        FieldList fl{};
        fl.n = std::min(kFilterFields, n - f0);
        for (int i = 0; i < fl.n; ++i) {
            fl.in[i] = reinterpret_cast<const double*>(in[f0 + i]);
            fl.out[i] = reinterpret_cast<double*>(out[f0 + i]);
        }
        TimerScope ts(h, "sgs_filter3");
        if (rowtile) {
            const int FJ = FR * 512 / d.nx;  // the thread map's rows (rows past ny are masked)
            const int nyb = (d.ny + FJ - 1) / FJ;
            const size_t es = f32 ? sizeof(float) : sizeof(double);
            // TMA row loads need 128-byte rows (the destinations' alignment); the built-in
            // choice (filter_staging 0) is TMA for FP64 rows and cp.async for FP32 ones (at
            // 256 x 64 x 129: FP64 172 -> 167 us per step with TMA; FP32 112 -> 129 us)
            FiltMaps tm;
            std::memset(&tm, 0, sizeof(tm));
            const bool tma_ok = (d.nx * es) % 128 == 0;
            bool tma = tma_ok && (h->sched.filter_staging == 2 || (h->sched.filter_staging == 0 && !f32));
            for (int i = 0; tma && i < fl.n; ++i)
                tma = tmap_rows(&tm.m[i], fl.in[i], (uint32_t)es, (uint64_t)d.nx, (uint64_t)d.nzp * d.ny,
                                (uint32_t)std::min(d.nx, 256));
            if (!tma && h->sched.filter_staging == 2) sfail(LSB_ERR_UNSUPPORTED, "filter_staging 2: no TMA row maps for this grid");
            const size_t tiles = (size_t)RT_ST * (FJ + 2) * d.nx * es;
            // (TMA: 128-byte alignment slack) tiles, the TMA barriers and the abort flag, the z
            // coefficients (FP64)
            const size_t sm = (tma ? 128 : 0) + tiles + (RT_ST + 1) * sizeof(uint64_t) +
                              (f32 ? 0 : 3 * (size_t)d.nzp * sizeof(double));
            const void* kf = f32 ? (tma ? (const void*)k_filter3p<float, true> : (const void*)k_filter3p<float, false>)
                                 : (tma ? (const void*)k_filter3p<double, true> : (const void*)k_filter3p<double, false>);
            if (!allow_smem(kf, sm)) sfail(LSB_ERR_UNSUPPORTED, "SGS filter: shared memory of the plane ring refused");
            // z chunks: a block marches zch planes plus the two halo planes; pick the chunk
            // count with the least (waves of resident blocks) x (planes per block)
            const long long slots = std::max(1LL, (long long)resident_blocks(kf, 256, sm) * sm_count());
            int zch = d.nzp;
            double best = -1.0;
            for (int c = 1; c <= std::max(1, (d.nzp + 3) / 4); ++c) {
                const int zc = (d.nzp + c - 1) / c;
                const int nc = (d.nzp + zc - 1) / zc;
                const long long blocks = (long long)nyb * nc * fl.n;
                const double cost = (double)((blocks + slots - 1) / slots) * (zc + 2);
                if (best < 0.0 || cost < best) best = cost, zch = zc;
            }
            const int force = h->sched.filter_zchunks;  // a tuned schedule overrides the model
            if (force >= 1 && force <= std::max(1, (d.nzp + 3) / 4)) zch = (d.nzp + force - 1) / force;
            const int nzc = (d.nzp + zch - 1) / zch;
            dim3 grid(nyb, nzc, fl.n);
            const double* z0 = zf;
            const double* z1 = zf + d.nzp;
            const double* z2 = zf + 2 * d.nzp;
            lsb::note_launch();
            if (f32) {
                if (tma) k_filter3p<float, true><<<grid, 256, sm, h->stream>>>(fl, lgx, d.ny, d.nzp, FJ, zch, (float)a, (float)b, z0, z1, z2, tm, h->uerr);
                else k_filter3p<float, false><<<grid, 256, sm, h->stream>>>(fl, lgx, d.ny, d.nzp, FJ, zch, (float)a, (float)b, z0, z1, z2, tm, h->uerr);
            } else {
                if (tma) k_filter3p<double, true><<<grid, 256, sm, h->stream>>>(fl, lgx, d.ny, d.nzp, FJ, zch, a, b, z0, z1, z2, tm, h->uerr);
                else k_filter3p<double, false><<<grid, 256, sm, h->stream>>>(fl, lgx, d.ny, d.nzp, FJ, zch, a, b, z0, z1, z2, tm, h->uerr);
            }
        } else {
            const int nzc = (d.nzp + FZC - 1) / FZC;
            dim3 grid((d.nx + FIB - 1) / FIB, (d.ny + FJB - 1) / FJB, nzc * fl.n);
            { lsb::note_launch(); k_filter3<<<grid, 256, 0, h->stream>>>(fl, d.nx, d.ny, d.nzp, a, b, zf, zf + d.nzp, zf + 2 * d.nzp, nzc); }
        }
    }
}

void filter3(lsb_handle* h, const double* const* in, double* const* out, int n, double a, double b, int which) {
    filter3_any(h, reinterpret_cast<const void* const*>(in), reinterpret_cast<void* const*>(out), n, a, b, which, false);
}

// ---------------------------------------------------------------- dynamic Smagorinsky
struct DynArgs {
    const double* g[9];     // du_l/dx_m
    double* sij[6];
    double* sijhat[6];
    double* lij[6];
    double* mij[6];
    const double* uihat[3];
    double* lf[6];          // filtered u_i u_j
    double* numc;
    double* denomc;
    const double* ctot;
    const double* cdd;
    double* tau[9];
    const double* delta;    // [nzp]
    long long P;
    int nxy;
    int full9;              // 0: only the 6 components l <= m are written (tau is symmetric)
};

// The pointwise SGS kernels are templated on the working type T (double for the FP64 form,
// float for the mixed form); pointer fields of the argument blocks are reinterpreted as T.
template <class T> __device__ __forceinline__ const T* cp_(const double* p) { return reinterpret_cast<const T*>(p); }
template <class T> __device__ __forceinline__ T* wp_(double* p) { return reinterpret_cast<T*>(p); }


template <class T>
__global__ void k_dyn1(DynArgs a) {  // S_ij and L'_ij = delta^2 |S| S_ij
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.P; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((unsigned)e / (unsigned)a.nxy);  // P < 2^31 (checked at create)
        const T dl = (T)a.delta[k];
        T s6[6];
        for (int l = 0; l < 3; ++l)
            for (int m = l; m < 3; ++m) s6[sym6(l, m)] = dyn_sij<T>(cp_<T>(a.g[3 * l + m])[e], cp_<T>(a.g[3 * m + l])[e]);
        const T sn = snorm6<T>(s6);
        for (int q = 0; q < 6; ++q) {
            wp_<T>(a.sij[q])[e] = s6[q];
            wp_<T>(a.lij[q])[e] = dyn_lij<T>(dl, sn, s6[q]);
        }
    }
}

template <class T>
__global__ void k_dyn3(DynArgs a) {  // M_ij, L_ij, <M L>, <M M> integrands
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.P; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((unsigned)e / (unsigned)a.nxy);
        const T cd = (T)2 * (T)a.delta[k];
        T sh6[6];
        for (int q = 0; q < 6; ++q) sh6[q] = cp_<T>(a.sijhat[q])[e];
        const T sh = snorm6<T>(sh6);  // |[S]|
        const T f = mul_rn(mul_rn(cd, cd), sh);
        T m6[6], l6[6];
        // M_ij = 2 ([delta^2 |S| S_ij] - [delta]^2 |[S]| [S_ij])
        for (int q = 0; q < 6; ++q) m6[q] = (T)2 * (cp_<T>(a.mij[q])[e] - mul_rn(f, sh6[q]));
        for (int l = 0; l < 3; ++l)
            for (int m = l; m < 3; ++m)
                l6[sym6(l, m)] = cp_<T>(a.lf[sym6(l, m)])[e] - cp_<T>(a.uihat[l])[e] * cp_<T>(a.uihat[m])[e];
        T num = (T)0, den = (T)0;
        for (int m = 0; m < 3; ++m)
            for (int l = 0; l < 3; ++l) {
                const int q = sym6(l, m);
                num = num + m6[q] * l6[q];
                den = den + m6[q] * m6[q];
            }
        wp_<T>(a.numc)[e] = num;
        wp_<T>(a.denomc)[e] = den;
    }
}

template <class T>
__global__ void k_dyn4(DynArgs a) {  // C clip, nu_sgs, tau = -2 nu S_ij
    const T cmax = (T)(0.2 * 0.2);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.P; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((unsigned)e / (unsigned)a.nxy);  // P < 2^31 (checked at create)
        const T dl = (T)a.delta[k];
        T s6[6];
        for (int q = 0; q < 6; ++q) s6[q] = cp_<T>(a.sij[q])[e];
        T c = cp_<T>(a.ctot)[e] / cp_<T>(a.cdd)[e];
        if (c < (T)0 || isnan(c)) c = (T)0;
        if (c > cmax) c = cmax;
        const T nu = c * dl * dl * snorm6<T>(s6);
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m)
                if (a.full9 || m >= l) wp_<T>(a.tau[3 * l + m])[e] = (T)-2 * nu * s6[sym6(l, m)];
    }
}

// ---------------------------------------------------------------- static Smagorinsky
template <class T>
__global__ void k_utau(const double* __restrict__ dudz_, const int* __restrict__ wall, int nwall, long long C,
                       double xnu, int nxy, double* out) {
    const T* dudz = cp_<T>(dudz_);
    __shared__ double red[256];
    double acc = 0.0;
    for (long long c = threadIdx.x; c < C; c += blockDim.x) {
        double u = 0.0;
        for (int w = 0; w < nwall; ++w) u = u + xnu * (double)dudz[(long long)wall[w] * C + c];
        acc += u / nwall;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sqrt(fabs(red[0] / (double)nxy));
}

template <class T>
__global__ void k_static(P9 g, W9 tau, const double* __restrict__ sdelta,
                         const double* __restrict__ zpts, const double* __restrict__ utau, double cs, double xnu,
                         long long P, int nxy) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((unsigned)e / (unsigned)nxy);  // P < 2^31 (checked at create)
        T sn = (T)0;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const T v = (T)0.5 * (cp_<T>(g.p[3 * i + j])[e] + cp_<T>(g.p[3 * j + i])[e]);
                sn = sn + v * v;
            }
        sn = sqrt((T)2 * sn);
        const double zplus = zpts[k] * utau[0] / xnu;
        const T f = (T)(cs * sdelta[k] * (1. - exp(-zplus / 25.)));
        const T nu = -(f * f) * sn;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i)
                wp_<T>(tau.p[3 * i + j])[e] = nu * (T)0.5 * (cp_<T>(g.p[3 * i + j])[e] + cp_<T>(g.p[3 * j + i])[e]);
    }
}

// ---------------------------------------------------------------- sigma model
// The FP64 sigma model rounds every operation as the reference's expressions do, one at a
// time and left to right (no fused multiply-adds): its stresses are a near-cancellation
// of singular values, so a contraction moves them far more than the operation's ulp.
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double r_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
// x**3. (a real power, pow of the C library in the reference): x*x and x*x*x formed with
// their exact rounding errors (Dekker's two-product by fma), so the result is the exact
// cube rounded once, up to a few units in the last bit's last half
__device__ __forceinline__ double r_cube(double x) {
    const double p = x * x, e = fma(x, x, -p);
    const double q = p * x, f = fma(p, x, -q);
    return q + fma(e, x, f);
}
__device__ __forceinline__ float r_cube(float x) { return x * x * x; }

template <class T>
__global__ void k_sigma(P9 g, W9 tau, const double* __restrict__ delta, long long P, int nxy) {
    const T pi = (T)3.141592653589793;  // 4 atan(1)
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((unsigned)e / (unsigned)nxy);  // P < 2^31 (checked at create)
        T gij[3][3], G[3][3], G2[3][3];
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m) gij[l][m] = cp_<T>(g.p[3 * l + m])[e];
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m)  // (g^T g)(l,m), summed over q = 1, 2, 3 in order
                G[l][m] = r_add(r_add(r_mul(gij[0][l], gij[0][m]), r_mul(gij[1][l], gij[1][m])), r_mul(gij[2][l], gij[2][m]));
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m)
                G2[l][m] = r_add(r_add(r_mul(G[l][0], G[0][m]), r_mul(G[l][1], G[1][m])), r_mul(G[l][2], G[2][m]));
        const T i1 = r_add(r_add(G[0][0], G[1][1]), G[2][2]);
        const T i2 = r_mul((T)0.5, r_sub(r_mul(i1, i1), r_add(r_add(G2[0][0], G2[1][1]), G2[2][2])));
        const T i3 = r_add(r_sub(r_mul(G[0][0], r_sub(r_mul(G[1][1], G[2][2]), r_mul(G[1][2], G[2][1]))),
                                 r_mul(G[0][1], r_sub(r_mul(G[1][0], G[2][2]), r_mul(G[1][2], G[2][0])))),
                           r_mul(G[0][2], r_sub(r_mul(G[1][0], G[2][1]), r_mul(G[1][1], G[2][0]))));
        T a1 = r_sub(r_mul(i1, i1) / (T)9, i2 / (T)3);
        const T a2 = r_add(r_sub(r_cube(i1) / (T)27, r_mul(i1, i2) / (T)6), r_mul((T)0.5, i3));
        if (a1 < (T)0) a1 = fabs(a1);
        const T sq = sqrt(a1);
        const T pre = a2 / r_cube(sq);
        T a3;
        if (pre >= (T)1 || isnan(pre)) a3 = (T)0;
        else if (pre <= (T)-1) a3 = pi / (T)3;
        else a3 = acos(pre) / (T)3;
        const T sq2 = r_mul((T)2, sq);
        const T s1 = sqrt(fabs(r_add(i1 / (T)3, r_mul(sq2, cos(a3)))));
        const T s2 = sqrt(fabs(r_sub(i1 / (T)3, r_mul(sq2, cos(r_add(pi / (T)3, a3))))));
        const T s3 = sqrt(fabs(r_sub(i1 / (T)3, r_mul(sq2, cos(r_sub(pi / (T)3, a3))))));
        T ds = r_mul(r_mul(s3, r_sub(s1, s2)), r_sub(s2, s3));
        if (s1 != (T)0) ds = ds / r_mul(s1, s1);
        if (ds < (T)0 || isnan(ds)) ds = (T)0;
        const T cd = (T)(1.35 * delta[k]);
        const T nu = r_mul(-r_mul(cd, cd), ds);
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m)
                wp_<T>(tau.p[3 * l + m])[e] = r_mul(r_mul(r_mul((T)2, nu), (T)0.5), r_add(gij[l][m], gij[m][l]));
    }
}

// ---------------------------------------------------------------- interscale
template <class T>
__global__ void k_prod9(P9 a, P9 b, W9 out, long long P) {
    // out[3l+m] = a[l] * b[m]
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P; e += (long long)gridDim.x * blockDim.x)
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m) wp_<T>(out.p[3 * l + m])[e] = cp_<T>(a.p[l])[e] * cp_<T>(b.p[m])[e];
}

template <class T>
__global__ void k_interscale(P9 u, P9 ub, P9 ub2, P9 uibujbar, W9 tau, long long P) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P; e += (long long)gridDim.x * blockDim.x)
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m)
                wp_<T>(tau.p[3 * l + m])[e] = cp_<T>(uibujbar.p[3 * l + m])[e] - cp_<T>(ub2.p[l])[e] * cp_<T>(ub2.p[m])[e] -
                                              cp_<T>(ub.p[l])[e] * (cp_<T>(u.p[m])[e] - cp_<T>(ub.p[m])[e]);
}

template <class T>
__global__ void k_uiuj(P9 u, W9 out, long long P) {
    // out[sym(l,m)] = u_l u_m   (src/navierstokes.f90:744)
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < P; e += (long long)gridDim.x * blockDim.x)
        for (int l = 0; l < 3; ++l)
            for (int m = l; m < 3; ++m) wp_<T>(out.p[sym6(l, m)])[e] = cp_<T>(u.p[m])[e] * cp_<T>(u.p[l])[e];
}

__global__ void k_mul(double* y, const double* x, long long n) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = y[e] * x[e];
}

}  // namespace

void sgs_mul(double* y, const double* x, long long n, cudaStream_t s) { lsb::note_launch(); k_mul<<<nblk(n), 256, 0, s>>>(y, x, n); }

static void zfilter_coeffs(const std::vector<double>& zp, int mapping, double a, double b, double* az, double* bz,
                           double* cz) {
    const int n = (int)zp.size();
    for (int k = 0; k < n; ++k) az[k] = bz[k] = cz[k] = 0.0;
    if (mapping == 1 || mapping == 2) {
        for (int k = 1; k < n - 1; ++k) {
            const double dltm = zp[k] - zp[k - 1], dltp = zp[k + 1] - zp[k];
            az[k] = a * 2.0 * dltm / (dltp + dltm);
            bz[k] = a * 2.0 * (1. - dltm / dltp) + b;
            cz[k] = a * 2.0 * dltm * dltm / (dltp * (dltp + dltm));
        }
        if (mapping == 1) { az[1] = 0.0; bz[1] = 2.0 * a + b; cz[1] = 0.0; }
    } else {
        const int m = (n + 1) / 2;
        for (int k = 2; k <= m - 1; ++k) {
            const double dltm = zp[k - 1] - zp[k - 2], dltp = zp[k] - zp[k - 1];
            az[k - 1] = a * 2.0 * dltm / (dltp + dltm);
            bz[k - 1] = a * 2.0 * (1. - dltm / dltp) + b;
            cz[k - 1] = a * 2.0 * dltm * dltm / (dltp * (dltp + dltm));
        }
        for (int k = m + 1; k <= n - 1; ++k) {
            const double dltm = zp[k - 1] - zp[k - 2], dltp = zp[k] - zp[k - 1];
            az[k - 1] = a * 2.0 * dltp * dltp / (dltm * (dltm + dltp));
            bz[k - 1] = a * 2.0 * (1. - dltp / dltm) + b;
            cz[k - 1] = a * 2.0 * dltp / (dltm + dltp);
        }
        az[m - 1] = a; bz[m - 1] = b; cz[m - 1] = a;
    }
}

void filters_init(lsb_handle* h) {
    const Dims& d = h->d;
    const lsb_config& c = h->cfg;
    const double ab[4][2] = {{c.a, c.b}, {1.0, 1.0}, {1.0, 6.0}, {1.0, 2.0}};
    std::vector<double> zf(12 * (size_t)d.nzp);
    for (int w = 0; w < 4; ++w)
        zfilter_coeffs(h->h_zpts, c.mapping, ab[w][0], ab[w][1], &zf[(3 * w) * d.nzp], &zf[(3 * w + 1) * d.nzp],
                       &zf[(3 * w + 2) * d.nzp]);
    h->sgs.zf = h->upload(zf.data(), zf.size());
}

void sgs_init(lsb_handle* h) {
    const Dims& d = h->d;
    const lsb_config& c = h->cfg;
    SgsWork& s = h->sgs;
    s.nonsym = (c.sgsmodel == 3);
    s.tau = h->alloc(9 * h->P);
    if (s.nonsym) s.H9 = h->alloc(9 * d.S());
    s.nw = 40;
    s.w = h->alloc((size_t)s.nw * h->P);
    // delta of the dynamic and sigma models (src/sgsterm.f90:159-164, 367-376)
    const std::vector<double>& zp = h->h_zpts;
    const int n = d.nzp;
    std::vector<double> dl(n), sd(n, 0.0);
    for (int k = 0; k < n; ++k) {
        double dz;
        if (k == 0) dz = zp[0] - zp[1];
        else if (k == n - 1) dz = zp[n - 2] - zp[n - 1];
        else dz = 0.5 * (zp[k - 1] - zp[k + 1]);
        dl[k] = std::pow(h->dx * h->dy * dz, 1. / 3.);
    }
    // static Smagorinsky (src/sgsterm.f90:96-103): delta(1) overwritten, delta(nzp) unset
    for (int k = 1; k < n - 1; ++k) sd[k] = std::pow(h->dx * h->dy * ((zp[k - 1] - zp[k + 1]) / 2.), 1. / 3.);
    sd[0] = std::pow(h->dx * h->dy * std::fabs(zp[n - 1] - zp[n - 2]), 1. / 3.);
    sd[n - 1] = 0.0;
    s.delta = h->upload(dl.data(), n);
    s.sdelta = h->upload(sd.data(), n);
    s.scal = h->alloc(16);
    // wall planes for u_tau: zpts == 0 or |zpts| == 0.5 (src/sgsterm.f90:62-67)
    std::vector<int> wall;
    for (int k = 0; k < n; ++k)
        if (zp[k] == 0.0 || std::fabs(zp[k]) == 0.5) wall.push_back(k);
    if (c.sgsmodel == 0 && wall.empty()) sfail(LSB_ERR_UNSUPPORTED, "static Smagorinsky needs a wall plane");
    double* wbuf = h->alloc(8);
    std::vector<int> wi(16, 0);
    for (size_t i = 0; i < wall.size() && i < 16; ++i) wi[i] = wall[i];
    CK(cudaMemcpyAsync(wbuf, wi.data(), 16 * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    h->sgs_wall = (int*)wbuf;
    h->sgs_nwall = (int)wall.size();
}

// field i of an array of P-point fields of type T (T = float in the mixed form)
template <class T>
double* fld(double* base, long long i, long long P) {
    return reinterpret_cast<double*>(reinterpret_cast<T*>(base) + i * P);
}

// tau (9 components, index 3l+m) from physical u_l, g = du_l/dx_m (9), uiuj (9, index 3l+m or sym)
// full9: write all 9 stress components (the tier-1 tau_sgs); the step only reads l <= m
template <class T>
static void model_tau(lsb_handle* h, const double* const* u, const double* const* g, const double* const* uu6,
                      double* tau, bool full9 = true) {
    const Dims& d = h->d;
    const lsb_config& c = h->cfg;
    const long long P = h->P;
    const int nxy = d.nx * d.ny;
    const bool f32 = sizeof(T) == 4;
    SgsWork& s = h->sgs;
    cudaStream_t st = h->stream;
    double* w = s.w;
    auto W = [&](int i) { return fld<T>(w, i, P); };
    auto F3 = [&](const double* const* in, double* const* out, int n, double fa, double fb, int which) {
        filter3_any(h, reinterpret_cast<const void* const*>(in), reinterpret_cast<void* const*>(out), n, fa, fb,
                    which, f32);
    };
    double* Tq[9];
    for (int q = 0; q < 9; ++q) Tq[q] = fld<T>(tau, q, P);
    if (c.sgsmodel == 1) {
        DynArgs a{};
        for (int q = 0; q < 9; ++q) a.g[q] = g[q];
        for (int q = 0; q < 6; ++q) {
            a.sij[q] = W(q);
            a.sijhat[q] = W(6 + q);
            a.lij[q] = W(12 + q);
            a.mij[q] = W(18 + q);
            a.lf[q] = W(24 + q);
        }
        for (int l = 0; l < 3; ++l) a.uihat[l] = W(30 + l);
        a.numc = W(34);
        a.denomc = W(35);
        a.ctot = W(36);
        a.cdd = W(37);
        for (int q = 0; q < 9; ++q) a.tau[q] = Tq[q];
        a.delta = s.delta;
        a.P = P;
        a.nxy = nxy;
        a.full9 = full9 ? 1 : 0;
        if (!s.dyn1_fused) { lsb::note_launch(); k_dyn1<T><<<nblk(P), 256, 0, st>>>(a); }
        {  // one launch: [S_ij], [delta^2 |S| S_ij], [u_i], [u_i u_j]
            const double* fin[21];
            double* fout[21];
            for (int q = 0; q < 6; ++q) {
                fin[q] = a.sij[q];
                fout[q] = a.sijhat[q];
                fin[6 + q] = a.lij[q];
                fout[6 + q] = a.mij[q];
                fin[15 + q] = uu6[q];
                fout[15 + q] = a.lf[q];
            }
            for (int l = 0; l < 3; ++l) {
                fin[12 + l] = u[l];
                fout[12 + l] = W(30 + l);
            }
            F3(fin, fout, 21, c.a, c.b, 0);
        }
        { lsb::note_launch(); k_dyn3<T><<<nblk(P), 256, 0, st>>>(a); }
        const double* nd[2] = {a.numc, a.denomc};
        double* cc[2] = {W(36), W(37)};
        F3(nd, cc, 2, 1.0, 1.0, 1);
        if (!s.dyn4_fused) { lsb::note_launch(); k_dyn4<T><<<nblk(P), 256, 0, st>>>(a); }
    } else if (c.sgsmodel == 0) {
        P9 gt{};
        W9 tt{};
        for (int q = 0; q < 9; ++q) {
            gt.p[q] = g[q];
            tt.p[q] = Tq[q];
        }
        { lsb::note_launch(); k_utau<T><<<1, 256, 0, st>>>(g[2], h->sgs_wall, h->sgs_nwall, d.C(), c.xnu, nxy, s.scal); }
        { lsb::note_launch(); k_static<T><<<nblk(P), 256, 0, st>>>(gt, tt, s.sdelta, h->zpts, s.scal, c.cs, c.xnu, P, nxy); }
    } else if (c.sgsmodel == 2) {
        P9 gt{};
        W9 tt{};
        for (int q = 0; q < 9; ++q) {
            gt.p[q] = g[q];
            tt.p[q] = Tq[q];
        }
        { lsb::note_launch(); k_sigma<T><<<nblk(P), 256, 0, st>>>(gt, tt, s.delta, P, nxy); }
    } else if (c.sgsmodel == 3) {
        double* ub[3] = {W(0), W(1), W(2)};
        double* ub2[3] = {W(3), W(4), W(5)};
        double* pr[9];
        double* pb[9];
        for (int q = 0; q < 9; ++q) {
            pr[q] = W(6 + q);
            pb[q] = W(15 + q);
        }
        F3(u, ub, 3, c.a, c.b, 0);
        F3((const double* const*)ub, ub2, 3, c.a, c.b, 0);
        P9 ubt{}, ut{}, ub2t{}, pbt{};
        W9 prt{}, tt{};
        for (int l = 0; l < 3; ++l) {
            ubt.p[l] = ub[l];
            ut.p[l] = u[l];
            ub2t.p[l] = ub2[l];
        }
        for (int q = 0; q < 9; ++q) {
            prt.p[q] = pr[q];
            pbt.p[q] = pb[q];
            tt.p[q] = Tq[q];
        }
        { lsb::note_launch(); k_prod9<T><<<nblk(P), 256, 0, st>>>(ubt, ut, prt, P); }
        F3((const double* const*)pr, pb, 9, c.a, c.b, 0);
        { lsb::note_launch(); k_interscale<T><<<nblk(P), 256, 0, st>>>(ut, ubt, ub2t, pbt, tt, P); }
    } else {
        CK(cudaMemsetAsync(tau, 0, 9 * P * sizeof(T), st));
    }
}

// nlterm hook: ph[0..2] = u_l (+ubar), ph[3+3l+m] = du_l/dx_m (physical fields of the
// working type: FP32 in the mixed form); adds the forward transform of tau into the
// spectral h fields.
void sgs_add_tau(lsb_handle* h, double* const* ph, bool dealias, const double* const* xin, double* const* xout, int nx,
                 const double* xlam, const double* const* xmeans) {
    const Dims& d = h->d;
    const long long P = h->P, S = d.S();
    SgsWork& s = h->sgs;
    cudaStream_t st = h->stream;
    const bool f32 = h->cfg.precision == 1;
    auto PH = [&](long long i) { return f32 ? fld<float>(h->phys, i, P) : fld<double>(h->phys, i, P); };
    auto TAU = [&](long long i) { return f32 ? fld<float>(s.tau, i, P) : fld<double>(s.tau, i, P); };
    // u_i u_j on the unpadded grid: the dealiased products (2 * horfft(+1) of h) or plain products
    double* uu6[6];
    for (int q = 0; q < 6; ++q) uu6[q] = PH(12 + q);
    const double* u3[3] = {ph[0], ph[1], ph[2]};
    if (dealias) {
        const double* hs[6];
        for (int q = 0; q < 6; ++q) hs[q] = h->H + q * S;
        spec_to_phys(h, hs, uu6, 6, d.nzp, nullptr, nullptr, f32, 2.0);  // u_i u_j = 2 h_ij
    } else {
        P9 ut{};
        W9 ot{};
        for (int l = 0; l < 3; ++l) ut.p[l] = ph[l];
        for (int q = 0; q < 6; ++q) ot.p[q] = uu6[q];
        lsb::note_launch();
        if (f32) k_uiuj<float><<<nblk(P), 256, 0, st>>>(ut, ot, P);
        else k_uiuj<double><<<nblk(P), 256, 0, st>>>(ut, ot, P);
    }
    const double* g[9];
    for (int q = 0; q < 9; ++q) g[q] = ph[3 + q];
    // with the fused first pass (same row plan), the dynamic model's last pass goes into the
    // forward row pass of the stresses too
    s.dyn4_fused = s.dyn1_fused && h->cfg.sgsmodel == 1 && !s.nonsym;
    if (f32) model_tau<float>(h, u3, g, (const double* const*)uu6, s.tau, s.nonsym);
    else model_tau<double>(h, u3, g, (const double* const*)uu6, s.tau, s.nonsym);
    // add T(tau_lm) to h_lm (6 independent components, or all 9 when tau is not symmetric),
    // after the caller's extra fields, in one batch of forward transforms
    const double* tp[kMaxJobs];
    double* hp[kMaxJobs];
    int n = 0;
    for (int i = 0; i < nx; ++i) {
        tp[n] = xin[i];
        hp[n++] = xout[i];
    }
    if (!s.nonsym) {
        for (int l = 0; l < 3; ++l)
            for (int m = l; m < 3; ++m) {
                tp[n] = TAU(3 * l + m);
                hp[n++] = h->H + sym6(l, m) * S;
            }
    } else {
        for (int l = 0; l < 3; ++l)
            for (int m = 0; m < 3; ++m) {
                CK(cudaMemcpyAsync(s.H9 + (3 * l + m) * S, h->H + sym6(l, m) * S, S * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
                tp[n] = TAU(3 * l + m);
                hp[n++] = s.H9 + (3 * l + m) * S;
            }
    }
    TauRowArgs ta{};
    if (s.dyn4_fused) {
        // model_tau's work fields: S_ij, and the filtered contractions (W 36, 37)
        for (int q = 0; q < 6; ++q) ta.sij[q] = sgs_dyn_field(h, q);
        ta.ctot = f32 ? fld<float>(s.w, 36, P) : fld<double>(s.w, 36, P);
        ta.cdd = f32 ? fld<float>(s.w, 37, P) : fld<double>(s.w, 37, P);
        ta.delta = s.delta;
    }
    phys_to_spec(h, tp, hp, n, d.nzp, 1.0, 1.0, nullptr, f32, xlam, xmeans, nx, s.dyn4_fused ? &ta : nullptr);
    s.dyn4_fused = false;
}

double* sgs_dyn_field(lsb_handle* h, int i) {
    const int w = (i < 6) ? i : 12 + (i - 6);  // model_tau's sij (0..5) and lij (12..17)
    return h->cfg.precision == 1 ? fld<float>(h->sgs.w, w, h->P) : fld<double>(h->sgs.w, w, h->P);
}

void sgs_tau_phys(lsb_handle* h, const double* ui, const double* g, const double* uiuj, double* tau) {
    const long long P = h->P;
    const double* u3[3] = {ui, ui + P, ui + 2 * P};
    const double* g9[9];
    for (int q = 0; q < 9; ++q) g9[q] = g + q * P;
    const double* uu6[6];
    for (int l = 0; l < 3; ++l)
        for (int m = l; m < 3; ++m) uu6[sym6(l, m)] = uiuj + (3 * l + m) * P;
    h->sgs.dyn1_fused = h->sgs.dyn4_fused = false;  // the gradients and the stresses are the caller's fields
    model_tau<double>(h, u3, g9, uu6, tau);
}

// ---------------------------------------------------------------- filtering hook
namespace {
// per plane: sum over the 3 velocity fields and the plane of (q - qf)^2
__global__ void k_plane_sqdiff(P9 q, P9 qf, int nx, int ny, double* out) {
    const int k = blockIdx.x;
    const long long base = (long long)k * nx * ny;
    __shared__ double red[256];
    double acc = 0.0;
    for (int f = 0; f < 3; ++f)
        for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
            const double dd = q.p[f][base + e] - qf.p[f][base + e];
            acc += dd * dd;
        }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = red[0];
}

// modecutFC (src/filters.f90:617-654): qb = sum_l coef_l F^l(q), coef = (6,-15,20,-15,6,-1)
void modecut(lsb_handle* h, double* const* q, double* const* qb, double* const* ping, double* const* pong, int nf,
             double a, double b, int which) {
    const double coef[6] = {6., -15., 20., -15., 6., -1.};
    const long long P = h->P;
    const double* cur[4];
    for (int f = 0; f < nf; ++f) cur[f] = q[f];
    for (int l = 0; l < 6; ++l) {
        double* const* dst = (l % 2 == 0) ? ping : pong;
        filter3(h, cur, dst, nf, a, b, which);
        for (int f = 0; f < nf; ++f) {
            launch_axpby(qb[f], dst[f], coef[l], l == 0 ? 0.0 : 1.0, P, h->stream);
            cur[f] = dst[f];
        }
    }
}
}  // namespace

void filter_hook(lsb_handle* h) {
    const Dims& d = h->d;
    const lsb_config& c = h->cfg;
    const long long S = d.S(), P = h->P;
    TimerScope ts(h, "filter_hook");
    double* q[4];
    double* A[4];
    double* B[4];
    double* pi[4];
    double* po[4];
    for (int f = 0; f < 4; ++f) {
        q[f] = h->phys + f * P;
        A[f] = h->phys + (4 + f) * P;
        B[f] = h->phys + (8 + f) * P;
        pi[f] = h->phys + (12 + f) * P;
        po[f] = h->phys + (16 + f) * P;
    }
    const double* spec[4] = {h->vel, h->vel + S, h->vel + 2 * S, h->p};
    spec_to_phys(h, spec, q, 4, d.nzp, nullptr, nullptr);
    double* outs[4] = {h->vel, h->vel + S, h->vel + 2 * S, h->p};
    if (c.sgsflag == 1 && c.sgsmodel == 4) {
        // tns_automatic_filtering (src/filters.f90:62-161)
        modecut(h, q, A, pi, po, 4, 1.0, 6.0, 2);  // q_filt_2kc
        modecut(h, q, B, pi, po, 4, 1.0, 2.0, 3);  // q_filt
        P9 qq{}, qa{}, qb{};
        for (int f = 0; f < 3; ++f) {
            qq.p[f] = q[f];
            qa.p[f] = A[f];
            qb.p[f] = B[f];
        }
        double* e = h->red;
        { lsb::note_launch(); k_plane_sqdiff<<<d.nzp, 256, 0, h->stream>>>(qq, qb, d.nx, d.ny, e); }             // energy(:,3)
        { lsb::note_launch(); k_plane_sqdiff<<<d.nzp, 256, 0, h->stream>>>(qq, qa, d.nx, d.ny, e + d.nzp); }     // energy(:,4)
        std::vector<double> en(2 * (size_t)d.nzp);
        CK(cudaMemcpyAsync(en.data(), e, en.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const double nxy = (double)d.ny * d.nx;
        const std::vector<double>& zp = h->h_zpts;
        double ih = 0.0, idel = 0.0;
        for (int k = d.nz - 1; k >= 0; --k) {
            const double dz = zp[k] - zp[k + 1];
            ih += 0.5 * (en[d.nzp + k] / nxy + en[d.nzp + k + 1] / nxy) * dz;
            idel += 0.5 * (en[k] / nxy + en[k + 1] / nxy) * dz;
        }
        h->tns_ratio = ih / idel;
        if (ih / idel > 0.007) phys_to_spec(h, (const double* const*)A, outs, 4, d.nzp, 1.0, 0.0, nullptr);
    } else {
        // filterall3pt (src/filters.f90:9-59)
        modecut(h, q, A, pi, po, 4, c.a, c.b, 0);
        phys_to_spec(h, (const double* const*)A, outs, 4, d.nzp, 1.0, 0.0, nullptr);
    }
}

// ---------------------------------------------------------------- diagnostics
namespace {
struct PlaneStats {
    double e_tot, e_pert, umax, umin, vmax, vmin, wmax, wmin, uabs, vabs, wcfl, divabs, nonfinite;
};
constexpr int kStats = 13;

__global__ void k_plane_stats(const double* __restrict__ u, const double* __restrict__ v,
                              const double* __restrict__ w, const double* __restrict__ up,
                              const double* __restrict__ vp, const double* __restrict__ wp,
                              const double* __restrict__ div, const double* __restrict__ wscale, int findex, int nx,
                              int ny, double* out) {
    const int k = blockIdx.x;
    const long long base = (long long)k * nx * ny;
    __shared__ double red[kStats][256];
    double et = 0, ep = 0, umax = -INFINITY, umin = INFINITY, vmax = -INFINITY, vmin = INFINITY, wmax = -INFINITY,
           wmin = INFINITY, ua = 0, va = 0, wc = 0, da = 0, nf = 0;
    for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
        const double a = u[base + e], b = v[base + e], c = w[base + e];
        et += 0.5 * (a * a + b * b + c * c);
        const double pa = up[base + e], pb = vp[base + e], pc = wp[base + e];
        ep += 0.5 * (pa * pa + pb * pb + pc * pc);
        umax = fmax(umax, a); umin = fmin(umin, a);
        vmax = fmax(vmax, b); vmin = fmin(vmin, b);
        wmax = fmax(wmax, c); wmin = fmin(wmin, c);
        ua = fmax(ua, fabs(a)); va = fmax(va, fabs(b));
        const int i = e % nx;
        if (i < findex) wc = fmax(wc, fabs(c * wscale[k]));
        da += fabs(div[base + e]);
        if (!isfinite(a) || !isfinite(b) || !isfinite(c)) nf = 1;
    }
    const double vals[kStats] = {et, ep, umax, umin, vmax, vmin, wmax, wmin, ua, va, wc, da, nf};
    for (int q = 0; q < kStats; ++q) red[q][threadIdx.x] = vals[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            for (int q = 0; q < kStats; ++q) {
                const double x = red[q][threadIdx.x], y = red[q][threadIdx.x + s];
                double r;
                if (q == 0 || q == 1 || q == 11) r = x + y;
                else if (q == 3 || q == 5 || q == 7) r = fmin(x, y);
                else r = fmax(x, y);
                red[q][threadIdx.x] = r;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < kStats) out[(long long)k * kStats + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_zero_mean(double* f, long long S, long long C, int nzp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nzp) {
        f[(long long)k * C] = 0.0;
        f[(long long)k * C + 1] = 0.0;
    }
}
}  // namespace

void diag_compute(lsb_handle* h, lsb_diagnostics* out) {
    const Dims& d = h->d;
    const long long S = d.S(), C = d.C(), P = h->P;
    cudaStream_t st = h->stream;
    // physical u (+ubar), v, w; perturbation copies (mean mode removed); divergence
    double* io = h->io;
    CK(cudaMemcpyAsync(io, h->vel, 3 * S * sizeof(double), cudaMemcpyDeviceToDevice, st));
    for (int l = 0; l < 3; ++l) { lsb::note_launch(); k_zero_mean<<<(d.nzp + 127) / 128, 128, 0, st>>>(io + l * S, S, C, d.nzp); }
    // divergence = dfdx(u) + dfdy(v) + dfdz(w)
    double* dv = io + 3 * S;
    zgemm(h, h->m_dz1, h->vel + 2 * S, dv, 1, EPI_STORE, 1.0, 0.0, nullptr);
    launch_dxy(h->vel, io + 4 * S, h->wavx, h->wavy, d.nx, S, C, 0, st);
    launch_dxy(h->vel + S, io + 5 * S, h->wavx, h->wavy, d.nx, S, C, 1, st);
    launch_axpby(dv, io + 4 * S, 1.0, 1.0, S, st);
    launch_axpby(dv, io + 5 * S, 1.0, 1.0, S, st);
    double* ph[7];
    for (int i = 0; i < 7; ++i) ph[i] = h->phys + i * P;
    const double* sp[7] = {h->vel, h->vel + S, h->vel + 2 * S, io, io + S, io + 2 * S, dv};
    const double* means[7] = {h->ubar, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    spec_to_phys(h, sp, ph, 7, d.nzp, means, nullptr);
    // w CFL scale per plane (maxcalc, src/navierstokes.f90:430-437)
    const std::vector<double>& zp = h->h_zpts;
    const int nz = d.nz;
    std::vector<double> ws(d.nzp);
    for (int k = 0; k < nz; ++k) ws[k] = h->dt / (zp[k] - zp[k + 1]);
    ws[0] = ws[0] * h->dt / (zp[0] - zp[1]);
    ws[nz] = h->dt / (zp[nz - 1] - zp[nz]);
    double* wsd = h->red;
    CK(cudaMemcpyAsync(wsd, ws.data(), d.nzp * sizeof(double), cudaMemcpyHostToDevice, st));
    const double fsz = h->cfg.fsize;
    int findex = d.nx;
    if (h->t > h->cfg.istartbound) findex = (int)((1. - 0.8 * fsz) * d.nx);
    double* stats = h->T;
    { lsb::note_launch(); k_plane_stats<<<d.nzp, 256, 0, st>>>(ph[0], ph[1], ph[2], ph[3], ph[4], ph[5], ph[6], wsd, findex, d.nx, d.ny,
                                         stats); }
    std::vector<double> hs((size_t)d.nzp * kStats);
    CK(cudaMemcpyAsync(hs.data(), stats, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memset(out, 0, sizeof(*out));
    double umax = -INFINITY, umin = INFINITY, vmax = 0.0, vmin = 0.0, wmax = 0.0, wmin = 0.0, ua = 0, va = 0, wc = 0,
           da = 0, nf = 0;
    for (int k = 0; k < d.nzp; ++k) {
        const double* r = &hs[(size_t)k * kStats];
        umax = std::fmax(umax, r[2]); umin = std::fmin(umin, r[3]);
        vmax = std::fmax(vmax, r[4]); vmin = std::fmin(vmin, r[5]);
        wmax = std::fmax(wmax, r[6]); wmin = std::fmin(wmin, r[7]);
        ua = std::fmax(ua, r[8]); va = std::fmax(va, r[9]);
        wc = std::fmax(wc, r[10]);
        da += r[11];
        nf = std::fmax(nf, r[12]);
    }
    // the reference's maxima include the two pad columns: 0 + ubar(k) for u, 0 for v and w
    for (double ub : h->h_ubar) {
        umax = std::fmax(umax, ub);
        umin = std::fmin(umin, ub);
        ua = std::fmax(ua, std::fabs(ub));
    }
    // ener (src/orrsomm.f90:660-664): trapezoid from k = nz down to 2, ceiling plane excluded
    double et = 0.0, ep = 0.0;
    for (int k = nz - 1; k >= 1; --k) {
        et = et + 0.5 * (hs[(size_t)(k + 1) * kStats + 0] + hs[(size_t)k * kStats + 0]) * (zp[k] - zp[k + 1]);
        ep = ep + 0.5 * (hs[(size_t)(k + 1) * kStats + 1] + hs[(size_t)k * kStats + 1]) * (zp[k] - zp[k + 1]);
    }
    out->divergence = da / (double)(d.nx * d.ny * d.nzp);
    out->umax = umax; out->umin = umin; out->vmax = vmax; out->vmin = vmin; out->wmax = wmax; out->wmin = wmin;
    out->cflx = ua * h->dt / h->dx;
    out->cfly = va * h->dt / h->dy;
    out->cflz = wc;
    out->energy_total = et;
    out->energy_pert = ep;
    out->t = h->t;
    out->dt = h->dt;
    out->istep = h->istep;
    out->nonfinite = nf != 0.0 ? 1 : 0;
}

}  // namespace lsb
