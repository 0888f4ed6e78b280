// Warp-group register FFTs for the horizontal transforms (horfft, src/horfft.f90:61-150,
// and the padded passes of dealiasing_2d_fftw, src/dealiasing.f90:262-447).
//
// A line of N = G*R complex values is held by a group of G lanes (G a power of two <= 32),
// lane g holding the R elements n = g + G*r.  The transform is the four-step split
// N = R x G: an R-point DFT in registers, the twiddles exp(-+2 pi i g k1 / N), then a
// G-point decimation-in-frequency network across the group's lanes with shfl_xor.  Lane g
// ends with X[k1 + R*bitrev(g)] in register k1.  Shared memory is only used to turn the
// strided/bit-reversed orders into coalesced global accesses; there is no block barrier
// inside a transform.  Lengths whose R is not in {1,2,3,4,6,8} use fft_kernels.cu.
#include <stdexcept>

#include <cstring>

#include "lsb_fftdev.cuh"
#include "lsb_internal.cuh"
#include "lsb_sgs.cuh"
#include "lsb_tma.cuh"

namespace lsb {
namespace {

constexpr int WKC = 16;  // kx columns per spanwise work item

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

__device__ __forceinline__ int brev(int g, int lgg) {
    return lgg ? (int)(__brev((unsigned)g) >> (32 - lgg)) : 0;
}

// SEL = true: the butterflies as a per-lane select of both branches (fewer live registers,
// more arithmetic; the FP64 product rows use it to stay within their register budget)
template <int R, int SIGN, bool SEL = false, class V>
__device__ __forceinline__ void wfft(V (&v)[R], int G, int g, const V* __restrict__ tw) {
    dft_reg<R, SIGN>(v);
    if (R > 1 && g != 0) {
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            V w = __ldg(&tw[g * k1]);
            if (SIGN > 0) w.y = -w.y;
            v[k1] = cmul(v[k1], w);
        }
    }
    // butterfly of the pair (g, g ^ h): the lower lane keeps v + o, the upper (o - v) w.
    // Both are t = sg v + o times w', with sg = -1, w' = w on the upper lane and sg = 1,
    // w' = 1 on the lower one, so no lane evaluates the other's branch (exactly the same
    // roundings: fma(-1, v, o) = o - v and t * (1, 0) = t).
    using S = typename CT<V>::S;
    int st = R;  // N / (2h) for 2h = G
    for (int h = G >> 1; h >= 1; h >>= 1) {
        const int j = g & (h - 1);
        const bool up = (g & h) != 0;
        V w = __ldg(&tw[j * st]);
        if (SIGN > 0) w.y = -w.y;
        if (SEL) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                V o;
                o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
                o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
                v[k1] = up ? cmul(csub(o, v[k1]), w) : cadd(v[k1], o);
            }
            st <<= 1;
            continue;
        }
        if (!up) w = CT<V>::make((S)1, (S)0);
        const S sg = up ? (S)-1 : (S)1;
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) {
            V o;
            o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
            o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
            const V tt = CT<V>::make(fma(sg, v[k1].x, o.x), fma(sg, v[k1].y, o.y));
            v[k1] = cmul(tt, w);
        }
        st <<= 1;
    }
}

// Inverse of the order produced by wfft: input "slot" layout (lane g' register k1 holds
// z[k1 + R*bitrev(g')]), cross-lane decimation-in-time network, twiddles, R-point DFT in
// registers; output in natural order (lane g register r holds X[g + G*r]).
template <int R, int SIGN, bool SEL = false, class V>
__device__ __forceinline__ void wfft_dit(V (&v)[R], int G, int g, const V* __restrict__ tw) {
    // butterfly of the pair (g, g ^ h): the lower lane keeps v + w o, the upper o - w v.  The
    // upper lane multiplies its own value by w before the exchange (the lower lane's factor is
    // 1, exactly), so each lane then takes sg x + o_x with sg = 1 below and -1 above: the same
    // roundings as forming w o on the lower lane, and no lane evaluates the other's branch
    using S = typename CT<V>::S;
    int st = R * (G >> 1);  // N / (2h) for h = 1
    for (int h = 1; h < G; h <<= 1) {
        const int j = g & (h - 1);
        const bool up = (g & h) != 0;
        V w = __ldg(&tw[j * st]);
        if (SIGN > 0) w.y = -w.y;
        if (SEL) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                V o;
                o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
                o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
                v[k1] = up ? csub(o, cmul(w, v[k1])) : cadd(v[k1], cmul(w, o));
            }
            st >>= 1;
            continue;
        }
        if (!up) w = CT<V>::make((S)1, (S)0);
        const S sg = up ? (S)-1 : (S)1;
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) {
            const V x = cmul(w, v[k1]);
            V o;
            o.x = __shfl_xor_sync(0xffffffffu, x.x, h);
            o.y = __shfl_xor_sync(0xffffffffu, x.y, h);
            v[k1] = CT<V>::make(fma(sg, x.x, o.x), fma(sg, x.y, o.y));
        }
        st >>= 1;
    }
    if (R > 1 && g != 0) {
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            V w = __ldg(&tw[g * k1]);
            if (SIGN > 0) w.y = -w.y;
            v[k1] = cmul(v[k1], w);
        }
    }
    dft_reg<R, SIGN>(v);
}

// lane g of a group receives the registers of lane bitrev(g): after wfft, lane g then
// holds X[k1 + R*g] (R consecutive outputs)
template <int R, class V>
__device__ __forceinline__ void lane_bitrev(V (&v)[R], int G, int lane, int g, int lgg) {
    const int src = (lane & ~(G - 1)) | brev(g, lgg);
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
        v[k1].x = __shfl_sync(0xffffffffu, v[k1].x, src);
        v[k1].y = __shfl_sync(0xffffffffu, v[k1].y, src);
    }
}

// Exchange networks for lane groups of G = 16 or 32 lanes with an even register count
// R = 2H.  In the lane-pair networks above both lanes of a pair evaluate a butterfly branch
// for every register.  Here, at each stage, a lane sends half of its registers to its partner
// and receives the partner's matching half, so that it holds H whole butterflies: half the
// shuffles and half the butterfly arithmetic per stage.  Invariant before the stage on lane
// bit h: register i (i < H) of the lane with bit h clear and register H + i of its partner
// hold the two inputs of one butterfly, and the other way round; the upper lane's operand
// order is reversed, which the twiddle's sign absorbs ((r - k)(-w) = (k - r) w exactly).
// The outputs are stored in the order the next stage's invariant needs (swapped on lanes
// whose next bit is set), and lanes with bit G/2 set start with their halves rotated.
// DIF (wfft_x): dft_reg, twiddles, rotation, stages h = G/2 .. 1.  Lane g, register k then
// holds X[m], m = xslot<R, G>(g, k) = k%H + H*g_top + R*bitrev(g mod G/2) + (N/2)*(k/H)
// with N = R G and g_top the lane's bit G/2 -- the lane bit reversal of wfft is not needed.
// DIT (wfft_dit_x): the conjugate transpose of that network (stages h = 1 .. G/2, the
// butterfly s +- w d, the data routing inverted), from that layout to natural order.
template <int R, int G>
__device__ __forceinline__ int xslot(int g, int k) {
    constexpr int H = R / 2, LG = ilog2c(G);
    return (k % H) + H * ((g >> (LG - 1)) & 1) + R * brev(g & (G / 2 - 1), LG - 1) + (G / 2) * R * (k / H);
}

template <int R, class V>
__device__ __forceinline__ void rotate_halves(V (&v)[R], bool on) {
    constexpr int H = R / 2;
#pragma unroll
    for (int i = 0; i < H; ++i) {
        const V a = v[i], b = v[H + i];
        v[i] = on ? b : a;
        v[H + i] = on ? a : b;
    }
}

template <int R, int SIGN, int G, class V>
__device__ __forceinline__ void wfft_x(V (&v)[R], int g, const V* __restrict__ tw) {
    static_assert(R % 2 == 0 && (G == 16 || G == 32), "exchange network: even R, 16- or 32-lane groups");
    constexpr int H = R / 2;
    dft_reg<R, SIGN>(v);
    if (g != 0) {
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            V w = __ldg(&tw[g * k1]);
            if (SIGN > 0) w.y = -w.y;
            v[k1] = cmul(v[k1], w);
        }
    }
    rotate_halves<R>(v, (g & (G / 2)) != 0);
    int st = R;
#pragma unroll
    for (int h = G / 2; h >= 1; h >>= 1) {
        V w = __ldg(&tw[(g & (h - 1)) * st]);
        if (SIGN > 0) w.y = -w.y;
        if (g & h) w = CT<V>::make(-w.x, -w.y);
        const bool sw = (h > 1) && (g & (h >> 1)) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            V r;
            r.x = __shfl_xor_sync(0xffffffffu, v[H + i].x, h);
            r.y = __shfl_xor_sync(0xffffffffu, v[H + i].y, h);
            const V sm = cadd(v[i], r);
            const V df = cmul(csub(v[i], r), w);
            v[i] = sw ? df : sm;
            v[H + i] = sw ? sm : df;
        }
        st <<= 1;
    }
}

template <int R, int SIGN, int G, class V>
__device__ __forceinline__ void wfft_dit_x(V (&v)[R], int g, const V* __restrict__ tw) {
    static_assert(R % 2 == 0 && (G == 16 || G == 32), "exchange network: even R, 16- or 32-lane groups");
    constexpr int H = R / 2;
    int st = (G / 2) * R;
#pragma unroll
    for (int h = 1; h <= G / 2; h <<= 1) {
        V w = __ldg(&tw[(g & (h - 1)) * st]);
        if (SIGN > 0) w.y = -w.y;
        if (g & h) w = CT<V>::make(-w.x, -w.y);
        const bool sw = (h > 1) && (g & (h >> 1)) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const V sm = sw ? v[H + i] : v[i];
            const V df = sw ? v[i] : v[H + i];
            const V t = cmul(w, df);
            const V bk = csub(sm, t);
            v[i] = cadd(sm, t);
            v[H + i].x = __shfl_xor_sync(0xffffffffu, bk.x, h);
            v[H + i].y = __shfl_xor_sync(0xffffffffu, bk.y, h);
        }
        st >>= 1;
    }
    rotate_halves<R>(v, (g & (G / 2)) != 0);
    if (g != 0) {
#pragma unroll
        for (int k1 = 1; k1 < R; ++k1) {
            V w = __ldg(&tw[g * k1]);
            if (SIGN > 0) w.y = -w.y;
            v[k1] = cmul(v[k1], w);
        }
    }
    dft_reg<R, SIGN>(v);
}

// physical pair index of register k of lane g after a product-row c2r (the slot layout)
template <int R>
__device__ __forceinline__ int nl_pair(int g, int k) {
    if constexpr (R % 2 == 0) return xslot<R, 32>(g, k);
    else return k + R * brev(g, 5);
}

__device__ __forceinline__ void cpa16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ int pad_row_w(int j, int ny, int nyl, int layout) {
    if (layout == 0 || nyl == ny) return j;
    return (j < ny / 2) ? j : j + (nyl - ny);
}
// inverse of pad_row_w: padded row -> input row, or -1 for a zero-pad row
__device__ __forceinline__ int unpad_row(int n, int ny, int nyl, int layout) {
    if (layout == 0 || nyl == ny) return n < ny ? n : -1;
    if (n < ny / 2) return n;
    if (n >= nyl - (ny - ny / 2)) return n - (nyl - ny);
    return -1;
}

// FP64 spanwise tile [nyl][WKC] (16-byte elements, no padding): the column of a row is
// XOR-swizzled by a function of the row, chosen per R so that the 8 lanes of a quarter warp
// hit 8 distinct banks both when a lane group reads a column in natural row order
// (rows g + G r) and when it writes it back after the lane bit reversal (rows R g + k1);
// lane-contiguous row accesses only permute a row's columns.
template <int R>
__device__ __forceinline__ int yswz(int row) {
    if (R == 2 || R == 4) return row ^ (row >> 1) ^ (row >> 2);
    if (R == 6) return row ^ (row >> 1) ^ (row << 1);
    if (R == 8) return row ^ (row >> 1) ^ (row >> 3);
    return row;
}
template <int R>
__device__ __forceinline__ int ytix(int row, int col) { return row * WKC + (col ^ (yswz<R>(row) & 7)); }

// FP64 spanwise tile staged by TMA: the two 8-column halves of a row are 128-byte lines of
// two regions [nyl][8], each 1024-byte aligned, under the TMA's 128-byte swizzle (16-byte
// chunk c of line r at c ^ (r & 7)): a lane group reading a column in natural row order hits
// 8 distinct banks per quarter warp
__device__ __forceinline__ int ytix_tma(int row, int col, int nyl) {
    return (col >> 3) * (nyl * 8) + row * 8 + ((col & 7) ^ (row & 7));
}

// tensor maps of a launch's input fields (one per job), passed as a grid constant
struct alignas(64) YTmaMaps {
    CUtensorMap m[kMaxJobs];
};

// ----------------------------------------------------------------------------- spanwise
// One kernel for both directions.  Work item = (job, z, chunk of WKC kx columns); the tile
// [nyl][WKC] is staged double-buffered -- by cp.async (TMA = false) or by TMA tile loads that
// complete on an mbarrier per buffer (TMA = true, 2 or 4 box loads issued by one thread) --,
// each column is transformed by a lane group, and the tile is written back in coalesced rows.
// (A three-buffer ring measured slower at 256 x 64 x 129: on the unpadded grid, where it keeps
// 4 blocks per SM, 5-8 us per pass -- the larger shared-memory carve-out leaves less L1 --,
// and on the padded grid it costs a block per SM.)
// GC: the lane-group width as a compile-time constant (0: the plan's, at run time), so that
// the transform's cross-lane stages unroll and their twiddle loads are issued up front;
// 64 registers (4 blocks per SM) fit the unrolled FP64 form without spills
template <int R, bool INV, int GC = 0, bool TMA = false>
__global__ void __launch_bounds__(256, 4) k_ywarp(YInvJobList ij, YFwdJobList fj, YPassArgs a, int nch,
                                                  const __grid_constant__ YTmaMaps tm) {
    extern __shared__ __align__(1024) unsigned char ysm_raw[];
    // the TMA's 128-byte swizzle wants 1024-byte aligned destinations
    double2* smem = reinterpret_cast<double2*>(
        ysm_raw + ((1024u - (unsigned)(__cvta_generic_to_shared(ysm_raw) & 1023u)) & 1023u));
    const int ny = a.ny, nyl = a.nyl, G = GC ? GC : a.plan.g, lgg = GC ? ilog2c(GC) : a.plan.lgg;
    auto Buf = [&](int b) { return smem + b * (nyl * WKC); };
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * nyl * WKC);  // [2] (TMA)
    int* sabort = reinterpret_cast<int*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int njobs = INV ? ij.n : fj.n;
    const int nitems = njobs * a.nzp * nch;
    const int lpw = 32 / G;              // lines per warp per pass
    const int q = lane / G, g = lane - q * G;
    auto IX = [&](int row, int col) { return TMA ? ytix_tma(row, col, nyl) : ytix<R>(row, col); };
    // TMA: the input rows of a tile land in tile rows [0, h0) and [nyl - (ny - h0), nyl) when
    // the padded tile splits the spectrum (the textbook 3/2 layout), else in rows [0, rows)
    const bool split = INV && a.layout != 0 && nyl != ny;
    const int h0 = split ? ny / 2 : (INV ? ny : nyl);
    const uint32_t tile_bytes = 2u * (uint32_t)(INV ? ny : nyl) * 128u;
    // per buffer b: bit b of phm is the mbarrier phase to wait for, bit b of infm marks a load
    // in flight (bits of a register: indexed arrays of these went to local memory)
    uint32_t phm = 0u, infm = 0u;
    if (TMA) {
        if (tid == 0) {
            tma::mbar_init(&bar[0], 1);
            tma::mbar_init(&bar[1], 1);
            tma::fence_init();
            *sabort = 0;
        }
        __syncthreads();
    }
    auto issue = [&](int item, int b) {
        double2* T = Buf(b);
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const int c0 = ch * WKC;
        if (TMA) {
            if (INV && nyl != ny) {  // the padded rows hold zeros (generic stores, rows the TMA does not write)
                const int r0 = split ? h0 : ny;
                for (int idx = tid; idx < (nyl - ny) * WKC; idx += 256) {
                    const int r = idx / WKC, cc = idx - r * WKC;
                    T[IX(r0 + r, cc)] = make_double2(0.0, 0.0);
                }
            }
            if (tid == 0) {
                // the block's earlier generic accesses of this buffer (ordered by the barrier
                // before this call) come before the TMA's writes
                tma::fence_proxy_async();
                tma::mbar_expect_tx(&bar[b], tile_bytes);
                const CUtensorMap* map = &tm.m[jb];
                for (int hf = 0; hf < 2; ++hf) {
                    double2* dst = T + hf * (nyl * 8);
                    tma::load_3d(dst, map, 2 * c0 + 16 * hf, 0, z, &bar[b]);
                    if (split) tma::load_3d(dst + (nyl - (ny - h0)) * 8, map, 2 * c0 + 16 * hf, h0, z, &bar[b]);
                }
            }
            infm |= 1u << b;
            return;
        }
        if (INV) {
            const double* in = ij.j[jb].in;
            for (int idx = tid; idx < ny * WKC; idx += 256) {
                const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                double2* d = &T[IX(pad_row_w(j, ny, nyl, a.layout), cc)];
                if (c < a.kxc) cpa16(d, in + ((long long)z * ny + j) * a.nx + 2 * c);
                else *d = make_double2(0.0, 0.0);
            }
            const int npad = nyl - ny;
            for (int idx = tid; idx < npad * WKC; idx += 256) {
                const int r = idx / WKC, cc = idx - r * WKC;
                const int jl = (a.layout == 0 || nyl == ny) ? ny + r : ny / 2 + r;
                T[IX(jl, cc)] = make_double2(0.0, 0.0);
            }
        } else {
            const double* in = fj.j[jb].in;
            for (int idx = tid; idx < nyl * WKC; idx += 256) {
                const int jl = idx / WKC, cc = idx - jl * WKC, c = c0 + cc;
                double2* d = &T[IX(jl, cc)];
                if (c < a.kxc) cpa16(d, in + ((long long)z * nyl + jl) * a.nx + 2 * c);
                else *d = make_double2(0.0, 0.0);
            }
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, 0);
    for (; item < nitems; item += gridDim.x) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const int c0 = ch * WKC;
        double2* T = Buf(cur);
        if (TMA) {
            if (tma::mbar_wait(&bar[cur], (phm >> cur) & 1u)) {
                phm ^= 1u << cur;
                infm &= ~(1u << cur);
            } else {
                *sabort = 1;  // the buffer stays in flight for the clean-up at the end
            }
        } else {
            cpa_wait_all();
        }
        __syncthreads();
        if (TMA && *sabort != 0) break;
        const int next = item + gridDim.x;
        if (next < nitems) issue(next, cur ^ 1);
        const int mode = INV ? ij.j[jb].mode : YM_COPY;
        for (int L0 = warp * lpw; L0 < WKC; L0 += 8 * lpw) {
            const int L = L0 + q;
            const bool act = L < WKC;
            const int Lc = act ? L : 0;
            double2 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = g + G * r;
                double2 x = T[IX(n, Lc)];
                if (INV && mode != YM_COPY) {
                    double k = 0.0;
                    if (mode == YM_IKY) {
                        const int j = unpad_row(n, ny, nyl, a.layout);
                        k = (j >= 0) ? a.wavy[j] : 0.0;
                    } else {
                        const int c = min(c0 + Lc, a.kxc - 1);
                        k = a.wavx[2 * c];
                    }
                    x = make_double2(-k * x.y, k * x.x);
                }
                v[r] = x;
            }
            if constexpr (GC == 16 && R % 2 == 0) {
                // exchange network: register k1 holds output xslot(g, k1)
                wfft_x<R, INV ? +1 : -1, 16>(v, g, a.plan.tw);
                if (act) {
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) T[IX(xslot<R, 16>(g, k1), L)] = v[k1];
                }
            } else {
                wfft<R, INV ? +1 : -1>(v, G, g, a.plan.tw);
                lane_bitrev<R>(v, G, lane, g, lgg);
                if (act) {
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) T[IX(R * g + k1, L)] = v[k1];
                }
            }
        }
        __syncthreads();
        if (INV) {
            double* out = ij.j[jb].out;
            for (int idx = tid; idx < nyl * WKC; idx += 256) {
                const int jl = idx / WKC, cc = idx - jl * WKC, c = c0 + cc;
                if (c >= a.kxc) continue;
                *reinterpret_cast<double2*>(out + ((long long)z * nyl + jl) * a.nx + 2 * c) = T[IX(jl, cc)];
            }
        } else {
            const YFwdJob job = fj.j[jb];
            if (job.beta == 0.0) {
                for (int idx = tid; idx < ny * WKC; idx += 256) {
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    if (c >= a.kxc) continue;
                    double2 v = T[IX(pad_row_w(j, ny, nyl, a.layout), cc)];
                    if (job.sym && c == 0) {
                        const int jm = (ny - j) % ny;
                        const double2 w = T[IX(pad_row_w(jm, ny, nyl, a.layout), cc)];
                        v = make_double2(0.5 * (v.x + w.x), 0.5 * (v.y - w.y));
                    }
                    v.x *= a.scale;
                    v.y *= a.scale;
                    *reinterpret_cast<double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c) =
                        make_double2(job.alpha * v.x, job.alpha * v.y);
                }
            } else
            // an accumulating job: groups of four elements per thread, the destination values
            // loaded together before the group's stores
            for (int i0 = tid; i0 < ny * WKC; i0 += 4 * 256) {
                double2 old[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int idx = i0 + e * 256;
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    old[e] = make_double2(0.0, 0.0);
                    if (job.beta != 0.0 && idx < ny * WKC && c < a.kxc)
                        old[e] = *reinterpret_cast<const double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c);
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int idx = i0 + e * 256;
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    if (idx >= ny * WKC || c >= a.kxc) continue;
                    double2 v = T[IX(pad_row_w(j, ny, nyl, a.layout), cc)];
                    if (job.sym && c == 0) {
                        const int jm = (ny - j) % ny;
                        const double2 w = T[IX(pad_row_w(jm, ny, nyl, a.layout), cc)];
                        v = make_double2(0.5 * (v.x + w.x), 0.5 * (v.y - w.y));
                    }
                    v.x *= a.scale;
                    v.y *= a.scale;
                    double2* o = reinterpret_cast<double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c);
                    double2 rr;
                    if (job.beta != 0.0) {
                        rr = make_double2(fma(job.alpha, v.x, job.beta * old[e].x), fma(job.alpha, v.y, job.beta * old[e].y));
                    } else {
                        rr = make_double2(job.alpha * v.x, job.alpha * v.y);
                    }
                    *o = rr;
                }
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    if (TMA) {
        // after a time-out: the loads this block still has in flight end before it exits (a
        // bounded wait again), and the launch's error word is raised
        if (*sabort != 0) {
            for (int b = 0; b < 2; ++b)
                if ((infm >> b) & 1u) tma::mbar_wait(&bar[b], (phm >> b) & 1u);
            if (tid == 0 && a.err) atomicExch(a.err, 1);
        }
    } else {
        cpa_wait_all();
    }
}

// ----------------------------------------------------------------------------- rows
// c2r of the modes in X (N+1 entries; zero beyond kxc, DC imaginary part dropped) into
// registers: lane g returns z[k1 + R*bitrev(g)] in v[k1] (z = x[2m] + i x[2m+1]).
// row-buffer index under an XOR swizzle within blocks of 8 elements for FP64 rows (16-byte
// elements): lane-contiguous and stride-4 accesses (the staging of a bit-reversed row,
// R = 4) both avoid bank conflicts; indices N .. N + 7 stay in their block, so a row needs
// N + 8 slots.  FP32 rows keep the plain layout (measured faster there).
template <class V>
__device__ __forceinline__ int xsw(int n) { return sizeof(V) == 16 ? (n ^ ((n >> 3) & 7)) : n; }

template <int R, bool XN, class V>
__device__ __forceinline__ void row_c2r_regs(const V* X, int N, int G, int g, const V* __restrict__ twr,
                                             const V* __restrict__ tw, V (&v)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int n = g + G * r;
        const V xa = X[xsw<V>(n)];
        const V xb = cconj(X[xsw<V>(N - n)]);
        const V e = cadd(xa, xb);
        const V o = cmul(csub(xa, xb), cconj(__ldg(&twr[n])));
        v[r] = CT<V>::make(e.x - o.y, e.y + o.x);
    }
    if constexpr (XN) wfft_x<R, +1, 32>(v, g, tw);
    else wfft<R, +1>(v, G, g, tw);
}

template <class V>
__device__ __forceinline__ V r2c_mode_w(const V* Z, int k, int N, const V* __restrict__ twr) {
    using S = typename CT<V>::S;
    const V za = Z[k];
    const V zb = cconj(Z[k == 0 ? 0 : N - k]);
    const V e = CT<V>::make((S)0.5 * (za.x + zb.x), (S)0.5 * (za.y + zb.y));
    const V o = CT<V>::make((S)0.5 * (za.x - zb.x), (S)0.5 * (za.y - zb.y));
    const V t = cmul(__ldg(&twr[k]), o);
    return CT<V>::make(e.x + t.y, e.y - t.x);
}

// Generic row transforms: each lane group of each warp owns one row at a time.
template <int R, class V, int GC = 0>
__global__ void __launch_bounds__(256) k_row_c2r_w(RowJobList jobs, RowArgs a) {
    using S = typename CT<V>::S;
    extern __shared__ unsigned char rsm_raw[];
    V* smem = reinterpret_cast<V*>(rsm_raw);
    const V* twr = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.twrf) : reinterpret_cast<const V*>(a.rp.twr);
    const V* tw = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.half.twf) : reinterpret_cast<const V*>(a.rp.half.tw);
    const int N = a.nxl / 2, G = GC ? GC : a.rp.half.g, lgg = GC ? ilog2c(GC) : a.rp.half.lgg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpw = 32 / G, q = lane / G, g = lane - q * G;
    V* X = smem + (warp * lpw + q) * (N + 8);
    const int nrows = a.nyl * a.nzp;
    const int nunits = jobs.n * nrows;
    const int gw = blockIdx.x * 8 + warp, TW = gridDim.x * 8;
    const V zero = CT<V>::make((S)0, (S)0);
    // the next row's modes are loaded while the current row is transformed
    auto load_unit = [&](int u0_, V (&ld_)[R + 1]) {
        const int uu = u0_ + q;
        const int ucc = uu < nunits ? uu : u0_;
        const int jbb = ucc / nrows, roww = ucc - jbb * nrows;
        const S* yr = reinterpret_cast<const S*>(jobs.j[jbb].yin) + (long long)roww * 2 * a.kxc;
#pragma unroll
        for (int it = 0; it <= R; ++it) {
            const int k = g + G * it;
            ld_[it] = (k < a.kxc) ? *reinterpret_cast<const V*>(yr + 2 * k) : zero;
        }
    };
    V nx_ld[R + 1];
    if (gw * lpw < nunits) load_unit(gw * lpw, nx_ld);
    for (int u0 = gw * lpw; u0 < nunits; u0 += TW * lpw) {
        const int u = u0 + q;
        const bool act = u < nunits;
        const int uc = act ? u : u0;
        const int jb = uc / nrows, row = uc - jb * nrows;
        const RowIO job = jobs.j[jb];
        V ld[R + 1];
#pragma unroll
        for (int it = 0; it <= R; ++it) ld[it] = nx_ld[it];
        if (u0 + TW * lpw < nunits) load_unit(u0 + TW * lpw, nx_ld);
#pragma unroll
        for (int it = 0; it <= R; ++it) {
            const int k = g + G * it;
            if (k > N) break;
            V v = ld[it];
            if (job.mode == YM_IKX && k < a.kxc) {
                const S kk = (S)a.wavx[2 * k];
                v = CT<V>::make(-kk * v.y, kk * v.x);
            }
            if (k == 0) v.y = (S)0;
            X[xsw<V>(k)] = v;
        }
        __syncwarp();
        V v[R];
        constexpr bool XN = (GC == 32 && R % 2 == 0);  // exchange network
        row_c2r_regs<R, XN>(X, N, G, g, twr, tw, v);
        S m = (S)0;
        if (job.mean != nullptr && job.add_mean != 0.0) m = (S)(job.mean[row / a.nyl] * job.add_mean);
        const S sc = (S)job.scale;
        if constexpr (!XN) lane_bitrev<R>(v, G, lane, g, lgg);
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) {
            int n = R * g + k1;
            if constexpr (XN) n = xslot<R, 32>(g, k1);
            X[xsw<V>(n)] = CT<V>::make(sc * v[k1].x + m, sc * v[k1].y + m);
        }
        __syncwarp();
        if (act) {
            V* o = reinterpret_cast<V*>(reinterpret_cast<S*>(job.out) + (long long)row * a.row_pitch);
            for (int k = g; k < N; k += G) o[k] = X[xsw<V>(k)];
        }
        __syncwarp();
    }
}

// The dynamic model's physical fields with its first pointwise pass (k_dyn1 in
// sgs_kernels.cu) fused in, for full-warp row plans with even R: one warp per (z, y) row runs
// 12 c2r -- u_l, then the gradients in the order g_11, g_22, g_33, (g_12, g_21), (g_13, g_31),
// (g_23, g_32), so that each off-diagonal S_lm is formed as soon as its pair is in registers
// -- keeps S_ij in per-warp shared-memory slots of the exchange network's layout, and writes
// u_l, S_ij and delta^2 |S| S_ij (the same expressions in the same order as k_dyn1, so the
// same values bit for bit).  The nine gradient rows never go to HBM.
template <int R>
__host__ __device__ constexpr int dyn_row_slots() { return 32 * R + 8 + 6 * R * 32; }

template <int R, class V>
__global__ void __launch_bounds__(128) k_row_c2r_dyn(DynRowArgs a) {
    using S = typename CT<V>::S;
    const RowArgs& r = a.r;
    extern __shared__ unsigned char dsm_raw[];
    const V* twr = sizeof(S) == 4 ? reinterpret_cast<const V*>(r.rp.twrf) : reinterpret_cast<const V*>(r.rp.twr);
    const V* tw = sizeof(S) == 4 ? reinterpret_cast<const V*>(r.rp.half.twf) : reinterpret_cast<const V*>(r.rp.half.tw);
    constexpr int N = 32 * R;
    const int g = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V* X = reinterpret_cast<V*>(dsm_raw) + warp * dyn_row_slots<R>();
    V* Ss = X + N + 8;  // [6][R][32]
    auto SL = [&](int q, int k1) -> V& { return Ss[(q * R + k1) * 32 + g]; };
    const int nrows = r.nyl * r.nzp;
    const int W = gridDim.x * 4;
    const V zero = CT<V>::make((S)0, (S)0);
    // the 12 input rows of a row in transform order (the order of the c2r calls below):
    // u_l (3), du_1/dx, du_2/dy, du_3/dz, (du_1/dy, du_2/dx), (du_1/dz, du_3/dx), (du_2/dz, du_3/dy)
    auto src_of = [&](int rw, int i) -> const S* {
        if (rw >= nrows) return nullptr;
        const double* p;
        switch (i) {
            case 0: case 3: p = a.yu[0]; break;
            case 1: case 7: p = a.yu[1]; break;
            case 2: case 9: p = a.yu[2]; break;
            case 4: p = a.ydy[1]; break;
            case 5: p = a.ydz[2]; break;
            case 6: p = a.ydy[0]; break;
            case 8: p = a.ydz[0]; break;
            case 10: p = a.ydz[1]; break;
            default: p = a.ydy[2]; break;
        }
        return reinterpret_cast<const S*>(p) + (long long)rw * 2 * r.kxc;
    };
    // the next input row's modes, loaded while the current row is transformed
    V nx_ld[R + 1];
    auto load_row = [&](const S* yr) {
#pragma unroll
        for (int it = 0; it <= R; ++it) {
            const int k = g + 32 * it;
            nx_ld[it] = (yr != nullptr && k < r.kxc) ? *reinterpret_cast<const V*>(yr + 2 * k) : zero;
        }
    };
    load_row(src_of(blockIdx.x * 4 + warp, 0));
    for (int row = blockIdx.x * 4 + warp; row < nrows; row += W) {
        const int z = row / r.nyl;
        // c2r of input i (staged from the prefetched modes) into the slot layout, as
        // k_row_c2r_w; the next input's loads are issued before the transform
        auto c2r = [&](int i, V (&v)[R]) {
            const bool ikx = (i == 3 || i == 7 || i == 9);
            __syncwarp();  // the row buffer is free
#pragma unroll
            for (int it = 0; it <= R; ++it) {
                const int k = g + 32 * it;
                if (k > N) break;
                V x = nx_ld[it];
                if (ikx && k < r.kxc) {
                    const S kk = (S)r.wavx[2 * k];
                    x = CT<V>::make(-kk * x.y, kk * x.x);
                }
                if (k == 0) x.y = (S)0;
                X[xsw<V>(k)] = x;
            }
            load_row(i < 11 ? src_of(row, i + 1) : src_of(row + W, 0));
            __syncwarp();
            row_c2r_regs<R, true>(X, N, 32, g, twr, tw, v);
        };
        // a physical row from the slot layout, written in coalesced order through the buffer
        auto store = [&](double* out, const V (&v)[R]) {
            __syncwarp();
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) X[xsw<V>(xslot<R, 32>(g, k1))] = v[k1];
            __syncwarp();
            V* o = reinterpret_cast<V*>(reinterpret_cast<S*>(out) + (long long)row * r.row_pitch);
#pragma unroll
            for (int k = g; k < N; k += 32) o[k] = X[xsw<V>(k)];
        };
        V v[R], w[R];
        // u_l (u_1 + ubar)
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            c2r(l, v);
            if (l == 0 && a.uprime != nullptr) store(a.uprime, v);
            const S m = (l == 0) ? (S)(a.ubar[z] * 1.0) : (S)0;
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = CT<V>::make(v[k1].x + m, v[k1].y + m);
            store(a.u[l], v);
        }
        // diagonal S_ll from g_ll (du_1/dx, du_2/dy, du_3/dz)
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            c2r(3 + l, v);
            const int q = sym6(l, l);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1)
                SL(q, k1) = CT<V>::make(dyn_sij<S>(v[k1].x, v[k1].x), dyn_sij<S>(v[k1].y, v[k1].y));
        }
        // off-diagonal S_lm from (g_lm, g_ml): (du_1/dy, du_2/dx), (du_1/dz + ubarp, du_3/dx),
        // (du_2/dz, du_3/dy)
#pragma unroll 1
        for (int p = 0; p < 3; ++p) {
            const int l = (p < 2) ? 0 : 1, m = (p == 0) ? 1 : 2;
            c2r(6 + 2 * p, v);
            if (p == 1) {
                const S mz = (S)(a.ubarp[z] * 1.0);
#pragma unroll
                for (int k1 = 0; k1 < R; ++k1) v[k1] = CT<V>::make(v[k1].x + mz, v[k1].y + mz);
            }
            c2r(7 + 2 * p, w);
            const int q = sym6(l, m);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1)
                SL(q, k1) = CT<V>::make(dyn_sij<S>(v[k1].x, w[k1].x), dyn_sij<S>(v[k1].y, w[k1].y));
        }
        // |S| per point, then S_ij and delta^2 |S| S_ij
        const S dl = (S)a.delta[z];
        V sn[R];
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) {
            S sx[6], sy[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                sx[q] = SL(q, k1).x;
                sy[q] = SL(q, k1).y;
            }
            sn[k1] = CT<V>::make(snorm6<S>(sx), snorm6<S>(sy));
        }
#pragma unroll 1
        for (int q = 0; q < 6; ++q) {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = SL(q, k1);
            store(a.sij[q], v);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1)
                v[k1] = CT<V>::make(dyn_lij<S>(dl, sn[k1].x, v[k1].x), dyn_lij<S>(dl, sn[k1].y, v[k1].y));
            store(a.lij[q], v);
        }
    }
}

template <int R, class V, int GC = 0>
__global__ void __launch_bounds__(256) k_row_r2c_w(RowJobList jobs, RowArgs a) {
    using S = typename CT<V>::S;
    extern __shared__ unsigned char rsm_raw[];
    V* smem = reinterpret_cast<V*>(rsm_raw);
    const V* twr = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.twrf) : reinterpret_cast<const V*>(a.rp.twr);
    const V* tw = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.half.twf) : reinterpret_cast<const V*>(a.rp.half.tw);
    const int N = a.nxl / 2, G = GC ? GC : a.rp.half.g, lgg = GC ? ilog2c(GC) : a.rp.half.lgg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpw = 32 / G, q = lane / G, g = lane - q * G;
    V* Z = smem + (warp * lpw + q) * (N + 1);
    const int nrows = a.nyl * a.nzp;
    const int nunits = jobs.n * nrows;
    const int gw = blockIdx.x * 8 + warp, TW = gridDim.x * 8;
    // the next row is loaded while the current one is transformed
    auto load_unit = [&](int u0_, V (&v_)[R]) {
        const int uu = u0_ + q;
        const int ucc = uu < nunits ? uu : u0_;
        const int jbb = ucc / nrows, roww = ucc - jbb * nrows;
        const V* in = reinterpret_cast<const V*>(reinterpret_cast<const S*>(jobs.j[jbb].yin) + (long long)roww * a.row_pitch);
#pragma unroll
        for (int r = 0; r < R; ++r) v_[r] = in[g + G * r];
    };
    V nx_v[R];
    if (gw * lpw < nunits) load_unit(gw * lpw, nx_v);
    for (int u0 = gw * lpw; u0 < nunits; u0 += TW * lpw) {
        const int u = u0 + q;
        const bool act = u < nunits;
        const int uc = act ? u : u0;
        const int jb = uc / nrows, row = uc - jb * nrows;
        const RowIO job = jobs.j[jb];
        V v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = nx_v[r];
        if (u0 + TW * lpw < nunits) load_unit(u0 + TW * lpw, nx_v);
        if (job.lam != nullptr) {  // fringe forcing lambda(x) (m - q) on the fly
            const S m = (job.mean != nullptr && job.add_mean != 0.0) ? (S)(job.mean[row / a.nyl] * job.add_mean) : (S)0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int x = 2 * (g + G * r);
                const S l0 = (S)job.lam[x], l1 = (S)job.lam[x + 1];
                v[r] = CT<V>::make(l0 * (m - v[r].x), l1 * (m - v[r].y));
            }
        }
        wfft<R, -1>(v, G, g, tw);
        lane_bitrev<R>(v, G, lane, g, lgg);
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1) Z[R * g + k1] = v[k1];
        __syncwarp();
        if (act) {
            S* yrow = reinterpret_cast<S*>(job.out) + (long long)row * 2 * a.kxc;
            for (int k = g; k < a.kxc; k += G)
                *reinterpret_cast<V*>(yrow + 2 * k) = r2c_mode_w(Z, k, N, twr);
        }
        __syncwarp();
    }
}

// r2c row pass for full-warp plans (G = 32, N = 32 R): one warp per row, the physical row
// staged in shared memory under an XOR swizzle, so that both its natural-order writes
// (lane-contiguous) and its slot-order reads (stride R, lanes bit-reversed) are free of
// bank conflicts; the decimation-in-time network then ends in natural order, where the
// (k, N - k) pairs of the real-to-complex split are one shuffle apart: no lane bit
// reversal, no second staging.  (The same scheme for c2r measured slower than
// k_row_c2r_w: its register footprint cost a block per SM.)
__device__ __forceinline__ int rsw(int n) { return n ^ ((n >> 4) & 7); }  // stays in n's block of 8
// the row buffer's swizzle per register count: conflict-free for the natural-order writes
// and for the gather in the exchange network's slot order at R = 2, 4, 8 (2-way at R = 6);
// for odd R the slot order of the lane-pair network (k1 + R bitrev(g))
template <int R>
__device__ __forceinline__ int rsw_x(int n) {
    if constexpr (R % 2 == 1 || R == 8) return rsw(n);
    else return n ^ ((n >> 3) & 7);
}

template <int R, class V>
__global__ void __launch_bounds__(256) k_row_r2c_s(RowJobList jobs, RowArgs a) {
    using S = typename CT<V>::S;
    constexpr int N = 32 * R, LS = N + 8;
    extern __shared__ unsigned char rsm_raw[];
    const V* twr = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.twrf) : reinterpret_cast<const V*>(a.rp.twr);
    const V* tw = sizeof(S) == 4 ? reinterpret_cast<const V*>(a.rp.half.twf) : reinterpret_cast<const V*>(a.rp.half.tw);
    const int g = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V* Z = reinterpret_cast<V*>(rsm_raw) + warp * LS;
    const int K = a.kxc, mb = R * brev(g, 5);
    const int nrows = a.nyl * a.nzp;
    const int nunits = jobs.n * nrows;
    const int gw = blockIdx.x * 8 + warp, TW = gridDim.x * 8;
    const int src = (32 - g) & 31;
    const S h = (S)0.5;
    auto load_unit = [&](int u, V (&v_)[R]) {
        const int jbb = u / nrows, roww = u - jbb * nrows;
        const V* in = reinterpret_cast<const V*>(reinterpret_cast<const S*>(jobs.j[jbb].yin) + (long long)roww * a.row_pitch);
#pragma unroll
        for (int r = 0; r < R; ++r) v_[r] = in[g + 32 * r];
    };
    V nx_v[R];
    if (gw < nunits) load_unit(gw, nx_v);
    (void)N;
    for (int u = gw; u < nunits; u += TW) {
        const int jb = u / nrows, row = u - jb * nrows;
        const RowIO job = jobs.j[jb];
        V v[R];
        if (job.lam != nullptr) {  // fringe forcing lambda(x) (m - q) on the fly
            const S m = (job.mean != nullptr && job.add_mean != 0.0) ? (S)(job.mean[row / a.nyl] * job.add_mean) : (S)0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int x = 2 * (g + 32 * r);
                const S l0 = (S)job.lam[x], l1 = (S)job.lam[x + 1];
                nx_v[r] = CT<V>::make(l0 * (m - nx_v[r].x), l1 * (m - nx_v[r].y));
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) Z[rsw_x<R>(g + 32 * r)] = nx_v[r];
        if (u + TW < nunits) load_unit(u + TW, nx_v);
        __syncwarp();
        if constexpr (R % 2 == 0) {
            // the exchange network's input layout: register k1 holds z[xslot(g, k1)]
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = Z[rsw_x<R>(xslot<R, 32>(g, k1))];
        } else {
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = Z[rsw_x<R>(k1 + mb)];
        }
        __syncwarp();  // the row buffer is free for the next row
        if constexpr (R % 2 == 0) wfft_dit_x<R, -1, 32>(v, g, tw);
        else wfft_dit<R, -1>(v, 32, g, tw);
        // natural order: lane g register rr holds Z[g + 32 rr]; Z[N-k] for k = g + 32 rr is
        // lane (32-g) register R-1-rr (g > 0), or lane 0 register R-rr (g = 0, rr > 0)
        V* yrow = reinterpret_cast<V*>(reinterpret_cast<S*>(job.out) + (long long)row * 2 * K);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
            V zb;
            zb.x = __shfl_sync(0xffffffffu, v[R - 1 - rr].x, src);
            zb.y = __shfl_sync(0xffffffffu, v[R - 1 - rr].y, src);
            if (g == 0) zb = v[rr == 0 ? 0 : R - rr];
            const int k = g + 32 * rr;
            if (k < K) {
                const V za = v[rr];
                zb = cconj(zb);
                const V e = CT<V>::make(h * (za.x + zb.x), h * (za.y + zb.y));
                const V o = CT<V>::make(h * (za.x - zb.x), h * (za.y - zb.y));
                const V tt = cmul(__ldg(&twr[k]), o);
                yrow[k] = CT<V>::make(e.x + tt.y, e.y - tt.x);
            }
        }
    }
}

// The dynamic model's last pointwise pass (k_dyn4 in sgs_kernels.cu) fused into the forward
// row pass of its stresses, for full-warp row plans with even R: one warp per (z, y) row
// reads S_ij and the filtered contractions in natural order, forms nu = C delta^2 |S| per
// point (C = <L M> / <M M> clipped to [0, 0.2^2], NaN to 0) and, per component, tau_ij =
// -2 nu S_ij -- the same expressions in the same order as k_dyn4 -- which it stages, gathers
// in the exchange network's slot order and transforms as k_row_r2c_s does.  The six stress
// fields never go to HBM.
template <int R, class V>
__global__ void __launch_bounds__(128, 5) k_row_r2c_tau(TauRowArgs a) {
    using S = typename CT<V>::S;
    const RowArgs& r = a.r;
    constexpr int N = 32 * R, LS = N + 8;
    extern __shared__ unsigned char rsm_raw[];
    const V* twr = sizeof(S) == 4 ? reinterpret_cast<const V*>(r.rp.twrf) : reinterpret_cast<const V*>(r.rp.twr);
    const V* tw = sizeof(S) == 4 ? reinterpret_cast<const V*>(r.rp.half.twf) : reinterpret_cast<const V*>(r.rp.half.tw);
    const int g = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V* Z = reinterpret_cast<V*>(rsm_raw) + warp * LS;
    const int K = r.kxc;
    const int nrows = r.nyl * r.nzp;
    const int gw = blockIdx.x * 4 + warp, TW = gridDim.x * 4;  // 4 warps per block
    const int src = (32 - g) & 31;
    const S h = (S)0.5;
    const S cmax = (S)(0.2 * 0.2);
    for (int row = gw; row < nrows; row += TW) {
        const int z = row / r.nyl;
        const S dl = (S)a.delta[z];
        const long long ro = (long long)row * r.row_pitch;
        auto at = [&](const double* f) { return reinterpret_cast<const V*>(reinterpret_cast<const S*>(f) + ro); };
        // nu at the pair g + 32 rr of this lane
        V nu[R];
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
            const int m = g + 32 * rr;
            S sx[6], sy[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const V sv = at(a.sij[q])[m];
                sx[q] = sv.x;
                sy[q] = sv.y;
            }
            const V ct = at(a.ctot)[m], cd = at(a.cdd)[m];
            S cx = ct.x / cd.x, cy = ct.y / cd.y;
            if (cx < (S)0 || isnan(cx)) cx = (S)0;
            if (cx > cmax) cx = cmax;
            if (cy < (S)0 || isnan(cy)) cy = (S)0;
            if (cy > cmax) cy = cmax;
            nu[rr] = CT<V>::make(cx * dl * dl * snorm6<S>(sx), cy * dl * dl * snorm6<S>(sy));
        }
#pragma unroll 1
        for (int q = 0; q < 6; ++q) {
            V v[R];
            __syncwarp();  // the row buffer is free
#pragma unroll
            for (int rr = 0; rr < R; ++rr) {
                const V sv = at(a.sij[q])[g + 32 * rr];
                Z[rsw_x<R>(g + 32 * rr)] = CT<V>::make((S)-2 * nu[rr].x * sv.x, (S)-2 * nu[rr].y * sv.y);
            }
            __syncwarp();
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = Z[rsw_x<R>(xslot<R, 32>(g, k1))];
            wfft_dit_x<R, -1, 32>(v, g, tw);
            V* yrow = reinterpret_cast<V*>(reinterpret_cast<S*>(a.out[q]) + (long long)row * 2 * K);
#pragma unroll
            for (int rr = 0; rr < R; ++rr) {
                V zb;
                zb.x = __shfl_sync(0xffffffffu, v[R - 1 - rr].x, src);
                zb.y = __shfl_sync(0xffffffffu, v[R - 1 - rr].y, src);
                if (g == 0) zb = v[rr == 0 ? 0 : R - rr];
                const int k = g + 32 * rr;
                if (k < K) {
                    const V za = v[rr];
                    zb = cconj(zb);
                    const V e = CT<V>::make(h * (za.x + zb.x), h * (za.y + zb.y));
                    const V o = CT<V>::make(h * (za.x - zb.x), h * (za.y - zb.y));
                    const V tt = cmul(__ldg(&twr[k]), o);
                    yrow[k] = CT<V>::make(e.x + tt.y, e.y - tt.x);
                }
            }
        }
    }
}

// The fused nonlinear-product row: 12 c2r (u_l, du_l/dx, du_l/dy, du_l/dz), the skew-
// symmetric products and fringe of nlterm_skewsym (src/navierstokes.f90:725-769), 9 r2c.
// A block owns one (z, y) row at a time; the 9 input rows of the next row are staged with
// cp.async while the current one is transformed.
template <int R>
__global__ void __launch_bounds__(256, 2) k_row_nl_w(NlRowArgs a) {
    extern __shared__ double2 smem[];
    const RowArgs& r = a.r;
    const int N = r.nxl / 2, G = r.rp.half.g, lgg = r.rp.half.lgg, K = r.kxc;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lpw = 32 / G, q = lane / G, g = lane - q * G;
    double2* Stg[2] = {smem, smem + 9 * K};   // staged rows: U0..2, DY0..2, DZ0..2
    double2* P = smem + 18 * K;               // 12 physical rows of N complex (2N reals)
    double2* W = P + 12 * N + (warp * lpw + q) * (N + 1);
    const int nitems = r.nyl * r.nzp;
    auto issue = [&](int row, double2* S) {
        for (int idx = tid; idx < 9 * K; idx += 256) {
            const int f = idx / K, k = idx - f * K;
            const int l = f % 3, kind = f / 3;
            const double* src = (kind == 0) ? a.U[l] : (kind == 1 ? a.DY[l] : a.DZ[l]);
            cpa16(&S[idx], src + (long long)row * 2 * K + 2 * k);
        }
        cpa_commit();
    };
    int cur = 0;
    int row = blockIdx.x;
    if (row < nitems) issue(row, Stg[0]);
    for (; row < nitems; row += gridDim.x) {
        const int z = row / r.nyl;
        const double2* S = Stg[cur];
        cpa_wait_all();
        __syncthreads();
        const int next = row + gridDim.x;
        if (next < nitems) issue(next, Stg[cur ^ 1]);
        // 12 c2r: field f = 3*kind + l with kind 0 u, 1 du/dx (= i kx u), 2 du/dy, 3 du/dz
        for (int f0 = warp * lpw; f0 < 12; f0 += 8 * lpw) {
            const int f = f0 + q;
            const bool act = f < 12;
            const int fc = act ? f : f0;
            const int l = fc % 3, kind = fc / 3;
            const double2* Xs = S + (kind <= 1 ? l : 3 * (kind - 1) + l) * K;
            double2 v[R];
#pragma unroll
            for (int rr = 0; rr < R; ++rr) {
                const int n = g + G * rr;
                double2 xa = (n < K) ? Xs[n] : make_double2(0.0, 0.0);
                double2 xb = (N - n < K) ? Xs[N - n] : make_double2(0.0, 0.0);
                if (kind == 1) {
                    const double ka = (n < K) ? r.wavx[2 * n] : 0.0;
                    const double kb = (N - n < K) ? r.wavx[2 * (N - n)] : 0.0;
                    xa = make_double2(-ka * xa.y, ka * xa.x);
                    xb = make_double2(-kb * xb.y, kb * xb.x);
                }
                if (n == 0) xa.y = 0.0;  // FFTW c2r ignores Im of the DC input
                xb = cconj(xb);
                const double2 e = cadd(xa, xb);
                const double2 o = cmul(csub(xa, xb), cconj(__ldg(&r.rp.twr[n])));
                v[rr] = make_double2(e.x - o.y, e.y + o.x);
            }
            wfft<R, +1>(v, G, g, r.rp.half.tw);
            if (act) {
                // slot layout: slot k1*G + g holds z[k1 + R*bitrev(g)] (conflict-free)
#pragma unroll
                for (int k1 = 0; k1 < R; ++k1) P[fc * N + k1 * G + g] = v[k1];
            }
        }
        __syncthreads();
        const double* p = reinterpret_cast<const double*>(P);
        double* qo = reinterpret_cast<double*>(P);
        const int n = r.nxl, L2 = 2 * N;
        const double ub = a.ubar[z], ubp = a.ubarp[z];
        for (int xs = tid; xs < n; xs += 256) {
            // physical point of the slot value: complex slot s = xs/2 holds z[m], m = k1 + R*bitrev(g)
            const int sl = xs >> 1, k1s = sl / G, gs = sl - k1s * G;
            const int x = 2 * (k1s + R * brev(gs, lgg)) + (xs & 1);
            double u[3], gr[3][3];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                u[l] = p[(0 + l) * L2 + xs];
                gr[l][0] = p[(3 + l) * L2 + xs];
                gr[l][1] = p[(6 + l) * L2 + xs];
                gr[l][2] = p[(9 + l) * L2 + xs];
            }
            u[0] += ub;
            gr[0][2] += ubp;
            double nl[3];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                double acc = 0.0;
                acc = acc - 0.5 * (u[0] * gr[l][0]);
                acc = acc - 0.5 * (u[1] * gr[l][1]);
                acc = acc - 0.5 * (u[2] * gr[l][2]);
                nl[l] = acc;
            }
            if (a.lamx != nullptr) {
                const double lx = a.lamx[x];
                nl[0] = nl[0] + lx * (ub - u[0]);
                nl[1] = nl[1] + lx * (0.0 - u[1]);
                nl[2] = nl[2] + lx * (0.0 - u[2]);
            }
            qo[0 * L2 + xs] = nl[0];
            qo[1 * L2 + xs] = nl[1];
            qo[2 * L2 + xs] = nl[2];
            qo[3 * L2 + xs] = 0.5 * (u[0] * u[0]);
            qo[4 * L2 + xs] = 0.5 * (u[0] * u[1]);
            qo[5 * L2 + xs] = 0.5 * (u[0] * u[2]);
            qo[6 * L2 + xs] = 0.5 * (u[1] * u[1]);
            qo[7 * L2 + xs] = 0.5 * (u[1] * u[2]);
            qo[8 * L2 + xs] = 0.5 * (u[2] * u[2]);
        }
        __syncthreads();
        for (int f0 = warp * lpw; f0 < 9; f0 += 8 * lpw) {
            const int f = f0 + q;
            const bool act = f < 9;
            const int fc = act ? f : f0;
            double2 v[R];
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) v[k1] = P[fc * N + k1 * G + g];
            wfft_dit<R, -1>(v, G, g, r.rp.half.tw);
            // natural order: lane g register rr holds Z[g + G*rr]
#pragma unroll
            for (int rr = 0; rr < R; ++rr) W[g + G * rr] = v[rr];
            __syncwarp();
            if (act) {
                double* dst = (fc < 3) ? a.N[fc] : a.H[fc - 3];
                double* yrow = dst + (long long)row * 2 * K;
                for (int k = g; k < K; k += G)
                    *reinterpret_cast<double2*>(yrow + 2 * k) = r2c_mode_w(W, k, N, r.rp.twr);
            }
            __syncwarp();
        }
        __syncthreads();
        cur ^= 1;
    }
}

// Register-resident variant for rows of N = 32*R complex (G = 32): each warp owns a whole
// (z, y) row.  Its lanes read the 9 input rows straight from global memory (coalesced),
// and the 12 c2r, the products and the 9 r2c all stay in registers: every c2r leaves the
// same slot layout (lane g, register k1 -> physical pair m = k1 + R*bitrev(g)), so the
// products are lane-local, and the r2c (decimation in time from that layout) ends in
// natural order, where the pair Z[k], Z[N-k] of the real-to-complex split is one shuffle
// apart.  No shared memory and no block barrier.
#ifndef NLR_MINB
#define NLR_MINB 3
#endif
#ifndef NLR_SEL
#define NLR_SEL 1
#endif
template <int R, class S, class V, bool SEL = (sizeof(S) == 8 && NLR_SEL)>
__device__ __forceinline__ void nl_c2r_r(const S* __restrict__ src, bool ikx, int K, int N, int g,
                                         const double* __restrict__ wavx, const V* __restrict__ twr,
                                         const V* __restrict__ tw, V (&v)[R]) {
    const V zero = CT<V>::make((S)0, (S)0);
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
        const int n = g + 32 * rr;
        V xa = zero, xb = zero;
        if (n < K) xa = __ldg(reinterpret_cast<const V*>(src) + n);
        if (N - n < K) xb = __ldg(reinterpret_cast<const V*>(src) + (N - n));
        if (ikx) {
            const S ka = (n < K) ? (S)__ldg(&wavx[2 * n]) : (S)0;
            const S kb = (N - n < K) ? (S)__ldg(&wavx[2 * (N - n)]) : (S)0;
            xa = CT<V>::make(-ka * xa.y, ka * xa.x);
            xb = CT<V>::make(-kb * xb.y, kb * xb.x);
        }
        if (n == 0) xa.y = (S)0;  // FFTW c2r ignores Im of the DC input
        xb = cconj(xb);
        const V e = cadd(xa, xb);
        const V o = cmul(csub(xa, xb), cconj(__ldg(&twr[n])));
        v[rr] = CT<V>::make(e.x - o.y, e.y + o.x);
    }
    if constexpr (R % 2 == 0) wfft_x<R, +1, 32>(v, g, tw);
    else wfft<R, +1, SEL>(v, 32, g, tw);
}

// r2c of a slot-layout row; writes the K stored modes of the row at dst
template <int R, class S, class V, bool SEL = (sizeof(S) == 8 && NLR_SEL)>
__device__ __forceinline__ void nl_r2c_r(V (&v)[R], S* __restrict__ dst, int K, int g, const V* __restrict__ twr,
                                         const V* __restrict__ tw) {
    if constexpr (R % 2 == 0) wfft_dit_x<R, -1, 32>(v, g, tw);
    else wfft_dit<R, -1, SEL>(v, 32, g, tw);
    // natural order: lane g register rr holds Z[g + 32 rr]; Z[N-k] for k = g + 32 rr is
    // lane (32-g) register R-1-rr (g > 0), or lane 0 register R-rr (g = 0, rr > 0)
    const int src = (32 - g) & 31;
    const S h = (S)0.5;
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
        V zb;
        zb.x = __shfl_sync(0xffffffffu, v[R - 1 - rr].x, src);
        zb.y = __shfl_sync(0xffffffffu, v[R - 1 - rr].y, src);
        if (g == 0) zb = v[rr == 0 ? 0 : R - rr];
        const int k = g + 32 * rr;
        if (32 * rr < K && k < K) {
            const V za = v[rr];
            zb = cconj(zb);
            const V e = CT<V>::make(h * (za.x + zb.x), h * (za.y + zb.y));
            const V o = CT<V>::make(h * (za.x - zb.x), h * (za.y - zb.y));
            const V tt = cmul(__ldg(&twr[k]), o);
            reinterpret_cast<V*>(dst)[k] = CT<V>::make(e.x + tt.y, e.y - tt.x);
        }
    }
}

// shared memory of k_row_nl_r: per warp, the three velocity rows and the convective sum
template <int R>
constexpr size_t nl_r_smem() { return (size_t)4 * 4 * R * 32 * sizeof(double2); }

template <int R>
__global__ void __launch_bounds__(128, (R <= 6 ? NLR_MINB : 3)) k_row_nl_r(NlRowArgs a) {
    const RowArgs& r = a.r;
    const int N = 32 * R, K = r.kxc;
    const int g = threadIdx.x & 31;
    const int nitems = r.nyl * r.nzp;
    const int W = gridDim.x * (blockDim.x >> 5);
    // the physical velocity rows of this warp's row, lane-private slots [l][k1][lane]: kept
    // in shared memory rather than registers, so that more warps fit per SM
    extern __shared__ double2 nl_r_sm[];
    double2* us = nl_r_sm + (threadIdx.x >> 5) * (4 * R * 32);
    auto U = [&](int l, int k1) -> double2& { return us[(l * R + k1) * 32 + g]; };
    for (int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < nitems; row += W) {
        const int z = row / r.nyl;
        const long long off = (long long)row * 2 * K;
        const double ub = a.ubar[z], ubp = a.ubarp[z];
        // the row's 21 transforms as one loop, so that each direction's code is inlined once
        // (instruction fetch was a top stall with the transforms inlined per call site):
        // ops 0..2   c2r of u_l into the slots (u_1 + ubar)
        // ops 3..8   r2c of the fluxes 0.5 u_l u_m for (11, 12, 13, 22, 23, 33)
        // ops 9..20  per component l: c2r of du_l/dx, du_l/dy, du_l/dz, accumulating
        //            -0.5 u_m d_m u_l in slot 3, then the r2c of that sum (+ the fringe)
        // (the FP32 rows and the dynamic-model row pass measured slower in this form)
#pragma unroll 1
        for (int op = 0; op < 21; ++op) {
            const int cl = (op - 9) >> 2, ct = (op - 9) & 3;  // component and step of ops 9..20
            double2 v[R];
            if (op < 3 || (op >= 9 && ct < 3)) {
                const double* src = (op < 3) ? a.U[op] : (ct == 0 ? a.U[cl] : (ct == 1 ? a.DY[cl] : a.DZ[cl]));
                nl_c2r_r<R>(src + off, op >= 9 && ct == 0, K, N, g, r.wavx, r.rp.twr, r.rp.half.tw, v);
                if (op < 3) {
                    const double add = (op == 0) ? ub : 0.0;
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) U(op, k1) = make_double2(v[k1].x + add, v[k1].y + add);
                } else {
                    const double dzb = (ct == 2 && cl == 0) ? ubp : 0.0;
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) {
                        const double2 um = U(ct, k1);
                        const double2 c = (ct == 0) ? make_double2(0.0, 0.0) : U(3, k1);
                        U(3, k1) = make_double2(c.x - 0.5 * (um.x * (v[k1].x + dzb)),
                                                c.y - 0.5 * (um.y * (v[k1].y + dzb)));
                    }
                }
            } else {
                double* dst;
                if (op < 9) {
                    const int p = op - 3;
                    const int l = (p < 3) ? 0 : (p < 5 ? 1 : 2);
                    const int m = (p < 3) ? p : (p < 5 ? p - 2 : 2);
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) {
                        const double2 ul = U(l, k1), um = U(m, k1);
                        v[k1] = make_double2(0.5 * (ul.x * um.x), 0.5 * (ul.y * um.y));
                    }
                    dst = a.H[p];
                } else {
                    const double ut = (cl == 0) ? ub : 0.0;
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) {
                        double2 c = U(3, k1);
                        if (a.lamx != nullptr) {
                            const int x = 2 * nl_pair<R>(g, k1);  // physical x of the pair in register k1
                            const double lx0 = __ldg(&a.lamx[x]), lx1 = __ldg(&a.lamx[x + 1]);
                            const double2 ul = U(cl, k1);
                            c.x = c.x + lx0 * (ut - ul.x);
                            c.y = c.y + lx1 * (ut - ul.y);
                        }
                        v[k1] = c;
                    }
                    dst = a.N[cl];
                }
                nl_r2c_r<R>(v, dst + off, K, g, r.rp.twr, r.rp.half.tw);
            }
        }
    }
}

// ----------------------------------------------------------------------------- mixed form
// FP32 variants for the mixed-precision step: y-intermediates are FP32, the transforms run
// in FP32 with FP32 twiddles; the spectral fields on either side stay FP64 (converted on
// load and store).  Same work items and layouts as k_ywarp.
// column swizzle of the FP32 compact spanwise tile (16 columns of 8 bytes per row): conflict-free
// for the natural-order reads (rows g + 16 r) and the exchange network's slot-order writes
// (rows xslot(g, k)) of 16-lane groups, checked for every column and R = 2, 4, 6, 8
template <int R>
__device__ __forceinline__ int fsw(int row) {
    return R == 6 ? (row & 15) : ((row ^ (row >> 4)) & 15);
}

__device__ __forceinline__ void cpa8(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc));
}

// The tile is the FP64 pass's: [nyl][WKC] 16-byte slots under its row swizzle, double-buffered
// by cp.async -- the inverse stages its FP64 spectral input as it is (converted to FP32 when
// the transform reads it), the forward its FP32 input in the first half of each slot --, and
// the transform's FP32 results go to the first half of the slots.  (The single-buffered form
// that converted on load left each item's load latency exposed.)
template <int R, bool INV, int GC = 0>
__global__ void __launch_bounds__(256, 4) k_ywarp_f(YInvJobList ij, YFwdJobList fj, YPassArgs a, int nch) {
    extern __shared__ __align__(16) double2 fsm2[];
    const int ny = a.ny, nyl = a.nyl, G = GC ? GC : a.plan.g, lgg = GC ? ilog2c(GC) : a.plan.lgg;
    auto Buf = [&](int b) { return fsm2 + b * (nyl * WKC); };
    auto SL = [&](double2* T, int row, int col) { return reinterpret_cast<float2*>(T + ytix<R>(row, col)); };
    // the exchange-network form keeps its FP32 values in a compact tile of 128-byte rows (column
    // c of row r at r * WKC + (c ^ fsw<R>(r))): 16 lanes then reach 16 distinct 8-byte
    // positions of a line in the natural-order reads, the slot-order write-back and the row
    // stores (8-byte values in 16-byte slots reach half of a line's banks: 2-way conflicts)
    constexpr bool CMP = (GC == 16 && R % 2 == 0);
    auto OUT = [&](double2* T, int row, int col) {
        return CMP ? reinterpret_cast<float2*>(T) + row * WKC + (col ^ fsw<R>(row)) : SL(T, row, col);
    };
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int njobs = INV ? ij.n : fj.n;
    const int nitems = njobs * a.nzp * nch;
    const int lpw = 32 / G;
    const int q = lane / G, g = lane - q * G;
    auto issue = [&](int item, int b) {
        double2* T = Buf(b);
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const int c0 = ch * WKC;
        if (INV) {
            const double* in = ij.j[jb].in;
            for (int idx = tid; idx < nyl * WKC; idx += 256) {
                const int jl = idx / WKC, cc = idx - jl * WKC, c = c0 + cc;
                const int j = unpad_row(jl, ny, nyl, a.layout);
                double2* d = T + ytix<R>(jl, cc);
                if (j >= 0 && c < a.kxc) cpa16(d, in + ((long long)z * ny + j) * a.nx + 2 * c);
                else *d = make_double2(0.0, 0.0);
            }
        } else {
            const float* in = reinterpret_cast<const float*>(fj.j[jb].in);
            for (int idx = tid; idx < nyl * WKC; idx += 256) {
                const int jl = idx / WKC, cc = idx - jl * WKC, c = c0 + cc;
                float2* d = OUT(T, jl, cc);
                if (c < a.kxc) cpa8(d, in + ((long long)z * nyl + jl) * a.nx + 2 * c);
                else *d = make_float2(0.f, 0.f);
            }
        }
        cpa_commit();
    };
    int cur = 0;
    int item = blockIdx.x;
    if (item < nitems) issue(item, 0);
    for (; item < nitems; item += gridDim.x) {
        const int ch = item % nch, rest = item / nch, z = rest % a.nzp, jb = rest / a.nzp;
        const int c0 = ch * WKC;
        double2* T = Buf(cur);
        cpa_wait_all();
        __syncthreads();  // this item's tile has landed; every thread is done with the other buffer
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x, cur ^ 1);
        const int mode = INV ? ij.j[jb].mode : YM_COPY;
        for (int L0 = warp * lpw; L0 < WKC; L0 += 8 * lpw) {
            const int L = L0 + q;
            const bool act = L < WKC;
            const int Lc = act ? L : 0;
            float2 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = g + G * r;
                float2 x;
                if (INV) {
                    const double2 d = T[ytix<R>(n, Lc)];
                    x = make_float2((float)d.x, (float)d.y);
                } else {
                    x = *OUT(T, n, Lc);
                }
                if (INV && mode != YM_COPY) {
                    float k = 0.f;
                    if (mode == YM_IKY) {
                        const int j = unpad_row(n, ny, nyl, a.layout);
                        k = (j >= 0) ? (float)a.wavy[j] : 0.f;
                    } else {
                        const int c = min(c0 + Lc, a.kxc - 1);
                        k = (float)a.wavx[2 * c];
                    }
                    x = make_float2(-k * x.y, k * x.x);
                }
                v[r] = x;
            }
            if constexpr (GC == 16 && R % 2 == 0) {
                wfft_x<R, INV ? +1 : -1, 16>(v, g, a.plan.twf);
                // the inverse's compact results overlay FP64 input slots of other columns: every
                // warp has read its columns first (this loop runs once per warp at 16-lane groups)
                if (INV) __syncthreads();
                else __syncwarp();
                if (act) {
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) *OUT(T, xslot<R, 16>(g, k1), L) = v[k1];
                }
            } else {
                wfft<R, INV ? +1 : -1>(v, G, g, a.plan.twf);
                lane_bitrev<R>(v, G, lane, g, lgg);
                __syncwarp();
                if (act) {
#pragma unroll
                    for (int k1 = 0; k1 < R; ++k1) *SL(T, R * g + k1, L) = v[k1];
                }
            }
        }
        __syncthreads();
        if (INV) {
            float* out = reinterpret_cast<float*>(ij.j[jb].out);
            for (int idx = tid; idx < nyl * WKC; idx += 256) {
                const int jl = idx / WKC, cc = idx - jl * WKC, c = c0 + cc;
                if (c >= a.kxc) continue;
                *reinterpret_cast<float2*>(out + ((long long)z * nyl + jl) * a.nx + 2 * c) = *OUT(T, jl, cc);
            }
        } else {
            const YFwdJob job = fj.j[jb];
            if (job.beta == 0.0) {
                for (int idx = tid; idx < ny * WKC; idx += 256) {
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    if (c >= a.kxc) continue;
                    const float2 vf = *OUT(T, pad_row_w(j, ny, nyl, a.layout), cc);
                    double2 v = make_double2((double)vf.x, (double)vf.y);
                    if (job.sym && c == 0) {
                        const int jm = (ny - j) % ny;
                        const float2 wf = *OUT(T, pad_row_w(jm, ny, nyl, a.layout), cc);
                        v = make_double2(0.5 * (v.x + (double)wf.x), 0.5 * (v.y - (double)wf.y));
                    }
                    v.x *= a.scale;
                    v.y *= a.scale;
                    *reinterpret_cast<double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c) =
                        make_double2(job.alpha * v.x, job.alpha * v.y);
                }
            } else
            // as in k_ywarp: an accumulating job's destination values are loaded four at a time
            for (int i0 = tid; i0 < ny * WKC; i0 += 4 * 256) {
                double2 old[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int idx = i0 + e * 256;
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    old[e] = make_double2(0.0, 0.0);
                    if (job.beta != 0.0 && idx < ny * WKC && c < a.kxc)
                        old[e] = *reinterpret_cast<const double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c);
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int idx = i0 + e * 256;
                    const int j = idx / WKC, cc = idx - j * WKC, c = c0 + cc;
                    if (idx >= ny * WKC || c >= a.kxc) continue;
                    const float2 vf = *OUT(T, pad_row_w(j, ny, nyl, a.layout), cc);
                    double2 v = make_double2((double)vf.x, (double)vf.y);
                    if (job.sym && c == 0) {
                        const int jm = (ny - j) % ny;
                        const float2 wf = *OUT(T, pad_row_w(jm, ny, nyl, a.layout), cc);
                        v = make_double2(0.5 * (v.x + (double)wf.x), 0.5 * (v.y - (double)wf.y));
                    }
                    v.x *= a.scale;
                    v.y *= a.scale;
                    double2* o = reinterpret_cast<double2*>(job.out + ((long long)z * ny + j) * a.nx + 2 * c);
                    double2 rr;
                    if (job.beta != 0.0) {
                        rr = make_double2(fma(job.alpha, v.x, job.beta * old[e].x), fma(job.alpha, v.y, job.beta * old[e].y));
                    } else {
                        rr = make_double2(job.alpha * v.x, job.alpha * v.y);
                    }
                    *o = rr;
                }
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    cpa_wait_all();
}

// k_row_nl_r in FP32: FP32 rows in and out, same slot layout.  The streamwise velocity is
// kept as the perturbation u' and the mean ubar(z) is added inside each product, so that
// FP32 rounding of ubar + u' (|ubar| ~ 1 >> |u'|) never enters the perturbation terms:
//   h_11 = u'(ubar + u'/2)   (0.5 ubar^2 dropped: a kx = 0 function of z that only ever
//                              enters the step through d/dx, where it vanishes)
//   h_1m = (ubar + u') u_m / 2,  fringe lambda (ubar - u) = -lambda u'.
#ifndef NLF_MINB
#define NLF_MINB 6
#endif
// shared memory of k_row_nl_f: per warp, u', v, w and the convective sum (FP32)
template <int R>
constexpr size_t nl_f_smem() { return (size_t)4 * 4 * R * 32 * sizeof(float2); }

template <int R>
__global__ void __launch_bounds__(128, NLF_MINB) k_row_nl_f(NlRowArgs a) {
    const RowArgs& r = a.r;
    const int N = 32 * R, K = r.kxc;
    const int g = threadIdx.x & 31;
    const int nitems = r.nyl * r.nzp;
    const int W = gridDim.x * (blockDim.x >> 5);
    auto F = [](const double* p) { return reinterpret_cast<const float*>(p); };
    // lane-private slots [l][k1][lane] of u', v, w (l = 0..2) and the convective sum (l = 3)
    extern __shared__ float2 nl_f_sm[];
    float2* us = nl_f_sm + (threadIdx.x >> 5) * (4 * R * 32);
    auto U = [&](int l, int k1) -> float2& { return us[(l * R + k1) * 32 + g]; };
    for (int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < nitems; row += W) {
        const int z = row / r.nyl;
        const long long off = (long long)row * 2 * K;
        const float ub = (float)a.ubar[z], ubp = (float)a.ubarp[z];
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            float2 t[R];
            nl_c2r_r<R>(F(a.U[l]) + off, false, K, N, g, r.wavx, r.rp.twrf, r.rp.half.twf, t);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) U(l, k1) = t[k1];
        }
#pragma unroll 1
        for (int p = 0; p < 6; ++p) {
            float2 f[R];
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const float2 up = U(0, k1);
                if (p == 0) {
                    f[k1] = make_float2(up.x * (ub + 0.5f * up.x), up.y * (ub + 0.5f * up.y));
                } else if (p < 3) {
                    const float2 um = U(p, k1);
                    f[k1] = make_float2(0.5f * ((ub + up.x) * um.x), 0.5f * ((ub + up.y) * um.y));
                } else {
                    const int l = (p < 5) ? 1 : 2;
                    const int m = (p < 5) ? p - 2 : 2;
                    const float2 ul = U(l, k1), um = U(m, k1);
                    f[k1] = make_float2(0.5f * (ul.x * um.x), 0.5f * (ul.y * um.y));
                }
            }
            nl_r2c_r<R>(f, reinterpret_cast<float*>(a.H[p]) + off, K, g, r.rp.twrf, r.rp.half.twf);
        }
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            float2 d[R];
            // the three c2r of a component share one loop body (as in k_row_nl_r)
#pragma unroll 1
            for (int t = 0; t < 3; ++t) {
                const double* src = (t == 0) ? a.U[l] : (t == 1 ? a.DY[l] : a.DZ[l]);
                nl_c2r_r<R>(F(src) + off, t == 0, K, N, g, r.wavx, r.rp.twrf, r.rp.half.twf, d);
                const float dzb = (t == 2 && l == 0) ? ubp : 0.f;
                const float um0 = (t == 0) ? ub : 0.f;  // u' carries the mean ubar only in u_1
#pragma unroll
                for (int k1 = 0; k1 < R; ++k1) {
                    const float2 um = U(t, k1);
                    const float2 c = (t == 0) ? make_float2(0.f, 0.f) : U(3, k1);
                    U(3, k1) = make_float2(c.x - 0.5f * ((um0 + um.x) * (d[k1].x + dzb)),
                                           c.y - 0.5f * ((um0 + um.y) * (d[k1].y + dzb)));
                }
            }
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                float2 c = U(3, k1);
                if (a.lamx != nullptr) {
                    const int x = 2 * nl_pair<R>(g, k1);  // physical x of the pair in register k1
                    const float lx0 = (float)__ldg(&a.lamx[x]), lx1 = (float)__ldg(&a.lamx[x + 1]);
                    const float2 ul = U(l, k1);
                    c.x = c.x - lx0 * ul.x;
                    c.y = c.y - lx1 * ul.y;
                }
                d[k1] = c;
            }
            nl_r2c_r<R>(d, reinterpret_cast<float*>(a.N[l]) + off, K, g, r.rp.twrf, r.rp.half.twf);
        }
    }
}

template <class K>
int persistent_grid_w(K kern, size_t smem, long long nitems) {
    const long long gsz = (long long)resident_blocks((const void*)kern, 256, smem) * sm_count();
    return (int)(gsz < nitems ? gsz : (nitems > 0 ? nitems : 1));
}

template <int R, bool INV>
void ylaunch(const YInvJobList& ij, const YFwdJobList& fj, const YPassArgs& a, cudaStream_t s) {
    const int nch = (a.kxc + WKC - 1) / WKC;
    const int nitems = (INV ? ij.n : fj.n) * a.nzp * nch;
    if (a.f32) {
        const size_t smf = (size_t)2 * a.nyl * WKC * sizeof(double2);
        lsb::note_launch();
        if (a.plan.g == 16) k_ywarp_f<R, INV, 16><<<persistent_grid_w(k_ywarp_f<R, INV, 16>, smf, nitems), 256, smf, s>>>(ij, fj, a, nch);
        else k_ywarp_f<R, INV><<<persistent_grid_w(k_ywarp_f<R, INV>, smf, nitems), 256, smf, s>>>(ij, fj, a, nch);
        return;
    }
    YTmaMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    // TMA staging (the handle's schedule): one tensor map per job's input field; a grid or
    // field the maps do not fit (tile rows not a multiple of 8, a box over 256 rows, the
    // driver call missing) takes the cp.async staging
    const int njobs = INV ? ij.n : fj.n;
    const bool split = INV && a.layout != 0 && a.nyl != a.ny;
    // every box lands on a 1024-byte boundary (the swizzle's atom): tile rows, and the row at
    // which the split's second box starts, multiples of 8
    bool use_tma = a.y_tma == 1 && a.nyl % 8 == 0 && a.nyl <= 256 && a.ny % 2 == 0 &&
                   (!split || (a.nyl - a.ny / 2) % 8 == 0);
    for (int jb = 0; use_tma && jb < njobs; ++jb) {
        const double* in = INV ? ij.j[jb].in : fj.j[jb].in;
        const uint64_t rows = INV ? (uint64_t)a.ny : (uint64_t)a.nyl;
        const uint32_t box_rows = split ? (uint32_t)(a.ny / 2) : (uint32_t)rows;
        use_tma = tmap_f64_3d(&tm.m[jb], in, (uint64_t)a.nx, rows, (uint64_t)a.nzp, 16, box_rows);
    }
    // the two buffers (TMA: 1024-byte alignment slack and the barriers)
    const size_t sm = use_tma ? (size_t)2 * a.nyl * WKC * sizeof(double2) + 64 + 1024
                              : (size_t)2 * a.nyl * (WKC + 1) * sizeof(double2);
    lsb::note_launch();
    auto go = [&](auto kern) { kern<<<persistent_grid_w(kern, sm, nitems), 256, sm, s>>>(ij, fj, a, nch, tm); };
    if (use_tma) {
        if (a.plan.g == 16) go(k_ywarp<R, INV, 16, true>);
        else go(k_ywarp<R, INV, 0, true>);
        return;
    }
    if (a.plan.g == 16) go(k_ywarp<R, INV, 16>);
    else go(k_ywarp<R, INV>);
}

template <bool INV>
bool ydispatch(const YInvJobList& ij, const YFwdJobList& fj, const YPassArgs& a, cudaStream_t s) {
    switch (a.plan.r) {
        case 1: ylaunch<1, INV>(ij, fj, a, s); return true;
        case 2: ylaunch<2, INV>(ij, fj, a, s); return true;
        case 3: ylaunch<3, INV>(ij, fj, a, s); return true;
        case 4: ylaunch<4, INV>(ij, fj, a, s); return true;
        case 6: ylaunch<6, INV>(ij, fj, a, s); return true;
        case 8: ylaunch<8, INV>(ij, fj, a, s); return true;
        default: return false;
    }
}

template <int R, class V>
void rowlaunch_t(const RowJobList& jobs, const RowArgs& a, cudaStream_t s, bool c2r) {
    const int N = a.nxl / 2;
    const size_t sm = (size_t)8 * 32 * (N + 8) * sizeof(V) / a.rp.half.g;  // row stride N + 8 (swizzle)
    const long long units = (long long)jobs.n * a.nyl * a.nzp;
    const long long blocks = (units + 8 * 32 / a.rp.half.g - 1) / (8 * 32 / a.rp.half.g);
    const bool g32 = a.rp.half.g == 32;
    if (!c2r && g32 && N == 32 * R) {
        const size_t ss = (size_t)8 * (N + 8) * sizeof(V);
        const long long b32 = (units + 7) / 8;
        lsb::note_launch();
        k_row_r2c_s<R, V><<<persistent_grid_w(k_row_r2c_s<R, V>, ss, b32), 256, ss, s>>>(jobs, a);
        return;
    }
    lsb::note_launch();
    if (c2r) {
        if (g32) k_row_c2r_w<R, V, 32><<<persistent_grid_w(k_row_c2r_w<R, V, 32>, sm, blocks), 256, sm, s>>>(jobs, a);
        else k_row_c2r_w<R, V><<<persistent_grid_w(k_row_c2r_w<R, V>, sm, blocks), 256, sm, s>>>(jobs, a);
    } else {
        if (g32) k_row_r2c_w<R, V, 32><<<persistent_grid_w(k_row_r2c_w<R, V, 32>, sm, blocks), 256, sm, s>>>(jobs, a);
        else k_row_r2c_w<R, V><<<persistent_grid_w(k_row_r2c_w<R, V>, sm, blocks), 256, sm, s>>>(jobs, a);
    }
}

template <int R>
void rowlaunch(const RowJobList& jobs, const RowArgs& a, cudaStream_t s, bool c2r) {
    if (a.f32) rowlaunch_t<R, float2>(jobs, a, s, c2r);
    else rowlaunch_t<R, double2>(jobs, a, s, c2r);
}

bool rowdispatch(const RowJobList& jobs, const RowArgs& a, cudaStream_t s, bool c2r) {
    switch (a.rp.half.r) {
        case 1: rowlaunch<1>(jobs, a, s, c2r); return true;
        case 2: rowlaunch<2>(jobs, a, s, c2r); return true;
        case 3: rowlaunch<3>(jobs, a, s, c2r); return true;
        case 4: rowlaunch<4>(jobs, a, s, c2r); return true;
        case 6: rowlaunch<6>(jobs, a, s, c2r); return true;
        case 8: rowlaunch<8>(jobs, a, s, c2r); return true;
        default: return false;
    }
}

template <int R>
void nllaunch(const NlRowArgs& a, cudaStream_t s) {
    const int N = a.r.nxl / 2;
    const int nitems = a.r.nyl * a.r.nzp;
    if (a.r.f32) {
        if (a.r.rp.half.g != 32) throw std::runtime_error("mixed precision: x transform length has no full-warp plan");
        constexpr size_t sm = nl_f_smem<R>();
        if (!allow_smem((const void*)k_row_nl_f<R>, sm))
            throw std::runtime_error("product rows: shared memory of the register plan refused");
        const int occ = resident_blocks((const void*)k_row_nl_f<R>, 128, sm);
        long long blocks = (long long)occ * sm_count(), need = (nitems + 3) / 4;
        if (blocks > need) blocks = need > 0 ? need : 1;
        { lsb::note_launch(); k_row_nl_f<R><<<(int)blocks, 128, sm, s>>>(a); }
        return;
    }
    if (a.r.rp.half.g == 32) {
        constexpr size_t sm = nl_r_smem<R>();
        if (!allow_smem((const void*)k_row_nl_r<R>, sm))
            throw std::runtime_error("product rows: shared memory of the register plan refused");
        const int occ = resident_blocks((const void*)k_row_nl_r<R>, 128, sm);
        long long blocks = (long long)occ * sm_count(), need = (nitems + 3) / 4;
        if (blocks > need) blocks = need > 0 ? need : 1;
        { lsb::note_launch(); k_row_nl_r<R><<<(int)blocks, 128, sm, s>>>(a); }
        return;
    }
    const size_t sm =
        ((size_t)18 * a.r.kxc + (size_t)12 * N + (size_t)8 * 32 / a.r.rp.half.g * (N + 1)) * sizeof(double2);
    { lsb::note_launch(); k_row_nl_w<R><<<persistent_grid_w(k_row_nl_w<R>, sm, nitems), 256, sm, s>>>(a); }
}

}  // namespace

bool launch_yinv_warp(const YInvJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (a.plan.g == 0) return false;
    YFwdJobList none{};
    return ydispatch<true>(jobs, none, a, s);
}

bool launch_yfwd_warp(const YFwdJobList& jobs, const YPassArgs& a, cudaStream_t s) {
    if (a.plan.g == 0) return false;
    YInvJobList none{};
    return ydispatch<false>(none, jobs, a, s);
}

bool launch_row_c2r_warp(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (a.rp.half.g == 0) return false;
    return rowdispatch(jobs, a, s, true);
}

bool launch_row_r2c_warp(const RowJobList& jobs, const RowArgs& a, cudaStream_t s) {
    if (a.rp.half.g == 0) return false;
    return rowdispatch(jobs, a, s, false);
}

namespace {
template <int R>
void dynlaunch(const DynRowArgs& a, cudaStream_t s) {
    const size_t sm = (size_t)4 * dyn_row_slots<R>() * (a.r.f32 ? sizeof(float2) : sizeof(double2));
    const void* k = a.r.f32 ? (const void*)k_row_c2r_dyn<R, float2> : (const void*)k_row_c2r_dyn<R, double2>;
    if (!allow_smem(k, sm)) throw std::runtime_error("dynamic-model row pass: shared memory refused");
    const int nrows = a.r.nyl * a.r.nzp;
    long long blocks = (long long)resident_blocks(k, 128, sm) * sm_count(), need = (nrows + 3) / 4;
    if (blocks > need) blocks = need > 0 ? need : 1;
    lsb::note_launch();
    if (a.r.f32) k_row_c2r_dyn<R, float2><<<(int)blocks, 128, sm, s>>>(a);
    else k_row_c2r_dyn<R, double2><<<(int)blocks, 128, sm, s>>>(a);
}
}  // namespace

namespace {
template <int R>
void taulaunch(const TauRowArgs& a, cudaStream_t s) {
    // 4-warp blocks: at ~100 registers, 5 blocks (20 warps) fit an SM where 8-warp blocks fit 2
    const size_t sm = (size_t)4 * (32 * R + 8) * (a.r.f32 ? sizeof(float2) : sizeof(double2));
    const void* k = a.r.f32 ? (const void*)k_row_r2c_tau<R, float2> : (const void*)k_row_r2c_tau<R, double2>;
    if (!allow_smem(k, sm)) throw std::runtime_error("dynamic-model stress row pass: shared memory refused");
    const int nrows = a.r.nyl * a.r.nzp;
    long long blocks = (long long)resident_blocks(k, 128, sm) * sm_count(), need = (nrows + 3) / 4;
    if (blocks > need) blocks = need > 0 ? need : 1;
    lsb::note_launch();
    if (a.r.f32) k_row_r2c_tau<R, float2><<<(int)blocks, 128, sm, s>>>(a);
    else k_row_r2c_tau<R, double2><<<(int)blocks, 128, sm, s>>>(a);
}
}  // namespace

bool row_r2c_tau_plan(const RowArgs& r) { return row_c2r_dyn_plan(r); }

void launch_row_r2c_tau(const TauRowArgs& a, cudaStream_t s) {
    switch (row_r2c_tau_plan(a.r) ? a.r.rp.half.r : 0) {
        case 2: taulaunch<2>(a, s); break;
        case 4: taulaunch<4>(a, s); break;
        case 6: taulaunch<6>(a, s); break;
        case 8: taulaunch<8>(a, s); break;
        default: throw std::runtime_error("dynamic-model stress row pass: no fused plan for this length");
    }
}

bool row_c2r_dyn_plan(const RowArgs& r) {
    const int R = r.rp.half.r;
    return r.rp.half.g == 32 && (R == 2 || R == 4 || R == 6 || R == 8);
}

void launch_row_c2r_dyn(const DynRowArgs& a, cudaStream_t s) {
    switch (row_c2r_dyn_plan(a.r) ? a.r.rp.half.r : 0) {
        case 2: dynlaunch<2>(a, s); break;
        case 4: dynlaunch<4>(a, s); break;
        case 6: dynlaunch<6>(a, s); break;
        case 8: dynlaunch<8>(a, s); break;
        default: throw std::runtime_error("dynamic-model row pass: no fused plan for this length");
    }
}

bool launch_row_nl_warp(const NlRowArgs& a, cudaStream_t s) {
    if (a.r.rp.half.g == 0) return false;
    switch (a.r.rp.half.r) {
        case 1: nllaunch<1>(a, s); return true;
        case 2: nllaunch<2>(a, s); return true;
        case 3: nllaunch<3>(a, s); return true;
        case 4: nllaunch<4>(a, s); return true;
        case 6: nllaunch<6>(a, s); return true;
        case 8: nllaunch<8>(a, s); return true;
        default: return false;
    }
}

}  // namespace lsb
