// The library handle (shared by lsbgpu.cu and sgs_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "lsb_internal.cuh"
#include "lsbgpu.h"

namespace lsb {

struct LsbError {
    int code;
    std::string msg;
};

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess)                                                                   \
            throw ::lsb::LsbError{LSB_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

struct Mat {
    double* p = nullptr;
    int M = 0, K = 0, Mp = 0, Kp = 0;
};

// SGS working set (physical fields on the unpadded grid, [nzp][ny][nx] each)
struct SgsWork {
    bool nonsym = false;        // interscale model: tau is not symmetric
    double* tau = nullptr;      // 9 fields, index 3*l + m
    double* H9 = nullptr;       // 9 spectral fields h(l,m) when tau is not symmetric
    double* w = nullptr;        // model work fields
    int nw = 0;
    double* zf = nullptr;       // z filter coefficients az, bz, cz (3*nzp each set) for the weight
                                // pairs (a, b), (1, 1), (1, 6), (1, 2)
    double* delta = nullptr;    // [nzp] (dx dy dz)^(1/3) of dynamic/sigma
    double* sdelta = nullptr;   // [nzp] static-Smagorinsky delta (its own quirks)
    double* scal = nullptr;     // device scalars (u_tau average)
    bool dyn1_fused = false;    // this step's row pass already wrote S_ij and delta^2 |S| S_ij
    bool dyn4_fused = false;    // the stresses are formed by the forward row pass (k_dyn4 skipped)
};

}  // namespace lsb

struct lsb_handle {
    lsb_config cfg{};
    lsb::Dims d;
    cudaStream_t own = nullptr, stream = nullptr;
    std::vector<void*> allocs;

    // set-up arrays
    double *wavx = nullptr, *wavy = nullptr, *zpts = nullptr, *ubar = nullptr, *ubarp = nullptr, *ubarpp = nullptr;
    double *hb = nullptr, *ht = nullptr, *d2hb = nullptr, *d2ht = nullptr, *lam = nullptr, *lamx = nullptr;
    std::vector<double> h_xpts, h_ypts, h_zpts, h_ubar;
    double dx = 0, dy = 0;
    lsb::Mat m_dz1, m_dz2, m_dz2rows, m_ei, m_eext;
    // FFT plans: y (ny), y padded (nyl), x real (nx), x real padded (nxl)
    lsb::FftPlan py, pyl;
    lsb::RealPlan rx, rxl;
    // state
    double *vel = nullptr, *veln = nullptr, *velnm = nullptr;  // 3S each
    double *nlc = nullptr, *nln = nullptr, *nlnm = nullptr;   // 3S each
    double *p = nullptr, *pn = nullptr;                       // S each
    // scratch
    double *filt = nullptr, *dz = nullptr, *H = nullptr, *rhs = nullptr, *T = nullptr, *divf = nullptr;
    lsb::OzMat oz_dz1, oz_ei, oz_eext;  // mixed form: int8 digits of D, E^-1, E (tensor cores)
    int* uerr = nullptr;         // device word raised by a tensor-core kernel whose wait timed out
    double *Y = nullptr;     // 18 y-intermediates on the (padded) transform grid
    double *Yu = nullptr;    // 12 y-intermediates on the unpadded grid
    double *phys = nullptr;  // physical scratch (unpadded grid), kPhys fields
    double *bc = nullptr, *bcp = nullptr, *bshape = nullptr;
    double *io = nullptr;    // host-transfer staging, 12 S
    double *red = nullptr;   // reduction scratch
    lsb::SgsWork sgs;
    double* tavg = nullptr;  // on-the-fly averages of u, v, w, p (4 S)
    double tns_ratio = 0.0;  // last TNS <I(h)>/<I(delta)>
    int* sgs_wall = nullptr;
    int sgs_nwall = 0;
    // per kernel-group CUDA-event timers (lsb_timers / lsb_timer_report)
    bool timing = false;
    // mixed form: the nonlinear term's padded-grid transforms and products in FP32 (false when
    // the padded x length has no full-warp register plan: those passes then run in FP64)
    bool nl_f32 = false;
    std::map<std::string, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> timers;
    static constexpr int kPhys = 24;
    long long Yl = 0, Yu1 = 0, P = 0;
    // scalars
    double t = 0, dt = 0, dt2 = 0, dt3 = 0;
    int istep = 0;
    double abfac[3] = {0, 0, 0}, bdf[3] = {0, 0, 0}, bdfv = 0;
    double bshape_norm = 0.0;  // bctype 1: S_top(0,0) / S_wall(0,0) helper

    // CUDA graphs of single steady steps (lsb_step), keyed by the history pointers (they
    // rotate with period 6) and the scalars that the launches carry
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        const void* key[8] = {};
        double dt = 0, ctop = 0, cwa = 0, cwb = 0;
        unsigned long long kernels = 0;  // kernels in one replay
    };
    std::vector<StepGraph> graphs;
    bool graphs_on = true;
    lsb_schedule sched{};  // launch schedule (lsb_set_schedule); zeros: the built-in models
    // bumped whenever the step graphs are dropped (a new schedule, graphs switched): the
    // ensemble graphs that captured this member's launches carry it in their key
    unsigned long long graph_gen = 0;
    void drop_graphs() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        ++graph_gen;
    }

    size_t device_bytes = 0;  // sum of this handle's device allocations
    double* alloc(size_t n) {
        void* q = nullptr;
        CK(cudaMalloc(&q, n * sizeof(double) > 0 ? n * sizeof(double) : 8));
        device_bytes += n * sizeof(double) > 0 ? n * sizeof(double) : 8;
        CK(cudaMemsetAsync(q, 0, n * sizeof(double), stream));
        allocs.push_back(q);
        return (double*)q;
    }
    double* upload(const double* h, size_t n) {
        double* q = alloc(n);
        CK(cudaMemcpyAsync(q, h, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        return q;
    }
    ~lsb_handle() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (void* q : allocs) cudaFree(q);
        if (own) cudaStreamDestroy(own);
    }
};


namespace lsb {
// an NVTX range around a piece of host code that launches work (seen by profilers that
// attach an NVTX tool; without one the calls return at once)
struct NvtxRange {
    explicit NvtxRange(const char* n) { nvtxRangePushA(n); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
// records CUDA events around the launches of one kernel group when timing is on, and an
// NVTX range of the group's name around them always.  Steps replayed from a CUDA graph run
// no host code, so their groups show inside the graph launch only.
struct TimerScope {
    lsb_handle* h;
    const char* name;
    cudaEvent_t a = nullptr, b = nullptr;
    TimerScope(lsb_handle* h_, const char* n) : h(h_), name(n) {
        nvtxRangePushA(n);
        if (h->timing) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, h->stream);
        }
    }
    ~TimerScope() {
        if (h->timing) {
            cudaEventRecord(b, h->stream);
            h->timers[name].emplace_back(a, b);
        }
        nvtxRangePop();
    }
};
// sgs_kernels.cu
void filters_init(lsb_handle* h);
void sgs_init(lsb_handle* h);
// the ifilt hook of timestep (src/navierstokes.f90:33-40) on the current u, v, w, p
void filter_hook(lsb_handle* h);
// xin/xout: nx further physical fields accumulated into spectral ones by the same forward
// transform launch (the fringe forcing into N)
void sgs_add_tau(lsb_handle* h, double* const* ph, bool dealias, const double* const* xin = nullptr,
                 double* const* xout = nullptr, int nx = 0, const double* xlam = nullptr,
                 const double* const* xmeans = nullptr);
void sgs_tau_phys(lsb_handle* h, const double* ui, const double* g, const double* uiuj, double* tau);
// the dynamic model's work fields S_ij (i = 0..5) and delta^2 |S| S_ij (i = 6..11), in the
// working type of the handle's precision
double* sgs_dyn_field(lsb_handle* h, int i);
void sgs_mul(double* y, const double* x, long long n, cudaStream_t s);
void diag_compute(lsb_handle* h, lsb_diagnostics* out);
// lsbgpu.cu helpers used by sgs_kernels.cu
// f32: physical fields and y-intermediates in FP32 (mixed form); spectral fields are FP64
// lam / lmeans / nlam: the first nlam fields enter as the fringe forcing lambda(x) (m - q),
// m = lmeans[i][z] (or 0), formed by the row transform as it reads them.  tau: the last six
// fields are the dynamic model's stresses, formed and transformed by the fused row pass from
// its inputs (their phys entries are not read)
void phys_to_spec(lsb_handle* h, const double* const* phys, double* const* spec, int nf, int nzp, double alpha,
                  double beta, double* const* ybuf, bool f32 = false, const double* lam = nullptr,
                  const double* const* lmeans = nullptr, int nlam = 0, const TauRowArgs* tau = nullptr);
void spec_to_phys(lsb_handle* h, const double* const* spec, double* const* phys, int nf, int nzp,
                  const double* const* means, const int* modes, bool f32 = false, double scale = 1.0);
void zgemm(lsb_handle* h, const Mat& m, const double* in, double* out, int nf, int epi, double alpha, double beta,
           const double* aux);
}  // namespace lsb
