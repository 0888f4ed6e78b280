/* lsbgpu.h -- C ABI of the B200 (sm_100a) implementation of LSBFLOW's per-time-step
 * hot path.  It is the drop-in boundary a Fortran driver binds through iso_c_binding
 * (bind(C) interfaces with the same argument order as the subroutines they replace)
 * or a Python/C host binds through ctypes / dlopen.
 *
 * Conventions
 *  - Every function returns an int status: 0 = LSB_OK, negative = error; the message
 *    of the last error of the calling thread is returned by lsb_last_error().
 *  - Arrays are FP64 in the reference's Fortran storage order (first index fastest):
 *      spectral  (nx, ny, nzp)     : nx reals = nx/2 complex kx modes interleaved Re/Im,
 *                                    ky in FFT order, k = 1 the ceiling, k = nzp the wall
 *      physical  (nx+2, ny, nzp)   : two pad columns per x row (written as 0, never read)
 *    nx, ny, nz are the reference's &dimen values, nzp = nz + 1, nzm = nz - 1.
 *  - Caller-owned host arrays are not retained after a call returns, except by the
 *    asynchronous copies of lsb_upload_velocity, lsb_download_velocity and
 *    lsb_snapshot_async, which use them when the handle's stream reaches the copy.
 *    Device state belongs to the handle.
 *  - A handle is one CUDA stream; it is not thread-safe, distinct handles are.
 *  - Temperature is not carried: the reference's set-up keeps T and its mean at exactly
 *    zero (src/init.f90:353-355,429), which makes every temperature term vanish.
 */
#ifndef LSBGPU_H
#define LSBGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define LSB_OK 0
#define LSB_ERR_ARG (-1)
#define LSB_ERR_CUDA (-2)
#define LSB_ERR_UNSUPPORTED (-3)
#define LSB_ERR_STATE (-4)
#define LSB_ERR_NONFINITE (-5)

typedef struct lsb_handle lsb_handle;

/* Run switches; the reference's namelists &dimen, &run, &param, &sgsin
 * (src/common.f90:20,78,92,107) restricted to what the time step reads. */
typedef struct {
    int nx, ny, nz;
    int dealiasflag;       /* 0 none, 1 3/2-rule products, 2 (3) exponential spectral filter  */
    int dealias_layout;    /* 0 = the reference's spanwise padding (src/dealiasing.f90:329,435),
                              1 = the textbook 3/2 layout                                        */
    int sgsflag, sgsmodel; /* sgsmodel 0 Smagorinsky, 1 dynamic, 2 sigma, 3 interscale, 4 TNS */
    int forcing;           /* 1: fringe forcing of src/navierstokes.f90:92-211                 */
    int bctype;            /* 0 homogeneous, 1 Spalart suction/blowing, 2 H-type strip,
                              3 ceiling dipole w = A (x-xc)/s exp(-((x-xc)/s)^2)                */
    int ifrz;
    int nstart;            /* 0: Euler/BDF2 start-up as src/navierstokes.f90:1500-1590       */
    int mapping;
    double xnu, u0, x0, xlen, ylen, zlen;
    double a, b, cs;       /* 3-point filter weights and the Smagorinsky constant             */
    double kc, filt_order, filt_amp;
    double istartbound, samp;
    double bc3_amp, bc3_xc, bc3_s;
    double fsize;          /* fringe fraction (bounds the z-CFL region in the diagnostics) */
    int dtadapt, iomod;    /* maxcalc every 5 steps and every iomod steps (src/navierstokes.f90:78-87) */
    int ifilt, modfilt;    /* filtering hook at the start of timestep (src/navierstokes.f90:33-40):
                              TNS automatic filtering when sgsmodel = 4, else filterall3pt */
    int otfavg, istartavg; /* on-the-fly time averages of u, v, w, p (src/main.f90:70-76) */
    int precision;         /* 0: FP64 throughout (the reference's arithmetic); 1: mixed form --
                              the nonlinear-term transforms, products and SGS model in FP32
                              with FP32 y-intermediates (the padded passes in FP64 when the
                              3/2-rule x length has no full-warp register plan), the nonlinear
                              term's z derivatives and the three velocity Helmholtz solves on
                              the int8 tensor cores (five int8 digits per operand with power-
                              of-two scales, exact int32 accumulation); the state, time
                              integration, boundary conditions, Poisson solve, pressure and
                              projection in FP64 (no reference counterpart) */
    int bc3_top;           /* ceiling condition for u, v with bctype 3 (no reference counterpart):
                              0 = the reference's u, v = -rhs/(k^2 + sigma/beta) on the ceiling
                              row (src/navierstokes.f90:1340-1347), an outflow condition that the
                              dipole's blowing half makes ill-posed (perturbations grow there);
                              1 = the free stream, u' = v = 0 on the ceiling in the velocity
                              Helmholtz solves (the projection then leaves a slip of
                              dt beta dp/dx, dt beta dp/dy there) */
} lsb_config;

/* Host set-up arrays (inputs, as the reference passes diag/smat/simat): see
 * src/init.f90:130-293 and src/helmholtz.f90:13-126.  Matrices are row-major [row][col]. */
typedef struct {
    const double* xpts;    /* [nx]  */
    const double* ypts;    /* [ny]  */
    const double* zpts;    /* [nzp] */
    const double* wavx;    /* [nx]  interleaved (wavx[2i] = wavx[2i+1] = i*alpha) */
    const double* wavy;    /* [ny]  FFT order */
    double dx, dy;
    const double* dz1;     /* [nzp][nzp] matrix applied by dfdz  */
    const double* dz2;     /* [nzp][nzp] matrix applied by d2fdz2 */
    const double* lam;     /* [nzm] eigenvalues of D2(2:nz,2:nz)   */
    const double* e;       /* [nzm][nzm] eigenvectors (columns)   */
    const double* ei;      /* [nzm][nzm] inverse                  */
    const double* ubar; const double* ubarp; const double* ubarpp;   /* [nzp] */
    const double* hbot; const double* htop; const double* d2hbot; const double* d2htop; /* [nzp] */
    const double* lamx;    /* [nx] fringe lambda(x) */
} lsb_setup;

typedef struct {
    double divergence;     /* mean |div u|, divcheck (src/derivatives.f90:348-392)    */
    double umax, umin, vmax, vmin, wmax, wmin;
    double cflx, cfly, cflz;
    double energy_total, energy_pert;  /* ener (src/orrsomm.f90:625-666) */
    double t, dt;
    int istep;
    int nonfinite;         /* 1 if any NaN/Inf was found in u, v, w */
} lsb_diagnostics;

const char* lsb_last_error(void);
int lsb_version(void);
/* kernels this library has launched since it was loaded, over all handles (no reference
   counterpart: a launch count for profiling and for checking that the GPU path ran) */
unsigned long long lsb_kernel_launches(void);
/* device memory held by a handle, in bytes (no reference counterpart: the serving loop
   admits runs by this footprint) */
int lsb_device_bytes(lsb_handle* h, unsigned long long* bytes);

/* ---------------- Tier 2: resident state --------------------------------------------- */
/* replaces initialize()'s device-side part (src/init.f90:7-127) */
int lsb_create(const lsb_config* cfg, const lsb_setup* setup, lsb_handle** out);
int lsb_destroy(lsb_handle* h);
/* run on a caller stream (cudaStream_t passed as void*); NULL restores the handle's own */
int lsb_set_stream(lsb_handle* h, void* stream);
/* the module ``core`` state (src/common.f90:162-175) and the ``time`` scalars */
int lsb_upload_state(lsb_handle* h, const double* uf, const double* vf, const double* wf,
                     const double* pf, const double* pnf,
                     const double* unif, const double* unmif, const double* nlnif, const double* nlnmif,
                     double t, double dt, double dt2, double dt3, int istep);
int lsb_download_state(lsb_handle* h, double* uf, double* vf, double* wf, double* pf, double* pnf,
                       double* unif, double* unmif, double* nlnif, double* nlnmif,
                       double* t, double* dt, double* dt2, double* dt3, int* istep);
/* device-resident variants: pointers are device addresses of the same layouts */
int lsb_upload_state_device(lsb_handle* h, const double* uf, const double* vf, const double* wf);
int lsb_download_velocity_device(lsb_handle* h, double* uf, double* vf, double* wf);
/* nsteps calls of timestep() (src/navierstokes.f90:10-90) on the device.  Steady steps
 * (after the start-up steps, constant dt, no timers, dt adaptation or filter hook, a
 * boundary forcing amplitude that no longer depends on t) are replayed from CUDA graphs
 * captured on the handle's stream, one per rotation of the history buffers (at most 6);
 * the results are those of ordinary launches, bit for bit. */
int lsb_step(lsb_handle* h, int nsteps);
/* enable = 0: drop the step graphs and launch every kernel of every step (no reference
 * counterpart) */
int lsb_graphs(lsb_handle* h, int enable);
/* Launch schedule of a handle (no reference counterpart; FFTW's plan search is the nearest
 * analogue).  Zero fields keep the built-in models; a tuner (lsbflow_b200/autotune.py)
 * times candidates through lsb_step and persists the fastest per grid as JSON.  Every
 * schedule gives the same results bit for bit: it moves work between blocks, never the
 * order of a sum. */
typedef struct {
    int gemm_warps;      /* FP64 z contractions: warps (8 columns each) per CTA, 4..8;
                            0 = the wave-quantization model.  The Helmholtz / Poisson
                            solves run as one fused launch at 0, 4 and 6, as their two
                            contractions at 5, 7 and 8 */
    int filter_zchunks;  /* 3-point SGS test filter: z chunks a block column is split into,
                            1..(nzp+3)/4; 0 = the waves x planes-per-block model */
    int y_staging;       /* FP64 spanwise passes: tiles staged by cp.async (1) or by TMA tile
                            loads (2); 0 = the built-in choice (TMA on the padded grid,
                            cp.async on the unpadded one) */
    int filter_staging;  /* 3-point SGS test filter: plane ring filled by cp.async (1) or by TMA
                            row loads (2, rows of a multiple of 128 bytes); 0 = the built-in
                            choice (TMA for FP64 rows, cp.async for the FP32 rows of the mixed
                            form) */
} lsb_schedule;
/* out-of-range fields return LSB_ERR_ARG; the step graphs are dropped and re-captured */
int lsb_set_schedule(lsb_handle* h, const lsb_schedule* s);
int lsb_get_schedule(lsb_handle* h, lsb_schedule* s);
int lsb_diag(lsb_handle* h, lsb_diagnostics* out);
int lsb_synchronize(lsb_handle* h);
/* asynchronous host<->device copies of u, v, w only (the histories stay resident);
 * host buffers should be pinned for the copies to overlap */
int lsb_upload_velocity(lsb_handle* h, const double* uf, const double* vf, const double* wf);
int lsb_download_velocity(lsb_handle* h, double* uf, double* vf, double* wf);
/* CUDA-event timers per kernel group: enable=1 clears and starts, 0 stops;
 * the report has one "group launches total_ms" line per group */
int lsb_timers(lsb_handle* h, int enable);
/* the on-the-fly time averages (src/main.f90:70-76, sum of q/iomod since the last reset);
 * reset = 1 zeroes them afterwards as main.f90:104-106 does after writing qavg files */
int lsb_tavg(lsb_handle* h, double* uf, double* vf, double* wf, double* pf, int reset);
int lsb_timer_report(lsb_handle* h, char* buf, int buflen);
/* spanwise mean of u + ubar, v, w, p over y (run/spanwiseavg.m:1-7, the reference's
 * post-processing of q snapshots, here on the device from the current state) and the rms
 * about it, sqrt(mean_y (f - mean_y f)^2); mean and rms are host arrays [4][nzp][nx]
 * (field u, v, w, p; z; x) */
int lsb_spanwise_stats(lsb_handle* h, double* mean, double* rms);
/* the fields mpi_snapshot writes to a q file (src/mpi_io.f90:339-497): horfft(+1) of the
 * current state on the device, u + ubar, v, w, p as q[4][nzp][ny][nx] (x fastest, no pad
 * columns), copied to the host array q on the handle's stream WITHOUT waiting: q must stay
 * valid, and is complete only, once the stream has passed this point (an event recorded on
 * the stream set by lsb_set_stream, or lsb_synchronize).  Pinned memory lets the copies
 * overlap; steps queued afterwards run after them. */
int lsb_snapshot_async(lsb_handle* h, double* q);

/* ---------------- Ensembles: runs stepped together ----------------------------------- */
/* No counterpart in the reference (one run per mpiexec there).  A batch steps several
 * handles (ensemble members: same or different grids, Re, boundary forcing, precision)
 * together: lsb_batch_step(b, n) advances every member by n calls of timestep(), with the
 * results of lsb_step on each member alone, bit for bit.  When every member's step is
 * steady (the lsb_step graph conditions), the members' steps are captured as parallel
 * branches of one CUDA graph and each ensemble step is one graph launch on the batch's
 * stream; otherwise the members are stepped one by one on their own streams.  The batch
 * does not own its members: destroy the batch before any member.  The batch's steps
 * follow the work already queued on the members' streams, and work queued on a member's
 * stream after lsb_batch_step follows them.  All members and the batch belong to the
 * device that is current at lsb_batch_create.  Not
 * thread-safe; a member must not be stepped by another batch or thread meanwhile. */
typedef struct lsb_batch lsb_batch;
int lsb_batch_create(lsb_handle* const* members, int nmembers, lsb_batch** out);
int lsb_batch_destroy(lsb_batch* b);
int lsb_batch_step(lsb_batch* b, int nsteps);
int lsb_batch_synchronize(lsb_batch* b);
/* launch the ensemble graphs on a caller stream (cudaStream_t as void*; NULL restores the
 * batch's own); an event recorded there after lsb_batch_step follows every member's steps */
int lsb_batch_set_stream(lsb_batch* b, void* stream);
/* enable = 0: drop the ensemble graphs and step the members one by one; enable = 1 (the
 * default) captures them again when needed.  A member's lsb_set_schedule or lsb_graphs
 * changes its graph generation, which is part of the ensemble graphs' key: the batch then
 * captures new ensemble graphs by itself (or steps members one by one while that member's
 * graphs are off) */
int lsb_batch_graphs(lsb_batch* b, int enable);

/* ---------------- Tier 1: the reference's subroutine interfaces (host arrays) --------- */
/* horfft(ain, ainf, is)             src/horfft.f90:61      is = -1 phys->spec, +1 spec->phys */
int lsb_horfft(lsb_handle* h, double* ain, double* ainf, int is);
/* dealiasing_2d_fftw(a, b, ab)      src/dealiasing.f90:262 (physical in/out)   */
int lsb_dealias_product(lsb_handle* h, const double* a, const double* b, double* ab);
/* dfdx / dfdy / dfdz / d2fdz2 / lapl src/derivatives.f90:261,283,112,161,306 */
int lsb_dfdx(lsb_handle* h, const double* uf, double* out);
int lsb_dfdy(lsb_handle* h, const double* uf, double* out);
int lsb_dfdz(lsb_handle* h, const double* uf, double* out);
int lsb_d2fdz2(lsb_handle* h, const double* uf, double* out);
int lsb_lapl(lsb_handle* h, const double* uf, double* out);
/* divuv(uf, vf, divf)               src/derivatives.f90:394 */
int lsb_divuv(lsb_handle* h, const double* uf, const double* vf, double* out);
/* solve_helmholtz(rhs, dtnui, n, diag, smat, simat)   src/helmholtz.f90:130 (n = nzm;
 * the eigenbasis given at lsb_create is used) */
int lsb_solve_helmholtz(lsb_handle* h, double* rhs, double dtnui);
/* solve_nhom_helmholtz(rhs, bc, dtnui, diag, smat, simat)   src/helmholtz.f90:211 */
int lsb_solve_nhom_helmholtz(lsb_handle* h, double* rhs, const double* bc, double dtnui);
/* nlterm_skewsym(uif, tempf, nltermif, nltempf, sgsflag)  src/navierstokes.f90:658
 * velocity part: uif = 3 spectral fields, nltermif = 3 spectral fields */
int lsb_nlterm(lsb_handle* h, const double* uif, double* nltermif);
/* tau_sgs(ui, uiuj, duidxj, tauij)  src/sgsterm.f90:10  (physical (nx+2,ny,nzp,3[,3]) arrays) */
int lsb_tau_sgs(lsb_handle* h, const double* ui, const double* uiuj, const double* duidxj, double* tauij);

/* ---------------- Allocation-free Helmholtz solve ------------------------------------ */
/* No counterpart in the reference.  solve_helmholtz (homogeneous Dirichlet BCs) for
 * callers that may not allocate GPU memory: programs whose device memory belongs to a
 * pool allocator or framework that forbids direct cudaMalloc, or time-stepping loops
 * that cannot pay for cudaMalloc/cudaFree's device-wide synchronisation.  No handle is
 * needed and nothing is allocated: every pointer is a device address the caller owns
 * (rhs, out: spectral (nx, ny, nzp); lam: nzm; e, ei: nzm x nzm row-major; wavx: nx;
 * wavy: ny), and the work memory is a static device array of LSB_NOALLOC_SCRATCH_BYTES
 * that every GPU loading the library keeps until exit.  Limit: nzp <= 129 (any nx*ny;
 * columns are processed in chunks that fit the array); larger nz returns
 * LSB_ERR_UNSUPPORTED.  The first call on a device looks up the array's address, so make
 * it before any stream capture.  Calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller.  stream is a cudaStream_t of the current
 * device (NULL = default); a stream of another device returns LSB_ERR_ARG.  The address
 * found on the first call is kept for the life of the process: a device reset
 * (cudaDeviceReset, or the primary context destroyed and made again) is not supported
 * afterwards. */
#define LSB_NOALLOC_SCRATCH_BYTES (8u << 20)
int lsb_solve_helmholtz_noalloc(int nx, int ny, int nz, const double* rhs, double* out, const double* lam,
                                const double* e, const double* ei, const double* wavx, const double* wavy,
                                double dtnui, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LSBGPU_H */
