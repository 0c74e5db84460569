/*
 * gpe.h -- C ABI of the B200 (sm_100a) dipolar Gross-Pitaevskii solver.
 *
 * Drop-in for the hot path of DBEC-GP-MPI-CUDA's imag3d-mpicuda and
 * real3d-mpicuda: the split-step Crank-Nicolson propagator in imaginary time
 * (real FP64 psi, renormalised every step) and in real time (complex128 psi).
 * The reference keeps its state in file-scope globals and exposes C functions
 * on cudaPitchedPtr arguments (src/imag3d-mpicuda/imag3d-mpicuda.cuh:48-159);
 * here every piece of device state is owned by a handle, so solvers are
 * re-entrant and several can live in one process.
 *
 * Conventions
 *  - Host arrays are x-major [nx][ny][nz] with z contiguous, as the reference
 *    host tensors (src/utils/mem.c:104-130).  Complex psi is interleaved
 *    (re, im) doubles like the reference's cuDoubleComplex tensor
 *    (real3d-mpicuda.cu:40); page-locked buffers are copied without staging.
 *  - Every call returns a gpe_status; the library never calls exit().
 *    gpe_last_error() returns a thread-local message for the last failure.
 *  - One host thread per handle.  Work is queued on the handle's stream
 *    (the caller's cudaStream_t if one was given to gpe_create).
 *  - The library owns all device memory; callers own host buffers.
 */
#ifndef GPE_H
#define GPE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
   GPE_OK = 0,
   GPE_ERR_PARAM = 1,       /* invalid argument or unsupported grid */
   GPE_ERR_CUDA = 2,        /* a CUDA runtime call failed */
   GPE_ERR_OOM = 3,         /* device allocation failed */
   GPE_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
   GPE_ERR_STATE = 5,       /* call not valid in the handle's state */
   GPE_ERR_IO = 6,          /* file could not be read or written */
   GPE_ERR_UNSUPPORTED = 7, /* feature not available in this build */
   GPE_ERR_BUDGET = 8,      /* admission refused by the memory budget */
   GPE_ERR_CANCELLED = 9    /* request cancelled (gpe_server_cancel) */
} gpe_status;

enum { GPE_MODE_IMAG = 0, GPE_MODE_REAL = 1 };
enum { GPE_PREC_FP64 = 0, GPE_PREC_MIXED = 1 };

/* Density outputs, the reference's out* writers
 * (src/imag3d-mpicuda/imag3d-mpicuda.cu:1944-2399). */
enum {
   GPE_DEN_1D_X = 0, GPE_DEN_1D_Y = 1, GPE_DEN_1D_Z = 2,
   GPE_DEN_2D_XY = 3, GPE_DEN_2D_XZ = 4, GPE_DEN_2D_YZ = 5,
   GPE_DEN_3D_XY0 = 6, GPE_DEN_3D_X0Z = 7, GPE_DEN_3D_0YZ = 8,
   GPE_DEN_3D = 9
};

/* Physical and numerical parameters: the keys of readpar()
 * (src/imag3d-mpicuda/imag3d-mpicuda.cu:650-829).  g and gd are not part of
 * the handle; they are passed per run so that ramps and quenches follow the
 * reference's phase loops exactly. */
typedef struct {
   int mode;         /* GPE_MODE_IMAG or GPE_MODE_REAL */
   int precision;    /* GPE_PREC_FP64 or GPE_PREC_MIXED */
   int opt;          /* OPTION: par = 2 if opt == 2, else 1 */
   int device;       /* CUDA device, -1 = current (DEVICE key) */
   long nx, ny, nz;  /* even, in [8, 1024], prime factors 2, 3 and 5 only */
   double dx, dy, dz, dt;
   double gamma, nu, lambda;
   double cutoff;
} gpe_params;

typedef struct gpe_solver gpe_solver;

/* Replaces initdevice() + the cudaMalloc3D calls of main()
 * (imag3d-mpicuda.cu:103-176, 982-1154).  stream may be NULL. */
gpe_status gpe_create(const gpe_params *p, void *stream, gpe_solver **out);
void gpe_destroy(gpe_solver *s);
const char *gpe_last_error(void);
/* Device bytes the handle would allocate for these parameters. */
gpe_status gpe_device_bytes(const gpe_params *p, long long *bytes);

/* initpsi Gaussian (imag3d-mpicuda.cu:835-867, real3d-mpicuda.cu:914-923). */
gpe_status gpe_init_gaussian(gpe_solver *s);
/* real3d initpsi from imag3d-den.bin: psi = (sqrt(rho), 0)
 * (real3d-mpicuda.cu:925-947); rho is a host [nx][ny][nz] array. */
gpe_status gpe_init_density(gpe_solver *s, const double *rho);
/* Host <-> device psi (the psiparam cudaMemcpy3D of imag3d-mpicuda.cu:226-236):
 * nx*ny*nz doubles in imaginary time, 2*nx*ny*nz interleaved doubles in real
 * time.  Both calls return when the copy has completed. */
gpe_status gpe_set_psi(gpe_solver *s, const double *psi);
gpe_status gpe_get_psi(gpe_solver *s, double *psi);

/* calcnorm (imag3d-mpicuda.cu:1194-1233; real3d-mpicuda.cu:1304-1322).
 * renormalize != 0 divides psi by the norm as imag3d does. */
gpe_status gpe_calcnorm(gpe_solver *s, int renormalize, double *norm);
/* The step loops of imag3d-mpicuda.cu:309-325,397-404,472-479 and
 * real3d-mpicuda.cu:328-339,411-424,496-508.  Before each step
 * *g += g_inc, *gd += gd_inc.  In imaginary time every step ends with the
 * renormalisation and *last_norm (may be NULL) receives the last
 * pre-renormalisation norm (left untouched when nsteps == 0 or in real
 * time).  rms_every > 0 evaluates calcrms after every step whose index c
 * satisfies c % rms_every == 0 (DYNAOUT, real3d:419-423)
 * into rms_out[4 * (c / rms_every)]; rms_every <= 0 disables it. */
gpe_status gpe_run(gpe_solver *s, long nsteps, double *g, double *gd, double g_inc, double gd_inc,
                   double *last_norm, long rms_every, double *rms_out);
/* calcmuen (imag3d-mpicuda.cu:1250-1450): mu and E, not divided by par. */
gpe_status gpe_calcmuen(gpe_solver *s, double g, double gd, double *mu, double *en);
/* calcrms (imag3d-mpicuda.cu:1639-1744): rms[0] = <r>, rms[1..3] = <x>,<y>,<z>. */
gpe_status gpe_calcrms(gpe_solver *s, double *rms);
/* |psi(Nx/2, Ny/2, Nz/2)|^2 (psiNx2Ny2Nz2param, imag3d-mpicuda.cu:231-236). */
gpe_status gpe_psi_center2(gpe_solver *s, double *value);
/* Density outputs (out* writers, imag3d-mpicuda.cu:1944-2399).  Writes the
 * doubles the reference writes to the file (pairs, triples or raw 3D) into
 * out (capacity cap doubles); *count receives the number written. */
gpe_status gpe_density(gpe_solver *s, int kind, long outstpx, long outstpy, long outstpz,
                       double *out, long cap, long *count);

/* Operator-level entry points, one per reference routine, for parity tests. */
gpe_status gpe_calcpsidd2(gpe_solver *s);               /* calcpsidd2_mem, imag3d:1460-1510 */
gpe_status gpe_get_phi(gpe_solver *s, double *phi);     /* psidd2 real view [nx][ny][nz] */
gpe_status gpe_calcnu(gpe_solver *s, double g, double gd); /* calcnu, imag3d:1752-1783 */
gpe_status gpe_calclux(gpe_solver *s);                  /* calclux, imag3d:1790-1844 */
gpe_status gpe_calcluy(gpe_solver *s);                  /* calcluy, imag3d:1851-1900 */
gpe_status gpe_calcluz(gpe_solver *s);                  /* calcluz, imag3d:1907-1942 */
gpe_status gpe_synchronize(gpe_solver *s);

/* Self-test of the bounded device waits (no reference counterpart: the
 * reference's kernels never wait on the device).  Queues one CTA that waits,
 * polling at most `spins` times (1..65536), on an mbarrier expecting a
 * transaction that no copy delivers; no copy is issued, so nothing is in
 * flight when it gives up.  The next gpe_synchronize (or gpe_run) returns
 * GPE_ERR_TIMEOUT and clears the handle's status word, after which the handle
 * works normally. */
gpe_status gpe_selftest_wait_timeout(gpe_solver *s, unsigned spins);
/* Kernel launches queued by this handle since creation (for accounting). */
gpe_status gpe_launch_count(gpe_solver *s, long long *count);
/* Step timing on the handle's stream: runs nsteps plain steps (fixed g, gd)
 * bracketed by CUDA events and returns the elapsed milliseconds. */
gpe_status gpe_time_steps(gpe_solver *s, long nsteps, double g, double gd, double *ms);
/* Timing of the dipolar convolution alone (calcpsidd2, imag3d-mpicuda.cu:
 * 1460-1510): after one untimed call, nrep calls bracketed by CUDA events on
 * the handle's stream; *ms receives the mean milliseconds per call (the
 * figure gpe_cufft_convolution in gpe_cufft.h is compared with). */
gpe_status gpe_time_calcpsidd2(gpe_solver *s, long nrep, double *ms);
/* Per-kernel timing: runs nsteps plain steps with a CUDA event around every
 * kernel of the step and returns, per kernel of one step, the mean duration in
 * milliseconds (ms[i], i < *count <= cap).  gpe_step_kernel_name(i) names
 * kernel i, gpe_step_kernel_bytes(s, i) its algorithmic bytes per launch. */
gpe_status gpe_profile_step(gpe_solver *s, long nsteps, double g, double gd, double *ms, int cap, int *count);
const char *gpe_step_kernel_name(gpe_solver *s, int i);
double gpe_step_kernel_bytes(gpe_solver *s, int i);

/* Tile configuration of a handle (no reference counterpart: the reference
 * has one fixed cuFFT + one-thread-per-line layout).  Zero fields select the
 * built-in heuristic. */
typedef struct gpe_tuning {
   int sweep_tw[3];     /* lines per CTA of the x, y, z sweeps (a power of two) */
   int sweep_stages[3]; /* TMA pipeline depth of the x, y, z sweeps: 2 or 3 */
   int fft_tile[2];     /* kz columns per tile of the y and x FFT passes */
   int fft_max_radix;   /* largest radix of the FFT plans: 16 (mixed precision only), 8, 4 or 2 */
   int sweep_seg[3];    /* points per recurrence segment of the x, y, z sweeps: 8, 16 or
                           32 (32: mixed-precision imaginary time only; complex FP64
                           lines: 8) at most 256 threads per CTA */
} gpe_tuning;
/* The configuration in use (every field filled in). */
gpe_status gpe_get_tuning(gpe_solver *s, gpe_tuning *t);
/* Re-plans the tiles with t (NULL = all defaults); psi and the state are kept.
 * GPE_ERR_PARAM (and the previous configuration restored) when a value does not
 * fit this grid. */
gpe_status gpe_set_tuning(gpe_solver *s, const gpe_tuning *t);
/* Autotuner: times candidate configurations with gpe_profile_step (nsteps
 * steps each at couplings g, gd) and picks, per sweep axis, the fastest lines
 * per CTA, segment length and pipeline depth, and for the FFT passes the
 * fastest tile widths and largest radix; the picks are kept only if whole
 * steps (gpe_time_steps, best of two runs of 2 nsteps) are faster with them
 * than with the configuration the call started from.  psi and the state are
 * restored afterwards; the configuration in use is returned in *best (may be
 * NULL). */
gpe_status gpe_autotune(gpe_solver *s, double g, double gd, int nsteps, gpe_tuning *best);

/* Snapshot of a solve (no reference counterpart: the reference's
 * imag3d-den.bin keeps sqrt(density) only and loses the phase).  The file
 * holds a 192-byte header (magic "GPESNAP1", format version 1, the handle's
 * gpe_params, couplings g and gd, the caller's step counter, payload size
 * and a 64-bit FNV-1a checksum of the payload) followed by psi exactly as the
 * handle stores it (FP64 or FP32, real or interleaved complex, x-major).  A
 * pending imaginary-time renormalisation is applied before writing. */
gpe_status gpe_snapshot_save(gpe_solver *s, const char *path, double g, double gd, long long step);
/* Loads a snapshot into a handle with the same grid, mode and precision
 * (GPE_ERR_PARAM otherwise; GPE_ERR_IO for a short, corrupt or foreign file);
 * returns the stored couplings and step counter (pointers may be NULL). */
gpe_status gpe_snapshot_load(gpe_solver *s, const char *path, double *g, double *gd, long long *step);

/* ---------------------------------------------------------------- batch
 * Many independent solves with their own grids and parameters (no reference
 * counterpart: the reference runs one solve per MPI job).  Each instance is a
 * full handle (its own stream and device memory); one batch step runs one
 * split step of every instance: the instances' kernels, captured once into a
 * CUDA graph with one branch per instance, are relaunched as one graph per
 * step, so small instances run concurrently on the GPU. */
typedef struct gpe_batch gpe_batch;
/* params[i] and couplings g[i], gd[i] of instance i (n >= 1).  Instances in
 * mixed-precision imaginary time start with 32-point segments in their y and z
 * sweeps (gpe_tuning.sweep_seg), the batched launches' faster choice; any
 * instance's tiles can be changed with gpe_set_tuning on its handle. */
gpe_status gpe_batch_create(const gpe_params *params, const double *g, const double *gd, int n, gpe_batch **out);
void gpe_batch_destroy(gpe_batch *b);
/* The handle of instance i (owned by the batch): initial state, observables. */
gpe_status gpe_batch_solver(gpe_batch *b, int i, gpe_solver **s);
/* New couplings for every instance (the step graph is captured again). */
gpe_status gpe_batch_set_couplings(gpe_batch *b, const double *g, const double *gd);
/* Autotunes one instance per distinct (grid, mode, precision) with
 * gpe_autotune (nsteps per trial) and applies its choice to the others, then
 * keeps those choices only if a timed batch step (best of two runs of nsteps)
 * is faster with them than with the tiles the instances had before; psi and
 * the step state of every instance are as before the call. */
gpe_status gpe_batch_autotune(gpe_batch *b, int nsteps);
/* nsteps batch steps, then the pending renormalisation of imaginary-time
 * instances; returns after the GPU finished. */
gpe_status gpe_batch_run(gpe_batch *b, long nsteps);
/* nsteps batch steps bracketed by CUDA events: elapsed milliseconds. */
gpe_status gpe_batch_time_steps(gpe_batch *b, long nsteps, double *ms);
/* Per-pass timing of batch steps: nsteps steps launched pass by pass with a
 * CUDA event after every pass; ms[q] (q < *count = 10, cap >= 10) receives the
 * mean milliseconds of pass q per step, summed over the groups, in the order
 * z forward FFT, y FFT, x convolution, inverse y FFT, z inverse FFT, phi
 * boundary planes, x sweep with calcnu, y sweep, z sweep, norm. */
gpe_status gpe_batch_profile_step(gpe_batch *b, long nsteps, double *ms, int cap, int *count);
/* Kernel launches executed by batch steps so far. */
gpe_status gpe_batch_launch_count(gpe_batch *b, long long *count);

/* --------------------------------------------------------------- server
 * Request server with continuous batching (no reference counterpart).  A
 * worker thread admits queued requests while the summed gpe_device_bytes of
 * the active solves stays within the HBM budget and fewer than max_active are
 * running, keeps each psi resident on the device, runs all active solves
 * concurrently in chunks (each on its own stream), and retires a solve when it
 * has converged (ground state) or done its steps (evolution); requests that
 * arrive meanwhile are admitted at the next chunk boundary. */
typedef struct gpe_server gpe_server;
enum { GPE_REQ_GROUND = 0, GPE_REQ_EVOLVE = 1 };
typedef struct gpe_request {
   gpe_params p;       /* p.mode: GPE_MODE_IMAG for GROUND, GPE_MODE_REAL for EVOLVE */
   int kind;           /* GPE_REQ_GROUND or GPE_REQ_EVOLVE */
   double g, gd;       /* couplings */
   double tol;         /* GROUND: stop when |mu_k - mu_{k-1}| / |mu_k| < tol between checks */
   long check_every;   /* GROUND: steps between mu checks; EVOLVE: steps per chunk */
   long max_steps;     /* GROUND: step cap; EVOLVE: steps to run */
} gpe_request;
typedef struct gpe_result {
   long long id;
   int status;         /* gpe_status of the solve */
   long steps;         /* steps run */
   double mu, en;      /* calcmuen at the end */
   double norm;        /* calcnorm at the end (before any renormalisation) */
   double rms[4];      /* calcrms at the end */
   double t_submit, t_start, t_done;  /* seconds since the server started */
} gpe_result;
/* device: CUDA ordinal (-1 = current); hbm_budget_bytes: admission budget. */
gpe_status gpe_server_create(int device, long long hbm_budget_bytes, int max_active, gpe_server **out);
/* Stops the worker after the queued and active requests finished. */
void gpe_server_destroy(gpe_server *sv);
gpe_status gpe_server_submit(gpe_server *sv, const gpe_request *rq, long long *id);
/* Waits (at most timeout_s seconds, < 0 = forever) for request id; fills res.
 * GPE_ERR_TIMEOUT when it has not finished in time. */
gpe_status gpe_server_wait(gpe_server *sv, long long id, double timeout_s, gpe_result *res);
/* Cancels request id.  A queued request is finished at once; an admitted one
 * stops at its next chunk boundary (no kernels of it in flight), its memory
 * is freed, and its result (gpe_server_wait) has status GPE_ERR_CANCELLED and
 * the steps it ran.  GPE_ERR_STATE when the request has already finished,
 * GPE_ERR_PARAM for an unknown id. */
gpe_status gpe_server_cancel(gpe_server *sv, long long id);
/* stats[0] requests done, [1] peak active, [2] peak bytes admitted, [3] chunks run. */
gpe_status gpe_server_stats(gpe_server *sv, double *stats);

/* Norm of a device-resident psi with no device allocation.  No counterpart in
 * the reference: it serves callers that cannot call cudaMalloc where they need
 * the norm (a latency-critical loop that must not take cudaMalloc/cudaFree's
 * implicit synchronisation, or a process whose device memory belongs to
 * another allocator).  psi_dev: nx*ny*nz doubles (mode GPE_MODE_IMAG, 8-byte
 * aligned) or interleaved complex doubles (GPE_MODE_REAL, 16-byte aligned),
 * x-major; norm_dev: one 8-byte aligned device double that receives
 * sqrt(Simpson integral of |psi|^2), as calcnorm.  Work is queued on stream
 * (NULL = default stream) and nothing is allocated: the per-row partials live
 * in a 2 MiB file-scope device array, so nx*ny must be at most 262144 and nx,
 * nz at most 1024; sizes beyond that and misaligned pointers are refused with
 * GPE_ERR_PARAM before anything is launched.  The first call in a CUDA context
 * looks up that array's address and caches it for the context (a context
 * created after cudaDeviceReset looks it up again); make that first call
 * before any stream capture.  Calls that overlap on the GPU share the array
 * and race. */
gpe_status gpe_norm_noalloc(const void *psi_dev, int mode, long nx, long ny, long nz, double dx, double dy, double dz,
                            double *norm_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GPE_H */
