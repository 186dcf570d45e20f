/* laminocam_b200 C ABI: the MBIR reconstruction hot path of LaminoCam
 * (aryabhatt/laminocam) on one NVIDIA B200.
 *
 * Conventions
 *  - Every function returns 0 on success or a non-zero LC_ERR_* code; the
 *    message of the last failure is lc_last_error(ctx).  This replaces the
 *    reference's std::runtime_error / std::invalid_argument throws
 *    (include/gpu/utils.h:31-49, include/finufft_plan.h:97-107).
 *  - Arrays are row-major float32 with the last dimension fastest, exactly the
 *    reference's Array<T> / DeviceArray<T> layout {n1, n2, n3}
 *    (include/dtypes.h:29-60).
 *  - Functions whose array arguments are described as "device" take device
 *    pointers that the caller owns; functions named lc_mbir* take host
 *    pointers and copy internally.
 *  - All device work is issued on the context's stream; a context is used by
 *    one host thread at a time.  Destroy handles before their context.
 *  - NUFFT tolerance arguments follow FINUFFT (include/finufft_plan.h:48,71;
 *    include/gpu/cufinufft_plan.h:49,75); pass <= 0 for the default 1e-6.
 */
#ifndef LAMINOCAM_H
#define LAMINOCAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LC_OK 0
#define LC_ERR_INVALID 1  /* bad argument or size */
#define LC_ERR_NOMEM 2    /* device allocation failed / over the memory budget */
#define LC_ERR_CUDA 3     /* CUDA runtime error */
#define LC_ERR_INTERNAL 4 /* anything else */
#define LC_ERR_TOO_LARGE 5 /* sizes beyond a fixed maximum or above a server's HBM budget */
#define LC_ERR_TIMEOUT 6   /* lc_server_wait gave up before the job ended */

typedef struct lc_context_s *lc_context;
typedef struct lc_geometry_s *lc_geometry;
typedef struct lc_psf_s *lc_psf;

/* ---- context ---------------------------------------------------------- */
int lc_version(void);
/* stream: a cudaStream_t or NULL for a private non-blocking stream */
int lc_context_create(int device, void *stream, lc_context *out);
int lc_context_destroy(lc_context ctx);
int lc_context_set_stream(lc_context ctx, void *stream);
int lc_context_synchronize(lc_context ctx);
const char *lc_last_error(lc_context ctx);

/* ---- geometry --------------------------------------------------------- */
/* Replaces cpu::PolarGrid2D / gpu::PolarGrid2D (include/polar_grid2d.h:35-66,
 * include/gpu/polar_grid2d.h): x = r cos(theta), y = r sin(theta),
 * r_k = (k+1/2) 2pi/nradial - pi.  theta: host, radians, ntheta values. */
int lc_geometry2d_create(lc_context ctx, const double *theta, int ntheta, int nradial,
                         lc_geometry *out);
/* Replaces cpu::PolarGrid / gpu::PolarGrid (include/polar_grid.h:34-95,
 * include/rotation.h:28-56) plus the per-projection centre-of-rotation shifts
 * of backproj() (src/projection.cpp:100-131).  theta, gamma, beta: host,
 * radians, one per projection; shifts: host, 2 floats (dx, dy) per projection
 * in pixels, or NULL. */
int lc_geometry3d_create(lc_context ctx, const double *theta, const double *gamma,
                         const double *beta, const float *shifts, int ntheta, int nrows,
                         int ncols, lc_geometry *out);
int lc_geometry_destroy(lc_geometry g);

/* ---- projection operators (device pointers) ---------------------------- */
/* forward2d (src/projection.cpp:146-160): volume {ns, n2, n3} -> sino {ns, ntheta, nradial} */
int lc_forward2d(lc_context ctx, lc_geometry g, const float *volume, int ns, int n2, int n3,
                 float *sino, double tol);
/* backproj2d (src/projection.cpp:168-182): sino {ns, ntheta, nradial} -> volume {ns, n2, n3} */
int lc_backproj2d(lc_context ctx, lc_geometry g, const float *sino, int ns, int n2, int n3,
                  float *volume, double tol);
/* sysmat2d(x, PolarGrid2D) (src/gradient.cpp:55-69): Re(NUFFT1(NUFFT2(x))) / nradial */
int lc_sysmat2d_nufft(lc_context ctx, lc_geometry g, const float *x, int ns, int n2, int n3,
                      float *y, double tol);
/* forward (src/projection.cpp:42-64, CPU semantics incl. the |q|<=pi mask):
 * volume {n1, n2, n3} -> projections {ntheta, nrows, ncols} */
int lc_forward3d(lc_context ctx, lc_geometry g, const float *volume, int n1, int n2, int n3,
                 float *proj, double tol);
/* backproj (src/projection.cpp:69-131): projections -> volume {n1, n2, n3};
 * apply_shifts != 0 uses the geometry's per-projection shifts */
int lc_backproj3d(lc_context ctx, lc_geometry g, const float *proj, int n1, int n2, int n3,
                  int apply_shifts, float *volume, double tol);
/* sysmat(x, PolarGrid) (src/gradient.cpp:32-45): Re(NUFFT1(NUFFT2(x))) / (nrows*ncols) */
int lc_sysmat3d_nufft(lc_context ctx, lc_geometry g, const float *x, int n1, int n2, int n3,
                      float *y, double tol);

/* ---- Toeplitz PSF ------------------------------------------------------ */
/* Replaces cpu/gpu::PointSpreadFunction2D (include/toeplitz2d.h:40-126) for a
 * 2D geometry (n1 = number of slices, n2 == n3 = image size) and
 * cpu/gpu::PointSpreadFunction (include/toeplitz.h:35-130) for a 3D geometry
 * (volume {n1, n2, n3}).  The kernel is generated in FP64 on the device. */
int lc_psf_create(lc_context ctx, lc_geometry g, int n1, int n2, int n3, lc_psf *out);
/* lc_psf_create with flags: LC_PSF_FP32_NUFFT builds the kernel as the
 * reference GPU does (include/gpu/toeplitz2d.h:84-115), a FP32 type-1 NUFFT of
 * ones at tol 1e-6, instead of the exact FP64 closed form. */
#define LC_PSF_FP32_NUFFT 1
int lc_psf_create_ex(lc_context ctx, lc_geometry g, int n1, int n2, int n3, int flags, lc_psf *out);
int lc_psf_destroy(lc_psf psf);
/* P[3]: PSF grid (P[0] = 1 for 2D); spectrum_elems: stored real spectrum size */
int lc_psf_info(lc_psf psf, int *P, long *spectrum_elems);
/* FP64 PSF K on the P grid in mode order (index k + P/2), host buffer; the
 * planes of mode -P/2 along even axes are zero (the cropped convolution never
 * reads them) */
int lc_psf_kernel(lc_context ctx, lc_psf psf, double *host_out);
/* real R2C half spectrum {P0, P1, P2/2+1} of the zero-centred PSF (its
 * unpaired -P/2 planes zeroed), host buffer.  A 3D PSF whose kernel is even
 * in z applies its z stage from taps and builds this spectrum on the first
 * call: like lc_psf_kernel, it needs the PSF's geometry then. */
int lc_psf_spectrum(lc_context ctx, lc_psf psf, float *host_out);
/* sysmat(x, PSF) / sysmat2d(x, PSF2D) (src/gradient.cpp:49-52,76-79):
 * y = A^T A x, x and y device {n1, n2, n3} */
int lc_sysmat_toeplitz(lc_context ctx, lc_psf psf, const float *x, float *y);

/* ---- solvers ------------------------------------------------------------ */
typedef struct {
    int max_iters;    /* CG iterations, or Split-Bregman outer iterations */
    int inner_iters;  /* CG iterations per Split-Bregman outer iteration */
    float tol;        /* residual tolerance (0 disables) */
    float xtol;       /* relative-step tolerance (0 disables) */
    float lambda;     /* TV weight */
    float mu;         /* Bregman penalty */
    int fp32_scalars; /* 1: float dot products as the reference GPU path */
    int poll_every;   /* iterations between host checks of the stop flag */
    int use_graph;    /* 1: replay iterations as CUDA graphs (CG: a chunk of iterations,
                         Split-Bregman: one outer iteration); ignored while profiling */
    int residual_refresh; /* Split-Bregman: recompute the operator product A x of the
                             warm-started CG residual every this many outer iterations
                             (1, the default: every one); in between it is carried by
                             the CG updates (ax += alpha A p), equal up to rounding, which
                             saves one operator application per outer iteration */
} lc_solver_params;

typedef struct {
    int iters;          /* CG iterations, or Split-Bregman outer iterations */
    int cg_iters_total;
    double residual;    /* last CG ||r|| / (||y|| + 1e-8) */
    double dx;          /* last relative change */
    int stop_reason;    /* 0 max iters, 1 residual, 2 step, 3 |pAp| < 1e-10 */
    double elapsed_ms;  /* device time of the call */
} lc_solver_stats;

void lc_solver_params_default(lc_solver_params *p);

/* opt::cgsolver (include/optimize.h:89-91, src/conjgrad.cpp:33-76) with the
 * Toeplitz operator of psf.  rhs, x: device {n1, n2, n3}; x holds x0 on entry. */
int lc_cgsolver(lc_context ctx, lc_psf psf, const float *rhs, float *x, const lc_solver_params *p,
                lc_solver_stats *stats);
/* opt::split_bregman (include/optimize.h:74-77, src/bregman.cpp:36-94) */
int lc_split_bregman(lc_context ctx, lc_psf psf, const float *rhs, float *x,
                     const lc_solver_params *p, lc_solver_stats *stats);

/* The solvers over any linear operator, given as a callback: the
 * opt::Function<T> argument of opt::cgsolver / opt::split_bregman
 * (include/optimize.h:30-31, 74-91), e.g. the NUFFT normal operator of
 * tests/test_cg_normal.cpp:47-101 or a preconditioned one.  Each application
 * calls op(user, in, out, n, stream): in and out are device vectors of n
 * floats, stream the cudaStream_t to issue the work on; return 0 on success
 * (any other value stops the solve with LC_ERR_INVALID).  With
 * p->use_graph = 1 the iterations are captured into a CUDA graph, so op must
 * then only enqueue work on stream (no synchronisation, allocation or host
 * copies); with use_graph = 0 it may do anything.  The split-Bregman operator
 * is A^T A alone (mu times the negative Laplacian is added by the solver);
 * dims {n1, n2, n3} shape the finite differences. */
typedef int (*lc_operator_fn)(void *user, const float *in, float *out, long n, void *stream);
int lc_cgsolver_op(lc_context ctx, lc_operator_fn op, void *user, long n, const float *rhs, float *x,
                   const lc_solver_params *p, lc_solver_stats *stats);
int lc_split_bregman_op(lc_context ctx, lc_operator_fn op, void *user, const int *dims, const float *rhs,
                        float *x, const lc_solver_params *p, lc_solver_stats *stats);

/* ---- reconstruction drivers (host buffers) ------------------------------ */
typedef struct {
    int method;           /* 0: CG (UNCONSTRAINED), 1: Split-Bregman */
    lc_solver_params solver;
    double nufft_tol;     /* <= 0: 1e-6 */
    float pad_factor;     /* 3D only, ReconParams::PAD_FACTOR (1.4142) */
    int psf_fp32;         /* 0: the PSF kernel exactly in FP64 (default); 1: as the
                             reference GPU builds it, a FP32 type-1 NUFFT of ones at
                             tol 1e-6 (include/gpu/toeplitz2d.h:84-115); the PSF
                             cache is bypassed */
} lc_recon_params;

void lc_recon_params_default(lc_recon_params *p);

/* gpu::MBIR2D (src/gpu/mbir2d.cu:36-85) on a prepared sinogram
 * {ns, ntheta, nradial} (include/mbir2d_prep.h:44-65); recon {ns, n, n} with
 * recon_dims = {ns, n, n}. */
int lc_mbir2d(lc_context ctx, const float *sino, int ns, int ntheta, int nradial,
              const double *theta, const int *recon_dims, const lc_recon_params *p, float *recon,
              lc_solver_stats *stats);
/* gpu::MBIR (src/gpu/mbir.cu:41-167): stacked projections {ntheta, nrows, ncols}
 * with per-projection angles (radians); normalises by the maximum, pads by
 * pad_factor (odd sizes), backprojects, builds the PSF, solves and crops to
 * recon_dims {n1, n2, n3}. */
int lc_mbir3d(lc_context ctx, const float *projs, int ntheta, int nrows, int ncols,
              const double *theta, const double *gamma, const double *beta, const float *shifts,
              const int *recon_dims, const lc_recon_params *p, float *recon,
              lc_solver_stats *stats);

/* As lc_mbir3d with device pointers: projs {ntheta, nrows, ncols} and recon
 * {n1, n2, n3} stay in device memory (the DeviceArray overload of gpu::MBIR).
 * Returns when the reconstruction is complete. */
int lc_mbir3d_device(lc_context ctx, const float *projs, int ntheta, int nrows, int ncols,
                     const double *theta, const double *gamma, const double *beta,
                     const float *shifts, const int *recon_dims, const lc_recon_params *p,
                     float *recon, lc_solver_stats *stats);

/* ---- cross-job batching (replaces the reference's one-slice-at-a-time loops,
 * include/gpu/nufft.h:92-95 and include/gpu/toeplitz2d.h:68-76, for many
 * independent slices) -------------------------------------------------------
 * One 2D reconstruction job: a prepared sinogram {1, ntheta, nradial} in host
 * memory, its angles (radians), the image size n and a host output {n, n}. */
typedef struct {
    const float *sinogram;
    int ntheta, nradial;
    const double *theta;
    int n;
    float *recon;
} lc_job2d;
/* gpu::MBIR2D with CG (method 0) for njobs independent slices of any sizes:
 * each job's setup (upload, backprojection, FP64 PSF) runs on one of
 * setup_workers worker streams (<= 0: 8), then all jobs iterate in lockstep,
 * every CG stage one launch over the whole batch (p->solver.use_graph replays
 * eight iterations as a CUDA graph).  Each job stops on its own tests.  A
 * job's result does not depend on the other jobs of the batch.  stats (NULL,
 * or njobs entries) receives each job's iteration count and stop reason.
 * Returns when every recon is in host memory. */
int lc_mbir2d_batch(lc_context ctx, const lc_job2d *jobs, int njobs, const lc_recon_params *p,
                    int setup_workers, lc_solver_stats *stats);

/* ---- profiling (no counterpart in the reference, which has only a wall-clock
 * Timer, include/timer.h:30-64) ---------------------------------------- */
typedef struct {
    char name[32];   /* kernel section, e.g. "toeplitz_z_mid" */
    long count;      /* launches timed */
    double total_ms; /* summed CUDA-event time */
    double bytes;    /* summed algorithmic bytes */
} lc_profile_entry;

/* on != 0 starts timing every kernel section with CUDA events on the context
 * stream (and clears the totals); 0 stops */
int lc_profile_enable(lc_context ctx, int on);
int lc_profile_read(lc_context ctx, lc_profile_entry *out, int max_entries, int *n_entries);
/* number of kernels this library has launched in the process so far */
long lc_kernel_launches(void);

/* ---- allocation-free Toeplitz apply --------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while running (for example a reconstruction inside a detector's
 * acquisition loop that reserves all device memory up front, or a host that
 * forbids cudaMalloc/cudaFree after start-up because they can synchronise the
 * device): y = A^T A x for nslices slices of n x n, like lc_sysmat_toeplitz on
 * a 2D PSF, without any allocation.  The intermediate spectrum lives in a
 * 16 MiB array and the transform's twiddles in a 32 KiB array, both compiled
 * into the library (held by every GPU that loads it until the process exits).
 *   stream:   cudaStream_t the work is issued on (NULL = legacy default stream)
 *   spectrum: device, the PSF's real half spectrum {P, P/2+1}, as returned by
 *             lc_psf_spectrum for a 2D PSF of image size n
 *   P:        the PSF grid, next 2^p 3^q >= 2n-1 (lc_psf_info)
 *   x, y:     device {nslices, n, n}
 * Limits: P <= 4096 and nslices * n * (P/2+1) <= 2^21; larger sizes return
 * LC_ERR_TOO_LARGE.  CUDA loads the library's device code on its first use on
 * a device, and that load places the two arrays in device memory: make one
 * call on each device before reserving its memory and before any stream
 * capture.  The set-up call lc_sysmat2d_toeplitz_noalloc(NULL, NULL, 0, NULL,
 * NULL, 0, 0) does only that (the current device) and returns LC_OK.  Every
 * call looks up the arrays' device addresses again, so a cudaDeviceReset in
 * between is harmless.  All calls share both arrays, which keep the previous
 * call's contents, and each call rewrites the twiddles for its own P: calls
 * that overlap on the GPU (other streams, other threads) race, even on
 * disjoint outputs, and must be serialised by the caller. */
int lc_sysmat2d_toeplitz_noalloc(void *stream, const float *spectrum, int P, const float *x,
                                 float *y, int nslices, int n);

/* ---- reconstruction server ----------------------------------------------
 * Replaces running one recon_tomo / recon_lamino process per reconstruction
 * (src/recon.cpp:40-118, src/mbir2d.cpp:66-100) with a long-lived server on
 * one GPU.  Jobs submitted from any thread queue in FIFO order; a fixed set of
 * workers (one context and stream each) starts the head job once its
 * estimated device footprint fits the HBM budget next to the running jobs, so
 * jobs that arrive while others run overlap with them on the device.  While
 * the head does not fit, later jobs that do fit may start first (backfill, at
 * most `backfill` of them per head, so the head is not starved).  Toeplitz
 * spectra are kept in a geometry-keyed cache (key: the exact angles, the
 * detector size and the padded dims); a job whose geometry is cached skips
 * the PSF construction.  A job computes what lc_mbir2d / lc_mbir3d compute for
 * the same arguments.  Its input and output host buffers must stay valid
 * until lc_server_wait has returned for it; angle arrays are copied at
 * submission. */
typedef struct lc_server_s *lc_server;

typedef struct {
    int device;
    int workers;             /* concurrent jobs (one context and stream each), 1..64 */
    double hbm_budget_bytes; /* admission budget; 0: 85% of the free memory at creation */
    double psf_cache_bytes;  /* cap of the Toeplitz spectrum cache; 0: 16 GiB */
    int psf_cache;           /* 0 disables the cache */
    int backfill;            /* max jobs that may start ahead of a queue head that does not
                                fit the budget yet (0: strict FIFO; default 16) */
    int priority_2d;         /* 1 (default): 2D jobs run on high-priority streams, so a slice
                                next to a running volume gets SMs first */
} lc_server_params;

typedef struct {
    double queue_ms;     /* submission to start */
    double run_ms;       /* start to result in host memory */
    double latency_ms;   /* submission to result */
    int psf_hit;         /* 1 if the Toeplitz spectrum came from the cache */
    int worker;
    double device_bytes; /* the footprint admission charged for the job */
    char error[160];     /* message of a failed job */
} lc_job_info;

typedef struct {
    long completed, failed, queued, running, peak_running;
    double p50_ms, p99_ms, mean_ms; /* latency of completed jobs (nearest rank) */
    double span_s;                  /* first submission to last completion */
    double recons_per_s;            /* completed / span_s */
    double hbm_budget_bytes, peak_admitted_bytes;
    long psf_hits, psf_misses, psf_cache_entries;
    double psf_cache_bytes;
    double p50_2d_ms, p99_2d_ms;    /* latency of the completed 2D jobs */
    double p50_3d_ms, p99_3d_ms;    /* latency of the completed laminography jobs */
    long backfilled;                /* jobs that started ahead of a waiting queue head */
} lc_server_stats;

void lc_server_params_default(lc_server_params *p);
int lc_server_create(const lc_server_params *p, lc_server *out);
/* runs the jobs still queued, then releases everything */
int lc_server_destroy(lc_server server);
/* gpu::MBIR2D as a job, with the arguments of lc_mbir2d; LC_ERR_TOO_LARGE if
 * the job alone would exceed the HBM budget */
int lc_server_submit2d(lc_server server, const float *sino, int ns, int ntheta, int nradial,
                       const double *theta, const int *recon_dims, const lc_recon_params *p,
                       float *recon, long long *job_id);
/* gpu::MBIR as a job, with the arguments of lc_mbir3d */
int lc_server_submit3d(lc_server server, const float *projs, int ntheta, int nrows, int ncols,
                       const double *theta, const double *gamma, const double *beta,
                       const float *shifts, const int *recon_dims, const lc_recon_params *p,
                       float *recon, long long *job_id);
/* Blocks until the job ends (timeout_ms <= 0: no limit) and returns the job's
 * status, LC_OK or its error; LC_ERR_TIMEOUT leaves the job registered. */
int lc_server_wait(lc_server server, long long job_id, double timeout_ms, lc_solver_stats *stats,
                   lc_job_info *info);
int lc_server_get_stats(lc_server server, lc_server_stats *out);
/* clears the latency record and the counters (the PSF cache stays) */
int lc_server_reset_stats(lc_server server);
/* drops the cached Toeplitz spectra and zeroes the hit / miss counts; running
 * jobs keep the spectrum they hold */
int lc_server_clear_psf_cache(lc_server server);
/* message of the last failed submit / wait on the server */
const char *lc_server_last_error(lc_server server);

#ifdef __cplusplus
}
#endif

#endif /* LAMINOCAM_H */
