/*
 * nsrno_b200 -- C ABI of the B200 frequency-domain Helmholtz solve.
 *
 * Conventions (mirroring the reference's native ABI, nsrno/native_time.cu:117-155
 * and nsrno/native_time.py:25-41):
 *   - every entry point returns 0 on success, a cudaError_t value (< 1000) or an
 *     NSR_ERR_* code (>= 1000); nsr_error_string() describes either;
 *   - every buffer is a caller-owned DEVICE pointer unless stated otherwise;
 *     complex values are interleaved (re, im) pairs: "c64" = 2 x float,
 *     "c128" = 2 x double;
 *   - work runs on the caller's stream (a cudaStream_t passed as void*);
 *     entry points do not synchronise it, except the *_sync variants, the
 *     dense solve (one small read per restart cycle) and the queries that say so;
 *   - no exceptions cross the ABI; nothing here allocates device memory
 *     except where stated (nsr_solve_batched takes a caller workspace sized by
 *     nsr_solve_workspace_size).
 *
 * Fields are [z, x] row-major (x contiguous), nz rows by nx columns, like the
 * reference grid of nsrno/theranostic/wave.py:29-87.
 */
#ifndef NSRNO_B200_H
#define NSRNO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes of one solved system.  They map one to one onto the reason
 * strings of the reference Krylov drivers (nsrno/dense_wave.py:127-147,
 * nsrno/wave_solver.py:17-37). */
enum {
  NSR_CONVERGED = 0,
  NSR_ITERATION_BUDGET = 1,
  NSR_BREAKDOWN = 2,
  NSR_DIVERGED = 3,
  NSR_NONFINITE = 4,
  NSR_TIMEOUT = 5,        /* NsrSolveParams.time_limit_s ran out first        */
  NSR_NOT_RUN = 6
};

/* Library error codes (cudaError_t values stay below 1000). */
enum {
  NSR_ERR_ARGUMENT = 1001,       /* null pointer, bad size or bad parameter   */
  NSR_ERR_UNSUPPORTED_SIZE = 1002, /* nz or nx outside [8, 2048] or with a
                                    prime factor above 61 (FFT sizes)    */
  NSR_ERR_WORKSPACE = 1003,      /* workspace smaller than the query returned */
  NSR_ERR_INTERNAL = 1004,       /* solver loop did not drain its queue       */
  NSR_ERR_CAPACITY = 1005,       /* request exceeds a fixed capacity          */
  NSR_ERR_TIMEOUT = 1006         /* a kernel gave up waiting on its copy ring */
};

/* Grid, PML and acquisition geometry of one record.  Mirrors the reference
 * Grid/Solver parameters (theranostic/wave.py:29-125) plus the plane-wave array
 * row of nsrno/conditioned_wave.py:29-30. */
typedef struct NsrGrid {
  int32_t nz, nx;            /* rows (z) and columns (x)                       */
  int32_t n_pml;             /* PML thickness in nodes on every side           */
  int32_t face;              /* row of the source line and receivers           */
  double h;                  /* node spacing [m]                               */
  double c0;                 /* reference speed for k0 and the PML [m/s]       */
  double rho0;               /* reference density [kg/m^3]                     */
  double pml_strength;       /* sigma_max = strength * c0 / (n_pml h)          */
  double alpha_power;        /* power-law exponent y of alpha [dB/cm/MHz^y]    */
  double aperture_half_width;/* cosine taper half width of the source line [m] */
} NsrGrid;

/* Launch shapes of nsr_solve_batched (all zero: the built-in defaults).
 * Chosen per grid and device by the autotuner of nsrno_b200.tune; every
 * choice gives bitwise the same results for a fixed slot count. */
typedef struct NsrTiles {
  int32_t stencil_width;     /* columns per stencil work item: 256 or 512      */
  int32_t stencil_depth;     /* row buffers of the second half's stencil ring:
                                4 (default), 5, 6 (width 512: 4; one column per
                                thread: 4); the first half's smaller rows fill
                                the same bytes (7, 8 or 10 of them)            */
  int32_t stencil_rows;      /* rows per stencil work item (band): 4..64       */
  int32_t stencil_ctas;      /* resident stencil CTAs per SM (0: occupancy)    */
  int32_t cols_width;        /* columns per column-FFT CTA: 8 or 16            */
  int32_t row_tile;          /* rows per row-FFT CTA: 1..8                     */
  int32_t slot_groups;       /* independent slot groups on graph branches: 1..4 */
  int32_t stencil_cols;      /* adjacent columns per stencil thread: 1 or 2    */
  int32_t cols_staged;       /* 1: column transform staged wholly through shared
                                memory; 0: first and last stages fused into the
                                global load and store (sizes 256..2048 of 2^a 3^b) */
  int32_t rows_staged;       /* 1: row transforms staged wholly through shared
                                memory; 0: first and last stages between
                                registers and global memory (widths 256..2048
                                of 2^a 3^b)                                    */
  int32_t reserved[2];
} NsrTiles;

/* Krylov parameters of nsr_solve_batched. */
/* Learned preconditioner of the reference's LearnedPreconditioner
 * (nsrno/conditioned_wave.py:94-117, learned_apply nsrno/dense_wave.py:150-165)
 * on the 5-point grid:  M r = outer * IFFT(m * FFT(inner * r)), the complex
 * conjugate of the reference map (exp(-i omega t) convention) in the units of
 * the h^2-scaled operator.  `params` is the flat float32 parameter vector in the
 * reference module's state_dict order: spectral[2][4], log_shift,
 * context.0.weight[16][5][3][3], context.0.bias[16], context.2.weight[16][16][3][3],
 * context.2.bias[16], context.4.weight[4][16][3][3], context.4.bias[4]. */
#define NSR_LEARNED_PARAMS 3645

typedef struct NsrLearned {
  const float* params;       /* device float[NSR_LEARNED_PARAMS]                */
  const void* gains;         /* device c64 [n_gain][2][nz][nx] (inner, outer)
                                from nsr_learned_setup; NULL: spectral
                                multiplier only (no diagonal gains)            */
  const int32_t* gain_index; /* device int32 [n_systems]: gain pair of each
                                system; NULL: system s uses pair s. Checked on
                                the host (one small copy) before any launch     */
  int32_t n_gain;            /* gain pairs in `gains`                          */
  int32_t reserved;
} NsrLearned;

typedef struct NsrSolveParams {
  double tolerance;          /* relative true residual ||b-Ax||/||b||          */
  double shift;              /* shifted-Laplace preconditioner shift (0.15)    */
  double restart_factor;     /* restart (fresh shadow vector) once the true
                                residual fell by this factor since the last
                                restart (1e-2; 0 disables)                     */
  double warm_gate;          /* an initial field x0 whose relative residual
                                exceeds this is discarded and the system starts
                                from zero (1.0; 0 accepts every x0)            */
  int32_t max_iterations;    /* BiCGSTAB iterations per system                 */
  int32_t replace_every;     /* true-residual replacement period (40)          */
  int32_t n_slots;           /* systems resident at once                       */
  int32_t adjoint;           /* 0: A x = b; 1: A^H x = b                       */
  int32_t graph_iterations;  /* iterations per captured CUDA graph (16)        */
  int32_t profile_iterations;/* first iterations launched one by one with CUDA
                                events between kernels (0: none); their average
                                durations are reported in NsrSolveStats          */
  int32_t fields_fp64;       /* 0: fields output is c64; 1: c128 (the FP64 iterate) */
  int32_t reserved;
  const NsrLearned* learned; /* host pointer; NULL: fixed shifted-Laplace
                                preconditioner. Otherwise the learned one
                                (`shift` is then unused)                        */
  double time_limit_s;       /* wall-clock limit per system measured on the
                                device from its start (0: none); a system still
                                iterating then stops at its next true residual
                                with status NSR_TIMEOUT                          */
  const NsrTiles* tiles;     /* host pointer; NULL: built-in launch shapes      */
} NsrSolveParams;

/* Optional host-side statistics of one nsr_solve_batched call. */
typedef struct NsrSolveStats {
  double loop_ms;            /* device time of the solve loop                   */
  double kernel_ms[16];      /* mean duration per launch, in launch order: fwd,
                                cols, rinv, inv of the first half; fwd, cols,
                                rinv, res, inv of the second half; [9..15]
                                unused                                          */
  int32_t kernel_timed[16];  /* launches averaged in kernel_ms                  */
  int64_t launches;          /* kernels launched by the call                    */
  int32_t graph_launches;    /* CUDA graph launches                             */
  int32_t warm_accepted;     /* initial fields kept                             */
  int32_t warm_rejected;     /* initial fields discarded by the warm_gate       */
  int32_t reserved;
} NsrSolveStats;

/* Version of this ABI (major * 100 + minor). */
int nsr_version(void);

/* Text for a return code (status, NSR_ERR_* or cudaError_t). */
const char* nsr_error_string(int code);

/* Size in bytes of the material buffer of a grid (0 for an invalid grid). */
size_t nsr_material_bytes(const NsrGrid* grid);

/* Material planes: c [m/s], rho [kg/m^3], alpha [dB/cm/MHz^y] (float, [nz,nx])
 * -> material buffer (nsr_material_bytes bytes): a = rho0/rho (1 + m_eta),
 * b = rho0 c0^2/(rho c^2) (1 + m_kappa), t = attenuation slope with
 * e(f) = t (f/1 MHz)^(y-1) = alpha_Np(f) c / omega, computed in double; the
 * buffer holds them as float planes [3][nz][nx] at offset 0 (for the FP32
 * Krylov kernels) and as double planes [3][nz][nx] at the next 256-byte
 * boundary after them (for the FP64 residual, FP64 apply and gradient).
 * Replaces the material part of Solver.matrix (theranostic/wave.py:158-180)
 * and of WaveResidualOperator.setup (nsrno/wave_operator.py:48-67). */
int nsr_setup_material(const NsrGrid* grid, const float* c, const float* rho,
                       const float* alpha_db, void* material, void* stream);

/* y = A x (adjoint = 0) or A^H x (adjoint = 1) for S systems of frequencies
 * freq_hz[S] (device, double), fields [S][nz][nx].  A is the h^2-scaled
 * 5-point operator (the reference matrix of theranostic/wave.py:174-188 times
 * h^2, with the attenuation mass term).  precision 0: c64 in/out, float math;
 * precision 1: c128 in/out, double math on the double planes.  Replaces
 * Solver.matrix @ x and
 * WaveResidualOperator.apply_operator (nsrno/wave_operator.py:105-109). */
int nsr_apply(const NsrGrid* grid, const void* material, const double* freq_hz,
              int32_t n_systems, int32_t adjoint, int32_t precision,
              const void* x, void* y, void* stream);

/* y = M^-1 x: the fixed shifted-Laplace preconditioner
 * M^-1 = IFFT[ 1 / (h^2 L(q) + (k0 h)^2 (1 + i shift)) FFT ], periodic 5-point
 * Laplacian symbol, c64 fields [S][nz][nx].  Replaces the fixed preconditioner
 * of nsrno/dense_wave.py:194-196 and conditioned_wave.py:90-92.  Requires
 * workspace of nsr_precondition_workspace_size bytes. */
size_t nsr_precondition_workspace_size(const NsrGrid* grid, int32_t n_systems);
int nsr_precondition(const NsrGrid* grid, const double* freq_hz, int32_t n_systems,
                     double shift, int32_t adjoint, const float* x, float* y,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free y = M^-1 x, for callers that cannot allocate device memory
 * where they need it (for example while another framework captures a CUDA
 * graph, under a latency budget that forbids the device-wide synchronisation
 * of cudaMalloc, or inside a host application that owns all device memory).
 * This entry point has no counterpart in the reference.  Same arguments and
 * result as nsr_precondition, but its scratch space is a fixed 16 MiB
 * file-scope device array (reserved on each device where the library's module
 * is loaded -- with lazy module loading, at the first call on that device --
 * and held until the process exits), so nothing is allocated.  Requests whose
 * nsr_precondition_workspace_size exceeds 16 MiB return NSR_ERR_CAPACITY
 * (e.g. at most two 1024 x 768 systems per call).  The first call in a CUDA
 * context (normally the device's primary context) looks up the array's device
 * address with that device current and caches it for that context only; make
 * that first call before any stream capture.  Every call shares the array and it
 * keeps the last call's contents: calls that overlap on the GPU (different
 * streams or threads, same device) race and must be serialised by the caller. */
int nsr_precondition_noalloc(const NsrGrid* grid, const double* freq_hz, int32_t n_systems,
                             double shift, int32_t adjoint, const float* x, float* y, void* stream);

/* Plane-wave right-hand side in SI units, b = -line(x)/h^2 on row `face`,
 * line = taper(x) exp(-i k0 x sin(theta)) (nsrno/wave_operator.py:111-115 and
 * theranostic/wave.py:260).  b: c128 [S][nz][nx]. */
int nsr_plane_wave_rhs(const NsrGrid* grid, const double* freq_hz, const double* angle_rad,
                       int32_t n_systems, void* b, void* stream);

/* Batched right-preconditioned BiCGSTAB over a queue of S systems held in
 * params->n_slots resident slots; converged systems retire and their slots
 * refill.  Replaces solve_system/bicgstab (nsrno/dense_wave.py:118-148,
 * 167-225) and the GMRES loop of solve_frequency (nsrno/wave_solver.py:38-67)
 * for whole records.
 *   material      material buffer from nsr_setup_material
 *   freq_hz[S]    device double
 *   angle_rad[S]  device double (plane-wave source; ignored when rhs != NULL)
 *   rhs           NULL or c64 [S][nz][nx] explicit right-hand sides (SI units)
 *   x0            NULL or c64 [S][nz][nx] initial fields (warm start)
 *   rx_index[n_rx] device int32 flat node indices of the receivers
 * Outputs (device): iq c128 [S][n_rx], residual f64 [S] (true relative
 * residual, FP64), iterations i32 [S], status i32 [S] (NSR_CONVERGED ...),
 * fields NULL or [S][nz][nx] (c64, or c128 when params->fields_fp64);
 * stats NULL or a host NsrSolveStats.
 *
 * nsr_solve_batched does not block: it enqueues the whole solve on the
 * caller's stream and returns.  The iteration loop runs on the device, as a
 * CUDA graph whose conditional WHILE node repeats graph_iterations
 * iterations until every system has finished (or a round budget derived
 * from max_iterations is spent; systems never finished keep NSR_NOT_RUN).
 * Inputs, outputs and the workspace must stay valid until the stream passes
 * the solve.  stats (if given) gets only what is known at enqueue time;
 * profile_iterations must be 0.  A kernel that gives up on its copy ring
 * ends the loop; nsr_solve_progress reports it.
 *
 * nsr_solve_batched_sync runs the same solve with a host-driven loop: it
 * relaunches the captured iterations and polls a completion counter, fills
 * every field of stats (device loop time, per-kernel event timings of the
 * first profile_iterations iterations), returns NSR_ERR_TIMEOUT for a
 * kernel that gave up, and returns once the solve has finished. */
size_t nsr_solve_workspace_size(const NsrGrid* grid, int32_t n_slots);
int nsr_solve_batched(const NsrGrid* grid, const void* material,
                      const double* freq_hz, const double* angle_rad, int32_t n_systems,
                      const float* rhs, const float* x0,
                      const int32_t* rx_index, int32_t n_rx,
                      const NsrSolveParams* params,
                      void* workspace, size_t workspace_bytes,
                      double* iq, double* residual, int32_t* iterations, int32_t* status,
                      void* fields, NsrSolveStats* stats, void* stream);
int nsr_solve_batched_sync(const NsrGrid* grid, const void* material,
                           const double* freq_hz, const double* angle_rad, int32_t n_systems,
                           const float* rhs, const float* x0,
                           const int32_t* rx_index, int32_t n_rx,
                           const NsrSolveParams* params,
                           void* workspace, size_t workspace_bytes,
                           double* iq, double* residual, int32_t* iterations, int32_t* status,
                           void* fields, NsrSolveStats* stats, void* stream);

/* Progress of the last solve in `workspace` (n_slots as given to it): systems
 * finished, device loop rounds run, and 1 if a kernel gave up on its copy
 * ring.  Synchronises `stream` (reads a few words). */
int nsr_solve_progress(const NsrGrid* grid, int32_t n_slots, const void* workspace, int32_t* done,
                       int64_t* rounds, int32_t* error, void* stream);
/* Byte offset in the workspace of the progress record read by
 * nsr_solve_progress: int32 words [1] systems finished, [4] error, and the
 * int64 at word 6 the device loop rounds; a caller may copy these 32 bytes
 * asynchronously after a non-blocking solve.  0 for invalid arguments. */
size_t nsr_solve_progress_offset(const NsrGrid* grid, int32_t n_slots);

/* Parameters of nsr_gmres_batched. */
typedef struct NsrGmresParams {
  double tolerance;          /* relative true residual ||b-Ax||/||b||          */
  double shift;              /* shifted-Laplace preconditioner shift (0.15)    */
  int32_t max_iterations;    /* Arnoldi steps per system                       */
  int32_t restart;           /* restart length m (1..64)                       */
  int32_t n_slots;           /* systems per batch                              */
  int32_t adjoint;           /* 0: A x = b; 1: A^H x = b                       */
  int32_t fields_fp64;       /* fields output c128 when set, else c64          */
  int32_t reserved;
  const NsrLearned* learned; /* host pointer; NULL: fixed preconditioner      */
} NsrGmresParams;

/* Restarted right-preconditioned GMRES(m) with two classical Gram-Schmidt
 * passes, FP64 Hessenberg/Givens recurrence and FP64 true residual at every
 * restart, for S systems in batches of params->n_slots.  Replaces `gmres`
 * (nsrno/wave_solver.py:9-36) as used by solve_frequency
 * (nsrno/wave_solver.py:38-67) and the GMRES path of solve_system
 * (nsrno/dense_wave.py:212-220).  Arguments and outputs as nsr_solve_batched;
 * `iterations` counts Arnoldi steps (operator applications).  Synchronises
 * its stream once per restart cycle. */
size_t nsr_gmres_workspace_size(const NsrGrid* grid, int32_t n_slots, int32_t restart);
int nsr_gmres_batched(const NsrGrid* grid, const void* material, const double* freq_hz,
                      const double* angle_rad, int32_t n_systems, const float* rhs, const float* x0,
                      const int32_t* rx_index, int32_t n_rx, const NsrGmresParams* params,
                      void* workspace, size_t workspace_bytes, double* iq, double* residual,
                      int32_t* iterations, int32_t* status, void* fields, void* stream);

/* g_logc, g_logrho (double [nz][nx]) += -Re(lambda^H dA/dm u) summed over S
 * systems, u and lambda [S][nz][nx] SI fields (precision 0: c64, 1: c128),
 * m = log c and log rho.
 * The exact derivative of the 5-point discretisation that
 * theranostic/wave.py:331-389 (born_jacobian) forms column by column and
 * nsrno/dense_wave.py:250-255 obtains by autograd. */
int nsr_grad_accum(const NsrGrid* grid, const void* material, const double* freq_hz,
                   int32_t n_systems, int32_t precision, const void* u, const void* lam,
                   double* g_logc, double* g_logrho, void* stream);

/* ---------------------------------------------------------------------------
 * The dense path's 8th-order staggered split-PML operator
 * (nsrno/conditioned_wave.py:52-80 projected as nsrno/dense_wave.py:66-68) and
 * its analytic adjoint (nsrno/dense_wave.py:70-82), evaluated as a direct
 * radius-4 stencil on the padded grid instead of 11 FFTs.
 * ------------------------------------------------------------------------- */
typedef struct NsrDenseGrid {
  int32_t H, W;              /* padded grid (rows, columns)                    */
  int32_t pz, px;            /* offset of the native region                    */
  int32_t h, w;              /* native region (the mask)                       */
  double dx;                 /* node spacing [m]                               */
} NsrDenseGrid;

/* Coefficients of one medium at one frequency, double, packed as
 * ax[H][W], az[H][W], mass[H][W] (c128), then along x (c128 [W] each)
 * svx, gvx, lx = mx/(D-arx), rx = 1 + (1-mx)/(D-arx), then along z
 * (c128 [H] each) svz, gvz, lz, rz.  Built by nsrno_b200.dense. */
size_t nsr_dense_coef_bytes(const NsrDenseGrid* grid);
size_t nsr_dense_workspace_size(const NsrDenseGrid* grid, int32_t n_fields, int32_t precision);

/* y = A x (adjoint 0) or A^H x (adjoint 1) for n_fields fields [n][H][W]
 * sharing one coefficient set; scal = (D-1)/(D k0^2).  precision 0: c64,
 * 1: c128.  Replaces projected_operator / adjoint_operator
 * (nsrno/dense_wave.py:66-82). */
int nsr_dense_apply(const NsrDenseGrid* grid, const double* coef, double scal_re, double scal_im,
                    int32_t n_fields, int32_t adjoint, int32_t precision, const void* x, void* y,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Cotangents of the dense operator's medium-dependent coefficient planes for
 * L = -Re sum_f conj(lam_f) . mask . A(m)(mask u_f): g_ax, g_az double [H][W]
 * (dL/d ax, dL/d az) and g_mass double [2][H][W] (dL/d Re mass, dL/d Im
 * mass), over n_fields c128 fields u, lam [n][H][W]; the chain rule through
 * the coefficient construction turns them into dL/d(c, rho).  Replaces the
 * operator part of the autograd in ImplicitChannels.backward
 * (nsrno/dense_wave.py:250-255). */
int nsr_dense_grad(const NsrDenseGrid* grid, const double* coef, double scal_re, double scal_im,
                   int32_t n_fields, const double* u, const double* lam, double* g_ax, double* g_az,
                   double* g_mass, void* stream);

/* Tangent (Born) right-hand side rhs = -dA[dm] u of n_systems background
 * fields u for the material direction dm = (dlogc, dlogrho) (double [nz][nx],
 * shared by all systems), in SI units like the solver's rhs: solving
 * A du = rhs gives the tangent field of the Gauss-Newton Hessian-vector
 * product.  precision 0: u, rhs c64; 1: c128.  Replaces the perturbation
 * assembly of Solver.born_data (theranostic/wave.py:280-329). */
int nsr_tangent_rhs(const NsrGrid* grid, const void* coef, const double* freq_hz, int32_t n_systems,
                    int32_t precision, const void* u, const double* dlogc, const double* dlogrho,
                    void* rhs, void* stream);

/* Fixed preconditioner of the dense path, y = mask * IFFT(m * FFT(x)) with
 * m = 1/(1 + lap/k0^2 - i shift) and the 8th-order staggered symbols in lap
 * (nsrno/conditioned_wave.py:90-92, nsrno/dense_wave.py:194-196); adjoint = 1
 * conjugates m as the reference's adjoint solve does.  k0dx2 = (k0 dx)^2 with
 * the system's k0 = 2 sin(pi f dt)/(dt c0).  H and W must be FFT sizes (see NSR_ERR_UNSUPPORTED_SIZE) in
 * [8, 2048].  x, y: c64 [n_fields][H][W]. */
size_t nsr_dense_precondition_workspace_size(const NsrDenseGrid* grid, int32_t n_fields);
int nsr_dense_precondition(const NsrDenseGrid* grid, double k0dx2, double shift, int32_t n_fields,
                           int32_t adjoint, const float* x, float* y, void* workspace, size_t workspace_bytes,
                           void* stream);

/* Converged dense-path solve A x = b (adjoint 0) or A^H x = b (adjoint 1) of
 * n_fields fields sharing one coefficient set, all fields treated as one
 * vector as the reference does: restarted right-preconditioned GMRES(restart)
 * with two classical Gram-Schmidt passes and the fixed preconditioner of
 * nsr_dense_precondition; complex64 Krylov vectors, FP64 inner products,
 * Hessenberg/Givens recurrence and triangular solve on the device, a
 * complex128 iterate and an FP64 true residual at every restart.  Replaces
 * the GMRES branch of solve_system (nsrno/dense_wave.py:212-220, gmres of
 * nsrno/wave_solver.py:9-36) and its mixed FP32 inverse / FP64 residual
 * refinement (nsrno/dense_wave.py:168-191).  rhs and x: c128
 * [n_fields][H][W] (x holds the initial field on entry, the solution on
 * return); field_residual: NULL or device double [n_fields], the final
 * relative residual of every field.  Synchronises its stream once per
 * restart cycle. */
typedef struct NsrDenseSolveParams {
  double tolerance;          /* FP64 relative residual over all fields         */
  double shift;              /* preconditioner shift (0.15)                    */
  double k0dx2;              /* (k0 dx)^2 of the preconditioner                */
  double scal_re, scal_im;   /* (D-1)/(D k0^2), as nsr_dense_apply             */
  int32_t restart;           /* Arnoldi steps per cycle (1..64; 24 or 32)      */
  int32_t max_cycles;        /* restart cycles                                 */
  int32_t adjoint;           /* 0: A x = b; 1: A^H x = b                       */
  int32_t reserved;
} NsrDenseSolveParams;

typedef struct NsrDenseSolveInfo {
  int32_t status;            /* NSR_CONVERGED, NSR_ITERATION_BUDGET, NSR_NONFINITE */
  int32_t steps;             /* Arnoldi steps (operator applications)          */
  int32_t cycles;            /* restart cycles                                 */
  int32_t reserved;
  double residual;           /* FP64 relative residual of the returned x        */
} NsrDenseSolveInfo;

size_t nsr_dense_solve_workspace_size(const NsrDenseGrid* grid, int32_t n_fields, int32_t restart);
int nsr_dense_solve(const NsrDenseGrid* grid, const double* coef, const NsrDenseSolveParams* params,
                    int32_t n_fields, const double* rhs, double* x, double* field_residual,
                    NsrDenseSolveInfo* info, void* workspace, size_t workspace_bytes, void* stream);

/* Band-limited RF traces rf[ch][t] (double) from receiver spectra
 * spectrum[ch][b] (c128) on positive bins 0 < bins[b] < n_samples/2:
 * the irfft with 'forward' normalisation of predict_band_rf
 * (nsrno/wave_operator.py:169-180).  Bins must be valid (checked by the
 * host wrapper); a spectrum with no bins gives zero traces. */
int nsr_band_rf(int32_t n_channels, int32_t n_bins, int32_t n_samples, const double* spectrum,
                const int32_t* bins, double* rf, void* stream);

/* FP64 true relative residual ||b - A x|| / ||b|| (or A^H) of n_systems c128
 * fields x; b is rhs (c128, SI) or, when rhs is NULL, the plane-wave source of
 * (freq, angle).  Deterministic order of summation.  Replaces the acceptance
 * residual of nsrno/dense_wave.py:146-147,221-225 and the diagnostics of
 * theranostic/wave.py:320-323. */
size_t nsr_true_residual_workspace_size(const NsrGrid* grid, int32_t n_systems);
int nsr_true_residual(const NsrGrid* grid, const void* coef, const double* freq_hz, const double* angle_rad,
                      int32_t n_systems, int32_t adjoint, const double* x, const double* rhs, double* residual,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ---- Learned preconditioner: inference -------------------------------- */

/* Arithmetic of the network: FP32, or BF16 weights and activations with FP32
 * accumulation (the state then holds bfloat16 planes). */
#define NSR_LEARNED_FP32 0
#define NSR_LEARNED_BF16 1

/* Bytes of the low-resolution network state of n_freq frequencies. */
size_t nsr_learned_state_bytes(const NsrGrid* grid, int32_t n_freq);

/* Network and gains of one medium at n_freq frequencies: the 8x pooled context
 * (log(c/1540)/.06, log(rho/1000)/.08, log1p(alpha), f/6e6-1, 1), three 3x3
 * convolutions with tanh, bilinear upsampling and the gains
 * inner = (1 + tanh(m0)/2) exp(-i tanh(m1)/2), outer likewise of m2, m3.
 * Replaces LearnedPreconditioner.setup (nsrno/conditioned_wave.py:103-117).
 * c, rho, alpha: float [nz][nx]; state: nsr_learned_state_bytes; gains: c64
 * [n_freq][2][nz][nx] (NULL: network only). */
int nsr_learned_setup(const NsrGrid* grid, const float* c, const float* rho, const float* alpha,
                      const double* freq_hz, int32_t n_freq, const float* params, void* state,
                      void* gains, void* stream);
/* The same with the network's precision (NSR_LEARNED_FP32 / NSR_LEARNED_BF16);
 * a BF16 state must be passed to the _ex backward entry points with the same
 * precision. */
int nsr_learned_setup_ex(const NsrGrid* grid, const float* c, const float* rho, const float* alpha,
                         const double* freq_hz, int32_t n_freq, const float* params, int32_t precision,
                         void* state, void* gains, void* stream);

/* y = M x (adjoint = 0) or M^H x (adjoint = 1) of the learned preconditioner
 * for n_systems c64 fields; workspace of nsr_precondition_workspace_size.
 * Replaces learned_apply (nsrno/dense_wave.py:150-165). */
int nsr_learned_precondition(const NsrGrid* grid, const NsrLearned* learned, const double* freq_hz,
                             int32_t n_systems, int32_t adjoint, const float* x, float* y,
                             void* workspace, size_t workspace_bytes, void* stream);

/* ---- Learned preconditioner: training (backward kernels) ---------------- */
/* Replace the autograd of DenseTrainingModel / differentiable_gmres
 * (nsrno/train_dense_wave.py:14-21, nsrno/conditioned_wave.py:119-139).
 * Cotangents follow dL = 2 Re sum conj(G) dz for complex z. */

size_t nsr_learned_backward_workspace_size(const NsrGrid* grid, int32_t n_freq);

/* Gain cotangents g_inner, g_outer (c64 [n_freq][nz][nx], dL/d conj(gain)) ->
 * map cotangents d_maps (float [n_freq][4][nz/8][nx/8], overwritten). */
int nsr_learned_map_backward(const NsrGrid* grid, const void* state, int32_t n_freq,
                             const float* g_inner, const float* g_outer, float* d_maps,
                             void* workspace, size_t workspace_bytes, void* stream);
int nsr_learned_map_backward_ex(const NsrGrid* grid, const void* state, int32_t precision, int32_t n_freq,
                                const float* g_inner, const float* g_outer, float* d_maps,
                                void* workspace, size_t workspace_bytes, void* stream);

/* Map cotangents -> gradients of the convolution weights and biases, ADDED to
 * d_params[9 .. NSR_LEARNED_PARAMS). */
int nsr_learned_network_backward(const NsrGrid* grid, const float* params, const void* state,
                                 int32_t n_freq, const float* d_maps, float* d_params,
                                 void* workspace, size_t workspace_bytes, void* stream);
int nsr_learned_network_backward_ex(const NsrGrid* grid, const float* params, const void* state,
                                    int32_t precision, int32_t n_freq, const float* d_maps, float* d_params,
                                    void* workspace, size_t workspace_bytes, void* stream);

size_t nsr_learned_spectral_workspace_size(const NsrGrid* grid, int32_t n_systems);

/* Gradient of the spectral weights and log_shift, ADDED to d_params[0..9), for
 * z = outer * F^-1(m * F(x)) with x = inner * r and y = conj(outer) * dL/d conj(z)
 * (c64 [n_systems][nz][nx]). */
int nsr_learned_spectral_backward(const NsrGrid* grid, const float* params, const double* freq_hz,
                                  int32_t n_systems, const float* x, const float* y, float* d_params,
                                  void* workspace, size_t workspace_bytes, void* stream);

/* One Adam step with gradient-norm clipping (clip_norm <= 0: none), in place on
 * params, m, v (float [n]); writes the unclipped gradient norm to grad_norm
 * (device float, may be NULL).  The optimiser of nsrno/train_dense_wave.py:37,72-76. */
int nsr_learned_adam(float* params, const float* grad, float* m, float* v, int32_t n, int32_t step,
                     double lr, double beta1, double beta2, double eps, double clip_norm,
                     float* grad_norm, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NSRNO_B200_H */
